"""Materials of the oracle's pinning tests (test infrastructure only).

Each entry is a node graph in the exporter's format.  Together they cover the
node subset the configs use (Noise -> ColorRamp -> Mix -> Principled) and the
other nodes the oracle restates: every Principled lobe (diffuse, metallic
specular, transmission, clearcoat, sheen, anisotropy, alpha, emission), the
Diffuse / Glossy / Glass / Transparent BSDFs, Mix and Add shaders, Math,
Vector Math, Checker, Texture Coordinate, MixRGB, Fresnel, Layer Weight,
Invert, Gamma, RGB to BW, Separate/Combine XYZ and Map Range, and the next
node set: Mapping, Normal Map (tangent and world space), Hue/Saturation,
Bright/Contrast and Blackbody.
"""
from __future__ import annotations

import sys
from pathlib import Path
from typing import Any

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
from raymond_b200 import materials as M  # noqa: E402


def _v(t, value=None, link=None):
    d: dict[str, Any] = {"type": t}
    if link is not None:
        d["links"] = [list(link)]
    elif value is not None:
        d["value"] = list(value) if isinstance(value, (list, tuple)) else value
    return d


def _out(link):
    return {"type": "OUTPUT_MATERIAL", "inputs": {"Surface": _v("SHADER", link=link)}, "parameters": {}}


# inputs the exporter writes for every node of a type (Blender's defaults)
_DEFAULTS = {
    "BSDF_DIFFUSE": {"Color": ("RGBA", [0.8, 0.8, 0.8, 1]), "Roughness": ("VALUE", 0.0),
                     "Normal": ("VECTOR", [0, 0, 0]), "Weight": ("VALUE", 0.0)},
    "BSDF_GLOSSY": {"Color": ("RGBA", [0.8, 0.8, 0.8, 1]), "Roughness": ("VALUE", 0.5),
                    "Normal": ("VECTOR", [0, 0, 0]), "Weight": ("VALUE", 0.0)},
    "BSDF_GLASS": {"Color": ("RGBA", [1, 1, 1, 1]), "Roughness": ("VALUE", 0.0), "IOR": ("VALUE", 1.45),
                   "Normal": ("VECTOR", [0, 0, 0]), "Weight": ("VALUE", 0.0)},
    "BSDF_TRANSPARENT": {"Color": ("RGBA", [1, 1, 1, 1]), "Weight": ("VALUE", 0.0)},
    "EMISSION": {"Color": ("RGBA", [1, 1, 1, 1]), "Strength": ("VALUE", 1.0), "Weight": ("VALUE", 0.0)},
    "MIX_SHADER": {"Fac": ("VALUE", 0.5)},
    "LAYER_WEIGHT": {"Blend": ("VALUE", 0.5), "Normal": ("VECTOR", [0, 0, 0])},
    "FRESNEL": {"IOR": ("VALUE", 1.45), "Normal": ("VECTOR", [0, 0, 0])},
    "TEX_CHECKER": {"Vector": ("VECTOR", [0, 0, 0]), "Color1": ("RGBA", [0.8, 0.8, 0.8, 1]),
                    "Color2": ("RGBA", [0.2, 0.2, 0.2, 1]), "Scale": ("VALUE", 5.0)},
    "MATH": {"Value": ("VALUE", 0.5), "Value_001": ("VALUE", 0.5), "Value_002": ("VALUE", 0.5)},
    "VECT_MATH": {"Vector": ("VECTOR", [0, 0, 0]), "Vector_001": ("VECTOR", [0, 0, 0]),
                  "Vector_002": ("VECTOR", [0, 0, 0]), "Scale": ("VALUE", 1.0)},
    "SEPXYZ": {"Vector": ("VECTOR", [0, 0, 0])},
    "COMBXYZ": {"X": ("VALUE", 0.0), "Y": ("VALUE", 0.0), "Z": ("VALUE", 0.0)},
    "MAP_RANGE": {"Value": ("VALUE", 1.0), "From Min": ("VALUE", 0.0), "From Max": ("VALUE", 1.0),
                  "To Min": ("VALUE", 0.0), "To Max": ("VALUE", 1.0), "Steps": ("VALUE", 4.0),
                  "Vector": ("VECTOR", [0, 0, 0]), "From_Min_FLOAT3": ("VECTOR", [0, 0, 0]),
                  "From_Max_FLOAT3": ("VECTOR", [1, 1, 1]), "To_Min_FLOAT3": ("VECTOR", [0, 0, 0]),
                  "To_Max_FLOAT3": ("VECTOR", [1, 1, 1]), "Steps_FLOAT3": ("VECTOR", [4, 4, 4])},
    "GAMMA": {"Color": ("RGBA", [1, 1, 1, 1]), "Gamma": ("VALUE", 1.0)},
    "INVERT": {"Fac": ("VALUE", 1.0), "Color": ("RGBA", [0, 0, 0, 1])},
    "MIX_RGB": {"Fac": ("VALUE", 0.5), "Color1": ("RGBA", [0.5, 0.5, 0.5, 1]), "Color2": ("RGBA", [0.5, 0.5, 0.5, 1])},
    "RGBTOBW": {"Color": ("RGBA", [0.5, 0.5, 0.5, 1])},
    "MAPPING": {"Vector": ("VECTOR", [0, 0, 0]), "Location": ("VECTOR", [0, 0, 0]), "Rotation": ("VECTOR", [0, 0, 0]),
                "Scale": ("VECTOR", [1, 1, 1])},
    "NORMAL_MAP": {"Strength": ("VALUE", 1.0), "Color": ("RGBA", [0.5, 0.5, 1, 1])},
    "HUE_SAT": {"Hue": ("VALUE", 0.5), "Saturation": ("VALUE", 1.0), "Value": ("VALUE", 1.0), "Fac": ("VALUE", 1.0),
                "Color": ("RGBA", [0.8, 0.8, 0.8, 1])},
    "BRIGHTCONTRAST": {"Color": ("RGBA", [1, 1, 1, 1]), "Bright": ("VALUE", 0.0), "Contrast": ("VALUE", 0.0)},
    "BLACKBODY": {"Temperature": ("VALUE", 1500.0)},
    "TEX_IMAGE": {"Vector": ("VECTOR", [0, 0, 0])},
    "TEX_ENVIRONMENT": {"Vector": ("VECTOR", [0, 0, 0])},
}


def _bsdf(t, params=None, **inputs):
    full = {k: _v(tv, v) for k, (tv, v) in _DEFAULTS.get(t, {}).items()}
    full.update(inputs)
    return {"type": t, "inputs": full, "parameters": params or {}}


def materials() -> list[tuple[str, dict]]:
    mats: list[tuple[str, dict]] = []
    mats.append(("principled_default", M.principled()))
    mats.append(("principled_metal", M.principled(base_color=(0.9, 0.6, 0.3, 1), roughness=0.2, metallic=1.0)))
    mats.append(("principled_coat", M.principled(base_color=(0.2, 0.5, 0.8, 1), roughness=0.4, clearcoat=0.7,
                                                 sheen=0.5, anisotropic=0.4, specular=0.8)))
    mats.append(("principled_glass", M.principled(base_color=(0.95, 0.95, 0.9, 1), roughness=0.1,
                                                  transmission=1.0, ior=1.5)))
    mats.append(("principled_alpha_emit", M.principled(base_color=(0.3, 0.8, 0.3, 1), alpha=0.6,
                                                       emission=(1.0, 0.5, 0.2, 1.0), emission_strength=3.0)))
    mats.append(("noise_ramp_mix", M.principled_noise_ramp((0.7, 0.2, 0.1, 1), 0.35, 0.0)))
    mats.append(("noise_ramp_mix_metal", M.principled_noise_ramp((0.1, 0.3, 0.9, 1), 0.6, 1.0, noise_detail=3.5,
                                                                 noise_scale=2.0)))
    mats.append(("diffuse_glossy_mix", {
        "Diffuse": _bsdf("BSDF_DIFFUSE", Color=_v("RGBA", [0.8, 0.2, 0.2, 1]), Roughness=_v("VALUE", 0.0)),
        "Glossy": _bsdf("BSDF_GLOSSY", {"distribution": "GGX"}, Color=_v("RGBA", [0.9, 0.9, 0.9, 1]),
                        Roughness=_v("VALUE", 0.25)),
        "Mix Shader": _bsdf("MIX_SHADER", Fac=_v("VALUE", 0.3), Shader=_v("SHADER", link=("Diffuse", "BSDF")),
                            Shader_001=_v("SHADER", link=("Glossy", "BSDF"))),
        "Material Output": _out(("Mix Shader", "Shader")),
    }))
    mats.append(("glass_add_emission", {
        "Glass": _bsdf("BSDF_GLASS", {"distribution": "GGX"}, Color=_v("RGBA", [1, 1, 1, 1]),
                       Roughness=_v("VALUE", 0.2), IOR=_v("VALUE", 1.45)),
        "Emission": _bsdf("EMISSION", Color=_v("RGBA", [0.2, 0.4, 1.0, 1]), Strength=_v("VALUE", 0.5)),
        "Add Shader": _bsdf("ADD_SHADER", Shader=_v("SHADER", link=("Glass", "BSDF")),
                            Shader_001=_v("SHADER", link=("Emission", "Emission"))),
        "Material Output": _out(("Add Shader", "Shader")),
    }))
    mats.append(("transparent_mix", {
        "Transparent": _bsdf("BSDF_TRANSPARENT", Color=_v("RGBA", [0.9, 0.9, 0.5, 1])),
        "Diffuse": _bsdf("BSDF_DIFFUSE", Color=_v("RGBA", [0.2, 0.6, 0.2, 1])),
        "Layer Weight": _bsdf("LAYER_WEIGHT", Blend=_v("VALUE", 0.4)),
        "Mix Shader": _bsdf("MIX_SHADER", Fac=_v("VALUE", link=("Layer Weight", "Facing")),
                            Shader=_v("SHADER", link=("Transparent", "BSDF")),
                            Shader_001=_v("SHADER", link=("Diffuse", "BSDF"))),
        "Material Output": _out(("Mix Shader", "Shader")),
    }))
    mats.append(("checker_math_roughness", {
        "Texture Coordinate": _bsdf("TEX_COORD"),
        "Checker": _bsdf("TEX_CHECKER", Vector=_v("VECTOR", link=("Texture Coordinate", "Object")),
                         Color1=_v("RGBA", [0.9, 0.9, 0.9, 1]), Color2=_v("RGBA", [0.1, 0.2, 0.3, 1]),
                         Scale=_v("VALUE", 7.0)),
        "Math": _bsdf("MATH", {"operation": "MULTIPLY", "use_clamp": True},
                      Value=_v("VALUE", link=("Checker", "Fac")), Value_001=_v("VALUE", 0.8),
                      Value_002=_v("VALUE", 0.0)),
        "Principled BSDF": {"type": "BSDF_PRINCIPLED",
                            "inputs": dict(M.principled_inputs(metallic=0.3),
                                           **{"Base Color": _v("RGBA", link=("Checker", "Color")),
                                              "Roughness": _v("VALUE", link=("Math", "Value"))}),
                            "parameters": {"distribution": "GGX", "subsurface_method": "RANDOM_WALK"}},
        "Material Output": _out(("Principled BSDF", "BSDF")),
    }))
    mats.append(("vector_math_colors", {
        "Texture Coordinate": _bsdf("TEX_COORD"),
        "Vector Math": _bsdf("VECT_MATH", {"operation": "MULTIPLY_ADD"},
                             Vector=_v("VECTOR", link=("Texture Coordinate", "Normal")),
                             Vector_001=_v("VECTOR", [0.3, -0.5, 0.8]), Vector_002=_v("VECTOR", [0.1, 0.2, -0.3])),
        "Separate XYZ": _bsdf("SEPXYZ", Vector=_v("VECTOR", link=("Vector Math", "Vector"))),
        "Map Range": _bsdf("MAP_RANGE", {"data_type": "FLOAT", "interpolation_type": "LINEAR", "clamp": True},
                           Value=_v("VALUE", link=("Separate XYZ", "X")),
                           **{"From Min": _v("VALUE", -1.0), "From Max": _v("VALUE", 1.0),
                              "To Min": _v("VALUE", 0.05), "To Max": _v("VALUE", 0.9)}),
        "Combine XYZ": _bsdf("COMBXYZ", X=_v("VALUE", link=("Map Range", "Result")), Y=_v("VALUE", 0.4),
                             Z=_v("VALUE", link=("Separate XYZ", "Z"))),
        "Gamma": _bsdf("GAMMA", Color=_v("RGBA", link=("Combine XYZ", "Vector")), Gamma=_v("VALUE", 2.2)),
        "Invert": _bsdf("INVERT", Fac=_v("VALUE", 0.25), Color=_v("RGBA", link=("Gamma", "Color"))),
        "MixRGB": _bsdf("MIX_RGB", {"blend_type": "MULTIPLY", "use_clamp": False},
                        Fac=_v("VALUE", 0.6), Color1=_v("RGBA", link=("Invert", "Color")),
                        Color2=_v("RGBA", [0.8, 0.7, 0.6, 1])),
        "RGB to BW": _bsdf("RGBTOBW", Color=_v("RGBA", link=("MixRGB", "Color"))),
        "Fresnel": _bsdf("FRESNEL", IOR=_v("VALUE", 1.6)),
        "Principled BSDF": {"type": "BSDF_PRINCIPLED",
                            "inputs": dict(M.principled_inputs(),
                                           **{"Base Color": _v("RGBA", link=("MixRGB", "Color")),
                                              "Roughness": _v("VALUE", link=("RGB to BW", "Val")),
                                              "Specular": _v("VALUE", link=("Fresnel", "Fac"))}),
                            "parameters": {"distribution": "GGX", "subsurface_method": "RANDOM_WALK"}},
        "Material Output": _out(("Principled BSDF", "BSDF")),
    }))
    mats.append(("emission_only", M.emission((1.0, 0.8, 0.6, 1.0), 4.0)))
    # the "next" node set: Mapping, Hue/Saturation, Bright/Contrast, Normal Map (tangent and world), Blackbody
    mats.append(("mapping_hue_normal_map", {
        "Texture Coordinate": _bsdf("TEX_COORD"),
        "Mapping": _bsdf("MAPPING", {"type": "MAPPING"}, Vector=_v("VECTOR", link=("Texture Coordinate", "Object")),
                         Location=_v("VECTOR", [0.1, -0.2, 0.3]), Rotation=_v("VECTOR", [0.3, -0.4, 1.1]),
                         Scale=_v("VECTOR", [2.0, 1.5, 0.7])),
        "Checker": _bsdf("TEX_CHECKER", Vector=_v("VECTOR", link=("Mapping", "Vector")),
                         Color1=_v("RGBA", [0.9, 0.4, 0.1, 1]), Color2=_v("RGBA", [0.1, 0.5, 0.8, 1]),
                         Scale=_v("VALUE", 3.0)),
        "Hue Saturation": _bsdf("HUE_SAT", Hue=_v("VALUE", 0.3), Saturation=_v("VALUE", 1.4), Value=_v("VALUE", 0.9),
                                Fac=_v("VALUE", 0.8), Color=_v("RGBA", link=("Checker", "Color"))),
        "Bright Contrast": _bsdf("BRIGHTCONTRAST", Color=_v("RGBA", link=("Hue Saturation", "Color")),
                                 Bright=_v("VALUE", 0.05), Contrast=_v("VALUE", 0.3)),
        "Normal Map": _bsdf("NORMAL_MAP", {"space": "TANGENT", "uv_map": ""}, Strength=_v("VALUE", 0.7),
                            Color=_v("RGBA", link=("Checker", "Color"))),
        "Principled BSDF": {"type": "BSDF_PRINCIPLED",
                            "inputs": dict(M.principled_inputs(roughness=0.35),
                                           **{"Base Color": _v("RGBA", link=("Bright Contrast", "Color")),
                                              "Normal": _v("VECTOR", link=("Normal Map", "Normal"))}),
                            "parameters": {"distribution": "GGX", "subsurface_method": "RANDOM_WALK"}},
        "Material Output": _out(("Principled BSDF", "BSDF")),
    }))
    mats.append(("blackbody_world_normal", {
        "Texture Coordinate": _bsdf("TEX_COORD"),
        "Separate XYZ": _bsdf("SEPXYZ", Vector=_v("VECTOR", link=("Texture Coordinate", "Generated"))),
        "Map Range": _bsdf("MAP_RANGE", {"data_type": "FLOAT", "interpolation_type": "LINEAR", "clamp": False},
                           Value=_v("VALUE", link=("Separate XYZ", "X")),
                           **{"From Min": _v("VALUE", 0.0), "From Max": _v("VALUE", 1.0),
                              "To Min": _v("VALUE", 500.0), "To Max": _v("VALUE", 13000.0)}),
        "Blackbody": _bsdf("BLACKBODY", Temperature=_v("VALUE", link=("Map Range", "Result"))),
        "Normal Map": _bsdf("NORMAL_MAP", {"space": "WORLD", "uv_map": ""}, Strength=_v("VALUE", 0.9),
                            Color=_v("RGBA", link=("Texture Coordinate", "Generated"))),
        "Principled BSDF": {"type": "BSDF_PRINCIPLED",
                            "inputs": dict(M.principled_inputs(roughness=0.5, emission_strength=0.2),
                                           **{"Base Color": _v("RGBA", link=("Blackbody", "Color")),
                                              "Emission": _v("RGBA", link=("Blackbody", "Color")),
                                              "Normal": _v("VECTOR", link=("Normal Map", "Normal"))}),
                            "parameters": {"distribution": "GGX", "subsurface_method": "RANDOM_WALK"}},
        "Material Output": _out(("Principled BSDF", "BSDF")),
    }))
    # image textures: flat projection of a mapped UV in sRGB, a single-channel
    # linear image, an equirectangular environment in XYZ, and a missing file
    mats.append(("image_textures", {
        "Texture Coordinate": _bsdf("TEX_COORD"),
        "Mapping": _bsdf("MAPPING", {"type": "MAPPING"}, Vector=_v("VECTOR", link=("Texture Coordinate", "Generated")),
                         Location=_v("VECTOR", [0.3, -0.1, 0.0]), Rotation=_v("VECTOR", [0.0, 0.0, 0.4]),
                         Scale=_v("VECTOR", [2.5, 1.7, 1.0])),
        "Albedo": _bsdf("TEX_IMAGE", _image_params("textures/albedo.png", "sRGB"),
                        Vector=_v("VECTOR", link=("Mapping", "Vector"))),
        "Rough": _bsdf("TEX_IMAGE", _image_params("textures/rough.png", "Non-Color")),
        "Sky": _bsdf("TEX_ENVIRONMENT", _image_params("textures/sky.exr", "XYZ", "EQUIRECTANGULAR"),
                     Vector=_v("VECTOR", link=("Texture Coordinate", "Normal"))),
        "Missing": _bsdf("TEX_IMAGE", _image_params("textures/not_exported.jpg", "sRGB")),
        "Mix": _bsdf("MIX_RGB", {"blend_type": "ADD", "use_clamp": False}, Fac=_v("VALUE", link=("Albedo", "Alpha")),
                     Color1=_v("RGBA", link=("Albedo", "Color")), Color2=_v("RGBA", link=("Missing", "Color"))),
        "Principled BSDF": {"type": "BSDF_PRINCIPLED",
                            "inputs": dict(M.principled_inputs(emission_strength=0.05),
                                           **{"Base Color": _v("RGBA", link=("Mix", "Color")),
                                              "Roughness": _v("VALUE", link=("Rough", "Color")),
                                              "Emission": _v("RGBA", link=("Sky", "Color"))}),
                            "parameters": {"distribution": "GGX", "subsurface_method": "RANDOM_WALK"}},
        "Material Output": _out(("Principled BSDF", "BSDF")),
    }))
    # the Nishita sky as an emissive colour (its node reads the shading point's wo); a large sun disc so that
    # some records look into it
    mats.append(("sky_emission", {
        "Sky Texture": _bsdf("TEX_SKY", dict(SKY, sky_type="NISHITA"), Vector=_v("VECTOR", [0.0, 0.0, 0.0])),
        "Emission": _bsdf("EMISSION", Color=_v("RGBA", link=("Sky Texture", "Color")),
                          Strength=_v("VALUE", 1e-3)),
        "Material Output": _out(("Emission", "Emission")),
    }))
    return mats


# parameters of the pinning sky (Blender's TEX_SKY node as the exporter writes them)
SKY = {"sun_elevation": 0.35, "sun_rotation": 0.7, "sun_disc": True, "sun_size": 0.6, "sun_intensity": 1.5,
       "altitude": 200.0, "air_density": 1.2, "dust_density": 0.8, "ozone_density": 1.1}


def install_ref_textures(R) -> None:
    """The reference build's Context.textures for the pinning materials: the
    image textures in order, then the sky texture of the sky material made by
    the reference's own sky model (its texture follows the scene's images)."""
    tex = textures()
    R.set_textures(tex)
    xyz = R.sky_texture(512, 512, SKY["sun_elevation"], SKY["altitude"], SKY["air_density"], SKY["dust_density"],
                        SKY["ozone_density"])
    import numpy as np

    rgba = np.concatenate([xyz, np.ones(xyz.shape[:2] + (1,), np.float32)], axis=-1)
    R.set_texture(len(tex), rgba)


def _image_params(path, colorspace, projection="FLAT"):
    return {"filepath": path, "interpolation": "Linear", "projection": projection, "extension": "REPEAT",
            "source": "FILE", "colorspace": colorspace, "alpha": "STRAIGHT"}


def textures() -> dict:
    """The pinning textures, by file name: an sRGB RGBA byte image, a
    single-channel 16-bit image and a float RGB environment."""
    import numpy as np

    rng = np.random.default_rng(31)
    return {
        "textures/albedo.png": rng.integers(0, 256, (13, 17, 4), dtype=np.uint8),
        "textures/rough.png": rng.integers(0, 65536, (9, 6), dtype=np.uint16),
        "textures/sky.exr": rng.exponential(1.0, (8, 16, 3)).astype(np.float32),
    }


def scene() -> dict:
    """A one-quad scene carrying the pinning materials (for the oracle and the codegen)."""
    import numpy as np

    from raymond_b200 import scenes

    sc = scenes.cornell(seed=1, envmap_exponent=2)
    sc["materials"] = materials()
    sc["textures"] = textures()
    for sh in sc["shapes"]:
        sh["materials"] = np.zeros_like(sh["materials"])
    return sc


def ref_scenes() -> dict[str, dict]:
    """Scenes whose materials the host build of the reference carries (one
    dispatch table each), by name: the pinning material set and the scenes of
    the reference-render comparison."""
    from raymond_b200 import scenes

    return {
        "pin": scene(),
        "cornell": scenes.cornell(seed=1, envmap_exponent=6),
        "cornell_all_lights": scenes.cornell_all_lights(seed=4, envmap_exponent=5),
        "spheres_small": scenes.spheres_terrain(seed=3, num_spheres=12, terrain_cells=64, envmap_exponent=6),
        # the benchmark scene (bench.py's reference arm)
        "spheres_terrain": scenes.spheres_terrain(seed=1),
    }
