"""Node graphs in the reference's exporter format.

A material is a dict node-name -> {"type", "inputs", "parameters"} exactly as
scripts/blender_exporter/raymond_blender/materials.py writes it (inputs keyed
by Blender socket identifier, each with "type" and either "value" or
"links": [[node, output-socket]]).  The defaults below are Blender's node
defaults, the same values the exporter's library/*.default.json carries.
"""
from __future__ import annotations

from typing import Any, Sequence


def _v(t: str, value=None, link: tuple[str, str] | None = None) -> dict[str, Any]:
    d: dict[str, Any] = {"type": t}
    if link is not None:
        d["links"] = [list(link)]
    elif value is not None:
        d["value"] = list(value) if isinstance(value, (list, tuple)) else value
    return d


def principled_inputs(base_color: Sequence[float] = (0.8, 0.8, 0.8, 1.0), roughness: float = 0.5,
                      metallic: float = 0.0, specular: float = 0.5, transmission: float = 0.0,
                      ior: float = 1.45, emission: Sequence[float] = (0.0, 0.0, 0.0, 1.0),
                      emission_strength: float = 1.0, alpha: float = 1.0, clearcoat: float = 0.0,
                      sheen: float = 0.0, anisotropic: float = 0.0) -> dict[str, Any]:
    bc = list(base_color) + [1.0] * (4 - len(base_color))
    return {
        "Base Color": _v("RGBA", bc),
        "Subsurface": _v("VALUE", 0.0),
        "Subsurface Radius": _v("VECTOR", [1.0, 0.2, 0.1]),
        "Subsurface Color": _v("RGBA", [0.8, 0.8, 0.8, 1.0]),
        "Subsurface IOR": _v("VALUE", 1.4),
        "Subsurface Anisotropy": _v("VALUE", 0.0),
        "Metallic": _v("VALUE", metallic),
        "Specular": _v("VALUE", specular),
        "Specular Tint": _v("VALUE", 0.0),
        "Roughness": _v("VALUE", roughness),
        "Anisotropic": _v("VALUE", anisotropic),
        "Anisotropic Rotation": _v("VALUE", 0.0),
        "Sheen": _v("VALUE", sheen),
        "Sheen Tint": _v("VALUE", 0.5),
        "Clearcoat": _v("VALUE", clearcoat),
        "Clearcoat Roughness": _v("VALUE", 0.03),
        "IOR": _v("VALUE", ior),
        "Transmission": _v("VALUE", transmission),
        "Transmission Roughness": _v("VALUE", 0.0),
        "Emission": _v("RGBA", list(emission)),
        "Emission Strength": _v("VALUE", emission_strength),
        "Alpha": _v("VALUE", alpha),
        "Normal": _v("VECTOR", [0.0, 0.0, 0.0]),
        "Clearcoat Normal": _v("VECTOR", [0.0, 0.0, 0.0]),
        "Tangent": _v("VECTOR", [0.0, 0.0, 0.0]),
        "Weight": _v("VALUE", 0.0),
    }


def _principled_node(**kw) -> dict[str, Any]:
    return {"type": "BSDF_PRINCIPLED", "inputs": principled_inputs(**kw),
            "parameters": {"distribution": "GGX", "subsurface_method": "RANDOM_WALK"}}


def _output(link: tuple[str, str]) -> dict[str, Any]:
    return {"type": "OUTPUT_MATERIAL",
            "inputs": {"Surface": _v("SHADER", link=link), "Volume": _v("SHADER"),
                       "Displacement": _v("VECTOR", [0.0, 0.0, 0.0]), "Thickness": _v("VALUE", 0.0)},
            "parameters": {}}


def principled(**kw) -> dict[str, Any]:
    """Principled BSDF -> Material Output (the exporter's default material)."""
    return {"Principled BSDF": _principled_node(**kw), "Material Output": _output(("Principled BSDF", "BSDF"))}


def principled_noise_ramp(base_color: Sequence[float], roughness: float, metallic: float,
                          noise_scale: float = 5.0, noise_detail: float = 2.0,
                          ramp: Sequence[tuple[float, Sequence[float]]] = ((0.3, (0.05, 0.05, 0.05, 1.0)),
                                                                           (0.7, (0.95, 0.95, 0.95, 1.0))),
                          mix_factor: float = 0.5) -> dict[str, Any]:
    """Noise Texture -> ColorRamp -> Mix(A = base colour, B = ramp) -> Principled Base Color."""
    bc = list(base_color) + [1.0] * (4 - len(base_color))
    pnode = _principled_node(roughness=roughness, metallic=metallic)
    pnode["inputs"]["Base Color"] = _v("RGBA", link=("Mix", "Result_Color"))
    return {
        "Noise Texture": {
            "type": "TEX_NOISE",
            "inputs": {"Vector": _v("VECTOR", [0.0, 0.0, 0.0]), "W": _v("VALUE", 0.0),
                       "Scale": _v("VALUE", noise_scale), "Detail": _v("VALUE", noise_detail),
                       "Roughness": _v("VALUE", 0.5), "Distortion": _v("VALUE", 0.0)},
            "parameters": {"noise_dimensions": "3D"},
        },
        "ColorRamp": {
            "type": "VALTORGB",
            "inputs": {"Fac": _v("VALUE", link=("Noise Texture", "Fac"))},
            "parameters": {"color_mode": "RGB", "interpolation": "LINEAR", "hue_interpolation": "NEAR",
                           "elements": [{"position": p, "color": list(c)} for p, c in ramp]},
        },
        "Mix": {
            "type": "MIX",
            "inputs": {"Factor_Float": _v("VALUE", mix_factor), "Factor_Vector": _v("VECTOR", [0.5, 0.5, 0.5]),
                       "A_Float": _v("VALUE", 0.0), "B_Float": _v("VALUE", 0.0),
                       "A_Vector": _v("VECTOR", [0.0, 0.0, 0.0]), "B_Vector": _v("VECTOR", [0.0, 0.0, 0.0]),
                       "A_Color": _v("RGBA", bc), "B_Color": _v("RGBA", link=("ColorRamp", "Color"))},
            "parameters": {"type": "RGBA", "clamp_result": False, "clamp_factor": True,
                           "factor_mode": "UNIFORM", "blend_type": "MIX"},
        },
        "Principled BSDF": pnode,
        "Material Output": _output(("Principled BSDF", "BSDF")),
    }


def emission(color: Sequence[float] = (1.0, 1.0, 1.0, 1.0), strength: float = 1.0) -> dict[str, Any]:
    """Emission -> Material Output (an emissive surface: becomes a shape light)."""
    c = list(color) + [1.0] * (4 - len(color))
    return {
        "Emission": {"type": "EMISSION",
                     "inputs": {"Color": _v("RGBA", c), "Strength": _v("VALUE", strength),
                                "Weight": _v("VALUE", 0.0)},
                     "parameters": {}},
        "Material Output": _output(("Emission", "Emission")),
    }


def world(color: Sequence[float] = (0.051, 0.051, 0.051, 1.0), strength: float = 1.0) -> dict[str, Any]:
    """Background -> World Output (library/world.default.json)."""
    c = list(color) + [1.0] * (4 - len(color))
    return {
        "World Output": {"type": "OUTPUT_WORLD",
                         "inputs": {"Surface": _v("SHADER", link=("Background", "Background")),
                                    "Volume": _v("SHADER")},
                         "parameters": {}},
        "Background": {"type": "BACKGROUND",
                       "inputs": {"Color": _v("RGBA", c), "Strength": _v("VALUE", strength),
                                  "Weight": _v("VALUE", 0.0)},
                       "parameters": {}},
    }


def light(color: Sequence[float] = (1.0, 1.0, 1.0, 1.0), strength: float = 1.0) -> dict[str, Any]:
    """Emission -> Light Output (library/light.default.json)."""
    c = list(color) + [1.0] * (4 - len(color))
    return {
        "Emission": {"type": "EMISSION",
                     "inputs": {"Color": _v("RGBA", c), "Strength": _v("VALUE", strength),
                                "Weight": _v("VALUE", 0.0)},
                     "parameters": {}},
        "Light Output": {"type": "OUTPUT_LIGHT",
                         "inputs": {"Surface": _v("SHADER", link=("Emission", "Emission"))},
                         "parameters": {}},
    }
