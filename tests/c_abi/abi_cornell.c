/*
 * A C11 caller of include/raymond.h, built and run by tests/test_c_abi.py.
 *
 *   abi_cornell layout          prints size, alignment and every field offset
 *                               of the header's structs (compared with the
 *                               Python ctypes mirror, and with the reference's
 *                               bridge layout, on the CPU)
 *   abi_cornell render OUT.bin  builds a Cornell box lit by a shape light and
 *                               one light record of each type (area, point,
 *                               spot, sun) from C arrays, renders it on GPU 0
 *                               and writes float32 images to OUT.bin:
 *                                 1. rmd_render, PCG32 seed 1, sample 0,
 *                                    depth 8, MIS: film sums, W*H*3
 *                                 2. rmd_render_frame with the reference's
 *                                    Uniforms (TEA, random_seed 1, then 2,
 *                                    accumulating) and rmd_film_normalize with
 *                                    exposure 1.5 and the Hable tonemap: W*H*4
 *                               and prints the per-instance records.
 * The scene's numbers are repeated in tests/test_c_abi.py (cabi_scene), which
 * renders the same scene with the oracle.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "raymond.h"

#define W 96
#define H 96

/* ------------------------------------------------------------------ layout */

#define S(T) printf("struct %s %zu %zu\n", #T, sizeof(T), _Alignof(T))
#define F(T, f) printf("field %s %s %zu\n", #T, #f, offsetof(T, f))

static void print_layout(void) {
    S(rmd_node_param); F(rmd_node_param, key); F(rmd_node_param, kind); F(rmd_node_param, string_value);
    F(rmd_node_param, number_value); F(rmd_node_param, numbers); F(rmd_node_param, num_numbers);
    S(rmd_node_input); F(rmd_node_input, name); F(rmd_node_input, type); F(rmd_node_input, num_values);
    F(rmd_node_input, values); F(rmd_node_input, link_node); F(rmd_node_input, link_socket);
    F(rmd_node_input, num_links);
    S(rmd_node); F(rmd_node, name); F(rmd_node, type); F(rmd_node, num_inputs); F(rmd_node, inputs);
    F(rmd_node, num_params); F(rmd_node, params);
    S(rmd_material); F(rmd_material, name); F(rmd_material, num_nodes); F(rmd_material, nodes);
    S(rmd_shape); F(rmd_shape, num_vertices); F(rmd_shape, num_faces); F(rmd_shape, vertices);
    F(rmd_shape, normals); F(rmd_shape, texcoords); F(rmd_shape, indices); F(rmd_shape, materials);
    S(rmd_entity); F(rmd_entity, shape); F(rmd_entity, visibility); F(rmd_entity, matrix);
    S(rmd_light_info); F(rmd_light_info, shader_index); F(rmd_light_info, casts_shadows); F(rmd_light_info, uses_mis);
    S(rmd_area_light); F(rmd_area_light, info); F(rmd_area_light, transform); F(rmd_area_light, color);
    F(rmd_area_light, is_circular);
    S(rmd_point_light); F(rmd_point_light, info); F(rmd_point_light, location); F(rmd_point_light, radius);
    F(rmd_point_light, color);
    S(rmd_sun_light); F(rmd_sun_light, info); F(rmd_sun_light, direction); F(rmd_sun_light, cos_angle);
    F(rmd_sun_light, color);
    S(rmd_spot_light); F(rmd_spot_light, info); F(rmd_spot_light, location); F(rmd_spot_light, direction);
    F(rmd_spot_light, radius); F(rmd_spot_light, color); F(rmd_spot_light, spot_size); F(rmd_spot_light, spot_blend);
    S(rmd_camera); F(rmd_camera, transform); F(rmd_camera, near_clip); F(rmd_camera, far_clip);
    F(rmd_camera, focal_length); F(rmd_camera, shift);
    S(rmd_per_instance_data); F(rmd_per_instance_data, vertex_offset); F(rmd_per_instance_data, face_offset);
    F(rmd_per_instance_data, light_face_offset); F(rmd_per_instance_data, light_face_count);
    F(rmd_per_instance_data, light_index); F(rmd_per_instance_data, bounds_min);
    F(rmd_per_instance_data, bounds_size); F(rmd_per_instance_data, point_transform);
    F(rmd_per_instance_data, normal_transform); F(rmd_per_instance_data, visibility);
    S(rmd_uniforms); F(rmd_uniforms, num_lens_surfaces); F(rmd_uniforms, frame_index); F(rmd_uniforms, random_seed);
    F(rmd_uniforms, accumulate); F(rmd_uniforms, lens_spectral); F(rmd_uniforms, sensor_scale);
    F(rmd_uniforms, camera_scale); F(rmd_uniforms, focus); F(rmd_uniforms, exposure); F(rmd_uniforms, stop_index);
    F(rmd_uniforms, relative_stop); F(rmd_uniforms, num_aperture_blades); F(rmd_uniforms, sampling_mode);
    F(rmd_uniforms, tonemapping); F(rmd_uniforms, rr); F(rmd_uniforms, rr_depth); F(rmd_uniforms, output_channel);
    S(rmd_texture); F(rmd_texture, name); F(rmd_texture, width); F(rmd_texture, height); F(rmd_texture, channels);
    F(rmd_texture, format); F(rmd_texture, data);
    S(rmd_scene_desc); F(rmd_scene_desc, num_surface_materials); F(rmd_scene_desc, surface_materials);
    F(rmd_scene_desc, num_light_materials); F(rmd_scene_desc, light_materials); F(rmd_scene_desc, num_shapes);
    F(rmd_scene_desc, shapes); F(rmd_scene_desc, num_entities); F(rmd_scene_desc, entities);
    F(rmd_scene_desc, world_shader); F(rmd_scene_desc, envmap_exponent); F(rmd_scene_desc, num_area_lights);
    F(rmd_scene_desc, area_lights); F(rmd_scene_desc, num_point_lights); F(rmd_scene_desc, point_lights);
    F(rmd_scene_desc, num_sun_lights); F(rmd_scene_desc, sun_lights); F(rmd_scene_desc, num_spot_lights);
    F(rmd_scene_desc, spot_lights); F(rmd_scene_desc, camera); F(rmd_scene_desc, num_textures);
    F(rmd_scene_desc, textures);
    S(rmd_render_settings); F(rmd_render_settings, spp); F(rmd_render_settings, max_depth);
    F(rmd_render_settings, sampling_mode); F(rmd_render_settings, rng); F(rmd_render_settings, seed);
    F(rmd_render_settings, first_sample); F(rmd_render_settings, film_fp64); F(rmd_render_settings, reserved);
    S(rmd_stats); F(rmd_stats, paths); F(rmd_stats, segments); F(rmd_stats, shadow_rays); F(rmd_stats, iterations);
    F(rmd_stats, ms_total); F(rmd_stats, ms_trace); F(rmd_stats, ms_shade); F(rmd_stats, ms_shadow);
    F(rmd_stats, ms_film); F(rmd_stats, pool_size); F(rmd_stats, errors); F(rmd_stats, rays); F(rmd_stats, ms_guide);
    F(rmd_stats, ms_guide_train); F(rmd_stats, invalid_samples);
    S(rmd_bvh_stats); F(rmd_bvh_stats, builder); F(rmd_bvh_stats, levels); F(rmd_bvh_stats, nodes);
    F(rmd_bvh_stats, build_ms); F(rmd_bvh_stats, sah_cost); F(rmd_bvh_stats, cluster_iterations);
    S(rmd_tune_result); F(rmd_tune_result, shade_min_blocks); F(rmd_tune_result, trace_blocks_per_sm);
    F(rmd_tune_result, pool_size); F(rmd_tune_result, calibration_spp); F(rmd_tune_result, ms_default);
    F(rmd_tune_result, ms_best);
    S(rmd_guide_settings); F(rmd_guide_settings, sampling); F(rmd_guide_settings, training);
    F(rmd_guide_settings, batch_size); F(rmd_guide_settings, learning_rate); F(rmd_guide_settings, reset);
    F(rmd_guide_settings, seed); F(rmd_guide_settings, step_records); F(rmd_guide_settings, replay_records);
    F(rmd_guide_settings, steps_per_batch); F(rmd_guide_settings, skip_light_records);
    F(rmd_guide_settings, guided_depth);
    S(rmd_guide_stats); F(rmd_guide_stats, steps); F(rmd_guide_stats, samples); F(rmd_guide_stats, records);
    F(rmd_guide_stats, last_loss);
    S(rmd_batch_view); F(rmd_batch_view, scene); F(rmd_batch_view, width); F(rmd_batch_view, height);
    F(rmd_batch_view, camera);
}

/* ------------------------------------------------------------------- scene */

/* one quad (two triangles) with a flat normal */
typedef struct {
    float v[4][3];
    float n[3];
} quad;

static const quad kWalls[5] = {
    {{{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}}, {0, 1, 0}},   /* floor */
    {{{0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}}, {0, -1, 0}},  /* ceiling */
    {{{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}}, {0, 0, 1}},   /* back */
    {{{0, 0, 0}, {0, 1, 0}, {0, 1, 1}, {0, 0, 1}}, {1, 0, 0}},   /* left */
    {{{1, 0, 0}, {1, 1, 0}, {1, 1, 1}, {1, 0, 1}}, {-1, 0, 0}},  /* right */
};
static const quad kLamp = {{{0.375f, 0.999f, 0.375f}, {0.625f, 0.999f, 0.375f}, {0.625f, 0.999f, 0.625f},
                            {0.375f, 0.999f, 0.625f}},
                           {0, -1, 0}};
static const float kColors[6][3] = {{0.7f, 0.7f, 0.7f}, {0.6f, 0.6f, 0.6f}, {0.5f, 0.6f, 0.7f},
                                    {0.7f, 0.2f, 0.2f}, {0.2f, 0.7f, 0.3f}, {0.3f, 0.3f, 0.6f}};
/* box [0.2, 0.5] x [0, 0.4] x [0.3, 0.6] */
static const float kBoxLo[3] = {0.2f, 0.0f, 0.3f}, kBoxHi[3] = {0.5f, 0.4f, 0.6f};

typedef struct {
    float vertices[4 * 3 * 6];
    float normals[4 * 3 * 6];
    float texcoords[4 * 2 * 6];
    uint32_t indices[6 * 6];
    uint16_t materials[2 * 6];
} mesh;

/* appends quad q as vertices 4k..4k+3, triangles (0,1,2) and (0,2,3) turned to face q.n */
static void add_quad(mesh *m, int k, const float v[4][3], const float n[3], uint16_t material) {
    for (int j = 0; j < 4; j++) {
        for (int c = 0; c < 3; c++) {
            m->vertices[3 * (4 * k + j) + c] = v[j][c];
            m->normals[3 * (4 * k + j) + c] = n[c];
        }
        m->texcoords[2 * (4 * k + j) + 0] = (float)(j == 1 || j == 2);
        m->texcoords[2 * (4 * k + j) + 1] = (float)(j >= 2);
    }
    /* winding: the geometric normal (v1 - v0) x (v2 - v0) should agree with n */
    float e1[3], e2[3], g[3];
    for (int c = 0; c < 3; c++) {
        e1[c] = v[1][c] - v[0][c];
        e2[c] = v[2][c] - v[0][c];
    }
    g[0] = e1[1] * e2[2] - e1[2] * e2[1];
    g[1] = e1[2] * e2[0] - e1[0] * e2[2];
    g[2] = e1[0] * e2[1] - e1[1] * e2[0];
    const int flip = g[0] * n[0] + g[1] * n[1] + g[2] * n[2] < 0;
    const uint32_t b = 4 * (uint32_t)k;
    const uint32_t t[6] = {b, flip ? b + 2 : b + 1, flip ? b + 1 : b + 2, b, flip ? b + 3 : b + 2, flip ? b + 2 : b + 3};
    memcpy(m->indices + 6 * k, t, sizeof t);
    m->materials[2 * k] = m->materials[2 * k + 1] = material;
}

static rmd_node_input value(const char *name, const char *type, int n, float a, float b, float c, float d) {
    rmd_node_input in;
    memset(&in, 0, sizeof in);
    in.name = name;
    in.type = type;
    in.num_values = n;
    in.values[0] = a;
    in.values[1] = b;
    in.values[2] = c;
    in.values[3] = d;
    return in;
}
static rmd_node_input link(const char *name, const char *type, const char *node, const char *socket) {
    rmd_node_input in = value(name, type, 0, 0, 0, 0, 0);
    in.link_node = node;
    in.link_socket = socket;
    in.num_links = 1;
    return in;
}

static int check(rmd_status s, const char *what) {
    if (s != RMD_OK) {
        fprintf(stderr, "%s failed (%d): %s\n", what, (int)s, rmd_last_error());
        exit(1);
    }
    return 0;
}

static int render(const char *out_path) {
    /* materials: six Principled surfaces and one emissive surface */
    static rmd_node_input pin[6][5], oin[7][1], ein[2];
    static rmd_node pnodes[6][2], enodes[2];
    static rmd_material surf[7];
    static const char *names[7] = {"floor", "ceiling", "back", "left", "right", "box", "lamp_quad"};
    for (int i = 0; i < 6; i++) {
        pin[i][0] = value("Base Color", "RGBA", 4, kColors[i][0], kColors[i][1], kColors[i][2], 1.0f);
        pin[i][1] = value("Roughness", "VALUE", 1, 0.5f, 0, 0, 0);
        pin[i][2] = value("Metallic", "VALUE", 1, 0.0f, 0, 0, 0);
        pin[i][3] = value("Specular", "VALUE", 1, 0.5f, 0, 0, 0);
        pin[i][4] = value("Normal", "VECTOR", 3, 0, 0, 0, 0); /* unlinked: the shading normal */
        oin[i][0] = link("Surface", "SHADER", "Principled BSDF", "BSDF");
        pnodes[i][0] = (rmd_node){"Principled BSDF", "BSDF_PRINCIPLED", 5, pin[i], 0, NULL};
        pnodes[i][1] = (rmd_node){"Material Output", "OUTPUT_MATERIAL", 1, oin[i], 0, NULL};
        surf[i] = (rmd_material){names[i], 2, pnodes[i]};
    }
    ein[0] = value("Color", "RGBA", 4, 1.0f, 1.0f, 1.0f, 1.0f);
    ein[1] = value("Strength", "VALUE", 1, 15.0f, 0, 0, 0);
    oin[6][0] = link("Surface", "SHADER", "Emission", "Emission");
    enodes[0] = (rmd_node){"Emission", "EMISSION", 2, ein, 0, NULL};
    enodes[1] = (rmd_node){"Material Output", "OUTPUT_MATERIAL", 1, oin[6], 0, NULL};
    surf[6] = (rmd_material){names[6], 2, enodes};

    /* light materials: a black world and a warm lamp */
    static rmd_node_input win[2], wout[1], lin[2], lout[1];
    static rmd_node wnodes[2], lnodes[2];
    win[0] = value("Color", "RGBA", 4, 0.0f, 0.0f, 0.0f, 1.0f);
    win[1] = value("Strength", "VALUE", 1, 1.0f, 0, 0, 0);
    wout[0] = link("Surface", "SHADER", "Background", "Background");
    wnodes[0] = (rmd_node){"Background", "BACKGROUND", 2, win, 0, NULL};
    wnodes[1] = (rmd_node){"World Output", "OUTPUT_WORLD", 1, wout, 0, NULL};
    lin[0] = value("Color", "RGBA", 4, 1.0f, 0.9f, 0.8f, 1.0f);
    lin[1] = value("Strength", "VALUE", 1, 1.0f, 0, 0, 0);
    lout[0] = link("Surface", "SHADER", "Emission", "Emission");
    lnodes[0] = (rmd_node){"Emission", "EMISSION", 2, lin, 0, NULL};
    lnodes[1] = (rmd_node){"Light Output", "OUTPUT_LIGHT", 1, lout, 0, NULL};
    rmd_material lmat[2] = {{"world", 2, wnodes}, {"lamp", 2, lnodes}};

    /* geometry: one shape for the walls, one for the box, one for the lamp quad */
    static mesh walls, box, lamp;
    for (int k = 0; k < 5; k++) add_quad(&walls, k, kWalls[k].v, kWalls[k].n, (uint16_t)k);
    const float *lo = kBoxLo, *hi = kBoxHi;
    const quad faces[6] = {
        {{{lo[0], lo[1], lo[2]}, {hi[0], lo[1], lo[2]}, {hi[0], lo[1], hi[2]}, {lo[0], lo[1], hi[2]}}, {0, -1, 0}},
        {{{lo[0], hi[1], lo[2]}, {hi[0], hi[1], lo[2]}, {hi[0], hi[1], hi[2]}, {lo[0], hi[1], hi[2]}}, {0, 1, 0}},
        {{{lo[0], lo[1], lo[2]}, {hi[0], lo[1], lo[2]}, {hi[0], hi[1], lo[2]}, {lo[0], hi[1], lo[2]}}, {0, 0, -1}},
        {{{lo[0], lo[1], hi[2]}, {hi[0], lo[1], hi[2]}, {hi[0], hi[1], hi[2]}, {lo[0], hi[1], hi[2]}}, {0, 0, 1}},
        {{{lo[0], lo[1], lo[2]}, {lo[0], hi[1], lo[2]}, {lo[0], hi[1], hi[2]}, {lo[0], lo[1], hi[2]}}, {-1, 0, 0}},
        {{{hi[0], lo[1], lo[2]}, {hi[0], hi[1], lo[2]}, {hi[0], hi[1], hi[2]}, {hi[0], lo[1], hi[2]}}, {1, 0, 0}},
    };
    for (int k = 0; k < 6; k++) add_quad(&box, k, faces[k].v, faces[k].n, 5);
    add_quad(&lamp, 0, kLamp.v, kLamp.n, 6);
    rmd_shape shapes[3] = {
        {20, 10, walls.vertices, walls.normals, walls.texcoords, walls.indices, walls.materials},
        {24, 12, box.vertices, box.normals, box.texcoords, box.indices, box.materials},
        {4, 2, lamp.vertices, lamp.normals, lamp.texcoords, lamp.indices, lamp.materials},
    };
    const uint32_t all = RMD_RAY_CAMERA | RMD_RAY_DIFFUSE | RMD_RAY_GLOSSY | RMD_RAY_TRANSMISSION |
                         RMD_RAY_VOLUME | RMD_RAY_SHADOW;
    rmd_entity entities[3];
    memset(entities, 0, sizeof entities);
    for (int e = 0; e < 3; e++) {
        entities[e].shape = (uint32_t)e;
        entities[e].visibility = all;
        for (int d = 0; d < 4; d++) entities[e].matrix[5 * d] = 1.0f;
    }

    /* one light record of each type, all shaded by the lamp material */
    rmd_light_info info = {1, 1, 0};
    rmd_area_light area;
    memset(&area, 0, sizeof area);
    area.info = info;
    /* float3x4 columns: rows of the world matrix [[0.2,0,0,0.5],[0,0,0.2,0.95],[0,-0.2,0,0.5]] */
    const float tr[3][4] = {{0.2f, 0, 0, 0.5f}, {0, 0, 0.2f, 0.95f}, {0, -0.2f, 0, 0.5f}};
    for (int c = 0; c < 3; c++)
        for (int rr = 0; rr < 4; rr++) area.transform[4 * c + rr] = tr[c][rr];
    area.color[0] = 4.0f, area.color[1] = 4.0f, area.color[2] = 4.0f;
    area.is_circular = 1;
    rmd_point_light point;
    memset(&point, 0, sizeof point);
    point.info = info;
    point.location[0] = 0.3f, point.location[1] = 0.7f, point.location[2] = 0.6f;
    point.radius = 0.05f;
    point.color[0] = 2.0f, point.color[1] = 2.0f, point.color[2] = 2.0f;
    rmd_spot_light spot;
    memset(&spot, 0, sizeof spot);
    spot.info = info;
    spot.location[0] = 0.5f, spot.location[1] = 0.9f, spot.location[2] = 0.8f;
    spot.direction[0] = 0.0f, spot.direction[1] = -1.0f, spot.direction[2] = 0.0f;
    spot.radius = 0.03f;
    spot.color[0] = 6.0f, spot.color[1] = 6.0f, spot.color[2] = 6.0f;
    spot.spot_size = 0.8f;
    spot.spot_blend = 0.05f;
    rmd_sun_light sun;
    memset(&sun, 0, sizeof sun);
    sun.info = info;
    sun.direction[0] = 0.0f, sun.direction[1] = 0.6f, sun.direction[2] = 0.8f;
    sun.cos_angle = 0.999f;
    sun.color[0] = 1.0f, sun.color[1] = 1.0f, sun.color[2] = 1.0f;

    rmd_camera cam;
    memset(&cam, 0, sizeof cam);
    /* camera at (0.5, 0.5, 2.3) looking down -z (column-major identity rotation) */
    cam.transform[0] = cam.transform[5] = cam.transform[10] = cam.transform[15] = 1.0f;
    cam.transform[12] = 0.5f, cam.transform[13] = 0.5f, cam.transform[14] = 2.3f;
    cam.near_clip = 0.1f;
    cam.far_clip = 100.0f;
    cam.focal_length = 2.5f;

    rmd_scene_desc d;
    memset(&d, 0, sizeof d);
    d.num_surface_materials = 7;
    d.surface_materials = surf;
    d.num_light_materials = 2;
    d.light_materials = lmat;
    d.num_shapes = 3;
    d.shapes = shapes;
    d.num_entities = 3;
    d.entities = entities;
    d.world_shader = 0;
    d.envmap_exponent = 4;
    d.num_area_lights = 1;
    d.area_lights = &area;
    d.num_point_lights = 1;
    d.point_lights = &point;
    d.num_sun_lights = 1;
    d.sun_lights = &sun;
    d.num_spot_lights = 1;
    d.spot_lights = &spot;
    d.camera = cam;

    rmd_context *ctx;
    rmd_scene *scene;
    rmd_renderer *r;
    check(rmd_context_create(0, &ctx), "rmd_context_create");
    check(rmd_scene_create(ctx, &d, &scene), "rmd_scene_create");
    check(rmd_renderer_create(scene, W, H, 0, &r), "rmd_renderer_create");

    rmd_per_instance_data inst[4];
    int32_t count = 0;
    check(rmd_scene_instance_data(scene, inst, 4, &count), "rmd_scene_instance_data");
    for (int i = 0; i < count; i++)
        printf("instance %d vertex_offset %u face_offset %u light_index %d light_face_count %u visibility %u "
               "bounds_min %g %g %g bounds_size %g %g %g\n",
               i, inst[i].vertex_offset, inst[i].face_offset, (int)inst[i].light_index, inst[i].light_face_count,
               (unsigned)inst[i].visibility, inst[i].bounds_min[0], inst[i].bounds_min[1], inst[i].bounds_min[2],
               inst[i].bounds_size[0], inst[i].bounds_size[1], inst[i].bounds_size[2]);

    FILE *f = fopen(out_path, "wb");
    if (!f) return 1;
    float *img = malloc(sizeof(float) * W * H * 4);
    rmd_render_settings s;
    memset(&s, 0, sizeof s);
    s.spp = 1;
    s.max_depth = 8;
    s.sampling_mode = RMD_SAMPLING_MIS;
    s.rng = RMD_RNG_PCG32;
    s.seed = 1;
    s.first_sample = 0;
    check(rmd_render(r, &s), "rmd_render");
    check(rmd_film_read(r, img, 0, RMD_TONEMAP_LINEAR, 1.0f), "rmd_film_read");
    fwrite(img, sizeof(float), (size_t)W * H * 3, f);

    /* two frames as Renderer.execute runs them (updateState advances the seed and frame index) */
    rmd_uniforms u;
    memset(&u, 0, sizeof u);
    u.accumulate = 0; /* the first frame also clears the film left by rmd_render */
    u.exposure = 1.5f;
    u.sampling_mode = RMD_SAMPLING_MIS;
    u.tonemapping = RMD_TONEMAP_HABLE;
    u.rr = RMD_RR_THROUGHPUT;
    u.output_channel = RMD_OUTPUT_IMAGE;
    for (uint32_t frame = 0; frame < 2; frame++) {
        u.frame_index = frame;
        u.random_seed = frame + 1;
        check(rmd_render_frame(r, &u, 8), "rmd_render_frame");
        u.accumulate = 1;
    }
    check(rmd_film_normalize(r, &u, img), "rmd_film_normalize");
    fwrite(img, sizeof(float), (size_t)W * H * 4, f);
    fclose(f);
    free(img);

    rmd_stats st;
    check(rmd_renderer_stats(r, &st), "rmd_renderer_stats");
    printf("paths %llu segments %llu\n", (unsigned long long)st.paths, (unsigned long long)st.segments);
    rmd_renderer_destroy(r);
    rmd_scene_destroy(scene);
    rmd_context_destroy(ctx);
    return 0;
}

int main(int argc, char **argv) {
    if (argc >= 2 && strcmp(argv[1], "layout") == 0) {
        print_layout();
        return 0;
    }
    if (argc >= 3 && strcmp(argv[1], "render") == 0) return render(argv[2]);
    fprintf(stderr, "usage: %s layout | render OUT.bin\n", argv[0]);
    return 2;
}
