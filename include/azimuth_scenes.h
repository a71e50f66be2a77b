/*
 * azimuth_scenes.h -- seeded procedural scenes built in azimuth's structs.
 *
 * azimuth loads scenes from XML (src/azimuth_xml.cpp:3021-3930); these
 * generators build the same in-memory result directly: spheres, meshes,
 * materials, lights and textures finalised exactly as the importer's
 * post-processing does (src/azimuth_xml.cpp:3632-3915), including azimuth's own
 * binary BVHs (src/azimuth_bvh.cpp).  The scene returned is therefore a valid
 * input both for azimuth's ProduceImageInLinearSpace and for
 * az_gpu_produce_image.
 */
#ifndef AZIMUTH_SCENES_H
#define AZIMUTH_SCENES_H

#include "azimuth_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    AZ_SCENE_CORNELL = 0,        /* Cornell box, 10+2 triangles, 2 spheres (mirror + diffuse) */
    AZ_SCENE_DENSE_MESH = 1,     /* Cornell walls + light around a Perlin-displaced icosphere,
                                    faces split round-robin over the 7 BRDF models */
    AZ_SCENE_MOTION_ENV = 2,     /* moving spheres, 30% dielectric, HDR environment map */
    AZ_SCENE_INTERIOR = 3,       /* three rooms joined by doorways, one light */
    AZ_SCENE_FEATURES = 100,     /* every light type, textures, Perlin bump, glossy mirror,
                                    dielectric, motion, transformed instance, ambient */
    AZ_SCENE_ENV_SPHERES = 101   /* a few spheres under an HDR environment map */
};

typedef struct az_gen_params {
    uint32_t width, height;      /* 0 = scene default */
    uint32_t spp;                /* camera SampleCount; 0 = default */
    uint32_t max_depth;          /* scene MaxRecursionDepth; 0 = default */
    uint32_t detail;             /* icosphere subdivisions / sphere count / triangle budget; 0 = default */
    int32_t  filter;             /* -1 = default, else AZ_Filter_* */
    int32_t  importance_sampling;/* -1 = default, 0 = uniform hemisphere, 1 = cosine */
    uint32_t env_width, env_height; /* environment map size; 0 = default */
    uint32_t flags;              /* AZ_GEN_* */
} az_gen_params;

enum {
    /* Leave the meshes as the importer has them before its post-processing:
     * no triangles, areas or entity BVHs (BVHRoot holds the other entities
     * only); az_generated_scene.soup is then the only copy of the geometry,
     * for az_gpu_scene_create_from_meshes. */
    AZ_GEN_SOUP_ONLY = 1
};

typedef struct az_generated_scene {
    az_scene *scene;
    az_camera *camera;
    az_epsilon_values *epsilons;
    int32_t filter_type;         /* filter the scene is meant to be rendered with */
    uint32_t backface_culling;
    const float *perlin_gradients;  /* 256*3 floats used by its Perlin textures, or NULL */
    uint64_t triangle_count;
    uint64_t sphere_count;
    void *owner;                 /* internal */
    const az_mesh_soup *soup;    /* the meshes before post-processing (vertices, faces, UVs, descriptions) */
} az_generated_scene;

/* Returns 0 on success. `params` may be NULL. */
int az_scene_generate(int32_t scene_id, uint64_t seed, const az_gen_params *params,
                      az_generated_scene *out);
void az_scene_release(az_generated_scene *scene);

#ifdef __cplusplus
}
#endif
#endif
