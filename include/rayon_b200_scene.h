/*
 * rayon_b200_scene.h - plain-data scene types of the rayon_b200 C-ABI
 * (material description and the enum numberings shared with the reference's
 * Scene::SceneDescription). Included by rayon_b200.h.
 */
#ifndef RAYON_B200_SCENE_H
#define RAYON_B200_SCENE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Numbering of Scene::MaterialType (scene_description.hpp:29-43). */
typedef enum rb_material_type {
  RB_MAT_LAMBERTIAN = 0, RB_MAT_METAL, RB_MAT_MIRROR, RB_MAT_ROUGH_MIRROR, RB_MAT_GLASS,
  RB_MAT_DIELECTRIC, RB_MAT_LIGHT, RB_MAT_CONSTANT, RB_MAT_SHOW_NORMALS, RB_MAT_SDF_MATERIAL,
  RB_MAT_ANISOTROPIC_METAL, RB_MAT_THIN_FILM, RB_MAT_CLEAR_COAT
} rb_material_type;

/* Numbering of Scene::GeometryType (scene_description.hpp:252-260). */
typedef enum rb_geometry_type {
  RB_GEOM_SPHERE = 0, RB_GEOM_RECTANGLE, RB_GEOM_CUBE, RB_GEOM_DISPLACED_SPHERE,
  RB_GEOM_TRIANGLE, RB_GEOM_TRIANGLE_MESH, RB_GEOM_SDF_PRIMITIVE
} rb_geometry_type;

/* Numbering of Scene::SDFType (scene_description.hpp:296-309); ROUND_BOX is
 * an addition (a box with rounded edges, parameters = half extents, radius in
 * `rotation[0]`-independent field `round_radius`). */
typedef enum rb_sdf_type {
  RB_SDF_SPHERE = 0, RB_SDF_BOX, RB_SDF_TORUS, RB_SDF_CAPSULE, RB_SDF_CYLINDER, RB_SDF_PLANE,
  RB_SDF_MANDELBULB, RB_SDF_DEATH_STAR, RB_SDF_CUT_HOLLOW_SPHERE, RB_SDF_OCTAHEDRON,
  RB_SDF_PYRAMID, RB_SDF_CUSTOM, RB_SDF_ROUND_BOX = 32
} rb_sdf_type;

/* Mirrors Scene::MaterialDesc (scene_description.hpp:58-101): vectors FP64,
 * scalars FP32. rb_material_default() gives MaterialDesc()'s defaults. */
typedef struct rb_material_desc {
  int32_t type;
  double albedo[3];
  double emission[3];
  float roughness, metallic, refractive_index, transmission, anisotropy;
  double eta[3];
  double k[3];
  int32_t texture_id;
  float film_thickness, film_ior;
  int32_t pattern;
  double pattern_color[3];
  float pattern_param1, pattern_param2;
} rb_material_desc;


#ifdef __cplusplus
}
#endif
#endif /* RAYON_B200_SCENE_H */
