/*
 * rayon_b200.h - C-ABI of the B200 path-tracing render path.
 *
 * Two groups of entry points:
 *
 *  1. The drop-in group. Same names, argument lists and semantics as the
 *     extern "C" block of RayON's CUDA renderer
 *     (src/rayon/gpu_renderers/renderer_cuda_device.cuh:8-67), so the
 *     unmodified host renderers (renderer_cuda_host.hpp,
 *     renderer_cuda_progressive_host.hpp) link against this library in place
 *     of the reference's .cu objects. Like the reference these return no
 *     status; failures are recorded and readable through rb_last_error().
 *
 *  2. The rb_* group: scene construction (the SceneDescription builder
 *     interface and its SAH BVH build), primary-hit queries, the batched
 *     multi-job wavefront engine and the serving loop. These return
 *     rb_status codes (0 = success, negative = error) and take an explicit
 *     CUDA stream (passed as void*, NULL = legacy default stream).
 *
 * No torch types cross this boundary: plain pointers, sizes and PODs.
 */
#ifndef RAYON_B200_H
#define RAYON_B200_H

#include <stddef.h>
#include <stdint.h>

#include "rayon_b200_scene.h"

#ifdef __cplusplus
namespace CudaScene { struct Scene; }
typedef CudaScene::Scene rb_cuda_scene;
extern "C" {
#define RB_DEFAULT(x) = x
#else
typedef struct CudaScene_Scene rb_cuda_scene;
#define RB_DEFAULT(x)
#include <stdbool.h>
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum rb_status {
  RB_OK = 0,
  RB_ERR_INVALID_ARG = -1,
  RB_ERR_CUDA = -2,
  RB_ERR_OUT_OF_MEMORY = -3,
  RB_ERR_NOT_FOUND = -4,
  RB_ERR_CAPACITY = -5,   /* admission refused: slot or memory budget */
  RB_ERR_STATE = -6,      /* call made in the wrong state */
  RB_ERR_UNSUPPORTED = -7
} rb_status;

/* Last error message of the calling thread ("" when none). */
const char *rb_last_error(void);
/* Library version string. */
const char *rb_version(void);

/* ======================================================================== */
/* 1. Drop-in group (renderer_cuda_device.cuh:8-67)                          */
/* ======================================================================== */

/* Replaces initCudaStreams / cleanupCudaStreams
 * (renderer_cuda_device.cuh:12-13; renderer_cuda_device.cu:35-54):
 * create / destroy the display stream and its pinned staging buffer. */
void initCudaStreams(void);
void cleanupCudaStreams(void);

/* Replaces renderPixelsCUDAAccumulative (renderer_cuda_device.cuh:18-24,
 * renderer_cuda_device.cu:157-322). Adds samples_to_add samples per pixel to
 * the accumulation buffer behind *d_accum_buffer_ptr (allocated on first use;
 * uploaded from the host float3 accum_buffer when that is non-NULL, zeroed
 * otherwise; downloaded into accum_buffer after every call when non-NULL).
 * `image` is unused, as in the reference. Returns W*H*samples_to_add, or 0
 * when scene is NULL or the call failed (see rb_last_error()). */
unsigned long long renderPixelsCUDAAccumulative(
    unsigned char *image, float *accum_buffer, rb_cuda_scene *scene, int width, int height,
    double cam_center_x, double cam_center_y, double cam_center_z, double pixel00_x,
    double pixel00_y, double pixel00_z, double delta_u_x, double delta_u_y, double delta_u_z,
    double delta_v_x, double delta_v_y, double delta_v_z, int samples_to_add,
    int total_samples_so_far, int max_depth, void **d_rand_states_ptr,
    void **d_accum_buffer_ptr, double cam_u_x, double cam_u_y, double cam_u_z, double cam_v_x,
    double cam_v_y, double cam_v_z, void *d_pixel_sample_counts RB_DEFAULT(NULL),
    int min_adaptive_samples RB_DEFAULT(32), float adaptive_threshold RB_DEFAULT(0.01f));

/* Replace freeDeviceRandomStates / freeDeviceAccumBuffer / resetDeviceAccumBuffer
 * (renderer_cuda_device.cuh:27-33; renderer_cuda_device.cu:108-130). */
void freeDeviceRandomStates(void *d_rand_states);
void freeDeviceAccumBuffer(void *d_accum_buffer);
void resetDeviceAccumBuffer(void *d_accum_buffer, int num_pixels);

/* Replace the global shading setters (renderer_cuda_device.cuh:36-50;
 * renderer_cuda_device.cu:57-79). Defaults match the reference's
 * __constant__ initialisers (renderer_cuda_device.cu:18-26): light 1.0,
 * background 1.0, metal fuzziness 0.8, glass IOR 1.5, DOF off, aperture 0.1
 * (a disk radius), focus distance 10. */
void setLightIntensity(float intensity);
void setBackgroundIntensity(float intensity);
void setMetalFuzziness(float fuzziness);
void setGlassRefractionIndex(float index);
void setDOFEnabled(bool enabled);
void setDOFAperture(float aperture);
void setDOFFocusDistance(float distance);

/* Replaces convertAccumToDisplayCUDA (renderer_cuda_device.cuh:54-55;
 * renderer_cuda_device.cu:340-393): sum/spp -> gamma -> clamp 0.999 -> u8. */
void convertAccumToDisplayCUDA(void *d_accum_buffer, unsigned char *display_image, int width,
                               int height, int channels, int num_samples, float gamma,
                               void *d_pixel_sample_counts RB_DEFAULT(NULL));

/* No counterpart in the reference. Same conversion and output as
 * convertAccumToDisplayCUDA, for callers that cannot allocate device memory
 * when they ask for a frame (device memory owned by another allocator or held
 * to a fixed budget; loops that must avoid cudaMalloc's implicit device-wide
 * synchronisation). The 8-bit image is staged in a fixed 8 MiB device array
 * that is part of the library (held on every GPU that loads it until exit):
 * width * height * channels above 8388608 is rejected with RB_ERR_CAPACITY.
 * Allocates nothing. The array's device address is looked up on the first call
 * per device (make that call before any stream capture) and cached; the cache
 * does not survive cudaDeviceReset. Calls share the array, so calls that
 * overlap on the GPU race. The kernel and the copy run on the legacy default
 * stream. Returns an rb_status. */
int convertAccumToDisplayNoAlloc(void *d_accum_buffer, unsigned char *display_image, int width,
                                 int height, int channels, int num_samples, float gamma,
                                 void *d_pixel_sample_counts);

/* Replace the adaptive-sampling buffer helpers (renderer_cuda_device.cuh:58-63;
 * renderer_cuda_device.cu:397-437). countConvergedPixels reduces on the device
 * and copies back one integer. */
void allocateAdaptiveBuffer(void **d_pixel_sample_counts, int num_pixels);
void resetAdaptiveBuffer(void *d_pixel_sample_counts, int num_pixels);
void freeAdaptiveBuffer(void *d_pixel_sample_counts);
int countConvergedPixels(void *d_pixel_sample_counts, int num_pixels);

/* Replaces renderSampleHeatmapCUDA (renderer_cuda_device.cuh:66-67;
 * renderer_cuda_device.cu:440-478). */
void renderSampleHeatmapCUDA(void *d_pixel_sample_counts, unsigned char *display_image, int width,
                             int height, int channels, int max_samples_for_scale);

/* ======================================================================== */
/* 2. Scene description (host, FP64)                                         */
/* ======================================================================== */

void rb_material_default(rb_material_desc *out);

typedef struct rb_scene_desc rb_scene_desc; /* opaque host scene */

rb_scene_desc *rb_scene_create(void);
void rb_scene_destroy(rb_scene_desc *s);

/* Builder interface, after SceneDescription (scene_description.hpp:487-711).
 * Bounds are computed exactly as the reference computes them (FP64; triangle
 * boxes padded by 1e-4). Geometry adders return the geometry index. */
int rb_scene_add_material(rb_scene_desc *s, const rb_material_desc *m);
int rb_scene_add_sphere(rb_scene_desc *s, const double center[3], double radius, int mat_id);
int rb_scene_add_displaced_sphere(rb_scene_desc *s, const double center[3], double radius,
                                  int mat_id, float displacement_scale, int pattern_type);
int rb_scene_add_rectangle(rb_scene_desc *s, const double corner[3], const double u[3],
                           const double v[3], int mat_id);
int rb_scene_add_triangle(rb_scene_desc *s, const double v0[3], const double v1[3],
                          const double v2[3], int mat_id);
int rb_scene_add_triangle_with_normals(rb_scene_desc *s, const double v0[3], const double v1[3],
                                       const double v2[3], const double n0[3],
                                       const double n1[3], const double n2[3], int mat_id);
int rb_scene_add_sdf(rb_scene_desc *s, int sdf_type, const double position[3],
                     const double params[3], const double rotation[3], int mat_id);
/* Bulk adders (same per-item semantics; n items, row-major):
 * spheres: cr = n x 4 (cx, cy, cz, r); triangles: v = n x 9, nrm = n x 9 or NULL.
 * mat_ids may be NULL (then mat_id is used for all). Return first index. */
int64_t rb_scene_add_spheres(rb_scene_desc *s, const double *cr, const int32_t *mat_ids,
                             int mat_id, int64_t n);
int64_t rb_scene_add_triangles(rb_scene_desc *s, const double *v, const double *nrm,
                               const int32_t *mat_ids, int mat_id, int64_t n);
/* Wavefront OBJ mesh (replaces Scene::OBJLoader::loadOBJ,
 * src/rayon/scenes/obj_loader.hpp:34-140, with its semantics: positions
 * scaled then translated, fan triangulation, 1-based and negative indices,
 * vertex normals only when all three are valid, invalid triangles skipped).
 * position / scale may be NULL (0 and 1). Returns the number of triangles
 * added, RB_ERR_NOT_FOUND when the file cannot be opened, RB_ERR_INVALID_ARG
 * on a malformed face index (where the reference throws; triangles of earlier
 * faces stay added). */
int64_t rb_scene_load_obj(rb_scene_desc *s, const char *path, int mat_id, const double position[3],
                          const double scale[3]);
int rb_scene_set_visible(rb_scene_desc *s, int64_t geom_index, int visible);
int64_t rb_scene_num_geometries(const rb_scene_desc *s);
int rb_scene_num_materials(const rb_scene_desc *s);
/* Smooth-union blend radius for the SDF primitives of this scene (0 = hard union). */
int rb_scene_set_sdf_blend(rb_scene_desc *s, float k, int max_steps, float epsilon);

/* SAH BVH build. Replaces SceneDescription::buildBVH
 * (scene_description.hpp:717-778, 793-925) with the same node array, the same
 * pre-order numbering and the same leaf-order geometry permutation for
 * max_leaf = 4, built in parallel across subtrees with `threads` host threads
 * (0 = all cores). max_leaf other than 4 is the tunable variant. */
int rb_scene_build_bvh(rb_scene_desc *s);
int rb_scene_build_bvh_ex(rb_scene_desc *s, int max_leaf, int threads);

/* Host BVH node export (for parity): arrays of length rb_scene_num_bvh_nodes.
 * Any pointer may be NULL. bounds = n x 6 (min xyz, max xyz) FP64. a/b =
 * left/right child (interior) or first_geom_idx/geom_count (leaf). */
int64_t rb_scene_num_bvh_nodes(const rb_scene_desc *s);
int rb_scene_bvh_root(const rb_scene_desc *s);
int rb_scene_export_bvh(const rb_scene_desc *s, double *bounds, int32_t *a, int32_t *b,
                        uint8_t *is_leaf, uint8_t *split_axis);
/* Original insertion index of the geometry now at each position (n). */
int rb_scene_export_order(const rb_scene_desc *s, int64_t *orig_index);
/* Geometry export (post-reorder), for the oracle: n x 20 doubles per item:
 * [type, material_id, visible, has_normals, p0..p15] where p holds the
 * type's parameters (sphere: c, r; rect: corner, u, v; tri: v0, v1, v2, n0,
 * n1, n2 truncated to 16 -> see rb_scene_export_geometry_full). */
int rb_scene_export_geometry_full(const rb_scene_desc *s, double *out /* n x 32 */);
int rb_scene_export_materials(const rb_scene_desc *s, rb_material_desc *out);

/* Camera frame. Replaces CameraBase::initialize (camera_base.hpp:76-99),
 * FP64. out: center, pixel00, delta_u, delta_v, u, v, w (7 x 3 doubles). */
void rb_camera_frame(const double look_from[3], const double look_at[3], const double vup[3],
                     double vfov_deg, int width, int height, double out[21]);

/* ======================================================================== */
/* 3. Device scene                                                           */
/* ======================================================================== */

typedef struct rb_upload_opts {
  int quantized_bvh;   /* 1: 8-bit child bounds relative to the parent */
  int use_bvh;         /* 0: linear scan (reference use_bvh == false)   */
  int layout;          /* RB_LAYOUT_*: how the render kernels see the scene */
  int max_leaf;        /* RB_LAYOUT_LEAF: BVH leaf size to rebuild with */
  int tune_depth;      /* path depth of the autotuner's probe (0 = 8) */
  int probe_width, probe_height;  /* frame size probe_frame was made for */
  const double *probe_frame;      /* autotune on this camera (rb_camera_frame), or NULL */
  int traversal_budget;           /* testing: traversal step budget per ray (0: 2 * (primitives + 4) + 64,
                                     which no well-formed tree reaches) */
  int wide_bvh;                   /* 0 (default) or 1: the render kernels traverse a 4-wide copy of
                                     the BVH (the same FP32 child boxes and leaves, four per 128-byte
                                     node); primary hits and exact-order traversal keep the binary
                                     tree. -1: binary tree only. Not with quantized_bvh. */
} rb_upload_opts;

/* RB_LAYOUT_AS_BUILT: the scene's BVH as built (the reference's leaf-4 tree
 * from rb_scene_build_bvh: primary-hit ids bit-exact against the reference).
 * RB_LAYOUT_AUTOTUNE: time a probe render (256 x 256 samples of probe_frame's
 * view, 8 spp; without a frame, views from inside and outside the scene's box)
 * on each candidate layout (linear scan and groups of 8 / 16 for small
 * scenes, BVH leaf sizes 1/2/4/8) and keep the fastest; decisions are cached
 * per scene.
 * RB_LAYOUT_LINEAR: no BVH. RB_LAYOUT_LEAF: rebuild the BVH with max_leaf.
 * RB_LAYOUT_GROUPS: no traversal stack: the built BVH's largest subtrees of at
 * most max_leaf primitives become groups, tested in leaf order (the group's
 * box, then its primitives); the primitives are tested in the linear scan's
 * order. */
enum { RB_LAYOUT_AS_BUILT = 0, RB_LAYOUT_AUTOTUNE = 1, RB_LAYOUT_LINEAR = 2, RB_LAYOUT_LEAF = 3,
       RB_LAYOUT_GROUPS = 4 };

/* Layout the upload chose: kind (RB_LAYOUT_LINEAR, RB_LAYOUT_LEAF or
 * RB_LAYOUT_GROUPS), leaf or group size (0 for linear) and, when autotuned,
 * the probe time of the winner. */
int rb_scene_layout_info(const rb_cuda_scene *scene, int *kind, int *leaf, float *probe_ms);

/* Everything the autotuner (RB_LAYOUT_AUTOTUNE) chose for a scene. Decisions
 * are cached per (GPU, scene fingerprint): a second upload of the same scene
 * on the same GPU reuses them without probing (from_cache = 1). Zeros mean
 * the class defaults (an upload that was not autotuned). */
typedef struct rb_tuning {
  int layout;           /* RB_LAYOUT_LINEAR, RB_LAYOUT_LEAF or RB_LAYOUT_GROUPS */
  int leaf;             /* BVH leaf size or group size (0 for linear) */
  int blocks_per_sm;    /* per-frame kernel: resident 256-thread blocks per SM (register budget) */
  int block_x, block_y; /* per-frame kernel: block shape */
  int short_stack;      /* traversal stack entries kept in shared memory */
  int wavefront_queue;  /* wavefront engine path slots (smooth-SDF scenes; 0: not tuned) */
  float probe_ms;       /* probe time of the chosen configuration */
  int from_cache;       /* 1: the decision came from the per-(GPU, scene) cache */
  int reserved_[3];
} rb_tuning;
int rb_scene_tuning(const rb_cuda_scene *scene, rb_tuning *out);

/* Upload to the current device. Returns an opaque device-scene handle that is
 * also accepted wherever the drop-in group takes a CudaScene::Scene*. */
rb_cuda_scene *rb_scene_upload(const rb_scene_desc *s, const rb_upload_opts *opts, void *stream);
void rb_scene_free_device(rb_cuda_scene *scene);
/* Device bytes held by a device scene. */
int64_t rb_scene_device_bytes(const rb_cuda_scene *scene);
/* Rays of this scene whose BVH traversal ran out of its step budget since the
 * upload (or the last reset): the loop then stops and the ray keeps the
 * closest hit found so far. A well-formed tree never reaches the budget, so a
 * nonzero count reports a corrupt tree (or a test's budget override,
 * rb_upload_opts.traversal_budget). Waits for the device. reset != 0 zeroes
 * the counter after reading it. */
int rb_scene_traversal_faults(const rb_cuda_scene *scene, uint64_t *count, int reset);

/* Host-only check of the 4-wide copy of a built scene's BVH (no device
 * needed): builds the upload layout on the host and verifies that every
 * binary-tree leaf is reached exactly once, every wide node once, child refs
 * stay in range and each child node's boxes lie inside its slot's box. out:
 * [wide nodes, leaves reached, binary-tree leaves, depth]. RB_OK when
 * consistent. */
int rb_scene_check_wide(const rb_scene_desc *s, int64_t out[4]);

/* Primary hits: pixel-centre rays (no jitter, no DOF), closest hit over the
 * device BVH; ids[w*h] = leaf-order geometry index or -1; t may be NULL.
 * ids / t are DEVICE pointers. */
int rb_primary_hits(const rb_cuda_scene *scene, int width, int height, const double frame[21],
                    int32_t *ids, float *t, void *stream);

/* Global options of the drop-in group beyond the reference's setters. */
typedef struct rb_render_opts {
  int nee;            /* 1: next-event estimation with MIS on area lights   */
  int kahan;          /* 1: Kahan-compensated FP32 accumulation (default 1) */
  uint32_t seed;      /* RNG seed of the per-path counter-based streams     */
  int block_x, block_y; /* launch shape of the per-pixel kernel (0 = tuned per class) */
  int reserved[4];      /* [0]: resident 256-thread blocks per SM the kernel is
                           compiled for (1-4; 0 = tuned per material class);
                           [1]: sample slices per pixel of the per-pixel kernel
                           (0 = automatic: frames with fewer pixels than four
                           times the GPU's resident threads split their samples,
                           up to 8 slices);
                           [2]: schedule of the per-pixel kernel: 1 grid (one
                           thread per pixel of a 2-D grid), 2 fetch (a persistent
                           grid whose warps take 8x4-pixel tiles of a sample
                           slice from a counter; the same sums bit for bit);
                           0 = the scene's tuned schedule, fetch by default) */
} rb_render_opts;
void rb_get_render_opts(rb_render_opts *out);
void rb_set_render_opts(const rb_render_opts *in);

/* Device-resident accumulation into caller-owned DEVICE buffers (no lazy
 * allocation, no host copies): accum = w*h float4 sums, comp = w*h float4
 * Kahan compensation or NULL. sample_base = index of the first sample (the
 * counter-based RNG key). counters (device, may be NULL) receives
 * [segments, paths] as two uint64 added atomically. */
int rb_render_accumulate(const rb_cuda_scene *scene, int width, int height, const double frame[21],
                         int samples_to_add, int sample_base, int max_depth, float *accum,
                         float *comp, uint64_t *counters, void *stream);

/* Several views of one scene in ONE persistent launch (the batched kernel):
 * n_views camera frames (frames: HOST, n_views x 21 doubles as rb_camera_frame
 * writes them), all width x height, each adding samples [sample_base,
 * sample_base + samples) per pixel. accum (DEVICE): n_views blocks of
 * 2*width*height float4, each the view's FP32 sums followed by its Kahan
 * compensation terms (true sum = sum - compensation). View v draws the sample
 * streams of salt v, so view 0 repeats rb_render_accumulate's streams.
 * counters (DEVICE, may be NULL) are overwritten with [segments, paths, stack
 * overflows]. Extends RendererCUDAProgressive's one-view-per-launch loop
 * (renderer_cuda_progressive_host.hpp:677-685, 904) to many views per launch. */
int rb_render_views(const rb_cuda_scene *scene, int n_views, int width, int height, const double *frames,
                    int samples, int sample_base, int max_depth, float *accum, uint64_t *counters,
                    void *stream);

/* Wavefront engine (an alternative to the per-pixel kernel of
 * rb_render_accumulate): SoA ray/hit queues of queue_capacity paths (0 = 2^20),
 * extend and shade kernels per bounce, warp-ballot compaction of surviving
 * paths with in-place regeneration of ended ones, iterations replayed from a
 * CUDA graph. Adds samples [sample_base, sample_base + samples) of every pixel
 * to accum (DEVICE, w*h*4 doubles: FP64 sums x y z, pad) with FP64 atomics.
 * counters (DEVICE, may be NULL): [segments, paths, stack overflows,
 * iterations]. Same sample streams as rb_render_accumulate. */
int rb_render_wavefront(const rb_cuda_scene *scene, int width, int height, const double frame[21],
                        int samples, int sample_base, int max_depth, double *accum,
                        int queue_capacity, uint64_t *counters, void *stream);

/* Number of kernel launches this library has made (all entry points). */
/* rb_render_views on the wavefront engine: the rays of all n_views views run
 * in one persistent wavefront (shared SoA queues, one job table, paths
 * regenerated across views), with FP64 accumulation. accum (DEVICE): n_views
 * blocks of width*height*4 doubles (xyz sums, pad), added to. Same sample
 * streams as rb_render_views (view v on salt v). counters (DEVICE, may be
 * NULL): [segments, paths, stack overflows, iterations]. */
int rb_render_views_wavefront(const rb_cuda_scene *scene, int n_views, int width, int height,
                              const double *frames, int samples, int sample_base, int max_depth,
                              double *accum, int queue_capacity, uint64_t *counters, void *stream);

/* Number of this library's kernel launches so far (all entry points). */
unsigned long long rb_launch_count(void);

/* Per-kernel timing for measurement (no counterpart in the reference). While
 * enabled, each launch of the per-frame render kernel (k_render) is bracketed
 * by two CUDA events recorded on the stream it is launched on.
 * rb_kernel_timer_read waits for the recorded events, returns the summed
 * elapsed milliseconds and the number of launches since the last read, and
 * releases the events. Off by default; not for use while a stream that
 * launches k_render is being captured into a graph. */
void rb_kernel_timer_enable(int on);
int rb_kernel_timer_read(double *ms, int64_t *launches);

/* Host-side fault injection for tests (no counterpart in the reference): the
 * next `count` device allocations at `site` fail as if the device were out of
 * memory, without any call into CUDA. Sites: "server_job" (a job's buffers at
 * admission: the job is rejected with RB_ERR_OUT_OF_MEMORY, the server keeps
 * serving the others) and "wavefront_queue" (the wavefront engine's queues:
 * the run returns RB_ERR_OUT_OF_MEMORY and the next run allocates afresh).
 * count 0 clears pending failures. */
int rb_inject_alloc_failures(const char *site, int count);

/* ======================================================================== */
/* 4. Batched multi-job engine and serving loop (additions; the reference    */
/*    renders one job per call, renderer_cuda_progressive_host.hpp:884-922)  */
/* ======================================================================== */

/* One render job. The scene is an index returned by rb_server_add_scene. */
typedef struct rb_job_request {
  int scene;
  int width, height;
  int spp;               /* total samples per pixel */
  int max_depth;
  double frame[21];      /* rb_camera_frame output */
  float light_intensity, background_intensity, metal_fuzziness, glass_ior;
  int dof_enabled;
  float dof_aperture, dof_focus;
  int nee;
  uint32_t seed;         /* job key of the counter-based sample streams */
  int fp64_accum;        /* 1: FP64 accumulation (always used above 65536 spp) */
  double arrival_time;   /* seconds on the server clock (rb_server_run_trace) */
  /* Per-job convergence (0 = off): after each iteration that gave the job
   * samples, a pixel counts as converged when, with at least
   * converge_min_spp samples, its mean luminance changed by less than
   * converge_threshold relative to the new mean (the per-pixel test of
   * render_acc_kernel.cu:241-271) and stays converged; the job completes
   * early when at least converge_fraction of its pixels are converged. */
  float converge_threshold;
  int converge_min_spp;
  float converge_fraction;
  int converge_pad;
} rb_job_request;

/* Defaults for rb_job_request: the reference's __constant__ shading values. */
void rb_job_default(rb_job_request *out);

typedef struct rb_server_opts {
  int64_t memory_budget_bytes;  /* HBM admission budget: accumulation + frame buffers */
  int max_active_jobs;          /* slots of the batched launch (<= 1024) */
  int64_t paths_per_iteration;  /* work quantum of one batched launch */
  int max_spp_per_iteration;    /* per-job cap of samples per pixel per launch of the batched
                                   kernel (jobs on the per-frame kernel take what the path
                                   quantum allows) */
  int use_graph;                /* 1: each iteration is a CUDA graph launch */
  int frames_every;             /* > 0: write each active job's u8 frame every N iterations */
  int occupancy;                /* resident 256-thread blocks per SM (0 = tuned) */
  int wavefront_field;          /* 1 (default): jobs of scenes with a smooth SDF field run on the
                                   wavefront engine (FP64 accumulation); 0: batched kernel */
  float target_iteration_ms;    /* > 0: latency-target controller. After each iteration the path
                                   quantum is scaled by clamp(target / measured, 0.5, 2) within
                                   [2^18, paths_per_iteration], the rule of the progressive
                                   renderer's batch controller (renderer_cuda_progressive_host.hpp:
                                   677-685) applied to the server's quantum. 0: fixed quantum */
  int per_frame_classes;        /* bit c set: planned jobs of material class c (1 diffuse, 2 classic,
                                   3 full, 4 SDF without a smooth field) with FP32 accumulation run
                                   on the per-frame kernel, one launch per job and iteration over the
                                   job's planned sample range, instead of the batched kernel */
} rb_server_opts;

void rb_server_default_opts(rb_server_opts *out);

typedef struct rb_job_status {
  int state;             /* 0 queued, 1 active, 2 done, -1 rejected */
  int spp_done;
  double t_arrival, t_admit, t_done;  /* server clock, seconds */
  int64_t device_bytes;
  int error;             /* why a rejected job was rejected: RB_ERR_CAPACITY (can never fit the
                            budget or slots) or RB_ERR_OUT_OF_MEMORY (its buffers could not be
                            allocated); RB_OK otherwise */
  int reserved_;
} rb_job_status;

typedef struct rb_server_stats {
  int64_t jobs_done, jobs_rejected, iterations, frames;
  int64_t paths, segments;
  double device_seconds;   /* sum of iteration device times (CUDA events) */
  double wall_seconds;     /* first arrival to last completion */
  int64_t peak_device_bytes;
  double p50_latency, p99_latency, mean_latency;  /* arrival -> done, seconds */
  int64_t quantum_paths;      /* path quantum of the next iteration */
  double last_iteration_ms;   /* device time of the last iteration */
} rb_server_stats;

typedef struct rb_server rb_server;

rb_server *rb_server_create(const rb_server_opts *opts, void *stream);
void rb_server_destroy(rb_server *s);
/* Keeps a device scene resident for the server's jobs; returns its index. */
int rb_server_add_scene(rb_server *s, const rb_cuda_scene *scene);
/* Queues a job (FIFO); returns its id (>= 0) or an rb_status. */
int64_t rb_server_submit(rb_server *s, const rb_job_request *req);
/* Admits queued jobs while slots and budget allow, runs one batched
 * iteration over all active jobs, retires finished ones. Returns the number
 * of jobs still active or queued (0 = idle), or an rb_status. */
int rb_server_step(rb_server *s);
int rb_server_job_status(rb_server *s, int64_t job, rb_job_status *out);
/* Copies a job's radiance sums (w*h*3 FP32, true sum = sum - compensation
 * or the FP64 sum rounded) and/or its latest u8 RGBA frame to host memory. */
int rb_server_fetch(rb_server *s, int64_t job, float *rgb_sum, uint8_t *rgba_frame);
/* Returns a finished job's device memory to the budget. */
int rb_server_release(rb_server *s, int64_t job);
/* Runs a whole request stream: requests are submitted when the server clock
 * passes their arrival_time (realtime = 1) or all at once (0); finished jobs
 * are released unless keep_results. latencies[n] (may be NULL) receives
 * arrival -> done seconds. */
int rb_server_run_trace(rb_server *s, const rb_job_request *reqs, int64_t n, int realtime, int keep_results,
                        double *latencies);
int rb_server_get_stats(rb_server *s, rb_server_stats *out);

#ifdef __cplusplus
}
#endif
#undef RB_DEFAULT
#endif /* RAYON_B200_H */
