/*
 * raygen_b200.h - C ABI of the B200 wavefront path tracer.
 *
 * This is the drop-in boundary for RayGen's shader-5 (BSDF) render path.
 * Every entry point takes plain pointers and sizes, returns an rg_status
 * (0 = OK, negative = error), never throws across the boundary, and is
 * thread-safe per handle (one render in flight per handle).
 *
 * Reference interfaces replaced (paths relative to the RayGen project):
 *   rg_settings            <- RendererSettings            src/raygen/rayrenderer.h:98-153
 *   rg_create              <- RayRenderer::RayRenderer    src/raygen/rayrenderer.cpp:53-86
 *   rg_set_scene           <- Renderer::setScene          src/raygen/renderer.h:48-50
 *                             + RayRenderer::transformScene src/raygen/rayrenderer.cpp:157-363
 *                             + TriangleBVH::build        src/raygen/bvh.cpp:76-98
 *   rg_render              <- RayRenderer::render         src/raygen/rayrenderer.cpp:478-596
 *   rg_set_progress_cb     <- RayRenderer::progressCallback src/raygen/rayrenderer.h:317
 *   rg_cancel              <- RayRenderer::cancelRequested  src/raygen/rayrenderer.h:427
 *   rg_render_async, rg_poll, rg_wait, rg_job_free
 *                          <- the threaded RayRenderer::render + progressCallback
 *                             src/raygen/rayrenderer.cpp:748-809
 *   rg_get_hdr             <- RayRenderer::getHdrResult   src/raygen/rayrenderer.h:411
 *   rg_get_ldr             <- RayRenderer::getRenderResult src/raygen/rayrenderer.h:404
 *   rg_reapply_postprocess <- RayRenderer::reapplyPostProcess src/raygen/rayrenderer.cpp:698-711
 *   rg_save_image          <- saveImage in the CLI's output step src/main.cpp:479-485
 *   rg_load_image          <- Texture::loadFromFile         src/raygen/texture.cpp:170-195
 *   rg_trace_closest       <- TriangleBVH::intersectClosest src/raygen/bvh.cpp:233-285
 *   rg_trace_any           <- TriangleBVH::intersectAny   src/raygen/bvh.h:63-101
 *   rg_denoise_atrous      <- RayRenderer::denoiseImage   src/raygen/rayrenderer.cpp:2649-2772
 *   rg_tonemap             <- RayRenderer::applyTonemapGamma src/raygen/rayrenderer.cpp:2610-2647
 *   rg_bloom               <- RayRenderer::applyPostProcess src/raygen/rayrenderer.cpp:598-696
 *   rg_scene_builtin       <- (procedural stand-ins for the sample scenes; no reference symbol)
 *   rg_load_scene_json     <- RendererSceneLoader::load   src/raygen/sceneloader.cpp:1113-1137
 *   rg_server_*            <- the viewer's render-job worker (src/viewer/main.cpp:775-850),
 *                             generalised to many resident jobs (batching / serving)
 */
#ifndef RAYGEN_B200_H
#define RAYGEN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int rg_status;
#define RG_OK 0
#define RG_ERR_INVALID_ARGUMENT (-1)
#define RG_ERR_NO_SCENE (-2)
#define RG_ERR_UNSUPPORTED (-3)      /* shader id 4 (reserved in the reference) */
#define RG_ERR_CUDA (-4)
#define RG_ERR_OUT_OF_MEMORY (-5)
#define RG_ERR_CANCELLED (-6)
#define RG_ERR_DEVICE_STATUS (-7)    /* a kernel raised its error flag */
#define RG_ERR_IO (-8)
#define RG_ERR_PARSE (-9)
#define RG_ERR_BUSY (-10)
#define RG_ERR_NO_DEVICE (-11)

/* Mix-shader evaluation: the reference sums every lobe (tree); the GPU picks
 * one lobe per vertex with probability proportional to its weight (select). */
#define RG_MIX_SELECT 0

/* Adaptive sampling granularity. */
#define RG_ADAPTIVE_PIXEL 0   /* per-pixel relative SEM (16 -> 256 spp)      */
#define RG_ADAPTIVE_TILE 1    /* reference: per 32x32 tile mean relative SEM */

/* Mirrors RendererSettings (rayrenderer.h:98-153) plus the tracer's own knobs. */
typedef struct rg_settings {
  int32_t resolution_width, resolution_height;
  int32_t threads;            /* host threads (loader / CPU helpers)          */
  int32_t samples;            /* samples per pixel (adaptive: maximum)        */
  int32_t shader_provider;    /* 0,1,2,3,5 ; 4 -> RG_ERR_UNSUPPORTED          */
  int32_t enable_antialias;
  int32_t enable_point_light_antialias;
  int32_t enable_color_sampling;
  int32_t enable_rendering_postprocess; /* bloom                              */
  int32_t enable_denoise;     /* A-Trous                                      */
  int32_t cull_back_face;
  int32_t denoise_levels;
  float denoise_sigma_color, denoise_sigma_normal, denoise_sigma_depth;
  float denoise_intensity;
  float firefly_clamp;
  int32_t enable_adaptive_sampling;
  int32_t adaptive_base_samples;
  float adaptive_threshold;
  int32_t adaptive_mode;      /* RG_ADAPTIVE_PIXEL / RG_ADAPTIVE_TILE         */
  float bloom_threshold, bloom_strength, bloom_radius, bloom_size_aspect, bloom_curve;
  float world_color[3];
  float back_color[4];
  /* tracer knobs (no reference counterpart; reference values in brackets) */
  uint32_t seed;              /* counter-based RNG seed [1]                   */
  int32_t max_depth;          /* MAX_TRACE_DEPTH [32]                         */
  int32_t rr_depth;           /* MIN_RR_DEPTH [3]                             */
  int32_t light_pick_fix;     /* 1: weight NEE by the light count [0]         */
  int32_t paths_per_wave;     /* wavefront size; 0 = automatic: up to 64 Mi
                               * paths (about 330 B of queues each), at most a
                               * fifth of the free device memory             */
  int32_t bvh_bins;           /* SAH bins for the device build [32]           */
  int32_t bvh_width;          /* 8: 8-wide BVH (default), 2: binary */
} rg_settings;

typedef struct rg_material {
  float color[3];
  float diffuse, glossy, roughness, transparency, refraction, refraction_ratio;
  float chroma_dispersion, metallic, anisotropy, aniso_rotation, emission, spot_range;
  int32_t texture;            /* index into rg_scene_desc.textures, -1 none   */
  float tex_tiling[2];
} rg_material;

/* One control point of a path-mode emission tube (HomogeneousMedium::PathSample,
 * medium.h:55-59). */
typedef struct rg_medium_path_point {
  float p[3];                 /* world space                                  */
  float radius;               /* tube radius here (lerped along a segment)    */
  float t;                    /* axial parameter: inner -> outer colour blend */
} rg_medium_path_point;

enum { RG_EMISSION_CONSTANT = 0, RG_EMISSION_CONE = 1, RG_EMISSION_PATH = 2 };
enum { RG_DENSITY_NONE = 0, RG_DENSITY_FBM = 1 };

/* Participating medium (HomogeneousMedium, medium.h:37-334; readMedium,
 * sceneloader.cpp:202-334).  A zero-initialised medium past `density` is the
 * homogeneous constant-emission medium; rg_medium_defaults() fills the
 * reference's defaults for the procedural fields (medium.h:80-199).
 *  - emission_mode CONE: sigma_e(p) is the afterburner profile around the
 *    axis cone_origin + s * cone_axis, s in [0, cone_length] (emissionAt,
 *    medium.cpp:303-404); PATH: a tube along path_points (medium.cpp:310-354).
 *    Both are integrated along each segment with cone/path_emission_samples
 *    stratified samples (emissionIntegralAlongRay, medium.cpp:443-473).
 *  - cone_origin / cone_axis and path_points are world space for the CONE and
 *    PATH modes respectively (the loader applies the owning object's transform
 *    when coneFollowObject / pathFollowObject is set).  In every other mode
 *    the renderer uses cone_origin / cone_axis as given, in camera space, as
 *    the reference's un-baked values are (only the heat-haze falloff reads
 *    them then; HomogeneousMedium::bake, medium.cpp:59-101).
 *  - density_field FBM: every sigma is scaled by a fractal value-noise field
 *    evaluated in camera space, max(0, noise_amplitude * fbm + noise_bias),
 *    and free flights use delta tracking (medium.cpp:276-301, 406-441).
 *  - heat_haze: rays crossing the medium are bent by the gradient of
 *    n(p) = 1 + ior_amplitude * (2 fbm - 1) over ior_march_steps steps and
 *    the sigma terms are ignored (bendRay, medium.cpp:191-274).
 * Octave, sample and march-step counts above 64 are clamped to 64. */
typedef struct rg_medium {
  float sigma_a[3], sigma_s[3], sigma_e[3];
  float g, density;
  int32_t emission_mode;      /* RG_EMISSION_*                                */
  float cone_origin[3], cone_axis[3];
  float cone_length, cone_radius;
  float cone_inner[3], cone_outer[3];
  float cone_intensity, cone_peak_axial, cone_peak_sharpness;
  int32_t cone_emission_samples;
  int32_t num_path_points;
  const rg_medium_path_point* path_points;
  float path_inner[3], path_outer[3];
  float path_intensity, path_falloff_power;
  int32_t path_emission_samples;
  int32_t density_field;      /* RG_DENSITY_*                                 */
  float noise_frequency;
  int32_t noise_octaves;
  float noise_gain, noise_lacunarity, noise_amplitude, noise_bias;
  float noise_offset[3];
  int32_t heat_haze;          /* 0 off                                        */
  float ior_amplitude, ior_frequency;
  int32_t ior_octaves;
  float ior_gain, ior_lacunarity;
  int32_t ior_march_steps;
  float ior_offset[3];
  float ior_falloff;
} rg_medium;

typedef struct rg_object {
  int32_t material;
  int32_t interior_medium;    /* -1 none */
  /* SceneObject::location (local to the parent).  An object whose interior
   * medium emits with constant sigma_e is a volume light anchored at this
   * point taken as camera-relative world coordinates (sampleVolumeLightForNEE,
   * rayrenderer.cpp:2091-2100).  An object may have no meshes: such an object
   * only contributes its medium as a volume light. */
  float location[3];
} rg_object;

/* A mesh-less emissive object of the reference (a point or spot light). */
typedef struct rg_point_light {
  float position[3];          /* world space */
  float normal[3];            /* world space */
  int32_t material;
} rg_point_light;

typedef struct rg_camera {
  float location[3];
  float angle[3];             /* degrees; R = Ry(y) Rx(x) Rz(z)             */
  float field_of_view;        /* vertical, degrees                           */
  float view_near, view_far;
  float depth_of_field, aperture;
  int32_t aperture_blades;
  float aperture_rotation;    /* degrees */
  float exposure;
} rg_camera;

typedef struct rg_texture {
  int32_t width, height;
  int32_t is_hdr;             /* 0: sRGB-decoded on sample                   */
  const float* rgba;          /* width*height*4                              */
} rg_texture;

/* Flattened scene: world-space triangle soup grouped into meshes and objects.
 * Triangle order is the reference's DFS order (objects -> meshes -> triangles)
 * and is the triangle id used by rg_trace_closest. */
typedef struct rg_scene_desc {
  int32_t num_triangles;
  const float* positions;     /* [num_triangles][3][3]                       */
  const float* normals;       /* [num_triangles][3][3]                       */
  const float* uvs;           /* [num_triangles][3][2] or NULL               */
  const int32_t* tri_mesh;    /* [num_triangles]                             */
  int32_t num_meshes;
  const int32_t* mesh_object; /* [num_meshes]                                */
  int32_t num_objects;
  const rg_object* objects;
  int32_t num_materials;
  const rg_material* materials;
  int32_t num_media;
  const rg_medium* media;
  int32_t global_medium;      /* -1 none */
  int32_t num_point_lights;
  const rg_point_light* point_lights;
  int32_t num_textures;
  const rg_texture* textures;
  rg_camera camera;
  /* Environment map (Scene::envmap / envmapIntensity / envmapRotation,
   * scene.h:187-190; sampleEnvironment, rayrenderer.cpp:1299-1348): an
   * equirectangular texture looked up by the VIEW-space ray direction (as in
   * the reference), rotated by envmap_rotation degrees about +Y, times
   * envmap_intensity; importance-sampled by luminance x sin(theta)
   * (Scene::buildEnvmapCDF, scene.cpp:330-463).  A zero-initialised
   * description has no environment map. */
  int32_t has_envmap;         /* 0 none */
  int32_t envmap_texture;     /* index into textures                          */
  float envmap_intensity;
  float envmap_rotation;      /* degrees */
  /* Cubemap environment (Scene::envCubemapFaces, scene.h:198-222): six square
   * faces of one size, texture indices in the order +X -X +Y -Y +Z -Z (px nx
   * py ny pz nz).  When envmap_cube is set it takes precedence over the
   * equirectangular map for lookups, and is importance-sampled per face by
   * luminance x texel solid angle (scene.cpp:343-410); intensity and rotation
   * are shared. */
  int32_t envmap_cube;        /* 0 none */
  int32_t envmap_cube_faces[6];
} rg_scene_desc;

typedef struct rg_stats {
  double trace_ms;            /* device time of the last render's trace     */
  double post_ms;             /* device time of denoise / tonemap            */
  double build_ms;            /* device time of the last BVH build           */
  uint64_t samples;           /* primary samples traced                      */
  uint64_t closest_rays, shadow_rays;
  uint64_t nodes_visited, tris_tested;          /* closest-hit kernels        */
  uint64_t shadow_nodes_visited, shadow_tris_tested;
  double extend_ms, shade_ms, connect_ms;       /* per-kernel device time     */
  int32_t bvh_nodes;
  int32_t waves;
  int32_t kernel_launches;
  int32_t device_error;       /* first device error code, 0 = none           */
  /* host wall time of the last rg_render: entry -> first wave launched, and
   * entry -> return (set-up, waves, post, stats read-back) */
  double host_setup_ms, host_total_ms;
} rg_stats;

typedef struct rg_handle rg_handle;
typedef void (*rg_progress_fn)(float progress, void* user);

void rg_settings_default(rg_settings* s);
/* Zero-fill `m` and set the reference's defaults of every medium field
 * (density 1, cone / path / noise / heat-haze defaults of medium.h:80-199). */
void rg_medium_defaults(rg_medium* m);
rg_status rg_create(const rg_settings* s, rg_handle** out);
rg_status rg_destroy(rg_handle* h);
rg_status rg_update_settings(rg_handle* h, const rg_settings* s);
/* Copies the scene to the device and builds its BVH.  The handle rebuilds in
 * place: the previous scene's device buffers and the build's working arrays are
 * reused (they only grow), so a scene no larger than the last one allocates no
 * device memory.  A scene with less than half the previous one's triangles
 * starts from fresh buffers. */
rg_status rg_set_scene(rg_handle* h, const rg_scene_desc* scene);
/* Blocking render (RayRenderer::render, rayrenderer.cpp:478-596).  Waves are
 * paced one behind the device, so progress is reported for completed waves and
 * rg_cancel ends the render within about one wave (RG_ERR_CANCELLED; the
 * handle stays usable).  RG_ERR_BUSY while an rg_render_async job of the same
 * handle is in flight. */
rg_status rg_render(rg_handle* h);
/* Asynchronous render: the reference's render() runs its tiles on worker
 * threads and reports through progressCallback (rayrenderer.cpp:748-809,
 * :804-806); here one host thread per job runs the render of `h` and the
 * caller polls or waits.  One in-flight render per handle: while a job runs,
 * rg_render_async, rg_render, rg_set_scene and rg_update_settings on the
 * handle return RG_ERR_BUSY.  rg_poll: done (0/1) and progress in [0, 1]; rg_wait: the render's
 * status, or RG_ERR_BUSY when timeout_ms (< 0: no limit) passes first;
 * rg_job_free waits for the render to end, then frees the job.  rg_destroy on
 * the handle waits for the job's render; a job that is done stays pollable
 * after its handle is destroyed. */
typedef struct rg_job rg_job;
rg_status rg_render_async(rg_handle* h, rg_job** job);
rg_status rg_poll(rg_job* job, int32_t* done, float* progress);
rg_status rg_wait(rg_job* job, double timeout_ms);
rg_status rg_job_free(rg_job* job);
/* Progress callback (RayRenderer::progressCallback, rayrenderer.h:317): called
 * from the rendering host thread (the caller's, or the async job's), never
 * from the device, with non-decreasing values; 1.0 when a render completes. */
rg_status rg_set_progress_cb(rg_handle* h, rg_progress_fn fn, void* user);
/* Request cancellation of the handle's render in flight (cancelRequested,
 * rayrenderer.h:427, polled per tile at rayrenderer.cpp:766). */
rg_status rg_cancel(rg_handle* h);
/* Linear HDR result (width*height*4 floats, alpha = 1). */
rg_status rg_get_hdr(rg_handle* h, float* rgba, size_t count);
/* Re-run the post-processing (HDR bloom when enable_rendering_postprocess,
 * then the tonemap) from the last render's denoised, not yet bloomed HDR,
 * with the current settings (set them with rg_update_settings first). */
rg_status rg_reapply_postprocess(rg_handle* h);
/* Tonemapped result in [0,1] (width*height*4 floats). */
rg_status rg_get_ldr(rg_handle* h, float* rgba, size_t count);
/* Guide buffers of the last render (normal*0.5+0.5, albedo, depth), 3 floats
 * per pixel each, as the denoiser saw them; NULL pointers are skipped. */
rg_status rg_get_aovs(rg_handle* h, float* normal, float* albedo, float* depth, size_t count);
/* Per-pixel sample counts of the last render (int32 per pixel). */
rg_status rg_get_sample_counts(rg_handle* h, int32_t* counts, size_t count);
rg_status rg_get_stats(rg_handle* h, rg_stats* out);
const char* rg_last_error(void);
const char* rg_version(void);

/* Ray-batch queries against the scene's view-space BVH.
 * rays: n x 6 floats (origin xyz, dir xyz) in view space.
 * closest: out_tuv n x 3 (t, u, v), out_prim n (DFS triangle id, -1 = miss).
 * any: tmax n floats; predicate 0 = area-light occluder, 1 = point/env
 *      occluder, 2 = AO occluder, 3 = every triangle, 4 = volume-light
 *      occluder (rayrenderer.cpp:2167-2171); out_hit n bytes. */
rg_status rg_trace_closest(rg_handle* h, const float* rays, int32_t n, float* out_tuv, int32_t* out_prim);
rg_status rg_trace_any(rg_handle* h, const float* rays, const float* tmax, int32_t n, int32_t predicate, uint8_t* out_hit);
/* Medium field queries on the scene's camera-space media (device work).
 * eval: points n x 3 -> out n x 5 (densityAt, emissionAt rgb, iorAt;
 *       medium.cpp:186-215, 276-404).
 * bend: rays n x 7 (origin xyz, dir xyz, march length) -> out n x 6 (the
 *       bent ray's origin and direction; bendRay, medium.cpp:237-274). */
rg_status rg_medium_eval(rg_handle* h, int32_t medium, const float* points, int32_t n, float* out);
rg_status rg_medium_bend(rg_handle* h, int32_t medium, const float* rays, int32_t n, float* out);
/* Failure-detection test hooks (no reference counterpart).  Both change a
 * process-wide bound of this library on the current device; pass 0 to restore
 * the built-in bound, and make no other render of the process overlap the call.
 *   rg_debug_set_traversal_step_cap: node steps a traversal may take per ray
 *     before it stops, raises its error flag and the render returns
 *     RG_ERR_DEVICE_STATUS (built-in: 4,194,304);
 *   rg_debug_set_tc_wait_limit: polls the learned denoiser's strip pipeline
 *     makes on a barrier before it gives up, raises its error word (the call
 *     returns RG_ERR_DEVICE_STATUS) and drains its copies and MMAs under the
 *     built-in bound before freeing tensor memory (built-in: 67,108,864). */
rg_status rg_debug_set_traversal_step_cap(int32_t cap);
rg_status rg_debug_set_tc_wait_limit(uint32_t polls);
/* Sampling-helper probes (device work, host pointers), one row per input;
 * each row runs the device function the shade kernel uses:
 *   0 sampleGGXVNDF      <- bsdf.cpp:139-161  in (Ve xyz, ax, ay, u1, u2) -> H xyz
 *   1 smithG1            <- bsdf.cpp:164-170  in (w xyz, ax, ay)          -> G1
 *   2 fresnelSchlick     <- bsdf.cpp:32-37    in (cosTheta, ior)          -> F
 *   3 refract            <- bsdf.cpp:39-52    in (d xyz, n xyz, ior)      -> dir xyz
 *   4 buildTangentFrame  <- bsdf.cpp:129-135  in (n xyz)                  -> t xyz, b xyz
 *   5 cosineWeightedDirection <- raycommon.cpp:94-115, on LDS dims dim, dim+1
 *                              in (x, y, sample, dim, n xyz)           -> dir xyz
 *   6 ldsPointInTriangle <- raycommon.cpp:117-122, on LDS dims dim, dim+1
 *                              in (x, y, sample, dim, v1 v2 v3 xyz)    -> p xyz
 *   7 ldsNext1D          <- raycommon.cpp:71-87 in (x, y, sample, dim) -> u
 *   8 samplePhase (HG)   <- medium.cpp:496-517  in (wo xyz, g, u1, u2)   -> wi xyz
 *   9 phasePdf (HG)      <- medium.cpp:519-525  in (wo xyz, wi xyz, g)   -> pdf
 *  10 sampleFreeFlight   <- medium.cpp:475-480  in (sigma_t hero, u)     -> t
 * LDS rows use seed 1 (the reference's unsalted scramble). */
rg_status rg_probe_sampling(int32_t which, const float* in, int32_t n, float* out);
/* View-space camera transform the scene was flattened with (4x4 row-major,
 * row-vector convention: p_view = [p 1] * M). */
rg_status rg_get_view_matrix(rg_handle* h, float* m16);

/* Stand-alone post passes on caller buffers (device work, host pointers).
 * color/out: w*h*3 floats; normal/albedo: w*h*3 (encoded as the AOVs);
 * albedo_alpha: w*h floats (1 = geometry hit); depth: w*h floats.
 * levels in [1, 16] (the settings' denoise_levels obeys the same bound), and
 * w*h*3 at most INT_MAX; otherwise RG_ERR_INVALID_ARGUMENT. */
rg_status rg_denoise_atrous(int32_t w, int32_t h, const float* color, const float* normal,
                            const float* depth, const float* albedo, const float* albedo_alpha,
                            int32_t levels, float sigma_color, float sigma_normal,
                            float sigma_depth, float intensity, float* out);
/* The same A-Trous filter on DEVICE buffers, without allocating.  No
 * counterpart in the reference: it exists for callers that cannot let the
 * library allocate device memory (a preview loop that must not take the
 * device-wide synchronisation of cudaFree, an application whose device memory
 * all comes from its own pool).  The library makes no cudaMalloc/cudaFree or
 * other allocating call here; the filter's working buffers are one static
 * device array per device.
 *   color_rgba, out_rgba: w*h float4 (RGBA, alpha ignored / written as 1),
 *                         16-byte aligned device memory of the current device;
 *   normal, albedo: w*h*3 floats; depth, albedo_alpha: w*h floats (device).
 *   stream: a cudaStream_t, NULL for the default stream.  The work is
 *   enqueued on it and the call returns; out_rgba is ready when it completes.
 * Limit: w*h <= 1,048,576 pixels and levels in [1, 16], else
 * RG_ERR_INVALID_ARGUMENT.  Host or foreign-device pointers, and an out_rgba
 * that overlaps any input, give RG_ERR_INVALID_ARGUMENT.  Buffer sizes cannot
 * be checked: each must hold w*h elements of the layout above.
 * Calls whose device work overlaps (other streams, unsynchronised threads)
 * share the working buffers and race; serialise them.  The first call in a
 * CUDA context (once per device, and again after a device reset) resolves the
 * working array's address; make it before any stream capture begins.
 * Results equal rg_denoise_atrous on the same inputs bit for bit. */
rg_status rg_denoise_atrous_noalloc(int32_t w, int32_t h, const float* color_rgba, const float* normal,
                                    const float* depth, const float* albedo, const float* albedo_alpha,
                                    int32_t levels, float sigma_color, float sigma_normal,
                                    float sigma_depth, float intensity, float* out_rgba, void* stream);
/* Test hook of the no-allocation entry point's address cache, which is keyed
 * by CUDA context id: runs ids[0..n) through a fresh cache (no CUDA call) and
 * writes whether each lookup had to resolve (1) or hit (0), and the ordinal
 * of the address returned.  No reference counterpart. */
rg_status rg_noalloc_cache_probe(const uint64_t* ids, int32_t n, int32_t* out_resolved, int32_t* out_slot);
rg_status rg_tonemap(int32_t w, int32_t h, const float* hdr_rgba, float* ldr_rgba);
/* Energy-based HDR bloom on caller buffers (device work, host pointers):
 * out = hdr + strength * blur(excess luminance above threshold), w*h RGBA. */
rg_status rg_bloom(int32_t w, int32_t h, const float* hdr_rgba, float threshold, float strength, float radius,
                   float size_aspect, float curve, float* out_rgba);

/* Tensor-core (tcgen05) BF16 GEMM of the learned denoiser, exposed for tests:
 * D[M x N] = A[M x K] * B[N x K]^T with FP32 accumulation; A, B row-major
 * BF16 bit patterns (K contiguous), D row-major FP32, host pointers.
 * N in 16..128 and K in 16..256, both multiples of 16.  No reference
 * counterpart (the reference has no learned denoiser). */
rg_status rg_tc_gemm_bf16(int32_t M, int32_t N, int32_t K, const uint16_t* A, const uint16_t* B, float* D);

/* ---- learned denoiser (kernel-predicting CNN on the tensor cores) --------
 * No reference counterpart: the reference denoises with A-Trous only, which
 * stays the renderer's default and its fallback.  Six 3x3 convolutions (11
 * input features: log radiance, albedo, normal and depth guides and the noise
 * level log2(1 + spp) / 12; 32 channels) predict a 5x5 filter per pixel that
 * is applied to the noisy radiance.  `spp` below is the samples per pixel of
 * the noisy image (>= 0); the renderer and the job server pass their
 * per-pixel sample counts instead (adaptive sampling included).
 * Convolutions run forward and backward as BF16 tcgen05 GEMMs with FP32
 * accumulation; training (relMSE loss against a high-spp render, Adam) runs
 * on the device.  Images: noisy/ref w*h RGBA floats, normal and albedo w*h*3
 * floats as returned by rg_get_aovs (normal * 0.5 + 0.5), depth w*h floats. */
typedef struct rg_denoiser rg_denoiser;
int32_t rg_denoiser_num_params(void);
/* He-initialised weights from `seed`. */
rg_status rg_denoiser_create(uint32_t seed, rg_denoiser** out);
rg_status rg_denoiser_destroy(rg_denoiser* d);
rg_status rg_denoiser_get_params(rg_denoiser* d, float* out, size_t n);
rg_status rg_denoiser_set_params(rg_denoiser* d, const float* in, size_t n);
/* Training pairs (all of one size) kept on the device. */
rg_status rg_denoiser_add_example(rg_denoiser* d, int32_t w, int32_t h, const float* noisy_rgba, const float* normal,
                                  const float* albedo, const float* depth, float spp, const float* ref_rgba);
rg_status rg_denoiser_clear_examples(rg_denoiser* d);
/* `steps` Adam steps on random batches of `batch` examples; losses[steps] (may be NULL). */
rg_status rg_denoiser_train(rg_denoiser* d, int32_t steps, int32_t batch, float lr, float* losses);
/* Loss and gradient (rg_denoiser_num_params floats) on `count` images of w x h. */
rg_status rg_denoiser_gradients(rg_denoiser* d, int32_t count, int32_t w, int32_t h, const float* noisy_rgba,
                                const float* normal, const float* albedo, const float* depth, float spp,
                                const float* ref_rgba, float* loss, float* grad);
rg_status rg_denoiser_apply(rg_denoiser* d, int32_t w, int32_t h, const float* noisy_rgba, const float* normal,
                            const float* albedo, const float* depth, float spp, float* out_rgba);
/* Device time (CUDA events) of the last rg_denoiser_apply (features, six
 * convolutions, kernel application) and of the mean step of the last
 * rg_denoiser_train call (batch gather, forward, backward, Adam, repacking). */
rg_status rg_denoiser_timing(rg_denoiser* d, float* apply_ms, float* train_step_ms);
/* Use `d` instead of A-Trous when enable_denoise is set (NULL: back to A-Trous).
 * The handle keeps the pointer; destroy `d` only after detaching it. */
rg_status rg_set_denoiser(rg_handle* h, rg_denoiser* d);

/* Procedural scenes (host C++, no device work).
 * kind 1: cube room (10 walls, two boxes, one 2.5x2.5 ceiling light).
 * kind 2: displaced icosphere x4 in a 20x20 room with 16 ceiling lights;
 *         iparams[0] = triangles per sphere (default 1,003,520).
 * kind 3: kind 2 + a global homogeneous medium (sigma_t 0.05, albedo 0.8, g 0.3).
 * kind 4: one job of the heterogeneous batch: iparams[0] = triangles,
 *         iparams[1] = emitters.
 * The returned description is owned by the library: free with rg_scene_free. */
rg_status rg_scene_builtin(int32_t kind, uint32_t seed, const int32_t* iparams, int32_t n_iparams,
                           rg_scene_desc** out);
rg_status rg_scene_free(rg_scene_desc* scene);
/* Reference scene JSON (sceneloader.cpp schema) -> flattened description. */
rg_status rg_load_scene_json(const char* path, rg_scene_desc** out);
/* Write width*height RGBA floats (row 0 at the top) to an image file chosen by
 * extension: .hdr (Radiance RGBE, RLE scanlines) and .pfm keep linear values;
 * .jpg / .jpeg (baseline JPEG, quality 92, 4:4:4), .png and .ppm store
 * round(clamp(v, 0, 1) * 255).  Host work only. */
rg_status rg_save_image(const char* path, int32_t width, int32_t height, const float* rgba);
/* Read an image file as a texture is read: Radiance .hdr by name (linear,
 * is_hdr 1), otherwise JPEG (baseline / extended sequential) or PNG by
 * content, and .pfm by name.  LDR images give their stored values in [0, 1]
 * (is_hdr 0; the renderer sRGB-decodes them when it samples).  Call with
 * rgba NULL to get the size; then with count >= width*height*4 floats.
 * Row 0 at the top.  Host work only. */
rg_status rg_load_image(const char* path, int32_t* width, int32_t* height, int32_t* is_hdr, float* rgba,
                        size_t count);

/* ---- resident multi-job server (batched and served rendering) ----------- */
#define RG_JOB_QUEUED 0
#define RG_JOB_RESIDENT 1
#define RG_JOB_DONE 2
#define RG_JOB_FAILED 3
#define RG_JOB_ADMITTING 4  /* slot reserved; scene upload / BVH build in progress */

typedef struct rg_server rg_server;

typedef struct rg_server_config {
  uint64_t hbm_budget_bytes;  /* admission budget for resident jobs [120 GiB]  */
  int32_t max_resident_jobs;  /* job slots [256]                               */
  int32_t paths_per_wave;     /* wavefront size shared by all jobs [8 Mi]      */
  int32_t max_depth_cap;      /* largest max_depth a job may use [10]          */
  int32_t shade_blocks_per_sm;  /* shade / generate / accumulate width [0: 4]  */
  int32_t trace_blocks_per_sm;  /* traversal width [0: occupancy limit]        */
  int32_t wave_fill;          /* 0: each wave shared evenly by the resident jobs;
                                 1: each wave filled from as few jobs as possible,
                                 in rotating order (fewer scenes per wave, more
                                 cache reuse; a large job delays the others) [0] */
} rg_server_config;

/* One render request.  The scene description is borrowed: it must stay valid
 * until the job reaches RG_JOB_DONE or RG_JOB_FAILED. */
typedef struct rg_job_desc {
  const rg_scene_desc* scene;
  int32_t width, height, samples;
  int32_t max_depth, rr_depth;  /* <= 0: the server's base settings */
  uint32_t seed;                /* RNG key: results do not depend on the mix */
  int32_t denoise;              /* 1: A-Trous on the finished image; 2: the learned
                                   denoiser set with rg_server_set_denoiser (A-Trous
                                   when none is set) */
} rg_job_desc;

typedef struct rg_job_status {
  int32_t state;                /* RG_JOB_* */
  rg_status error;
  double submit_ms, start_ms, done_ms, latency_ms;
  int64_t samples_issued, samples_total;
} rg_job_status;

typedef struct rg_server_stats {
  int64_t jobs_done;
  double p50_ms, p99_ms, mean_ms, max_ms;  /* submit -> result latency */
  double images_per_s;                     /* done jobs / (last done - first submit) */
  uint64_t samples_done;
  double device_ms;                        /* device time of all waves */
  int64_t waves;
  int32_t resident_peak;
  int32_t pending;
  uint64_t bytes_peak;                     /* peak admitted footprint estimate */
} rg_server_stats;

void rg_server_config_default(rg_server_config* c);
rg_status rg_server_create(const rg_settings* base, const rg_server_config* cfg, rg_server** out);
/* Queue a job.  RG_ERR_OUT_OF_MEMORY when the job's admission estimate alone
 * exceeds the whole HBM budget (it could never be admitted).  The admission
 * estimate reserves budget before the upload; once the job is resident its
 * measured device footprint replaces the reservation (bytes_peak is measured). */
rg_status rg_server_submit(rg_server* s, const rg_job_desc* job, int64_t* job_id);
rg_status rg_server_poll(rg_server* s, int64_t job_id, rg_job_status* out);
/* RG_ERR_BUSY on timeout. */
rg_status rg_server_wait(rg_server* s, int64_t job_id, double timeout_ms);
/* Resident scenes: a scene uploaded and built once (BVH, triangles, textures,
 * light and medium tables stay on the device), then rendered by any number of
 * jobs without a second upload or build.  rg_server_add_scene copies the
 * description, builds on the caller's thread and counts the scene's measured
 * bytes against the HBM budget (RG_ERR_OUT_OF_MEMORY when it does not fit);
 * the camera is the description's.  rg_server_submit_scene queues a job on it
 * (job->scene is ignored and may be NULL).  rg_server_remove_scene forgets the
 * id; the memory is freed when the last job rendering it ends.  No reference
 * counterpart (the reference renders one scene per process). */
rg_status rg_server_add_scene(rg_server* s, const rg_scene_desc* scene, int64_t* scene_id);
rg_status rg_server_submit_scene(rg_server* s, int64_t scene_id, const rg_job_desc* job, int64_t* job_id);
rg_status rg_server_remove_scene(rg_server* s, int64_t scene_id);
/* Cancel a job (the viewer's cancel button sets cancelRequested on the running
 * render, src/viewer/MainPanel.cpp:44-47): a
 * queued job leaves the queue; an admitting or resident job is dropped between
 * waves and its slot and memory are freed.  The job then polls as
 * RG_JOB_FAILED with error RG_ERR_CANCELLED, and a waiter returns
 * RG_ERR_CANCELLED.  RG_ERR_BUSY when the job has finished rendering already
 * (its result stays available). */
rg_status rg_server_cancel(rg_server* s, int64_t job_id);
/* Linear HDR result (width*height*4 floats); release != 0 forgets the job. */
rg_status rg_server_get_result(rg_server* s, int64_t job_id, float* hdr_rgba, size_t count, int32_t release);
/* Progressive result of a resident job (current sample mean), taken between waves. */
rg_status rg_server_snapshot(rg_server* s, int64_t job_id, float* hdr_rgba, size_t count, double timeout_ms);
rg_status rg_server_get_stats(rg_server* s, rg_server_stats* out);
/* Autotuner: renders the probe jobs with candidate wave sizes (paths_per_wave)
 * and launch widths (shade_blocks_per_sm, trace_blocks_per_sm) on servers
 * built from `cfg`, by coordinate descent on the wall time of the whole mix
 * (a candidate replaces the incumbent when it is more than 3% faster), and
 * writes the fastest into `cfg`.  best_ms (may be NULL): its wall time.  The
 * probe should be a sample of the real mix (its spp included). */
rg_status rg_server_autotune(const rg_settings* base, const rg_job_desc* probe, int32_t count, rg_server_config* cfg,
                             double* best_ms);
/* Learned denoiser for jobs submitted with denoise = 2 (NULL: A-Trous).  Keep
 * `d` alive while it is set. */
rg_status rg_server_set_denoiser(rg_server* s, rg_denoiser* d);
rg_status rg_server_destroy(rg_server* s);

#ifdef __cplusplus
}
#endif
#endif /* RAYGEN_B200_H */
