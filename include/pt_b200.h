/*
 * pt_b200 -- C ABI of the B200 (sm_100a) path tracer that stands in for the
 * render path of LSystemEditor's PathTracerLib.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes.  No
 * CUDA, Qt, OpenGL or torch types cross this boundary (streams are passed as
 * void*).  Every entry point names the reference interface it replaces
 * (paths are relative to the reference project root).
 *
 * Record layouts are byte-compatible with the reference structs, so a caller
 * that already fills MaterialGpu / TextureDescGpu / CameraGpu / RenderParamsGpu
 * can pass them through unchanged.
 */
#ifndef PT_B200_H
#define PT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__cplusplus)
#define PT_ALIGN16 alignas(16)
#else
#define PT_ALIGN16 _Alignas(16)
#endif

/* ------------------------------------------------------------------------ */
/* Status codes (the reference returns bool + AppLog text; PathTracer.cu:568-574). */
enum pt_status {
    PT_OK = 0,
    PT_ERR_INVALID_ARGUMENT = 1, /* null handle / pointer, bad size              */
    PT_ERR_CUDA = 2,             /* a CUDA runtime call failed                    */
    PT_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed                      */
    PT_ERR_NO_SCENE = 4,         /* render before a scene was set                 */
    PT_ERR_NOT_CONFIGURED = 5,   /* render before pt_configure                    */
    PT_ERR_TIMEOUT = 6,          /* a bounded device-side wait gave up            */
    PT_ERR_UNSUPPORTED = 7,      /* feature not available in this build           */
    PT_ERR_INTERNAL = 8          /* device-side consistency check failed          */
};

/* ------------------------------------------------------------------------ */
/* Records.                                                                 */

/* MaterialGpu (PathTracerLib/src/MeshAccel/MeshAccelTypes.h:49-86), 96 bytes.
 * `sheen` occupies the reference's tail padding (no reference counterpart). */
typedef struct PT_ALIGN16 pt_material {
    float r, g, b;
    float roughness;
    float metallic;
    float transmission;
    float thin;
    float ior;
    float subsurface;
    float emission;
    float diffuse_roughness;
    float scatter_radius_r, scatter_radius_g, scatter_radius_b;
    float specular;
    uint32_t albedo_tex, roughness_tex, metallic_tex, transmission_tex;
    uint32_t thin_tex, ior_tex, subsurface_tex, emission_tex;
    float sheen;
} pt_material;

/* TextureDescGpu (MeshAccelTypes.h:22-28), 64 bytes. kind: 0 constant scalar,
 * 1 constant rgb, 2 grid 2D, 3 stripe 1D (MeshAccelTypes.h:13-19). */
typedef struct PT_ALIGN16 pt_texture {
    uint32_t kind;
    uint32_t pad[3];
    float p0[4];
    float p1[4];
    float p2[4];
} pt_texture;

/* CameraGpu (PathTracerLib/src/CameraGpu.h:5-16), 80 bytes. orientation is a
 * unit quaternion (w, x, y, z); the camera looks down its local -Z. */
typedef struct PT_ALIGN16 pt_camera {
    float position[3];
    float pad0;
    float orientation[4];
    float fov_y;
    float aspect;
    float near_plane;
    float far_plane;
    float aperture_radius;
    float focus_distance;
    float focus_point[3];
    int32_t focus_valid;
    float pad1[2];
} pt_camera;

/* RenderParamsGpu (PathTracerLib/src/RenderTypes.h:15-28): the first 44 bytes
 * are the reference struct; the tail holds extensions whose zero value keeps
 * the reference behaviour. 64 bytes. */
typedef struct pt_render_params {
    float background_r, background_g, background_b;
    float environment_intensity;
    int32_t max_path_depth;             /* 0 = 256 bounces, <0 = 32 (reference default) */
    int32_t russian_roulette_min_depth; /* <0 = 3 */
    int32_t min_samples;
    int32_t max_samples_per_pixel;      /* <=0 = unlimited */
    int32_t debug_overlay_mode;         /* accepted, display-only in the reference */
    int32_t brdf_debug_flags;           /* BrdfDebugFlags (Brdf/BrdfDebug.h:6-19) */
    float relative_error_threshold;
    /* --- extensions --- */
    int32_t seed_mode;          /* 0: reference seed (Sampling/RandCore.h:7-12); 1: hash(x, y, seed_value) */
    uint32_t seed_value;
    int32_t adaptive_criterion; /* 0: relative std-dev (reference); 1: relative std-error; 2: as 1, and a
                                   pixel all of whose samples are black stops after max(min_samples, 64) */
    int32_t samples_per_launch; /* waves traced per launch; 0 = automatic */
    int32_t spectral_wavelengths; /* 0: RGB (reference); 4 or 8: hero-wavelength spectral samples */
    int32_t emitter_mis;        /* 0: reference emissive NEE (its shadow ray runs to 1e6 and the sampled
                                   emitter blocks it, so emitters are found by BSDF sampling only);
                                   1: at opaque vertices (no transmission, no subsurface, no BRDF debug
                                   flags, flat scenes) the shadow ray stops short of the light sample and
                                   BSDF-sampled emitter hits are balance-weighted against it: the same
                                   expected image, far less noise from small lights (no reference
                                   counterpart) */
    int32_t reserved[3];        /* zero */
} pt_render_params;

/* Triangle soup in structure-of-arrays form: HostMesh + HostTriangle
 * (Application/src/MeshBuilder/HostMesh.h:9-28). All pointers are HOST memory. */
typedef struct pt_mesh {
    uint32_t triangle_count;
    const float* positions;      /* 9 floats per triangle: v0, v1, v2           */
    const float* normals;        /* 9 floats per triangle: n0, n1, n2 (shading) */
    const float* uvs;            /* 6 floats per triangle: uv0, uv1, uv2        */
    const uint32_t* material_ids;
    uint32_t material_count;
    const pt_material* materials;
    uint32_t texture_count;
    const pt_texture* textures;
} pt_mesh;

/* Placement of one object in an instanced scene (no reference counterpart:
 * the reference flattens its ProceduralInstance list into one mesh,
 * Application/src/MeshBuilder/MeshSceneContent.h:16-20). */
typedef struct pt_instance {
    float object_to_world[12]; /* 3 x 4 row-major: linear part | translation */
    uint32_t object;           /* index into the objects of pt_set_instances  */
    uint32_t pad[3];
} pt_instance;

/* Statistics of the accumulation (PathTracer.h:94-99 plus timings). */
typedef struct pt_stats {
    int64_t waves;              /* currentSampleCount: full-resolution waves taken */
    int64_t active_pixels;      /* currentActivePixelCount                          */
    int64_t samples;            /* path samples accumulated since reset             */
    int64_t rays;               /* primary + continuation + shadow rays traced      */
    int64_t launches;           /* device kernel launches issued                    */
    double render_ms;           /* device time of the last pt_render call           */
    double build_ms;            /* device time of the last scene build              */
    int32_t budget_exhausted;   /* isSampleBudgetExhausted                          */
    int32_t bvh_nodes;          /* compressed 8-wide nodes                          */
    int32_t tape_underruns;     /* reserved                                         */
    int32_t stack_overflows;    /* traversal stack overflows (rays truncated)       */
} pt_stats;

/* Per-stage device timings and traversal counters of the last pt_render call
 * (enabled with pt_set_profiling; no reference counterpart beyond the
 * PATHTRACER_PROFILE wait log of PathTracer.cpp:1087-1123). */
typedef struct pt_profile {
    double ms_generate, ms_extend, ms_shade, ms_shadow, ms_finalize, ms_accumulate, ms_compact;
    int64_t launches_extend, launches_shadow;
    int64_t rays_extend, rays_shadow;   /* rays traced by the closest-hit / any-hit stages */
    int64_t nodes_extend, tris_extend;  /* compressed nodes / triangles visited (counting mode) */
    int64_t nodes_shadow, tris_shadow;
} pt_profile;

enum pt_profile_flags {
    PT_PROFILE_STAGE_TIMES = 1,   /* CUDA events around every stage launch */
    PT_PROFILE_COUNT_VISITS = 2   /* count BVH nodes and triangles visited per stage */
};

typedef struct pt_renderer pt_renderer;

/* ------------------------------------------------------------------------ */
/* Renderer object: replaces class PathTracer (PathTracerLib/src/PathTracer.h:30-152). */

/* PathTracer::PathTracer + cudaSetDevice.  device < 0 selects the current one. */
int pt_create(pt_renderer** out, int device);
/* PathTracer::~PathTracer. Releases every device buffer. */
int pt_destroy(pt_renderer* r);
/* Text of the last error on this renderer (never NULL). */
const char* pt_last_error(const pt_renderer* r);

/* PathTracer::configure (PathTracer.h:45-51) minus the GL PBOs: allocates the
 * accumulation state for width x height pixels (PathTracer.cpp:323-419). */
int pt_configure(pt_renderer* r, int width, int height);

/* MeshAccelScene::build + upload (MeshAccel/MeshAccelScene.h:22-27,
 * MeshAccelScene.cpp:141-341) and PathTracer::rebuildMeshScene (PathTracer.h:130-132):
 * uploads the mesh and builds the acceleration structure ON THE GPU
 * (LBVH -> compressed 8-wide BVH). Resets accumulation. */
int pt_set_mesh(pt_renderer* r, const pt_mesh* mesh);

/* PathTracer::setCamera / lastSampleCamera (PathTracer.h:101-103). */
int pt_set_camera(pt_renderer* r, const pt_camera* camera);
int pt_get_camera(const pt_renderer* r, pt_camera* out);

/* Snapshot of the setters setMaxSamplesPerPixel, setMinSamples,
 * setRelativeErrorThreshold, setRussianRouletteMinDepth, setBrdfDebugFlags,
 * setClearColor, setEnvironmentIntensity (PathTracer.h:73-124) as one record
 * (RenderParamsGpu, RenderTypes.h:15-28). Resets accumulation.  Values are
 * clamped as those setters clamp them (PathTracer.cpp:126-190): max spp to
 * [0, 1e6], min spp to [1, 1e4], relative error threshold to [0.001, 1], RR
 * depth to >= 0; pt_get_params returns the clamped record. */
int pt_set_params(pt_renderer* r, const pt_render_params* params);
int pt_get_params(const pt_renderer* r, pt_render_params* out);
/* RenderParamsGpu{} defaults (RenderTypes.h:15-28) with a zero extension tail. */
void pt_default_params(pt_render_params* out);

/* PathTracer::setEnvironmentHdrPath (PathTracer.h:115-121) with the decoded
 * image instead of a file: linear RGB lat-long, width x height x 3 floats
 * (host). rgb == NULL restores the solid background. Builds the importance
 * tables of EnvironmentMap.cpp:76-128. Resets accumulation. */
int pt_set_environment(pt_renderer* r, int width, int height, const float* rgb);

/* PathTracer::resetAccumulation + clearAccumulatorKernel (PathTracer.cu:275-303). */
int pt_reset(pt_renderer* r);

/* The render loop (PathTracer::renderLoop, PathTracer.cpp:2220-2543) as a
 * synchronous call: traces `waves` full-resolution adaptive waves, one sample
 * per active pixel per wave, compacting the active list as it goes. Pixels
 * stop at max_samples_per_pixel or when converged. waves <= 0 runs until no
 * pixel is active. */
int pt_render(pt_renderer* r, int waves);

/* Headless replacement of the PBO publish (PathTracer.cu:464-512): copies the
 * running-mean RGBA accumulator (float4 per pixel), sample counts and the
 * convergence mask to HOST memory. Any output pointer may be NULL. */
int pt_readback(pt_renderer* r, float* rgba, uint32_t* counts, uint8_t* converged);

/* Device pointers of the accumulation state (borrowed; valid until the next
 * pt_configure / pt_destroy): float4 rgba[P], uint32 counts[P], uint8 converged[P]. */
int pt_device_buffers(pt_renderer* r, void** rgba, void** counts, void** converged);

/* currentSampleCount / currentActivePixelCount / isSampleBudgetExhausted
 * (PathTracer.h:94-99) and timings. */
int pt_get_stats(const pt_renderer* r, pt_stats* out);

/* PathTracer::pickSurface (PathTracer.h:111, PathTracer.cpp:1991-2013) generalised
 * to n rays: closest hit through the GPU BVH. All pointers HOST memory.
 * origins/dirs: 3 floats per ray; tmin/tmax per ray. Outputs: hit flag, t,
 * ORIGINAL triangle index, shading normal (3 floats), uv (2 floats); any
 * output except hit may be NULL. Semantics of meshAccelTraceRay
 * (MeshAccel/MeshAccelIntersectCore.h:110-221). */
int pt_trace_rays(pt_renderer* r, int n, const float* origins, const float* dirs, const float* tmin,
    const float* tmax, uint8_t* hit, float* t, uint32_t* tri, float* normal, float* uv);

/* Same with DEVICE pointers on the given CUDA stream (void* = cudaStream_t). */
int pt_trace_rays_device(pt_renderer* r, int n, const float* origins, const float* dirs, const float* tmin,
    const float* tmax, uint8_t* hit, float* t, uint32_t* tri, float* normal, float* uv, void* stream);

/* Runs all work of the renderer on the caller's CUDA stream (void* =
 * cudaStream_t; the reference's launch API takes one per call,
 * PathTracerCuda.h:12-126). NULL restores the renderer's own stream. */
int pt_set_stream(pt_renderer* r, void* stream);

/* Profiling switches (pt_profile_flags) and the profile of the last pt_render. */
int pt_set_profiling(pt_renderer* r, int flags);
int pt_get_profile(const pt_renderer* r, pt_profile* out);

/* Work-size tuning (no reference counterpart): paths in flight per launch
 * (0 = default 2^24) and resident blocks per SM of the persistent stage grids
 * (0 = from the occupancy calculator). */
int pt_set_tuning(pt_renderer* r, int path_capacity, int blocks_per_sm);

/* Closest-hit and shadow-ray scheduling (no reference counterpart; images are
 * identical in every mode).  AUTO: per-lane ray replacement (closest hit and
 * shadow rays; two-level traversal in instanced scenes) with a slot-ordered
 * next-bounce queue when the largest flat scene or instanced object has at
 * least 32768 BVH nodes, else one warp per 32 queued rays.  WARP / LANE force
 * either form. */
enum pt_extend_mode { PT_EXTEND_MODE_AUTO = 0, PT_EXTEND_MODE_WARP = 1, PT_EXTEND_MODE_LANE = 2 };
int pt_set_extend_mode(pt_renderer* r, int mode);

/* Parity hook (no reference counterpart): writes, for waves [first_wave,
 * first_wave + waves) and every pixel, the first `stride` uniforms that the
 * renderer's generator draws for that (pixel, sample) -- curand_init /
 * curand_uniform with the seed of Sampling/RandCore.h:7-12 -- to HOST memory
 * laid out [wave][pixel][stride]. The active pixels at the time of the call are
 * assumed to have counts == first_wave (a fresh accumulation). */
int pt_rng_tape(pt_renderer* r, int first_wave, int waves, int stride, float* out);

/* ---- Batched form (no counterpart in the reference) ----------------------
 * One renderer can hold several independent scenes (meshes, cameras, image
 * sizes) that pt_render advances together: their pixels form one work queue,
 * so small scenes fill the GPU jointly instead of one launch sequence each.
 * Every scene renders exactly as it would alone (seeds and film coordinates
 * use the pixel's index within its own image); the render parameters and the
 * environment are shared.  pt_configure returns a renderer to one scene; the
 * single-scene calls (pt_set_mesh, pt_set_camera, pt_readback, pt_trace_rays)
 * address scene 0, and pt_device_buffers returns the concatenated pixels of
 * all scenes (scene after scene). */
int pt_batch_configure(pt_renderer* r, int scene_count, const int* widths, const int* heights);
int pt_batch_set_mesh(pt_renderer* r, int scene, const pt_mesh* mesh);
int pt_batch_set_camera(pt_renderer* r, int scene, const pt_camera* camera);
int pt_batch_readback(pt_renderer* r, int scene, float* rgba, uint32_t* counts, uint8_t* converged);

/* ---- Scene generation on the device (no reference counterpart) ----------
 * Turtle output as tubes and leaves, lofted into triangles on the GPU and fed
 * straight to the BVH build (replaces the host loft of
 * Application/src/Procedural/Loft.cpp:108-155 and the HostMesh upload).  Tube
 * t spans rings ring_start[t] .. ring_start[t + 1] - 1 (each ring: centre,
 * tangent, radius, in double); every ring contributes 2 * sides triangles
 * (side quads to the next ring, a flat cap at each tube end) and every leaf a
 * two-triangle quad of size leaf_size * leaf[9] spanning (tangent x up) and
 * the tangent.  The mesh is [tubes in order, leaves in order, extra]; all
 * material ids index the material bank of `extra`.  Per tube the triangles
 * follow buildLoftHostMeshFromFrames: side walls ring by ring (the seam vertex
 * shared with side 0), then start and end caps interleaved per side with rim
 * uvs 0.5 + 0.5 (sin, cos).  cos_sin may be NULL (the library then tabulates
 * the reference's angles k * 6.283185307f / sides, cosine and sine rounded to
 * single precision). */
typedef struct pt_tubes {
    uint32_t tube_count;
    uint32_t sides;
    const uint32_t* ring_start;   /* tube_count + 1 offsets, ring_start[0] = 0 */
    const double* points;         /* 3 per ring */
    const double* tangents;       /* 3 per ring */
    const double* radii;          /* 1 per ring */
    const uint32_t* materials;    /* 1 per tube */
    const double* cos_sin;        /* 2 * (sides + 1) or NULL */
    uint32_t leaf_count;
    const double* leaves;         /* 10 per leaf: position, tangent, up, size */
    double leaf_size;
    uint32_t leaf_material;
    const double* frames;         /* 6 per ring: unit normal, unit binormal (e.g. the reference's
                                     spline frames, Spline.cpp:102-255), or NULL: a frame derived
                                     from the ring tangent (+Y reference axis, the last ring of a
                                     tube takes the tangent of the one before it) */
} pt_tubes;

/* Builds scene `scene` (0 for a single-scene renderer) from tubes, leaves and
 * an extra triangle soup (ground, lights; may have no triangles but carries
 * the material bank). */
int pt_batch_set_tubes(pt_renderer* r, int scene, const pt_tubes* tubes, const pt_mesh* extra);

/* Copies scene `scene`'s triangles back to host memory in their original
 * order (for OBJ export; MeshAccelWavefrontExport.cpp:64-142 exports from the
 * host mesh instead): 9 + 9 + 6 floats and 1 material id per triangle.  Any
 * output may be NULL; *triangle_count receives the count. */
int pt_export_mesh(pt_renderer* r, int scene, uint32_t* triangle_count, float* positions, float* normals,
    float* uvs, uint32_t* material_ids);

/* Headless display output: replaces the GL publish path
 * (PathTracer::publishDisplayFrame, PathTracer.cu:421-512 writeDisplayToPboKernel
 * without downscale).  Writes scene `scene`'s image as 8-bit RGBA to HOST memory
 * (width x height x 4 bytes): background colour where a pixel has no sample,
 * rgb x exposure, Reinhard x / (1 + x), clamp to [0, 1], x 255 truncated; with
 * debug_overlay_mode 2 the adaptive-sampling overlay (green converged, red
 * active). */
int pt_tonemap(pt_renderer* r, int scene, float exposure, uint8_t* rgba8);

/* PhysicalCamera::exposureMultiplier (PhysicalCamera.cpp:392-397):
 * shutter x (max(iso, 1) / 100) / max(f_stop, 0.1)^2. */
float pt_exposure_multiplier(float f_stop, float shutter_seconds, float iso);

/* ---- Differentiation (no counterpart in the reference) --------------------
 * Replaces the material bank of scene `scene` (same meaning of the material
 * ids; textures kept) without rebuilding its BVH; the emissive list follows. */
int pt_set_materials(pt_renderer* r, int scene, uint32_t material_count, const pt_material* materials);

/* Keeps, from the next render onwards, the radiance of samples 0 .. spp - 1 of
 * every pixel (16 bytes each, spp x pixels) so that pt_backward reads it
 * instead of tracing each path a first time.  It is used when the last
 * pt_render drew exactly spp samples per pixel (min_samples ==
 * max_samples_per_pixel == spp) with the current scene, camera and
 * parameters; 0 releases it.  Single-scene renderers. */
int pt_record_samples(pt_renderer* r, int spp);

/* Path-replay backpropagation of an image loss.  d_image: HOST array of
 * d loss / d image, `channels` (3 or 4) floats per pixel, for the image that
 * pt_render draws with `spp` samples per pixel from a reset accumulator with
 * the current scene, camera and parameters (single-scene renderer).  Writes
 * grad[m * 7 + j], j = r, g, b, roughness, metallic, sheen, emission, for
 * materials m < grad_materials (at most 16 materials; textured channels get
 * 0).  Sampling decisions, Russian roulette and MIS weights are treated as
 * constants.  *device_ms (may be NULL) receives the kernel's device time. */
int pt_backward(pt_renderer* r, const float* d_image, int channels, int spp, float* grad, uint32_t grad_materials,
    double* device_ms);

/* The environment's importance tables as built on the device
 * (EnvironmentMap.cpp:76-128): marginal CDF (height + 1 floats) and row CDFs
 * (height x (width + 1)), HOST outputs, either may be NULL. */
int pt_environment_tables(pt_renderer* r, float* marginal, float* row);

/* ---- Instanced scenes and the distant light (extensions) -----------------
 * pt_set_instances: `object_count` meshes (HOST arrays; the material and
 * texture banks of objects[0] serve all objects) placed by `instance_count`
 * instances.  Every object gets its own BVH and the instances a top-level BVH,
 * all built on the device; rays are traversed in two levels (object-space rays
 * for the objects).  Emissive triangles inside objects are reached by BSDF
 * sampling only.  pt_export_mesh and pt_backward reject instanced scenes. */
int pt_set_instances(pt_renderer* r, int scene, uint32_t object_count, const pt_mesh* objects,
    uint32_t instance_count, const pt_instance* instances);

/* Batch view: scene `scene` renders the geometry and materials of scene
 * `source` (set before or after) with its own camera and image, so several
 * views of one scene share their BVHs in one render.  Setting a mesh on
 * `scene` ends the sharing. */
int pt_batch_share_scene(pt_renderer* r, int scene, int source);

/* Distant light: constant radiance inside a cone of half-angle `half_angle`
 * (radians, 0 < half_angle < 1.5) around `direction` (towards the light).
 * Radiance: `radiance` (RGB) when temperature_k <= 0, else a blackbody of that
 * temperature whose linear sRGB has Rec. 709 luminance `luminance` (and whose
 * spectrum is Planck's law in spectral mode).  It is sampled together with
 * the environment: the next-event sample of the sky takes one extra random
 * number, drawn just before the environment sample's two, to pick the light
 * (probability 1/2, or 1 when the sky is black) or the environment, and is
 * MIS-weighted against BSDF sampling by the
 * mixture's density; escaping rays see environment plus light.  NULL or
 * enabled = 0 removes it (the reference's estimator then runs unchanged).
 * Preview passes show the environment only; pt_backward rejects a scene lit
 * by it. */
typedef struct pt_distant_light {
    float direction[3];
    float half_angle;
    float radiance[3];
    float temperature_k;
    float luminance;
    int32_t enabled;
} pt_distant_light;

int pt_set_distant_light(pt_renderer* r, const pt_distant_light* light);

/* ---- Autotuner (no reference counterpart) ---------------------------------
 * Chooses the scheduling knobs for the current scene(s), camera(s) and
 * parameters: path capacity (paths in flight, 2^21 .. 2^24), blocks per SM of
 * the stage kernels (occupancy calculator, 2, 3, 4) and waves per launch
 * (pt_render_params.samples_per_launch: automatic, 4, 16, 64), one knob at a
 * time from the current configuration, each candidate timed on the device
 * over `waves` waves from a reset accumulator.  The fastest is kept (also in
 * the params) and the accumulation is reset.  The knobs change only how the
 * work is scheduled: every candidate renders the same image. */
typedef struct pt_tuning {
    int32_t path_capacity;
    int32_t blocks_per_sm;       /* 0 = occupancy calculator */
    int32_t samples_per_launch;  /* 0 = automatic */
    int32_t trials;
    double ms_default;           /* probe time of the configuration it started from */
    double ms_best;
} pt_tuning;

int pt_autotune(pt_renderer* r, int waves, pt_tuning* out);

/* L2-resident read bandwidth of this GPU (no reference counterpart; the roof
 * of kernels whose working set fits in L2): 128-bit loads that bypass L1 over
 * a `bytes` buffer (keep it well under the L2 size), `reps` passes after one
 * warming pass, timed with events on the renderer's stream.  *gb_per_s
 * receives bytes read / time. */
int pt_measure_l2(pt_renderer* r, uint64_t bytes, int reps, double* gb_per_s);

/* BVH build quality knob (no reference counterpart; the reference's host
 * median split has none): the number of treelet SAH reordering passes of the
 * GPU build (Karras & Aila 2013), 0 = the plain Karras LBVH; default 1.
 * Applies to the following mesh / instance / batch builds. */
int pt_set_bvh_options(pt_renderer* r, int treelet_passes);
/* SAH cost of scene `scene`'s binary BVH as built (before the collapse to
 * 8-wide nodes; one triangle per leaf): (1.2 * sum of inner node areas +
 * sum of leaf areas) / root area.  A quality measure for tests and tuning. */
int pt_bvh_sah_cost(pt_renderer* r, int scene, double* cost);

/* Stable LSD radix sort of n (key, value) pairs of 32-bit unsigned integers on
 * the low `bits` bits of the keys, over DEVICE buffers, on `stream` (no
 * counterpart in the reference, whose BVH is a host median split; the GPU BVH
 * build sorts its 30-bit Morton keys with it).  keys/vals are left unchanged,
 * keys_out/vals_out (not aliasing them) receive the sorted pairs; temp is
 * device scratch of at least pt_radix_sort_temp_bytes(n) bytes.  Returns
 * PT_ERR_INVALID_ARGUMENT for null pointers, bits outside 1..32 or too little
 * scratch. */
size_t pt_radix_sort_temp_bytes(uint32_t n);
int pt_radix_sort_pairs(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out, uint32_t* vals_out, uint32_t n,
    int bits, void* temp, size_t temp_bytes, void* stream);

/* ---- Spectral mode (extension; the reference's integrator is RGB) ---------
 * With pt_render_params.spectral_wavelengths = 4 or 8, every path carries
 * that many wavelengths spread evenly over [380, 780] nm from a hero
 * wavelength drawn per (pixel, sample) (Wilkie et al., EGSR 2014); colours
 * (materials, textures, background, environment texels, emitters) become
 * spectra s(lambda) = scale * (1/2 + x / (2 sqrt(1 + x^2))),
 * x = c0 lambda^2 + c1 lambda + c2 (the function space of the reference's
 * Spectral/Rgb2Spec.h:58-66, Jakob and Hanika 2019), and each sample is
 * converted to linear sRGB through CIE 1931 x 2-degree colour matching
 * weighted by D65 (Spectral/SpectralCore.h:128-139) before accumulation.
 * Previews and pt_backward stay RGB (pt_backward rejects a spectral render
 * with PT_ERR_UNSUPPORTED). */

/* The sRGB response per nm, 401 entries (380 .. 780 nm) x 3 floats, HOST
 * output: a spectrum L gives RGB = integral L(lambda) response(lambda) dlambda;
 * each channel sums to 1 by the trapezoid rule, so L = 1 gives (1, 1, 1).
 * Optionally (each output may be NULL) the data it is built from: cie =
 * x-bar, y-bar, z-bar and D65 at 380 .. 780 nm every 10 nm (41 x 4 floats),
 * xyz_to_rgb = the XYZ -> linear sRGB matrix (3 x 3, row-major).  Needs no GPU. */
int pt_spectral_response(float* rgb, float* cie, float* xyz_to_rgb);

/* Spectrum coefficients (c0, c1, c2, scale; lambda in nm) of `count` RGB
 * colours (radiance rules: negative channels 0, colours brighter than 1 scaled
 * by their largest channel), HOST arrays, as the renderer uses them.  Needs
 * no GPU. */
int pt_spectral_uplift(uint32_t count, const float* rgb, float* coef);

/* ---- Preview passes and region render ------------------------------------ */
/* PathTracer::setPreviewStepsPerLevel (PathTracer.h:89-92): with n > 0 (at
 * most 128), pt_render first renders n low-resolution preview passes, level i
 * at 1 / 2^(n - i) of the image (PathTracerPreviewLevels.h:17-49), one sample
 * per pixel at the pixel centre, depth 4, global seed i + 1; full-resolution
 * wave w then draws with global seed n + w + 1, as the reference's iteration
 * count includes the previews.  Until the first full-resolution wave,
 * pt_tonemap shows the finest preview upsampled.  Single-scene renderers. */
int pt_set_preview_levels(pt_renderer* r, int levels);
/* Renders the preview passes not yet rendered since the last reset (pt_render
 * does it first anyway), so that a display can show them before any wave. */
int pt_render_previews(pt_renderer* r);
/* A preview level's float RGBA image (HOST, width x height x 4) and size. */
int pt_preview_readback(pt_renderer* r, int level, float* rgba, int* width, int* height);

/* setRegionRenderEnabled + setRenderRegion (PathTracer.h:134-138,
 * PathTracer.cpp:1447-1463): only the pixels of the rectangle (corners ordered
 * and clamped to the image) take samples; enabling clears the region and keeps
 * the rest of the image.  A reset (parameter change) clears the whole image and
 * keeps sampling only the region. */
int pt_set_region(pt_renderer* r, int enabled, int min_x, int min_y, int max_x, int max_y);
/* resetRegionAccumulation (PathTracer.h:140): clears the region only. */
int pt_reset_region(pt_renderer* r);

/* Largest triangle count pt_trace_soup_noalloc accepts. */
#define PT_NOALLOC_MAX_TRIANGLES 16384u

/* Closest-hit queries against a small triangle soup that allocates no device
 * memory (no counterpart in the reference).  For callers that cannot allocate:
 * hosts whose allocator owns the whole device and hands out every byte itself
 * (a cudaMalloc behind its back can fail or break its accounting), and
 * latency-critical callbacks such as a viewport's surface pick, for which
 * cudaMalloc/cudaFree cost an implicit device synchronisation each time.  Every input and output
 * is a DEVICE pointer supplied by the caller (positions 9 floats/triangle;
 * normals and uvs may be NULL: without normals the reported normal is the
 * triangle's geometric normal facing the ray, without uvs the uv is 0; results
 * as in pt_trace_rays); work runs on `stream` (NULL = default stream) of the
 * current device.  The BVH build waits for `stream` once per tree level, so
 * the call blocks the host until the build is done and returns with the
 * traversal enqueued.  All temporaries live in one 8 MiB device array,
 * reserved on a GPU when the library's module is first loaded there (at the
 * latest at the first call) and kept for the life of the process; up to
 * PT_NOALLOC_MAX_TRIANGLES triangles (larger inputs are rejected with
 * PT_ERR_INVALID_ARGUMENT and a message).  The first call in a CUDA context
 * (per device, and again after that context is destroyed and recreated, e.g.
 * by cudaDeviceReset) looks up that array's device address -- make it before
 * any stream capture.  Calls share the array, so calls whose GPU work overlaps
 * race and must be serialised by the caller.  error_message (may be NULL)
 * receives the reason of a failure. */
int pt_trace_soup_noalloc(uint32_t triangle_count, const float* positions, const float* normals, const float* uvs,
    int n, const float* origins, const float* dirs, const float* tmin, const float* tmax, uint8_t* hit, float* t,
    uint32_t* tri, float* normal, float* uv, void* stream, char* error_message, size_t error_capacity);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* PT_B200_H */
