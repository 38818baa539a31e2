/* pcr_cuda.h -- C ABI of the B200 (sm_100a) wavefront spectral path tracer.
 *
 * This is the drop-in boundary for pcr's GPU backend.  In the reference the
 * GPU renderer is chosen by a compile-time alias (code/Gpu/GpuRenderer.h:15-21)
 * and driven through the OpenglRenderer/MetalRenderer surface
 * (code/Gpu/Opengl/OpenglRenderer.h:29-117): a constructor taking
 * (width, height, depth, samples, shadowSamples), public quality knobs, and
 * render(const Scenes::SceneData&, start, outputDir).  A CudaRenderer class
 * with that surface (pcr_b200/csrc/cuda_renderer.h) wraps the calls below.
 *
 * Conventions: plain C types only; every call returns a pcr_status; no
 * exception crosses the boundary; host buffers are caller-owned; a context
 * owns all device memory it allocates.  pcr_last_error() gives the message
 * of the last failing call on the calling thread.
 */
#ifndef PCR_CUDA_H
#define PCR_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PCR_OK = 0,
    PCR_ERR_INVALID = 1,      /* bad argument or descriptor */
    PCR_ERR_CUDA = 2,         /* CUDA runtime error */
    PCR_ERR_NO_MEMORY = 3,    /* device memory budget exceeded */
    PCR_ERR_NOT_FOUND = 4,    /* unknown scene / request id */
    PCR_ERR_SCENE = 5,        /* scene file could not be loaded */
    PCR_ERR_TIMEOUT = 6,      /* a bounded wait expired */
    PCR_ERR_CANCELLED = 7,
    PCR_ERR_DEVICE_STATUS = 8 /* a kernel reported an error status word */
} pcr_status;

#define PCR_SPECTRUM_SAMPLES 61

typedef struct pcr_ctx pcr_ctx;
typedef int32_t pcr_scene_id;
typedef int64_t pcr_request_id;

/* ------------------------------------------------------------- scene POD
 * Field meaning follows the reference SceneData (code/Scenes/Scene.h:58-83)
 * after loadSceneFromFile (code/Scenes/SceneLoader.cpp:475-516): triangles
 * already in BVH-leaf order and the binary SAH BVH (code/Bvh/Bvh.h:28-35)
 * prebuilt; material spectral fits populated (code/Includes/Material.h:125-139). */
typedef struct {
    float albedo[3], emissive[3];
    int32_t metallic, transparent, use_tab_albedo, use_tab_emissive;
    float ior, cauchy_b;
    float albedo_fit[4], emissive_fit[4];          /* c0 c1 c2 scale */
    float tab_albedo[PCR_SPECTRUM_SAMPLES], tab_emissive[PCR_SPECTRUM_SAMPLES];
} pcr_material;

typedef struct { float origin[3], u[3], v[3], n[3], area; int32_t mat; } pcr_plane;
typedef struct { float center[3], radius; int32_t mat; } pcr_sphere;
typedef struct {
    float v0[3], v1[3], v2[3], n0[3], n1[3], n2[3], flat_n[3];
    int32_t smooth, mat;
} pcr_triangle;
typedef struct { float bmin[3], bmax[3]; int32_t left_or_first, right_child, count; } pcr_bvh_node;
/* kind 0: plane light (plane); kind 1: triangle set
 * (light_triangles[tri_offset .. tri_offset+tri_count), cumulative areas alongside) */
typedef struct { int32_t kind; float total_area; pcr_plane plane; int32_t tri_offset, tri_count; } pcr_light;

typedef struct {
    const char *name, *version;
    float cam_pos[3], fov;
    int32_t n_materials; const pcr_material *materials;
    int32_t n_spheres;   const pcr_sphere *spheres;
    int32_t n_planes;    const pcr_plane *planes;       /* light planes first, then walls */
    int32_t n_triangles; const pcr_triangle *triangles; /* BVH-leaf order */
    int32_t n_bvh_nodes; const pcr_bvh_node *bvh_nodes; /* may be 0: the library builds it */
    int32_t n_lights;    const pcr_light *lights;
    const pcr_triangle *light_triangles; const float *light_cum_area;
    const int32_t *triangle_ids; /* optional id reported per triangle; NULL = index */
} pcr_scene_desc;

/* ------------------------------------------------------------- render POD
 * Knobs of the reference Renderer (code/Includes/Renderer.h:45-102) with the
 * GPU backends' meaning of `samples`: paths per pixel
 * (code/Gpu/Opengl/OpenglRenderer.cpp:1302). */
typedef struct {
    int32_t width, height, depth, samples, shadow_samples;
    int32_t spectral, hero_samples, mis, russian, stratified;
    /* aa_samples: jittered camera rounds per pixel, each of `samples` paths.
     * adaptive (with aa_samples > 1): a pixel stops after 4 or more rounds
     * once every channel's relative variance of the round means is below
     * 0.05 (code/Gpu/Opengl/OpenglRenderer.cpp:1288-1383).  denoise: two
     * 5x5 bilateral passes on the 8-bit image, on the device
     * (code/Denoise.cpp:14-86). */
    int32_t aa_samples, adaptive, aces, denoise;
    uint64_t seed;           /* 0 -> 1 */
    int32_t priority;        /* batched / served: pending requests are admitted lowest value
                              * first, in submit order among equals (0 default) */
    /* plain method only: 0 = one sample per pixel per pass, the reference
     * wavefront's default (code/Includes/GpuDefaults.h:44-50); 1 = passes
     * as large as the queue (wavefrontMultiSample) */
    int32_t multi_sample;
    /* Sample range [sample_begin, sample_end) of `samples` (0, 0 = all).  A
     * render split across GPUs gives each one a range; the HDR images are
     * then partial sums (each already divided by samples * aa) that add up
     * to the full image, and pcr_tonemap makes the 8-bit image of the sum.
     * Not with adaptive sampling. */
    int32_t sample_begin, sample_end;
    /* spectral_fork = false of the GPU backends (code/Includes/GpuDefaults.h:55-71,
     * code/Gpu/Metal/MetalRenderer.mm:2155-2252): at the first dispersive
     * refraction a path keeps its hero wavelength alone, scaled by the number
     * of hero wavelengths, instead of forking one sub-path per wavelength.
     * 0 = fork (default, as the CPU renderer). */
    int32_t spectral_terminate;
} pcr_render_desc;

typedef struct {
    double device_ms;        /* first issue -> last path retired, device clock */
    double latency_ms;       /* submit -> result ready (host clock) */
    double queue_ms;         /* submit -> admission */
    uint64_t paths, rays, shadow_rays;
} pcr_render_stats;

typedef struct {
    int32_t device;          /* CUDA ordinal */
    int64_t memory_budget;   /* bytes the context may hold for requests (0: 40 GiB) */
    int32_t queue_capacity;  /* paths in flight (0: autotuned / default) */
    int32_t block_size;      /* threads per block for the trace/shade kernels (0: default) */
    int32_t chunk_paths;     /* per-request issue chunk per iteration (0: default) */
    int32_t regen_every;     /* refill cadence in iterations (0: 1) */
    int32_t use_graph;       /* capture the iteration loop in a CUDA graph (default 1) */
    int32_t profile;         /* time each stage with CUDA events */
    const char *tuning_cache;/* autotuner cache file (NULL: none) */
} pcr_ctx_opts;

/* ------------------------------------------------------------- context */
const char *pcr_last_error(void);
const char *pcr_version(void);
pcr_status pcr_ctx_create(pcr_ctx **out, const pcr_ctx_opts *opts);
pcr_status pcr_ctx_destroy(pcr_ctx *ctx);
/* Pins the calling thread's current device to the context's device. */
pcr_status pcr_ctx_set_device(pcr_ctx *ctx);
/* The CUDA stream (cudaStream_t) every kernel of this context runs on, so a
 * caller can order its own work or time the engine with CUDA events. */
pcr_status pcr_ctx_stream(pcr_ctx *ctx, void **stream);

/* ------------------------------------------------------------- scenes */
/* Upload a loaded scene (flat POD arrays) into the device scene cache.
 * Replaces the GPU upload of code/Gpu/Opengl/OpenglRenderer.cpp:1657-1912. */
pcr_status pcr_scene_upload(pcr_ctx *ctx, const pcr_scene_desc *desc, pcr_scene_id *out);
/* Load a scene JSON (schema 1.x, code/Scenes/SceneLoader.cpp:475-516) with the
 * library's own loader and upload it.  data_root holds spd/ (may be NULL:
 * the JSON's directory).  lut_path: PLUT file for the RGB->spectrum fit
 * (code/RGBToSpectrum.cpp:420-451) or NULL for the runtime fit. */
pcr_status pcr_scene_load_json(pcr_ctx *ctx, const char *path, const char *data_root,
                               const char *lut_path, pcr_scene_id *out);
pcr_status pcr_scene_release(pcr_ctx *ctx, pcr_scene_id id);

/* Host-side scene admission without a device: loads a scene JSON into flat
 * arrays (what pcr_scene_load_json uploads) and fills *desc with pointers
 * into them, valid until pcr_host_scene_free.  Same loader semantics as
 * code/Scenes/SceneLoader.cpp:475-516 (BVH built, spectra populated). */
typedef struct pcr_host_scene pcr_host_scene;
pcr_status pcr_host_scene_load(const char *path, const char *data_root, const char *lut_path,
                               pcr_host_scene **out, pcr_scene_desc *desc);
pcr_status pcr_host_scene_free(pcr_host_scene *scene);
/* RGBToSpectrum::fitSigmoidCoefficients (code/RGBToSpectrum.cpp:256-293) for n
 * RGB triples; lut (3*16^3*3 floats) or NULL for the runtime homotopy. */
pcr_status pcr_fit_sigmoid(const float *rgb, int64_t n, const float *lut, float *out4);
/* RGBToSpectrum::buildLUT (code/RGBToSpectrum.cpp:332-385): 3*16^3*3 floats. */
pcr_status pcr_lut_build(float *out);
/* Device bytes held by a scene (its cache entry). */
pcr_status pcr_scene_bytes(pcr_ctx *ctx, pcr_scene_id id, int64_t *bytes);

/* ------------------------------------------------------------- rendering */
/* Plain method: one render through its own launch sequence, synchronous.
 * hdr_out: W*H*3 linear sRGB floats (may be NULL); rgb8_out: W*H*3 tone-mapped
 * 8-bit pixels (may be NULL).  Mirrors Renderer::render's framebuffer and
 * quantised output (code/Renderer.cpp:113-382). */
pcr_status pcr_render(pcr_ctx *ctx, pcr_scene_id scene, const pcr_render_desc *desc,
                      float *hdr_out, uint8_t *rgb8_out, pcr_render_stats *stats);

/* Plain render that allocates nothing.  This entry point has no counterpart
 * in the reference; it exists for callers that may not allocate device
 * memory while they render: a host that has handed all device memory to its
 * own pool allocator, or a real-time loop that cannot afford cudaMalloc /
 * cudaFree, which synchronize the whole device and stall every other stream.
 * All working memory (path and shadow queues, hit records, the FP64 pixel
 * accumulator, request and counter words) comes from one fixed array of
 * about 21 MiB compiled into the library, which every GPU that loads the
 * library holds until the process exits.
 *   - scene: a scene already uploaded to ctx (an input; not copied again).
 *   - hdr_out_dev / rgb8_out_dev: caller-owned DEVICE buffers of W*H*3 floats /
 *     bytes (either may be NULL, not both), written as pcr_render writes them.
 *   - Limits: at most 65536 pixels (e.g. 256x256) and at most 8 shadow samples
 *     per hit; larger requests return PCR_ERR_INVALID.
 * The first call on a device looks up the array's device address on that
 * device (cudaGetSymbolAddress); make that first call before any stream
 * capture.  Every call shares the one array and clears what must start at
 * zero, so calls that overlap on the GPU (from several threads, or several
 * contexts on one device) race; serialise them.  Synchronous. */
pcr_status pcr_render_noalloc(pcr_ctx *ctx, pcr_scene_id scene, const pcr_render_desc *desc,
                              float *hdr_out_dev, uint8_t *rgb8_out_dev);

/* Batched / served method.  pcr_submit is thread-safe and returns at once;
 * the request is admitted into the shared wavefront when the memory budget
 * and queue allow.  pcr_run_until_idle drives the engine on the calling
 * thread until every submitted request is finished; pcr_serve_start runs it
 * on a background thread instead (continuous batching). */
pcr_status pcr_submit(pcr_ctx *ctx, pcr_scene_id scene, const pcr_render_desc *desc,
                      pcr_request_id *out);
pcr_status pcr_run_until_idle(pcr_ctx *ctx);
pcr_status pcr_serve_start(pcr_ctx *ctx);
pcr_status pcr_serve_stop(pcr_ctx *ctx);
/* done = 1 when the request's result is ready. */
pcr_status pcr_poll(pcr_ctx *ctx, pcr_request_id id, int32_t *done);
/* Waits up to timeout_ms (<0: forever) for the request. */
pcr_status pcr_wait(pcr_ctx *ctx, pcr_request_id id, int64_t timeout_ms);
/* Copies the finished result out and frees the request's device memory. */
pcr_status pcr_fetch(pcr_ctx *ctx, pcr_request_id id, float *hdr_out, uint8_t *rgb8_out,
                     pcr_render_stats *stats);
/* Cancels a request, the counterpart of the reference renderers'
 * cancelRequested flag (code/Renderer.cpp:170-181,
 * code/Gpu/Opengl/OpenglRenderer.cpp:2170-2175).  A request waiting for
 * admission is dropped at once; a running one stops issuing paths at the
 * next block of iterations and ends when the paths in flight retire (within
 * its depth in iterations), its partial result discarded; a finished one
 * keeps its result (the call is then a no-op).  pcr_wait on a cancelled
 * request returns PCR_ERR_CANCELLED; pcr_fetch returns PCR_ERR_CANCELLED
 * and releases it. */
pcr_status pcr_cancel(pcr_ctx *ctx, pcr_request_id id);
/* Share of a request's paths traced to the end, in [0, 1], from the device
 * state copied after each block of iterations: 0 while it waits for
 * admission, 1 once it is resolved.  The counterpart of the reference's
 * progressRows counter (code/Includes/Renderer.h:41-43), which the
 * CudaRenderer surface fills as fraction x height. */
pcr_status pcr_progress(pcr_ctx *ctx, pcr_request_id id, double *fraction);

/* ------------------------------------------------------------- engine info */
typedef struct {
    double stage_ms[8];      /* regen, extend, shade, shadow, resolve, schedule, status, other */
    int64_t stage_launches[8];
    int64_t iterations, paths, rays, shadow_rays;
    int64_t device_bytes;
    int32_t queue_capacity, block_size, chunk_paths, regen_every;
} pcr_engine_stats;
pcr_status pcr_engine_stats_get(pcr_ctx *ctx, pcr_engine_stats *out);
/* Measures the device's L2 read bandwidth (GB/s): a kernel reads an
 * L2-resident buffer of `bytes` (1..96 MiB; 32 MiB fits the 126 MB L2 of a
 * B200 with room to spare) `reps` times with loads that bypass L1.  The
 * denominator of the BVH-fetch roofline's L2 fraction: a mesh's nodes and
 * triangles (a few MB to ~60 MB) stay in L2 while rays traverse it.  No
 * reference counterpart (measurement only). */
pcr_status pcr_l2_bandwidth(pcr_ctx *ctx, int64_t bytes, int32_t reps, double *gbs);
pcr_status pcr_engine_stats_reset(pcr_ctx *ctx);
/* Picks queue capacity (512K..16M paths in flight), block size, chunk and
 * refill cadence by timing short trial batches of the given requests; stores
 * the choice (and the cache file when one was given).  The path and shadow
 * queues grow with the capacity: about 10 GB at 4M and 40 GB at 16M with up
 * to 8 shadow rays per hit, more when requests ask for more (S slots per
 * path slot); capacities whose path slots times the sample's shadow rays per
 * hit reach 2^31 shadow records are not tried. */
pcr_status pcr_autotune(pcr_ctx *ctx, const pcr_scene_id *scenes, const pcr_render_desc *descs,
                        int32_t n, int32_t *chosen /* 4 ints, may be NULL */);

/* ------------------------------------------------------------- kernels for parity
 * Closest hit for n rays (origin3 dir3 floats each) against a scene, the
 * reference's sceneIntersect (code/Renderer.cpp:891-949): writes material
 * index (-1 miss), primitive code (kind<<30 | id; kind 1 sphere, 2 plane,
 * 3 triangle id from triangle_ids) and t.  Host buffers. */
pcr_status pcr_trace_closest(pcr_ctx *ctx, pcr_scene_id scene, const float *rays, int64_t n,
                             int32_t *mat, int32_t *prim, float *t);
/* Bvh::intersect over the triangles only (code/Bvh/Bvh.cpp:353-444), with
 * per-ray counts of internal nodes visited and triangles tested (may be NULL). */
pcr_status pcr_trace_bvh(pcr_ctx *ctx, pcr_scene_id scene, const float *rays, int64_t n,
                         int32_t *tri_id, float *t, int32_t *counts);
/* Reinhard / ACES tone map and 8-bit quantisation of a linear sRGB image
 * (code/Renderer.cpp:365-382), with the bilateral denoise when asked; the
 * last step of a render split across GPUs. */
pcr_status pcr_tonemap(pcr_ctx *ctx, const float *hdr, int32_t width, int32_t height, int32_t aces, int32_t denoise,
                       uint8_t *rgb8_out);

/* ------------------------------------------------------------- router
 * Request router over several contexts, typically one per GPU of a node
 * (the scale-out of the serving path; the reference renders on one device
 * and has no counterpart).  The router borrows the contexts (they must
 * outlive it), replicates scenes into each one's scene cache, and sends
 * each request to the context with the fewest paths outstanding (submitted
 * and not yet fetched).  Requests are independent, so there is no data
 * exchange between devices; a request's image is the same whichever
 * context renders it.  Tickets name (context, request).  Thread-safe. */
typedef struct pcr_router pcr_router;
pcr_status pcr_router_create(pcr_router **out, pcr_ctx *const *ctxs, int32_t n);
pcr_status pcr_router_destroy(pcr_router *r);
pcr_status pcr_router_scene_load_json(pcr_router *r, const char *path, const char *data_root,
                                      const char *lut_path, pcr_scene_id *out);
pcr_status pcr_router_serve_start(pcr_router *r);
pcr_status pcr_router_serve_stop(pcr_router *r);
pcr_status pcr_router_submit(pcr_router *r, pcr_scene_id scene, const pcr_render_desc *desc, int64_t *ticket);
pcr_status pcr_router_wait(pcr_router *r, int64_t ticket, int64_t timeout_ms);
pcr_status pcr_router_fetch(pcr_router *r, int64_t ticket, float *hdr_out, uint8_t *rgb8_out,
                            pcr_render_stats *stats);
/* per-context paths outstanding (n entries) and requests routed (n entries) */
pcr_status pcr_router_load(pcr_router *r, int64_t *outstanding_paths, int64_t *routed);

/* The shadow test of one light sample (code/Renderer.cpp:852-860) on caller
 * rays: rays = n x (origin xyz, unit direction xyz), light_dist2 = squared
 * distance to the light sample; blocked[i] = 1 when the closest hit is
 * non-emissive and closer than light_dist2 - 1e-3 (compared in double). */
pcr_status pcr_trace_shadow(pcr_ctx *ctx, pcr_scene_id scene, const float *rays, const float *light_dist2,
                            int64_t n, int32_t *blocked);
/* Bvh::build (code/Bvh/Bvh.cpp:122-325) on the context's device: the binary
 * SAH tree over tris[0..n) in the reference's depth-first layout, equal bit
 * for bit to the host builder's, and order_out[i] = index in `tris` of the
 * triangle at leaf position i (the reference permutes its triangle vector in
 * place; tris here is left as it is).  nodes_out holds max_nodes entries
 * (2n - 1 always suffices); *n_nodes receives the count.  Synchronous.
 * pcr_scene_upload runs this builder when the descriptor has no BVH. */
pcr_status pcr_bvh_build(pcr_ctx *ctx, const pcr_triangle *tris, int32_t n, pcr_bvh_node *nodes_out,
                         int32_t max_nodes, int32_t *n_nodes, int32_t *order_out);
/* Device evaluations of the FP32 stage functions on a wavelength / colour grid:
 * what 0 sigmoid fit at lambda (fit=4 floats) | 1 tabulated spectrum (61) |
 * 2 CIE xbar/ybar/zbar (3 out) | 3 singleLambdaXYZ(lambda, in[i]) (3 out) |
 * 4 XYZ->linear sRGB (3 in/out) | 5 Reinhard (3) | 6 ACES (3) | 7 8-bit quantise (3) |
 * 8 singleLambdaXYZ(lambda, in[i]) as the hot path forms it (3 out): the
 * interpolated colour-matching table that raygen reads, times the radiance
 * (code/Includes/CIE.h:140-159). */
pcr_status pcr_eval_stage(pcr_ctx *ctx, int32_t what, const float *params, const float *in,
                          int64_t n, float *out);

#ifdef __cplusplus
}
#endif
#endif
