// Device-resident data layout of the wavefront path tracer (HBM).
//
// Scene cache entries, the request table, the two path queues and the
// shadow-ray queue.  Everything the kernels read per ray is packed into
// 16-byte words so one thread issues 128-bit loads (LDG.128).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pcr {

constexpr int kSpecN = 61;          // 400..700 nm at 5 nm (code/Includes/Spectrum.h:167-170)
constexpr int kMaxActive = 1024;    // request slots in flight at once
constexpr int kMaxShadow = 64;      // shadow rays per diffuse vertex the kernels accept
constexpr int kStackSize = 64;      // BVH4 traversal stack entries per ray
constexpr int kMaxEmitPrims = 4;    // emissive spheres / planes listed per scene

// Primitive code in a hit record: kind in the top two bits.
constexpr uint32_t kPrimNone = 0u;
constexpr uint32_t kPrimSphere = 1u << 30;
constexpr uint32_t kPrimPlane = 2u << 30;
constexpr uint32_t kPrimTri = 3u << 30;
constexpr uint32_t kPrimKindMask = 3u << 30;
constexpr uint32_t kPrimIndexMask = (1u << 30) - 1u;

// Material flags
constexpr int kMatEmissive = 1, kMatMetallic = 2, kMatTransparent = 4, kMatTabA = 8, kMatTabE = 16;

// 592-byte material record (code/Includes/Material.h:8-101 fields used per bounce).
struct alignas(16) DMaterial {
    int flags;
    float ior, cauchyB, albedo_max;
    float4 albedo;      // rgb in xyz
    float4 emissive;    // rgb in xyz
    float4 afit, efit;  // c0 c1 c2 scale
    float tabA[64];
    float tabE[64];
};

// Parallelogram (code/Includes/Plane.h): 4 x 16 B.
struct alignas(16) DPlane {
    float4 o_mat;   // origin, matIdx (bits)
    float4 n_emit;  // unit normal, 1 when the plane's material is emissive (else 0)
    float4 u_uu;    // u, dot(u,u)
    float4 v_vv;    // v, dot(v,v)
};

struct alignas(16) DSphere {
    float4 c_r;     // centre, radius
    int4 mat;       // matIdx, 1 when the material is emissive (else 0), pad
};

// Triangle for Moller-Trumbore (code/Includes/Triangle.h:53-92): v0, e1 = v1-v0,
// e2 = v2-v0 computed on the host with the same float subtraction the
// reference does per test.  3 x 16 B.
struct alignas(16) DTri {
    float4 v0_id;     // v0, external id (bits)
    float4 e1_mat;    // e1, matIdx (bits)
    float4 e2_flags;  // e2, smooth flag (bits)
};

// 4-wide BVH node collapsed from the reference's binary SAH tree; child
// boxes are the binary nodes' boxes verbatim.  8 x 16 B = 128 B.
struct alignas(16) DNode4 {
    float4 lox, hix, loy, hiy, loz, hiz;
    int4 child;   // >= 0: internal node index; leaf: 0x80000000 | count<<24 | first; empty slot: 0x80000000
    int4 valid;   // 1 for a used slot, 0 for empty
};

struct alignas(16) DLight {
    int kind;           // 0 plane, 1 triangle set
    float total_area;
    int tri_offset, tri_count;
    float4 o_mat, u, v, n;  // plane
};

struct DScene {
    const DPlane* planes;
    const DSphere* spheres;
    const DNode4* nodes;
    const DTri* tris;
    const float4* tri_n;      // 3 per triangle (n0 n1 n2), smooth shading
    const float4* tri_flatn;  // 1 per triangle
    const DLight* lights;
    const DTri* light_tris;
    const float4* light_flatn;
    const float* light_cum;
    // Plane groups: runs of consecutive planes (a box's six faces) behind one
    // conservative bounding-box test.  2 words per group: (lo, first plane),
    // (hi, plane count); a group of one plane has no box test.
    const float4* pgroups;
    // The non-emissive planes again, grouped the same way, for the shadow
    // query (which tests emissive planes separately and needs no tie order).
    const DPlane* splanes;
    const float4* sgroups;
    int n_planes, n_spheres, n_nodes, n_tris, n_lights, mat_base, n_mats, n_pgroups;
    int n_sgroups;
    int emissive_tris;        // 1 when any triangle's material is emissive
    // The scene's only emissive material (scene-local index) when it has
    // exactly one and every light uses it, else -1.  Spectral paths of such
    // a scene carry emission x XYZ weight per wavelength instead of the
    // weight alone.
    int emit_mat;
    // Emissive spheres and planes (indices), for the shadow query's first
    // pass; n_emit_* = -1 when a scene has more than kMaxEmitPrims of a kind.
    int n_emit_spheres, n_emit_planes;
    int emit_spheres[kMaxEmitPrims], emit_planes[kMaxEmitPrims];
    float total_light_area;
};

// Request flags
constexpr int kReqSpectral = 1, kReqMIS = 2, kReqRussian = 4, kReqStratified = 8, kReqAdaptive = 16,
              kReqTerminate = 32, kReqCancelled = 64;

struct DRequest {
    int scene, width, height, depth;
    int paths_per_pixel;      // spp * aa
    int spp, aa, shadow, flags, hero, strata;
    float cam_x, cam_y, cam_z, scale, aspect;
    uint32_t seed_lo, seed_hi;
    long long total;          // width * height * paths_per_pixel (adaptive: paths issued through this round)
    double* accum;            // width * height * 3
    // Adaptive sampling (kReqAdaptive): the aa samples run as rounds; round
    // r traces spp paths for each pixel still in act[r & 1].  Per pixel the
    // round's mean enters a Welford mean / M2 (welford[2p] = mean, taken;
    // welford[2p+1] = M2); converged or finished pixels leave the list and
    // their final mean goes to accum.
    int* act[2];
    float4* welford;
    long long round_base;     // paths issued before this round
    int round;
    // sample range [sample0, sample0 + local_spp) of each aa round (a render
    // split across GPUs); paths_per_pixel = local_spp * aa
    int sample0, local_spp;
};

// Path state, structure of arrays, one entry per queued path.
struct PathQueue {
    float4* o;     // origin, hero lambda
    float4* d;     // direction, meta (bits): bounce | fork<<8 | single<<11 | n<<12
    float4* tp;    // throughput per channel
    int4* id;      // request slot, pixel, sample, scene (copied by continuations and forks)
    // XYZ weight of each carried wavelength, cmf(lambda_k) * 300/yBarIntegral / N
    // (spectral paths only): w[0] = x0 y0 z0 x1, w[1] = y1 z1 x2 y2, w[2] = z2 x3 y3 z3.
    // Computed once at raygen; a path's wavelengths never change.  In a scene
    // with one emissive material (DScene::emit_mat >= 0) each weight is
    // multiplied by that material's emission at the wavelength.
    float4* w[3];
};

struct ShadowQueue {
    float4* o;     // origin, lightDist2
    float4* d;     // direction, pixel (bits)
    float4* c;     // contribution (XYZ or RGB), request slot | scene << 16 (bits)
};

struct Counters {
    int queue_n[2];
    int shadow_n;
    int new_n;
    int new_base;
    int iter;
    int status;           // non-zero: a kernel reported an error
    int idle;             // 1 when no request has work left
    int n_rounds;         // adaptive requests whose round ended this iteration (k_status -> k_round)
    unsigned long long rays, shadow_rays, paths;
};

// Device view of the engine, passed by value to every kernel.
struct EngineView {
    const DScene* scenes;
    const DMaterial* mats;
    const DRequest* reqs;
    unsigned long long* issued;      // per slot
    long long* outstanding;          // per slot
    int* give;                       // per active position: paths this iteration
    int* give_base;                  // per active position: exclusive prefix
    int* active;                     // active slot list (admission order)
    int* n_active;
    int* done_flag;                  // per slot: 1 once finished
    unsigned long long* t_first;     // per slot: globaltimer at first issue
    unsigned long long* t_done;      // per slot: globaltimer at completion
    Counters* cnt;
    PathQueue q[2];
    float4* hit;
    ShadowQueue sq;
    long long* give_start;           // per active position: first path index issued
    int shadow_cap;                  // shadow-queue entries
    int queue_cap;                   // entries per path queue
    int n_mats;
    int* round_state;                // per slot: 1 while an adaptive round's per-pixel step is pending
    int* round_cnt;                  // per slot: pixels kept for the next adaptive round
    int* round_list;                 // slots of Counters::n_rounds
    const float4* cmf_table;         // CIE colour-matching functions at fine spacing (raygen)
};

}  // namespace pcr
