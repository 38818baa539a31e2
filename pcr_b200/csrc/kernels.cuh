// Wavefront stage kernels.  One iteration of the persistent wavefront is
//   schedule -> regen -> extend -> shade -> shadow -> status
// over the current path queue; shade writes surviving paths into the other
// queue.  Every kernel is a grid-stride loop over a device-side count, so
// a whole iteration (and several in a row) can be captured in one CUDA
// graph with no host round trip.  No kernel waits on another block or on
// the host: there is no spin anywhere.
#pragma once

#include <cooperative_groups.h>
#include <cooperative_groups/scan.h>
#include <cub/block/block_scan.cuh>

#include "device.cuh"

namespace pcr {

struct EngineParams {
    int fill;          // refill target (paths in flight)
    int chunk;         // per-request issue chunk per refill
    int regen_every;   // refill cadence in iterations
    int plain;         // 1: refill only when the queue is empty (pass-wise)
};

// ------------------------------------------------------------------ schedule
// One block.  Decides how many new camera paths each active request gets
// this iteration: first up to `chunk` each (round-robin fairness), then the
// remaining free slots oldest-first.
constexpr int kSchedThreads = 1024;

__global__ void __launch_bounds__(kSchedThreads) k_schedule(EngineView E, const EngineParams* P, int cur)
{
    typedef cub::BlockScan<long long, kSchedThreads> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ long long s_total;
    Counters* C = E.cnt;
    const int tid = threadIdx.x;
    const int n_act = *E.n_active;
    int qn = C->queue_n[cur];
    if (qn > E.queue_cap) {  // never expected: shade guards every append
        qn = E.queue_cap;
        if (tid == 0) atomicOr(&C->status, 4);
    }
    const EngineParams p = *P;
    long long free_slots = (long long)p.fill - qn;
    if (free_slots < 0) free_slots = 0;
    if (p.plain && qn > 0) free_slots = 0;
    if (p.regen_every > 1 && (C->iter % p.regen_every) != 0 && qn > 0) free_slots = 0;

    int slot = -1;
    long long rem = 0;
    if (tid < n_act) {
        slot = E.active[tid];
        if (E.round_state[slot] == 1) {
            // an adaptive round ended last iteration and k_round kept
            // round_cnt pixels: open the next round, or finish the request
            DRequest& R = const_cast<DRequest&>(E.reqs[slot]);
            // a cancelled request opens no further round
            const int kept = (R.flags & kReqCancelled) ? 0 : E.round_cnt[slot];
            E.round_cnt[slot] = 0;
            E.round_state[slot] = 0;
            R.round_base = R.total;
            R.round += 1;
            R.total += (long long)kept * R.spp;
            if (kept == 0) {
                unsigned long long t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                E.done_flag[slot] = 1;
                E.t_done[slot] = t;
            }
        }
        rem = E.reqs[slot].total - (long long)E.issued[slot];
        if (rem < 0) rem = 0;
    }
    // pass 1: up to chunk each, in active order
    long long w1 = rem < (long long)p.chunk ? rem : (long long)p.chunk;
    long long ex1, tot1;
    Scan(tmp).ExclusiveSum(w1, ex1, tot1);
    __syncthreads();
    long long g1 = free_slots - ex1;
    g1 = g1 < 0 ? 0 : (g1 > w1 ? w1 : g1);
    long long left = free_slots - (tot1 < free_slots ? tot1 : free_slots);
    long long rem2 = rem - g1;
    long long ex2, tot2;
    Scan(tmp).ExclusiveSum(rem2, ex2, tot2);
    __syncthreads();
    long long g2 = left - ex2;
    g2 = g2 < 0 ? 0 : (g2 > rem2 ? rem2 : g2);
    long long g = g1 + g2;
    long long exg, totg;
    Scan(tmp).ExclusiveSum(g, exg, totg);
    if (tid < n_act) {
        E.give[tid] = (int)g;
        E.give_base[tid] = (int)exg;
        E.give_start[tid] = (long long)E.issued[slot];
        if (g > 0) {
            if (E.issued[slot] == 0ull) {
                unsigned long long t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                E.t_first[slot] = t;
            }
            E.issued[slot] += (unsigned long long)g;
            E.outstanding[slot] += g;
        }
    }
    if (tid == 0) s_total = totg;
    __syncthreads();
    if (tid == 0) {
        C->n_rounds = 0;  // k_round of the last iteration has read the list
        C->new_base = qn;
        C->new_n = (int)s_total;
        C->queue_n[cur] = qn + (int)s_total;
        C->queue_n[cur ^ 1] = 0;
        C->shadow_n = 0;
        C->paths += (unsigned long long)s_total;
    }
}

// ------------------------------------------------------------------ spectral weights
// Per-channel XYZ weights of a path's wavelengths: w_k = cmf(lam_k) *
// (700-400)/yBarIntegral / N, so the pixel contribution of per-channel
// radiance c is sum_k c_k w_k = sum_k singleLambdaXYZ(lam_k, c_k) / N
// (code/Renderer.cpp:254-257, code/Includes/CIE.h:140-159).  Computed once
// per path at raygen; RGB mode passes the channels through.
struct XyzWeights {
    float3 w[4];
};

// The colour-matching functions tabulated every 1/kCmfPerNm nm over
// [kCmfLo, kCmfHi] (380..720 nm, wider than the 400..700 nm the hero
// wavelengths span) and read back with linear interpolation, so raygen
// evaluates four wavelengths per path without 28 exponentials.  Entries are
// the Wyman-Sloan-Shirley lobes (code/Includes/CIE.h:27-53, their float
// constants) evaluated in double at the exact grid wavelength, then rounded
// once; the lookup's fraction comes from one fused multiply-add of the exact
// difference lambda - kCmfLo, so the only error left is the interpolation's,
// below 2e-6 of each value.  In [kCmfXLo, kCmfXHi] x-bar's lobes cancel and
// the reference's own float evaluation (singleLambdaXYZ) carries rounding of
// up to 3e-5 of the result, which no smooth table follows; there x-bar is
// evaluated with the reference's float operations instead (xyz_weights).  Against the
// reference the result then stays below 1e-5 relative (1e-7 absolute near
// zero) over 380..720 nm.
constexpr float kCmfLo = 380.f, kCmfHi = 720.f, kCmfXLo = 495.f, kCmfXHi = 508.f;
constexpr int kCmfPerNm = 80;
constexpr int kCmfEntries = 340 * kCmfPerNm + 1;  // (kCmfHi - kCmfLo) * kCmfPerNm + 1
__device__ __forceinline__ double wyman_d(double l, float mu, float s1, float s2)
{
    const double t = (l < (double)mu) ? (l - (double)mu) * (double)s1 : (l - (double)mu) * (double)s2;
    return exp(-0.5 * t * t);
}
__global__ void k_cmf_table(float4* table)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kCmfEntries; i += gridDim.x * blockDim.x) {
        const double l = (double)kCmfLo + (double)i / (double)kCmfPerNm;
        const double x = (double)0.362f * wyman_d(l, 442.0f, 0.0624f, 0.0374f) +
                         (double)1.056f * wyman_d(l, 599.8f, 0.0264f, 0.0323f) -
                         (double)0.065f * wyman_d(l, 501.1f, 0.0490f, 0.0382f);
        const double y = (double)0.821f * wyman_d(l, 568.8f, 0.0213f, 0.0247f) +
                         (double)0.286f * wyman_d(l, 530.9f, 0.0613f, 0.0322f);
        const double z = (double)1.217f * wyman_d(l, 437.0f, 0.0845f, 0.0278f) +
                         (double)0.681f * wyman_d(l, 459.0f, 0.0385f, 0.0725f);
        table[i] = make_float4((float)x, (float)y, (float)z, 0.f);
    }
}
__device__ __forceinline__ float3 cmf_lut(const float4* __restrict__ table, float l)
{
    // l - kCmfLo is exact for l in [190, 760] (Sterbenz); fmaf rounds
    // d * kCmfPerNm - i once, so f carries no error from the product
    const float d = l - kCmfLo;
    const int i = min(max((int)floorf(d * (float)kCmfPerNm), 0), kCmfEntries - 2);
    const float f = fmaf(d, (float)kCmfPerNm, -(float)i);
    const float4 a = table[i], b = table[i + 1];
    return make_float3(a.x + (b.x - a.x) * f, a.y + (b.y - a.y) * f, a.z + (b.z - a.z) * f);
}
__device__ __forceinline__ bool in_cmf_x_window(float l) { return l >= kCmfXLo && l <= kCmfXHi; }

__device__ __noinline__ XyzWeights xyz_weights(bool spectral, const float* lam, int nch, float wN, float xyz_scale,
                                               const float4* cmf_table)
{
    XyzWeights W;
    if (!spectral) {
        W.w[0] = make_float3(1.f, 0.f, 0.f);
        W.w[1] = make_float3(0.f, 1.f, 0.f);
        W.w[2] = make_float3(0.f, 0.f, 1.f);
        W.w[3] = make_float3(0.f, 0.f, 0.f);
        return W;
    }
    const float s = xyz_scale * wN;
    int kx = -1;  // the wavelength in x-bar's exact window, if any
    for (int k = 0; k < 4; k++) {
        if (k < nch) {
            float3 c = cmf_lut(cmf_table, lam[k]);
            if (in_cmf_x_window(lam[k])) kx = k;
            W.w[k] = make_float3(c.x * s, c.y * s, c.z * s);
        } else {
            W.w[k] = make_float3(0.f, 0.f, 0.f);
        }
    }
    // a path's wavelengths lie 300/N nm apart (75 at N = 4) and the window is
    // 13 nm wide, so at most one of them is in it: one exact evaluation per
    // lane, outside the loop, keeps a warp from running it up to four times
    if (kx >= 0) {
        const float x = cmf_x(lam[kx]) * s;
        if (kx == 0) W.w[0].x = x;
        else if (kx == 1) W.w[1].x = x;
        else if (kx == 2) W.w[2].x = x;
        else W.w[3].x = x;
    }
    return W;
}
// Packed layout of the weights in the path queue (see PathQueue::w).
__device__ __forceinline__ void store_weights(const PathQueue& Q, int pos, const XyzWeights& W)
{
    Q.w[0][pos] = make_float4(W.w[0].x, W.w[0].y, W.w[0].z, W.w[1].x);
    Q.w[1][pos] = make_float4(W.w[1].y, W.w[1].z, W.w[2].x, W.w[2].y);
    Q.w[2][pos] = make_float4(W.w[2].z, W.w[3].x, W.w[3].y, W.w[3].z);
}
__device__ __forceinline__ XyzWeights load_weights(const PathQueue& Q, int pos)
{
    const float4 a = Q.w[0][pos], b = Q.w[1][pos], c = Q.w[2][pos];
    XyzWeights W;
    W.w[0] = make_float3(a.x, a.y, a.z);
    W.w[1] = make_float3(a.w, b.x, b.y);
    W.w[2] = make_float3(b.z, b.w, c.x);
    W.w[3] = make_float3(c.y, c.z, c.w);
    return W;
}
__device__ __forceinline__ XyzWeights rgb_weights()
{
    XyzWeights W;
    W.w[0] = make_float3(1.f, 0.f, 0.f);
    W.w[1] = make_float3(0.f, 1.f, 0.f);
    W.w[2] = make_float3(0.f, 0.f, 1.f);
    W.w[3] = make_float3(0.f, 0.f, 0.f);
    return W;
}

__device__ __forceinline__ float3 apply_xyz(const XyzWeights& W, float4 c)
{
    float3 s = make_float3(0.f, 0.f, 0.f);
    s.x += c.x * W.w[0].x; s.y += c.x * W.w[0].y; s.z += c.x * W.w[0].z;
    s.x += c.y * W.w[1].x; s.y += c.y * W.w[1].y; s.z += c.y * W.w[1].z;
    s.x += c.z * W.w[2].x; s.y += c.z * W.w[2].y; s.z += c.z * W.w[2].z;
    s.x += c.w * W.w[3].x; s.y += c.w * W.w[3].y; s.z += c.w * W.w[3].z;
    return s;
}

__device__ __forceinline__ float comp4(float4 v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }
__device__ __forceinline__ float4 mul4(float4 a, float4 b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
__device__ __forceinline__ float4 rgb4(float4 c) { return make_float4(c.x, c.y, c.z, 0.f); }

// A material spectrum at the four carried wavelengths (Material::albedoAt /
// emissiveAt, code/Includes/Material.h:92-101).  Kept out of line: one copy
// of the sigmoid / table code instead of one per call site keeps k_shade's
// instruction footprint small.
__device__ __noinline__ float4 spec4(const DMaterial& m, int emissive, float4 lam)
{
    const bool tab = (m.flags & (emissive ? kMatTabE : kMatTabA)) != 0;
    const float* table = emissive ? m.tabE : m.tabA;
    const float4 fit = emissive ? m.efit : m.afit;
    float v[4];
    const float l[4] = {lam.x, lam.y, lam.z, lam.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float x = tab ? spectrum_lerp(table, l[k]) : sigmoid_fit(fit, l[k]);
        if (!emissive && !tab && x > 1.f) x = 1.f;
        v[k] = x;
    }
    return make_float4(v[0], v[1], v[2], v[3]);
}


// ------------------------------------------------------------------ regen
// Camera rays for the new paths (code/Renderer.cpp:190-239): pixel centre,
// jitter when aa > 1, hero wavelength and its stratified companions.

__global__ void k_regen(EngineView E, int cur, float xyz_scale)
{
    __shared__ int s_base[kMaxActive];
    __shared__ int s_give[kMaxActive];
    __shared__ int s_slot[kMaxActive];
    __shared__ long long s_start[kMaxActive];
    const Counters* C = E.cnt;
    const int n_act = *E.n_active;
    for (int i = threadIdx.x; i < n_act; i += blockDim.x) {
        s_base[i] = E.give_base[i];
        s_give[i] = E.give[i];
        s_slot[i] = E.active[i];
        s_start[i] = E.give_start[i];
    }
    __syncthreads();
    const int n_new = C->new_n, base = C->new_base;
    const PathQueue Q = E.q[cur];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += gridDim.x * blockDim.x) {
        int lo = 0, hi = n_act - 1;
        while (lo < hi) {  // last r with base[r] <= i and give[r] > 0
            int mid = (lo + hi + 1) >> 1;
            if (s_base[mid] <= i) lo = mid; else hi = mid - 1;
        }
        while (lo > 0 && (s_give[lo] == 0 || s_base[lo] > i)) lo--;
        const int slot = s_slot[lo];
        const DRequest& R = E.reqs[slot];
        const long long path = s_start[lo] + (i - s_base[lo]);
        uint32_t pixel, sample;
        if (R.flags & kReqAdaptive) {
            // round r: spp paths for each pixel still in the round's list;
            // sample numbers r*spp.. as in the non-adaptive order
            const long long q = path - R.round_base;
            pixel = (uint32_t)R.act[R.round & 1][q / R.spp];
            sample = (uint32_t)(R.round * R.spp + (int)(q % R.spp));
        } else {
            pixel = (uint32_t)(path / R.paths_per_pixel);
            const int q = (int)(path % R.paths_per_pixel);  // local sample
            sample = (uint32_t)((q / R.local_spp) * R.spp + R.sample0 + q % R.local_spp);
        }
        const int px = (int)(pixel % (uint32_t)R.width), py = (int)(pixel / (uint32_t)R.width);
        float jx = 0.f, jy = 0.f;
        if (R.aa > 1) {
            float4 j = rand4(R, pixel, sample / (uint32_t)R.spp, 0, 254u, 0);
            jx = j.x - 0.5f;
            jy = j.y - 0.5f;
        }
        float x = ((2 * (px + 0.5f + jx) / (float)R.width) - 1) * R.scale * R.aspect;
        float y = -((2 * (py + 0.5f + jy) / (float)R.height) - 1) * R.scale;
        float inv = rsqrtf(x * x + y * y + 1.f);
        float3 d = make_float3(x * inv, y * inv, -inv);
        float lambda0 = 0.f;
        int nch = 4;
        const int pos = base + i;
        if (R.flags & kReqSpectral) {
            float4 u = rand4(R, pixel, sample, 0, 255u, 0);
            lambda0 = 400.f + u.x * 300.f;
            nch = R.hero;
            // hero wavelength and its stratified companions (code/Renderer.cpp:227-239)
            float lam[4];
            const float span = 300.f, stride_l = span / (float)nch;
            lam[0] = lambda0;
#pragma unroll
            for (int k = 1; k < 4; k++) {
                float l = lam[0] + stride_l * k;
                if (l > 700.f) l -= span;
                lam[k] = k < nch ? l : lam[0];
            }
            XyzWeights W = xyz_weights(true, lam, nch, 1.f / (float)nch, xyz_scale, E.cmf_table);
            const DScene& S = E.scenes[R.scene];
            if (S.emit_mat >= 0) {
                // emission of the scene's only emissive material, folded in
                const float4 e = spec4(E.mats[S.mat_base + S.emit_mat], 1, make_float4(lam[0], lam[1], lam[2], lam[3]));
                W.w[0] = f3mul(W.w[0], e.x);
                W.w[1] = f3mul(W.w[1], e.y);
                W.w[2] = f3mul(W.w[2], e.z);
                W.w[3] = f3mul(W.w[3], e.w);
            }
            store_weights(Q, pos, W);
        }
        Q.o[pos] = make_float4(R.cam_x, R.cam_y, R.cam_z, lambda0);
        Q.d[pos] = make_float4(d.x, d.y, d.z, __int_as_float(nch << 12));
        Q.tp[pos] = make_float4(1.f, 1.f, 1.f, 1.f);
        Q.id[pos] = make_int4(slot, (int)pixel, (int)sample, R.scene);
    }
}

// Brings the next grid-stride record's line into L2 while this one is
// processed (no register cost; the record is read again when its turn comes).
__device__ __forceinline__ void prefetch_l2(const void* p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// ------------------------------------------------------------------ extend
// The trace kernels are latency-bound (dependent IEEE arithmetic, scattered
// scene loads): their register budget is capped at 64 per thread (blocks of
// up to 256, 4 per SM) so 32 or more warps stay resident per SM.
#ifndef PCR_TRACE_MIN_BLOCKS
#define PCR_TRACE_MIN_BLOCKS 4
#endif
#ifndef PCR_SHADOW_MIN_BLOCKS
#define PCR_SHADOW_MIN_BLOCKS PCR_TRACE_MIN_BLOCKS
#endif
constexpr int kTraceMaxBlock = 256, kTraceMinBlocks = PCR_TRACE_MIN_BLOCKS, kShadowMinBlocks = PCR_SHADOW_MIN_BLOCKS;

// Closest hit for every queued path (trace_closest).
__global__ void __launch_bounds__(kTraceMaxBlock, kTraceMinBlocks) k_extend(EngineView E, int cur)
{
    const Counters* C = E.cnt;
    const int n = min(C->queue_n[cur], E.queue_cap);
    const PathQueue Q = E.q[cur];
    unsigned long long mine = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int nx = i + gridDim.x * blockDim.x;
        if (nx < n) { prefetch_l2(Q.o + nx); prefetch_l2(Q.d + nx); prefetch_l2(Q.id + nx); }
        const DScene& S = E.scenes[Q.id[i].w];
        float4 o = Q.o[i], d = Q.d[i];
        float t = FLT_MAX, u = 0.f, v = 0.f;
        uint32_t prim = scene_closest(S, xyz(o), xyz(d), FLT_MAX, t, u, v);
        E.hit[i] = make_float4(t, __uint_as_float(prim), u, v);
        mine++;
    }
    for (int off = 16; off > 0; off >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, off);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&E.cnt->rays, mine);
}

// ------------------------------------------------------------------ helpers

// Adds one sample's XYZ to a pixel's FP64 accumulator (device memory) with
// global-space reductions, which return nothing to the thread.
__device__ __forceinline__ void red_add(double* a, double v)
{
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(__cvta_generic_to_global(a)), "d"(v) : "memory");
}
__device__ __forceinline__ void add_xyz(double* acc, float3 c)
{
    red_add(acc + 0, (double)c.x);
    red_add(acc + 1, (double)c.y);
    red_add(acc + 2, (double)c.z);
}

// ------------------------------------------------------------------ shade
// Appends `count` records for the calling lane among the lanes that reach the
// call together (divergent code): one atomic per coalesced group.
__device__ __forceinline__ int group_append(int* counter, int count)
{
    namespace cg = cooperative_groups;
    cg::coalesced_group g = cg::coalesced_threads();
    const int ex = cg::exclusive_scan(g, count);
    const int tot = g.shfl(ex + count, g.size() - 1);
    int base = 0;
    if (g.thread_rank() == 0 && tot) base = atomicAdd(counter, tot);
    return g.shfl(base, 0) + ex;
}

// k_shade's block shape is fixed: its register budget (launch bounds) is
// set for 128-thread blocks, PCR_SHADE_MIN_BLOCKS per SM.
#ifndef PCR_SHADE_MIN_BLOCKS
#define PCR_SHADE_MIN_BLOCKS 5
#endif
constexpr int kShadeBlock = 128;

// Per-path shading of the hit found by k_extend (code/Renderer.cpp:656-889
// with samples = 1, the GPU's paths-per-pixel estimator): emission,
// mirror, dielectric (with the 4-way hero fork at dispersive glass),
// diffuse direct lighting via explicit shadow rays, Russian roulette and the
// cosine-hemisphere continuation.  Materials are staged in shared memory.
//
// A diffuse vertex reserves R.shadow shadow records with one append; samples
// whose geometry term is zero are written as skip records (lightDist2 < 0).
// The spectral product albedo * emission * XYZ weight is formed once per
// vertex and light material, so each shadow sample only scales it by its
// geometry term.
//
// Per-channel values live in float4 registers (no per-thread arrays, so no
// local memory); channels a path does not carry have zero XYZ weight, so
// they are evaluated but contribute nothing.
__global__ void __launch_bounds__(kShadeBlock, PCR_SHADE_MIN_BLOCKS) k_shade(EngineView E, int cur, int smem_mats)
{
    extern __shared__ DMaterial s_mat[];
    const DMaterial* M = E.mats;
    if (smem_mats) {
        const int words = E.n_mats * (int)(sizeof(DMaterial) / 16);
        const float4* src = reinterpret_cast<const float4*>(E.mats);
        float4* dst = reinterpret_cast<float4*>(s_mat);
        for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
        __syncthreads();
        M = s_mat;
    }
    Counters* C = E.cnt;
    const int n = min(C->queue_n[cur], E.queue_cap);
    const PathQueue Q = E.q[cur];
    const PathQueue NQ = E.q[cur ^ 1];
    const ShadowQueue SQ = E.sq;
    const float inv_pi = 1.f / 3.14159274f;
    const int lane = threadIdx.x & 31;
    // block-uniform trip count: every thread of a block runs the same
    // iterations, so the block-wide append at the bottom sees all of them
    __shared__ int s_app[2][kShadeBlock / 32 + 1];
    __shared__ int s_shd[2][kShadeBlock / 32 + 1];
    int parity = 0;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int i = base + threadIdx.x;
        const bool live = i < n;
        int4 id = make_int4(0, 0, 0, 0);
        float4 o4 = make_float4(0, 0, 0, 0), d4 = o4, tp4 = o4, h = o4;
        if (i + stride < n) {
            const int nx = i + stride;
            prefetch_l2(Q.id + nx); prefetch_l2(Q.o + nx); prefetch_l2(Q.d + nx); prefetch_l2(Q.tp + nx);
            prefetch_l2(E.hit + nx);
            prefetch_l2(Q.w[0] + nx); prefetch_l2(Q.w[1] + nx); prefetch_l2(Q.w[2] + nx);
        }
        if (live) { id = Q.id[i]; o4 = Q.o[i]; d4 = Q.d[i]; tp4 = Q.tp[i]; h = E.hit[i]; }
        const int slot = id.x;
        const uint32_t prim = __float_as_uint(h.y);
        const int meta = __float_as_int(d4.w);
        const int bounce = meta & 0xFF, fork = (meta >> 8) & 7, single = (meta >> 11) & 1, nHero = (meta >> 12) & 7;
        bool cont = false;    // continue into the next queue
        int forked = 0;       // sub-paths written by a dispersive fork
        float3 no = make_float3(0, 0, 0), nd = no;
        float4 ntp = make_float4(0, 0, 0, 0);
        bool term = false;    // continues with its hero wavelength alone
        double* acc = nullptr;
        float3 emit_xyz = make_float3(0, 0, 0);
        bool emit = false;
        bool spec_path = false;

        // Shadow records: a diffuse vertex with a light in its scene writes
        // R.shadow of them.  They are reserved for the whole block at once
        // (one contiguous range, its warps in order), so k_shadow's warps
        // rarely straddle two blocks' records, which may belong to
        // different scenes.
        int nee = 0;
        bool mesh = false;  // casts over a BVH
        if (live && (prim & kPrimKindMask) != kPrimNone) {
            const DScene& S0 = E.scenes[id.w];
            if (S0.total_light_area > 0.f) {
                const uint32_t k0 = prim & kPrimKindMask, p0 = prim & kPrimIndexMask;
                const int mi0 = k0 == kPrimSphere ? S0.spheres[p0].mat.x
                              : k0 == kPrimPlane  ? __float_as_int(S0.planes[p0].o_mat.w)
                                                  : __float_as_int(S0.tris[p0].e1_mat.w);
                if (!(M[S0.mat_base + mi0].flags & (kMatEmissive | kMatMetallic | kMatTransparent))) {
                    nee = E.reqs[slot].shadow;
                    mesh = S0.n_nodes > 0;
                }
            }
        }
        int spos_block, sstride;
        {
            int ex = nee;  // inclusive scan across the warp
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, ex, off);
                if (lane >= off) ex += v;
            }
            int* sw = s_shd[parity];
            const int wid = threadIdx.x >> 5;
            if (lane == 31) sw[wid] = ex;
            __syncthreads();
            if (threadIdx.x == 0) {
                int tot = 0;
                for (int k = 0; k < kShadeBlock / 32; k++) { const int c = sw[k]; sw[k] = tot; tot += c; }
                sw[kShadeBlock / 32] = tot ? atomicAdd(&C->shadow_n, tot) : 0;
            }
            __syncthreads();
            const int wbase = sw[kShadeBlock / 32] + sw[wid];
            // Sample-major order inside the warp when its vertices all cast
            // the same number of shadow rays (one request, the usual case)
            // into scenes without a mesh: record s of the warp's k-th
            // casting lane sits at wbase + s * casters + k, so each sample's
            // stores are one contiguous run.  Otherwise each lane's records
            // are adjacent: over a BVH, the rays of one vertex then share a
            // k_shadow warp and walk mostly the same nodes.
            const unsigned cm = __ballot_sync(0xffffffffu, nee > 0);
            const unsigned hi = __reduce_max_sync(0xffffffffu, (unsigned)nee);
            const unsigned lo = __reduce_min_sync(0xffffffffu, nee > 0 ? (unsigned)nee : 0xffffffffu);
            if (hi == lo && !__any_sync(0xffffffffu, mesh)) {
                spos_block = wbase + __popc(cm & ((1u << lane) - 1u));
                sstride = __popc(cm);
            } else {
                spos_block = wbase + ex - nee;
                sstride = 1;
            }
        }

        if (live && (prim & kPrimKindMask) != kPrimNone) {
            const DRequest& R = E.reqs[slot];
            const DScene& S = E.scenes[id.w];
            const bool spectral = (R.flags & kReqSpectral) != 0;
            spec_path = spectral;
            // wavelengths carried by this path (code/Renderer.cpp:227-239)
            float4 lam4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (spectral) {
                const float l0 = o4.w;
                if (single) {
                    lam4 = make_float4(l0, l0, l0, l0);
                } else {
                    const float span = 300.f, stride_l = span / (float)nHero;
                    float l1 = l0 + stride_l * 1, l2 = l0 + stride_l * 2, l3 = l0 + stride_l * 3;
                    if (l1 > 700.f) l1 -= span;
                    if (l2 > 700.f) l2 -= span;
                    if (l3 > 700.f) l3 -= span;
                    lam4 = make_float4(l0, 1 < nHero ? l1 : l0, 2 < nHero ? l2 : l0, 3 < nHero ? l3 : l0);
                }
            }
            acc = R.accum + (size_t)id.y * 3;
            const float3 o = xyz(o4), d = xyz(d4);
            const float t = h.x;
            const float3 hit = make_float3(o.x + d.x * t, o.y + d.y * t, o.z + d.z * t);
            float3 N;
            int mi;
            const uint32_t kind = prim & kPrimKindMask, pidx = prim & kPrimIndexMask;
            if (kind == kPrimSphere) {
                const float4 cr = S.spheres[pidx].c_r;
                float3 v = make_float3(hit.x - cr.x, hit.y - cr.y, hit.z - cr.z);
                N = f3mul(v, rsqrtf(f3dot(v, v)));
                mi = S.spheres[pidx].mat.x;
            } else if (kind == kPrimPlane) {
                const float4 na = S.planes[pidx].n_emit;
                N = make_float3(na.x, na.y, na.z);
                mi = __float_as_int(S.planes[pidx].o_mat.w);
            } else {
                const DTri& tr = S.tris[pidx];
                mi = __float_as_int(tr.e1_mat.w);
                if (__float_as_int(tr.e2_flags.w) & 1) {
                    const float4 n0 = S.tri_n[pidx * 3], n1 = S.tri_n[pidx * 3 + 1], n2 = S.tri_n[pidx * 3 + 2];
                    const float w = 1.f - h.z - h.w;
                    float3 in = make_float3(n0.x * w + n1.x * h.z + n2.x * h.w, n0.y * w + n1.y * h.z + n2.y * h.w,
                                            n0.z * w + n1.z * h.z + n2.z * h.w);
                    N = f3mul(in, rsqrtf(f3dot(in, in)));
                } else {
                    N = xyz(S.tri_flatn[pidx]);
                }
            }
            const bool entering = f3dot(d, N) < 0.f;
            if (!entering) N = f3neg(N);
            const DMaterial& m = M[S.mat_base + mi];
            const bool last = bounce + 1 >= R.depth;
            if (m.flags & kMatEmissive) {
                // with emit_mat the carried weights already hold the emission
                const float4 c = !spectral ? mul4(tp4, rgb4(m.emissive))
                               : S.emit_mat >= 0 ? tp4 : mul4(tp4, spec4(m, 1, lam4));
                const XyzWeights W = spectral ? load_weights(Q, i) : rgb_weights();
                emit_xyz = apply_xyz(W, c);
                emit = true;
            } else if (m.flags & kMatMetallic) {
                if (!last) {
                    const float cosI = -f3dot(d, N);
                    nd = f3add(d, f3mul(N, 2.f * cosI));
                    no = f3add(hit, f3mul(N, 1e-3f));
                    ntp = mul4(tp4, spectral ? spec4(m, 0, lam4) : rgb4(m.albedo));
                    cont = true;
                }
            } else if (m.flags & kMatTransparent) {
                if (!last) {
                    const float cosI = -f3dot(d, N);
                    const bool dispersive = spectral && m.cauchyB != 0.f && !single && nHero > 1;
                    // fork: one sub-path per wavelength (code/Renderer.cpp:736-753);
                    // terminate: the hero wavelength's bounce alone
                    // (code/Gpu/Metal/MetalRenderer.mm:2143-2252)
                    const bool terminate = dispersive && (R.flags & kReqTerminate);
                    const bool disperse = dispersive && !terminate;
                    const int ways = disperse ? nHero : 1;
                    const float4 coins = rand4(R, (uint32_t)id.y, (uint32_t)id.z, (uint32_t)fork, (uint32_t)bounce, 63u);
                    const float4 alg = spectral ? spec4(m, 0, lam4) : rgb4(m.albedo);
                    int fpos = 0;
                    if (disperse) {
                        fpos = group_append(&C->queue_n[cur ^ 1], ways);
                        forked = ways;
                    }
                    for (int k = 0; k < ways; k++) {
                        const float lk = comp4(lam4, k);
                        float ior = m.ior;
                        if (spectral && m.cauchyB != 0.f && (dispersive || single))
                            ior = m.ior + m.cauchyB * 1e4f / (lk * lk);  // Optics::cauchyIor
                        // Optics::dielectricBounce (code/Includes/Optics.h:59-82)
                        const float n1 = entering ? 1.f : ior, n2 = entering ? ior : 1.f;
                        const float eta = n1 / n2;
                        const float sinT2 = eta * eta * (1.f - cosI * cosI);
                        const float u = comp4(coins, k);
                        float3 bd, bo;
                        bool refl = sinT2 >= 1.f;
                        if (!refl) {
                            float F0 = (n1 - n2) / (n1 + n2);
                            F0 *= F0;
                            const float F = F0 + (1.f - F0) * __powf(1.f - cosI, 5.f);
                            refl = u < F;
                        }
                        if (refl) {
                            bd = f3add(d, f3mul(N, 2.f * cosI));
                            bo = f3add(hit, f3mul(N, 1e-3f));
                        } else {
                            const float cosT = sqrtf(1.f - sinT2);
                            bd = f3add(f3mul(d, eta), f3mul(N, eta * cosI - cosT));
                            bo = f3sub(hit, f3mul(N, 1e-3f));
                        }
                        if (disperse) {
                            // sub-path k carries wavelength k alone (code/Renderer.cpp:736-753)
                            const int pos = fpos + k;
                            if (pos < E.queue_cap) {
                                const float ftp = comp4(tp4, k) * comp4(alg, k);
                                const int fm = (bounce + 1) | ((k + 1) << 8) | (1 << 11) | (nHero << 12);
                                NQ.o[pos] = make_float4(bo.x, bo.y, bo.z, lk);
                                NQ.d[pos] = make_float4(bd.x, bd.y, bd.z, __int_as_float(fm));
                                NQ.tp[pos] = make_float4(ftp, ftp, ftp, ftp);
                                NQ.id[pos] = id;
                                // the sub-path keeps wavelength k's weight alone
                                const float4 w0 = Q.w[0][i], w1 = Q.w[1][i], w2 = Q.w[2][i];
                                const float3 wk = k == 0 ? make_float3(w0.x, w0.y, w0.z)
                                                : k == 1 ? make_float3(w0.w, w1.x, w1.y)
                                                : k == 2 ? make_float3(w1.z, w1.w, w2.x)
                                                         : make_float3(w2.y, w2.z, w2.w);
                                NQ.w[0][pos] = make_float4(wk.x, wk.y, wk.z, 0.f);
                                NQ.w[1][pos] = make_float4(0.f, 0.f, 0.f, 0.f);
                                NQ.w[2][pos] = make_float4(0.f, 0.f, 0.f, 0.f);
                            } else {
                                atomicOr(&C->status, 2);
                            }
                        } else {
                            no = bo;
                            nd = bd;
                            // a refraction ends the other wavelengths; the
                            // hero's share is scaled by their number so the
                            // estimate stays unbiased (a reflection does not
                            // depend on the wavelength and keeps them all)
                            term = terminate && !refl;
                        }
                    }
                    if (!disperse) {
                        ntp = mul4(tp4, alg);
                        if (term) {
                            const float h0 = ntp.x * (float)nHero;
                            ntp = make_float4(h0, h0, h0, h0);
                        }
                        cont = true;
                    }
                }
            } else {
                // diffuse
                const float4 al = spectral ? spec4(m, 0, lam4) : rgb4(m.albedo);
                // indirect origin: hit moved once by 1e-3*N (the reference's
                // mutating `hit + N * 1e-3`, code/Renderer.cpp:782 with samples = 1)
                float3 hc = f3add(hit, f3mul(N, 1e-3f));
                const float3 h1 = hc;
                if (S.total_light_area > 0.f) {
                    const float scaleS = S.total_light_area * inv_pi / (float)R.shadow;
                    const float4 tpal = mul4(tp4, al);
                    int cached = -1;
                    float3 V = make_float3(0.f, 0.f, 0.f);
                    if (spectral && S.emit_mat >= 0) {
                        // every light has the one emissive material, whose
                        // emission the carried weights already hold: the
                        // vertex's product is known before any sample
                        V = f3mul(apply_xyz(load_weights(Q, i), tpal), scaleS);
                        cached = S.emit_mat;
                    }
                    const int spos = spos_block;
                    const int nsh = spos + (R.shadow - 1) * sstride < E.shadow_cap ? R.shadow : 0;
                    if (nsh == 0) atomicOr(&C->status, 1);
                    for (int s = 0; s < nsh; s++) {
                        const float4 rr = rand4(R, (uint32_t)id.y, (uint32_t)id.z, (uint32_t)fork, (uint32_t)bounce,
                                                1u + (uint32_t)s);
                        int pick = 0;
                        if (S.n_lights > 1) {
                            const float target = rr.x * S.total_light_area;
                            float cum = 0.f;
                            for (int l = 0; l < S.n_lights; l++) {
                                cum += S.lights[l].total_area;
                                if (target <= cum) { pick = l; break; }
                            }
                        }
                        const DLight& L = S.lights[pick];
                        float3 P, Nl;
                        int lm;
                        if (L.kind == 0) {
                            P = make_float3(L.o_mat.x + L.u.x * rr.y + L.v.x * rr.z, L.o_mat.y + L.u.y * rr.y + L.v.y * rr.z,
                                            L.o_mat.z + L.u.z * rr.y + L.v.z * rr.z);
                            Nl = xyz(L.n);
                            lm = __float_as_int(L.o_mat.w);
                        } else {
                            const float4 r2 = rand4(R, (uint32_t)id.y, (uint32_t)id.z, (uint32_t)fork, (uint32_t)bounce,
                                                    1000u + (uint32_t)s);
                            const float rt = rr.y * L.total_area;
                            const float* cum = S.light_cum + L.tri_offset;
                            int lo = 0, hi = L.tri_count;
                            while (lo < hi) { int mid = (lo + hi) >> 1; if (cum[mid] < rt) lo = mid + 1; else hi = mid; }
                            const int ti = lo < L.tri_count - 1 ? lo : L.tri_count - 1;
                            const DTri& lt = S.light_tris[L.tri_offset + ti];
                            float a = rr.z, b = r2.x;
                            if (a + b > 1.f) { a = 1.f - a; b = 1.f - b; }
                            P = make_float3(lt.v0_id.x + lt.e1_mat.x * a + lt.e2_flags.x * b,
                                            lt.v0_id.y + lt.e1_mat.y * a + lt.e2_flags.y * b,
                                            lt.v0_id.z + lt.e1_mat.z * a + lt.e2_flags.z * b);
                            Nl = xyz(S.light_flatn[L.tri_offset + ti]);
                            lm = __float_as_int(lt.e1_mat.w);
                        }
                        const float3 Li = f3sub(P, hc);
                        const float d2 = f3dot(Li, Li);
                        const float inv_d = rsqrtf(d2);
                        const float3 wi = f3mul(Li, inv_d);
                        const float cosT = fmaxf(0.f, f3dot(wi, N));
                        float3 so;
                        // the lit-facing branch moves the shading point again
                        // (code/Renderer.cpp:857, mutating operator+)
                        if (cosT <= 0.f) so = f3sub(hc, f3mul(N, 1e-3f));
                        else { hc = f3add(hc, f3mul(N, 1e-3f)); so = hc; }
                        const float cosL = fmaxf(0.f, -f3dot(Nl, Li));
                        const float G = cosT * cosL * (inv_d * inv_d);
                        const int pos = spos + s * sstride;
                        if (!(G > 0.f)) {
                            SQ.o[pos] = make_float4(0.f, 0.f, 0.f, -1.f);  // skip record
                            continue;
                        }
                        if (lm != cached) {
                            // product of this light material, once per vertex
                            const DMaterial& lmat = M[S.mat_base + lm];
                            const float4 c = spectral ? mul4(tpal, spec4(lmat, 1, lam4)) : mul4(tpal, rgb4(lmat.emissive));
                            V = f3mul(apply_xyz(spectral ? load_weights(Q, i) : rgb_weights(), c), scaleS);
                            cached = lm;
                        }
                        float w = 1.f;
                        if ((R.flags & kReqMIS) && cosL > 1e-6f) {
                            const float pL = d2 / (cosL * S.total_light_area), pB = cosT * inv_pi;
                            w = (pL * pL) / (pL * pL + pB * pB);
                        }
                        const float f = G * w;
                        SQ.o[pos] = make_float4(so.x, so.y, so.z, d2);
                        SQ.d[pos] = make_float4(wi.x, wi.y, wi.z, __int_as_float(id.y));
                        SQ.c[pos] = make_float4(V.x * f, V.y * f, V.z * f, __int_as_float(slot | (id.w << 16)));
                    }
                }
                const float4 r0 = rand4(R, (uint32_t)id.y, (uint32_t)id.z, (uint32_t)fork, (uint32_t)bounce, 0u);
                bool survive = !last;
                float rr_scale = 1.f;
                if (survive && (R.flags & kReqRussian) && bounce >= 1) {
                    float pr = spectral ? al.x : fmaxf(fmaxf(al.x, al.y), al.z);
                    pr = fminf(0.95f, fmaxf(0.05f, pr));
                    if (r0.w > pr) survive = false;
                    else rr_scale = 1.f / pr;
                }
                if (survive) {
                    float r1 = r0.x, r2 = r0.y;
                    if ((R.flags & kReqStratified) && bounce == 0 && R.strata > 0) {
                        const int sin_ = id.z % R.spp;
                        const int sx = sin_ % R.strata, sy = (sin_ / R.strata) % R.strata;
                        r1 = ((float)sx + r0.x) / (float)R.strata;
                        r2 = ((float)sy + r0.y) / (float)R.strata;
                    }
                    nd = hemisphere(N, r1, r2);
                    no = h1;
                    ntp = make_float4(tp4.x * al.x * rr_scale, tp4.y * al.y * rr_scale, tp4.z * al.z * rr_scale,
                                      tp4.w * al.w * rr_scale);
                    cont = true;
                }
            }
        }

        // ---- emit work (block-uniform control flow from here)
        if (emit) add_xyz(acc, emit_xyz);
        {
            const int newMeta = (bounce + 1) | (fork << 8) | ((single | (term ? 1 : 0)) << 11) | (nHero << 12);
            // one contiguous range per block (its warps in order), so the
            // next launch's warps rarely straddle two blocks' outputs, which
            // may belong to different scenes
            int* sw = s_app[parity];
            parity ^= 1;
            const unsigned am = __ballot_sync(0xffffffffu, cont);
            const int wid = threadIdx.x >> 5;
            if (lane == 0) sw[wid] = __popc(am);
            __syncthreads();
            if (threadIdx.x == 0) {
                int tot = 0;
                for (int k = 0; k < kShadeBlock / 32; k++) { const int c = sw[k]; sw[k] = tot; tot += c; }
                sw[kShadeBlock / 32] = tot ? atomicAdd(&C->queue_n[cur ^ 1], tot) : 0;
            }
            __syncthreads();
            int pos = cont ? sw[kShadeBlock / 32] + sw[wid] + __popc(am & ((1u << lane) - 1u)) : -1;
            if (pos >= E.queue_cap) { atomicOr(&C->status, 2); pos = -1; }
            if (pos >= 0) {
                NQ.o[pos] = make_float4(no.x, no.y, no.z, o4.w);
                NQ.d[pos] = make_float4(nd.x, nd.y, nd.z, __int_as_float(newMeta));
                NQ.tp[pos] = ntp;
                NQ.id[pos] = id;
                if (spec_path) {
                    const float4 w0 = Q.w[0][i];
                    NQ.w[0][pos] = term ? make_float4(w0.x, w0.y, w0.z, 0.f) : w0;
                    NQ.w[1][pos] = term ? make_float4(0.f, 0.f, 0.f, 0.f) : Q.w[1][i];
                    NQ.w[2][pos] = term ? make_float4(0.f, 0.f, 0.f, 0.f) : Q.w[2][i];
                }
            }
        }
        // path bookkeeping per request, one atomic per request per warp:
        // -1 for a retired path, ways-1 for a fork
        const long long delta = live ? (long long)((cont ? 0 : -1) + forked) : 0;
        const unsigned same = __match_any_sync(0xffffffffu, live ? slot : -1);
        const int sum = __reduce_add_sync(same, (int)delta);
        if (live && sum != 0 && lane == __ffs(same) - 1)
            atomicAdd((unsigned long long*)&E.outstanding[slot], (unsigned long long)(long long)sum);
    }
}

// ------------------------------------------------------------------ shadow
// Shadow-ray test (code/Renderer.cpp:852-860): blocked when the closest hit
// within the light distance is non-emissive and closer than lightDist2 -
// 1e-3 (compared in double, as the reference's double literal promotes it);
// scene_blocked answers it with an early exit.  Lit samples add their XYZ
// contribution to the pixel's FP64 accumulator.
__global__ void __launch_bounds__(kTraceMaxBlock, kShadowMinBlocks) k_shadow(EngineView E)
{
    Counters* C = E.cnt;
    const int n = min(C->shadow_n, E.shadow_cap);
    const ShadowQueue SQ = E.sq;
    unsigned mine = 0;  // shadow rays of this thread (one launch: < 2^32)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int nx = i + gridDim.x * blockDim.x;
        if (nx < n) { prefetch_l2(SQ.o + nx); prefetch_l2(SQ.d + nx); prefetch_l2(SQ.c + nx); }
        const float4 o = SQ.o[i];
        if (!(o.w >= 0.f)) continue;  // skip record (zero geometry term)
        const float4 d = SQ.d[i];
        // only the scene is needed for the query; the contribution is read
        // afterwards, for lit samples, so it holds no registers across it
        const DScene& S = E.scenes[__float_as_int(SQ.c[i].w) >> 16];
        const float d2 = o.w;
        // a hit beyond the light cannot block: bound the query just past it
        const float tmax = sqrtf(d2) * 1.0001f + 1e-4f;
        mine++;
        if (!scene_blocked(S, E.mats, xyz(o), xyz(d), tmax, (double)d2 - 1e-3)) {
            const float4 c = SQ.c[i];
            const int pixel = __float_as_int(SQ.d[i].w);
            add_xyz(E.reqs[__float_as_int(c.w) & 0xFFFF].accum + (size_t)pixel * 3, make_float3(c.x, c.y, c.z));
        }
    }
    unsigned long long warp_rays = mine;
    for (int off = 16; off > 0; off >>= 1) warp_rays += __shfl_down_sync(0xffffffffu, warp_rays, off);
    if ((threadIdx.x & 31) == 0 && warp_rays) atomicAdd(&C->shadow_rays, warp_rays);
}

// ------------------------------------------------------------------ status
// End of iteration: marks requests whose paths are all issued and retired.
__global__ void k_status(EngineView E, int next)
{
    Counters* C = E.cnt;
    const int n_act = *E.n_active;
    __shared__ int s_busy;
    if (threadIdx.x == 0) s_busy = 0;
    __syncthreads();
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    for (int r = threadIdx.x; r < n_act; r += blockDim.x) {
        const int slot = E.active[r];
        if (E.done_flag[slot]) continue;
        if (E.round_state[slot]) { s_busy = 1; continue; }
        const bool all_issued = (long long)E.issued[slot] >= E.reqs[slot].total;
        if (all_issued && E.outstanding[slot] == 0) {
            // a cancelled adaptive request opens no further round
            if ((E.reqs[slot].flags & (kReqAdaptive | kReqCancelled)) == kReqAdaptive) {
                E.round_state[slot] = 1;  // k_round, then the next k_schedule
                E.round_list[atomicAdd(&C->n_rounds, 1)] = slot;
                s_busy = 1;
            } else {
                E.done_flag[slot] = 1;
                E.t_done[slot] = now;
            }
        } else {
            s_busy = 1;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        C->idle = (s_busy == 0 && C->queue_n[next] == 0) ? 1 : 0;
        C->iter++;
    }
}

// ------------------------------------------------------------------ adaptive rounds
// End of an adaptive aa round (the GPU backends' per-pixel Welford loop,
// code/Gpu/Opengl/OpenglRenderer.cpp:1288-1383): each pixel of the round
// takes the mean of its spp paths, updates its running mean / M2, and stops
// after 4 or more rounds once every channel's relative variance
// M2/(taken-1) / (mean^2 + 0.01) is below 0.05, or after aa rounds.
// Stopped pixels write their mean to the accumulator (resolved with weight
// 1); the others reset it and move to the next round's list.
__global__ void k_round(EngineView E)
{
    const int n_rounds = E.cnt->n_rounds;
    const int lane = threadIdx.x & 31;
    for (int r = 0; r < n_rounds; r++) {
        const int slot = E.round_list[r];
        const DRequest& R = E.reqs[slot];
        const int n = (int)((R.total - R.round_base) / R.spp);
        const int* list = R.act[R.round & 1];
        int* next = R.act[(R.round & 1) ^ 1];
        const float inv = 1.f / (float)R.spp;
        const int stride = gridDim.x * blockDim.x;
        for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {  // warp-uniform trips
            const int k = base + threadIdx.x;
            bool keep = false;
            int px = 0;
            if (k < n) {
                px = list[k];
                double* a = R.accum + (size_t)px * 3;
                const float3 c = make_float3((float)a[0] * inv, (float)a[1] * inv, (float)a[2] * inv);
                float4 m = R.welford[2 * (size_t)px], m2 = R.welford[2 * (size_t)px + 1];
                const float taken = m.w + 1.f;
                const float3 d1 = make_float3(c.x - m.x, c.y - m.y, c.z - m.z);
                m.x += d1.x / taken; m.y += d1.y / taken; m.z += d1.z / taken;
                const float3 d2 = make_float3(c.x - m.x, c.y - m.y, c.z - m.z);
                m2.x += d1.x * d2.x; m2.y += d1.y * d2.y; m2.z += d1.z * d2.z;
                m.w = taken;
                bool done = (int)taken >= R.aa;
                if (!done && taken >= 4.f) {
                    const float t1 = taken - 1.f;
                    const float rx = (m2.x / t1) / (m.x * m.x + 0.01f), ry = (m2.y / t1) / (m.y * m.y + 0.01f),
                                rz = (m2.z / t1) / (m.z * m.z + 0.01f);
                    done = fmaxf(fmaxf(rx, ry), rz) < 0.05f;
                }
                R.welford[2 * (size_t)px] = m;
                R.welford[2 * (size_t)px + 1] = m2;
                if (done) { a[0] = m.x; a[1] = m.y; a[2] = m.z; }
                else { a[0] = 0.0; a[1] = 0.0; a[2] = 0.0; keep = true; }
            }
            const unsigned km = __ballot_sync(0xffffffffu, keep);
            int b = 0;
            if (lane == 0 && km) b = atomicAdd(&E.round_cnt[slot], __popc(km));
            b = __shfl_sync(0xffffffffu, b, 0);
            if (keep) next[b + __popc(km & ((1u << lane) - 1u))] = px;
        }
    }
}

// ------------------------------------------------------------------ resolve
// Per-pixel mean -> linear sRGB (code/Renderer.cpp:300-302), then tone map
// and 8-bit quantise (code/Renderer.cpp:365-382) on the device.
__global__ void k_resolve(const double* __restrict__ acc, int npix, double inv_n, int spectral, int aces_tm,
                          float* __restrict__ hdr, unsigned char* __restrict__ rgb8)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        float3 c = make_float3((float)(acc[i * 3] * inv_n), (float)(acc[i * 3 + 1] * inv_n), (float)(acc[i * 3 + 2] * inv_n));
        if (spectral) c = xyz_to_srgb(c);
        if (hdr) { hdr[i * 3] = c.x; hdr[i * 3 + 1] = c.y; hdr[i * 3 + 2] = c.z; }
        if (rgb8) {
            float3 m = aces_tm ? make_float3(aces(c.x), aces(c.y), aces(c.z)) : make_float3(reinhard(c.x), reinhard(c.y), reinhard(c.z));
            rgb8[i * 3] = quantize(m.x);
            rgb8[i * 3 + 1] = quantize(m.y);
            rgb8[i * 3 + 2] = quantize(m.z);
        }
    }
}

// Tone map + quantise a linear sRGB image (the last step of k_resolve).
__global__ void k_tonemap(const float* __restrict__ hdr, int npix, int aces_tm, unsigned char* __restrict__ rgb8)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        const float3 c = make_float3(hdr[i * 3], hdr[i * 3 + 1], hdr[i * 3 + 2]);
        const float3 m = aces_tm ? make_float3(aces(c.x), aces(c.y), aces(c.z))
                                 : make_float3(reinhard(c.x), reinhard(c.y), reinhard(c.z));
        rgb8[i * 3] = quantize(m.x);
        rgb8[i * 3 + 1] = quantize(m.y);
        rgb8[i * 3 + 2] = quantize(m.z);
    }
}

// ------------------------------------------------------------------ denoise
// One pass of the 5x5 cross-bilateral on the 8-bit image (Denoise::
// bilateralRGB, code/Denoise.cpp:14-86, which runs two): spatial sigma 1.5
// px, colour sigma 10 levels, float arithmetic in the reference's order (no
// contraction), the weight's exponential taken in double and rounded once.
__global__ void k_bilateral(const unsigned char* __restrict__ src, unsigned char* __restrict__ dst, int width,
                            int height)
{
    using namespace ex;
    const float invSpatial2 = div(1.0f, mul(mul(2.0f, 1.5f), 1.5f));
    const float invColor2 = div(1.0f, mul(mul(2.0f, 10.0f), 10.0f));
    const int npix = width * height;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        const int y = p / width, x = p - y * width;
        const float cR = (float)src[p * 3], cG = (float)src[p * 3 + 1], cB = (float)src[p * 3 + 2];
        float sumW = 0.f, sumR = 0.f, sumG = 0.f, sumB = 0.f;
        for (int dy = -2; dy <= 2; dy++) {
            const int ny = y + dy;
            if (ny < 0 || ny >= height) continue;
            for (int dx = -2; dx <= 2; dx++) {
                const int nx = x + dx;
                if (nx < 0 || nx >= width) continue;
                const int q = (ny * width + nx) * 3;
                const float nR = (float)src[q], nG = (float)src[q + 1], nB = (float)src[q + 2];
                const float spatial = mul((float)(dx * dx + dy * dy), invSpatial2);
                const float dR = sub(nR, cR), dG = sub(nG, cG), dB = sub(nB, cB);
                const float color = mul(add(add(mul(dR, dR), mul(dG, dG)), mul(dB, dB)), invColor2);
                const float w = (float)exp(-(double)add(spatial, color));
                sumW = add(sumW, w);
                sumR = add(sumR, mul(w, nR));
                sumG = add(sumG, mul(w, nG));
                sumB = add(sumB, mul(w, nB));
            }
        }
        if (sumW > 0.f) {
            dst[p * 3] = (unsigned char)fminf(255.f, add(div(sumR, sumW), 0.5f));
            dst[p * 3 + 1] = (unsigned char)fminf(255.f, add(div(sumG, sumW), 0.5f));
            dst[p * 3 + 2] = (unsigned char)fminf(255.f, add(div(sumB, sumW), 0.5f));
        } else {
            dst[p * 3] = src[p * 3];
            dst[p * 3 + 1] = src[p * 3 + 1];
            dst[p * 3 + 2] = src[p * 3 + 2];
        }
    }
}

// ------------------------------------------------------------------ parity kernels
__global__ void k_trace_rays(const DScene* scene, const DMaterial* mats, const float* __restrict__ rays, long long n,
                             int* mat, int* prim_out, float* t_out, int bvh_only, int* counts)
{
    const DScene& S = *scene;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float3 o = make_float3(rays[i * 6], rays[i * 6 + 1], rays[i * 6 + 2]);
        const float3 d = make_float3(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5]);
        float t = FLT_MAX, u = 0.f, v = 0.f;
        if (bvh_only) {
            TraceCounts tc = {0, 0};
            int tri = counts ? bvh4_closest<true>(S, o, d, t, u, v, &tc) : bvh4_closest<false>(S, o, d, t, u, v, nullptr);
            prim_out[i] = tri >= 0 ? __float_as_int(S.tris[tri].v0_id.w) : -1;
            t_out[i] = tri >= 0 ? t : 0.f;
            if (counts) { counts[i * 2] = tc.nodes; counts[i * 2 + 1] = tc.tris; }
        } else {
            const uint32_t prim = scene_closest(S, o, d, FLT_MAX, t, u, v);
            const uint32_t kind = prim & kPrimKindMask, pidx = prim & kPrimIndexMask;
            int mi = -1;
            uint32_t code = 0;
            if (kind == kPrimSphere) { mi = S.spheres[pidx].mat.x; code = kind | pidx; }
            else if (kind == kPrimPlane) { mi = __float_as_int(S.planes[pidx].o_mat.w); code = kind | pidx; }
            else if (kind == kPrimTri) {
                mi = __float_as_int(S.tris[pidx].e1_mat.w);
                code = kind | ((uint32_t)__float_as_int(S.tris[pidx].v0_id.w) & kPrimIndexMask);
            }
            mat[i] = mi;
            prim_out[i] = (int)code;
            t_out[i] = kind ? t : 0.f;
        }
    }
}

// The shadow test of k_shadow on caller rays (origin, unit direction) with
// their squared light distances: 1 when blocked.
__global__ void k_trace_shadow(const DScene* scene, const DMaterial* mats, const float* __restrict__ rays,
                               const float* __restrict__ dist2, long long n, int* blocked)
{
    const DScene& S = *scene;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float3 o = make_float3(rays[i * 6], rays[i * 6 + 1], rays[i * 6 + 2]);
        const float3 d = make_float3(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5]);
        const float d2 = dist2[i];
        blocked[i] = scene_blocked(S, mats, o, d, sqrtf(d2) * 1.0001f + 1e-4f, (double)d2 - 1e-3) ? 1 : 0;
    }
}

__global__ void k_eval_stage(int what, const float* __restrict__ params, const float* __restrict__ in, long long n,
                             float* __restrict__ out, float xyz_scale, const float4* __restrict__ cmf_table)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        switch (what) {
        case 0: out[i] = sigmoid_fit(make_float4(params[0], params[1], params[2], params[3]), in[i]); break;
        case 1: out[i] = spectrum_lerp(params, in[i]); break;
        case 2: { float3 c = cmf(in[i]); out[i * 3] = c.x; out[i * 3 + 1] = c.y; out[i * 3 + 2] = c.z; } break;
        case 3: {
            float3 c = cmf(in[i * 2]);
            float r = in[i * 2 + 1];
            out[i * 3] = r * c.x * xyz_scale; out[i * 3 + 1] = r * c.y * xyz_scale; out[i * 3 + 2] = r * c.z * xyz_scale;
        } break;
        case 4: { float3 c = xyz_to_srgb(make_float3(in[i * 3], in[i * 3 + 1], in[i * 3 + 2]));
                  out[i * 3] = c.x; out[i * 3 + 1] = c.y; out[i * 3 + 2] = c.z; } break;
        case 5: for (int k = 0; k < 3; k++) out[i * 3 + k] = reinhard(in[i * 3 + k]); break;
        case 6: for (int k = 0; k < 3; k++) out[i * 3 + k] = aces(in[i * 3 + k]); break;
        case 7: for (int k = 0; k < 3; k++) out[i * 3 + k] = (float)quantize(in[i * 3 + k]); break;
        case 8: {
            // the XYZ weight raygen stores for a one-wavelength path (the
            // colour-matching table), times the radiance: singleLambdaXYZ
            const float lam[4] = {in[i * 2], in[i * 2], in[i * 2], in[i * 2]};
            const XyzWeights W = xyz_weights(true, lam, 1, 1.f, xyz_scale, cmf_table);
            const float r = in[i * 2 + 1];
            out[i * 3] = r * W.w[0].x; out[i * 3 + 1] = r * W.w[0].y; out[i * 3 + 2] = r * W.w[0].z;
        } break;
        default: break;
        }
    }
}

}  // namespace pcr
