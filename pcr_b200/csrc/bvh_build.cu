// Device build of the binary SAH BVH (code/Bvh/Bvh.cpp:122-325), producing
// the same node array (depth-first preorder, same boxes bit for bit) and the
// same triangle order as the host builder `build_bvh` in scene.cpp.
//
// Work split:
// * Nodes over more than kSmall triangles are processed level by level, all
//   nodes of a level at once, by blocks that each own a chunk of 1024
//   positions of one node: node bounds, centroid bounds, 3 x 16 bins, the SAH
//   decision (one thread per node), and the reference's two-cursor partition
//   restated in parallel (below).
// * A node of kSmall or fewer triangles is built to the end by one thread,
//   sequentially, exactly as the host recursion does.
// * The finished pieces are renumbered into depth-first preorder.
//
// Why the result is bit-equal to the sequential build:
// * A node's box keeps, per axis, the FIRST vertex (in position order, v0 v1
//   v2 within a triangle) whose value is the minimum (maximum), since the
//   sequential `if (p < mn) mn = p` never replaces an equal value; so -0 and
//   +0 are told apart exactly as there.  Each min / max is reduced as a
//   64-bit key (monotonic value, vertex sequence number), which makes the
//   reduction order irrelevant.
// * Centroid bounds and bin boxes are only used through differences and
//   areas, where -0 and +0 give the same decisions, so they are reduced as
//   plain monotonic 32-bit keys; counts are integers.
// * All decision arithmetic uses explicitly rounded operations (__fadd_rn ...)
//   in the host's operation order; the host side is compiled without
//   floating-point contraction.
// * The two-cursor partition (libstdc++ std::partition for bidirectional
//   iterators) swaps the k-th misplaced element from the left (a right-side
//   triangle before the split point) with the k-th misplaced element from the
//   right (a left-side triangle after it); every other triangle stays put.
//   The ranks come from a prefix count of the left-side flags.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <vector>

#include "bvh_build.h"
#include "engine.h"
#include "scene.h"

namespace pcr {
namespace {

constexpr int kChunk = 1024;      // positions per block in the level passes
constexpr int kLevelBlock = 256;  // threads per block in the level passes
constexpr int kSmall = 32;        // nodes at or below this size go to one thread
constexpr int kBins = 16;

// Per triangle, in input order: lo / hi = the triangle's per-axis min / max
// vertex value (first vertex among equals), lo.w packs which vertex holds
// each (2 bits per axis, min in bits 0-5, max in bits 8-13); c = centroid.
struct alignas(16) BTri {
    float4 lo, hi, c;
};

struct BTask {
    int begin, count, slot, cbase;
    int nchunks, axis, bin, r;
    int mid, pad0;
    float lo, scale;
    unsigned long long kmin[3], kmax[3];
    unsigned cmin[3], cmax[3];
};

struct TopNode {   // a node of the level-processed part, before renumbering
    float bmin[3], bmax[3];
    int left, right, count;   // kind 0: child slots; kind 1: first, -, count
    int kind, ref;            // kind 2: root of small task `ref`
};

struct SmallTask {
    int begin, count, slot, nnodes;
};

struct BuildCounters {
    int ntop, ntasks, nchunks, nsmall;
    int error;   // set by a bounds or consistency check; the host throws
};

struct Caps {
    int top, tasks, chunks, small;
};

__device__ __forceinline__ float getc(const float4& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// monotonic key of a float; -0 and +0 map to the same key
__device__ __forceinline__ unsigned ord_key(float f)
{
    unsigned u = f == 0.f ? 0u : __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_value(unsigned k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Box::area (host order: 2 * ((dx*dy + dy*dz) + dz*dx), 0 when inverted)
__device__ __forceinline__ float box_area(const float mn[3], const float mx[3])
{
    const float dx = __fsub_rn(mx[0], mn[0]), dy = __fsub_rn(mx[1], mn[1]), dz = __fsub_rn(mx[2], mn[2]);
    if (dx < 0.f || dy < 0.f || dz < 0.f) return 0.f;
    return __fmul_rn(2.f, __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx)));
}

__device__ __forceinline__ int bin_of(float c, float lo, float scale)
{
    const int b = __float2int_rz(__fmul_rn(__fsub_rn(c, lo), scale));
    return b < 0 ? 0 : (b > kBins - 1 ? kBins - 1 : b);
}

// One axis of the SAH sweep over filled bins, in the host's order: left
// prefix areas / counts, right suffix areas / counts, then costs for split
// s = 0..14 with a strict `<` against the best so far.
__device__ void sah_axis(const float (*bmn)[3], const float (*bmx)[3], const int* cnt, float parent, int axis,
                         float& best_cost, int& best_axis, int& best_bin, int& best_lc)
{
    float lSA[kBins - 1], rSA[kBins - 1];
    int lC[kBins - 1], rC[kBins - 1];
    float amn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, amx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    int ac = 0;
    for (int i = 0; i < kBins - 1; i++) {
        for (int a = 0; a < 3; a++) {
            if (bmn[i][a] < amn[a]) amn[a] = bmn[i][a];
            if (bmx[i][a] > amx[a]) amx[a] = bmx[i][a];
        }
        ac += cnt[i];
        lSA[i] = box_area(amn, amx);
        lC[i] = ac;
    }
    for (int a = 0; a < 3; a++) { amn[a] = FLT_MAX; amx[a] = -FLT_MAX; }
    ac = 0;
    for (int i = kBins - 1; i > 0; i--) {
        for (int a = 0; a < 3; a++) {
            if (bmn[i][a] < amn[a]) amn[a] = bmn[i][a];
            if (bmx[i][a] > amx[a]) amx[a] = bmx[i][a];
        }
        ac += cnt[i];
        rSA[i - 1] = box_area(amn, amx);
        rC[i - 1] = ac;
    }
    for (int s = 0; s < kBins - 1; s++) {
        if (lC[s] == 0 || rC[s] == 0) continue;
        const float sum = __fadd_rn(__fmul_rn(lSA[s], (float)lC[s]), __fmul_rn(rSA[s], (float)rC[s]));
        const float cost = __fadd_rn(1.f, __fdiv_rn(__fmul_rn(2.f, sum), parent));
        if (cost < best_cost) {
            best_cost = cost;
            best_axis = axis;
            best_bin = s;
            best_lc = lC[s];
        }
    }
}

__global__ void k_bvh_prep(const float* __restrict__ verts, int n, BTri* __restrict__ T, int* __restrict__ perm)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* v = verts + (size_t)i * 9;
    float lo[3], hi[3], c[3];
    int kb = 0;
    for (int a = 0; a < 3; a++) {
        int kl = 0, kh = 0;
        float l = v[a], h = v[a];
        for (int k = 1; k < 3; k++) {
            const float x = v[k * 3 + a];
            if (x < l) { l = x; kl = k; }
            if (x > h) { h = x; kh = k; }
        }
        lo[a] = l;
        hi[a] = h;
        kb |= kl << (2 * a) | kh << (8 + 2 * a);
        // (v0 + v1 + v2) * (1/3) as the host's centroid()
        c[a] = __fmul_rn(__fadd_rn(__fadd_rn(v[a], v[3 + a]), v[6 + a]), 1.f / 3.f);
    }
    T[i].lo = make_float4(lo[0], lo[1], lo[2], __int_as_float(kb));
    T[i].hi = make_float4(hi[0], hi[1], hi[2], 0.f);
    T[i].c = make_float4(c[0], c[1], c[2], 0.f);
    perm[i] = i;
}

__global__ void k_bvh_init(BTask* __restrict__ tasks, int ntasks, unsigned* __restrict__ bins, int* __restrict__ bcnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntasks * 3 * kBins) return;
    const int t = i / (3 * kBins);
    unsigned* b = bins + (size_t)i * 6;
    for (int k = 0; k < 3; k++) { b[k] = 0xffffffffu; b[3 + k] = 0u; }
    bcnt[i] = 0;
    if (i % (3 * kBins) == 0) {
        BTask& T = tasks[t];
        for (int a = 0; a < 3; a++) {
            T.kmin[a] = ~0ull;
            T.kmax[a] = 0ull;
            T.cmin[a] = 0xffffffffu;
            T.cmax[a] = 0u;
        }
    }
}

__device__ __forceinline__ unsigned long long shfl_min64(unsigned long long v)
{
    for (int o = 16; o; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
__device__ __forceinline__ unsigned long long shfl_max64(unsigned long long v)
{
    for (int o = 16; o; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Node bounds (first-occurrence keys) and centroid bounds of every large node.
__global__ void __launch_bounds__(kLevelBlock) k_bvh_bounds(const BTri* __restrict__ T, const int* __restrict__ perm,
                                                            BTask* __restrict__ tasks, const int2* __restrict__ chunks)
{
    const int2 ch = chunks[blockIdx.x];
    BTask& t = tasks[ch.x];
    const int p0 = t.begin + ch.y * kChunk, p1 = min(p0 + kChunk, t.begin + t.count);
    unsigned long long kmn[3] = {~0ull, ~0ull, ~0ull}, kmx[3] = {0ull, 0ull, 0ull};
    unsigned cmn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, cmx[3] = {0u, 0u, 0u};
    for (int p = p0 + (int)threadIdx.x; p < p1; p += kLevelBlock) {
        const BTri r = T[perm[p]];
        const int kb = __float_as_int(r.lo.w);
        const unsigned seq = 3u * (unsigned)p;
        for (int a = 0; a < 3; a++) {
            const unsigned long long kl =
                (unsigned long long)ord_key(getc(r.lo, a)) << 32 | (seq + ((kb >> (2 * a)) & 3));
            const unsigned long long kh =
                (unsigned long long)ord_key(getc(r.hi, a)) << 32 | (0xffffffffu - (seq + ((kb >> (8 + 2 * a)) & 3)));
            kmn[a] = kl < kmn[a] ? kl : kmn[a];
            kmx[a] = kh > kmx[a] ? kh : kmx[a];
            const unsigned kc = ord_key(getc(r.c, a));
            cmn[a] = min(cmn[a], kc);
            cmx[a] = max(cmx[a], kc);
        }
    }
    for (int a = 0; a < 3; a++) {
        kmn[a] = shfl_min64(kmn[a]);
        kmx[a] = shfl_max64(kmx[a]);
        cmn[a] = __reduce_min_sync(0xffffffffu, cmn[a]);
        cmx[a] = __reduce_max_sync(0xffffffffu, cmx[a]);
    }
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; a++) {
            if (kmn[a] != ~0ull) atomicMin(&t.kmin[a], kmn[a]);
            if (kmx[a] != 0ull) atomicMax(&t.kmax[a], kmx[a]);
            atomicMin(&t.cmin[a], cmn[a]);
            atomicMax(&t.cmax[a], cmx[a]);
        }
    }
}

struct AxisBin {
    bool use;
    float lo, scale;
};
__device__ __forceinline__ AxisBin axis_bin(const BTask& t, int a)
{
    AxisBin r;
    r.lo = key_value(t.cmin[a]);
    const float ext = __fsub_rn(key_value(t.cmax[a]), r.lo);
    r.use = !(ext < 1e-6f);
    r.scale = r.use ? __fdiv_rn((float)kBins, ext) : 0.f;
    return r;
}

// 3 x 16 bins (box keys and counts) of every large node.
__global__ void __launch_bounds__(kLevelBlock) k_bvh_bins(const BTri* __restrict__ T, const int* __restrict__ perm,
                                                          const BTask* __restrict__ tasks, const int2* __restrict__ chunks,
                                                          unsigned* __restrict__ bins, int* __restrict__ bcnt)
{
    __shared__ unsigned sb[3 * kBins][6];
    __shared__ int sc[3 * kBins];
    for (int i = threadIdx.x; i < 3 * kBins; i += kLevelBlock) {
        for (int k = 0; k < 3; k++) { sb[i][k] = 0xffffffffu; sb[i][3 + k] = 0u; }
        sc[i] = 0;
    }
    const int2 ch = chunks[blockIdx.x];
    const BTask& t = tasks[ch.x];
    AxisBin ab[3];
    for (int a = 0; a < 3; a++) ab[a] = axis_bin(t, a);
    __syncthreads();
    const int p0 = t.begin + ch.y * kChunk, p1 = min(p0 + kChunk, t.begin + t.count);
    for (int p = p0 + (int)threadIdx.x; p < p1; p += kLevelBlock) {
        const BTri r = T[perm[p]];
        const unsigned l[3] = {ord_key(r.lo.x), ord_key(r.lo.y), ord_key(r.lo.z)};
        const unsigned h[3] = {ord_key(r.hi.x), ord_key(r.hi.y), ord_key(r.hi.z)};
        for (int a = 0; a < 3; a++) {
            if (!ab[a].use) continue;
            const int b = a * kBins + bin_of(getc(r.c, a), ab[a].lo, ab[a].scale);
            for (int k = 0; k < 3; k++) {
                atomicMin(&sb[b][k], l[k]);
                atomicMax(&sb[b][3 + k], h[k]);
            }
            atomicAdd(&sc[b], 1);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * kBins; i += kLevelBlock) {
        if (sc[i] == 0) continue;
        const size_t g = (size_t)ch.x * 3 * kBins + i;
        for (int k = 0; k < 3; k++) {
            atomicMin(&bins[g * 6 + k], sb[i][k]);
            atomicMax(&bins[g * 6 + 3 + k], sb[i][3 + k]);
        }
        atomicAdd(&bcnt[g], sc[i]);
    }
}

struct LevelOut {
    BTask* tasks;
    int2* chunks;
};

// The SAH decision of every large node (one thread per node); writes the
// node, allocates its children and queues them for the next level or for a
// thread of their own.
__global__ void k_bvh_split(const BTri* __restrict__ T, const int* __restrict__ perm, BTask* __restrict__ tasks,
                            int ntasks, const unsigned* __restrict__ bins, const int* __restrict__ bcnt,
                            TopNode* __restrict__ top, SmallTask* __restrict__ small, LevelOut next,
                            BuildCounters* __restrict__ ctr, Caps cap)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntasks) return;
    BTask& t = tasks[i];
    TopNode& N = top[t.slot];
    float box_mn[3], box_mx[3];
    for (int a = 0; a < 3; a++) {
        const unsigned smin = (unsigned)(t.kmin[a] & 0xffffffffu);
        const unsigned smax = 0xffffffffu - (unsigned)(t.kmax[a] & 0xffffffffu);
        box_mn[a] = getc(T[perm[smin / 3]].lo, a);
        box_mx[a] = getc(T[perm[smax / 3]].hi, a);
        N.bmin[a] = box_mn[a];
        N.bmax[a] = box_mx[a];
    }
    const int count = t.count;
    int best_axis = -1, best_bin = -1, best_lc = 0;
    float best_cost = FLT_MAX;
    const float parent = box_area(box_mn, box_mx);
    if (parent > 0.f) {
        for (int a = 0; a < 3; a++) {
            const AxisBin ab = axis_bin(t, a);
            if (!ab.use) continue;
            float bmn[kBins][3], bmx[kBins][3];
            int cnt[kBins];
            for (int b = 0; b < kBins; b++) {
                const size_t g = (size_t)i * 3 * kBins + a * kBins + b;
                cnt[b] = bcnt[g];
                for (int k = 0; k < 3; k++) {
                    bmn[b][k] = cnt[b] ? key_value(bins[g * 6 + k]) : FLT_MAX;
                    bmx[b][k] = cnt[b] ? key_value(bins[g * 6 + 3 + k]) : -FLT_MAX;
                }
            }
            sah_axis(bmn, bmx, cnt, parent, a, best_cost, best_axis, best_bin, best_lc);
        }
    }
    t.axis = -1;
    const int mid = t.begin + best_lc;
    if (best_axis < 0 || best_cost >= __fmul_rn((float)count, 2.f) || mid == t.begin || mid == t.begin + count) {
        N.kind = 1;
        N.left = t.begin;
        N.right = 0;
        N.count = count;
        return;
    }
    const AxisBin ab = axis_bin(t, best_axis);
    t.axis = best_axis;
    t.bin = best_bin;
    t.lo = ab.lo;
    t.scale = ab.scale;
    t.mid = mid;
    N.kind = 0;
    N.count = 0;
    int child[2];
    const int cb[2] = {t.begin, mid}, ce[2] = {mid, t.begin + count};
    for (int k = 0; k < 2; k++) {
        const int slot = atomicAdd(&ctr->ntop, 1);
        child[k] = slot;
        if (slot >= cap.top) { ctr->error = 1; t.axis = -1; return; }
        const int n = ce[k] - cb[k];
        if (n > kSmall) {
            const int j = atomicAdd(&ctr->ntasks, 1);
            const int nc = (n + kChunk - 1) / kChunk;
            const int c0 = atomicAdd(&ctr->nchunks, nc);
            if (j >= cap.tasks || c0 + nc > cap.chunks) { ctr->error = 2; t.axis = -1; return; }
            BTask& u = next.tasks[j];
            u.begin = cb[k];
            u.count = n;
            u.slot = slot;
            u.cbase = c0;
            u.nchunks = nc;
            for (int q = 0; q < nc; q++) next.chunks[c0 + q] = make_int2(j, q);
            top[slot].kind = 0;
        } else {
            const int s = atomicAdd(&ctr->nsmall, 1);
            if (s >= cap.small) { ctr->error = 3; t.axis = -1; return; }
            small[s].begin = cb[k];
            small[s].count = n;
            small[s].slot = slot;
            small[s].nnodes = 0;
            top[slot].kind = 2;
            top[slot].ref = s;
        }
    }
    N.left = child[0];
    N.right = child[1];
}

// Left-side flags of every splitting node, and their count per chunk.
__global__ void __launch_bounds__(kLevelBlock) k_bvh_classify(const BTri* __restrict__ T, const int* __restrict__ perm,
                                                              const BTask* __restrict__ tasks,
                                                              const int2* __restrict__ chunks,
                                                              unsigned char* __restrict__ side, int* __restrict__ cleft)
{
    const int2 ch = chunks[blockIdx.x];
    const BTask& t = tasks[ch.x];
    if (t.axis < 0) return;
    const int p0 = t.begin + ch.y * kChunk, p1 = min(p0 + kChunk, t.begin + t.count);
    int n = 0;
    for (int p = p0 + (int)threadIdx.x; p < p1; p += kLevelBlock) {
        const float c = getc(T[perm[p]].c, t.axis);
        const int left = bin_of(c, t.lo, t.scale) <= t.bin;
        side[p] = (unsigned char)left;
        n += left;
    }
    n = __reduce_add_sync(0xffffffffu, n);
    __shared__ int s[kLevelBlock / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        int sum = 0;
        for (int w = 0; w < kLevelBlock / 32; w++) sum += s[w];
        cleft[blockIdx.x] = sum;
    }
}

// Per splitting node: chunk offsets of the left-flag prefix count, and r =
// the number of right-side triangles before the split point (= swaps).
__global__ void k_bvh_scan(BTask* __restrict__ tasks, int ntasks, const unsigned char* __restrict__ side,
                           const int* __restrict__ cleft, int* __restrict__ coff, BuildCounters* __restrict__ ctr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntasks) return;
    BTask& t = tasks[i];
    if (t.axis < 0) return;
    int off = 0;
    for (int k = 0; k < t.nchunks; k++) {
        coff[t.cbase + k] = off;
        off += cleft[t.cbase + k];
    }
    if (off != t.mid - t.begin) {   // the flags must agree with the bin counts
        ctr->error = 4;
        t.r = 0;
        return;
    }
    const int km = (t.mid - t.begin) / kChunk;
    int lp = coff[t.cbase + km];
    for (int p = t.begin + km * kChunk; p < t.mid; p++) lp += side[p];
    t.r = (t.mid - t.begin) - lp;
}

// Ranks of the misplaced triangles: R[k] = position of the k-th right-side
// triangle before the split point (from the left), L[k] = position of the
// k-th left-side triangle after it (from the right).
__global__ void __launch_bounds__(kLevelBlock) k_bvh_ranks(const BTask* __restrict__ tasks,
                                                           const int2* __restrict__ chunks,
                                                           const unsigned char* __restrict__ side,
                                                           const int* __restrict__ coff, int* __restrict__ R,
                                                           int* __restrict__ L)
{
    const int2 ch = chunks[blockIdx.x];
    const BTask& t = tasks[ch.x];
    if (t.axis < 0) return;
    const int p0 = t.begin + ch.y * kChunk, p1 = min(p0 + kChunk, t.begin + t.count);
    constexpr int kPer = kChunk / kLevelBlock;
    const int q0 = p0 + (int)threadIdx.x * kPer;
    int f[kPer], mine = 0;
    for (int k = 0; k < kPer; k++) {
        f[k] = (q0 + k < p1) ? side[q0 + k] : 0;
        mine += f[k];
    }
    // block exclusive scan of the per-thread counts
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    __shared__ int wsum[kLevelBlock / 32];
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int wbase = 0;
    for (int w = 0; w < warp; w++) wbase += wsum[w];
    int lp = coff[blockIdx.x] + wbase + incl - mine;   // left flags in [begin, q0)
    const int Lall = t.mid - t.begin, r = t.r;
    for (int k = 0; k < kPer; k++) {
        const int p = q0 + k;
        if (p >= p1) break;
        if (p < t.mid) {
            const int k2 = (p - t.begin) - lp;
            if (!f[k] && k2 >= 0 && k2 < r) R[t.begin + k2] = p;
        } else if (f[k]) {
            const int k2 = r - 1 - (lp - (Lall - r));
            if (k2 >= 0 && k2 < r) L[t.begin + k2] = p;
        }
        lp += f[k];
    }
}

__global__ void __launch_bounds__(kLevelBlock) k_bvh_swap(const BTask* __restrict__ tasks,
                                                          const int2* __restrict__ chunks, const int* __restrict__ R,
                                                          const int* __restrict__ L, int* __restrict__ perm,
                                                          BuildCounters* __restrict__ ctr)
{
    const int2 ch = chunks[blockIdx.x];
    const BTask& t = tasks[ch.x];
    if (t.axis < 0) return;
    const int k0 = ch.y * kChunk, k1 = min(k0 + kChunk, t.r);
    for (int k = k0 + (int)threadIdx.x; k < k1; k += kLevelBlock) {
        const int a = R[t.begin + k], b = L[t.begin + k];
        if (a < t.begin || a >= t.mid || b < t.mid || b >= t.begin + t.count) {
            ctr->error = 5;
            continue;
        }
        const int x = perm[a];
        perm[a] = perm[b];
        perm[b] = x;
    }
}

// The host recursion over one small node, run by one thread: nodes go to
// out[0 ..) in depth-first preorder with indices local to the subtree.
__global__ void __launch_bounds__(128) k_bvh_small(const BTri* __restrict__ T, int* __restrict__ perm,
                                                   SmallTask* __restrict__ small, int nsmall,
                                                   pcr_bvh_node* __restrict__ region)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsmall) return;
    SmallTask st = small[i];
    pcr_bvh_node* out = region + 2 * (size_t)st.begin;
    int stk_b[kSmall], stk_e[kSmall], stk_p[kSmall];
    int sp = 0, n = 0;
    int b = st.begin, e = st.begin + st.count, par = -1;
    for (;;) {
        const int idx = n++;
        if (par >= 0) out[par].right_child = idx;
        float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        float cmn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int p = b; p < e; p++) {
            const BTri r = T[perm[p]];
            for (int a = 0; a < 3; a++) {
                const float l = getc(r.lo, a), h = getc(r.hi, a), c = getc(r.c, a);
                if (l < mn[a]) mn[a] = l;
                if (h > mx[a]) mx[a] = h;
                if (c < cmn[a]) cmn[a] = c;
                if (c > cmx[a]) cmx[a] = c;
            }
        }
        pcr_bvh_node& N = out[idx];
        for (int a = 0; a < 3; a++) { N.bmin[a] = mn[a]; N.bmax[a] = mx[a]; }
        const int count = e - b;
        int best_axis = -1, best_bin = -1, best_lc = 0;
        if (count > 4) {
            float best_cost = FLT_MAX;
            const float parent = box_area(mn, mx);
            if (parent > 0.f) {
                for (int a = 0; a < 3; a++) {
                    const float lo = cmn[a], ext = __fsub_rn(cmx[a], lo);
                    if (ext < 1e-6f) continue;
                    const float scale = __fdiv_rn((float)kBins, ext);
                    float bmn[kBins][3], bmx[kBins][3];
                    int cnt[kBins];
                    for (int q = 0; q < kBins; q++) {
                        cnt[q] = 0;
                        for (int k = 0; k < 3; k++) { bmn[q][k] = FLT_MAX; bmx[q][k] = -FLT_MAX; }
                    }
                    for (int p = b; p < e; p++) {
                        const BTri r = T[perm[p]];
                        const int q = bin_of(getc(r.c, a), lo, scale);
                        for (int k = 0; k < 3; k++) {
                            const float l = getc(r.lo, k), h = getc(r.hi, k);
                            if (l < bmn[q][k]) bmn[q][k] = l;
                            if (h > bmx[q][k]) bmx[q][k] = h;
                        }
                        cnt[q]++;
                    }
                    sah_axis(bmn, bmx, cnt, parent, a, best_cost, best_axis, best_bin, best_lc);
                }
            }
            if (best_axis >= 0 && best_cost >= __fmul_rn((float)count, 2.f)) best_axis = -1;
        }
        int mid = b;
        if (best_axis >= 0) {
            const float lo = cmn[best_axis], scale = __fdiv_rn((float)kBins, __fsub_rn(cmx[best_axis], lo));
            // std::partition, bidirectional form: two cursors swapping
            // misplaced triangles
            int first = b, last = e;
            for (;;) {
                while (first != last && bin_of(getc(T[perm[first]].c, best_axis), lo, scale) <= best_bin) first++;
                if (first == last) break;
                last--;
                while (first != last && bin_of(getc(T[perm[last]].c, best_axis), lo, scale) > best_bin) last--;
                if (first == last) break;
                const int x = perm[first];
                perm[first] = perm[last];
                perm[last] = x;
                first++;
            }
            mid = first;
        }
        if (best_axis < 0 || mid == b || mid == e) {
            N.left_or_first = b;
            N.right_child = 0;
            N.count = count;
            if (sp == 0) break;
            sp--;
            b = stk_b[sp];
            e = stk_e[sp];
            par = stk_p[sp];
        } else {
            N.left_or_first = idx + 1;
            N.right_child = -1;
            N.count = 0;
            stk_b[sp] = mid;
            stk_e[sp] = e;
            stk_p[sp] = idx;
            sp++;
            e = mid;
            par = -1;
        }
    }
    small[i].nnodes = n;
}

// Renumbering into depth-first preorder: pre[slot] for the level-built
// nodes, and each small subtree shifted by its root's preorder index.
__global__ void k_bvh_emit_top(const TopNode* __restrict__ top, int ntop, const int* __restrict__ pre,
                               pcr_bvh_node* __restrict__ out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ntop) return;
    const TopNode N = top[s];
    if (N.kind == 2) return;
    pcr_bvh_node o;
    for (int a = 0; a < 3; a++) { o.bmin[a] = N.bmin[a]; o.bmax[a] = N.bmax[a]; }
    if (N.kind == 0) {
        o.left_or_first = pre[N.left];
        o.right_child = pre[N.right];
        o.count = 0;
    } else {
        o.left_or_first = N.left;
        o.right_child = 0;
        o.count = N.count;
    }
    out[pre[s]] = o;
}

__global__ void k_bvh_emit_small(const SmallTask* __restrict__ small, int nsmall, const int* __restrict__ pre,
                                 const pcr_bvh_node* __restrict__ region, pcr_bvh_node* __restrict__ out,
                                 int total)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nsmall) return;
    const SmallTask st = small[w];
    const int base = pre[st.slot];
    const pcr_bvh_node* src = region + 2 * (size_t)st.begin;
    if (base < 0 || base + st.nnodes > total) return;   // the host checked the sizes
    for (int j = lane; j < st.nnodes; j += 32) {
        pcr_bvh_node o = src[j];
        if (o.count == 0) {
            o.left_or_first += base;
            o.right_child += base;
        }
        out[base + j] = o;
    }
}

#define BK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            throw PcrError(e_ == cudaErrorMemoryAllocation ? PCR_ERR_NO_MEMORY : PCR_ERR_CUDA,     \
                           std::string("BVH build: ") + #call + ": " + cudaGetErrorString(e_));    \
    } while (0)

// Workspace from the caller's pool (stream-ordered), returned when the
// build ends or throws.
struct DevBuf {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    ~DevBuf()
    {
        if (p) {
            cudaFreeAsync(p, st);
            cudaStreamSynchronize(st);
        }
    }
};

inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

inline unsigned blocks(long long n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

void device_build_bvh_raw(int device, cudaStream_t st, cudaMemPool_t pool, const float* verts9, int n,
                          std::vector<pcr_bvh_node>& nodes, std::vector<int32_t>& order)
{
    nodes.clear();
    order.clear();
    if (n <= 0) return;
    if (n > (1 << 28)) throw PcrError(PCR_ERR_INVALID, "BVH build: more than 2^28 triangles");
    BK(cudaSetDevice(device));
    const size_t N = (size_t)n;
    const int cap_tasks = n / (kSmall + 1) + 1;          // large nodes of one level are disjoint
    const int cap_chunks = n / kChunk + cap_tasks + 1;
    // carve one allocation
    size_t off = 0;
    auto carve = [&](size_t bytes) { const size_t o = off; off += up256(bytes); return o; };
    const size_t o_verts = carve(N * 9 * sizeof(float)), o_T = carve(N * sizeof(BTri)), o_perm = carve(N * 4),
                 o_side = carve(N), o_R = carve(N * 4), o_L = carve(N * 4),
                 o_top = carve((2 * N + 1) * sizeof(TopNode)), o_small = carve((N + 1) * sizeof(SmallTask)),
                 o_region = carve(2 * N * sizeof(pcr_bvh_node)), o_out = carve(2 * N * sizeof(pcr_bvh_node)),
                 o_pre = carve((2 * N + 1) * 4), o_tasks0 = carve((size_t)cap_tasks * sizeof(BTask)),
                 o_tasks1 = carve((size_t)cap_tasks * sizeof(BTask)), o_ch0 = carve((size_t)cap_chunks * 8),
                 o_ch1 = carve((size_t)cap_chunks * 8), o_cleft = carve((size_t)cap_chunks * 4),
                 o_coff = carve((size_t)cap_chunks * 4), o_bins = carve((size_t)cap_tasks * 3 * kBins * 6 * 4),
                 o_bcnt = carve((size_t)cap_tasks * 3 * kBins * 4), o_ctr = carve(sizeof(BuildCounters));
    DevBuf mem;
    mem.st = st;
    if (pool) BK(cudaMallocFromPoolAsync(&mem.p, off, pool, st));
    else BK(cudaMallocAsync(&mem.p, off, st));
    char* base = static_cast<char*>(mem.p);
    float* d_verts = reinterpret_cast<float*>(base + o_verts);
    BTri* T = reinterpret_cast<BTri*>(base + o_T);
    int* perm = reinterpret_cast<int*>(base + o_perm);
    unsigned char* side = reinterpret_cast<unsigned char*>(base + o_side);
    int* R = reinterpret_cast<int*>(base + o_R);
    int* L = reinterpret_cast<int*>(base + o_L);
    TopNode* top = reinterpret_cast<TopNode*>(base + o_top);
    SmallTask* small = reinterpret_cast<SmallTask*>(base + o_small);
    pcr_bvh_node* region = reinterpret_cast<pcr_bvh_node*>(base + o_region);
    pcr_bvh_node* out = reinterpret_cast<pcr_bvh_node*>(base + o_out);
    int* pre = reinterpret_cast<int*>(base + o_pre);
    BTask* tasks[2] = {reinterpret_cast<BTask*>(base + o_tasks0), reinterpret_cast<BTask*>(base + o_tasks1)};
    int2* chunks[2] = {reinterpret_cast<int2*>(base + o_ch0), reinterpret_cast<int2*>(base + o_ch1)};
    int* cleft = reinterpret_cast<int*>(base + o_cleft);
    int* coff = reinterpret_cast<int*>(base + o_coff);
    unsigned* bins = reinterpret_cast<unsigned*>(base + o_bins);
    int* bcnt = reinterpret_cast<int*>(base + o_bcnt);
    BuildCounters* ctr = reinterpret_cast<BuildCounters*>(base + o_ctr);

    BK(cudaMemcpyAsync(d_verts, verts9, N * 9 * sizeof(float), cudaMemcpyHostToDevice, st));
    k_bvh_prep<<<blocks(n, 256), 256, 0, st>>>(d_verts, n, T, perm);
    BK(cudaGetLastError());

    // the root: a level task, or a small task on its own
    BuildCounters hc{1, 0, 0, 0, 0};
    const Caps cap{(int)(2 * N + 1), cap_tasks, cap_chunks, (int)(N + 1)};
    TopNode root{};
    int ntasks = 0, nchunks = 0;
    if (n > kSmall) {
        BTask t{};
        t.begin = 0;
        t.count = n;
        t.slot = 0;
        t.cbase = 0;
        t.nchunks = blocks(n, kChunk);
        std::vector<int2> ch(t.nchunks);
        for (int q = 0; q < t.nchunks; q++) ch[q] = make_int2(0, q);
        BK(cudaMemcpyAsync(tasks[0], &t, sizeof(t), cudaMemcpyHostToDevice, st));
        BK(cudaMemcpyAsync(chunks[0], ch.data(), ch.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
        BK(cudaStreamSynchronize(st));   // host sources go out of scope
        ntasks = 1;
        nchunks = t.nchunks;
    } else {
        SmallTask s{0, n, 0, 0};
        root.ref = 0;
        hc.nsmall = 1;
        BK(cudaMemcpyAsync(small, &s, sizeof(s), cudaMemcpyHostToDevice, st));
        BK(cudaStreamSynchronize(st));
    }
    root.kind = n > kSmall ? 0 : 2;
    BK(cudaMemcpyAsync(top, &root, sizeof(root), cudaMemcpyHostToDevice, st));
    BK(cudaMemcpyAsync(ctr, &hc, sizeof(hc), cudaMemcpyHostToDevice, st));
    BK(cudaStreamSynchronize(st));

    int cur = 0;
    while (ntasks > 0) {
        if (ntasks > cap_tasks || nchunks > cap_chunks) throw PcrError(PCR_ERR_DEVICE_STATUS, "BVH build: level overflow");
        const int nxt = cur ^ 1;
        k_bvh_init<<<blocks((long long)ntasks * 3 * kBins, 256), 256, 0, st>>>(tasks[cur], ntasks, bins, bcnt);
        k_bvh_bounds<<<nchunks, kLevelBlock, 0, st>>>(T, perm, tasks[cur], chunks[cur]);
        k_bvh_bins<<<nchunks, kLevelBlock, 0, st>>>(T, perm, tasks[cur], chunks[cur], bins, bcnt);
        BK(cudaMemsetAsync(&ctr->ntasks, 0, 2 * sizeof(int), st));
        k_bvh_split<<<blocks(ntasks, 128), 128, 0, st>>>(T, perm, tasks[cur], ntasks, bins, bcnt, top, small,
                                                         LevelOut{tasks[nxt], chunks[nxt]}, ctr, cap);
        k_bvh_classify<<<nchunks, kLevelBlock, 0, st>>>(T, perm, tasks[cur], chunks[cur], side, cleft);
        k_bvh_scan<<<blocks(ntasks, 128), 128, 0, st>>>(tasks[cur], ntasks, side, cleft, coff, ctr);
        k_bvh_ranks<<<nchunks, kLevelBlock, 0, st>>>(tasks[cur], chunks[cur], side, coff, R, L);
        k_bvh_swap<<<nchunks, kLevelBlock, 0, st>>>(tasks[cur], chunks[cur], R, L, perm, ctr);
        BK(cudaGetLastError());
        BK(cudaMemcpyAsync(&hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost, st));
        BK(cudaStreamSynchronize(st));
        if (hc.error) throw PcrError(PCR_ERR_DEVICE_STATUS, "BVH build: check " + std::to_string(hc.error) + " failed");
        ntasks = hc.ntasks;
        nchunks = hc.nchunks;
        cur = nxt;
    }
    const int ntop = hc.ntop, nsmall = hc.nsmall;
    if (nsmall > 0) k_bvh_small<<<blocks(nsmall, 128), 128, 0, st>>>(T, perm, small, nsmall, region);
    BK(cudaGetLastError());

    // preorder numbering of the level-built part (children always have
    // larger slots than their parent)
    std::vector<TopNode> ht(ntop);
    std::vector<SmallTask> hs(nsmall);
    BK(cudaMemcpyAsync(ht.data(), top, ntop * sizeof(TopNode), cudaMemcpyDeviceToHost, st));
    if (nsmall) BK(cudaMemcpyAsync(hs.data(), small, nsmall * sizeof(SmallTask), cudaMemcpyDeviceToHost, st));
    BK(cudaStreamSynchronize(st));
    std::vector<long long> size(ntop);
    for (int s = 0; s < ntop; s++) {
        const TopNode& t = ht[s];
        const bool ok = t.kind == 1 || (t.kind == 2 && t.ref >= 0 && t.ref < nsmall && hs[t.ref].nnodes > 0) ||
                        (t.kind == 0 && t.left > s && t.left < ntop && t.right > s && t.right < ntop);
        if (!ok) throw PcrError(PCR_ERR_DEVICE_STATUS, "BVH build: inconsistent node " + std::to_string(s));
    }
    for (int s = ntop - 1; s >= 0; s--) {
        const TopNode& t = ht[s];
        if (t.kind == 1) size[s] = 1;
        else if (t.kind == 2) size[s] = hs[t.ref].nnodes;
        else size[s] = 1 + size[t.left] + size[t.right];
    }
    const long long total = size[0];
    if (total <= 0 || total > 2 * (long long)n) throw PcrError(PCR_ERR_DEVICE_STATUS, "BVH build: bad node count");
    std::vector<int> hpre(ntop, 0);
    for (int s = 0; s < ntop; s++) {
        const TopNode& t = ht[s];
        if (t.kind != 0) continue;
        hpre[t.left] = hpre[s] + 1;
        hpre[t.right] = hpre[s] + 1 + (int)size[t.left];
    }
    BK(cudaMemcpyAsync(pre, hpre.data(), ntop * sizeof(int), cudaMemcpyHostToDevice, st));
    k_bvh_emit_top<<<blocks(ntop, 128), 128, 0, st>>>(top, ntop, pre, out);
    if (nsmall) k_bvh_emit_small<<<blocks((long long)nsmall * 32, 256), 256, 0, st>>>(small, nsmall, pre, region, out, (int)total);
    BK(cudaGetLastError());
    nodes.resize((size_t)total);
    order.resize(N);
    BK(cudaMemcpyAsync(nodes.data(), out, (size_t)total * sizeof(pcr_bvh_node), cudaMemcpyDeviceToHost, st));
    BK(cudaMemcpyAsync(order.data(), perm, N * 4, cudaMemcpyDeviceToHost, st));
    BK(cudaStreamSynchronize(st));
}

std::vector<pcr_bvh_node> device_build_bvh(int device, cudaStream_t st, cudaMemPool_t pool,
                                           std::vector<pcr_triangle>& tris, std::vector<int32_t>* ids)
{
    std::vector<pcr_bvh_node> nodes;
    std::vector<int32_t> order;
    const int n = (int)tris.size();
    std::vector<float> v((size_t)n * 9);
    parallel_for(n, [&](int lo, int hi) {
        for (int i = lo; i < hi; i++)
            for (int a = 0; a < 3; a++) {
                v[(size_t)i * 9 + a] = tris[i].v0[a];
                v[(size_t)i * 9 + 3 + a] = tris[i].v1[a];
                v[(size_t)i * 9 + 6 + a] = tris[i].v2[a];
            }
    });
    device_build_bvh_raw(device, st, pool, v.data(), n, nodes, order);
    std::vector<pcr_triangle> t2(tris.size());
    std::vector<int32_t> i2(ids ? ids->size() : 0);
    parallel_for(n, [&](int lo, int hi) {
        for (int i = lo; i < hi; i++) {
            t2[i] = tris[order[i]];
            if (ids) i2[i] = (*ids)[order[i]];
        }
    });
    tris.swap(t2);
    if (ids) ids->swap(i2);
    return nodes;
}

}  // namespace pcr
