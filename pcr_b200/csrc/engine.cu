// Host side of the wavefront engine.  See engine.h.
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "bvh_build.h"
#include "kernels.cuh"
#include "scene.h"

namespace pcr {

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            throw PcrError(e_ == cudaErrorMemoryAllocation ? PCR_ERR_NO_MEMORY : PCR_ERR_CUDA,     \
                           std::string(#call) + ": " + cudaGetErrorString(e_));                    \
    } while (0)

// ---------------------------------------------------------------- small setter kernels
// Request entries and the active list travel as kernel parameters, which
// the launch copies, so the host never races an in-flight copy.
struct ActiveList { int n; int slots[kMaxActive]; };

__global__ void k_admit(EngineView E, DRequest r, int slot)
{
    const_cast<DRequest*>(E.reqs)[slot] = r;
    E.issued[slot] = 0ull;
    E.outstanding[slot] = 0;
    E.done_flag[slot] = 0;
    E.t_first[slot] = 0ull;
    E.t_done[slot] = 0ull;
    E.round_state[slot] = 0;
    E.round_cnt[slot] = 0;
}

// First adaptive round: every pixel, in order.
__global__ void k_iota(int* a, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

__global__ void k_set_active(EngineView E, ActiveList L)
{
    for (int i = threadIdx.x; i < L.n; i += blockDim.x) E.active[i] = L.slots[i];
    if (threadIdx.x == 0) *E.n_active = L.n;
}

__global__ void k_set_params(EngineParams* P, EngineParams p) { *P = p; }

// Cancels a running request: no path of it is issued after this point
// (its total becomes what was issued so far), so it finishes once the paths
// already in flight retire, within `depth` iterations.  Launched between
// blocks of iterations on the engine stream, so no kernel reads the entry
// while it changes.
__global__ void k_cancel(EngineView E, int slot)
{
    DRequest& R = const_cast<DRequest&>(E.reqs[slot]);
    R.flags |= kReqCancelled;
    R.total = (long long)E.issued[slot];
}

// ---------------------------------------------------------------- helpers
static float host_ybar_integral()
{
    // CIE::yBarIntegral (code/Includes/CIE.h:79-88), float arithmetic in the
    // reference's order (this file's host code is built without FMA contraction).
    auto wy = [](float l, float mu, float s1, float s2) {
        float t = (l < mu) ? (l - mu) * s1 : (l - mu) * s2;
        return std::exp(-0.5f * t * t);
    };
    float sum = 0.f;
    for (int i = 0; i < kSpecN; i++) {
        float l = 400.f + i * 5.0f;
        sum += 0.821f * wy(l, 568.8f, 0.0213f, 0.0247f) + 0.286f * wy(l, 530.9f, 0.0613f, 0.0322f);
    }
    return sum * 5.0f;
}

template <typename T>
static T* dalloc(size_t n, std::vector<void*>& track)
{
    T* p = nullptr;
    if (n == 0) n = 1;
    CK(cudaMalloc(&p, n * sizeof(T)));
    track.push_back(p);
    return p;
}

template <typename T>
static T* dupload(const std::vector<T>& v, std::vector<void*>& track, int64_t& bytes)
{
    T* p = dalloc<T>(v.size(), track);
    if (!v.empty()) CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    bytes += (int64_t)std::max<size_t>(1, v.size()) * sizeof(T);
    return p;
}

// ---------------------------------------------------------------- ctor / dtor
Engine::Engine(const pcr_ctx_opts* o)
{
    if (o) {
        device_ = o->device;
        if (o->memory_budget > 0) budget_ = o->memory_budget;
        if (o->queue_capacity > 0) tune_.queue_capacity = o->queue_capacity;
        if (o->block_size > 0) tune_.block_size = o->block_size;
        if (o->chunk_paths > 0) tune_.chunk_paths = o->chunk_paths;
        if (o->regen_every > 0) tune_.regen_every = o->regen_every;
        use_graph_ = o->use_graph != 0;
        profile_ = o->profile != 0;
        if (o->tuning_cache) tuning_cache_ = o->tuning_cache;
    }
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (ndev <= 0) throw PcrError(PCR_ERR_CUDA, "no CUDA device");
    if (device_ < 0 || device_ >= ndev) throw PcrError(PCR_ERR_INVALID, "device ordinal out of range");
    CK(cudaSetDevice(device_));
    CK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_));
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&resolve_stream_, cudaStreamNonBlocking));
    xyz_scale_ = (700.f - 400.f) / host_ybar_integral();
    slot_owner_.assign(kMaxActive, -1);
    scenes_.reserve(256);
    for (auto& e : prof_ev_) CK(cudaEventCreate(&e));
    for (auto& e : ev_snaps_) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    // Per-request buffers come from the engine's own stream-ordered pool,
    // which keeps freed memory for reuse (release threshold: never) so that
    // a steady request stream does no device page mapping after warm-up.
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device_;
    CK(cudaMemPoolCreate(&pool_, &props));
    uint64_t keep = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep));
    alloc_buffers();
}

Engine::~Engine()
{
    try {
        serve_stop();
    } catch (...) {
    }
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);
    cudaStreamSynchronize(resolve_stream_);
    for (auto& kv : reqs_) {
        Request& r = *kv.second;
        if (r.accum) cudaFreeAsync(r.accum, stream_);
        for (int k = 0; k < 2; k++)
            if (r.act[k]) cudaFreeAsync(r.act[k], stream_);
        if (r.welford) cudaFreeAsync(r.welford, stream_);
        if (r.d_hdr) cudaFreeAsync(r.d_hdr, stream_);
        if (r.d_rgb) cudaFreeAsync(r.d_rgb, stream_);
        if (r.ev_ready) cudaEventDestroy(r.ev_ready);
    }
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(resolve_stream_);
    for (Staging& st : staging_idle_) {
        cudaStreamSynchronize(st.stream);
        if (st.buf) cudaFreeHost(st.buf);
        cudaStreamDestroy(st.stream);
    }
    for (auto& s : scenes_)
        for (void* p : s.allocs) cudaFree(p);
    free_buffers();
    for (auto& e : prof_ev_) cudaEventDestroy(e);
    for (auto& e : ev_snaps_) cudaEventDestroy(e);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (pool_) cudaMemPoolDestroy(pool_);
    cudaStreamDestroy(stream_);
}

void Engine::alloc_buffers()
{
    std::vector<void*>& T = qallocs_;
    d_scenes_ = dalloc<DScene>(256, T);
    mat_cap_ = 256;
    d_mats_ = dalloc<DMaterial>(mat_cap_, T);
    d_reqs_ = dalloc<DRequest>(kMaxActive, T);
    CK(cudaMemset(d_reqs_, 0, sizeof(DRequest) * kMaxActive));
    d_issued_ = dalloc<unsigned long long>(kMaxActive, T);
    d_tfirst_ = dalloc<unsigned long long>(kMaxActive, T);
    d_tdone_ = dalloc<unsigned long long>(kMaxActive, T);
    d_outstanding_ = dalloc<long long>(kMaxActive, T);
    d_give_start_ = dalloc<long long>(kMaxActive, T);
    d_give_ = dalloc<int>(kMaxActive, T);
    d_give_base_ = dalloc<int>(kMaxActive, T);
    d_active_ = dalloc<int>(kMaxActive, T);
    d_nactive_ = dalloc<int>(1, T);
    d_done_ = dalloc<int>(kMaxActive, T);
    d_round_state_ = dalloc<int>(kMaxActive, T);
    d_round_cnt_ = dalloc<int>(kMaxActive, T);
    d_round_list_ = dalloc<int>(kMaxActive, T);
    d_cnt_ = dalloc<Counters>(1, T);
    d_params_ = dalloc<EngineParams>(1, T);
    d_cmf_ = dalloc<float4>(kCmfEntries, T);
    k_cmf_table<<<(kCmfEntries + 255) / 256, 256, 0, stream_>>>(d_cmf_);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemset(d_issued_, 0, 8 * kMaxActive));
    CK(cudaMemset(d_outstanding_, 0, 8 * kMaxActive));
    CK(cudaMemset(d_done_, 0, 4 * kMaxActive));
    CK(cudaMemset(d_round_state_, 0, 4 * kMaxActive));
    CK(cudaMemset(d_round_cnt_, 0, 4 * kMaxActive));
    CK(cudaMemset(d_nactive_, 0, 4));
    CK(cudaMemset(d_cnt_, 0, sizeof(Counters)));
    for (auto& h : h_snaps_) {
        CK(cudaMallocHost(&h, sizeof(HostSnap)));
        std::memset(h, 0, sizeof(HostSnap));
    }
    h_snap_ = h_snaps_[0];
    snap_next_ = 0;
    snap_inflight_ = 0;
    CK(cudaMallocHost(&h_params_, sizeof(EngineParams)));

    const int fill = tune_.queue_capacity;
    queue_cap_ = fill * 4;   // a dispersive-glass fork turns one path into up to four
    shadow_cap_ = (int)std::min<int64_t>((int64_t)queue_cap_ * 8, (1ll << 31) - 1);
    for (int b = 0; b < 2; b++) {
        q_[b].o = dalloc<float4>(queue_cap_, T);
        q_[b].d = dalloc<float4>(queue_cap_, T);
        q_[b].tp = dalloc<float4>(queue_cap_, T);
        q_[b].id = dalloc<int4>(queue_cap_, T);
        for (int k = 0; k < 3; k++) q_[b].w[k] = dalloc<float4>(queue_cap_, T);
    }
    d_hit_ = dalloc<float4>(queue_cap_, T);
    sq_.o = dalloc<float4>(shadow_cap_, T);
    sq_.d = dalloc<float4>(shadow_cap_, T);
    sq_.c = dalloc<float4>(shadow_cap_, T);
    EngineParams p{fill, tune_.chunk_paths, tune_.regen_every, 0};
    CK(cudaMemcpy(d_params_, &p, sizeof(p), cudaMemcpyHostToDevice));
    graph_dirty_ = true;
}

void Engine::free_buffers()
{
    for (void* p : qallocs_) cudaFree(p);
    qallocs_.clear();
    for (auto& h : h_snaps_) {
        if (h) cudaFreeHost(h);
        h = nullptr;
    }
    if (h_params_) cudaFreeHost(h_params_);
    h_snap_ = nullptr;
    h_params_ = nullptr;
}

void Engine::set_tuning(const EngineTuning& t)
{
    std::lock_guard<std::mutex> g(run_mu_);
    for (int s : active_slots_)
        if (s >= 0) throw PcrError(PCR_ERR_INVALID, "cannot retune while requests are active");
    CK(cudaStreamSynchronize(stream_));
    // keep the scene and material tables; rebuild queues and the request table
    std::vector<DScene> sc(256);
    CK(cudaMemcpy(sc.data(), d_scenes_, sizeof(DScene) * 256, cudaMemcpyDeviceToHost));
    std::vector<DMaterial> mats(mat_count_);
    if (mat_count_) CK(cudaMemcpy(mats.data(), d_mats_, sizeof(DMaterial) * mat_count_, cudaMemcpyDeviceToHost));
    free_buffers();
    tune_ = t;
    if (tune_.iters_per_launch < 2) tune_.iters_per_launch = 2;
    if (tune_.iters_per_launch & 1) tune_.iters_per_launch++;
    alloc_buffers();
    if (mat_count_ > mat_cap_) {
        mat_cap_ = mat_count_;
    }
    CK(cudaMemcpy(d_scenes_, sc.data(), sizeof(DScene) * 256, cudaMemcpyHostToDevice));
    if (mat_count_) {
        if (mat_count_ > 256) {
            CK(cudaFree(d_mats_));
            qallocs_.erase(std::find(qallocs_.begin(), qallocs_.end(), (void*)d_mats_));
            d_mats_ = dalloc<DMaterial>(mat_cap_, qallocs_);
        }
        CK(cudaMemcpy(d_mats_, mats.data(), sizeof(DMaterial) * mat_count_, cudaMemcpyHostToDevice));
    }
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
    graph_dirty_ = true;
}

EngineView Engine::view() const
{
    EngineView E{};
    E.scenes = d_scenes_;
    E.mats = d_mats_;
    E.reqs = d_reqs_;
    E.issued = d_issued_;
    E.outstanding = d_outstanding_;
    E.give = d_give_;
    E.give_base = d_give_base_;
    E.active = d_active_;
    E.n_active = d_nactive_;
    E.done_flag = d_done_;
    E.t_first = d_tfirst_;
    E.t_done = d_tdone_;
    E.cnt = d_cnt_;
    E.q[0] = q_[0];
    E.q[1] = q_[1];
    E.hit = d_hit_;
    E.sq = sq_;
    E.give_start = d_give_start_;
    E.shadow_cap = shadow_cap_;
    E.queue_cap = queue_cap_;
    E.n_mats = mat_count_;
    E.round_state = d_round_state_;
    E.round_cnt = d_round_cnt_;
    E.round_list = d_round_list_;
    E.cmf_table = d_cmf_;
    return E;
}

// ---------------------------------------------------------------- scenes
// Splits the plane list into runs of consecutive planes, each run either one
// plane tested directly or several tested behind one box test (a box
// primitive's six faces), so the closest-hit loop skips a run the ray cannot
// reach.  The split minimises an expected cost by dynamic programming over
// run boundaries: a lone plane costs 1 test, a boxed run of k planes costs
// 0.6 (the box test) + k * P(hit).  P(hit) for rays that mostly start inside
// the scene is estimated as the run box's share of the whole plane set's
// volume (the origin lies inside it) plus its share of the surface area.  The order of the planes, and so the reference's
// first-tested-wins tie rule, is unchanged.  Boxes are padded by 1e-4 times
// the scene's largest coordinate (at least 1e-4), far above the rounding
// error of a computed hit point.
static std::vector<float4> plane_groups(const pcr_plane* p, int n)
{
    struct Box {
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        void add(float x, float y, float z) {
            const float v[3] = {x, y, z};
            for (int k = 0; k < 3; k++) { lo[k] = std::min(lo[k], v[k]); hi[k] = std::max(hi[k], v[k]); }
        }
        void add(const Box& b) { add(b.lo[0], b.lo[1], b.lo[2]); add(b.hi[0], b.hi[1], b.hi[2]); }
        double area() const {
            const double x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
            return 2.0 * (x * y + y * z + z * x);
        }
        double volume() const {
            return (double)(hi[0] - lo[0]) * (double)(hi[1] - lo[1]) * (double)(hi[2] - lo[2]);
        }
    };
    std::vector<Box> b(n);
    Box all;
    float big = 1.f;
    for (int i = 0; i < n; i++) {
        const float* o = p[i].origin;
        const float* u = p[i].u;
        const float* v = p[i].v;
        b[i].add(o[0], o[1], o[2]);
        b[i].add(o[0] + u[0], o[1] + u[1], o[2] + u[2]);
        b[i].add(o[0] + v[0], o[1] + v[1], o[2] + v[2]);
        b[i].add(o[0] + u[0] + v[0], o[1] + u[1] + v[1], o[2] + u[2] + v[2]);
        all.add(b[i]);
        for (int k = 0; k < 3; k++) big = std::max(big, std::max(std::fabs(b[i].lo[k]), std::fabs(b[i].hi[k])));
    }
    const double total = std::max(all.area(), 1e-30), total_v = std::max(all.volume(), 1e-30);
    // best[j]: cost of planes [0, j); from[j]: start of the last run
    std::vector<double> best(n + 1, 0.0);
    std::vector<int> from(n + 1, 0);
    for (int j = 1; j <= n; j++) {
        best[j] = best[j - 1] + 1.0;
        from[j] = j - 1;
        Box g = b[j - 1];
        for (int i = j - 2; i >= 0 && j - i <= 64; i--) {
            g.add(b[i]);
            const double c = best[i] + 0.6 + (j - i) * std::min(1.0, g.area() / total + g.volume() / total_v);
            if (c < best[j]) { best[j] = c; from[j] = i; }
        }
    }
    std::vector<std::pair<int, int>> runs;
    for (int j = n; j > 0; j = from[j]) runs.push_back({from[j], j});
    std::reverse(runs.begin(), runs.end());
    const float pad = 1e-4f * big;
    std::vector<float4> out;
    for (auto [i, j] : runs) {
        Box g;
        for (int k = i; k < j; k++) g.add(b[k]);
        out.push_back(make_float4(g.lo[0] - pad, g.lo[1] - pad, g.lo[2] - pad, __int_as_float_host(i)));
        out.push_back(make_float4(g.hi[0] + pad, g.hi[1] + pad, g.hi[2] + pad, __int_as_float_host(j - i)));
    }
    return out;
}

int Engine::upload_scene(const pcr_scene_desc& d)
{
    std::lock_guard<std::mutex> g(run_mu_);
    CK(cudaSetDevice(device_));
    if (d.n_materials <= 0 || !d.materials) throw PcrError(PCR_ERR_INVALID, "scene has no materials");
    if (d.n_lights <= 0 || !d.lights) throw PcrError(PCR_ERR_INVALID, "scene has no area light");
    if (d.n_planes < 0 || d.n_spheres < 0 || d.n_triangles < 0 || d.n_bvh_nodes < 0)
        throw PcrError(PCR_ERR_INVALID, "negative count in scene descriptor");
    if ((d.n_planes && !d.planes) || (d.n_spheres && !d.spheres) || (d.n_triangles && !d.triangles))
        throw PcrError(PCR_ERR_INVALID, "null array with non-zero count");
    int sid = -1;
    for (size_t i = 0; i < scenes_.size(); i++)
        if (!scenes_[i].live) { sid = (int)i; break; }
    if (sid < 0) {
        if (scenes_.size() >= 256) throw PcrError(PCR_ERR_NO_MEMORY, "scene cache full (256 scenes)");
        scenes_.emplace_back();
        sid = (int)scenes_.size() - 1;
    }
    SceneEntry e;
    e.name = d.name ? d.name : "";
    e.version = d.version ? d.version : "";
    std::memcpy(e.cam, d.cam_pos, sizeof(e.cam));
    e.fov = d.fov;

    // triangles + BVH (built here on the device, equal to the reference's
    // builder, when the descriptor has none)
    // (copies only when the triangles must be put into leaf order here)
    std::vector<pcr_triangle> own_tris;
    std::vector<int32_t> own_ids;
    const pcr_triangle* tris = d.triangles;
    const int32_t* ids = d.triangle_ids;
    std::vector<pcr_bvh_node> bvh;
    if (d.n_triangles > 0) {
        if (d.n_bvh_nodes > 0 && d.bvh_nodes) {
            bvh.assign(d.bvh_nodes, d.bvh_nodes + d.n_bvh_nodes);
        } else {
            own_tris.assign(d.triangles, d.triangles + d.n_triangles);
            own_ids.resize(d.n_triangles);
            for (int i = 0; i < d.n_triangles; i++) own_ids[i] = d.triangle_ids ? d.triangle_ids[i] : i;
            bvh = device_build_bvh(device_, stream_, pool_, own_tris, &own_ids);
            tris = own_tris.data();
            ids = own_ids.data();
        }
    }
    for (const auto& n : bvh)
        if (n.count == 0 && (n.left_or_first < 0 || n.left_or_first >= (int)bvh.size() || n.right_child < 0 ||
                             n.right_child >= (int)bvh.size()))
            throw PcrError(PCR_ERR_INVALID, "BVH child index out of range");
    std::vector<DNode4> nodes4 = collapse_bvh4(bvh, d.n_triangles);

    // materials
    for (int i = 0; i < d.n_materials; i++) {
        const pcr_material& m = d.materials[i];
        DMaterial M{};
        M.flags = (m.emissive[0] > 0 || m.emissive[1] > 0 || m.emissive[2] > 0 ? kMatEmissive : 0) |
                  (m.metallic ? kMatMetallic : 0) | (m.transparent ? kMatTransparent : 0) |
                  (m.use_tab_albedo ? kMatTabA : 0) | (m.use_tab_emissive ? kMatTabE : 0);
        M.ior = m.ior;
        M.cauchyB = m.cauchy_b;
        M.albedo_max = std::max(m.albedo[0], std::max(m.albedo[1], m.albedo[2]));
        M.albedo = make_float4(m.albedo[0], m.albedo[1], m.albedo[2], 0.f);
        M.emissive = make_float4(m.emissive[0], m.emissive[1], m.emissive[2], 0.f);
        M.afit = make_float4(m.albedo_fit[0], m.albedo_fit[1], m.albedo_fit[2], m.albedo_fit[3]);
        M.efit = make_float4(m.emissive_fit[0], m.emissive_fit[1], m.emissive_fit[2], m.emissive_fit[3]);
        for (int k = 0; k < kSpecN; k++) {
            M.tabA[k] = m.tab_albedo[k];
            M.tabE[k] = m.tab_emissive[k];
        }
        e.mats.push_back(M);
    }
    auto check_mat = [&](int m, const char* what) {
        if (m < 0 || m >= d.n_materials) throw PcrError(PCR_ERR_INVALID, std::string(what) + ": material index out of range");
    };

    std::vector<DPlane> planes(d.n_planes);
    for (int i = 0; i < d.n_planes; i++) {
        const pcr_plane& p = d.planes[i];
        check_mat(p.mat, "plane");
        DPlane P;
        P.o_mat = make_float4(p.origin[0], p.origin[1], p.origin[2], __int_as_float_host(p.mat));
        P.n_emit = make_float4(p.n[0], p.n[1], p.n[2], (e.mats[p.mat].flags & kMatEmissive) ? 1.f : 0.f);
        // u.dot(u) exactly as Plane::intersect computes it (code/Includes/Plane.h:46-47)
        float uu = p.u[0] * p.u[0] + p.u[1] * p.u[1] + p.u[2] * p.u[2];
        float vv = p.v[0] * p.v[0] + p.v[1] * p.v[1] + p.v[2] * p.v[2];
        P.u_uu = make_float4(p.u[0], p.u[1], p.u[2], uu);
        P.v_vv = make_float4(p.v[0], p.v[1], p.v[2], vv);
        planes[i] = P;
    }
    std::vector<DSphere> spheres(d.n_spheres);
    for (int i = 0; i < d.n_spheres; i++) {
        const pcr_sphere& s = d.spheres[i];
        check_mat(s.mat, "sphere");
        spheres[i].c_r = make_float4(s.center[0], s.center[1], s.center[2], s.radius);
        spheres[i].mat = make_int4(s.mat, (e.mats[s.mat].flags & kMatEmissive) ? 1 : 0, 0, 0);
    }
    auto to_dtri = [&](const pcr_triangle& t, int id) {
        DTri T;
        float e1[3], e2[3];
        for (int k = 0; k < 3; k++) {
            e1[k] = t.v1[k] - t.v0[k];
            e2[k] = t.v2[k] - t.v0[k];
        }
        T.v0_id = make_float4(t.v0[0], t.v0[1], t.v0[2], __int_as_float_host(id));
        T.e1_mat = make_float4(e1[0], e1[1], e1[2], __int_as_float_host(t.mat));
        T.e2_flags = make_float4(e2[0], e2[1], e2[2], __int_as_float_host(t.smooth ? 1 : 0));
        return T;
    };
    int emissive_tris = 0;
    for (int i = 0; i < d.n_triangles; i++) {
        check_mat(tris[i].mat, "triangle");
        if (e.mats[tris[i].mat].flags & kMatEmissive) emissive_tris = 1;
    }
    std::vector<DTri> dtris(d.n_triangles);
    std::vector<float4> tri_n((size_t)d.n_triangles * 3), tri_flat(d.n_triangles);
    parallel_for(d.n_triangles, [&](int lo, int hi) {
        for (int i = lo; i < hi; i++) {
            dtris[i] = to_dtri(tris[i], ids ? ids[i] : i);
            tri_n[i * 3 + 0] = make_float4(tris[i].n0[0], tris[i].n0[1], tris[i].n0[2], 0.f);
            tri_n[i * 3 + 1] = make_float4(tris[i].n1[0], tris[i].n1[1], tris[i].n1[2], 0.f);
            tri_n[i * 3 + 2] = make_float4(tris[i].n2[0], tris[i].n2[1], tris[i].n2[2], 0.f);
            tri_flat[i] = make_float4(tris[i].flat_n[0], tris[i].flat_n[1], tris[i].flat_n[2], 0.f);
        }
    });
    // lights
    std::vector<DLight> lights(d.n_lights);
    int n_lt = 0;
    for (int i = 0; i < d.n_lights; i++) {
        const pcr_light& L = d.lights[i];
        if (L.kind == 1) n_lt = std::max(n_lt, L.tri_offset + L.tri_count);
    }
    std::vector<DTri> ltris(n_lt);
    std::vector<float4> lflat(n_lt);
    std::vector<float> lcum(n_lt);
    float total_area = 0.f;
    for (int i = 0; i < d.n_lights; i++) {
        const pcr_light& L = d.lights[i];
        DLight D{};
        D.kind = L.kind;
        D.total_area = L.total_area;
        D.tri_offset = L.tri_offset;
        D.tri_count = L.tri_count;
        total_area += L.total_area;  // code/Renderer.cpp:134-136
        if (L.kind == 0) {
            check_mat(L.plane.mat, "light");
            D.o_mat = make_float4(L.plane.origin[0], L.plane.origin[1], L.plane.origin[2], __int_as_float_host(L.plane.mat));
            D.u = make_float4(L.plane.u[0], L.plane.u[1], L.plane.u[2], 0.f);
            D.v = make_float4(L.plane.v[0], L.plane.v[1], L.plane.v[2], 0.f);
            D.n = make_float4(L.plane.n[0], L.plane.n[1], L.plane.n[2], 0.f);
        } else {
            if (L.kind != 1 || L.tri_count <= 0 || L.tri_offset < 0 || !d.light_triangles || !d.light_cum_area)
                throw PcrError(PCR_ERR_INVALID, "bad triangle-set light");
            for (int k = L.tri_offset; k < L.tri_offset + L.tri_count; k++) {
                check_mat(d.light_triangles[k].mat, "light triangle");
                ltris[k] = to_dtri(d.light_triangles[k], k);
                lflat[k] = make_float4(d.light_triangles[k].flat_n[0], d.light_triangles[k].flat_n[1],
                                       d.light_triangles[k].flat_n[2], 0.f);
                lcum[k] = d.light_cum_area[k];
            }
        }
        lights[i] = D;
    }

    // material table growth
    if (mat_count_ + d.n_materials > mat_cap_) {
        int cap = std::max(mat_cap_ * 2, mat_count_ + d.n_materials);
        DMaterial* nm = nullptr;
        CK(cudaMalloc(&nm, sizeof(DMaterial) * cap));
        if (mat_count_) CK(cudaMemcpy(nm, d_mats_, sizeof(DMaterial) * mat_count_, cudaMemcpyDeviceToDevice));
        auto it = std::find(qallocs_.begin(), qallocs_.end(), (void*)d_mats_);
        if (it != qallocs_.end()) qallocs_.erase(it);
        CK(cudaStreamSynchronize(stream_));
        CK(cudaFree(d_mats_));
        d_mats_ = nm;
        qallocs_.push_back(nm);
        mat_cap_ = cap;
    }
    const int mat_base = mat_count_;
    CK(cudaMemcpy(d_mats_ + mat_base, e.mats.data(), sizeof(DMaterial) * d.n_materials, cudaMemcpyHostToDevice));
    mat_count_ += d.n_materials;

    int64_t bytes = (int64_t)sizeof(DMaterial) * d.n_materials;
    DScene S{};
    S.planes = dupload(planes, e.allocs, bytes);
    S.spheres = dupload(spheres, e.allocs, bytes);
    S.nodes = dupload(nodes4, e.allocs, bytes);
    S.tris = dupload(dtris, e.allocs, bytes);
    S.tri_n = dupload(tri_n, e.allocs, bytes);
    S.tri_flatn = dupload(tri_flat, e.allocs, bytes);
    S.lights = dupload(lights, e.allocs, bytes);
    S.light_tris = dupload(ltris, e.allocs, bytes);
    S.light_flatn = dupload(lflat, e.allocs, bytes);
    S.light_cum = dupload(lcum, e.allocs, bytes);
    const std::vector<float4> pgroups = plane_groups(d.planes, d.n_planes);
    S.pgroups = dupload(pgroups, e.allocs, bytes);
    S.n_pgroups = (int)pgroups.size() / 2;
    std::vector<pcr_plane> lit_src;
    std::vector<DPlane> splanes;
    for (int i = 0; i < d.n_planes; i++)
        if (planes[i].n_emit.w == 0.f) {
            lit_src.push_back(d.planes[i]);
            splanes.push_back(planes[i]);
        }
    const std::vector<float4> sgroups = plane_groups(lit_src.data(), (int)lit_src.size());
    S.splanes = dupload(splanes, e.allocs, bytes);
    S.sgroups = dupload(sgroups, e.allocs, bytes);
    S.n_sgroups = (int)sgroups.size() / 2;
    S.emissive_tris = emissive_tris;
    {
        int only = -1, n_emit = 0;
        for (int i = 0; i < d.n_materials; i++)
            if (e.mats[i].flags & kMatEmissive) { only = i; n_emit++; }
        bool all_lights = n_emit == 1;
        for (int i = 0; i < d.n_lights && all_lights; i++) {
            const pcr_light& L = d.lights[i];
            if (L.kind == 0) all_lights = L.plane.mat == only;
            else
                for (int k = L.tri_offset; k < L.tri_offset + L.tri_count; k++)
                    if (d.light_triangles[k].mat != only) all_lights = false;
        }
        S.emit_mat = all_lights ? only : -1;
    }
    S.n_emit_spheres = S.n_emit_planes = 0;
    for (int i = 0; i < d.n_spheres; i++)
        if (spheres[i].mat.y) {
            if (S.n_emit_spheres >= 0 && S.n_emit_spheres < kMaxEmitPrims) S.emit_spheres[S.n_emit_spheres++] = i;
            else S.n_emit_spheres = -1;
        }
    for (int i = 0; i < d.n_planes; i++)
        if (planes[i].n_emit.w != 0.f) {
            if (S.n_emit_planes >= 0 && S.n_emit_planes < kMaxEmitPrims) S.emit_planes[S.n_emit_planes++] = i;
            else S.n_emit_planes = -1;
        }
    S.n_planes = d.n_planes;
    S.n_spheres = d.n_spheres;
    S.n_nodes = (int)nodes4.size();
    S.n_tris = d.n_triangles;
    S.n_lights = d.n_lights;
    S.mat_base = mat_base;
    S.n_mats = d.n_materials;
    S.total_light_area = total_area;
    e.dev = S;
    e.bytes = bytes;
    e.live = true;
    CK(cudaMemcpy(d_scenes_ + sid, &S, sizeof(DScene), cudaMemcpyHostToDevice));
    scenes_[sid] = std::move(e);
    graph_dirty_ = true;
    return sid;
}

void Engine::release_scene(int id)
{
    std::lock_guard<std::mutex> g(run_mu_);
    if (id < 0 || id >= (int)scenes_.size() || !scenes_[id].live) throw PcrError(PCR_ERR_NOT_FOUND, "unknown scene");
    {
        std::lock_guard<std::mutex> l(mu_);
        for (auto& kv : reqs_)
            if (kv.second->scene == id && (kv.second->state == ReqState::Pending || kv.second->state == ReqState::Active))
                throw PcrError(PCR_ERR_INVALID, "scene is in use by a request");
    }
    CK(cudaStreamSynchronize(stream_));
    for (void* p : scenes_[id].allocs) cudaFree(p);
    scenes_[id].allocs.clear();
    scenes_[id].live = false;
    // material slots of released scenes are not compacted; the table only grows
}

int64_t Engine::scene_bytes(int id) const
{
    if (id < 0 || id >= (int)scenes_.size() || !scenes_[id].live) throw PcrError(PCR_ERR_NOT_FOUND, "unknown scene");
    return scenes_[id].bytes;
}

// ---------------------------------------------------------------- requests
void Engine::validate(int scene, const pcr_render_desc& d) const
{
    if (scene < 0 || scene >= (int)scenes_.size() || !scenes_[scene].live) throw PcrError(PCR_ERR_NOT_FOUND, "unknown scene");
    if (d.width <= 0 || d.height <= 0 || d.depth <= 0 || d.samples <= 0 || d.shadow_samples <= 0)
        throw PcrError(PCR_ERR_INVALID, "width, height, depth, samples and shadow samples must be positive");
    if (d.depth > 255) throw PcrError(PCR_ERR_INVALID, "depth above 255");
    if (d.shadow_samples > kMaxShadow) throw PcrError(PCR_ERR_INVALID, "more than 64 shadow samples per hit");
    const int64_t px = (int64_t)d.width * d.height;
    if (d.sample_end != 0 || d.sample_begin != 0) {
        if (d.sample_begin < 0 || d.sample_end <= d.sample_begin || d.sample_end > d.samples)
            throw PcrError(PCR_ERR_INVALID, "sample range must satisfy 0 <= sample_begin < sample_end <= samples");
        if (d.adaptive && d.aa_samples > 1)
            throw PcrError(PCR_ERR_INVALID, "a sample range cannot be combined with adaptive sampling");
    }
    const int64_t ppp = (int64_t)d.samples * std::max(1, d.aa_samples);
    if (px >= (1ll << 31) || ppp >= (1ll << 31) || px * ppp >= (1ll << 62))
        throw PcrError(PCR_ERR_INVALID, "render too large");
    if ((int64_t)queue_cap_ * d.shadow_samples >= (1ll << 31))
        throw PcrError(PCR_ERR_INVALID, "shadow samples x queue capacity above 2^31 shadow records");
}

// Adaptive sampling runs only with more than one aa sample per pixel (the
// convergence test needs 4 rounds; with aa = 1 there is a single round).
static bool adaptive_rounds(const pcr_render_desc& d) { return d.adaptive && d.aa_samples > 1; }

// The request's samples per aa round: [sample_begin, sample_end) of
// `samples`, or all of them.
static int local_spp(const pcr_render_desc& d)
{
    return d.sample_end > 0 ? d.sample_end - d.sample_begin : d.samples;
}

int64_t Engine::request_bytes(const pcr_render_desc& d) const
{
    const int64_t px = (int64_t)d.width * d.height;
    // accumulator, HDR, 8-bit (+ Welford state and two pixel lists when adaptive)
    return px * 3 * (8 + 4 + 1) + (adaptive_rounds(d) ? px * (32 + 8) : 0);
}

// The shadow queue holds shadow_samples records for every path slot of a
// launch (8 by default).  A request with more shadow samples grows it
// between iterations: shadow records never outlive the iteration that
// writes them, so the buffer can be replaced once the stream is drained.
// The caller holds run_mu_.
void Engine::ensure_shadow_capacity(int shadow_samples)
{
    const int64_t need = (int64_t)queue_cap_ * std::max(8, shadow_samples);
    if (need <= shadow_cap_) return;
    // shadow records are indexed with 32-bit ints (and 2^31 records would
    // take ~100 GB): the product must stay below 2^31
    if (need > (int64_t)INT32_MAX)
        throw PcrError(PCR_ERR_INVALID, std::to_string(shadow_samples) + " shadow samples per hit at " +
                                            std::to_string(tune_.queue_capacity) +
                                            " paths in flight exceed the 2^31-record shadow queue; use a smaller "
                                            "queue capacity");
    CK(cudaStreamSynchronize(stream_));
    for (float4* p : {sq_.o, sq_.d, sq_.c}) {
        auto it = std::find(qallocs_.begin(), qallocs_.end(), (void*)p);
        if (it != qallocs_.end()) qallocs_.erase(it);
        CK(cudaFree(p));
    }
    shadow_cap_ = (int)need;
    sq_.o = dalloc<float4>(shadow_cap_, qallocs_);
    sq_.d = dalloc<float4>(shadow_cap_, qallocs_);
    sq_.c = dalloc<float4>(shadow_cap_, qallocs_);
    graph_dirty_ = true;
}

int64_t Engine::submit(int scene, const pcr_render_desc& desc)
{
    validate(scene, desc);
    if ((int64_t)queue_cap_ * desc.shadow_samples > shadow_cap_) {
        std::lock_guard<std::mutex> g(run_mu_);
        ensure_shadow_capacity(desc.shadow_samples);
    }
    auto r = std::make_unique<Request>();
    r->scene = scene;
    r->desc = desc;
    r->bytes = request_bytes(desc);
    if (r->bytes > budget_) throw PcrError(PCR_ERR_NO_MEMORY, "request larger than the device memory budget");
    r->t_submit = std::chrono::steady_clock::now();
    int64_t id;
    {
        std::lock_guard<std::mutex> g(mu_);
        id = next_id_++;
        r->id = id;
        const int prio = desc.priority;
        reqs_[id] = std::move(r);
        // admission order: lower priority value first, submit order among equals
        auto at = pending_.end();
        while (at != pending_.begin()) {
            auto prev = std::prev(at);
            if (reqs_[*prev]->desc.priority <= prio) break;
            at = prev;
        }
        pending_.insert(at, id);
    }
    cv_.notify_all();
    return id;
}

void Engine::activate(Request& r, int slot)
{
    const pcr_render_desc& d = r.desc;
    const int64_t px = (int64_t)d.width * d.height;
    CK(cudaMallocFromPoolAsync(&r.accum, px * 3 * sizeof(double), pool_, stream_));
    CK(cudaMemsetAsync(r.accum, 0, px * 3 * sizeof(double), stream_));
    CK(cudaMallocFromPoolAsync(&r.d_hdr, px * 3 * sizeof(float), pool_, stream_));
    CK(cudaMallocFromPoolAsync(&r.d_rgb, px * 3, pool_, stream_));
    const SceneEntry& S = scenes_[r.scene];
    DRequest R{};
    R.scene = r.scene;
    R.width = d.width;
    R.height = d.height;
    R.depth = d.depth;
    R.aa = std::max(1, d.aa_samples);
    R.spp = d.samples;
    R.sample0 = d.sample_end > 0 ? d.sample_begin : 0;
    R.local_spp = local_spp(d);
    R.paths_per_pixel = R.aa * R.local_spp;
    R.shadow = d.shadow_samples;
    R.flags = (d.spectral ? kReqSpectral : 0) | (d.mis ? kReqMIS : 0) | (d.russian ? kReqRussian : 0) |
              (d.stratified ? kReqStratified : 0) | (d.spectral_terminate ? kReqTerminate : 0);
    R.hero = std::min(4, std::max(1, d.hero_samples <= 0 ? 4 : d.hero_samples));
    R.strata = d.stratified ? std::max(1, (int)std::lround(std::sqrt((float)d.samples))) : 0;
    R.cam_x = S.cam[0];
    R.cam_y = S.cam[1];
    R.cam_z = S.cam[2];
    // code/Renderer.cpp:149-150
    R.aspect = d.width / (float)d.height;
    R.scale = std::tan((float)3.14159265358979323846 / 180.f * 0.5f * S.fov);
    const uint64_t seed = d.seed ? d.seed : 1ull;
    R.seed_lo = (uint32_t)(seed & 0xffffffffu) * 0x9E3779B1u + 0x7F4A7C15u;
    R.seed_hi = (uint32_t)(seed >> 32) ^ (uint32_t)(seed * 0xD1B54A32D192ED03ull >> 17);
    R.total = px * R.paths_per_pixel;
    R.accum = r.accum;
    if (adaptive_rounds(d)) {
        R.flags |= kReqAdaptive;
        CK(cudaMallocFromPoolAsync(&r.act[0], px * sizeof(int), pool_, stream_));
        CK(cudaMallocFromPoolAsync(&r.act[1], px * sizeof(int), pool_, stream_));
        CK(cudaMallocFromPoolAsync(&r.welford, px * 2 * sizeof(float4), pool_, stream_));
        CK(cudaMemsetAsync(r.welford, 0, px * 2 * sizeof(float4), stream_));
        k_iota<<<std::max<int64_t>(1, std::min<int64_t>((px + 255) / 256, (int64_t)sms_ * 8)), 256, 0, stream_>>>(
            r.act[0], (int)px);
        R.act[0] = r.act[0];
        R.act[1] = r.act[1];
        R.welford = r.welford;
        R.round = 0;
        R.round_base = 0;
        R.total = px * R.spp;  // round 0 only; each round end adds the next
    }
    k_admit<<<1, 1, 0, stream_>>>(view(), R, slot);
    CK(cudaGetLastError());
    r.slot = slot;
    r.admit_block = blocks_launched_;
    r.state = ReqState::Active;
    r.t_admit = std::chrono::steady_clock::now();
    slot_owner_[slot] = r.id;
    active_slots_.push_back(slot);
    bytes_in_use_ += r.bytes;
    active_dirty_ = true;
}

void Engine::admit_locked()
{
    // first fit under the slot limit and the memory budget, in submit order
    for (auto it = pending_.begin(); it != pending_.end();) {
        Request& r = *reqs_[*it];
        if (r.state == ReqState::Cancelled) { it = pending_.erase(it); continue; }
        if ((int)active_slots_.size() >= kMaxActive) break;
        if (bytes_in_use_ + r.bytes > budget_) { ++it; continue; }
        int slot = -1;
        for (int s = 0; s < kMaxActive; s++)
            if (slot_owner_[s] < 0) { slot = s; break; }
        if (slot < 0) break;
        activate(r, slot);
        it = pending_.erase(it);
    }
}

void Engine::upload_active()
{
    if (!active_dirty_) return;
    ActiveList L;
    L.n = (int)active_slots_.size();
    for (int i = 0; i < L.n; i++) L.slots[i] = active_slots_[i];
    k_set_active<<<1, 256, 0, stream_>>>(view(), L);
    CK(cudaGetLastError());
    active_dirty_ = false;
}

void Engine::grid_for(const void* kernel, int block, size_t smem, int* grid)
{
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem));
    *grid = std::max(1, per_sm) * sms_;
}

void Engine::launch_iteration(int cur, bool prof)
{
    const EngineView E = view();
    const int B = tune_.block_size;
    if (prof) CK(cudaEventRecord(prof_ev_[0], stream_));
    k_schedule<<<1, kSchedThreads, 0, stream_>>>(E, (const EngineParams*)d_params_, cur);
    if (prof) CK(cudaEventRecord(prof_ev_[1], stream_));
    k_regen<<<grid_regen_, B, 0, stream_>>>(E, cur, xyz_scale_);
    if (prof) CK(cudaEventRecord(prof_ev_[2], stream_));
    k_extend<<<grid_extend_, B, 0, stream_>>>(E, cur);
    if (prof) CK(cudaEventRecord(prof_ev_[3], stream_));
    k_shade<<<grid_shade_, kShadeBlock, shade_smem_, stream_>>>(E, cur, smem_mats_);
    if (prof) CK(cudaEventRecord(prof_ev_[4], stream_));
    k_shadow<<<grid_shadow_, B, 0, stream_>>>(E);
    if (prof) CK(cudaEventRecord(prof_ev_[5], stream_));
    k_status<<<1, 1024, 0, stream_>>>(E, cur ^ 1);
    k_round<<<grid_round_, 256, 0, stream_>>>(E);
    if (prof) CK(cudaEventRecord(prof_ev_[6], stream_));
    CK(cudaGetLastError());
    if (prof) {
        CK(cudaEventSynchronize(prof_ev_[6]));
        // stage index: 0 regen 1 extend 2 shade 3 shadow 4 resolve 5 schedule 6 status
        const int map[6] = {5, 0, 1, 2, 3, 6};
        for (int k = 0; k < 6; k++) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, prof_ev_[k], prof_ev_[k + 1]));
            stage_ms_[map[k]] += ms;
            stage_launches_[map[k]]++;
        }
    } else {
        for (int k : {0, 1, 2, 3, 5, 6}) stage_launches_[k]++;
    }
    stage_launches_[7]++;  // k_round (timed with k_status)
    iterations_++;
}

// k_shade's limit on dynamic shared memory is one attribute of the function
// on the current device, shared by every context of the process.  It is only
// ever raised: a context with a smaller material table must not lower it
// below the size another context's launches (or captured graph) use.
static void raise_shade_smem(size_t bytes)
{
    static std::mutex mu;
    std::lock_guard<std::mutex> g(mu);
    cudaFuncAttributes a{};
    CK(cudaFuncGetAttributes(&a, (const void*)k_shade));
    if ((int)bytes > a.maxDynamicSharedSizeBytes)
        CK(cudaFuncSetAttribute((const void*)k_shade, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

void Engine::build_graph()
{
    const int B = tune_.block_size;
    // materials staged in shared memory when they fit
    const size_t mat_bytes = sizeof(DMaterial) * (size_t)std::max(1, mat_count_);
    smem_mats_ = mat_bytes <= 96 * 1024 ? 1 : 0;
    shade_smem_ = smem_mats_ ? mat_bytes : 0;
    raise_shade_smem(shade_smem_);
    grid_for((const void*)k_regen, B, 0, &grid_regen_);
    grid_for((const void*)k_extend, B, 0, &grid_extend_);
    grid_for((const void*)k_shade, kShadeBlock, shade_smem_, &grid_shade_);
    grid_for((const void*)k_shadow, B, 0, &grid_shadow_);
    grid_round_ = sms_ * 2;  // a round's per-pixel step is light; an idle launch reads one word
    if (graph_exec_) {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    if (use_graph_) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        for (int it = 0; it < tune_.iters_per_launch; it++) launch_iteration(it & 1, false);
        CK(cudaStreamEndCapture(stream_, &g));
        CK(cudaGraphInstantiate(&graph_exec_, g, 0));
        CK(cudaGraphDestroy(g));
        // capture counted launches that did not run
        for (int k : {0, 1, 2, 3, 5, 6, 7}) stage_launches_[k] -= tune_.iters_per_launch;
        iterations_ -= tune_.iters_per_launch;
    }
    graph_dirty_ = false;
}

void Engine::launch_block()
{
    if (graph_dirty_) build_graph();
    if (use_graph_ && !profile_) {
        CK(cudaGraphLaunch(graph_exec_, stream_));
        for (int k : {0, 1, 2, 3, 5, 6, 7}) stage_launches_[k] += tune_.iters_per_launch;
        iterations_ += tune_.iters_per_launch;
    } else {
        for (int it = 0; it < tune_.iters_per_launch; it++) launch_iteration(it & 1, profile_);
    }
}

void Engine::check_status()
{
    if (h_snap_->cnt.status)
        throw PcrError(PCR_ERR_DEVICE_STATUS, "device reported queue overflow (status " +
                                                  std::to_string(h_snap_->cnt.status) + ")");
}

void Engine::finish_request(Request& r, bool after_engine_stream)
{
    const pcr_render_desc& d = r.desc;
    const int64_t px = (int64_t)d.width * d.height;
    // adaptive requests hold each pixel's final mean already
    const double inv = adaptive_rounds(d) ? 1.0 : 1.0 / ((double)d.samples * std::max(1, d.aa_samples));
    int grid = std::min<int64_t>((px + 255) / 256, (int64_t)sms_ * 8);
    cudaStream_t rs = resolve_stream_;
    if (after_engine_stream) {
        // the plain method hands over with work it queued since its last
        // synchronisation: the resolve follows all of it
        if (!r.ev_ready) CK(cudaEventCreateWithFlags(&r.ev_ready, cudaEventDisableTiming));
        CK(cudaEventRecord(r.ev_ready, stream_));
        CK(cudaStreamWaitEvent(rs, r.ev_ready, 0));
    }
    k_resolve<<<std::max(1, grid), 256, 0, rs>>>(r.accum, (int)px, inv, d.spectral ? 1 : 0, d.aces ? 1 : 0, r.d_hdr,
                                                 r.d_rgb);
    CK(cudaGetLastError());
    if (d.denoise) {
        // two bilateral passes on the 8-bit image, the accumulator as scratch
        unsigned char* tmp = reinterpret_cast<unsigned char*>(r.accum);
        k_bilateral<<<std::max(1, grid), 256, 0, rs>>>(r.d_rgb, tmp, d.width, d.height);
        k_bilateral<<<std::max(1, grid), 256, 0, rs>>>(tmp, r.d_rgb, d.width, d.height);
        CK(cudaGetLastError());
    }
    // the resolved images stay on the device until fetch copies them out
    CK(cudaFreeAsync(r.accum, rs));
    r.accum = nullptr;
    for (int k = 0; k < 2; k++)
        if (r.act[k]) { CK(cudaFreeAsync(r.act[k], rs)); r.act[k] = nullptr; }
    if (r.welford) { CK(cudaFreeAsync(r.welford, rs)); r.welford = nullptr; }
    if (!r.ev_ready) CK(cudaEventCreateWithFlags(&r.ev_ready, cudaEventDisableTiming));
    CK(cudaEventRecord(r.ev_ready, rs));
    r.state = ReqState::Resolving;
}

// A cancelled request whose in-flight paths have retired: its device
// memory goes back to the pool (stream-ordered after the iterations that
// wrote it) and it waits in the Cancelled state for the fetch that reports
// and releases it.
void Engine::release_cancelled(Request& r)
{
    for (void** p : {(void**)&r.accum, (void**)&r.d_hdr, (void**)&r.d_rgb, (void**)&r.act[0], (void**)&r.act[1],
                     (void**)&r.welford})
        if (*p) { CK(cudaFreeAsync(*p, stream_)); *p = nullptr; }
    r.state = ReqState::Cancelled;
    r.t_ready = std::chrono::steady_clock::now();
}

// A pinned staging buffer of at least `bytes` with its copy stream: an idle
// one when one is large enough, else an idle one grown, else a new one.
Engine::Staging Engine::take_staging(size_t bytes)
{
    Staging st;
    {
        std::lock_guard<std::mutex> g(staging_mu_);
        int pick = -1;
        for (int k = 0; k < (int)staging_idle_.size(); k++) {
            const size_t have = staging_idle_[k].bytes;
            if (have >= bytes && (pick < 0 || have < staging_idle_[pick].bytes)) pick = k;
        }
        if (pick < 0 && !staging_idle_.empty()) pick = 0;
        if (pick >= 0) {
            st = staging_idle_[pick];
            staging_idle_.erase(staging_idle_.begin() + pick);
        }
    }
    if (!st.stream) CK(cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking));
    if (st.bytes < bytes) {
        if (st.buf) CK(cudaFreeHost(st.buf));
        st.buf = nullptr;
        st.bytes = 0;
        CK(cudaMallocHost(&st.buf, bytes));
        st.bytes = bytes;
    }
    return st;
}

void Engine::give_staging(const Staging& st)
{
    std::lock_guard<std::mutex> g(staging_mu_);
    staging_idle_.push_back(st);
}

// Copies a resolved request's images to caller host buffers through a
// pinned staging buffer on its own copy stream (ordered after the resolve by
// the request's event), then frees its device images.
void Engine::copy_out(Request& r, float* hdr, uint8_t* rgb)
{
    const int64_t px = (int64_t)r.desc.width * r.desc.height;
    const size_t need = (hdr || rgb) ? (size_t)px * 3 * (sizeof(float) + 1) : 0;
    struct Hold {  // hands the buffer back on every exit path
        Engine* e;
        Staging st;
        ~Hold() { e->give_staging(st); }
    } hold{this, take_staging(need)};
    const Staging& st = hold.st;
    CK(cudaStreamWaitEvent(st.stream, r.ev_ready, 0));
    float* sh = reinterpret_cast<float*>(st.buf);
    uint8_t* sr = st.buf ? st.buf + px * 3 * sizeof(float) : nullptr;
    if (hdr) CK(cudaMemcpyAsync(sh, r.d_hdr, px * 3 * sizeof(float), cudaMemcpyDeviceToHost, st.stream));
    if (rgb) CK(cudaMemcpyAsync(sr, r.d_rgb, px * 3, cudaMemcpyDeviceToHost, st.stream));
    CK(cudaFreeAsync(r.d_hdr, st.stream));
    CK(cudaFreeAsync(r.d_rgb, st.stream));
    r.d_hdr = nullptr;
    r.d_rgb = nullptr;
    CK(cudaStreamSynchronize(st.stream));
    if (hdr) std::memcpy(hdr, sh, px * 3 * sizeof(float));
    if (rgb) std::memcpy(rgb, sr, px * 3);
}

void Engine::harvest(bool)
{
    // h_snap_ holds the device state at the end of the last block
    check_status();
    std::vector<int> keep;
    for (int s : active_slots_) {
        Request& r = *reqs_[slot_owner_[s]];
        // a copy taken before the slot was set for this request still
        // holds the slot's previous owner's done flag
        if (h_snap_->done[s] && h_snap_block_ > r.admit_block) {
            const unsigned long long tf = h_snap_->tf[s], td = h_snap_->td[s];
            r.device_ms = (td > tf && tf) ? (double)(td - tf) * 1e-6 : 0.0;
            r.paths = h_snap_->issued[s];  // adaptive requests trace fewer than W*H*spp*aa
            if (r.cancel_running) release_cancelled(r);
            else finish_request(r);
            slot_owner_[s] = -1;
            bytes_in_use_ -= r.bytes;
            active_dirty_ = true;
        } else {
            keep.push_back(s);
        }
    }
    active_slots_.swap(keep);
    // results whose copies completed
    bool any = false;
    for (auto& kv : reqs_) {
        Request& r = *kv.second;
        if (r.state == ReqState::Resolving && cudaEventQuery(r.ev_ready) == cudaSuccess) {
            r.state = ReqState::Ready;
            r.t_ready = std::chrono::steady_clock::now();
            any = true;
        }
    }
    if (any) cv_done_.notify_all();
}

// One round of the device loop.  Returns false when nothing is left to do.
// Launches one block of iterations and copies the device state out after it;
// the host harvests the copies that have landed and waits only when
// kSnapRing blocks are queued, so later blocks are queued behind the one
// running.  A request harvested from block k's copy had no paths left, so the
// blocks already queued behind it do no work for it.
bool Engine::engine_step()
{
    CK(cudaSetDevice(device_));
    {
        std::lock_guard<std::mutex> g(mu_);
        admit_locked();
        upload_active();
        for (int s : active_slots_) {
            Request& r = *reqs_[slot_owner_[s]];
            if (r.cancel_running && !r.cancel_sent) {
                k_cancel<<<1, 1, 0, stream_>>>(view(), s);
                CK(cudaGetLastError());
                r.cancel_sent = true;
            }
        }
        bool resolving = false;
        for (auto& kv : reqs_)
            if (kv.second->state == ReqState::Resolving) { resolving = true; break; }
        if (active_slots_.empty()) {
            if (resolving || snap_inflight_) {
                CK(cudaStreamSynchronize(stream_));
                CK(cudaStreamSynchronize(resolve_stream_));
                if (snap_inflight_) {
                    const int last = (snap_next_ + kSnapRing - 1) % kSnapRing;
                    h_snap_ = h_snaps_[last];
                    h_snap_block_ = snap_block_[last];
                }
                snap_inflight_ = 0;
                harvest(true);
            }
            return !pending_.empty();
        }
    }
    launch_block();
    blocks_launched_++;
    const int b = snap_next_;
    snap_block_[b] = blocks_launched_;
    HostSnap* hs = h_snaps_[b];
    CK(cudaMemcpyAsync(&hs->cnt, d_cnt_, sizeof(Counters), cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(hs->done, d_done_, sizeof(int) * kMaxActive, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(hs->tf, d_tfirst_, 8 * kMaxActive, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(hs->td, d_tdone_, 8 * kMaxActive, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(hs->issued, d_issued_, 8 * kMaxActive, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(hs->outstanding, d_outstanding_, 8 * kMaxActive, cudaMemcpyDeviceToHost, stream_));
    CK(cudaEventRecord(ev_snaps_[b], stream_));
    snap_next_ = (snap_next_ + 1) % kSnapRing;
    snap_inflight_++;
    // harvest every copy that has landed; block only when the ring is full
    while (snap_inflight_ > 0) {
        const int old = (snap_next_ + kSnapRing - snap_inflight_) % kSnapRing;
        if (snap_inflight_ < kSnapRing) {
            const cudaError_t q = cudaEventQuery(ev_snaps_[old]);
            if (q == cudaErrorNotReady) break;
            CK(q);
        } else {
            CK(cudaEventSynchronize(ev_snaps_[old]));
        }
        snap_inflight_--;
        h_snap_ = h_snaps_[old];
        h_snap_block_ = snap_block_[old];
        std::lock_guard<std::mutex> g(mu_);
        harvest(false);
    }
    return true;
}

void Engine::run_until_idle()
{
    std::lock_guard<std::mutex> g(run_mu_);
    if (serving_) throw PcrError(PCR_ERR_INVALID, "engine is serving on its own thread");
    int64_t guard = 0;
    uint64_t last_paths = ~0ull, last_block = h_snap_block_;
    while (engine_step()) {
        if (h_snap_block_ == last_block) continue;  // no new copy harvested
        last_block = h_snap_block_;
        // no-progress guard: the loop must make progress every few blocks
        if (h_snap_->cnt.paths == last_paths && h_snap_->cnt.queue_n[0] == 0 && h_snap_->cnt.queue_n[1] == 0) {
            if (++guard > 64) throw PcrError(PCR_ERR_TIMEOUT, "engine made no progress");
        } else {
            guard = 0;
        }
        last_paths = h_snap_->cnt.paths;
    }
    CK(cudaStreamSynchronize(stream_));
    CK(cudaStreamSynchronize(resolve_stream_));
    std::lock_guard<std::mutex> l(mu_);
    harvest(true);
}

void Engine::serve_loop()
{
    try {
        cudaSetDevice(device_);
        while (!stop_) {
            bool work;
            {
                std::lock_guard<std::mutex> g(run_mu_);
                work = engine_step();
            }
            if (!work) {
                std::unique_lock<std::mutex> l(mu_);
                cv_.wait_for(l, std::chrono::milliseconds(2), [&] { return stop_.load() || !pending_.empty(); });
            }
        }
    } catch (const std::exception& e) {
        // waiters learn of it at once instead of running into their timeout
        const PcrError* pe = dynamic_cast<const PcrError*>(&e);
        {
            std::lock_guard<std::mutex> l(mu_);
            serve_error_ = e.what();
            serve_status_ = pe ? pe->status : PCR_ERR_CUDA;
        }
        std::fprintf(stderr, "pcr: serve loop stopped: %s\n", e.what());
        serving_ = false;
        cv_done_.notify_all();
    }
}

void Engine::serve_start()
{
    if (serving_) return;
    if (serve_thread_.joinable()) serve_thread_.join();  // a loop that stopped on an error
    {
        std::lock_guard<std::mutex> l(mu_);
        serve_error_.clear();
    }
    stop_ = false;
    serving_ = true;
    serve_thread_ = std::thread([this] { serve_loop(); });
}

void Engine::serve_stop()
{
    if (!serve_thread_.joinable()) return;
    stop_ = true;
    cv_.notify_all();
    serve_thread_.join();
    serving_ = false;
}

bool Engine::poll(int64_t id)
{
    std::lock_guard<std::mutex> g(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) throw PcrError(PCR_ERR_NOT_FOUND, "unknown request");
    Request& r = *it->second;
    if (r.state == ReqState::Resolving && cudaEventQuery(r.ev_ready) == cudaSuccess) {
        r.state = ReqState::Ready;
        r.t_ready = std::chrono::steady_clock::now();
    }
    return r.state == ReqState::Ready;
}

void Engine::wait(int64_t id, int64_t timeout_ms)
{
    auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? (int64_t)1 << 40 : timeout_ms);
    while (!poll(id)) {
        if (std::chrono::steady_clock::now() > deadline) throw PcrError(PCR_ERR_TIMEOUT, "wait timed out");
        {
            std::lock_guard<std::mutex> l(mu_);
            if (!serve_error_.empty()) throw PcrError(serve_status_, "serve loop stopped: " + serve_error_);
        }
        if (!serving_) {
            std::lock_guard<std::mutex> g(run_mu_);
            if (!engine_step()) {
                CK(cudaStreamSynchronize(stream_));
                CK(cudaStreamSynchronize(resolve_stream_));
                std::lock_guard<std::mutex> l(mu_);
                harvest(true);
            }
        } else {
            std::unique_lock<std::mutex> l(mu_);
            cv_done_.wait_for(l, std::chrono::milliseconds(1));
        }
        {
            std::lock_guard<std::mutex> l(mu_);
            if (reqs_[id]->state == ReqState::Cancelled) throw PcrError(PCR_ERR_CANCELLED, "request cancelled");
        }
    }
}

void Engine::fetch(int64_t id, float* hdr, uint8_t* rgb, pcr_render_stats* st)
{
    {
        // a cancelled request is released by its fetch, which reports it
        std::lock_guard<std::mutex> g(mu_);
        auto it = reqs_.find(id);
        if (it != reqs_.end() && it->second->state == ReqState::Cancelled) {
            reqs_.erase(it);
            throw PcrError(PCR_ERR_CANCELLED, "request cancelled");
        }
    }
    if (!poll(id)) throw PcrError(PCR_ERR_INVALID, "request not finished");
    std::unique_ptr<Request> owned;
    {
        std::lock_guard<std::mutex> g(mu_);
        auto it = reqs_.find(id);
        owned = std::move(it->second);
        reqs_.erase(it);
    }
    Request& r = *owned;
    copy_out(r, hdr, rgb);
    if (st) {
        st->device_ms = r.device_ms;
        st->latency_ms = std::chrono::duration<double, std::milli>(r.t_ready - r.t_submit).count();
        st->queue_ms = std::chrono::duration<double, std::milli>(r.t_admit - r.t_submit).count();
        st->paths = r.paths;
        st->rays = 0;
        st->shadow_rays = 0;
    }
    if (r.ev_ready) cudaEventDestroy(r.ev_ready);
}

void Engine::cancel(int64_t id)
{
    {
        std::lock_guard<std::mutex> g(mu_);
        auto it = reqs_.find(id);
        if (it == reqs_.end()) throw PcrError(PCR_ERR_NOT_FOUND, "unknown request");
        Request& r = *it->second;
        if (r.state == ReqState::Pending) {
            r.state = ReqState::Cancelled;
            return;
        }
        // a running request stops issuing paths at the next block of
        // iterations (engine_step sends it to the device); a finished one
        // keeps its result
        if (r.state != ReqState::Active) return;
        r.cancel_running = true;
    }
    cv_.notify_all();
}

// Share of a request's paths that have been traced to the end (issued and
// retired), from the device state copied after the last harvested block:
// 0 while it waits for admission, 1 once its images are resolved.
double Engine::progress(int64_t id)
{
    std::lock_guard<std::mutex> g(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) throw PcrError(PCR_ERR_NOT_FOUND, "unknown request");
    const Request& r = *it->second;
    if (r.state == ReqState::Pending) return 0.0;
    if (r.state != ReqState::Active) return 1.0;
    if (!h_snap_ || h_snap_block_ <= r.admit_block) return 0.0;
    const pcr_render_desc& d = r.desc;
    const double total = (double)d.width * d.height * local_spp(d) * std::max(1, d.aa_samples);
    const double retired = (double)h_snap_->issued[r.slot] - (double)h_snap_->outstanding[r.slot];
    return std::min(1.0, std::max(0.0, retired / std::max(1.0, total)));
}

// ---------------------------------------------------------------- plain method
void Engine::render_plain(int scene, const pcr_render_desc& desc, float* hdr, uint8_t* rgb, pcr_render_stats* st)
{
    if (adaptive_rounds(desc)) {
        // adaptive rounds are opened on the device between iterations: the
        // request runs alone through the batched loop
        {
            std::lock_guard<std::mutex> l(mu_);
            if (!active_slots_.empty() || !pending_.empty() || serving_)
                throw PcrError(PCR_ERR_INVALID, "plain render while batched work is active");
        }
        const int64_t id = submit(scene, desc);
        run_until_idle();
        fetch(id, hdr, rgb, st);
        return;
    }
    std::lock_guard<std::mutex> g(run_mu_);
    CK(cudaSetDevice(device_));
    validate(scene, desc);
    if (!active_slots_.empty() || serving_) throw PcrError(PCR_ERR_INVALID, "plain render while batched work is active");
    ensure_shadow_capacity(desc.shadow_samples);
    auto t0 = std::chrono::steady_clock::now();
    Request r;
    r.id = -1;
    r.scene = scene;
    r.desc = desc;
    r.bytes = request_bytes(desc);
    if (r.bytes > budget_) throw PcrError(PCR_ERR_NO_MEMORY, "request larger than the device memory budget");
    if (graph_dirty_) build_graph();
    // a pass holds one sample per pixel (W*H paths) unless multi_sample asks
    // for passes as large as the queue; no refill until a pass has drained
    const int64_t px = (int64_t)desc.width * desc.height;
    const int pass = desc.multi_sample ? tune_.queue_capacity : (int)std::min<int64_t>(px, tune_.queue_capacity);
    EngineParams p{pass, pass, 1, 1};
    k_set_params<<<1, 1, 0, stream_>>>((EngineParams*)d_params_, p);
    activate(r, 0);
    slot_owner_[0] = -1;  // the plain request is not in the request map
    upload_active();
    const int64_t total = px * local_spp(desc) * std::max(1, desc.aa_samples);
    const int64_t passes = (total + pass - 1) / pass;
    int cur = 0;
    for (int64_t it = 0; it < passes * (int64_t)desc.depth; it++) {
        launch_iteration(cur, profile_);
        cur ^= 1;
    }
    int extra = 0;
    while (true) {
        int done = 0;
        CK(cudaMemcpyAsync(&done, d_done_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        Counters c;
        CK(cudaMemcpy(&c, d_cnt_, sizeof(c), cudaMemcpyDeviceToHost));
        if (c.status) throw PcrError(PCR_ERR_DEVICE_STATUS, "device reported queue overflow");
        if (done) break;
        if (++extra > 4 * desc.depth + 8) throw PcrError(PCR_ERR_TIMEOUT, "plain render did not finish");
        launch_iteration(cur, profile_);
        cur ^= 1;
    }
    // a plain render always ends on queue parity 0 for the next user
    if (cur != 0) {
        launch_iteration(cur, false);
        cur ^= 1;
    }
    unsigned long long tf = 0, td = 0;
    CK(cudaMemcpy(&tf, d_tfirst_, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&td, d_tdone_, 8, cudaMemcpyDeviceToHost));
    finish_request(r, true);
    active_slots_.clear();
    active_dirty_ = true;
    bytes_in_use_ -= r.bytes;
    upload_active();
    EngineParams q{tune_.queue_capacity, tune_.chunk_paths, tune_.regen_every, 0};
    k_set_params<<<1, 1, 0, stream_>>>((EngineParams*)d_params_, q);
    copy_out(r, hdr, rgb);
    cudaEventDestroy(r.ev_ready);
    if (st) {
        st->device_ms = (td > tf && tf) ? (double)(td - tf) * 1e-6 : 0.0;
        st->latency_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        st->queue_ms = 0;
        st->paths = (uint64_t)total;
        st->rays = 0;
        st->shadow_rays = 0;
    }
}

// ---------------------------------------------------------------- render without allocating
// pcr_render_noalloc: a plain render whose working memory (path queues, hit
// records, shadow queue, FP64 pixel accumulator, request and counter words)
// is carved from one fixed-size array compiled into this library, for
// callers that may not allocate device memory during a render.  Inputs are
// a scene already uploaded to the context; outputs are caller-owned device
// buffers.  Every GPU that loads the library holds the array until exit.
constexpr int kNoAllocFill = 8192;                       // paths per pass
constexpr int kNoAllocQueue = kNoAllocFill * 4;          // room for 4-way forks
constexpr int kNoAllocShadowPerVertex = 8;
constexpr int kNoAllocShadow = kNoAllocQueue * kNoAllocShadowPerVertex;
constexpr int64_t kNoAllocMaxPixels = 256 * 256;
constexpr size_t kNoAllocAlign = 256;
constexpr size_t align_up(size_t x) { return (x + kNoAllocAlign - 1) / kNoAllocAlign * kNoAllocAlign; }
constexpr size_t kNoAllocHeader = 64 * 1024;             // counters, request table, per-slot words
constexpr size_t kNoAllocQueueBytes = align_up((size_t)kNoAllocQueue * 112);  // 7 x 16 B per path
constexpr size_t kNoAllocHitBytes = align_up((size_t)kNoAllocQueue * 16);
constexpr size_t kNoAllocShadowBytes = align_up((size_t)kNoAllocShadow * 48);
constexpr size_t kNoAllocAccumBytes = align_up((size_t)kNoAllocMaxPixels * 3 * sizeof(double));
constexpr size_t kNoAllocBytes =
    kNoAllocHeader + 2 * kNoAllocQueueBytes + kNoAllocHitBytes + kNoAllocShadowBytes + kNoAllocAccumBytes;

// The scratch array.  In host code `g_noalloc_scratch` is only a host-side
// stand-in for the symbol; its device address comes from
// cudaGetSymbolAddress (noalloc_scratch() below), once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[128] = {nullptr};
}  // namespace

// Device address of the scratch array on `device` (which must be current).
// Looked up on the first call per device; later calls reuse it.
static void* noalloc_scratch(int device)
{
    if (device < 0 || device >= 128) throw PcrError(PCR_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw PcrError(PCR_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_ptr[device] = p;
    }
    return g_noalloc_ptr[device];
}

// The request entry of a render (same fields Engine::activate writes).
DRequest Engine::make_request(const pcr_render_desc& d, int scene, double* accum) const
{
    const SceneEntry& S = scenes_[scene];
    DRequest R{};
    R.scene = scene;
    R.width = d.width;
    R.height = d.height;
    R.depth = d.depth;
    R.aa = std::max(1, d.aa_samples);
    R.spp = d.samples;
    R.sample0 = d.sample_end > 0 ? d.sample_begin : 0;
    R.local_spp = local_spp(d);
    R.paths_per_pixel = R.aa * R.local_spp;
    R.shadow = d.shadow_samples;
    R.flags = (d.spectral ? kReqSpectral : 0) | (d.mis ? kReqMIS : 0) | (d.russian ? kReqRussian : 0) |
              (d.stratified ? kReqStratified : 0) | (d.spectral_terminate ? kReqTerminate : 0);
    R.hero = std::min(4, std::max(1, d.hero_samples <= 0 ? 4 : d.hero_samples));
    R.strata = d.stratified ? std::max(1, (int)std::lround(std::sqrt((float)d.samples))) : 0;
    R.cam_x = S.cam[0];
    R.cam_y = S.cam[1];
    R.cam_z = S.cam[2];
    R.aspect = d.width / (float)d.height;
    R.scale = std::tan((float)3.14159265358979323846 / 180.f * 0.5f * S.fov);
    const uint64_t seed = d.seed ? d.seed : 1ull;
    R.seed_lo = (uint32_t)(seed & 0xffffffffu) * 0x9E3779B1u + 0x7F4A7C15u;
    R.seed_hi = (uint32_t)(seed >> 32) ^ (uint32_t)(seed * 0xD1B54A32D192ED03ull >> 17);
    R.total = (int64_t)d.width * d.height * R.paths_per_pixel;
    R.accum = accum;
    return R;
}

void Engine::render_noalloc(int scene, const pcr_render_desc& desc, float* hdr_dev, uint8_t* rgb_dev)
{
    std::lock_guard<std::mutex> g(run_mu_);
    CK(cudaSetDevice(device_));
    validate(scene, desc);
    const int64_t px = (int64_t)desc.width * desc.height;
    if (px > kNoAllocMaxPixels)
        throw PcrError(PCR_ERR_INVALID, "pcr_render_noalloc: " + std::to_string(desc.width) + "x" +
                                            std::to_string(desc.height) + " exceeds the " +
                                            std::to_string(kNoAllocMaxPixels) + "-pixel limit of its fixed scratch");
    if (desc.shadow_samples > kNoAllocShadowPerVertex)
        throw PcrError(PCR_ERR_INVALID, "pcr_render_noalloc: more than " + std::to_string(kNoAllocShadowPerVertex) +
                                            " shadow samples per hit");
    if (!hdr_dev && !rgb_dev) throw PcrError(PCR_ERR_INVALID, "pcr_render_noalloc: no output buffer");
    if (adaptive_rounds(desc))
        throw PcrError(PCR_ERR_INVALID, "pcr_render_noalloc: adaptive sampling needs per-pixel state; use pcr_render");
    if (!active_slots_.empty() || serving_)
        throw PcrError(PCR_ERR_INVALID, "pcr_render_noalloc while batched work is active");

    unsigned char* base = static_cast<unsigned char*>(noalloc_scratch(device_));
    // carve the array: header words first, then queues, hits, shadows, accumulator
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + off;
        off += align_up(bytes);
        return p;
    };
    Counters* cnt = reinterpret_cast<Counters*>(take(sizeof(Counters)));
    EngineParams* params = reinterpret_cast<EngineParams*>(take(sizeof(EngineParams)));
    DRequest* reqs = reinterpret_cast<DRequest*>(take(sizeof(DRequest)));
    unsigned long long* issued = reinterpret_cast<unsigned long long*>(take(8));
    long long* outstanding = reinterpret_cast<long long*>(take(8));
    unsigned long long* tfirst = reinterpret_cast<unsigned long long*>(take(8));
    unsigned long long* tdone = reinterpret_cast<unsigned long long*>(take(8));
    long long* give_start = reinterpret_cast<long long*>(take(8));
    int* give = reinterpret_cast<int*>(take(4));
    int* give_base = reinterpret_cast<int*>(take(4));
    int* active = reinterpret_cast<int*>(take(4));
    int* n_active = reinterpret_cast<int*>(take(4));
    int* done = reinterpret_cast<int*>(take(4));
    int* round_state = reinterpret_cast<int*>(take(4));
    int* round_cnt = reinterpret_cast<int*>(take(4));
    int* round_list = reinterpret_cast<int*>(take(4));
    const size_t header_used = off;
    off = kNoAllocHeader;
    PathQueue q[2];
    for (int b = 0; b < 2; b++) {
        unsigned char* p = take(kNoAllocQueueBytes);
        q[b].o = reinterpret_cast<float4*>(p);
        q[b].d = q[b].o + kNoAllocQueue;
        q[b].tp = q[b].d + kNoAllocQueue;
        q[b].id = reinterpret_cast<int4*>(q[b].tp + kNoAllocQueue);
        q[b].w[0] = reinterpret_cast<float4*>(q[b].id + kNoAllocQueue);
        q[b].w[1] = q[b].w[0] + kNoAllocQueue;
        q[b].w[2] = q[b].w[1] + kNoAllocQueue;
    }
    float4* hit = reinterpret_cast<float4*>(take(kNoAllocHitBytes));
    ShadowQueue sq;
    sq.o = reinterpret_cast<float4*>(take(kNoAllocShadowBytes));
    sq.d = sq.o + kNoAllocShadow;
    sq.c = sq.d + kNoAllocShadow;
    double* accum = reinterpret_cast<double*>(take(kNoAllocAccumBytes));
    if (off > kNoAllocBytes || header_used > kNoAllocHeader)
        throw PcrError(PCR_ERR_INVALID, "pcr_render_noalloc: scratch layout overflow");

    // the array keeps the previous call's contents: clear what starts at zero
    CK(cudaMemsetAsync(base, 0, header_used, stream_));
    CK(cudaMemsetAsync(accum, 0, (size_t)px * 3 * sizeof(double), stream_));

    EngineView E{};
    E.scenes = d_scenes_;
    E.mats = d_mats_;
    E.reqs = reqs;
    E.issued = issued;
    E.outstanding = outstanding;
    E.give = give;
    E.give_base = give_base;
    E.active = active;
    E.n_active = n_active;
    E.done_flag = done;
    E.t_first = tfirst;
    E.t_done = tdone;
    E.cnt = cnt;
    E.q[0] = q[0];
    E.q[1] = q[1];
    E.hit = hit;
    E.sq = sq;
    E.give_start = give_start;
    E.shadow_cap = kNoAllocShadow;
    E.round_state = round_state;
    E.round_cnt = round_cnt;
    E.round_list = round_list;
    E.cmf_table = d_cmf_;
    E.queue_cap = kNoAllocQueue;
    E.n_mats = mat_count_;

    DRequest R = make_request(desc, scene, accum);
    k_admit<<<1, 1, 0, stream_>>>(E, R, 0);
    ActiveList L;
    L.n = 1;
    L.slots[0] = 0;
    k_set_active<<<1, 32, 0, stream_>>>(E, L);
    const int pass = (int)std::min<int64_t>(px, kNoAllocFill);
    k_set_params<<<1, 1, 0, stream_>>>(params, EngineParams{pass, pass, 1, 1});
    CK(cudaGetLastError());

    // launch shapes from the occupancy calculator (no allocation involved)
    const int B = tune_.block_size;
    const size_t mat_bytes = sizeof(DMaterial) * (size_t)std::max(1, mat_count_);
    const int smem_mats = mat_bytes <= 96 * 1024 ? 1 : 0;
    const size_t smem = smem_mats ? mat_bytes : 0;
    raise_shade_smem(smem);
    int g_regen, g_extend, g_shade, g_shadow;
    grid_for((const void*)k_regen, B, 0, &g_regen);
    grid_for((const void*)k_extend, B, 0, &g_extend);
    grid_for((const void*)k_shade, kShadeBlock, smem, &g_shade);
    grid_for((const void*)k_shadow, B, 0, &g_shadow);
    int cur = 0;
    auto iteration = [&]() {
        k_schedule<<<1, kSchedThreads, 0, stream_>>>(E, params, cur);
        k_regen<<<g_regen, B, 0, stream_>>>(E, cur, xyz_scale_);
        k_extend<<<g_extend, B, 0, stream_>>>(E, cur);
        k_shade<<<g_shade, kShadeBlock, smem, stream_>>>(E, cur, smem_mats);
        k_shadow<<<g_shadow, B, 0, stream_>>>(E);
        k_status<<<1, 1024, 0, stream_>>>(E, cur ^ 1);
        CK(cudaGetLastError());
        cur ^= 1;
    };
    const int64_t total = px * local_spp(desc) * std::max(1, desc.aa_samples);
    const int64_t passes = (total + pass - 1) / pass;
    for (int64_t it = 0; it < passes * (int64_t)desc.depth; it++) iteration();
    for (int extra = 0;; extra++) {
        int flag = 0;
        Counters c;
        CK(cudaMemcpyAsync(&flag, done, sizeof(int), cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(&c, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        if (c.status) throw PcrError(PCR_ERR_DEVICE_STATUS, "pcr_render_noalloc: device reported queue overflow");
        if (flag) break;
        if (extra > 4 * desc.depth + 8) throw PcrError(PCR_ERR_TIMEOUT, "pcr_render_noalloc did not finish");
        iteration();
    }
    const double inv = 1.0 / ((double)desc.samples * std::max(1, desc.aa_samples));
    const int grid = (int)std::min<int64_t>((px + 255) / 256, (int64_t)sms_ * 8);
    k_resolve<<<std::max(1, grid), 256, 0, stream_>>>(accum, (int)px, inv, desc.spectral ? 1 : 0, desc.aces ? 1 : 0,
                                                       hdr_dev, rgb_dev);
    CK(cudaGetLastError());
    if (desc.denoise && rgb_dev) {
        // two bilateral passes; the accumulator region (24 B a pixel) is free now
        unsigned char* tmp = reinterpret_cast<unsigned char*>(accum);
        k_bilateral<<<std::max(1, grid), 256, 0, stream_>>>(rgb_dev, tmp, desc.width, desc.height);
        k_bilateral<<<std::max(1, grid), 256, 0, stream_>>>(tmp, rgb_dev, desc.width, desc.height);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(stream_));
}

// ---------------------------------------------------------------- parity entry points
void Engine::trace(int scene, const float* rays, int64_t n, int32_t* mat, int32_t* prim, float* t, int bvh_only,
                   int32_t* counts)
{
    std::lock_guard<std::mutex> g(run_mu_);
    CK(cudaSetDevice(device_));
    if (scene < 0 || scene >= (int)scenes_.size() || !scenes_[scene].live) throw PcrError(PCR_ERR_NOT_FOUND, "unknown scene");
    if (n <= 0) return;
    float* d_rays = nullptr;
    int *d_mat = nullptr, *d_prim = nullptr, *d_cnt = nullptr;
    float* d_t = nullptr;
    CK(cudaMallocFromPoolAsync(&d_rays, n * 6 * sizeof(float), pool_, stream_));
    CK(cudaMallocFromPoolAsync(&d_mat, n * sizeof(int), pool_, stream_));
    CK(cudaMallocFromPoolAsync(&d_prim, n * sizeof(int), pool_, stream_));
    CK(cudaMallocFromPoolAsync(&d_t, n * sizeof(float), pool_, stream_));
    if (counts) CK(cudaMallocFromPoolAsync(&d_cnt, n * 2 * sizeof(int), pool_, stream_));
    CK(cudaMemcpyAsync(d_rays, rays, n * 6 * sizeof(float), cudaMemcpyHostToDevice, stream_));
    int grid = 0;
    grid_for((const void*)k_trace_rays, 128, 0, &grid);
    if (profile_) CK(cudaEventRecord(prof_ev_[0], stream_));
    k_trace_rays<<<grid, 128, 0, stream_>>>(d_scenes_ + scene, d_mats_, d_rays, n, d_mat, d_prim, d_t, bvh_only, d_cnt);
    CK(cudaGetLastError());
    if (profile_) record_other(prof_ev_[0], prof_ev_[1]);
    if (mat) CK(cudaMemcpyAsync(mat, d_mat, n * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    if (prim) CK(cudaMemcpyAsync(prim, d_prim, n * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    if (t) CK(cudaMemcpyAsync(t, d_t, n * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    if (counts) CK(cudaMemcpyAsync(counts, d_cnt, n * 2 * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    CK(cudaFreeAsync(d_rays, stream_));
    CK(cudaFreeAsync(d_mat, stream_));
    CK(cudaFreeAsync(d_prim, stream_));
    CK(cudaFreeAsync(d_t, stream_));
    if (d_cnt) CK(cudaFreeAsync(d_cnt, stream_));
    CK(cudaStreamSynchronize(stream_));
}

// Profiled contexts time the parity-query kernels too, under stage "other".
void Engine::record_other(cudaEvent_t a, cudaEvent_t z)
{
    CK(cudaEventRecord(z, stream_));
    CK(cudaEventSynchronize(z));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, z));
    stage_ms_[7] += ms;
    stage_launches_[7]++;
}

void Engine::build_bvh(const pcr_triangle* tris, int n, std::vector<pcr_bvh_node>& nodes, std::vector<int32_t>& order)
{
    std::lock_guard<std::mutex> g(run_mu_);
    std::vector<float> v((size_t)n * 9);
    parallel_for(n, [&](int lo, int hi) {
        for (int i = lo; i < hi; i++)
            for (int a = 0; a < 3; a++) {
                v[(size_t)i * 9 + a] = tris[i].v0[a];
                v[(size_t)i * 9 + 3 + a] = tris[i].v1[a];
                v[(size_t)i * 9 + 6 + a] = tris[i].v2[a];
            }
    });
    device_build_bvh_raw(device_, stream_, pool_, v.data(), n, nodes, order);
}

void Engine::trace_shadow(int scene, const float* rays, const float* dist2, int64_t n, int32_t* blocked)
{
    std::lock_guard<std::mutex> g(run_mu_);
    CK(cudaSetDevice(device_));
    if (scene < 0 || scene >= (int)scenes_.size() || !scenes_[scene].live) throw PcrError(PCR_ERR_NOT_FOUND, "unknown scene");
    if (n <= 0) return;
    float *d_rays = nullptr, *d_d2 = nullptr;
    int* d_b = nullptr;
    CK(cudaMallocFromPoolAsync(&d_rays, n * 6 * sizeof(float), pool_, stream_));
    CK(cudaMallocFromPoolAsync(&d_d2, n * sizeof(float), pool_, stream_));
    CK(cudaMallocFromPoolAsync(&d_b, n * sizeof(int), pool_, stream_));
    CK(cudaMemcpyAsync(d_rays, rays, n * 6 * sizeof(float), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(d_d2, dist2, n * sizeof(float), cudaMemcpyHostToDevice, stream_));
    int grid = 0;
    grid_for((const void*)k_trace_shadow, 128, 0, &grid);
    if (profile_) CK(cudaEventRecord(prof_ev_[0], stream_));
    k_trace_shadow<<<grid, 128, 0, stream_>>>(d_scenes_ + scene, d_mats_, d_rays, d_d2, n, d_b);
    CK(cudaGetLastError());
    if (profile_) record_other(prof_ev_[0], prof_ev_[1]);
    CK(cudaMemcpyAsync(blocked, d_b, n * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    CK(cudaFreeAsync(d_rays, stream_));
    CK(cudaFreeAsync(d_d2, stream_));
    CK(cudaFreeAsync(d_b, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void Engine::tonemap(const float* hdr, int width, int height, int aces_tm, int denoise, uint8_t* rgb8)
{
    std::lock_guard<std::mutex> g(run_mu_);
    CK(cudaSetDevice(device_));
    if (width <= 0 || height <= 0) throw PcrError(PCR_ERR_INVALID, "width and height must be positive");
    const int64_t px = (int64_t)width * height;
    float* d_hdr = nullptr;
    unsigned char *d_rgb = nullptr, *d_tmp = nullptr;
    CK(cudaMallocFromPoolAsync(&d_hdr, px * 3 * sizeof(float), pool_, stream_));
    CK(cudaMallocFromPoolAsync(&d_rgb, px * 3, pool_, stream_));
    CK(cudaMemcpyAsync(d_hdr, hdr, px * 3 * sizeof(float), cudaMemcpyHostToDevice, stream_));
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((px + 255) / 256, (int64_t)sms_ * 8));
    k_tonemap<<<grid, 256, 0, stream_>>>(d_hdr, (int)px, aces_tm, d_rgb);
    if (denoise) {
        CK(cudaMallocFromPoolAsync(&d_tmp, px * 3, pool_, stream_));
        k_bilateral<<<grid, 256, 0, stream_>>>(d_rgb, d_tmp, width, height);
        k_bilateral<<<grid, 256, 0, stream_>>>(d_tmp, d_rgb, width, height);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(rgb8, d_rgb, px * 3, cudaMemcpyDeviceToHost, stream_));
    CK(cudaFreeAsync(d_hdr, stream_));
    CK(cudaFreeAsync(d_rgb, stream_));
    if (d_tmp) CK(cudaFreeAsync(d_tmp, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void Engine::eval_stage(int what, const float* params, const float* in, int64_t n, float* out)
{
    std::lock_guard<std::mutex> g(run_mu_);
    CK(cudaSetDevice(device_));
    if (what < 0 || what > 8 || n <= 0) throw PcrError(PCR_ERR_INVALID, "bad stage evaluation request");
    const int in_w = (what == 0 || what == 1 || what == 2) ? 1 : ((what == 3 || what == 8) ? 2 : 3);
    const int out_w = (what == 0 || what == 1) ? 1 : 3;
    const int np = what == 0 ? 4 : (what == 1 ? kSpecN : 0);
    float *d_in = nullptr, *d_out = nullptr, *d_p = nullptr;
    CK(cudaMallocFromPoolAsync(&d_in, n * in_w * sizeof(float), pool_, stream_));
    CK(cudaMallocFromPoolAsync(&d_out, n * out_w * sizeof(float), pool_, stream_));
    CK(cudaMallocFromPoolAsync(&d_p, 64 * sizeof(float), pool_, stream_));
    CK(cudaMemcpyAsync(d_in, in, n * in_w * sizeof(float), cudaMemcpyHostToDevice, stream_));
    if (np) {
        if (!params) throw PcrError(PCR_ERR_INVALID, "stage needs parameters");
        CK(cudaMemcpyAsync(d_p, params, np * sizeof(float), cudaMemcpyHostToDevice, stream_));
    }
    k_eval_stage<<<std::min<int64_t>((n + 255) / 256, 4096), 256, 0, stream_>>>(what, d_p, d_in, n, d_out, xyz_scale_,
                                                                                 d_cmf_);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, d_out, n * out_w * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    CK(cudaFreeAsync(d_in, stream_));
    CK(cudaFreeAsync(d_out, stream_));
    CK(cudaFreeAsync(d_p, stream_));
    CK(cudaStreamSynchronize(stream_));
}

// ---------------------------------------------------------------- L2 bandwidth
// Reads an L2-resident buffer `reps` times with loads that bypass L1
// (ld.global.cg), four 16-byte loads in flight per thread per step; each
// thread writes its sum so the loads are kept.
__global__ void __launch_bounds__(256) k_l2_read(const float4* __restrict__ buf, long long n4, int reps, float* out)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    float acc = 0.f;
    for (int r = 0; r < reps; r++) {
        long long i = t0;
        for (; i + 3 * stride < n4; i += 4 * stride) {
            const float4 a = __ldcg(buf + i), b = __ldcg(buf + i + stride), c = __ldcg(buf + i + 2 * stride),
                         d = __ldcg(buf + i + 3 * stride);
            acc += (a.x + b.y) + (c.z + d.w);
        }
        for (; i < n4; i += stride) acc += __ldcg(buf + i).x;
    }
    out[t0] = acc;
}

double Engine::l2_bandwidth(int64_t bytes, int reps)
{
    std::lock_guard<std::mutex> g(run_mu_);
    CK(cudaSetDevice(device_));
    if (bytes < (1 << 20) || bytes > (int64_t)96 << 20 || reps < 1)
        throw PcrError(PCR_ERR_INVALID, "l2 bandwidth probe: 1..96 MiB and at least one pass");
    const int block = 256, grid = sms_ * 8;
    const int64_t n4 = bytes / 16;
    float4* buf = nullptr;
    float* out = nullptr;
    CK(cudaMallocFromPoolAsync(&buf, n4 * 16, pool_, stream_));
    CK(cudaMallocFromPoolAsync(&out, (size_t)grid * block * sizeof(float), pool_, stream_));
    CK(cudaMemsetAsync(buf, 0, n4 * 16, stream_));
    k_l2_read<<<grid, block, 0, stream_>>>(buf, n4, 2, out);  // warm: brings the buffer into L2
    cudaEvent_t a, z;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&z));
    CK(cudaEventRecord(a, stream_));
    k_l2_read<<<grid, block, 0, stream_>>>(buf, n4, reps, out);
    CK(cudaEventRecord(z, stream_));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(z));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, z));
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    CK(cudaFreeAsync(buf, stream_));
    CK(cudaFreeAsync(out, stream_));
    CK(cudaStreamSynchronize(stream_));
    return (double)n4 * 16 * reps / (ms * 1e-3) / 1e9;
}

// ---------------------------------------------------------------- stats / tuning
void Engine::stats(pcr_engine_stats* o)
{
    std::lock_guard<std::mutex> g(run_mu_);
    Counters c;
    CK(cudaMemcpy(&c, d_cnt_, sizeof(c), cudaMemcpyDeviceToHost));
    std::memset(o, 0, sizeof(*o));
    for (int k = 0; k < 8; k++) {
        o->stage_ms[k] = stage_ms_[k];
        o->stage_launches[k] = stage_launches_[k];
    }
    o->iterations = iterations_;
    o->paths = (int64_t)(c.paths - base_paths_);
    o->rays = (int64_t)(c.rays - base_rays_);
    o->shadow_rays = (int64_t)(c.shadow_rays - base_shadow_);
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    o->device_bytes = (int64_t)(tot - fr);
    o->queue_capacity = tune_.queue_capacity;
    o->block_size = tune_.block_size;
    o->chunk_paths = tune_.chunk_paths;
    o->regen_every = tune_.regen_every;
}

void Engine::reset_stats()
{
    std::lock_guard<std::mutex> g(run_mu_);
    Counters c;
    CK(cudaMemcpy(&c, d_cnt_, sizeof(c), cudaMemcpyDeviceToHost));
    base_paths_ = c.paths;
    base_rays_ = c.rays;
    base_shadow_ = c.shadow_rays;
    std::memset(stage_ms_, 0, sizeof(stage_ms_));
    std::memset(stage_launches_, 0, sizeof(stage_launches_));
    iterations_ = 0;
}

// ---------------------------------------------------------------- autotuner
// Times short trial batches of the caller's sample workload under a small
// grid of (queue capacity, block size, issue chunk, refill cadence) and keeps
// the fastest.  The choice is written to the tuning cache file when one was
// given at context creation.
void Engine::autotune(const int32_t* scenes, const pcr_render_desc* descs, int n, int32_t* chosen)
{
    struct Cand { int q, b, c, r; };
    std::vector<Cand> cands;
    // up to 16M paths in flight (64M path slots; about 40 GB of path and
    // shadow queues at 8 shadow rays per hit).  Shadow records are indexed
    // with 32-bit ints, so a capacity whose slots times the sample requests'
    // shadow rays per hit reach 2^31 is skipped.
    int max_shadow = 8;
    for (int i = 0; i < n; i++) max_shadow = std::max(max_shadow, descs[i].shadow_samples);
    for (int q : {1 << 19, 1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24})
        for (int b : {64, 128, 256})
            for (int c : {1 << 14, 1 << 16})
                for (int r : {1, 2})
                    if ((int64_t)q * 4 * max_shadow <= (int64_t)INT32_MAX) cands.push_back({q, b, c, r});
    EngineTuning best = tune_;
    double best_ms = 1e30;
    cudaEvent_t a, z;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&z));
    for (const Cand& cd : cands) {
        EngineTuning t = tune_;
        t.queue_capacity = cd.q;
        t.block_size = cd.b;
        t.chunk_paths = cd.c;
        t.regen_every = cd.r;
        set_tuning(t);
        std::vector<int64_t> ids;
        for (int i = 0; i < n; i++) ids.push_back(submit(scenes[i], descs[i]));
        CK(cudaEventRecord(a, stream_));
        run_until_idle();
        CK(cudaEventRecord(z, stream_));
        CK(cudaEventSynchronize(z));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, a, z));
        for (int64_t id : ids) fetch(id, nullptr, nullptr, nullptr);
        if (ms < best_ms) { best_ms = ms; best = t; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    set_tuning(best);
    if (chosen) {
        chosen[0] = best.queue_capacity;
        chosen[1] = best.block_size;
        chosen[2] = best.chunk_paths;
        chosen[3] = best.regen_every;
    }
    if (!tuning_cache_.empty()) {
        if (FILE* f = std::fopen(tuning_cache_.c_str(), "w")) {
            std::fprintf(f, "{\"queue_capacity\": %d, \"block_size\": %d, \"chunk_paths\": %d, \"regen_every\": %d, \"ms\": %.3f}\n",
                         best.queue_capacity, best.block_size, best.chunk_paths, best.regen_every, best_ms);
            std::fclose(f);
        }
    }
}

}  // namespace pcr
