// Host side of the wavefront engine: device scene cache, request table,
// admission under a memory budget, the graph-captured iteration loop
// (batched / served method) and the plain per-request launch sequence.
#pragma once

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pcr_cuda.h"
#include "layout.h"

namespace pcr {

struct PcrError : std::runtime_error {
    pcr_status status;
    PcrError(pcr_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

struct SceneEntry {
    DScene dev{};
    std::vector<void*> allocs;
    int64_t bytes = 0;
    std::string name, version;
    float cam[3] = {0, 0, 0}, fov = 65.f;
    std::vector<DMaterial> mats;
    bool live = false;
};

enum class ReqState { Pending, Active, Resolving, Ready, Fetched, Cancelled };

struct Request {
    int64_t id = 0;
    int scene = 0;
    pcr_render_desc desc{};
    ReqState state = ReqState::Pending;
    int slot = -1;
    int64_t bytes = 0;
    double* accum = nullptr;
    float* d_hdr = nullptr;
    uint8_t* d_rgb = nullptr;
    cudaEvent_t ev_ready = nullptr;
    std::chrono::steady_clock::time_point t_submit, t_admit, t_ready;
    double device_ms = 0;
    uint64_t paths = 0;
    uint64_t admit_block = 0;  // blocks launched before this request's slot was (re)set
    bool cancel_running = false;        // cancel asked while Active
    bool cancel_sent = false;           // k_cancel launched for it
    int* act[2] = {nullptr, nullptr};   // adaptive: pixel lists of alternate rounds
    float4* welford = nullptr;          // adaptive: per-pixel mean / M2
};

struct EngineTuning {
    int queue_capacity = 1 << 20;  // fill target
    int block_size = 128;
    int chunk_paths = 1 << 16;
    int regen_every = 1;
    int iters_per_launch = 8;      // iterations per graph launch (even)
};

class Engine {
public:
    explicit Engine(const pcr_ctx_opts* opts);
    ~Engine();

    int upload_scene(const pcr_scene_desc& d);
    void release_scene(int id);
    int64_t scene_bytes(int id) const;

    void render_plain(int scene, const pcr_render_desc& desc, float* hdr, uint8_t* rgb, pcr_render_stats* st);
    // Plain render with all working memory in the library's fixed scratch
    // array; outputs are caller device buffers.  Allocates nothing.
    void render_noalloc(int scene, const pcr_render_desc& desc, float* hdr_dev, uint8_t* rgb_dev);
    int64_t submit(int scene, const pcr_render_desc& desc);
    void run_until_idle();
    void serve_start();
    void serve_stop();
    bool poll(int64_t id);
    void wait(int64_t id, int64_t timeout_ms);
    void fetch(int64_t id, float* hdr, uint8_t* rgb, pcr_render_stats* st);
    void cancel(int64_t id);
    double progress(int64_t id);

    void trace(int scene, const float* rays, int64_t n, int32_t* mat, int32_t* prim, float* t, int bvh_only,
               int32_t* counts);
    void record_other(cudaEvent_t a, cudaEvent_t z);
    void trace_shadow(int scene, const float* rays, const float* dist2, int64_t n, int32_t* blocked);
    void build_bvh(const pcr_triangle* tris, int n, std::vector<pcr_bvh_node>& nodes, std::vector<int32_t>& order);
    void tonemap(const float* hdr, int width, int height, int aces_tm, int denoise, uint8_t* rgb8);
    void eval_stage(int what, const float* params, const float* in, int64_t n, float* out);
    double l2_bandwidth(int64_t bytes, int reps);

    void stats(pcr_engine_stats* out);
    void reset_stats();
    void set_tuning(const EngineTuning& t);
    const EngineTuning& tuning() const { return tune_; }
    void autotune(const int32_t* scenes, const pcr_render_desc* descs, int n, int32_t* chosen);
    int device() const { return device_; }
    cudaStream_t stream() const { return stream_; }

private:
    void ensure_shadow_capacity(int shadow_samples);
    void alloc_buffers();
    void free_buffers();
    void validate(int scene, const pcr_render_desc& d) const;
    int64_t request_bytes(const pcr_render_desc& d) const;
    void admit_locked();
    void activate(Request& r, int slot);
    void upload_active();
    void launch_iteration(int cur, bool profile);
    void launch_block();
    void build_graph();
    void harvest(bool final_sync);
    void finish_request(Request& r, bool after_engine_stream = false);
    void release_cancelled(Request& r);
    void copy_out(Request& r, float* hdr, uint8_t* rgb);
    DRequest make_request(const pcr_render_desc& d, int scene, double* accum) const;
    void check_status();
    bool engine_step();
    void serve_loop();
    EngineView view() const;
    void grid_for(const void* kernel, int block, size_t smem, int* grid);

    int device_ = 0;
    int sms_ = 148;
    cudaStream_t stream_ = nullptr;
    // Resolves of finished requests run here, beside the iterations still
    // queued on stream_: a request is harvested from the device state copied
    // after the block it finished in, by which point its accumulator is final.
    cudaStream_t resolve_stream_ = nullptr;
    // Result copies: pinned staging buffers, each with its own copy stream,
    // kept idle between fetches.  A fetch takes one (or makes one), so
    // fetches from several threads copy at the same time.
    struct Staging {
        uint8_t* buf = nullptr;
        size_t bytes = 0;
        cudaStream_t stream = nullptr;
    };
    std::mutex staging_mu_;
    std::vector<Staging> staging_idle_;
    Staging take_staging(size_t bytes);
    void give_staging(const Staging& s);
    EngineTuning tune_;
    bool use_graph_ = true, profile_ = false;
    int64_t budget_ = 40ll << 30;
    std::string tuning_cache_;

    // scenes
    std::vector<SceneEntry> scenes_;
    DScene* d_scenes_ = nullptr;
    DMaterial* d_mats_ = nullptr;
    int mat_cap_ = 0, mat_count_ = 0;
    float xyz_scale_ = 0.f;

    // request table
    DRequest* d_reqs_ = nullptr;
    DRequest* h_reqs_ = nullptr;  // pinned mirror
    unsigned long long *d_issued_ = nullptr, *d_tfirst_ = nullptr, *d_tdone_ = nullptr;
    long long* d_outstanding_ = nullptr;
    long long* d_give_start_ = nullptr;
    int *d_give_ = nullptr, *d_give_base_ = nullptr, *d_active_ = nullptr, *d_nactive_ = nullptr, *d_done_ = nullptr;
    int *d_round_state_ = nullptr, *d_round_cnt_ = nullptr, *d_round_list_ = nullptr;
    float4* d_cmf_ = nullptr;  // colour-matching table for raygen
    int* h_active_ = nullptr;     // pinned: [0] = n, then slots
    Counters* d_cnt_ = nullptr;
    struct HostSnap {
        Counters cnt;
        int done[kMaxActive];
        unsigned long long tf[kMaxActive], td[kMaxActive], issued[kMaxActive];
        long long outstanding[kMaxActive];
    };
    // Device state copied out after each block of iterations, into a ring of
    // pinned buffers: the host keeps up to kSnapRing blocks queued and
    // harvests each block's copy once it has landed, so the GPU does not idle
    // while the host harvests or is briefly descheduled.
    static constexpr int kSnapRing = 4;
    cudaMemPool_t pool_ = nullptr;
    HostSnap* h_snaps_[kSnapRing] = {};
    cudaEvent_t ev_snaps_[kSnapRing] = {};
    HostSnap* h_snap_ = nullptr;  // the snapshot harvest reads (one of h_snaps_)
    int snap_next_ = 0;           // buffer the next block copies into
    int snap_inflight_ = 0;       // blocks launched whose copy is not harvested
    uint64_t blocks_launched_ = 0;
    uint64_t snap_block_[kSnapRing] = {};  // block count each buffer's copy follows
    uint64_t h_snap_block_ = 0;        // the same for h_snap_
    void* d_params_ = nullptr;
    void* h_params_ = nullptr;

    // queues
    PathQueue q_[2]{};
    float4* d_hit_ = nullptr;
    ShadowQueue sq_{};
    int queue_cap_ = 0, shadow_cap_ = 0;
    std::vector<void*> qallocs_;

    // graph
    cudaGraphExec_t graph_exec_ = nullptr;
    bool graph_dirty_ = true;
    int grid_regen_ = 0, grid_extend_ = 0, grid_shade_ = 0, grid_shadow_ = 0, grid_round_ = 0;
    size_t shade_smem_ = 0;
    int smem_mats_ = 0;

    // requests
    std::mutex mu_;
    std::condition_variable cv_, cv_done_;
    std::map<int64_t, std::unique_ptr<Request>> reqs_;
    std::deque<int64_t> pending_;
    std::vector<int64_t> slot_owner_;   // request id per slot (-1 free)
    std::vector<int> active_slots_;
    int64_t next_id_ = 1;
    int64_t bytes_in_use_ = 0;
    bool active_dirty_ = true;
    std::thread serve_thread_;
    std::atomic<bool> serving_{false}, stop_{false};
    std::string serve_error_;                 // why the serve loop stopped (guarded by mu_)
    pcr_status serve_status_ = PCR_OK;
    std::mutex run_mu_;   // one driver of the device loop at a time

    // stats
    double stage_ms_[8] = {0};
    int64_t stage_launches_[8] = {0};
    int64_t iterations_ = 0;
    uint64_t base_rays_ = 0, base_shadow_ = 0, base_paths_ = 0;
    cudaEvent_t prof_ev_[16]{};
};

}  // namespace pcr
