// extern "C" implementation of include/pcr_cuda.h.  No exception crosses
// this boundary: every entry point converts errors into a pcr_status and a
// thread-local message (pcr_last_error).
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pcr_cuda.h"
#include "engine.h"
#include "scene.h"

struct pcr_ctx {
    std::unique_ptr<pcr::Engine> eng;
};

struct pcr_host_scene {
    pcr::HostScene s;
};

// Least-outstanding-paths router over borrowed contexts.
struct pcr_router {
    std::vector<pcr::Engine*> eng;
    std::mutex mu;
    std::vector<std::vector<int>> scene_map;   // router scene id -> per-context scene id
    struct Ticket { int ctx; int64_t id; int64_t paths; };
    std::map<int64_t, Ticket> tickets;
    std::vector<int64_t> load, routed;
    int64_t next = 1;
};

namespace {
thread_local std::string g_err;

template <typename F>
pcr_status guard(F&& f)
{
    try {
        f();
        g_err.clear();
        return PCR_OK;
    } catch (const pcr::PcrError& e) {
        g_err = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        g_err = "host allocation failed";
        return PCR_ERR_NO_MEMORY;
    } catch (const std::exception& e) {
        g_err = e.what();
        return PCR_ERR_INVALID;
    }
}

pcr::Engine& E(pcr_ctx* c)
{
    if (!c || !c->eng) throw pcr::PcrError(PCR_ERR_INVALID, "null context");
    return *c->eng;
}

std::string parent_dir(const std::string& p)
{
    auto k = p.find_last_of('/');
    return k == std::string::npos ? std::string(".") : (k == 0 ? std::string("/") : p.substr(0, k));
}

pcr::HostScene host_scene_from_json(const char* path, const char* data_root, const char* lut_path,
                                    bool with_bvh = true)
{
    // default data root: the directory that holds the scene directory
    // (the reference ships <root>/Scenes/*.json beside <root>/spd/)
    std::string root = data_root ? std::string(data_root) : parent_dir(parent_dir(path));
    std::vector<float> lut;
    if (lut_path) {
        std::string err;
        if (!pcr::load_plut(lut_path, lut, &err))
            throw pcr::PcrError(PCR_ERR_SCENE, std::string("loadLUT(") + lut_path + "): " + err);
    }
    return pcr::load_scene_json(path, root, lut_path ? &lut : nullptr, with_bvh);
}

// The BVH of a scene loaded without one, built on `e`'s device; the
// triangles and their ids are put into leaf order as the host builder does.
void device_bvh(pcr::Engine& e, pcr::HostScene& s)
{
    const int n = (int)s.triangles.size();
    if (n == 0) return;
    std::vector<int32_t> order;
    e.build_bvh(s.triangles.data(), n, s.bvh, order);
    std::vector<pcr_triangle> t(n);
    std::vector<int32_t> ids(n);
    pcr::parallel_for(n, [&](int lo, int hi) {
        for (int i = lo; i < hi; i++) {
            t[i] = s.triangles[order[i]];
            ids[i] = s.triangle_ids[order[i]];
        }
    });
    s.triangles.swap(t);
    s.triangle_ids.swap(ids);
}
}  // namespace

extern "C" {

const char* pcr_last_error(void) { return g_err.c_str(); }
const char* pcr_version(void) { return "pcr-b200 0.1 (sm_100a)"; }

pcr_status pcr_ctx_create(pcr_ctx** out, const pcr_ctx_opts* opts)
{
    return guard([&] {
        if (!out) throw pcr::PcrError(PCR_ERR_INVALID, "null output pointer");
        auto c = std::make_unique<pcr_ctx>();
        c->eng = std::make_unique<pcr::Engine>(opts);
        *out = c.release();
    });
}

pcr_status pcr_ctx_destroy(pcr_ctx* ctx)
{
    return guard([&] { delete ctx; });
}

pcr_status pcr_ctx_set_device(pcr_ctx* ctx)
{
    return guard([&] {
        if (cudaSetDevice(E(ctx).device()) != cudaSuccess) throw pcr::PcrError(PCR_ERR_CUDA, "cudaSetDevice failed");
    });
}

pcr_status pcr_ctx_stream(pcr_ctx* ctx, void** stream)
{
    return guard([&] {
        if (!stream) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        *stream = (void*)E(ctx).stream();
    });
}

pcr_status pcr_scene_upload(pcr_ctx* ctx, const pcr_scene_desc* desc, pcr_scene_id* out)
{
    return guard([&] {
        if (!desc || !out) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        *out = E(ctx).upload_scene(*desc);
    });
}

pcr_status pcr_scene_load_json(pcr_ctx* ctx, const char* path, const char* data_root, const char* lut_path,
                               pcr_scene_id* out)
{
    return guard([&] {
        if (!path || !out) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        pcr::HostScene s = host_scene_from_json(path, data_root, lut_path, false);
        device_bvh(E(ctx), s);
        pcr_scene_desc d = s.desc();
        *out = E(ctx).upload_scene(d);
    });
}

pcr_status pcr_host_scene_load(const char* path, const char* data_root, const char* lut_path, pcr_host_scene** out,
                               pcr_scene_desc* desc)
{
    return guard([&] {
        if (!path || !out || !desc) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        std::string root = data_root ? std::string(data_root) : parent_dir(parent_dir(path));
        std::vector<float> lut;
        if (lut_path) {
            std::string err;
            if (!pcr::load_plut(lut_path, lut, &err)) throw pcr::PcrError(PCR_ERR_SCENE, std::string("loadLUT(") + lut_path + "): " + err);
        }
        auto h = std::make_unique<pcr_host_scene>();
        h->s = pcr::load_scene_json(path, root, lut_path ? &lut : nullptr);
        *desc = h->s.desc();
        *out = h.release();
    });
}

pcr_status pcr_host_scene_free(pcr_host_scene* scene)
{
    return guard([&] { delete scene; });
}

pcr_status pcr_fit_sigmoid(const float* rgb, int64_t n, const float* lut, float* out4)
{
    return guard([&] {
        if (!rgb || !out4 || n < 0) throw pcr::PcrError(PCR_ERR_INVALID, "bad argument");
        std::vector<float> L;
        if (lut) L.assign(lut, lut + 3 * 16 * 16 * 16 * 3);
        for (int64_t i = 0; i < n; i++) pcr::fit_sigmoid(rgb + i * 3, lut ? &L : nullptr, out4 + i * 4);
    });
}

pcr_status pcr_lut_build(float* out)
{
    return guard([&] {
        if (!out) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        std::vector<float> L;
        pcr::build_lut(L);
        std::memcpy(out, L.data(), L.size() * sizeof(float));
    });
}

pcr_status pcr_scene_release(pcr_ctx* ctx, pcr_scene_id id)
{
    return guard([&] { E(ctx).release_scene(id); });
}

pcr_status pcr_scene_bytes(pcr_ctx* ctx, pcr_scene_id id, int64_t* bytes)
{
    return guard([&] {
        if (!bytes) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        *bytes = E(ctx).scene_bytes(id);
    });
}

pcr_status pcr_render(pcr_ctx* ctx, pcr_scene_id scene, const pcr_render_desc* desc, float* hdr_out, uint8_t* rgb8_out,
                      pcr_render_stats* stats)
{
    return guard([&] {
        if (!desc) throw pcr::PcrError(PCR_ERR_INVALID, "null render descriptor");
        E(ctx).render_plain(scene, *desc, hdr_out, rgb8_out, stats);
    });
}

pcr_status pcr_render_noalloc(pcr_ctx* ctx, pcr_scene_id scene, const pcr_render_desc* desc, float* hdr_out_dev,
                              uint8_t* rgb8_out_dev)
{
    return guard([&] {
        if (!desc) throw pcr::PcrError(PCR_ERR_INVALID, "null render descriptor");
        E(ctx).render_noalloc(scene, *desc, hdr_out_dev, rgb8_out_dev);
    });
}

pcr_status pcr_submit(pcr_ctx* ctx, pcr_scene_id scene, const pcr_render_desc* desc, pcr_request_id* out)
{
    return guard([&] {
        if (!desc || !out) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        *out = E(ctx).submit(scene, *desc);
    });
}

pcr_status pcr_run_until_idle(pcr_ctx* ctx)
{
    return guard([&] { E(ctx).run_until_idle(); });
}

pcr_status pcr_serve_start(pcr_ctx* ctx)
{
    return guard([&] { E(ctx).serve_start(); });
}

pcr_status pcr_serve_stop(pcr_ctx* ctx)
{
    return guard([&] { E(ctx).serve_stop(); });
}

pcr_status pcr_poll(pcr_ctx* ctx, pcr_request_id id, int32_t* done)
{
    return guard([&] {
        if (!done) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        *done = E(ctx).poll(id) ? 1 : 0;
    });
}

pcr_status pcr_wait(pcr_ctx* ctx, pcr_request_id id, int64_t timeout_ms)
{
    return guard([&] { E(ctx).wait(id, timeout_ms); });
}

pcr_status pcr_fetch(pcr_ctx* ctx, pcr_request_id id, float* hdr_out, uint8_t* rgb8_out, pcr_render_stats* stats)
{
    return guard([&] { E(ctx).fetch(id, hdr_out, rgb8_out, stats); });
}

pcr_status pcr_cancel(pcr_ctx* ctx, pcr_request_id id)
{
    return guard([&] { E(ctx).cancel(id); });
}

pcr_status pcr_l2_bandwidth(pcr_ctx* ctx, int64_t bytes, int32_t reps, double* gbs)
{
    return guard([&] {
        if (!gbs) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        *gbs = E(ctx).l2_bandwidth(bytes, reps);
    });
}

pcr_status pcr_progress(pcr_ctx* ctx, pcr_request_id id, double* fraction)
{
    return guard([&] {
        if (!fraction) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        *fraction = E(ctx).progress(id);
    });
}

pcr_status pcr_engine_stats_get(pcr_ctx* ctx, pcr_engine_stats* out)
{
    return guard([&] {
        if (!out) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        E(ctx).stats(out);
    });
}

pcr_status pcr_engine_stats_reset(pcr_ctx* ctx)
{
    return guard([&] { E(ctx).reset_stats(); });
}

pcr_status pcr_autotune(pcr_ctx* ctx, const pcr_scene_id* scenes, const pcr_render_desc* descs, int32_t n,
                        int32_t* chosen)
{
    return guard([&] {
        if (!scenes || !descs || n <= 0) throw pcr::PcrError(PCR_ERR_INVALID, "autotune needs a sample workload");
        E(ctx).autotune(scenes, descs, n, chosen);
    });
}

pcr_status pcr_trace_closest(pcr_ctx* ctx, pcr_scene_id scene, const float* rays, int64_t n, int32_t* mat,
                             int32_t* prim, float* t)
{
    return guard([&] {
        if (!rays && n > 0) throw pcr::PcrError(PCR_ERR_INVALID, "null rays");
        E(ctx).trace(scene, rays, n, mat, prim, t, 0, nullptr);
    });
}

pcr_status pcr_trace_bvh(pcr_ctx* ctx, pcr_scene_id scene, const float* rays, int64_t n, int32_t* tri_id, float* t,
                         int32_t* counts)
{
    return guard([&] {
        if (!rays && n > 0) throw pcr::PcrError(PCR_ERR_INVALID, "null rays");
        E(ctx).trace(scene, rays, n, nullptr, tri_id, t, 1, counts);
    });
}

pcr_status pcr_tonemap(pcr_ctx* ctx, const float* hdr, int32_t width, int32_t height, int32_t aces, int32_t denoise,
                       uint8_t* rgb8_out)
{
    return guard([&] {
        if (!hdr || !rgb8_out) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        E(ctx).tonemap(hdr, width, height, aces, denoise, rgb8_out);
    });
}

pcr_status pcr_router_create(pcr_router** out, pcr_ctx* const* ctxs, int32_t n)
{
    return guard([&] {
        if (!out || !ctxs || n <= 0) throw pcr::PcrError(PCR_ERR_INVALID, "router needs at least one context");
        auto r = std::make_unique<pcr_router>();
        for (int i = 0; i < n; i++) r->eng.push_back(&E(ctxs[i]));
        r->load.assign(n, 0);
        r->routed.assign(n, 0);
        *out = r.release();
    });
}

pcr_status pcr_router_destroy(pcr_router* r)
{
    return guard([&] { delete r; });
}

namespace {
pcr_router& RT(pcr_router* r)
{
    if (!r) throw pcr::PcrError(PCR_ERR_INVALID, "null router");
    return *r;
}
}  // namespace

pcr_status pcr_router_scene_load_json(pcr_router* r, const char* path, const char* data_root, const char* lut_path,
                                      pcr_scene_id* out)
{
    return guard([&] {
        pcr_router& R = RT(r);
        if (!path || !out) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        pcr::HostScene hs = host_scene_from_json(path, data_root, lut_path, false);
        device_bvh(*R.eng[0], hs);   // built once, uploaded to every context
        const pcr_scene_desc d = hs.desc();
        std::vector<int> ids;
        for (pcr::Engine* e : R.eng) ids.push_back(e->upload_scene(d));
        std::lock_guard<std::mutex> g(R.mu);
        R.scene_map.push_back(ids);
        *out = (pcr_scene_id)R.scene_map.size() - 1;
    });
}

pcr_status pcr_router_serve_start(pcr_router* r)
{
    return guard([&] {
        for (pcr::Engine* e : RT(r).eng) e->serve_start();
    });
}

pcr_status pcr_router_serve_stop(pcr_router* r)
{
    return guard([&] {
        for (pcr::Engine* e : RT(r).eng) e->serve_stop();
    });
}

pcr_status pcr_router_submit(pcr_router* r, pcr_scene_id scene, const pcr_render_desc* desc, int64_t* ticket)
{
    return guard([&] {
        pcr_router& R = RT(r);
        if (!desc || !ticket) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        std::lock_guard<std::mutex> g(R.mu);
        if (scene < 0 || scene >= (int)R.scene_map.size()) throw pcr::PcrError(PCR_ERR_NOT_FOUND, "unknown scene");
        int best = 0;
        for (int i = 1; i < (int)R.eng.size(); i++)
            if (R.load[i] < R.load[best]) best = i;
        const int64_t paths = (int64_t)desc->width * desc->height * desc->samples * std::max(1, desc->aa_samples);
        const int64_t id = R.eng[best]->submit(R.scene_map[scene][best], *desc);
        R.load[best] += paths;
        R.routed[best]++;
        *ticket = R.next++;
        R.tickets[*ticket] = {best, id, paths};
    });
}

namespace {
pcr_router::Ticket ticket_of(pcr_router& R, int64_t t)
{
    std::lock_guard<std::mutex> g(R.mu);
    auto it = R.tickets.find(t);
    if (it == R.tickets.end()) throw pcr::PcrError(PCR_ERR_NOT_FOUND, "unknown ticket");
    return it->second;
}
}  // namespace

pcr_status pcr_router_wait(pcr_router* r, int64_t ticket, int64_t timeout_ms)
{
    return guard([&] {
        pcr_router& R = RT(r);
        const pcr_router::Ticket t = ticket_of(R, ticket);
        R.eng[t.ctx]->wait(t.id, timeout_ms);
    });
}

pcr_status pcr_router_fetch(pcr_router* r, int64_t ticket, float* hdr_out, uint8_t* rgb8_out,
                            pcr_render_stats* stats)
{
    return guard([&] {
        pcr_router& R = RT(r);
        const pcr_router::Ticket t = ticket_of(R, ticket);
        R.eng[t.ctx]->fetch(t.id, hdr_out, rgb8_out, stats);
        std::lock_guard<std::mutex> g(R.mu);
        R.load[t.ctx] -= t.paths;
        R.tickets.erase(ticket);
    });
}

pcr_status pcr_router_load(pcr_router* r, int64_t* outstanding_paths, int64_t* routed)
{
    return guard([&] {
        pcr_router& R = RT(r);
        std::lock_guard<std::mutex> g(R.mu);
        for (size_t i = 0; i < R.eng.size(); i++) {
            if (outstanding_paths) outstanding_paths[i] = R.load[i];
            if (routed) routed[i] = R.routed[i];
        }
    });
}

pcr_status pcr_trace_shadow(pcr_ctx* ctx, pcr_scene_id scene, const float* rays, const float* light_dist2, int64_t n,
                            int32_t* blocked)
{
    return guard([&] {
        if ((!rays || !light_dist2 || !blocked) && n > 0) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        E(ctx).trace_shadow(scene, rays, light_dist2, n, blocked);
    });
}

pcr_status pcr_bvh_build(pcr_ctx* ctx, const pcr_triangle* tris, int32_t n, pcr_bvh_node* nodes_out,
                         int32_t max_nodes, int32_t* n_nodes, int32_t* order_out)
{
    return guard([&] {
        if (n < 0 || max_nodes < 0) throw pcr::PcrError(PCR_ERR_INVALID, "negative count");
        if (!n_nodes || (n > 0 && (!tris || !order_out || !nodes_out))) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        std::vector<pcr_bvh_node> nodes;
        std::vector<int32_t> order;
        E(ctx).build_bvh(tris, n, nodes, order);
        if ((int64_t)nodes.size() > max_nodes) throw pcr::PcrError(PCR_ERR_INVALID, "nodes_out too small");
        std::copy(nodes.begin(), nodes.end(), nodes_out);
        std::copy(order.begin(), order.end(), order_out);
        *n_nodes = (int32_t)nodes.size();
    });
}

pcr_status pcr_eval_stage(pcr_ctx* ctx, int32_t what, const float* params, const float* in, int64_t n, float* out)
{
    return guard([&] {
        if (!in || !out) throw pcr::PcrError(PCR_ERR_INVALID, "null argument");
        E(ctx).eval_stage(what, params, in, n, out);
    });
}

}  // extern "C"
