// CudaRenderer: see cuda_renderer.h.
#include "cuda_renderer.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <iostream>
#include <random>

namespace pcr {

// ------------------------------------------------------------------ PNG
namespace {
void put32(std::vector<uint8_t>& o, uint32_t v)
{
    o.push_back((uint8_t)(v >> 24));
    o.push_back((uint8_t)(v >> 16));
    o.push_back((uint8_t)(v >> 8));
    o.push_back((uint8_t)v);
}
void chunk(std::vector<uint8_t>& o, const char* type, const std::vector<uint8_t>& data)
{
    put32(o, (uint32_t)data.size());
    size_t start = o.size();
    o.insert(o.end(), type, type + 4);
    o.insert(o.end(), data.begin(), data.end());
    uLong crc = crc32(0L, Z_NULL, 0);
    crc = crc32(crc, o.data() + start, (uInt)(o.size() - start));
    put32(o, (uint32_t)crc);
}

std::string compress_zone(const std::string& z)
{
    // strftime("%Z") gives long names on some platforms; keep the short
    // POSIX form (code/Renderer.cpp:37-74)
    if (z.find(' ') == std::string::npos) return z;
    std::string a;
    bool start = true;
    for (char c : z) {
        if (c == ' ') { start = true; continue; }
        if (start && std::isalpha((unsigned char)c)) a += (char)std::toupper((unsigned char)c);
        start = false;
    }
    return a.empty() ? z : a;
}

std::string timestamp()
{
    // "YYYYMMDD-HHMMSS-<ZONE>", local time (code/Renderer.cpp:79-105)
    std::time_t now = std::time(nullptr);
    std::tm tm{};
    localtime_r(&now, &tm);
    char buf[64], zone[64];
    std::strftime(buf, sizeof(buf), "%Y%m%d-%H%M%S", &tm);
    std::strftime(zone, sizeof(zone), "%Z", &tm);
    return std::string(buf) + "-" + compress_zone(zone);
}
}  // namespace

bool write_png(const std::string& path, const uint8_t* rgb, int width, int height,
               const std::vector<std::pair<std::string, std::string>>& text)
{
    std::vector<uint8_t> o = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    std::vector<uint8_t> ihdr;
    put32(ihdr, (uint32_t)width);
    put32(ihdr, (uint32_t)height);
    ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // 8-bit RGB
    chunk(o, "IHDR", ihdr);
    for (const auto& kv : text) {  // tEXt ahead of IDAT
        std::vector<uint8_t> t(kv.first.begin(), kv.first.end());
        t.push_back(0);
        t.insert(t.end(), kv.second.begin(), kv.second.end());
        chunk(o, "tEXt", t);
    }
    std::vector<uint8_t> raw((size_t)(width * 3 + 1) * height);
    for (int y = 0; y < height; y++) {
        raw[(size_t)y * (width * 3 + 1)] = 0;
        std::memcpy(&raw[(size_t)y * (width * 3 + 1) + 1], rgb + (size_t)y * width * 3, (size_t)width * 3);
    }
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<uint8_t> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) return false;
    z.resize(zlen);
    chunk(o, "IDAT", z);
    chunk(o, "IEND", {});
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = std::fwrite(o.data(), 1, o.size(), f) == o.size();
    ok = std::fclose(f) == 0 && ok;
    return ok;
}

// ------------------------------------------------------------------ renderer
CudaRenderer::CudaRenderer(int width, int height, int depth, int samples, int shadowSamples, GLFWwindow*)
    : _width(width), _height(height), _maxDepth(depth), _samples(samples), _shadowSamples(shadowSamples)
{
}

CudaRenderer::~CudaRenderer()
{
    if (_ctx) pcr_ctx_destroy(_ctx);
}

pcr_render_desc CudaRenderer::desc() const
{
    pcr_render_desc d{};
    d.width = _width;
    d.height = _height;
    d.depth = _maxDepth;
    d.samples = _samples;
    d.shadow_samples = _shadowSamples;
    d.spectral = useSpectral;
    d.hero_samples = heroSamples;
    d.mis = useMIS;
    d.russian = useRussian;
    d.stratified = useStratified;
    d.aa_samples = std::max(1, aaSamples);
    d.adaptive = useAdaptive;
    d.aces = useACES;
    d.denoise = useDenoise;
    d.multi_sample = wavefrontMultiSample;
    d.spectral_terminate = spectralFork ? 0 : 1;
    d.seed = seed ? seed : (uint64_t)std::random_device{}() << 32 | std::random_device{}();
    return d;
}

bool CudaRenderer::render_to(const pcr_scene_desc& scene, RenderOutput& out)
{
    if (!_ctx) {
        pcr_ctx_opts o{};
        const char* dev = std::getenv("PCR_DEVICE");
        o.device = dev ? std::atoi(dev) : 0;
        o.use_graph = 1;
        if (pcr_ctx_create(&_ctx, &o) != PCR_OK) {
            std::cerr << "pcr: " << pcr_last_error() << std::endl;
            _ctx = nullptr;
            return false;
        }
    }
    const void* key = scene.materials;
    if (_scene < 0 || key != _scene_key) {
        if (_scene >= 0) pcr_scene_release(_ctx, _scene);
        _scene = -1;
        if (pcr_scene_upload(_ctx, &scene, &_scene) != PCR_OK) {
            std::cerr << "pcr: scene upload failed: " << pcr_last_error() << std::endl;
            return false;
        }
        _scene_key = key;
    }
    pcr_render_desc d = desc();
    out.hdr.assign((size_t)_width * _height * 3, 0.f);
    out.rgb8.assign((size_t)_width * _height * 3, 0);
    pcr_render_stats st{};
    pcr_request_id id = -1;
    if (pcr_submit(_ctx, _scene, &d, &id) != PCR_OK) {
        std::cerr << "pcr: render failed: " << pcr_last_error() << std::endl;
        return false;
    }
    // The render runs as blocks of graph-captured iterations driven from this
    // thread.  Between blocks the loop reports progress and honours a cancel
    // request, as the reference renderers poll between pixels or tiles
    // (code/Renderer.cpp:170-181, code/Gpu/Opengl/OpenglRenderer.cpp:2170-2175).
    bool cancel_sent = false;
    while (true) {
        const pcr_status w = pcr_wait(_ctx, id, 20);
        if (w == PCR_OK) break;
        if (w == PCR_ERR_CANCELLED) {
            pcr_fetch(_ctx, id, nullptr, nullptr, nullptr);  // reports the cancel and releases the request
            if (progressRows) progressRows->store(0, std::memory_order_relaxed);
            std::cout << "GPU render cancelled." << std::endl;
            return false;
        }
        if (w != PCR_ERR_TIMEOUT) {
            std::cerr << "pcr: render failed: " << pcr_last_error() << std::endl;
            return false;
        }
        double f = 0.0;
        if (progressRows && pcr_progress(_ctx, id, &f) == PCR_OK)
            progressRows->store((int)(f * _height), std::memory_order_relaxed);
        if (!cancel_sent && cancelRequested && cancelRequested->load(std::memory_order_relaxed)) {
            pcr_cancel(_ctx, id);
            cancel_sent = true;
        }
    }
    if (pcr_fetch(_ctx, id, out.hdr.data(), out.rgb8.data(), &st) != PCR_OK) {
        std::cerr << "pcr: render failed: " << pcr_last_error() << std::endl;
        return false;
    }
    if (useOIDN)
        std::cerr << "warning: --oidn requested but binary was not built with PCR_USE_OIDN=ON; skipping denoise.\n";
    // the bilateral denoise (useDenoise) runs on the device after the resolve
    if (progressRows) progressRows->store(_height, std::memory_order_relaxed);
    if (onPartialFrame) {
        std::vector<std::array<float, 3>> fb((size_t)_width * _height);
        for (size_t i = 0; i < fb.size(); i++) fb[i] = {out.hdr[i * 3], out.hdr[i * 3 + 1], out.hdr[i * 3 + 2]};
        onPartialFrame(fb, _width, _height);
    }
    return true;
}

void CudaRenderer::render(const pcr_scene_desc& scene, std::chrono::steady_clock::time_point start,
                          const std::string& outputDir)
{
    lastOutputPath.clear();
    if (cancelRequested && cancelRequested->load(std::memory_order_relaxed)) {
        std::cout << "Render cancelled before write." << std::endl;
        return;
    }
    RenderOutput out;
    if (!render_to(scene, out)) return;
    if (cancelRequested && cancelRequested->load(std::memory_order_relaxed)) {
        std::cout << "Render cancelled before write." << std::endl;
        return;
    }
    auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - start).count();
    std::cout << "Render took " << ms << " ms" << std::endl;
    const std::string ts = timestamp();
    std::string name = std::string(scene.name ? scene.name : "scene") + "-" + (scene.version ? scene.version : "") +
                       "-" + ts + "-d" + std::to_string(_maxDepth) + "-s" + std::to_string(_samples) + "-S" +
                       std::to_string(_shadowSamples) + "-w" + std::to_string(_width);
    if (_width != _height) name += "-h" + std::to_string(_height);
    if (useSpectral) name += "-spectral";
    if (useACES) name += "-aces";
    name += "-t" + std::to_string(ms) + ".png";
    std::filesystem::path p = std::filesystem::path(outputDir) / name;
    std::error_code ec;
    std::filesystem::create_directories(p.parent_path(), ec);
    // tEXt keys of code/Renderer.cpp:429-447
    std::vector<std::pair<std::string, std::string>> text = {
        {"Software", binaryName}, {"Scene", scene.name ? scene.name : ""},
        {"SceneVersion", scene.version ? scene.version : ""}, {"CreationTime", ts},
        {"Depth", std::to_string(_maxDepth)}, {"Samples", std::to_string(_samples)},
        {"ShadowSamples", std::to_string(_shadowSamples)}, {"Width", std::to_string(_width)},
        {"Height", std::to_string(_height)}, {"RenderTimeMs", std::to_string(ms)},
        {"Denoise", useDenoise ? "1" : "0"}, {"MIS", useMIS ? "1" : "0"}, {"Russian", useRussian ? "1" : "0"},
        {"Stratified", useStratified ? "1" : "0"}, {"Tonemap", useACES ? "ACES" : "Reinhard"},
        {"AASamples", std::to_string(aaSamples)}, {"Adaptive", useAdaptive ? "1" : "0"},
        {"OIDN", useOIDN ? "1" : "0"}, {"Spectral", useSpectral ? "1" : "0"}};
    if (!write_png(p.string(), out.rgb8.data(), _width, _height, text)) {
        std::cerr << "png save error (path: " << p << ")" << std::endl;
        return;
    }
    std::cout << "Wrote " << p << std::endl;
    lastOutputPath = p.string();
}

}  // namespace pcr
