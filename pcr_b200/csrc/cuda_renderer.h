// CudaRenderer: the reference GPU renderer's public surface on top of the C
// ABI (include/pcr_cuda.h).
//
// Mirrors code/Gpu/Opengl/OpenglRenderer.h:29-117 and the CPU Renderer's
// knobs (code/Includes/Renderer.h:41-109): the (width, height, depth,
// samples, shadowSamples, sharedContext) constructor, the public quality
// fields, render(scene, start, outputDir) writing the tone-mapped PNG with
// the reference's filename and tEXt keys, and lastOutputPath.  `samples` is
// paths per pixel, as on the reference GPU backends.  No exception leaves
// render(): errors print to stderr and leave lastOutputPath empty.
#pragma once

#include <array>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "pcr_cuda.h"

struct GLFWwindow;

namespace pcr {

struct RenderOutput {
    std::vector<float> hdr;       // W*H*3 linear sRGB
    std::vector<uint8_t> rgb8;    // W*H*3 tone-mapped, quantised (and denoised)
};

// PNG (RGB8) with tEXt chunks ahead of IDAT (code/Includes/PngText.h:32-63).
bool write_png(const std::string& path, const uint8_t* rgb, int width, int height,
               const std::vector<std::pair<std::string, std::string>>& text);

class CudaRenderer {
public:
    CudaRenderer(int width, int height, int depth, int samples, int shadowSamples, GLFWwindow* sharedContext = nullptr);
    ~CudaRenderer();
    CudaRenderer(const CudaRenderer&) = delete;
    CudaRenderer& operator=(const CudaRenderer&) = delete;

    std::atomic<int>* progressRows = nullptr;
    std::atomic<bool>* cancelRequested = nullptr;
    std::function<void(const std::vector<std::array<float, 3>>&, int width, int height)> onPartialFrame;

    bool useDenoise = false;
    bool useMIS = false;
    bool useRussian = false;
    bool useStratified = false;
    bool useACES = false;
    int aaSamples = 1;
    bool useAdaptive = false;
    bool useOIDN = false;
    bool useSpectral = false;
    int heroSamples = 4;
    int threadgroupX = 8;     // accepted for surface compatibility; block size is autotuned
    int threadgroupY = 8;
    bool useWavefront = true; // always wavefront on this backend
    bool wavefrontMultiSample = false;
    bool spectralFork = true;
    uint64_t seed = 0;        // 0: a fresh seed per render

    // Renders `scene` and writes <outputDir>/<name>-<version>-<timestamp>-d#-s#-S#-w#[-h#][-spectral][-aces]-t<ms>.png
    void render(const pcr_scene_desc& scene, std::chrono::steady_clock::time_point start, const std::string& outputDir);
    // Renders without writing a file.
    bool render_to(const pcr_scene_desc& scene, RenderOutput& out);

    std::string lastOutputPath;
    std::string binaryName = "pcr-render";

private:
    pcr_render_desc desc() const;
    int _width, _height, _maxDepth, _samples, _shadowSamples;
    pcr_ctx* _ctx = nullptr;
    const void* _scene_key = nullptr;
    pcr_scene_id _scene = -1;
};

}  // namespace pcr
