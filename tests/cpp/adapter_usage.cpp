// Compile check of the reference-tree adapter (pcr_b200/csrc/adapter/
// CudaRenderer.h) against the reference's own headers: the GpuRenderer
// alias the adapter is written for, and the calls code/Cli/Main.cpp:445-473
// makes on it, in the same form.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <string>
#include <vector>

#include "CudaRenderer.h"

using GpuRenderer = CudaRenderer;

int cli_like(const Scenes::SceneData &sceneData, std::chrono::steady_clock::time_point start,
             const std::string &outputDir)
{
    int width = 64, height = 48, depth = 3, samples = 8, shadowSamples = 2, aaSamples = 4, heroSamples = 4;
    bool useDenoise = false, useMIS = true, useRussian = false, useStratified = false, useACES = false,
         useAA = true, useAdaptive = false, useOIDN = false, useSpectral = true, useWavefront = true,
         wavefrontMultiSample = false, spectralTerminate = false;
    int threadgroupX = 8, threadgroupY = 8;
    GLFWwindow *gpuShared = nullptr;
    GpuRenderer renderer{width, height, depth, samples, shadowSamples, gpuShared};
    renderer.useDenoise = useDenoise;
    renderer.useMIS = useMIS;
    renderer.useRussian = useRussian;
    renderer.useStratified = useStratified;
    renderer.useACES = useACES;
    renderer.aaSamples = useAA ? std::max(1, aaSamples) : 1;
    renderer.useAdaptive = useAdaptive;
    renderer.useOIDN = useOIDN;
    renderer.useSpectral = useSpectral;
    renderer.heroSamples = heroSamples;
    renderer.threadgroupX = threadgroupX;
    renderer.threadgroupY = threadgroupY;
    renderer.useWavefront = useWavefront;
    renderer.wavefrontMultiSample = wavefrontMultiSample;
    renderer.spectralFork = !spectralTerminate;
    // the GUI's hooks (code/Includes/Renderer.h:41-43)
    std::atomic<int> rows{0};
    std::atomic<bool> cancel{false};
    renderer.progressRows = &rows;
    renderer.cancelRequested = &cancel;
    renderer.onPartialFrame = [](const std::vector<Vec3f> &fb, int w, int h) { (void)fb; (void)w; (void)h; };
    renderer.render(sceneData, start, outputDir);
    return renderer.lastOutputPath.empty() ? 1 : 0;
}
