// Drives pcr::CudaRenderer the way the reference GUI drives a GpuRenderer on
// its worker thread (code/Gui/main.cpp job queue): progressRows and
// cancelRequested are atomics the caller owns.
//
//   renderer_cancel <scene.json> <data root> <out dir>
//
// 1. A large render is cancelled from another thread once progressRows has
//    moved: render() must return early, without writing a PNG.
// 2. A small render runs to the end: progressRows reaches the height and the
//    PNG is written.
// Prints one line of key=value results for the test to check.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <thread>

#include "cuda_renderer.h"
#include "pcr_cuda.h"

int main(int argc, char** argv)
{
    if (argc < 4) return 2;
    pcr_host_scene* hs = nullptr;
    pcr_scene_desc desc{};
    if (pcr_host_scene_load(argv[1], argv[2], nullptr, &hs, &desc) != PCR_OK) {
        std::fprintf(stderr, "load: %s\n", pcr_last_error());
        return 1;
    }
    using clock = std::chrono::steady_clock;
    // 1024 x 1024, depth 8, 1024 paths per pixel: about 1.1 G paths, seconds
    // of work on one GPU
    pcr::CudaRenderer big(1024, 1024, 8, 1024, 4, nullptr);
    big.useSpectral = true;
    big.seed = 7;
    std::atomic<int> rows{0};
    std::atomic<bool> cancel{false};
    big.progressRows = &rows;
    big.cancelRequested = &cancel;
    int rows_at_cancel = -1;
    clock::time_point t_cancel{};
    std::thread watcher([&] {
        const auto t0 = clock::now();
        while (rows.load() <= 0 && clock::now() - t0 < std::chrono::seconds(120))
            std::this_thread::sleep_for(std::chrono::milliseconds(1));
        rows_at_cancel = rows.load();
        t_cancel = clock::now();
        cancel.store(true);
    });
    const auto t0 = clock::now();
    big.render(desc, t0, argv[3]);
    const auto t1 = clock::now();
    watcher.join();
    const double big_s = std::chrono::duration<double>(t1 - t0).count();
    const double cancel_s = std::chrono::duration<double>(t1 - t_cancel).count();
    const bool big_written = !big.lastOutputPath.empty();

    pcr::CudaRenderer small(64, 48, 3, 8, 2, nullptr);
    small.useSpectral = true;
    small.seed = 8;
    std::atomic<int> rows2{0};
    std::atomic<bool> cancel2{false};
    small.progressRows = &rows2;
    small.cancelRequested = &cancel2;
    small.render(desc, clock::now(), argv[3]);
    std::printf("rows_at_cancel=%d big_seconds=%.3f cancel_to_return=%.3f big_written=%d small_rows=%d "
                "small_written=%d\n",
                rows_at_cancel, big_s, cancel_s, big_written ? 1 : 0, rows2.load(), small.lastOutputPath.empty() ? 0 : 1);
    pcr_host_scene_free(hs);
    return 0;
}
