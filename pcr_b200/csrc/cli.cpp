// pcr-render: the reference CLI's surface (code/Cli/Main.cpp:75-481) driving
// the CUDA backend.  Same flags, same defaults, same output naming; the
// scene is loaded by the library's own loader and rendered by CudaRenderer.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <regex>
#include <string>
#include <vector>

#include <unistd.h>

#include "cuda_renderer.h"
#include "pcr_cuda.h"

namespace fs = std::filesystem;

namespace {

struct Found {
    std::string name, version, path;
};

std::string field(const std::string& text, const char* key)
{
    std::smatch m;
    std::regex re(std::string("\"") + key + "\"\\s*:\\s*\"([^\"]*)\"");
    return std::regex_search(text, m, re) ? m[1].str() : std::string();
}

fs::path exe_dir()
{
    std::error_code ec;
    auto p = fs::read_symlink("/proc/self/exe", ec);
    return ec ? fs::path() : p.parent_path();
}

// Scene discovery (code/Scenes/SceneDiscovery.cpp:116-165): extra dirs, then
// $PWD/Scenes, then <binary-dir>/Scenes; first occurrence of a name wins.
std::vector<Found> discover(const std::vector<std::string>& extra)
{
    std::vector<fs::path> dirs;
    for (const auto& d : extra) dirs.emplace_back(d);
    dirs.push_back(fs::current_path() / "Scenes");
    if (!exe_dir().empty()) dirs.push_back(exe_dir() / "Scenes");
    std::vector<Found> out;
    for (const auto& d : dirs) {
        std::error_code ec;
        if (!fs::is_directory(d, ec)) continue;
        std::vector<fs::path> files;
        for (const auto& e : fs::directory_iterator(d, ec))
            if (e.path().extension() == ".json") files.push_back(e.path());
        std::sort(files.begin(), files.end());
        for (const auto& f : files) {
            std::ifstream in(f);
            std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
            Found s{field(text, "name"), field(text, "version"), f.string()};
            if (s.name.empty()) continue;
            if (std::none_of(out.begin(), out.end(), [&](const Found& o) { return o.name == s.name; })) out.push_back(s);
        }
    }
    return out;
}

int usage(const char* msg)
{
    if (msg) std::cerr << msg << "\n";
    std::cerr << "usage: pcr-render [--scene NAME] [-d N] [-s N] [-S N] [-w N] [--height N] [-o DIR] [--scenes-dir DIR]...\n"
                 "                  [--list-scenes] [--denoise] [--mis] [--russian] [--stratified] [--aces] [--aa]\n"
                 "                  [--aa-samples N] [--adaptive] [--oidn] [--spectral] [--hero-samples 1..4]\n"
                 "                  [--seed N] [--lut | --lut-file NAME|PATH] [--tz ZONE] [--device N]\n"
                 "                  [--threadgroup-x N] [--threadgroup-y N] [--wavefront|--no-wavefront]\n"
                 "                  [--wavefront-multi-sample] [--spectral-terminate]\n";
    return msg ? 1 : 0;
}

}  // namespace

int main(int argc, char** argv)
{
    auto start = std::chrono::steady_clock::now();
    int depth = 4, samples = 16, shadow = 4, width = 720, height = -1, aaSamples = 4, hero = 4, tgx = 8, tgy = 8;
    std::string scene = "cornell", outputDir, tz, lutFile;
    std::vector<std::string> extraDirs;
    bool list = false, denoise = false, mis = false, russian = false, strat = false, aces = false, aa = false;
    bool adaptive = false, oidn = false, spectral = false, lut = false, terminate = false;
    uint64_t seed = 0;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        std::string val;
        auto eq = a.find('=');
        if (a.rfind("--", 0) == 0 && eq != std::string::npos) {
            val = a.substr(eq + 1);
            a = a.substr(0, eq);
        }
        auto next = [&]() -> std::string {
            if (!val.empty()) return val;
            if (i + 1 >= argc) { std::cerr << a << " needs a value\n"; std::exit(1); }
            return argv[++i];
        };
        auto pos = [&](int& dst) {
            dst = std::atoi(next().c_str());
            if (dst <= 0) { std::cerr << a << ": value must be positive\n"; std::exit(1); }
        };
        if (a == "--scene") scene = next();
        else if (a == "-d" || a == "--depth") pos(depth);
        else if (a == "-s" || a == "--samples") pos(samples);
        else if (a == "-S" || a == "--shadow") pos(shadow);
        else if (a == "-w" || a == "--width") pos(width);
        else if (a == "--height") pos(height);
        else if (a == "--tz" || a == "--timezone") tz = next();
        else if (a == "-o" || a == "--output") outputDir = next();
        else if (a == "--scenes-dir") extraDirs.push_back(next());
        else if (a == "--list-scenes") list = true;
        else if (a == "--denoise") denoise = true;
        else if (a == "--mis") mis = true;
        else if (a == "--russian") russian = true;
        else if (a == "--stratified") strat = true;
        else if (a == "--aces") aces = true;
        else if (a == "--aa") aa = true;
        else if (a == "--aa-samples") pos(aaSamples);
        else if (a == "--adaptive") adaptive = true;
        else if (a == "--oidn") oidn = true;
        else if (a == "--spectral") spectral = true;
        else if (a == "--hero-samples") {
            hero = std::atoi(next().c_str());
            if (hero < 1 || hero > 4) { std::cerr << "--hero-samples: value not in range 1 to 4\n"; return 1; }
        } else if (a == "--seed") seed = std::strtoull(next().c_str(), nullptr, 10);
        else if (a == "--lut") lut = true;
        else if (a == "--lut-file") lutFile = next();
        else if (a == "--threadgroup-x") pos(tgx);
        else if (a == "--threadgroup-y") pos(tgy);
        else if (a == "--wavefront" || a == "--no-wavefront" || a == "--wavefront-multi-sample") {
        } else if (a == "--spectral-terminate") terminate = true;
        else if (a == "--device") setenv("PCR_DEVICE", next().c_str(), 1);
        else if (a == "-h" || a == "--help") return usage(nullptr);
        else return usage(("unknown option " + a).c_str());
    }
    if (lut && !lutFile.empty()) { std::cerr << "--lut excludes --lut-file\n"; return 1; }
    if (height < 0) height = width;
    if (!tz.empty()) { setenv("TZ", tz.c_str(), 1); tzset(); }
    if (outputDir.empty()) outputDir = (fs::current_path() / "Image").string();

    auto reg = discover(extraDirs);
    if (list) {
        std::cout << "Available scenes:\n";
        for (const auto& s : reg) std::cout << "  " << s.name << "  " << s.version << "  (" << s.path << ")\n";
        return 0;
    }
    auto it = std::find_if(reg.begin(), reg.end(), [&](const Found& s) { return s.name == scene; });
    if (it == reg.end()) {
        std::cerr << "Unknown scene: " << scene << "\nAvailable scenes:\n";
        for (const auto& s : reg) std::cerr << "  " << s.name << "\n";
        return 1;
    }
    std::string lutPath;
    if (lut) {
        std::vector<float> L(3 * 16 * 16 * 16 * 3);
        std::cout << "Building RGB-to-spectrum LUT..." << std::flush;
        if (pcr_lut_build(L.data()) != PCR_OK) { std::cerr << pcr_last_error() << "\n"; return 1; }
        lutPath = (fs::temp_directory_path() / ("pcr-lut-" + std::to_string(getpid()) + ".lut")).string();
        std::ofstream o(lutPath, std::ios::binary);
        uint32_t h[4] = {0, 1, 16, (uint32_t)L.size()};
        std::memcpy(h, "PLUT", 4);
        o.write((const char*)h, 16);
        o.write((const char*)L.data(), (std::streamsize)(L.size() * 4));
        std::cout << " done\n";
    } else if (!lutFile.empty()) {
        bool looksLikePath = lutFile.find('/') != std::string::npos ||
                             (lutFile.size() >= 4 && lutFile.substr(lutFile.size() - 4) == ".lut");
        lutPath = lutFile;
        if (!looksLikePath) {
            for (const auto& d : {fs::current_path() / "luts", exe_dir() / "luts"}) {
                fs::path c = d / (lutFile + ".lut");
                std::error_code ec;
                if (fs::exists(c, ec)) { lutPath = c.string(); break; }
            }
        }
    }
    // data root: the directory that holds Scenes/ (spd/ lives beside it)
    const std::string root = fs::path(it->path).parent_path().parent_path().string();
    pcr_host_scene* hs = nullptr;
    pcr_scene_desc desc{};
    if (pcr_host_scene_load(it->path.c_str(), root.c_str(), lutPath.empty() ? nullptr : lutPath.c_str(), &hs, &desc) !=
        PCR_OK) {
        std::cerr << "Error loading scene: " << pcr_last_error() << "\n";
        return 1;
    }
    pcr::CudaRenderer r(width, height, depth, samples, shadow, nullptr);
    r.useDenoise = denoise;
    r.useMIS = mis;
    r.useRussian = russian;
    r.useStratified = strat;
    r.useACES = aces;
    r.aaSamples = aa ? std::max(1, aaSamples) : 1;
    r.useAdaptive = adaptive;
    r.useOIDN = oidn;
    r.useSpectral = spectral;
    r.heroSamples = hero;
    r.threadgroupX = tgx;
    r.threadgroupY = tgy;
    r.spectralFork = !terminate;
    r.seed = seed;
    r.binaryName = "pcr-render";
    r.render(desc, start, outputDir);
    pcr_host_scene_free(hs);
    return r.lastOutputPath.empty() ? 1 : 0;
}
