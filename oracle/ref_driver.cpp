// Test infrastructure only: an extern "C" harness around the reference CPU
// renderer, compiled from the reference's own unmodified sources by
// oracle/Makefile into oracle/_ref/libpcrref.so.  It is the checker for the
// CUDA path and the timed CPU baseline; nothing in pcr_b200/ links it.
//
// What it exposes (each entry forwards to the reference function named):
//   * scene load        -> Scenes::loadSceneFromFile   (code/Scenes/SceneLoader.cpp:475-516)
//   * scene export      -> SceneData fields            (code/Scenes/Scene.h:58-83)
//   * PNG render        -> Renderer::render            (code/Renderer.cpp:113-466)
//   * HDR harness       -> Renderer::castRaySpectral / castRay
//                                                      (code/Renderer.cpp:468-889)
//   * sceneIntersect    -> Renderer::sceneIntersect    (code/Renderer.cpp:891-949)
//   * BVH build/query   -> Bvh::build / Bvh::intersect (code/Bvh/Bvh.cpp:122-325, 353-444)
//   * stage functions   -> RGBToSpectrum / CIE / ToneMap / Optics headers
//
// The private members of Renderer are reached by compiling this one file
// with `private` defined as `public` (access only; layout is unchanged).

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <functional>
#include <numbers>
#include <string>
#include <thread>
#include <vector>
#include <unistd.h>

#define private public
#include "Includes/Renderer.h"
#undef private

#include "Bvh/Bvh.h"
#include "Includes/CIE.h"
#include "Includes/NumGen.h"
#include "Includes/Optics.h"
#include "Includes/RGBToSpectrum.h"
#include "Includes/Spectrum.h"
#include "Includes/ToneMap.h"
#include "Scenes/Scene.h"
#include "Scenes/SceneLoader.h"

// Defined in numgen_shim.cpp (same translation unit as the reference's
// NumGen.cpp): rewinds the per-thread stream counter so a seeded render in
// a long-lived process draws the same stream a fresh CLI process would.
extern "C" void pcr_ref_numgen_reset(void);

namespace
{
    struct RefScene
    {
        Scenes::SceneData data;
    };

    void copyErr(const std::string &msg, char *err, int errlen)
    {
        if (!err || errlen <= 0) return;
        std::snprintf(err, (size_t)errlen, "%s", msg.c_str());
    }

    // Renderer::render fills _planes (light planes first, then walls) at
    // code/Renderer.cpp:123-130 before tracing; the harness does the same.
    void preparePlanes(Renderer &r, const Scenes::SceneData &s, float &totalLightArea)
    {
        r._planes.clear();
        for (const auto &L : s.areaLights)
            if (L.kind == Scenes::AreaLightKind::Plane) r._planes.push_back(L.plane);
        for (const auto &w : s.walls) r._planes.push_back(w);
        totalLightArea = 0.f;
        for (const auto &L : s.areaLights) totalLightArea += L.totalArea;
    }

    std::unique_ptr<RGBToSpectrum::LUT> g_lut;
}

// Render options shared by the PNG and HDR entry points.  Field meaning is
// that of the Renderer knobs (code/Includes/Renderer.h:41-102).
struct RefRenderOpts
{
    int width, height, depth, samples, shadow;
    int spectral, mis, russian, stratified, aces, denoise;
    int aa, adaptive, hero;
    uint64_t seed;
};

extern "C" {

// ---------------------------------------------------------------- scenes

void *ref_scene_load(const char *jsonPath, const char *dataRoot, char *err, int errlen)
{
    // SpdLoader resolves "<name>.spd" under $PWD/spd (code/SpdLoader.cpp:93-98).
    std::error_code ec;
    auto oldCwd = std::filesystem::current_path(ec);
    if (dataRoot && *dataRoot) std::filesystem::current_path(dataRoot, ec);
    RefScene *s = nullptr;
    try
    {
        s = new RefScene{Scenes::loadSceneFromFile(jsonPath)};
    }
    catch (const std::exception &e)
    {
        copyErr(e.what(), err, errlen);
        s = nullptr;
    }
    std::filesystem::current_path(oldCwd, ec);
    return s;
}

void ref_scene_free(void *h) { delete (RefScene *)h; }

// out: [materials, spheres, walls, triangles, bvhNodes, areaLights]
void ref_scene_sizes(void *h, int *out)
{
    auto &s = ((RefScene *)h)->data;
    out[0] = (int)s.materials.size();
    out[1] = (int)s.spheres.size();
    out[2] = (int)s.walls.size();
    out[3] = (int)s.triangles.size();
    out[4] = (int)s.triangleBvh.size();
    out[5] = (int)s.areaLights.size();
}

void ref_scene_name(void *h, char *name, int nlen, char *version, int vlen)
{
    auto &s = ((RefScene *)h)->data;
    copyErr(s.name, name, nlen);
    copyErr(s.version, version, vlen);
}

void ref_scene_camera(void *h, float *out)
{
    auto &s = ((RefScene *)h)->data;
    out[0] = s.camera.position[0]; out[1] = s.camera.position[1];
    out[2] = s.camera.position[2]; out[3] = s.camera.fov;
}

// 142 floats per material: albedo3 emissive3 metallic transparent ior cauchyB
// useTabA useTabE albedoFit4 emissiveFit4 tabA61 tabE61
void ref_scene_materials(void *h, float *out)
{
    auto &s = ((RefScene *)h)->data;
    for (size_t i = 0; i < s.materials.size(); i++)
    {
        const Material &m = s.materials[i];
        float *o = out + i * 142;
        for (int k = 0; k < 3; k++) { o[k] = m.albedo[k]; o[3 + k] = m.emissive[k]; }
        o[6] = m.metallic; o[7] = m.transparent; o[8] = m.ior; o[9] = m.cauchyB;
        o[10] = m.useTabulatedAlbedo; o[11] = m.useTabulatedEmissive;
        o[12] = m.albedoFit.c0; o[13] = m.albedoFit.c1; o[14] = m.albedoFit.c2; o[15] = m.albedoFit.scale;
        o[16] = m.emissiveFit.c0; o[17] = m.emissiveFit.c1; o[18] = m.emissiveFit.c2; o[19] = m.emissiveFit.scale;
        for (int k = 0; k < 61; k++) { o[20 + k] = m.tabulatedAlbedo[k]; o[81 + k] = m.tabulatedEmissive[k]; }
    }
}

// Planes in the renderer's test order (light planes, then walls).
// 14 floats: origin3 u3 v3 N3 area matIdx.  Returns the count.
int ref_scene_planes(void *h, float *out)
{
    auto &s = ((RefScene *)h)->data;
    Renderer r(1, 1, 1, 1, 1);
    float total;
    preparePlanes(r, s, total);
    for (size_t i = 0; out && i < r._planes.size(); i++)
    {
        const Plane &p = r._planes[i];
        float *o = out + i * 14;
        for (int k = 0; k < 3; k++)
        {
            o[k] = p.origin[k]; o[3 + k] = p.getU()[k]; o[6 + k] = p.getV()[k]; o[9 + k] = p.N[k];
        }
        o[12] = p.getArea(); o[13] = (float)p.matIdx;
    }
    return (int)r._planes.size();
}

// 5 floats per sphere: center3 radius matIdx
void ref_scene_spheres(void *h, float *out)
{
    auto &s = ((RefScene *)h)->data;
    for (size_t i = 0; i < s.spheres.size(); i++)
    {
        const Sphere &sp = s.spheres[i];
        float *o = out + i * 5;
        o[0] = sp.center[0]; o[1] = sp.center[1]; o[2] = sp.center[2];
        o[3] = sp.radius(); o[4] = (float)sp.matIdx;
    }
}

// 23 floats per triangle (BVH-leaf order): v0 v1 v2 n0 n1 n2 flatN smooth matIdx
void ref_scene_triangles(void *h, float *out)
{
    auto &s = ((RefScene *)h)->data;
    for (size_t i = 0; i < s.triangles.size(); i++)
    {
        const Triangle &t = s.triangles[i];
        float *o = out + i * 23;
        const Vec3f *vs[7] = {&t.v0, &t.v1, &t.v2, &t.n0, &t.n1, &t.n2, &t.flatN};
        for (int a = 0; a < 7; a++)
            for (int k = 0; k < 3; k++) o[a * 3 + k] = (*vs[a])[k];
        o[21] = t.smooth ? 1.f : 0.f; o[22] = (float)t.matIdx;
    }
}

void ref_scene_bvh(void *h, float *boxes, int *ints)
{
    auto &s = ((RefScene *)h)->data;
    for (size_t i = 0; i < s.triangleBvh.size(); i++)
    {
        const Bvh::Node &n = s.triangleBvh[i];
        for (int k = 0; k < 3; k++) { boxes[i * 6 + k] = n.boxMin[k]; boxes[i * 6 + 3 + k] = n.boxMax[k]; }
        ints[i * 3 + 0] = n.leftOrFirst; ints[i * 3 + 1] = n.rightChild; ints[i * 3 + 2] = n.count;
    }
}

// 16 floats per light: kind totalArea nTris origin3 u3 v3 N3 matIdx
void ref_scene_lights(void *h, float *out)
{
    auto &s = ((RefScene *)h)->data;
    for (size_t i = 0; i < s.areaLights.size(); i++)
    {
        const auto &L = s.areaLights[i];
        float *o = out + i * 16;
        o[0] = L.kind == Scenes::AreaLightKind::Plane ? 0.f : 1.f;
        o[1] = L.totalArea;
        o[2] = (float)L.triangles.size();
        for (int k = 0; k < 3; k++)
        {
            o[3 + k] = L.plane.origin[k]; o[6 + k] = L.plane.getU()[k];
            o[9 + k] = L.plane.getV()[k]; o[12 + k] = L.plane.N[k];
        }
        o[15] = (float)L.plane.matIdx;
    }
}

// 15 floats per light triangle: v0 v1 v2 flatN matIdx cumulativeArea
void ref_scene_light_tris(void *h, int light, float *out)
{
    auto &L = ((RefScene *)h)->data.areaLights[(size_t)light];
    for (size_t i = 0; i < L.triangles.size(); i++)
    {
        const Triangle &t = L.triangles[i];
        float *o = out + i * 14;
        const Vec3f *vs[4] = {&t.v0, &t.v1, &t.v2, &t.flatN};
        for (int a = 0; a < 4; a++)
            for (int k = 0; k < 3; k++) o[a * 3 + k] = (*vs[a])[k];
        o[12] = (float)t.matIdx; o[13] = L.cumulativeArea[i];
    }
}

float ref_material_albedo_at(void *h, int mat, float lambda)
{
    return ((RefScene *)h)->data.materials[(size_t)mat].albedoAt(lambda);
}

float ref_material_emissive_at(void *h, int mat, float lambda)
{
    return ((RefScene *)h)->data.materials[(size_t)mat].emissiveAt(lambda);
}

// ---------------------------------------------------------------- LUT

// mode 0: none, 1: build in process (--lut), 2: load PLUT file (--lut-file)
int ref_set_lut(int mode, const char *path, char *err, int errlen)
{
    if (mode == 0)
    {
        RGBToSpectrum::setActiveLUT(nullptr);
        g_lut.reset();
        return 0;
    }
    auto lut = std::make_unique<RGBToSpectrum::LUT>();
    if (mode == 1)
        RGBToSpectrum::buildLUT(*lut);
    else
    {
        std::string e;
        if (!RGBToSpectrum::loadLUT(path, *lut, &e))
        {
            copyErr(e, err, errlen);
            return 1;
        }
    }
    g_lut = std::move(lut);
    RGBToSpectrum::setActiveLUT(g_lut.get());
    return 0;
}

// Copies the active LUT's coefficient array (3*16^3*3 floats); returns its size.
int ref_lut_data(float *out)
{
    if (!g_lut) return 0;
    if (out) std::memcpy(out, g_lut->data.data(), g_lut->data.size() * sizeof(float));
    return (int)g_lut->data.size();
}

int ref_lut_save(const char *path)
{
    return g_lut && RGBToSpectrum::saveLUT(*g_lut, path) ? 0 : 1;
}

// ---------------------------------------------------------------- render

// Full reference render to PNG: exactly what the CPU CLI does after scene
// load (code/Cli/Main.cpp:445-473).  Writes the PNG under outDir and copies
// its path to outPath.
int ref_render_png(void *h, const RefRenderOpts *o, const char *outDir, char *outPath, int outlen)
{
    auto &s = ((RefScene *)h)->data;
    NumGen::setSeed(o->seed);
    pcr_ref_numgen_reset();
    Renderer r(o->width, o->height, o->depth, o->samples, o->shadow);
    r.useDenoise = o->denoise; r.useMIS = o->mis; r.useRussian = o->russian;
    r.useStratified = o->stratified; r.useACES = o->aces;
    r.aaSamples = std::max(1, o->aa); r.useAdaptive = o->adaptive;
    r.useSpectral = o->spectral; r.heroSamples = o->hero;
    r.render(s, std::chrono::steady_clock::now(), outDir);
    copyErr(r.lastOutputPath, outPath, outlen);
    return r.lastOutputPath.empty() ? 1 : 0;
}

// One camera sample through pixel (i=row, j=col) with the reference's own
// primary-ray and hero-lambda construction (code/Renderer.cpp:196-257).
// Returns XYZ/N (spectral) or RGB.
static Vec3f cameraSample(Renderer &r, const Scenes::SceneData &s, const RefRenderOpts *o,
                          float totalLightArea, int i, int j, bool jitter)
{
    Vec3f origin = s.camera.position;
    float aspect = o->width / (float)o->height;
    float scale = std::tan((float)std::numbers::pi / 180.f * 0.5f * s.camera.fov);
    float jx = jitter ? (NumGen::Epsilon() - 0.5f) : 0.f;
    float jy = jitter ? (NumGen::Epsilon() - 0.5f) : 0.f;
    auto x = ((2 * (j + 0.5f + jx) / (float)o->width) - 1) * scale * aspect;
    auto y = -((2 * (i + 0.5f + jy) / (float)o->height) - 1) * scale;
    Ray ray(Vec3f(x, y, -1.f).normalize(), origin);
    if (!o->spectral)
        return r.castRay(ray, s.materials, s.spheres, s.triangles, s.triangleBvh,
                         s.areaLights, totalLightArea, 0);
    int N = std::clamp(o->hero, 1, kHeroLambdaCount);
    constexpr float kSpan = Spectrum::kLambdaMax - Spectrum::kLambdaMin;
    float kStride = kSpan / (float)N;
    SpectralSample lambdas;
    lambdas[0] = Spectrum::kLambdaMin + NumGen::Epsilon() * kSpan;
    for (int k = 1; k < N; k++)
    {
        float l = lambdas[0] + kStride * k;
        if (l > Spectrum::kLambdaMax) l -= kSpan;
        lambdas[k] = l;
    }
    for (int k = N; k < kHeroLambdaCount; k++) lambdas[k] = lambdas[0];
    SpectralSample rad = r.castRaySpectral(ray, s.materials, s.spheres, s.triangles,
                                           s.triangleBvh, s.areaLights, totalLightArea, 0, lambdas);
    Vec3f xyz(0.f, 0.f, 0.f);
    for (int k = 0; k < N; k++) xyz = xyz + CIE::singleLambdaXYZ(lambdas[k], rad[k]);
    return xyz / (float)N;
}

// HDR render in linear sRGB, accumulated per pixel in FP64.
//   mode 0 ("branched"): the CPU renderer's own estimator: `samples` indirect
//          branches per diffuse vertex, aa primary rays per pixel (jittered
//          when aa > 1), mean over aa.
//   mode 1 ("paths"): the GPU estimator: Renderer built with samples = 1,
//          `spp` camera paths through the pixel centre, mean over spp.
// threads == 0 uses hardware_concurrency.  A non-zero seed with threads == 1
// reproduces the reference's seeded single-thread stream.
// Returns the render-loop wall time in seconds (scene load excluded).
double ref_render_hdr(void *h, const RefRenderOpts *o, int mode, int spp, int threads,
                      int rowBegin, int rowEnd, double *out)
{
    auto &s = ((RefScene *)h)->data;
    NumGen::setSeed(o->seed);
    pcr_ref_numgen_reset();
    int nThreads = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    if (rowEnd <= 0 || rowEnd > o->height) rowEnd = o->height;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < nThreads; t++)
    {
        pool.emplace_back([&, t]() {
            Renderer r(o->width, o->height, o->depth, mode == 0 ? o->samples : 1, o->shadow);
            r.useMIS = o->mis; r.useRussian = o->russian; r.useStratified = o->stratified;
            r.useSpectral = o->spectral; r.heroSamples = o->hero;
            float totalLightArea;
            preparePlanes(r, s, totalLightArea);
            for (int i = rowBegin + t; i < rowEnd; i += nThreads)
            {
                for (int j = 0; j < o->width; j++)
                {
                    double acc[3] = {0, 0, 0};
                    int n = mode == 0 ? std::max(1, o->aa) : spp;
                    bool jitter = mode == 0 && o->aa > 1;
                    if (mode == 0)
                    {
                        // Welford mean in float exactly as Renderer::render.
                        Vec3f mean{0, 0, 0};
                        int taken = 0;
                        for (int k = 0; k < n; k++)
                        {
                            Vec3f c = cameraSample(r, s, o, totalLightArea, i, j, jitter);
                            taken++;
                            for (int ch = 0; ch < 3; ch++) mean[ch] += (c[ch] - mean[ch]) / taken;
                        }
                        if (o->spectral) mean = CIE::xyzToLinearSRGB(mean);
                        for (int ch = 0; ch < 3; ch++) acc[ch] = mean[ch];
                    }
                    else
                    {
                        for (int k = 0; k < n; k++)
                        {
                            Vec3f c = cameraSample(r, s, o, totalLightArea, i, j, false);
                            for (int ch = 0; ch < 3; ch++) acc[ch] += c[ch];
                        }
                        for (int ch = 0; ch < 3; ch++) acc[ch] /= n;
                        if (o->spectral)
                        {
                            double X = acc[0], Y = acc[1], Z = acc[2];
                            acc[0] = 3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z;
                            acc[1] = -0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z;
                            acc[2] = 0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z;
                        }
                    }
                    double *px = out + ((size_t)(i - rowBegin) * o->width + j) * 3;
                    px[0] = acc[0]; px[1] = acc[1]; px[2] = acc[2];
                }
            }
        });
    }
    for (auto &th : pool) th.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// ref_render_hdr in paths mode (spp paths per pixel centre, samples = 1)
// over an explicit list of rows, e.g. a sample spread evenly over the image;
// the threads share the list.  out holds nrows x width x 3 (linear sRGB).
double ref_render_hdr_rows(void *h, const RefRenderOpts *o, int spp, int threads, const int *rows, int nrows,
                           double *out)
{
    auto &s = ((RefScene *)h)->data;
    NumGen::setSeed(o->seed);
    pcr_ref_numgen_reset();
    const int nThreads = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < nThreads; t++)
    {
        pool.emplace_back([&, t]() {
            Renderer r(o->width, o->height, o->depth, 1, o->shadow);
            r.useMIS = o->mis; r.useRussian = o->russian; r.useStratified = o->stratified;
            r.useSpectral = o->spectral; r.heroSamples = o->hero;
            float totalLightArea;
            preparePlanes(r, s, totalLightArea);
            for (int k = t; k < nrows; k += nThreads)
            {
                for (int j = 0; j < o->width; j++)
                {
                    double acc[3] = {0, 0, 0};
                    for (int q = 0; q < spp; q++)
                    {
                        Vec3f c = cameraSample(r, s, o, totalLightArea, rows[k], j, false);
                        for (int ch = 0; ch < 3; ch++) acc[ch] += c[ch];
                    }
                    for (int ch = 0; ch < 3; ch++) acc[ch] /= spp;
                    if (o->spectral)
                    {
                        const double X = acc[0], Y = acc[1], Z = acc[2];
                        acc[0] = 3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z;
                        acc[1] = -0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z;
                        acc[2] = 0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z;
                    }
                    double *px = out + ((size_t)k * o->width + j) * 3;
                    for (int ch = 0; ch < 3; ch++) px[ch] = acc[ch];
                }
            }
        });
    }
    for (auto &th : pool) th.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Renderer::sceneIntersect over n rays (origin3 dir3 each).  Writes matIdx
// (-1 on miss) and hit3 N3 per ray.
void ref_scene_intersect(void *h, const float *rays, int n, int *mat, float *hitN)
{
    auto &s = ((RefScene *)h)->data;
    Renderer r(1, 1, 1, 1, 1);
    float total;
    preparePlanes(r, s, total);
    for (int i = 0; i < n; i++)
    {
        Ray ray;
        ray.origin = Vec3f(rays[i * 6 + 0], rays[i * 6 + 1], rays[i * 6 + 2]);
        ray.dir = Vec3f(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5]);
        Vec3f hit, N;
        int m = -1;
        bool got = r.sceneIntersect(ray, s.spheres, s.triangles, s.triangleBvh, hit, N, m);
        mat[i] = got ? m : -1;
        for (int k = 0; k < 3; k++) { hitN[i * 6 + k] = got ? hit[k] : 0.f; hitN[i * 6 + 3 + k] = got ? N[k] : 0.f; }
    }
}

// ---------------------------------------------------------------- BVH

static std::vector<Triangle> trianglesFrom(const float *tris, int n)
{
    std::vector<Triangle> v;
    v.reserve((size_t)n);
    for (int i = 0; i < n; i++)
    {
        const float *t = tris + (size_t)i * 9;
        v.emplace_back(Vec3f(t[0], t[1], t[2]), Vec3f(t[3], t[4], t[5]), Vec3f(t[6], t[7], t[8]), i);
    }
    return v;
}

// Bvh::build over n flat triangles whose matIdx is their input index.
// Writes nodes (boxes6, ints3) and the permutation (input index per leaf slot).
int ref_bvh_build(const float *tris, int n, float *boxes, int *ints, int *perm)
{
    auto v = trianglesFrom(tris, n);
    auto nodes = Bvh::build(v);
    for (size_t i = 0; i < nodes.size(); i++)
    {
        for (int k = 0; k < 3; k++) { boxes[i * 6 + k] = nodes[i].boxMin[k]; boxes[i * 6 + 3 + k] = nodes[i].boxMax[k]; }
        ints[i * 3 + 0] = nodes[i].leftOrFirst; ints[i * 3 + 1] = nodes[i].rightChild; ints[i * 3 + 2] = nodes[i].count;
    }
    for (int i = 0; i < n; i++) perm[i] = v[(size_t)i].matIdx;
    return (int)nodes.size();
}

// Bvh::build then Bvh::intersect for each ray (origin3 dir3) with
// closest_t = FLT_MAX.  Writes the input index of the hit triangle (-1 on
// miss) and t.  Returns the build+query wall time of the query loop only.
double ref_bvh_intersect(const float *tris, int n, const float *rays, long nrays,
                         int *hitId, float *hitT, int threads)
{
    auto v = trianglesFrom(tris, n);
    auto nodes = Bvh::build(v);
    int nThreads = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < nThreads; t++)
    {
        pool.emplace_back([&, t]() {
            for (long i = t; i < nrays; i += nThreads)
            {
                Ray ray;
                ray.origin = Vec3f(rays[i * 6 + 0], rays[i * 6 + 1], rays[i * 6 + 2]);
                ray.dir = Vec3f(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5]);
                Vec3f hit, N;
                int m = -1;
                float tt = 0.f;
                bool got = Bvh::intersect(nodes, v, ray, hit, N, m, tt, std::numeric_limits<float>::max());
                hitId[i] = got ? m : -1;
                hitT[i] = got ? tt : 0.f;
            }
        });
    }
    for (auto &th : pool) th.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// ---------------------------------------------------------------- stage functions

float ref_ybar_integral(void) { return CIE::yBarIntegral(); }

void ref_eval_sigmoid_fit(const float *fit, const float *lam, int n, float *out)
{
    RGBToSpectrum::SigmoidFit f{fit[0], fit[1], fit[2], fit[3]};
    for (int i = 0; i < n; i++) out[i] = RGBToSpectrum::evalSigmoidFit(f, lam[i]);
}

void ref_eval_spectrum(const float *tab61, const float *lam, int n, float *out)
{
    std::array<float, 61> a;
    std::memcpy(a.data(), tab61, sizeof(float) * 61);
    Spectrum s(a);
    for (int i = 0; i < n; i++) out[i] = s(lam[i]);
}

void ref_eval_cmf(const float *lam, int n, float *out)
{
    for (int i = 0; i < n; i++)
    {
        out[i * 3 + 0] = CIE::xBar(lam[i]);
        out[i * 3 + 1] = CIE::yBar(lam[i]);
        out[i * 3 + 2] = CIE::zBar(lam[i]);
    }
}

void ref_single_lambda_xyz(const float *lam, const float *rad, int n, float *out)
{
    for (int i = 0; i < n; i++)
    {
        Vec3f v = CIE::singleLambdaXYZ(lam[i], rad[i]);
        out[i * 3 + 0] = v[0]; out[i * 3 + 1] = v[1]; out[i * 3 + 2] = v[2];
    }
}

void ref_xyz_to_srgb(const float *in, int n, float *out)
{
    for (int i = 0; i < n; i++)
    {
        Vec3f v = CIE::xyzToLinearSRGB(Vec3f(in[i * 3], in[i * 3 + 1], in[i * 3 + 2]));
        out[i * 3 + 0] = v[0]; out[i * 3 + 1] = v[1]; out[i * 3 + 2] = v[2];
    }
}

void ref_srgb_to_xyz(const float *in, int n, float *out)
{
    for (int i = 0; i < n; i++)
    {
        Vec3f v = CIE::linearSRGBToXYZ(Vec3f(in[i * 3], in[i * 3 + 1], in[i * 3 + 2]));
        out[i * 3 + 0] = v[0]; out[i * 3 + 1] = v[1]; out[i * 3 + 2] = v[2];
    }
}

void ref_spectrum_to_xyz(const float *tab61, float *out3)
{
    std::array<float, 61> a;
    std::memcpy(a.data(), tab61, sizeof(float) * 61);
    Vec3f v = CIE::spectrumToXYZ(Spectrum(a));
    out3[0] = v[0]; out3[1] = v[1]; out3[2] = v[2];
}

// mode 0 Reinhard, 1 ACES (code/Includes/ToneMap.h:14-39)
void ref_tonemap(const float *in, int n, int mode, float *out)
{
    for (int i = 0; i < n; i++)
    {
        Vec3f c(in[i * 3], in[i * 3 + 1], in[i * 3 + 2]);
        if (mode) ToneMap::aces(c); else ToneMap::reinhard(c);
        out[i * 3 + 0] = c[0]; out[i * 3 + 1] = c[1]; out[i * 3 + 2] = c[2];
    }
}

// fitSigmoidCoefficients for n RGB triples -> 4 floats each (honours the active LUT)
void ref_fit_sigmoid(const float *rgb, int n, float *out)
{
    for (int i = 0; i < n; i++)
    {
        auto f = RGBToSpectrum::fitSigmoidCoefficients(Vec3f(rgb[i * 3], rgb[i * 3 + 1], rgb[i * 3 + 2]));
        out[i * 4 + 0] = f.c0; out[i * 4 + 1] = f.c1; out[i * 4 + 2] = f.c2; out[i * 4 + 3] = f.scale;
    }
}

float ref_schlick(float cosTheta, float n1, float n2) { return Optics::schlickFresnel(cosTheta, n1, n2); }
float ref_cauchy(float ior, float b, float lam) { return Optics::cauchyIor(ior, b, lam); }

// Optics::dielectricBounce: in = dir3 N3 hit3, out = dir3 origin3
void ref_dielectric(const float *in, int entering, float ior, float u, float *out)
{
    auto b = Optics::dielectricBounce(Vec3f(in[0], in[1], in[2]), Vec3f(in[3], in[4], in[5]),
                                      Vec3f(in[6], in[7], in[8]), entering != 0, ior, u);
    for (int k = 0; k < 3; k++) { out[k] = b.dir[k]; out[3 + k] = b.origin[k]; }
}

} // extern "C"
