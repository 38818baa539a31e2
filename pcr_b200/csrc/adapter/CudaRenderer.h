// The reference-tree side of the CUDA backend: copied into the reference
// project as code/Gpu/Cuda/CudaRenderer.h, it is the class the
// `using GpuRenderer = CudaRenderer;` branch of code/Gpu/GpuRenderer.h names.
//
// It has the surface code/Cli/Main.cpp:445-473 and the GUI use on a
// GpuRenderer (code/Gpu/Opengl/OpenglRenderer.h:29-117): the
// (width, height, depth, samples, shadowSamples, GLFWwindow*) constructor,
// progressRows, cancelRequested, onPartialFrame taking the reference's
// Vec3f framebuffer, the quality knobs, render(const Scenes::SceneData&,
// start, outputDir) and lastOutputPath.  render() converts the loaded scene
// (triangles already in BVH-leaf order, triangleBvh built,
// code/Scenes/SceneLoader.cpp:504-513) into the flat pcr_scene_desc of the C
// ABI and hands it to pcr::CudaRenderer, which uploads it once and renders.
//
// Include paths: the reference's code/ directory (as its own targets use),
// this repository's include/ and pcr_b200/csrc/.  Link: libpcr_b200.so and
// pcr_b200/csrc/cuda_renderer.cpp.
#pragma once

#include <algorithm>
#include <array>
#include <chrono>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "Scenes/Scene.h"
#include "cuda_renderer.h"
#include "pcr_cuda.h"

class CudaRenderer : public pcr::CudaRenderer {
public:
    using pcr::CudaRenderer::CudaRenderer;

    // The reference's callback type (code/Includes/Renderer.h:41-43); it
    // replaces the base's std::array form for callers in the reference tree.
    std::function<void(const std::vector<Vec3f> &, int width, int height)> onPartialFrame;

    void render(const Scenes::SceneData &s, std::chrono::steady_clock::time_point start,
                const std::string &outputDir)
    {
        pcr::CudaRenderer::onPartialFrame = [this](const std::vector<std::array<float, 3>> &fb, int w, int h) {
            if (!onPartialFrame) return;
            std::vector<Vec3f> v(fb.size());
            for (size_t i = 0; i < fb.size(); i++) v[i] = Vec3f(fb[i][0], fb[i][1], fb[i][2]);
            onPartialFrame(v, w, h);
        };
        // The flat copy is kept while the same SceneData is rendered again,
        // so pcr::CudaRenderer (which keys its device scene on the
        // materials array) uploads a scene once.  A new scene builds new
        // arrays while the old ones are still alive, so the key changes.
        const void *key[4] = {&s, s.materials.data(), s.triangles.data(), s.walls.data()};
        if (!std::equal(key, key + 4, key_) || !flat_) {
            auto f = std::make_unique<Flat>();
            convert(s, *f);
            flat_ = std::move(f);
            std::copy(key, key + 4, key_);
        }
        pcr::CudaRenderer::render(flat_->desc, start, outputDir);
    }

private:
    struct Flat {
        std::vector<pcr_material> mats;
        std::vector<pcr_plane> planes;
        std::vector<pcr_sphere> sph;
        std::vector<pcr_triangle> tris, ltris;
        std::vector<pcr_bvh_node> nodes;
        std::vector<pcr_light> lights;
        std::vector<float> cum;
        pcr_scene_desc desc{};
    };
    std::unique_ptr<Flat> flat_;
    const void *key_[4] = {nullptr, nullptr, nullptr, nullptr};

    static void convert(const Scenes::SceneData &s, Flat &F)
    {
        auto &mats = F.mats;
        for (const Material &m : s.materials) {
            pcr_material o{};
            for (int k = 0; k < 3; k++) { o.albedo[k] = m.albedo[k]; o.emissive[k] = m.emissive[k]; }
            o.metallic = m.metallic;
            o.transparent = m.transparent;
            o.ior = m.ior;
            o.cauchy_b = m.cauchyB;
            o.use_tab_albedo = m.useTabulatedAlbedo;
            o.use_tab_emissive = m.useTabulatedEmissive;
            o.albedo_fit[0] = m.albedoFit.c0;
            o.albedo_fit[1] = m.albedoFit.c1;
            o.albedo_fit[2] = m.albedoFit.c2;
            o.albedo_fit[3] = m.albedoFit.scale;
            o.emissive_fit[0] = m.emissiveFit.c0;
            o.emissive_fit[1] = m.emissiveFit.c1;
            o.emissive_fit[2] = m.emissiveFit.c2;
            o.emissive_fit[3] = m.emissiveFit.scale;
            for (int i = 0; i < PCR_SPECTRUM_SAMPLES; i++) {
                o.tab_albedo[i] = m.tabulatedAlbedo[i];
                o.tab_emissive[i] = m.tabulatedEmissive[i];
            }
            mats.push_back(o);
        }
        auto plane = [](const Plane &p) {
            pcr_plane o{};
            for (int k = 0; k < 3; k++) {
                o.origin[k] = p.origin[k];
                o.u[k] = p.getU()[k];
                o.v[k] = p.getV()[k];
                o.n[k] = p.N[k];
            }
            o.area = p.getArea();
            o.mat = p.matIdx;
            return o;
        };
        auto tri = [](const Triangle &t) {
            pcr_triangle o{};
            for (int k = 0; k < 3; k++) {
                o.v0[k] = t.v0[k]; o.v1[k] = t.v1[k]; o.v2[k] = t.v2[k];
                o.n0[k] = t.n0[k]; o.n1[k] = t.n1[k]; o.n2[k] = t.n2[k];
                o.flat_n[k] = t.flatN[k];
            }
            o.smooth = t.smooth;
            o.mat = t.matIdx;
            return o;
        };
        // the renderer's plane order: light planes first, then walls
        // (code/Renderer.cpp:123-130)
        auto &planes = F.planes;
        for (const auto &L : s.areaLights)
            if (L.kind == Scenes::AreaLightKind::Plane) planes.push_back(plane(L.plane));
        for (const auto &w : s.walls) planes.push_back(plane(w));
        auto &sph = F.sph;
        for (const auto &x : s.spheres) sph.push_back({{x.center[0], x.center[1], x.center[2]}, x.radius(), x.matIdx});
        auto &tris = F.tris, &ltris = F.ltris;
        for (const auto &t : s.triangles) tris.push_back(tri(t));
        auto &nodes = F.nodes;
        for (const auto &n : s.triangleBvh)
            nodes.push_back({{n.boxMin[0], n.boxMin[1], n.boxMin[2]}, {n.boxMax[0], n.boxMax[1], n.boxMax[2]},
                             n.leftOrFirst, n.rightChild, n.count});
        auto &lights = F.lights;
        auto &cum = F.cum;
        for (const auto &L : s.areaLights) {
            pcr_light o{};
            o.kind = L.kind == Scenes::AreaLightKind::Plane ? 0 : 1;
            o.total_area = L.totalArea;
            if (o.kind == 0) {
                o.plane = plane(L.plane);
            } else {
                o.tri_offset = (int32_t)ltris.size();
                o.tri_count = (int32_t)L.triangles.size();
                for (size_t i = 0; i < L.triangles.size(); i++) {
                    ltris.push_back(tri(L.triangles[i]));
                    cum.push_back(L.cumulativeArea[i]);
                }
            }
            lights.push_back(o);
        }
        pcr_scene_desc &d = F.desc;
        d.name = s.name.c_str();
        d.version = s.version.c_str();
        for (int k = 0; k < 3; k++) d.cam_pos[k] = s.camera.position[k];
        d.fov = s.camera.fov;
        d.n_materials = (int32_t)mats.size();
        d.materials = mats.data();
        d.n_spheres = (int32_t)sph.size();
        d.spheres = sph.data();
        d.n_planes = (int32_t)planes.size();
        d.planes = planes.data();
        d.n_triangles = (int32_t)tris.size();
        d.triangles = tris.data();
        d.n_bvh_nodes = (int32_t)nodes.size();
        d.bvh_nodes = nodes.data();
        d.n_lights = (int32_t)lights.size();
        d.lights = lights.data();
        d.light_triangles = ltris.data();
        d.light_cum_area = cum.data();
    }
};
