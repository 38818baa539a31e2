// Host-side scene admission: the scene-JSON loader, SPD and OBJ readers,
// the RGB -> spectrum sigmoid fit (runtime homotopy or PLUT LUT), the
// reference-equal binary SAH BVH builder and its collapse into the 4-wide
// device BVH.  Everything here runs once per scene, before upload.
#pragma once

#include <cstdint>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/pcr_cuda.h"
#include "layout.h"

namespace pcr {

inline float __int_as_float_host(int x)
{
    float f;
    std::memcpy(&f, &x, 4);
    return f;
}

struct HostScene {
    std::string name, version;
    float cam[3] = {0, 0, 0};
    float fov = 65.f;
    std::vector<pcr_material> materials;
    std::vector<pcr_sphere> spheres;
    std::vector<pcr_plane> planes;          // light planes first, then walls
    std::vector<pcr_triangle> triangles;    // BVH-leaf order after finish()
    std::vector<int32_t> triangle_ids;
    std::vector<pcr_bvh_node> bvh;
    std::vector<pcr_light> lights;
    std::vector<pcr_triangle> light_tris;
    std::vector<float> light_cum;

    pcr_scene_desc desc() const;
};

// Scene JSON schema 1.x with // and /* */ comments (code/Scenes/SceneLoader.cpp:475-516).
// data_root holds spd/<name>.spd; lut (3*16^3*3 floats) selects the LUT fit.
// with_bvh = false leaves the triangles in file order and the BVH empty (for
// a build on the device).
HostScene load_scene_json(const std::string& path, const std::string& data_root, const std::vector<float>* lut,
                          bool with_bvh = true);

// Bvh::build (code/Bvh/Bvh.cpp:95-391): 16-bin SAH on centroids, leaf <= 4,
// depth-first layout; permutes tris (and ids) into leaf order.
std::vector<pcr_bvh_node> build_bvh(std::vector<pcr_triangle>& tris, std::vector<int32_t>* ids);

// Greedy collapse of the binary tree into 4-wide nodes whose child boxes are
// the binary nodes' boxes verbatim.
std::vector<DNode4> collapse_bvh4(const std::vector<pcr_bvh_node>& bvh, int n_tris);

// fn(lo, hi) over [0, n) in contiguous ranges on up to 16 host threads
// (inline below 64K items).
void parallel_for(int n, const std::function<void(int, int)>& fn);

// RGBToSpectrum::fitSigmoidCoefficients (code/RGBToSpectrum.cpp:256-293).
void fit_sigmoid(const float rgb[3], const std::vector<float>* lut, float out[4]);
// Material::populateSpectra (code/Includes/Material.h:125-139).
void populate_material(pcr_material& m, const std::vector<float>* lut);
// PLUT file (code/RGBToSpectrum.cpp:403-451) and in-process build (:332-385).
bool load_plut(const std::string& path, std::vector<float>& out, std::string* err);
bool save_plut(const std::string& path, const std::vector<float>& lut);
void build_lut(std::vector<float>& out);

pcr_plane make_plane(const float o[3], const float u[3], const float v[3], int mat);
pcr_triangle make_triangle(const float a[3], const float b[3], const float c[3], const float* n0, const float* n1,
                           const float* n2, int mat);

}  // namespace pcr
