// Device build of the reference's binary SAH BVH (code/Bvh/Bvh.cpp:122-325):
// same nodes, bit for bit, and the same triangle order as `build_bvh`.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/pcr_cuda.h"

namespace pcr {

// verts9: n triangles as v0 v1 v2 (9 floats each).  Returns the nodes in
// depth-first preorder and order[i] = input index of the triangle at leaf
// position i.  Synchronous on `st`; the workspace (about 360 bytes per
// triangle) comes from `pool` (null: the device's default pool).
void device_build_bvh_raw(int device, cudaStream_t st, cudaMemPool_t pool, const float* verts9, int n,
                          std::vector<pcr_bvh_node>& nodes, std::vector<int32_t>& order);

// As build_bvh: permutes tris (and ids) into leaf order and returns the nodes.
std::vector<pcr_bvh_node> device_build_bvh(int device, cudaStream_t st, cudaMemPool_t pool,
                                           std::vector<pcr_triangle>& tris, std::vector<int32_t>* ids);

}  // namespace pcr
