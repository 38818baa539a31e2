/* Test infrastructure only: the CPU restatement of the reference renderer's
 * hot path, used as the checker for the CUDA path.  Product code never
 * links this.  Every function cites the reference file:line it restates
 * (paths relative to the reference project root). */
#ifndef PCR_ORACLE_H
#define PCR_ORACLE_H

#include <stdint.h>

#define O_SPEC_N 61

typedef struct {
    float albedo[3], emissive[3];
    int metallic, transparent, useTabA, useTabE;
    float ior, cauchyB;
    float afit[4], efit[4]; /* c0 c1 c2 scale */
    float tabA[O_SPEC_N], tabE[O_SPEC_N];
} OMaterial;

typedef struct { float origin[3], u[3], v[3], N[3], area; int matIdx; } OPlane;
typedef struct { float center[3], radius; int matIdx; } OSphere;
typedef struct {
    float v0[3], v1[3], v2[3], n0[3], n1[3], n2[3], flatN[3];
    int smooth, matIdx;
} OTriangle;
typedef struct { float bmin[3], bmax[3]; int leftOrFirst, rightChild, count; } ONode;
typedef struct { int kind; float totalArea; OPlane plane; int triOffset, triCount; } OLight;

typedef struct {
    float camPos[3], fov;
    int nMat; const OMaterial *mats;
    int nSph; const OSphere *sph;
    int nPlanes; const OPlane *planes;      /* light planes first, then walls */
    int nTri; const OTriangle *tris;        /* BVH-leaf order */
    int nNodes; const ONode *nodes;
    int nLights; const OLight *lights;
    const OTriangle *lightTris; const float *lightCum;
} OScene;

typedef struct {
    int width, height, depth, samples, shadow;
    int spectral, mis, russian, stratified, aces, denoise;
    int aa, adaptive, hero;
    uint64_t seed;
} OOpts;

#endif
