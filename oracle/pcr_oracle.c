/* Test infrastructure only: CPU restatement of the reference renderer's hot
 * path (the checker for the CUDA path; never linked by the product).
 *
 * The arithmetic follows the reference's operation order exactly (built
 * with -ffp-contract=off, single-precision libm), so a seeded single-thread
 * render reproduces the reference's golden PNGs bit for bit.  Citations are
 * file:line in the reference project.
 *
 * Pinned by: the 17 golden PNGs (tests/render/golden), and by the compiled
 * reference itself (oracle/_ref) on scene load, BVH build/query,
 * sceneIntersect and the spectral stage functions.
 */
#include "pcr_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* (float)std::numbers::pi as used throughout Renderer.cpp and Ray.h */
#define PI_F ((float)3.14159265358979323846)
#define LMIN 400.f
#define LMAX 700.f
#define LSTEP 5.0f /* Spectrum::kStep, Spectrum.h:170 */

/* ------------------------------------------------------------ vectors
 * Vec3f (Includes/Vec3f.h:16-109): componentwise float ops, left-to-right. */
typedef struct { float x, y, z; } V3;
static inline V3 v3(float a, float b, float c) { V3 r = {a, b, c}; return r; }
static inline V3 vld(const float *p) { return v3(p[0], p[1], p[2]); }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vmul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 vmulv(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 vdiv(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 vcross(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float vlen(V3 a) { return sqrtf(vdot(a, a)); }
static inline V3 vnorm(V3 a) { float m = sqrtf(vdot(a, a)); return v3(a.x / m, a.y / m, a.z / m); }
static inline float vget(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
/* std::max / std::min argument order semantics (NaN in b is ignored) */
static inline float smax(float a, float b) { return (a < b) ? b : a; }
static inline float smin(float a, float b) { return (b < a) ? b : a; }
static inline float sclamp(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

/* ------------------------------------------------------------ RNG
 * NumGen (NumGen.cpp:24-35 pcgStep, :54-80 Epsilon with per-thread seed). */
typedef struct { uint64_t s; } ORng;
static inline uint32_t pcg_step(uint64_t *state)
{
    uint64_t old = *state;
    *state = old * 6364136223846793005ULL + 1442695040888963407ULL;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}
static inline float eps(ORng *r) { return (float)pcg_step(&r->s) * (1.0f / 4294967296.0f); }
static ORng rng_for_thread(uint64_t seed, uint64_t threadIdx)
{
    ORng r;
    uint64_t s = seed ^ (threadIdx * 6364136223846793005ULL + 1442695040888963407ULL);
    r.s = s == 0 ? 1ULL : s;
    return r;
}

/* ------------------------------------------------------------ spectra */
/* Spectrum::operator() (Spectrum.h:82-90) */
static float spec_eval(const float *s, float lambda)
{
    if (lambda < LMIN || lambda > LMAX) return 0.f;
    float t = (lambda - LMIN) / LSTEP;
    int i = (int)t;
    if (i >= O_SPEC_N - 1) return s[O_SPEC_N - 1];
    float f = t - i;
    return s[i] * (1.f - f) + s[i + 1] * f;
}
/* RGBToSpectrum::sigmoid / evalSigmoidFit (RGBToSpectrum.h:38-41, 118-125) */
static inline float sigmoidf_(float x) { return 0.5f + x / (2.f * sqrtf(1.f + x * x)); }
static inline float sigmoid_deriv(float x) { float t = 1.f + x * x; return 0.5f / (t * sqrtf(t)); }
static float eval_fit(const float *fit, float lambda)
{
    float L = (lambda - 550.f) / 150.f;
    float p = fit[0] + L * (fit[1] + L * fit[2]);
    return sigmoidf_(p) * fit[3];
}
/* Material::albedoAt / emissiveAt (Material.h:92-101) */
static float albedo_at(const OMaterial *m, float lambda)
{
    if (m->useTabA) return spec_eval(m->tabA, lambda);
    return smin(eval_fit(m->afit, lambda), 1.f);
}
static float emissive_at(const OMaterial *m, float lambda)
{
    if (m->useTabE) return spec_eval(m->tabE, lambda);
    return eval_fit(m->efit, lambda);
}
static int is_emissive(const OMaterial *m)
{
    return m->emissive[0] > 0 || m->emissive[1] > 0 || m->emissive[2] > 0;
}

/* CIE (Includes/CIE.h:27-53, 79-88, 115-123, 140-159) */
static inline float wyman(float l, float mu, float s1, float s2)
{
    float t = (l < mu) ? (l - mu) * s1 : (l - mu) * s2;
    return expf(-0.5f * t * t);
}
static float xbar(float l)
{
    return 0.362f * wyman(l, 442.0f, 0.0624f, 0.0374f) + 1.056f * wyman(l, 599.8f, 0.0264f, 0.0323f)
         - 0.065f * wyman(l, 501.1f, 0.0490f, 0.0382f);
}
static float ybar(float l)
{
    return 0.821f * wyman(l, 568.8f, 0.0213f, 0.0247f) + 0.286f * wyman(l, 530.9f, 0.0613f, 0.0322f);
}
static float zbar(float l)
{
    return 1.217f * wyman(l, 437.0f, 0.0845f, 0.0278f) + 0.681f * wyman(l, 459.0f, 0.0385f, 0.0725f);
}
static inline float lambda_at(int i) { return LMIN + i * LSTEP; }
static float ybar_integral(void)
{
    static float val = -1.f;
    if (val < 0.f)
    {
        float sum = 0.f;
        for (int i = 0; i < O_SPEC_N; i++) sum += ybar(lambda_at(i));
        val = sum * LSTEP;
    }
    return val;
}
static V3 single_lambda_xyz(float lambda, float rad)
{
    float scale = (LMAX - LMIN) / ybar_integral();
    return v3(rad * xbar(lambda) * scale, rad * ybar(lambda) * scale, rad * zbar(lambda) * scale);
}
static V3 xyz_to_srgb(V3 c)
{
    return v3(3.2404542f * c.x - 1.5371385f * c.y - 0.4985314f * c.z,
              -0.9692660f * c.x + 1.8760108f * c.y + 0.0415560f * c.z,
              0.0556434f * c.x - 0.2040259f * c.y + 1.0572252f * c.z);
}
static V3 srgb_to_xyz(V3 c)
{
    return v3(0.4124564f * c.x + 0.3575761f * c.y + 0.1804375f * c.z,
              0.2126729f * c.x + 0.7151522f * c.y + 0.0721750f * c.z,
              0.0193339f * c.x + 0.1191920f * c.y + 0.9503041f * c.z);
}
/* CIE::spectrumToXYZ (CIE.cpp:10-26) */
static V3 spectrum_to_xyz(const float *s)
{
    float X = 0.f, Y = 0.f, Z = 0.f;
    for (int i = 0; i < O_SPEC_N; i++)
    {
        float l = lambda_at(i), v = s[i];
        X += v * xbar(l);
        Y += v * ybar(l);
        Z += v * zbar(l);
    }
    float scale = LSTEP / ybar_integral();
    return v3(X * scale, Y * scale, Z * scale);
}

/* ------------------------------------------------------------ RGB -> spectrum fit
 * RGBToSpectrum.cpp:27-53 solve3x3, :59-166 newtonFit, :175-190 spikiness,
 * :192-254 fitCoefficients, :256-293 fitSigmoidCoefficients,
 * :453-521 lookupSigmoidFit, :332-385 buildLUT. */
static int solve3x3(float J[3][3], const float b[3], float x[3])
{
    float det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1])
              - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0])
              + J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    if (fabsf(det) < 1e-12f) return 0;
    float invDet = 1.f / det;
    float d0 = b[0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1])
             - J[0][1] * (b[1] * J[2][2] - J[1][2] * b[2])
             + J[0][2] * (b[1] * J[2][1] - J[1][1] * b[2]);
    float d1 = J[0][0] * (b[1] * J[2][2] - J[1][2] * b[2])
             - b[0] * (J[1][0] * J[2][2] - J[1][2] * J[2][0])
             + J[0][2] * (J[1][0] * b[2] - b[1] * J[2][0]);
    float d2 = J[0][0] * (J[1][1] * b[2] - b[1] * J[2][1])
             - J[0][1] * (J[1][0] * b[2] - b[1] * J[2][0])
             + b[0] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    x[0] = d0 * invDet; x[1] = d1 * invDet; x[2] = d2 * invDet;
    return 1;
}

static void integrate_fit(const float c[3], float xyz[3], float J[3][3])
{
    xyz[0] = xyz[1] = xyz[2] = 0.f;
    if (J) memset(J, 0, sizeof(float) * 9);
    for (int i = 0; i < O_SPEC_N; i++)
    {
        float lambda = lambda_at(i);
        float ln = (lambda - 550.f) / 150.f;
        float p = c[0] + ln * (c[1] + ln * c[2]);
        float s = sigmoidf_(p);
        float xb = xbar(lambda), yb = ybar(lambda), zb = zbar(lambda);
        xyz[0] += s * xb; xyz[1] += s * yb; xyz[2] += s * zb;
        if (J)
        {
            float ds = sigmoid_deriv(p);
            float ln2 = ln * ln;
            J[0][0] += ds * xb; J[0][1] += ds * ln * xb; J[0][2] += ds * ln2 * xb;
            J[1][0] += ds * yb; J[1][1] += ds * ln * yb; J[1][2] += ds * ln2 * yb;
            J[2][0] += ds * zb; J[2][1] += ds * ln * zb; J[2][2] += ds * ln2 * zb;
        }
    }
}

static void newton_fit(const float target[3], const float cIn[3], float cOut[3])
{
    float c[3] = {cIn[0], cIn[1], cIn[2]};
    for (int iter = 0; iter < 15; iter++)
    {
        float xyz[3], J[3][3];
        integrate_fit(c, xyz, J);
        float dl = LSTEP;
        for (int k = 0; k < 3; k++)
        {
            xyz[k] *= dl;
            for (int j = 0; j < 3; j++) J[k][j] *= dl;
        }
        float r[3] = {xyz[0] - target[0], xyz[1] - target[1], xyz[2] - target[2]};
        float rNorm = sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        if (rNorm < 1e-6f) break;
        float delta[3];
        if (!solve3x3(J, r, delta)) break;
        float prev[3] = {c[0], c[1], c[2]};
        float step = 1.f;
        int reduced = 0;
        for (int trial = 0; trial < 4; trial++)
        {
            c[0] = prev[0] - step * delta[0];
            c[1] = prev[1] - step * delta[1];
            c[2] = prev[2] - step * delta[2];
            float t[3];
            integrate_fit(c, t, NULL);
            t[0] *= dl; t[1] *= dl; t[2] *= dl;
            float tr[3] = {t[0] - target[0], t[1] - target[1], t[2] - target[2]};
            float tn = sqrtf(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]);
            if (tn < rNorm) { reduced = 1; break; }
            step *= 0.5f;
        }
        if (!reduced)
        {
            c[0] = prev[0]; c[1] = prev[1]; c[2] = prev[2];
            break;
        }
    }
    cOut[0] = c[0]; cOut[1] = c[1]; cOut[2] = c[2];
}

static int cmp_float(const void *a, const void *b)
{
    float x = *(const float *)a, y = *(const float *)b;
    return (x < y) ? -1 : (y < x) ? 1 : 0;
}

static float spikiness(const float c[3])
{
    float s[O_SPEC_N], maxV = 0.f;
    for (int i = 0; i < O_SPEC_N; i++)
    {
        float ln = (lambda_at(i) - 550.f) / 150.f;
        float p = c[0] + ln * (c[1] + ln * c[2]);
        s[i] = 0.5f + p / (2.f * sqrtf(1.f + p * p));
        if (s[i] > maxV) maxV = s[i];
    }
    qsort(s, O_SPEC_N, sizeof(float), cmp_float); /* nth_element(61/2) == sorted[30] */
    float median = s[O_SPEC_N / 2];
    if (median < 1e-8f) return (maxV < 1e-8f) ? 1.f : 1e30f;
    return maxV / median;
}

static inline float sigmoid_inverse(float y)
{
    y = sclamp(y, 1e-4f, 1.f - 1e-4f);
    float u = 2.f * y - 1.f;
    return u / sqrtf(1.f - u * u);
}

static void fit_coefficients(V3 target, float out[3])
{
    const float kXn = 0.95046f, kZn = 1.08906f;
    float gray[3] = {target.y * kXn, target.y, target.y * kZn};
    float tgt[3] = {target.x, target.y, target.z};
    float c[3] = {sigmoid_inverse(target.y / ybar_integral()), 0.f, 0.f};
    float good[3] = {c[0], c[1], c[2]};
    for (int step = 1; step <= 32; step++)
    {
        float t = (float)step / (float)32;
        float cur[3] = {(1.f - t) * gray[0] + t * tgt[0], (1.f - t) * gray[1] + t * tgt[1],
                        (1.f - t) * gray[2] + t * tgt[2]};
        float nx[3];
        newton_fit(cur, c, nx);
        if (spikiness(nx) > 200.f) break;
        c[0] = nx[0]; c[1] = nx[1]; c[2] = nx[2];
        good[0] = c[0]; good[1] = c[1]; good[2] = c[2];
    }
    out[0] = good[0]; out[1] = good[1]; out[2] = good[2];
}

#define LUT_RES 16
static inline int lut_idx(int l, int b, int x, int y)
{
    return ((l * LUT_RES + b) * LUT_RES + x) * LUT_RES * 3 + y * 3;
}

void oracle_lut_lookup(const float *lut, const float *rgb, float *out)
{
    float r = sclamp(rgb[0], 0.f, 1.f), g = sclamp(rgb[1], 0.f, 1.f), b = sclamp(rgb[2], 0.f, 1.f);
    if (r <= 0.f && g <= 0.f && b <= 0.f) { out[0] = out[1] = out[2] = out[3] = 0.f; return; }
    if (r >= 1.f && g >= 1.f && b >= 1.f)
    {
        float scale = ybar_integral();
        out[0] = sigmoid_inverse(1.f / scale); out[1] = out[2] = 0.f; out[3] = scale;
        return;
    }
    int l = 0;
    float maxV = r;
    if (g >= maxV) { l = 1; maxV = g; }
    if (b >= maxV) { l = 2; maxV = b; }
    float o1, o2;
    if (l == 0) { o1 = g; o2 = b; } else if (l == 1) { o1 = r; o2 = b; } else { o1 = r; o2 = g; }
    float xn = o1 / maxV, yn = o2 / maxV, bn = maxV;
    float xf = xn * (float)(LUT_RES - 1), yf = yn * (float)(LUT_RES - 1), bf = bn * (float)(LUT_RES - 1);
    int xi = (int)xf, yi = (int)yf, bi = (int)bf;
    xi = xi < 0 ? 0 : (LUT_RES - 2 < xi ? LUT_RES - 2 : xi);
    yi = yi < 0 ? 0 : (LUT_RES - 2 < yi ? LUT_RES - 2 : yi);
    bi = bi < 0 ? 0 : (LUT_RES - 2 < bi ? LUT_RES - 2 : bi);
    float xt = sclamp(xf - xi, 0.f, 1.f), yt = sclamp(yf - yi, 0.f, 1.f), bt = sclamp(bf - bi, 0.f, 1.f);
    out[3] = ybar_integral();
    for (int k = 0; k < 3; k++)
    {
#define S_(db, dx, dy) lut[lut_idx(l, bi + (db), xi + (dx), yi + (dy)) + k]
        float v000 = S_(0, 0, 0), v100 = S_(0, 1, 0), v010 = S_(0, 0, 1), v110 = S_(0, 1, 1);
        float v001 = S_(1, 0, 0), v101 = S_(1, 1, 0), v011 = S_(1, 0, 1), v111 = S_(1, 1, 1);
#undef S_
        float v00 = v000 + xt * (v100 - v000), v10 = v010 + xt * (v110 - v010);
        float v01 = v001 + xt * (v101 - v001), v11 = v011 + xt * (v111 - v011);
        float v0 = v00 + yt * (v10 - v00), v1 = v01 + yt * (v11 - v01);
        out[k] = v0 + bt * (v1 - v0);
    }
}

/* fitSigmoidCoefficients; lut == NULL uses the runtime homotopy */
void oracle_fit_sigmoid(const float *rgb, const float *lut, float *out)
{
    if (lut) { oracle_lut_lookup(lut, rgb, out); return; }
    float r = sclamp(rgb[0], 0.f, 1.f), g = sclamp(rgb[1], 0.f, 1.f), b = sclamp(rgb[2], 0.f, 1.f);
    if (r <= 0.f && g <= 0.f && b <= 0.f) { out[0] = out[1] = out[2] = out[3] = 0.f; return; }
    if (r >= 1.f && g >= 1.f && b >= 1.f)
    {
        float scale = ybar_integral();
        out[0] = sigmoid_inverse(1.f / scale); out[1] = out[2] = 0.f; out[3] = scale;
        return;
    }
    float c[3];
    fit_coefficients(srgb_to_xyz(v3(r, g, b)), c);
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = ybar_integral();
}

void oracle_lut_build(float *lut)
{
    for (int l = 0; l < 3; l++)
        for (int xi = 0; xi < LUT_RES; xi++)
            for (int yi = 0; yi < LUT_RES; yi++)
            {
                float x = (float)xi / (float)(LUT_RES - 1), y = (float)yi / (float)(LUT_RES - 1);
                for (int bi = 0; bi < LUT_RES; bi++)
                {
                    int idx = lut_idx(l, bi, xi, yi);
                    float b = (float)bi / (float)(LUT_RES - 1);
                    if (b <= 0.f) { lut[idx] = lut[idx + 1] = lut[idx + 2] = 0.f; continue; }
                    float v0 = b, v1 = x * b, v2 = y * b;
                    V3 rgb = l == 0 ? v3(v0, v1, v2) : (l == 1 ? v3(v1, v0, v2) : v3(v1, v2, v0));
                    float c[3];
                    fit_coefficients(srgb_to_xyz(rgb), c);
                    for (int k = 0; k < 3; k++) lut[idx + k] = sclamp(c[k], -200.f, 200.f);
                }
            }
}

/* Material::populateSpectra (Material.h:125-139) */
void oracle_populate_material(OMaterial *m, const float *lut)
{
    oracle_fit_sigmoid(m->albedo, lut, m->afit);
    if (is_emissive(m))
    {
        float e0 = m->emissive[0], e1 = m->emissive[1], e2 = m->emissive[2];
        float maxE = e0;
        if (maxE < e1) maxE = e1;
        if (maxE < e2) maxE = e2;
        float n[3] = {e0 / maxE, e1 / maxE, e2 / maxE};
        oracle_fit_sigmoid(n, lut, m->efit);
        m->efit[3] *= maxE;
    }
    else
        m->efit[0] = m->efit[1] = m->efit[2] = m->efit[3] = 0.f;
}

/* SceneLoader.cpp:141-145: RGB equivalent of an SPD-only material */
void oracle_spectrum_rgb(const float *tab61, float *out)
{
    V3 c = xyz_to_srgb(spectrum_to_xyz(tab61));
    out[0] = smax(0.f, c.x); out[1] = smax(0.f, c.y); out[2] = smax(0.f, c.z);
}

/* ------------------------------------------------------------ primitives */
/* Plane ctor (Plane.h:11-16) */
void oracle_make_plane(const float *o, const float *u, const float *v, int mat, OPlane *p)
{
    V3 c = vcross(vld(u), vld(v));
    V3 n = vnorm(c);
    memcpy(p->origin, o, 12); memcpy(p->u, u, 12); memcpy(p->v, v, 12);
    p->N[0] = n.x; p->N[1] = n.y; p->N[2] = n.z;
    p->area = vlen(c);
    p->matIdx = mat;
}

/* Triangle ctors (Triangle.h:12-36); normals may be NULL for flat */
void oracle_make_triangle(const float *a, const float *b, const float *c, const float *n0,
                          const float *n1, const float *n2, int mat, OTriangle *t)
{
    memcpy(t->v0, a, 12); memcpy(t->v1, b, 12); memcpy(t->v2, c, 12);
    V3 f = vnorm(vcross(vsub(vld(b), vld(a)), vsub(vld(c), vld(a))));
    t->flatN[0] = f.x; t->flatN[1] = f.y; t->flatN[2] = f.z;
    t->smooth = n0 != NULL;
    if (n0) { memcpy(t->n0, n0, 12); memcpy(t->n1, n1, 12); memcpy(t->n2, n2, 12); }
    else { memset(t->n0, 0, 12); memset(t->n1, 0, 12); memset(t->n2, 0, 12); }
    t->matIdx = mat;
}

/* Scene.h:110-129 makeTriangleSetLight: cumulative areas */
float oracle_triangle_cum_area(const OTriangle *tris, int n, float *cum)
{
    float acc = 0.f;
    for (int i = 0; i < n; i++)
    {
        V3 e1 = vsub(vld(tris[i].v1), vld(tris[i].v0)), e2 = vsub(vld(tris[i].v2), vld(tris[i].v0));
        acc += 0.5f * vlen(vcross(e1, e2));
        cum[i] = acc;
    }
    return acc;
}

/* MeshLoader.cpp:89-136: scale, Euler XYZ (degrees), translate; normals rotate
 * then normalize.  pts: n*3 in/out.  isNormal selects the normal transform. */
void oracle_mesh_transform(float *pts, int n, const float *pos, const float *rotDeg,
                           const float *scale, int isNormal)
{
    const float kPi = 3.14159265358979323846f;
    float rx = rotDeg[0] * (kPi / 180.f), ry = rotDeg[1] * (kPi / 180.f), rz = rotDeg[2] * (kPi / 180.f);
    for (int i = 0; i < n; i++)
    {
        float *v = pts + i * 3;
        if (!isNormal) { v[0] *= scale[0]; v[1] *= scale[1]; v[2] *= scale[2]; }
        if (rx != 0.f)
        {
            float c = cosf(rx), s = sinf(rx);
            float y = v[1] * c - v[2] * s, z = v[1] * s + v[2] * c;
            v[1] = y; v[2] = z;
        }
        if (ry != 0.f)
        {
            float c = cosf(ry), s = sinf(ry);
            float x = v[0] * c + v[2] * s, z = -v[0] * s + v[2] * c;
            v[0] = x; v[2] = z;
        }
        if (rz != 0.f)
        {
            float c = cosf(rz), s = sinf(rz);
            float x = v[0] * c - v[1] * s, y = v[0] * s + v[1] * c;
            v[0] = x; v[1] = y;
        }
        if (!isNormal) { v[0] += pos[0]; v[1] += pos[1]; v[2] += pos[2]; }
        else
        {
            V3 nn = vnorm(vld(v));
            v[0] = nn.x; v[1] = nn.y; v[2] = nn.z;
        }
    }
}

/* Sphere::intersect (Sphere.h:20-40) */
static int sphere_hit(const OSphere *s, V3 o, V3 d, float *t0)
{
    V3 cp = vsub(vld(s->center), o);
    float rayLen = vdot(d, cp);
    float tSq = vdot(cp, cp) - rayLen * rayLen;
    float r2 = s->radius * s->radius;
    if (tSq > r2) return 0;
    float tDist = sqrtf(r2 - tSq);
    *t0 = rayLen - tDist;
    float t1 = rayLen + tDist;
    if (*t0 < 0) *t0 = t1;
    if (*t0 < 0) return 0;
    return 1;
}

/* Plane::intersect (Plane.h:33-54) */
static int plane_hit(const OPlane *p, V3 o, V3 d, V3 *hit, float *t0, float closest)
{
    const float EPS = 1e-6f;
    V3 N = vld(p->N);
    float denom = vdot(d, N);
    if (fabsf(denom) <= EPS) return 0;
    float t = vdot(vsub(vld(p->origin), o), N) / denom;
    *t0 = t;
    if (t <= EPS || t > closest) return 0;
    V3 th = vadd(o, vmul(d, t));
    V3 lh = vsub(th, vld(p->origin));
    V3 u = vld(p->u), v = vld(p->v);
    float s = vdot(lh, u) / vdot(u, u);
    float q = vdot(lh, v) / vdot(v, v);
    if (s > 1 || s < 0 || q > 1 || q < 0) return 0;
    *hit = th;
    return 1;
}

/* Triangle::intersect (Triangle.h:53-92) */
static int tri_hit(const OTriangle *tr, V3 o, V3 d, V3 *hit, V3 *N, float *t0, float closest)
{
    const float EPS = 1e-6f;
    V3 v0 = vld(tr->v0);
    V3 e1 = vsub(vld(tr->v1), v0), e2 = vsub(vld(tr->v2), v0);
    V3 pvec = vcross(d, e2);
    float det = vdot(e1, pvec);
    if (fabsf(det) < EPS) return 0;
    float invDet = 1.f / det;
    V3 tvec = vsub(o, v0);
    float u = vdot(tvec, pvec) * invDet;
    if (u < 0.f || u > 1.f) return 0;
    V3 qvec = vcross(tvec, e1);
    float v = vdot(d, qvec) * invDet;
    if (v < 0.f || u + v > 1.f) return 0;
    float t = vdot(e2, qvec) * invDet;
    if (t <= EPS || t >= closest) return 0;
    *t0 = t;
    *hit = vadd(o, vmul(d, t));
    if (tr->smooth)
    {
        float w = 1.f - u - v;
        V3 in = v3(tr->n0[0] * w + tr->n1[0] * u + tr->n2[0] * v, tr->n0[1] * w + tr->n1[1] * u + tr->n2[1] * v,
                   tr->n0[2] * w + tr->n1[2] * u + tr->n2[2] * v);
        *N = vnorm(in);
    }
    else
        *N = vld(tr->flatN);
    return 1;
}

/* ------------------------------------------------------------ BVH build
 * Bvh.cpp:95-139 AABB, :149-157 centroid, :188-268 findSahSplit,
 * :274-292 partitionForSah (std::partition, bidirectional form),
 * :297-356 buildRecursive, :380-391 build. */
typedef struct { float mn[3], mx[3]; } OBox;
static void box_empty(OBox *b)
{
    for (int i = 0; i < 3; i++) { b->mn[i] = FLT_MAX; b->mx[i] = -FLT_MAX; }
}
static void box_vertex(OBox *b, const float *p)
{
    for (int i = 0; i < 3; i++)
    {
        if (p[i] < b->mn[i]) b->mn[i] = p[i];
        if (p[i] > b->mx[i]) b->mx[i] = p[i];
    }
}
static void box_tri(OBox *b, const OTriangle *t) { box_vertex(b, t->v0); box_vertex(b, t->v1); box_vertex(b, t->v2); }
static void box_merge(OBox *b, const OBox *o)
{
    for (int i = 0; i < 3; i++)
    {
        if (o->mn[i] < b->mn[i]) b->mn[i] = o->mn[i];
        if (o->mx[i] > b->mx[i]) b->mx[i] = o->mx[i];
    }
}
static float box_area(const OBox *b)
{
    float dx = b->mx[0] - b->mn[0], dy = b->mx[1] - b->mn[1], dz = b->mx[2] - b->mn[2];
    if (dx < 0 || dy < 0 || dz < 0) return 0.f;
    return 2.f * (dx * dy + dy * dz + dz * dx);
}
static inline float centroid(const OTriangle *t, int a) { return (t->v0[a] + t->v1[a] + t->v2[a]) * (1.f / 3.f); }

typedef struct { OTriangle *tris; ONode *nodes; int count; } OBuild;

static void centroid_box(const OTriangle *tris, int begin, int end, OBox *cb)
{
    box_empty(cb);
    for (int i = begin; i < end; i++)
    {
        float c[3] = {centroid(&tris[i], 0), centroid(&tris[i], 1), centroid(&tris[i], 2)};
        box_vertex(cb, c);
    }
}

static int bin_of(float c, float lo, float scale)
{
    int idx = (int)((c - lo) * scale);
    return idx < 0 ? 0 : (15 < idx ? 15 : idx);
}

static int build_rec(OBuild *B, int begin, int end)
{
    int nodeIdx = B->count++;
    ONode *nd = &B->nodes[nodeIdx];
    OBox box;
    box_empty(&box);
    for (int i = begin; i < end; i++) box_tri(&box, &B->tris[i]);
    for (int i = 0; i < 3; i++) { nd->bmin[i] = box.mn[i]; nd->bmax[i] = box.mx[i]; }
    int count = end - begin;
    if (count <= 4) goto leaf;
    {
        OBox cb;
        centroid_box(B->tris, begin, end, &cb);
        int bestAxis = -1, bestBin = -1;
        float bestCost = FLT_MAX;
        float parentSA = box_area(&box);
        if (parentSA > 0.f)
        {
            for (int axis = 0; axis < 3; axis++)
            {
                float lo = cb.mn[axis], hi = cb.mx[axis], extent = hi - lo;
                if (extent < 1e-6f) continue;
                float scale = (float)16 / extent;
                OBox bins[16];
                int cnt[16];
                for (int k = 0; k < 16; k++) { box_empty(&bins[k]); cnt[k] = 0; }
                for (int i = begin; i < end; i++)
                {
                    int idx = bin_of(centroid(&B->tris[i], axis), lo, scale);
                    box_tri(&bins[idx], &B->tris[i]);
                    cnt[idx]++;
                }
                float lSA[15], rSA[15];
                int lC[15], rC[15];
                OBox acc;
                box_empty(&acc);
                int ac = 0;
                for (int i = 0; i < 15; i++)
                {
                    box_merge(&acc, &bins[i]); ac += cnt[i];
                    lSA[i] = box_area(&acc); lC[i] = ac;
                }
                box_empty(&acc);
                ac = 0;
                for (int i = 15; i > 0; i--)
                {
                    box_merge(&acc, &bins[i]); ac += cnt[i];
                    rSA[i - 1] = box_area(&acc); rC[i - 1] = ac;
                }
                for (int s = 0; s < 15; s++)
                {
                    if (lC[s] == 0 || rC[s] == 0) continue;
                    float cost = 1.f + 2.f * (lSA[s] * lC[s] + rSA[s] * rC[s]) / parentSA;
                    if (cost < bestCost) { bestCost = cost; bestAxis = axis; bestBin = s; }
                }
            }
        }
        float leafCost = (float)count * 2.f;
        if (bestAxis < 0 || bestCost >= leafCost) goto leaf;
        /* partitionForSah: recompute the centroid box, then libstdc++'s
         * bidirectional std::partition (two-pointer swap). */
        float lo = cb.mn[bestAxis], hi = cb.mx[bestAxis];
        float scale = (float)16 / (hi - lo);
        int first = begin, last = end;
        for (;;)
        {
            for (;;)
            {
                if (first == last) goto done;
                if (bin_of(centroid(&B->tris[first], bestAxis), lo, scale) <= bestBin) first++;
                else break;
            }
            last--;
            for (;;)
            {
                if (first == last) goto done;
                if (!(bin_of(centroid(&B->tris[last], bestAxis), lo, scale) <= bestBin)) last--;
                else break;
            }
            OTriangle tmp = B->tris[first];
            B->tris[first] = B->tris[last];
            B->tris[last] = tmp;
            first++;
        }
    done:;
        int mid = first;
        if (mid == begin || mid == end) goto leaf;
        int l = build_rec(B, begin, mid);
        int r = build_rec(B, mid, end);
        nd = &B->nodes[nodeIdx];
        nd->leftOrFirst = l; nd->rightChild = r; nd->count = 0;
        return nodeIdx;
    }
leaf:
    nd = &B->nodes[nodeIdx];
    nd->leftOrFirst = begin; nd->rightChild = 0; nd->count = count;
    return nodeIdx;
}

/* Builds over tris (permuted in place); nodes must hold 2n entries. */
int oracle_bvh_build(OTriangle *tris, int n, ONode *nodes)
{
    if (n <= 0) return 0;
    OBuild B = {tris, nodes, 0};
    build_rec(&B, 0, n);
    return B.count;
}

/* ------------------------------------------------------------ BVH query
 * Bvh.cpp:294-311 rayAabb, :353-444 intersect.  counts (optional):
 * [0] internal nodes processed, [1] leaf triangles tested. */
static int ray_aabb(V3 o, V3 d, const float *mn, const float *mx, float segMax, float *tNear)
{
    float tmin = 0.f, tmax = segMax;
    for (int i = 0; i < 3; i++)
    {
        float invD = 1.f / vget(d, i);
        float t1 = (mn[i] - vget(o, i)) * invD;
        float t2 = (mx[i] - vget(o, i)) * invD;
        if (t1 > t2) { float s = t1; t1 = t2; t2 = s; }
        tmin = smax(tmin, t1);
        tmax = smin(tmax, t2);
        if (tmin > tmax) return 0;
    }
    *tNear = tmin;
    return 1;
}

static int bvh_intersect(const ONode *nodes, int nNodes, const OTriangle *tris, V3 o, V3 d,
                         V3 *hit, V3 *N, int *matIdx, float *tOut, float closest_t, long *counts)
{
    if (nNodes <= 0) return 0;
    struct { int idx; float tNear; } st[64];
    int top = 0;
    float tRoot;
    if (!ray_aabb(o, d, nodes[0].bmin, nodes[0].bmax, closest_t, &tRoot)) return 0;
    st[top].idx = 0; st[top].tNear = tRoot; top++;
    int any = 0;
    float closest = closest_t;
    while (top > 0)
    {
        top--;
        int ei = st[top].idx;
        float et = st[top].tNear;
        if (et > closest) continue;
        const ONode *n = &nodes[ei];
        if (n->count > 0)
        {
            for (int i = 0; i < n->count; i++)
            {
                int ti = n->leftOrFirst + i;
                V3 th, tn;
                float tt;
                if (counts) counts[1]++;
                if (!tri_hit(&tris[ti], o, d, &th, &tn, &tt, closest)) continue;
                closest = tt; *hit = th; *N = tn; *matIdx = tris[ti].matIdx; any = 1;
            }
            continue;
        }
        if (counts) counts[0]++;
        const ONode *cl = &nodes[n->leftOrFirst], *cr = &nodes[n->rightChild];
        float tL, tR;
        int hL = ray_aabb(o, d, cl->bmin, cl->bmax, closest, &tL);
        int hR = ray_aabb(o, d, cr->bmin, cr->bmax, closest, &tR);
        if (hL && hR)
        {
            if (top + 2 > 64) continue;
            if (tL <= tR)
            {
                st[top].idx = n->rightChild; st[top].tNear = tR; top++;
                st[top].idx = n->leftOrFirst; st[top].tNear = tL; top++;
            }
            else
            {
                st[top].idx = n->leftOrFirst; st[top].tNear = tL; top++;
                st[top].idx = n->rightChild; st[top].tNear = tR; top++;
            }
        }
        else if (hL)
        {
            if (top + 1 > 64) continue;
            st[top].idx = n->leftOrFirst; st[top].tNear = tL; top++;
        }
        else if (hR)
        {
            if (top + 1 > 64) continue;
            st[top].idx = n->rightChild; st[top].tNear = tR; top++;
        }
    }
    if (any) *tOut = closest;
    return any;
}

/* Closest hit per ray (origin3 dir3) with closest_t = FLT_MAX; hitId is the
 * hit triangle's matIdx (-1 on miss).  counts (optional, 2 per ray). */
void oracle_bvh_query(const ONode *nodes, int nNodes, const OTriangle *tris, const float *rays,
                      long nrays, int *hitId, float *hitT, long *counts)
{
    for (long i = 0; i < nrays; i++)
    {
        V3 o = vld(rays + i * 6), d = vld(rays + i * 6 + 3), h, N;
        int m = -1;
        float t = 0.f;
        long c[2] = {0, 0};
        int got = bvh_intersect(nodes, nNodes, tris, o, d, &h, &N, &m, &t, FLT_MAX, counts ? c : NULL);
        hitId[i] = got ? m : -1;
        hitT[i] = got ? t : 0.f;
        if (counts) { counts[i * 2] = c[0]; counts[i * 2 + 1] = c[1]; }
    }
}

/* ------------------------------------------------------------ work counts
 * While counting is on (oracle_count_begin .. oracle_count_end), every
 * scene query adds to process-wide totals: [0] rays (sceneIntersect calls:
 * camera, continuation and shadow rays alike, as the reference casts them),
 * [1] plane tests, [2] sphere tests, [3] BVH internal nodes processed (each
 * reads its two children's boxes), [4] leaf triangles tested.  These are the
 * reference traversal's work, the algorithmic units of the path's rooflines. */
static int g_counting = 0;
static long g_counts[5];

void oracle_count_begin(void)
{
    for (int i = 0; i < 5; i++) __atomic_store_n(&g_counts[i], 0, __ATOMIC_RELAXED);
    __atomic_store_n(&g_counting, 1, __ATOMIC_RELEASE);
}

void oracle_count_end(long *out)
{
    __atomic_store_n(&g_counting, 0, __ATOMIC_RELEASE);
    for (int i = 0; i < 5; i++) out[i] = __atomic_load_n(&g_counts[i], __ATOMIC_RELAXED);
}

/* ------------------------------------------------------------ scene query
 * Renderer::sceneIntersect (Renderer.cpp:891-949) */
static int scene_intersect(const OScene *S, V3 o, V3 d, V3 *hit, V3 *N, int *matIdx)
{
    float closest = FLT_MAX, t0 = 0.f;
    long bc[2] = {0, 0};
    const int counting = __atomic_load_n(&g_counting, __ATOMIC_RELAXED);
    for (int i = 0; i < S->nSph; i++)
    {
        if (!sphere_hit(&S->sph[i], o, d, &t0) || t0 >= closest) continue;
        closest = t0;
        *hit = vadd(o, vmul(d, t0));
        *N = vnorm(vsub(*hit, vld(S->sph[i].center)));
        *matIdx = S->sph[i].matIdx;
    }
    for (int i = 0; i < S->nPlanes; i++)
    {
        if (!plane_hit(&S->planes[i], o, d, hit, &t0, closest) || t0 >= closest) continue;
        closest = t0;
        *N = vld(S->planes[i].N);
        *matIdx = S->planes[i].matIdx;
    }
    if (S->nNodes > 0)
    {
        V3 th, tn;
        int tm;
        float tt;
        if (bvh_intersect(S->nodes, S->nNodes, S->tris, o, d, &th, &tn, &tm, &tt, closest, counting ? bc : NULL))
        {
            closest = tt; *hit = th; *N = tn; *matIdx = tm;
        }
    }
    else
    {
        V3 th, tn;
        for (int i = 0; i < S->nTri; i++)
        {
            if (!tri_hit(&S->tris[i], o, d, &th, &tn, &t0, closest) || t0 >= closest) continue;
            closest = t0; *hit = th; *N = tn; *matIdx = S->tris[i].matIdx;
        }
        bc[1] = S->nTri;
    }
    if (counting)
    {
        __atomic_fetch_add(&g_counts[0], 1, __ATOMIC_RELAXED);
        __atomic_fetch_add(&g_counts[1], (long)S->nPlanes, __ATOMIC_RELAXED);
        __atomic_fetch_add(&g_counts[2], (long)S->nSph, __ATOMIC_RELAXED);
        __atomic_fetch_add(&g_counts[3], bc[0], __ATOMIC_RELAXED);
        __atomic_fetch_add(&g_counts[4], bc[1], __ATOMIC_RELAXED);
    }
    return closest < FLT_MAX;
}

void oracle_scene_intersect(const OScene *S, const float *rays, int n, int *mat, float *hitN)
{
    for (int i = 0; i < n; i++)
    {
        V3 h = v3(0, 0, 0), N = v3(0, 0, 0);
        int m = -1;
        int got = scene_intersect(S, vld(rays + i * 6), vld(rays + i * 6 + 3), &h, &N, &m);
        mat[i] = got ? m : -1;
        float *o = hitN + i * 6;
        o[0] = got ? h.x : 0.f; o[1] = got ? h.y : 0.f; o[2] = got ? h.z : 0.f;
        o[3] = got ? N.x : 0.f; o[4] = got ? N.y : 0.f; o[5] = got ? N.z : 0.f;
    }
}

/* ------------------------------------------------------------ shading helpers */
/* Ray::genRayFromIntersection (Ray.h:28-53) */
static V3 hemisphere_dir(V3 N, float r1, float r2)
{
    V3 helper = fabsf(N.x) <= fabsf(N.y) ? v3(1, 0, 0) : v3(0, 1, 0);
    V3 T = vnorm(vcross(N, helper));
    V3 B = vcross(N, T);
    float r = sqrtf(r1);
    float phi = 2.f * PI_F * r2;
    float x = r * cosf(phi), y = r * sinf(phi);
    float z = sqrtf(smax(0.f, 1.f - x * x - y * y));
    return vadd(vadd(vmul(T, x), vmul(B, y)), vmul(N, z));
}

/* Optics (Optics.h:22-27 schlick, :37-40 cauchy, :59-82 dielectricBounce) */
static float schlick(float cosT, float n1, float n2)
{
    float F0 = (n1 - n2) / (n1 + n2);
    F0 *= F0;
    return F0 + (1.f - F0) * powf(1.f - cosT, 5.f);
}
static float cauchy_ior(float ior, float b, float lam) { return ior + b * 1e4f / (lam * lam); }
static void dielectric(V3 d, V3 N, V3 hit, int entering, float ior, float u, V3 *od, V3 *oo)
{
    float cosI = -vdot(d, N);
    float n1 = entering ? 1.f : ior, n2 = entering ? ior : 1.f;
    float eta = n1 / n2;
    float sinT2 = eta * eta * (1.f - cosI * cosI);
    if (sinT2 >= 1.f || u < schlick(cosI, n1, n2))
    {
        *od = vadd(d, vmul(N, 2.f * cosI));
        *oo = vadd(hit, vmul(N, 1e-3f));
        return;
    }
    float cosT = sqrtf(1.f - sinT2);
    *od = vadd(vmul(d, eta), vmul(N, eta * cosI - cosT));
    *oo = vsub(hit, vmul(N, 1e-3f));
}

typedef struct {
    const OScene *S;
    int maxDepth, samples, shadow, mis, russian, stratified;
    float totalLightArea;
} OCtx;

/* Light pick + sample (Renderer.cpp:574-615 / 812-850) */
static void sample_light(const OCtx *c, ORng *rng, V3 *P, V3 *Nl, int *lmat)
{
    const OScene *S = c->S;
    int pick = 0;
    if (S->nLights > 1)
    {
        float target = eps(rng) * c->totalLightArea, cum = 0.f;
        for (int i = 0; i < S->nLights; i++)
        {
            cum += S->lights[i].totalArea;
            if (target <= cum) { pick = i; break; }
        }
    }
    const OLight *L = &S->lights[pick];
    if (L->kind == 0)
    {
        float ru = eps(rng), rv = eps(rng);
        *P = vadd(vadd(vld(L->plane.origin), vmul(vld(L->plane.u), ru)), vmul(vld(L->plane.v), rv));
        *Nl = vld(L->plane.N);
        *lmat = L->plane.matIdx;
    }
    else
    {
        float rtri = eps(rng) * L->totalArea;
        const float *cum = S->lightCum + L->triOffset;
        int lo = 0, hi = L->triCount; /* std::lower_bound */
        while (lo < hi)
        {
            int mid = lo + (hi - lo) / 2;
            if (cum[mid] < rtri) lo = mid + 1; else hi = mid;
        }
        int ti = lo < L->triCount - 1 ? lo : L->triCount - 1;
        const OTriangle *t = &S->lightTris[L->triOffset + ti];
        float r1 = eps(rng), r2 = eps(rng);
        if (r1 + r2 > 1.f) { r1 = 1.f - r1; r2 = 1.f - r2; }
        V3 v0 = vld(t->v0);
        *P = vadd(vadd(v0, vmul(vsub(vld(t->v1), v0), r1)), vmul(vsub(vld(t->v2), v0), r2));
        *Nl = vld(t->flatN);
        *lmat = t->matIdx;
    }
}

/* Shadow test (Renderer.cpp:617-625 / 852-860); returns 1 when lit and sets
 * cosTheta, cosLight, lightDist2. */
static int shadow_lit(const OCtx *c, V3 *hit, V3 N, V3 P, V3 Nl, float *cosT, float *cosL, float *d2)
{
    V3 Li = vsub(P, *hit);
    V3 wi = vnorm(Li);
    float cosTheta = smax(0.f, vdot(wi, N));
    float lightDist2 = vdot(Li, Li);
    /* `hit + N * 1e-3` binds Vec3f's non-const operator+ (Vec3f.h:67-73),
     * which adds into `hit` itself: the lit-facing branch moves the shading
     * point by 1e-3*N for every later shadow sample. */
    V3 so;
    if (cosTheta <= 0) so = vsub(*hit, vmul(N, 1e-3f));
    else { *hit = vadd(*hit, vmul(N, 1e-3f)); so = *hit; }
    V3 sh, sn;
    int sm = -1;
    int blocked = 0;
    if (scene_intersect(c->S, so, wi, &sh, &sn, &sm))
    {
        V3 dd = vsub(sh, so);
        blocked = (double)lightDist2 - 1e-3 > (double)vdot(dd, dd) && !is_emissive(&c->S->mats[sm]);
    }
    *cosT = cosTheta;
    *cosL = smax(0.f, vdot(Nl, vmul(Li, -1.f)));
    *d2 = lightDist2;
    return !blocked;
}

static inline float mis_weight(const OCtx *c, float cosTheta, float cosLight, float d2)
{
    if (!c->mis || !(cosLight > 1e-6f)) return 1.f;
    float pL = d2 / (cosLight * c->totalLightArea);
    float pB = cosTheta / PI_F;
    return (pL * pL) / (pL * pL + pB * pB);
}

/* Renderer::castRay, RGB mode (Renderer.cpp:468-654) */
static V3 cast_rgb(const OCtx *c, ORng *rng, V3 o, V3 d, int depth)
{
    const OScene *S = c->S;
    V3 hit, N;
    int mi = -1;
    if (depth >= c->maxDepth || !scene_intersect(S, o, d, &hit, &N, &mi)) return v3(0, 0, 0);
    const OMaterial *m = &S->mats[mi];
    int entering = vdot(d, N) < 0.f;
    if (!entering) N = vmul(N, -1.f);
    V3 alb = vld(m->albedo);
    if (is_emissive(m)) return vld(m->emissive);
    if (m->metallic)
    {
        float cosI = -vdot(d, N);
        V3 r = cast_rgb(c, rng, vadd(hit, vmul(N, 1e-3f)), vadd(d, vmul(N, 2.f * cosI)), depth + 1);
        return vmulv(r, alb);
    }
    if (m->transparent)
    {
        V3 bd, bo;
        dielectric(d, N, hit, entering, m->ior, eps(rng), &bd, &bo);
        return vmulv(cast_rgb(c, rng, bo, bd, depth + 1), alb);
    }
    V3 ind = v3(0, 0, 0);
    int strata = 0;
    if (c->stratified)
    {
        strata = (int)roundf(sqrtf((float)c->samples));
        if (strata < 1) strata = 1;
    }
    for (int i = 0; i < c->samples; i++)
    {
        /* genRayFromIntersection(N, hit + N * 1e-3, ...) also goes through the
         * mutating operator+: each indirect sample starts 1e-3*N further out
         * and the shadow loop below sees the moved point. */
        hit = vadd(hit, vmul(N, 1e-3f));
        V3 ho = hit;
        float r1, r2;
        if (c->stratified)
        {
            int sx = i % strata, sy = (i / strata) % strata;
            r1 = (sx + eps(rng)) / (float)strata;
            r2 = (sy + eps(rng)) / (float)strata;
        }
        else { r1 = eps(rng); r2 = eps(rng); }
        V3 nd = hemisphere_dir(N, r1, r2);
        if (c->russian && depth >= 1)
        {
            float ma = smax(smax(alb.x, alb.y), alb.z);
            float p = smin(0.95f, smax(0.05f, ma));
            if (eps(rng) > p) continue;
            ind = vadd(ind, vdiv(vmulv(cast_rgb(c, rng, ho, nd, depth + 1), alb), p));
        }
        else
            ind = vadd(ind, vmulv(cast_rgb(c, rng, ho, nd, depth + 1), alb));
    }
    ind = vdiv(ind, (float)c->samples);
    V3 dir = v3(0, 0, 0);
    if (c->totalLightArea > 0.f)
    {
        for (int i = 0; i < c->shadow; i++)
        {
            V3 P, Nl;
            int lm;
            sample_light(c, rng, &P, &Nl, &lm);
            float cosT, cosL, d2;
            if (shadow_lit(c, &hit, N, P, Nl, &cosT, &cosL, &d2))
            {
                float G = (cosT * cosL) / d2;
                V3 contrib = vmul(vmul(vmulv(vdiv(alb, PI_F), vld(S->mats[lm].emissive)), G), c->totalLightArea);
                if (c->mis && cosL > 1e-6f) contrib = vmul(contrib, mis_weight(c, cosT, cosL, d2));
                dir = vadd(dir, contrib);
            }
        }
    }
    return vadd(vdiv(dir, (float)c->shadow), ind);
}

/* Renderer::castRaySpectral (Renderer.cpp:656-889) */
static void cast_spec(const OCtx *c, ORng *rng, V3 o, V3 d, int depth, const float lam[4], float out[4])
{
    const OScene *S = c->S;
    V3 hit, N;
    int mi = -1;
    out[0] = out[1] = out[2] = out[3] = 0.f;
    if (depth >= c->maxDepth || !scene_intersect(S, o, d, &hit, &N, &mi)) return;
    const OMaterial *m = &S->mats[mi];
    int entering = vdot(d, N) < 0.f;
    if (!entering) N = vmul(N, -1.f);
    if (is_emissive(m))
    {
        for (int k = 0; k < 4; k++) out[k] = emissive_at(m, lam[k]);
        return;
    }
    float r[4];
    if (m->metallic)
    {
        float cosI = -vdot(d, N);
        cast_spec(c, rng, vadd(hit, vmul(N, 1e-3f)), vadd(d, vmul(N, 2.f * cosI)), depth + 1, lam, r);
        for (int k = 0; k < 4; k++) out[k] = r[k] * albedo_at(m, lam[k]);
        return;
    }
    if (m->transparent)
    {
        if (m->cauchyB == 0.f)
        {
            V3 bd, bo;
            dielectric(d, N, hit, entering, m->ior, eps(rng), &bd, &bo);
            cast_spec(c, rng, bo, bd, depth + 1, lam, r);
            for (int k = 0; k < 4; k++) out[k] = r[k] * albedo_at(m, lam[k]);
            return;
        }
        for (int k = 0; k < 4; k++)
        {
            float iorK = cauchy_ior(m->ior, m->cauchyB, lam[k]);
            V3 bd, bo;
            dielectric(d, N, hit, entering, iorK, eps(rng), &bd, &bo);
            float single[4] = {lam[k], lam[k], lam[k], lam[k]};
            cast_spec(c, rng, bo, bd, depth + 1, single, r);
            out[k] = r[0] * albedo_at(m, lam[k]);
        }
        return;
    }
    float al[4];
    for (int k = 0; k < 4; k++) al[k] = albedo_at(m, lam[k]);
    float ind[4] = {0, 0, 0, 0};
    int strata = 0;
    if (c->stratified)
    {
        strata = (int)roundf(sqrtf((float)c->samples));
        if (strata < 1) strata = 1;
    }
    for (int i = 0; i < c->samples; i++)
    {
        /* genRayFromIntersection(N, hit + N * 1e-3, ...) also goes through the
         * mutating operator+: each indirect sample starts 1e-3*N further out
         * and the shadow loop below sees the moved point. */
        hit = vadd(hit, vmul(N, 1e-3f));
        V3 ho = hit;
        float r1, r2;
        if (c->stratified)
        {
            int sx = i % strata, sy = (i / strata) % strata;
            r1 = (sx + eps(rng)) / (float)strata;
            r2 = (sy + eps(rng)) / (float)strata;
        }
        else { r1 = eps(rng); r2 = eps(rng); }
        V3 nd = hemisphere_dir(N, r1, r2);
        if (c->russian && depth >= 1)
        {
            float p = smin(0.95f, smax(0.05f, al[0]));
            if (eps(rng) > p) continue;
            cast_spec(c, rng, ho, nd, depth + 1, lam, r);
            for (int k = 0; k < 4; k++) ind[k] += r[k] * al[k] / p;
        }
        else
        {
            cast_spec(c, rng, ho, nd, depth + 1, lam, r);
            for (int k = 0; k < 4; k++) ind[k] += r[k] * al[k];
        }
    }
    for (int k = 0; k < 4; k++) ind[k] /= (float)c->samples;
    float dir[4] = {0, 0, 0, 0};
    if (c->totalLightArea > 0.f)
    {
        for (int i = 0; i < c->shadow; i++)
        {
            V3 P, Nl;
            int lm;
            sample_light(c, rng, &P, &Nl, &lm);
            float cosT, cosL, d2;
            if (shadow_lit(c, &hit, N, P, Nl, &cosT, &cosL, &d2))
            {
                float G = (cosT * cosL) / d2;
                float w = mis_weight(c, cosT, cosL, d2);
                for (int k = 0; k < 4; k++)
                {
                    float eL = emissive_at(&S->mats[lm], lam[k]);
                    dir[k] += (al[k] / PI_F) * eL * G * c->totalLightArea * w;
                }
            }
        }
    }
    for (int k = 0; k < 4; k++) out[k] = dir[k] / (float)c->shadow + ind[k];
}

/* One camera sample (Renderer.cpp:196-257): XYZ/N in spectral mode, else RGB. */
static V3 camera_sample(const OCtx *c, const OOpts *op, ORng *rng, int i, int j, int jitter)
{
    const OScene *S = c->S;
    float aspect = op->width / (float)op->height;
    float scale = tanf(PI_F / 180.f * 0.5f * S->fov);
    float jx = jitter ? (eps(rng) - 0.5f) : 0.f;
    float jy = jitter ? (eps(rng) - 0.5f) : 0.f;
    float x = ((2 * (j + 0.5f + jx) / (float)op->width) - 1) * scale * aspect;
    float y = -((2 * (i + 0.5f + jy) / (float)op->height) - 1) * scale;
    V3 d = vnorm(v3(x, y, -1.f));
    V3 o = vld(S->camPos);
    if (!op->spectral) return cast_rgb(c, rng, o, d, 0);
    int N = op->hero < 1 ? 1 : (op->hero > 4 ? 4 : op->hero);
    const float span = LMAX - LMIN;
    float stride = span / (float)N;
    float lam[4];
    lam[0] = LMIN + eps(rng) * span;
    for (int k = 1; k < N; k++)
    {
        float l = lam[0] + stride * k;
        if (l > LMAX) l -= span;
        lam[k] = l;
    }
    for (int k = N; k < 4; k++) lam[k] = lam[0];
    float rad[4];
    cast_spec(c, rng, o, d, 0, lam, rad);
    V3 xyz = v3(0, 0, 0);
    for (int k = 0; k < N; k++) xyz = vadd(xyz, single_lambda_xyz(lam[k], rad[k]));
    return vdiv(xyz, (float)N);
}

typedef struct {
    const OCtx *c; const OOpts *op; int mode, spp, nThreads, t;
    float *hdr; double *acc;
} OJob;

static void *render_rows(void *arg)
{
    OJob *J = (OJob *)arg;
    const OOpts *op = J->op;
    ORng rng = rng_for_thread(op->seed, (uint64_t)J->t);
    for (int i = J->t; i < op->height; i += J->nThreads)
        for (int j = 0; j < op->width; j++)
        {
            size_t px = (size_t)i * op->width + j;
            if (J->mode == 0)
            {
                /* Renderer.cpp:190-302: Welford mean over aa samples */
                int aa = op->aa < 1 ? 1 : op->aa;
                float mean[3] = {0, 0, 0}, M2[3] = {0, 0, 0};
                int taken = 0;
                for (int s = 0; s < aa; s++)
                {
                    V3 cc = camera_sample(J->c, op, &rng, i, j, aa > 1);
                    float cv[3] = {cc.x, cc.y, cc.z};
                    taken++;
                    float dl[3], d2[3];
                    for (int ch = 0; ch < 3; ch++) { dl[ch] = cv[ch] - mean[ch]; }
                    for (int ch = 0; ch < 3; ch++) mean[ch] += dl[ch] / taken;
                    for (int ch = 0; ch < 3; ch++) d2[ch] = cv[ch] - mean[ch];
                    for (int ch = 0; ch < 3; ch++) M2[ch] += dl[ch] * d2[ch];
                    if (op->adaptive && taken >= 4)
                    {
                        int conv = 1;
                        for (int ch = 0; ch < 3; ch++)
                        {
                            float v = M2[ch] / (float)(taken - 1);
                            float rel = v / (mean[ch] * mean[ch] + 0.01f);
                            if (rel >= 0.05f) { conv = 0; break; }
                        }
                        if (conv) break;
                    }
                }
                V3 m = v3(mean[0], mean[1], mean[2]);
                if (op->spectral) m = xyz_to_srgb(m);
                J->hdr[px * 3 + 0] = m.x; J->hdr[px * 3 + 1] = m.y; J->hdr[px * 3 + 2] = m.z;
            }
            else
            {
                double a[3] = {0, 0, 0};
                for (int s = 0; s < J->spp; s++)
                {
                    V3 cc = camera_sample(J->c, op, &rng, i, j, 0);
                    a[0] += cc.x; a[1] += cc.y; a[2] += cc.z;
                }
                for (int ch = 0; ch < 3; ch++) a[ch] /= J->spp;
                if (op->spectral)
                {
                    double X = a[0], Y = a[1], Z = a[2];
                    a[0] = 3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z;
                    a[1] = -0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z;
                    a[2] = 0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z;
                }
                J->acc[px * 3 + 0] = a[0]; J->acc[px * 3 + 1] = a[1]; J->acc[px * 3 + 2] = a[2];
            }
        }
    return NULL;
}

static void run_threads(OJob *proto, int nThreads)
{
    pthread_t th[256];
    OJob jobs[256];
    if (nThreads > 256) nThreads = 256;
    for (int t = 0; t < nThreads; t++)
    {
        jobs[t] = *proto;
        jobs[t].nThreads = nThreads;
        jobs[t].t = t;
        pthread_create(&th[t], NULL, render_rows, &jobs[t]);
    }
    for (int t = 0; t < nThreads; t++) pthread_join(th[t], NULL);
}

static float scene_light_area(const OScene *S)
{
    float total = 0.f;
    for (int i = 0; i < S->nLights; i++) total += S->lights[i].totalArea;
    return total;
}

/* 8-bit quantisation (Renderer.cpp:379-381): (unsigned char)(255*c + 0.5f)
 * as x86-64 g++ lowers it (cvttss2si to int32, keep the low byte). */
static unsigned char quantize(float c)
{
    float v = 255 * c + 0.5f;
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0;
    return (unsigned char)((int)v & 0xFF);
}

/* Denoise::bilateralRGB (Denoise.cpp:14-86) */
void oracle_bilateral(unsigned char *rgb, int w, int h)
{
    const int radius = 2;
    const float is2 = 1.0f / (2.0f * 1.5f * 1.5f), ic2 = 1.0f / (2.0f * 10.0f * 10.0f);
    size_t n = (size_t)w * h * 3;
    unsigned char *out = (unsigned char *)malloc(n);
    for (int pass = 0; pass < 2; pass++)
    {
        const unsigned char *src = pass == 0 ? rgb : out;
        unsigned char *dst = pass == 0 ? out : rgb;
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++)
            {
                size_t ci = ((size_t)y * w + x) * 3;
                float cR = src[ci], cG = src[ci + 1], cB = src[ci + 2];
                float sW = 0, sR = 0, sG = 0, sB = 0;
                for (int dy = -radius; dy <= radius; dy++)
                {
                    int ny = y + dy;
                    if (ny < 0 || ny >= h) continue;
                    for (int dx = -radius; dx <= radius; dx++)
                    {
                        int nx = x + dx;
                        if (nx < 0 || nx >= w) continue;
                        size_t ni = ((size_t)ny * w + nx) * 3;
                        float nR = src[ni], nG = src[ni + 1], nB = src[ni + 2];
                        float sp = (float)(dx * dx + dy * dy) * is2;
                        float dR = nR - cR, dG = nG - cG, dB = nB - cB;
                        float col = (dR * dR + dG * dG + dB * dB) * ic2;
                        float wgt = expf(-(sp + col));
                        sW += wgt; sR += wgt * nR; sG += wgt * nG; sB += wgt * nB;
                    }
                }
                if (sW > 0.0f)
                {
                    dst[ci] = (unsigned char)smin(255.0f, sR / sW + 0.5f);
                    dst[ci + 1] = (unsigned char)smin(255.0f, sG / sW + 0.5f);
                    dst[ci + 2] = (unsigned char)smin(255.0f, sB / sW + 0.5f);
                }
                else { dst[ci] = src[ci]; dst[ci + 1] = src[ci + 1]; dst[ci + 2] = src[ci + 2]; }
            }
    }
    free(out);
}

/* ToneMap (ToneMap.h:14-39) */
static void tonemap(float *c, int aces)
{
    for (int i = 0; i < 3; i++)
    {
        float x = c[i];
        if (aces)
        {
            float v = (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
            if (v < 0.f) v = 0.f;
            if (v > 1.f) v = 1.f;
            c[i] = v;
        }
        else
            c[i] = x / (x + 1.f);
    }
}

/* Renderer::render without the PNG write: hdr = pre-tonemap framebuffer
 * (linear sRGB), rgb8 = tone-mapped, quantised (and denoised) pixels.
 * A non-zero seed forces one thread (Renderer.cpp:158-160). */
void oracle_render(const OScene *S, const OOpts *op, int threads, float *hdr, unsigned char *rgb8)
{
    OCtx c = {S, op->depth, op->samples, op->shadow, op->mis, op->russian, op->stratified, scene_light_area(S)};
    OJob job = {&c, op, 0, 0, 1, 0, hdr, NULL};
    int nt = op->seed != 0 ? 1 : (threads > 0 ? threads : 1);
    run_threads(&job, nt);
    if (!rgb8) return;
    size_t n = (size_t)op->width * op->height;
    for (size_t i = 0; i < n; i++)
    {
        float px[3] = {hdr[i * 3], hdr[i * 3 + 1], hdr[i * 3 + 2]};
        tonemap(px, op->aces);
        for (int k = 0; k < 3; k++) rgb8[i * 3 + k] = quantize(px[k]);
    }
    if (op->denoise) oracle_bilateral(rgb8, op->width, op->height);
}

/* The GPU estimator on the CPU: spp camera paths through each pixel centre
 * with one indirect continuation per diffuse vertex (samples = 1), FP64
 * per-pixel mean, linear sRGB out. */
void oracle_render_paths(const OScene *S, const OOpts *op, int spp, int threads, double *out)
{
    OCtx c = {S, op->depth, 1, op->shadow, op->mis, op->russian, op->stratified, scene_light_area(S)};
    OJob job = {&c, op, 1, spp, 1, 0, NULL, out};
    run_threads(&job, threads > 0 ? threads : 1);
}

/* ------------------------------------------------------------ stage grids */
float oracle_ybar_integral(void) { return ybar_integral(); }
void oracle_eval_fit(const float *fit, const float *lam, int n, float *out)
{
    for (int i = 0; i < n; i++) out[i] = eval_fit(fit, lam[i]);
}
void oracle_eval_spectrum(const float *tab, const float *lam, int n, float *out)
{
    for (int i = 0; i < n; i++) out[i] = spec_eval(tab, lam[i]);
}
void oracle_eval_cmf(const float *lam, int n, float *out)
{
    for (int i = 0; i < n; i++) { out[i * 3] = xbar(lam[i]); out[i * 3 + 1] = ybar(lam[i]); out[i * 3 + 2] = zbar(lam[i]); }
}
void oracle_single_lambda_xyz(const float *lam, const float *rad, int n, float *out)
{
    for (int i = 0; i < n; i++)
    {
        V3 v = single_lambda_xyz(lam[i], rad[i]);
        out[i * 3] = v.x; out[i * 3 + 1] = v.y; out[i * 3 + 2] = v.z;
    }
}
void oracle_xyz_to_srgb(const float *in, int n, float *out)
{
    for (int i = 0; i < n; i++)
    {
        V3 v = xyz_to_srgb(vld(in + i * 3));
        out[i * 3] = v.x; out[i * 3 + 1] = v.y; out[i * 3 + 2] = v.z;
    }
}
void oracle_tonemap(const float *in, int n, int aces, float *out, unsigned char *q)
{
    for (int i = 0; i < n; i++)
    {
        float px[3] = {in[i * 3], in[i * 3 + 1], in[i * 3 + 2]};
        tonemap(px, aces);
        for (int k = 0; k < 3; k++)
        {
            out[i * 3 + k] = px[k];
            if (q) q[i * 3 + k] = quantize(px[k]);
        }
    }
}
void oracle_spectrum_to_xyz(const float *tab, float *out)
{
    V3 v = spectrum_to_xyz(tab);
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
}
float oracle_schlick(float c, float n1, float n2) { return schlick(c, n1, n2); }
float oracle_cauchy(float ior, float b, float lam) { return cauchy_ior(ior, b, lam); }
void oracle_dielectric(const float *in, int entering, float ior, float u, float *out)
{
    V3 od, oo;
    dielectric(vld(in), vld(in + 3), vld(in + 6), entering, ior, u, &od, &oo);
    out[0] = od.x; out[1] = od.y; out[2] = od.z; out[3] = oo.x; out[4] = oo.y; out[5] = oo.z;
}
void oracle_hemisphere_dir(const float *N, float r1, float r2, float *out)
{
    V3 d = hemisphere_dir(vld(N), r1, r2);
    out[0] = d.x; out[1] = d.y; out[2] = d.z;
}
