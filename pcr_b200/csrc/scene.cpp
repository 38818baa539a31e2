// Host-side scene admission.  Float arithmetic follows the reference's
// operation order; this file is compiled with -ffp-contract=off so the fit
// coefficients, plane/triangle constants and BVH boxes come out bit-equal to
// the reference loader's.
#include "scene.h"

#include <algorithm>
#include <array>
#include <charconv>
#include <cfloat>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <future>
#include <thread>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include "engine.h"

namespace pcr {

// ============================================================ JSON (JSONC)
namespace {

struct JVal {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double num = 0;
    bool is_int = false;
    long long inum = 0;
    std::string str;
    std::vector<JVal> arr;
    std::map<std::string, JVal> obj;  // key order, as nlohmann::json iterates
    const JVal* get(const std::string& k) const
    {
        auto it = obj.find(k);
        return it == obj.end() ? nullptr : &it->second;
    }
    float as_float() const { return is_int ? (float)inum : (float)num; }
};

struct JParser {
    const std::string& s;
    size_t i = 0;
    std::string path;
    explicit JParser(const std::string& t, const std::string& p) : s(t), path(p) {}
    [[noreturn]] void fail(const std::string& m)
    {
        int line = 1, col = 1;
        for (size_t k = 0; k < i && k < s.size(); k++) {
            if (s[k] == '\n') { line++; col = 1; } else col++;
        }
        throw PcrError(PCR_ERR_SCENE, path + ":" + std::to_string(line) + ":" + std::to_string(col) + ": JSON parse error: " + m);
    }
    void ws()
    {
        for (;;) {
            while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) i++;
            if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '/') {
                while (i < s.size() && s[i] != '\n') i++;
            } else if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '*') {
                size_t e = s.find("*/", i + 2);
                if (e == std::string::npos) fail("unterminated comment");
                i = e + 2;
            } else {
                break;
            }
        }
    }
    JVal value()
    {
        ws();
        if (i >= s.size()) fail("unexpected end of input");
        char c = s[i];
        JVal v;
        if (c == '{') {
            v.kind = JVal::Obj;
            i++;
            ws();
            if (i < s.size() && s[i] == '}') { i++; return v; }
            for (;;) {
                ws();
                if (i >= s.size() || s[i] != '"') fail("expected object key");
                std::string k = string_();
                ws();
                if (i >= s.size() || s[i] != ':') fail("expected ':'");
                i++;
                v.obj[k] = value();
                ws();
                if (i < s.size() && s[i] == ',') { i++; continue; }
                if (i < s.size() && s[i] == '}') { i++; break; }
                fail("expected ',' or '}'");
            }
        } else if (c == '[') {
            v.kind = JVal::Arr;
            i++;
            ws();
            if (i < s.size() && s[i] == ']') { i++; return v; }
            for (;;) {
                v.arr.push_back(value());
                ws();
                if (i < s.size() && s[i] == ',') { i++; continue; }
                if (i < s.size() && s[i] == ']') { i++; break; }
                fail("expected ',' or ']'");
            }
        } else if (c == '"') {
            v.kind = JVal::Str;
            v.str = string_();
        } else if (s.compare(i, 4, "true") == 0) {
            v.kind = JVal::Bool; v.b = true; i += 4;
        } else if (s.compare(i, 5, "false") == 0) {
            v.kind = JVal::Bool; v.b = false; i += 5;
        } else if (s.compare(i, 4, "null") == 0) {
            v.kind = JVal::Null; i += 4;
        } else if (c == '-' || (c >= '0' && c <= '9')) {
            size_t st = i;
            if (s[i] == '-') i++;
            while (i < s.size() && isdigit((unsigned char)s[i])) i++;
            bool integral = true;
            if (i < s.size() && s[i] == '.') { integral = false; i++; while (i < s.size() && isdigit((unsigned char)s[i])) i++; }
            if (i < s.size() && (s[i] == 'e' || s[i] == 'E')) {
                integral = false;
                i++;
                if (i < s.size() && (s[i] == '+' || s[i] == '-')) i++;
                while (i < s.size() && isdigit((unsigned char)s[i])) i++;
            }
            std::string tok = s.substr(st, i - st);
            v.kind = JVal::Num;
            v.num = std::strtod(tok.c_str(), nullptr);
            if (integral) { v.is_int = true; v.inum = std::strtoll(tok.c_str(), nullptr, 10); }
        } else {
            fail(std::string("unexpected character '") + c + "'");
        }
        return v;
    }
    std::string string_()
    {
        std::string out;
        i++;
        while (i < s.size() && s[i] != '"') {
            if (s[i] == '\\' && i + 1 < s.size()) {
                char e = s[i + 1];
                out += e == 'n' ? '\n' : e == 't' ? '\t' : e;
                i += 2;
            } else {
                out += s[i++];
            }
        }
        if (i >= s.size()) fail("unterminated string");
        i++;
        return out;
    }
};

std::string read_file(const std::string& p)
{
    std::ifstream in(p, std::ios::binary);
    if (!in) throw PcrError(PCR_ERR_SCENE, "Cannot open scene file: " + p);
    std::ostringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

// ============================================================ spectral math (host)
// code/Includes/CIE.h:27-53 and :79-123; code/Includes/Spectrum.h:167-229
inline float wy(float l, float mu, float s1, float s2)
{
    float t = (l < mu) ? (l - mu) * s1 : (l - mu) * s2;
    return std::exp(-0.5f * t * t);
}
inline float xbar(float l)
{
    return 0.362f * wy(l, 442.0f, 0.0624f, 0.0374f) + 1.056f * wy(l, 599.8f, 0.0264f, 0.0323f) -
           0.065f * wy(l, 501.1f, 0.0490f, 0.0382f);
}
inline float ybar(float l) { return 0.821f * wy(l, 568.8f, 0.0213f, 0.0247f) + 0.286f * wy(l, 530.9f, 0.0613f, 0.0322f); }
inline float zbar(float l) { return 1.217f * wy(l, 437.0f, 0.0845f, 0.0278f) + 0.681f * wy(l, 459.0f, 0.0385f, 0.0725f); }
inline float lambda_at(int i) { return 400.f + i * 5.0f; }
float ybar_integral()
{
    static float v = [] {
        float sum = 0.f;
        for (int i = 0; i < kSpecN; i++) sum += ybar(lambda_at(i));
        return sum * 5.0f;
    }();
    return v;
}
void srgb_to_xyz(const float c[3], float o[3])
{
    o[0] = 0.4124564f * c[0] + 0.3575761f * c[1] + 0.1804375f * c[2];
    o[1] = 0.2126729f * c[0] + 0.7151522f * c[1] + 0.0721750f * c[2];
    o[2] = 0.0193339f * c[0] + 0.1191920f * c[1] + 0.9503041f * c[2];
}
void xyz_to_srgb(const float c[3], float o[3])
{
    o[0] = 3.2404542f * c[0] - 1.5371385f * c[1] - 0.4985314f * c[2];
    o[1] = -0.9692660f * c[0] + 1.8760108f * c[1] + 0.0415560f * c[2];
    o[2] = 0.0556434f * c[0] - 0.2040259f * c[1] + 1.0572252f * c[2];
}
void spectrum_to_xyz(const float* s, float o[3])
{
    float X = 0.f, Y = 0.f, Z = 0.f;
    for (int i = 0; i < kSpecN; i++) {
        float l = lambda_at(i), v = s[i];
        X += v * xbar(l);
        Y += v * ybar(l);
        Z += v * zbar(l);
    }
    float scale = 5.0f / ybar_integral();
    o[0] = X * scale; o[1] = Y * scale; o[2] = Z * scale;
}
inline float sclamp(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
inline float sigm(float x) { return 0.5f + x / (2.f * std::sqrt(1.f + x * x)); }
inline float sigm_d(float x) { float t = 1.f + x * x; return 0.5f / (t * std::sqrt(t)); }
inline float sigm_inv(float y)
{
    y = sclamp(y, 1e-4f, 1.f - 1e-4f);
    float u = 2.f * y - 1.f;
    return u / std::sqrt(1.f - u * u);
}

// ============================================================ sigmoid fit
// code/RGBToSpectrum.cpp:27-53 solve3x3
bool solve3x3(const float J[3][3], const float b[3], float x[3])
{
    float det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    if (std::fabs(det) < 1e-12f) return false;
    float inv = 1.f / det;
    float d0 = b[0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (b[1] * J[2][2] - J[1][2] * b[2]) +
               J[0][2] * (b[1] * J[2][1] - J[1][1] * b[2]);
    float d1 = J[0][0] * (b[1] * J[2][2] - J[1][2] * b[2]) - b[0] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
               J[0][2] * (J[1][0] * b[2] - b[1] * J[2][0]);
    float d2 = J[0][0] * (J[1][1] * b[2] - b[1] * J[2][1]) - J[0][1] * (J[1][0] * b[2] - b[1] * J[2][0]) +
               b[0] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    x[0] = d0 * inv; x[1] = d1 * inv; x[2] = d2 * inv;
    return true;
}

void integrate(const float c[3], float xyz[3], float (*J)[3])
{
    xyz[0] = xyz[1] = xyz[2] = 0.f;
    if (J) for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) J[a][b] = 0.f;
    for (int i = 0; i < kSpecN; i++) {
        float l = lambda_at(i);
        float ln = (l - 550.f) / 150.f;
        float p = c[0] + ln * (c[1] + ln * c[2]);
        float s = sigm(p);
        float xb = xbar(l), yb = ybar(l), zb = zbar(l);
        xyz[0] += s * xb; xyz[1] += s * yb; xyz[2] += s * zb;
        if (J) {
            float ds = sigm_d(p), ln2 = ln * ln;
            J[0][0] += ds * xb; J[0][1] += ds * ln * xb; J[0][2] += ds * ln2 * xb;
            J[1][0] += ds * yb; J[1][1] += ds * ln * yb; J[1][2] += ds * ln2 * yb;
            J[2][0] += ds * zb; J[2][1] += ds * ln * zb; J[2][2] += ds * ln2 * zb;
        }
    }
}

// code/RGBToSpectrum.cpp:59-166 newtonFit
void newton_fit(const float tgt[3], const float cin[3], float cout[3])
{
    float c[3] = {cin[0], cin[1], cin[2]};
    for (int it = 0; it < 15; it++) {
        float xyz[3], J[3][3];
        integrate(c, xyz, J);
        for (int k = 0; k < 3; k++) {
            xyz[k] *= 5.0f;
            for (int j = 0; j < 3; j++) J[k][j] *= 5.0f;
        }
        float r[3] = {xyz[0] - tgt[0], xyz[1] - tgt[1], xyz[2] - tgt[2]};
        float rn = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        if (rn < 1e-6f) break;
        float dl[3];
        if (!solve3x3(J, r, dl)) break;
        float prev[3] = {c[0], c[1], c[2]};
        float step = 1.f;
        bool reduced = false;
        for (int trial = 0; trial < 4; trial++) {
            c[0] = prev[0] - step * dl[0];
            c[1] = prev[1] - step * dl[1];
            c[2] = prev[2] - step * dl[2];
            float t[3];
            integrate(c, t, nullptr);
            t[0] *= 5.0f; t[1] *= 5.0f; t[2] *= 5.0f;
            float tr[3] = {t[0] - tgt[0], t[1] - tgt[1], t[2] - tgt[2]};
            float tn = std::sqrt(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]);
            if (tn < rn) { reduced = true; break; }
            step *= 0.5f;
        }
        if (!reduced) {
            c[0] = prev[0]; c[1] = prev[1]; c[2] = prev[2];
            break;
        }
    }
    cout[0] = c[0]; cout[1] = c[1]; cout[2] = c[2];
}

// code/RGBToSpectrum.cpp:175-190: max sample over the median sample
float spikiness(const float c[3])
{
    float s[kSpecN], mx = 0.f;
    for (int i = 0; i < kSpecN; i++) {
        float ln = (lambda_at(i) - 550.f) / 150.f;
        float p = c[0] + ln * (c[1] + ln * c[2]);
        s[i] = 0.5f + p / (2.f * std::sqrt(1.f + p * p));
        if (s[i] > mx) mx = s[i];
    }
    std::nth_element(s, s + kSpecN / 2, s + kSpecN);
    float med = s[kSpecN / 2];
    if (med < 1e-8f) return (mx < 1e-8f) ? 1.f : 1e30f;
    return mx / med;
}

// code/RGBToSpectrum.cpp:192-254: homotopy from the grey of equal Y
void fit_coefficients(const float tgt[3], float out[3])
{
    const float kXn = 0.95046f, kZn = 1.08906f;
    float gray[3] = {tgt[1] * kXn, tgt[1], tgt[1] * kZn};
    float c[3] = {sigm_inv(tgt[1] / ybar_integral()), 0.f, 0.f};
    float good[3] = {c[0], c[1], c[2]};
    for (int step = 1; step <= 32; step++) {
        float t = (float)step / (float)32;
        float cur[3] = {(1.f - t) * gray[0] + t * tgt[0], (1.f - t) * gray[1] + t * tgt[1], (1.f - t) * gray[2] + t * tgt[2]};
        float nx[3];
        newton_fit(cur, c, nx);
        if (spikiness(nx) > 200.f) break;
        c[0] = nx[0]; c[1] = nx[1]; c[2] = nx[2];
        good[0] = c[0]; good[1] = c[1]; good[2] = c[2];
    }
    out[0] = good[0]; out[1] = good[1]; out[2] = good[2];
}

constexpr int kLutRes = 16;
inline int lut_idx(int l, int b, int x, int y) { return ((l * kLutRes + b) * kLutRes + x) * kLutRes * 3 + y * 3; }

// code/RGBToSpectrum.cpp:453-521 trilinear lookup
void lut_lookup(const std::vector<float>& lut, const float rgb[3], float out[4])
{
    float r = sclamp(rgb[0], 0.f, 1.f), g = sclamp(rgb[1], 0.f, 1.f), b = sclamp(rgb[2], 0.f, 1.f);
    if (r <= 0.f && g <= 0.f && b <= 0.f) { out[0] = out[1] = out[2] = out[3] = 0.f; return; }
    if (r >= 1.f && g >= 1.f && b >= 1.f) {
        float sc = ybar_integral();
        out[0] = sigm_inv(1.f / sc); out[1] = out[2] = 0.f; out[3] = sc;
        return;
    }
    int l = 0;
    float mx = r;
    if (g >= mx) { l = 1; mx = g; }
    if (b >= mx) { l = 2; mx = b; }
    float o1, o2;
    if (l == 0) { o1 = g; o2 = b; } else if (l == 1) { o1 = r; o2 = b; } else { o1 = r; o2 = g; }
    float xf = (o1 / mx) * (float)(kLutRes - 1), yf = (o2 / mx) * (float)(kLutRes - 1), bf = mx * (float)(kLutRes - 1);
    int xi = std::clamp((int)xf, 0, kLutRes - 2), yi = std::clamp((int)yf, 0, kLutRes - 2), bi = std::clamp((int)bf, 0, kLutRes - 2);
    float xt = sclamp(xf - xi, 0.f, 1.f), yt = sclamp(yf - yi, 0.f, 1.f), bt = sclamp(bf - bi, 0.f, 1.f);
    out[3] = ybar_integral();
    for (int k = 0; k < 3; k++) {
        auto S = [&](int db, int dx, int dy) { return lut[lut_idx(l, bi + db, xi + dx, yi + dy) + k]; };
        float v00 = S(0, 0, 0) + xt * (S(0, 1, 0) - S(0, 0, 0));
        float v10 = S(0, 0, 1) + xt * (S(0, 1, 1) - S(0, 0, 1));
        float v01 = S(1, 0, 0) + xt * (S(1, 1, 0) - S(1, 0, 0));
        float v11 = S(1, 0, 1) + xt * (S(1, 1, 1) - S(1, 0, 1));
        float v0 = v00 + yt * (v10 - v00), v1 = v01 + yt * (v11 - v01);
        out[k] = v0 + bt * (v1 - v0);
    }
}

}  // namespace

void fit_sigmoid(const float rgb[3], const std::vector<float>* lut, float out[4])
{
    if (lut) { lut_lookup(*lut, rgb, out); return; }
    float r = sclamp(rgb[0], 0.f, 1.f), g = sclamp(rgb[1], 0.f, 1.f), b = sclamp(rgb[2], 0.f, 1.f);
    if (r <= 0.f && g <= 0.f && b <= 0.f) { out[0] = out[1] = out[2] = out[3] = 0.f; return; }
    if (r >= 1.f && g >= 1.f && b >= 1.f) {
        float sc = ybar_integral();
        out[0] = sigm_inv(1.f / sc); out[1] = out[2] = 0.f; out[3] = sc;
        return;
    }
    float c3[3] = {r, g, b}, xyz[3], c[3];
    srgb_to_xyz(c3, xyz);
    fit_coefficients(xyz, c);
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = ybar_integral();
}

void populate_material(pcr_material& m, const std::vector<float>* lut)
{
    fit_sigmoid(m.albedo, lut, m.albedo_fit);
    if (m.emissive[0] > 0 || m.emissive[1] > 0 || m.emissive[2] > 0) {
        float mx = std::max({m.emissive[0], m.emissive[1], m.emissive[2]});
        float n[3] = {m.emissive[0] / mx, m.emissive[1] / mx, m.emissive[2] / mx};
        fit_sigmoid(n, lut, m.emissive_fit);
        m.emissive_fit[3] *= mx;
    } else {
        m.emissive_fit[0] = m.emissive_fit[1] = m.emissive_fit[2] = m.emissive_fit[3] = 0.f;
    }
}

void build_lut(std::vector<float>& out)
{
    out.assign(3 * kLutRes * kLutRes * kLutRes * 3, 0.f);
    for (int l = 0; l < 3; l++)
        for (int xi = 0; xi < kLutRes; xi++)
            for (int yi = 0; yi < kLutRes; yi++) {
                float x = float(xi) / float(kLutRes - 1), y = float(yi) / float(kLutRes - 1);
                for (int bi = 0; bi < kLutRes; bi++) {
                    int idx = lut_idx(l, bi, xi, yi);
                    float b = float(bi) / float(kLutRes - 1);
                    if (b <= 0.f) continue;
                    float v0 = b, v1 = x * b, v2 = y * b;
                    float rgb[3];
                    if (l == 0) { rgb[0] = v0; rgb[1] = v1; rgb[2] = v2; }
                    else if (l == 1) { rgb[0] = v1; rgb[1] = v0; rgb[2] = v2; }
                    else { rgb[0] = v1; rgb[1] = v2; rgb[2] = v0; }
                    float xyz[3], c[3];
                    srgb_to_xyz(rgb, xyz);
                    fit_coefficients(xyz, c);
                    for (int k = 0; k < 3; k++) out[idx + k] = std::clamp(c[k], -200.f, 200.f);
                }
            }
}

bool load_plut(const std::string& path, std::vector<float>& out, std::string* err)
{
    auto fail = [&](const char* m) { if (err) *err = m; return false; };
    std::ifstream in(path, std::ios::binary);
    if (!in) return fail("cannot open file");
    char h[16];
    in.read(h, 16);
    if (in.gcount() != 16) return fail("header truncated");
    if (std::memcmp(h, "PLUT", 4) != 0) return fail("bad magic (not a PLUT file)");
    uint32_t ver, res, nf;
    std::memcpy(&ver, h + 4, 4);
    std::memcpy(&res, h + 8, 4);
    std::memcpy(&nf, h + 12, 4);
    if (ver != 1) return fail("unsupported version");
    if (res != (uint32_t)kLutRes) return fail("res mismatch (recompile pcr or rebuild this LUT)");
    const uint32_t expect = 3u * kLutRes * kLutRes * kLutRes * 3u;
    if (nf != expect) return fail("nFloats mismatch (corrupt header)");
    out.assign(expect, 0.f);
    in.read(reinterpret_cast<char*>(out.data()), (std::streamsize)(expect * sizeof(float)));
    if (in.gcount() != (std::streamsize)(expect * sizeof(float))) return fail("payload truncated");
    return true;
}

bool save_plut(const std::string& path, const std::vector<float>& lut)
{
    std::ofstream o(path, std::ios::binary | std::ios::trunc);
    if (!o) return false;
    uint32_t hdr[4];
    std::memcpy(hdr, "PLUT", 4);
    hdr[1] = 1;
    hdr[2] = kLutRes;
    hdr[3] = (uint32_t)lut.size();
    o.write(reinterpret_cast<const char*>(hdr), 16);
    o.write(reinterpret_cast<const char*>(lut.data()), (std::streamsize)(lut.size() * sizeof(float)));
    return o.good();
}

// ============================================================ primitives
namespace {
inline void cross3(const float a[3], const float b[3], float o[3])
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
inline float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
}  // namespace

// Plane ctor (code/Includes/Plane.h:11-16)
pcr_plane make_plane(const float o[3], const float u[3], const float v[3], int mat)
{
    pcr_plane p{};
    std::memcpy(p.origin, o, 12);
    std::memcpy(p.u, u, 12);
    std::memcpy(p.v, v, 12);
    float c[3];
    cross3(u, v, c);
    float m = std::sqrt(dot3(c, c));
    p.area = m;
    p.n[0] = c[0] / m; p.n[1] = c[1] / m; p.n[2] = c[2] / m;
    p.mat = mat;
    return p;
}

// Triangle ctors (code/Includes/Triangle.h:12-36)
pcr_triangle make_triangle(const float a[3], const float b[3], const float c[3], const float* n0, const float* n1,
                           const float* n2, int mat)
{
    pcr_triangle t{};
    std::memcpy(t.v0, a, 12);
    std::memcpy(t.v1, b, 12);
    std::memcpy(t.v2, c, 12);
    float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]}, x[3];
    cross3(e1, e2, x);
    float m = std::sqrt(dot3(x, x));
    t.flat_n[0] = x[0] / m; t.flat_n[1] = x[1] / m; t.flat_n[2] = x[2] / m;
    t.smooth = n0 ? 1 : 0;
    if (n0) {
        std::memcpy(t.n0, n0, 12);
        std::memcpy(t.n1, n1, 12);
        std::memcpy(t.n2, n2, 12);
    }
    t.mat = mat;
    return t;
}

// ============================================================ BVH build
namespace {
struct Box {
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void vert(const float* p)
    {
        for (int i = 0; i < 3; i++) {
            if (p[i] < mn[i]) mn[i] = p[i];
            if (p[i] > mx[i]) mx[i] = p[i];
        }
    }
    void tri(const pcr_triangle& t) { vert(t.v0); vert(t.v1); vert(t.v2); }
    void merge(const Box& o)
    {
        for (int i = 0; i < 3; i++) {
            if (o.mn[i] < mn[i]) mn[i] = o.mn[i];
            if (o.mx[i] > mx[i]) mx[i] = o.mx[i];
        }
    }
    float area() const
    {
        float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
        if (dx < 0 || dy < 0 || dz < 0) return 0.f;
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
};
inline float centroid(const pcr_triangle& t, int a) { return (t.v0[a] + t.v1[a] + t.v2[a]) * (1.f / 3.f); }
inline int bin_of(float c, float lo, float scale) { return std::clamp((int)((c - lo) * scale), 0, 15); }

// Runs fn(chunk, lo, hi) over [begin, end) split into `parts` ordered chunks
// on parallel threads.
template <typename F>
void parallel_chunks(int begin, int end, int parts, F&& fn)
{
    std::vector<std::thread> th;
    const int n = end - begin;
    for (int k = 0; k < parts; k++) {
        const int lo = begin + (int)((int64_t)n * k / parts), hi = begin + (int)((int64_t)n * (k + 1) / parts);
        th.emplace_back([&fn, k, lo, hi] { fn(k, lo, hi); });
    }
    for (auto& t : th) t.join();
}

// The reference's recursive binned-SAH build (code/Bvh/Bvh.cpp:122-325).
// Large ranges are processed by several host threads with the same result
// as the sequential build: boxes and bin boxes are merged by min / max and
// counts by addition, with chunks merged in range order (so even the choice
// among equal signed zeros matches); sibling subtrees of large nodes are
// built concurrently into their own node lists and spliced in depth-first
// order (parent, left subtree, right subtree) with their indices shifted.
// The two-cursor partition stays sequential per node.
constexpr int kParallelRange = 1 << 16;   // triangles for chunked passes / concurrent children

struct Builder {
    std::vector<pcr_triangle>& tris;
    std::vector<int32_t>* ids;
    std::vector<pcr_bvh_node>& nodes;
    int threads;   // threads this builder may use

    void swap_tri(int a, int b)
    {
        std::swap(tris[a], tris[b]);
        if (ids) std::swap((*ids)[a], (*ids)[b]);
    }

    int rec(int begin, int end)
    {
        int idx = (int)nodes.size();
        nodes.emplace_back();
        const int count = end - begin;
        const int parts = (count >= kParallelRange && threads > 1) ? threads : 1;
        Box box, cb;
        {
            std::vector<Box> pb(parts), pc(parts);
            parallel_or_inline(begin, end, parts, [&](int k, int lo, int hi) {
                for (int i = lo; i < hi; i++) {
                    pb[k].tri(tris[i]);
                    float c[3] = {centroid(tris[i], 0), centroid(tris[i], 1), centroid(tris[i], 2)};
                    pc[k].vert(c);
                }
            });
            for (int k = 0; k < parts; k++) { box.merge(pb[k]); cb.merge(pc[k]); }
        }
        for (int i = 0; i < 3; i++) { nodes[idx].bmin[i] = box.mn[i]; nodes[idx].bmax[i] = box.mx[i]; }
        auto leaf = [&] {
            nodes[idx].left_or_first = begin;
            nodes[idx].right_child = 0;
            nodes[idx].count = count;
            return idx;
        };
        if (count <= 4) return leaf();
        int best_axis = -1, best_bin = -1;
        float best_cost = FLT_MAX;
        const float parent = box.area();
        if (parent > 0.f) {
            for (int axis = 0; axis < 3; axis++) {
                float lo = cb.mn[axis], hi = cb.mx[axis], ext = hi - lo;
                if (ext < 1e-6f) continue;
                float scale = (float)16 / ext;
                std::vector<std::array<Box, 16>> pbins(parts);
                std::vector<std::array<int, 16>> pcnt(parts);
                for (auto& c : pcnt) c.fill(0);
                parallel_or_inline(begin, end, parts, [&](int k, int lo_i, int hi_i) {
                    for (int i = lo_i; i < hi_i; i++) {
                        int b = bin_of(centroid(tris[i], axis), lo, scale);
                        pbins[k][b].tri(tris[i]);
                        pcnt[k][b]++;
                    }
                });
                Box bins[16];
                int cnt[16] = {0};
                for (int k = 0; k < parts; k++)
                    for (int b = 0; b < 16; b++) { bins[b].merge(pbins[k][b]); cnt[b] += pcnt[k][b]; }
                float lSA[15], rSA[15];
                int lC[15], rC[15];
                Box acc;
                int ac = 0;
                for (int i = 0; i < 15; i++) { acc.merge(bins[i]); ac += cnt[i]; lSA[i] = acc.area(); lC[i] = ac; }
                acc = Box();
                ac = 0;
                for (int i = 15; i > 0; i--) { acc.merge(bins[i]); ac += cnt[i]; rSA[i - 1] = acc.area(); rC[i - 1] = ac; }
                for (int s = 0; s < 15; s++) {
                    if (lC[s] == 0 || rC[s] == 0) continue;
                    float cost = 1.f + 2.f * (lSA[s] * lC[s] + rSA[s] * rC[s]) / parent;
                    if (cost < best_cost) { best_cost = cost; best_axis = axis; best_bin = s; }
                }
            }
        }
        if (best_axis < 0 || best_cost >= (float)count * 2.f) return leaf();
        // std::partition as libstdc++ implements it for bidirectional
        // iterators (two cursors swapping misplaced elements)
        const float lo = cb.mn[best_axis], hi = cb.mx[best_axis];
        const float scale = (float)16 / (hi - lo);
        auto left = [&](int i) { return bin_of(centroid(tris[i], best_axis), lo, scale) <= best_bin; };
        int first = begin, last = end;
        for (;;) {
            for (;;) {
                if (first == last) goto done;
                if (left(first)) first++; else break;
            }
            last--;
            for (;;) {
                if (first == last) goto done;
                if (!left(last)) last--; else break;
            }
            swap_tri(first, last);
            first++;
        }
    done:
        const int mid = first;
        if (mid == begin || mid == end) return leaf();
        int l, r;
        if (threads > 1 && mid - begin >= kParallelRange / 2 && end - mid >= kParallelRange / 2) {
            // the two subtrees on their own threads, spliced depth-first
            std::vector<pcr_bvh_node> ln, rn;
            const int tl = std::max(1, threads / 2), tr = std::max(1, threads - tl);
            auto fut = std::async(std::launch::async, [&] {
                Builder sub{tris, ids, ln, tl};
                sub.rec(begin, mid);
            });
            Builder sub{tris, ids, rn, tr};
            sub.rec(mid, end);
            fut.get();
            const int bl = (int)nodes.size(), br = bl + (int)ln.size();
            for (auto& n : ln)
                if (n.count == 0) { n.left_or_first += bl; n.right_child += bl; }
            for (auto& n : rn)
                if (n.count == 0) { n.left_or_first += br; n.right_child += br; }
            nodes.insert(nodes.end(), ln.begin(), ln.end());
            nodes.insert(nodes.end(), rn.begin(), rn.end());
            l = bl;
            r = br;
        } else {
            l = rec(begin, mid);
            r = rec(mid, end);
        }
        nodes[idx].left_or_first = l;
        nodes[idx].right_child = r;
        nodes[idx].count = 0;
        return idx;
    }

    template <typename F>
    void parallel_or_inline(int begin, int end, int parts, F&& fn)
    {
        if (parts <= 1) fn(0, begin, end);
        else parallel_chunks(begin, end, parts, fn);
    }
};
}  // namespace

std::vector<pcr_bvh_node> build_bvh(std::vector<pcr_triangle>& tris, std::vector<int32_t>* ids)
{
    std::vector<pcr_bvh_node> nodes;
    if (tris.empty()) return nodes;
    nodes.reserve(2 * tris.size());
    const int threads = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
    Builder b{tris, ids, nodes, threads};
    b.rec(0, (int)tris.size());
    return nodes;
}

std::vector<DNode4> collapse_bvh4(const std::vector<pcr_bvh_node>& bvh, int n_tris)
{
    std::vector<DNode4> out;
    if (bvh.empty()) return out;
    auto area = [&](int i) {
        const pcr_bvh_node& n = bvh[i];
        float dx = n.bmax[0] - n.bmin[0], dy = n.bmax[1] - n.bmin[1], dz = n.bmax[2] - n.bmin[2];
        return dx * dy + dy * dz + dz * dx;
    };
    out.reserve(bvh.size() / 2 + 1);
    // depth-first preorder: a 4-wide node takes the next index when it is
    // reached, its internal children are visited in slot order
    struct Item { int b, parent, slot; };
    std::vector<Item> stack{{0, -1, 0}};
    while (!stack.empty()) {
        const Item it = stack.back();
        stack.pop_back();
        if (out.size() >= bvh.size()) throw PcrError(PCR_ERR_INVALID, "BVH is not a tree");
        const int me = (int)out.size();
        out.emplace_back();
        if (it.parent >= 0) reinterpret_cast<int*>(&out[it.parent].child)[it.slot] = me;
        int ch[4], nc = 0;
        if (bvh[it.b].count > 0) ch[nc++] = it.b;
        else { ch[nc++] = bvh[it.b].left_or_first; ch[nc++] = bvh[it.b].right_child; }
        while (nc < 4) {   // open the internal child with the largest area
            int pick = -1;
            float best = -1.f;
            for (int k = 0; k < nc; k++)
                if (bvh[ch[k]].count == 0 && area(ch[k]) > best) { best = area(ch[k]); pick = k; }
            if (pick < 0) break;
            const int c = ch[pick];
            for (int k = nc; k > pick + 1; k--) ch[k] = ch[k - 1];
            ch[pick] = bvh[c].left_or_first;
            ch[pick + 1] = bvh[c].right_child;
            nc++;
        }
        float lo[3][4], hi[3][4];
        // empty slots: the code of a leaf with no triangles
        const int empty = (int)0x80000000u;
        int code[4] = {empty, empty, empty, empty}, valid[4] = {0, 0, 0, 0};
        for (int k = 0; k < 4; k++)
            for (int a = 0; a < 3; a++) { lo[a][k] = 0.f; hi[a][k] = 0.f; }
        for (int k = 0; k < nc; k++) {
            const pcr_bvh_node& n = bvh[ch[k]];
            for (int a = 0; a < 3; a++) { lo[a][k] = n.bmin[a]; hi[a][k] = n.bmax[a]; }
            valid[k] = 1;
            if (n.count > 0) {
                if (n.count > 127) throw PcrError(PCR_ERR_INVALID, "BVH leaf with more than 127 triangles");
                if (n.left_or_first < 0 || n.left_or_first + n.count > n_tris || n.left_or_first >= (1 << 24))
                    throw PcrError(PCR_ERR_INVALID, "BVH leaf range out of bounds");
                code[k] = (int)(0x80000000u | ((uint32_t)n.count << 24) | (uint32_t)n.left_or_first);
            } else {
                code[k] = -1;   // set when the child is reached
            }
        }
        DNode4& N = out[me];
        N.lox = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
        N.hix = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
        N.loy = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
        N.hiy = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
        N.loz = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
        N.hiz = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
        N.child = make_int4(code[0], code[1], code[2], code[3]);
        N.valid = make_int4(valid[0], valid[1], valid[2], valid[3]);
        for (int k = nc - 1; k >= 0; k--)
            if (bvh[ch[k]].count == 0) stack.push_back({ch[k], me, k});
    }
    return out;
}

void parallel_for(int n, const std::function<void(int, int)>& fn)
{
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int parts = n < (1 << 16) ? 1 : std::min(16, hw);
    if (parts <= 1) {
        if (n > 0) fn(0, n);
        return;
    }
    parallel_chunks(0, n, parts, [&](int, int lo, int hi) { fn(lo, hi); });
}

// ============================================================ SPD / OBJ
namespace {
// SpdLoader::loadSpdFile + interp (code/SpdLoader.cpp:20-80)
std::vector<float> load_spd(const std::string& path)
{
    std::ifstream in(path);
    if (!in) throw PcrError(PCR_ERR_SCENE, "cannot open file: " + path);
    std::vector<std::pair<float, float>> pairs;
    std::string line;
    int ln = 0;
    while (std::getline(in, line)) {
        ln++;
        size_t s = 0;
        while (s < line.size() && (line[s] == ' ' || line[s] == '\t')) s++;
        if (s >= line.size() || line[s] == '#') continue;
        std::istringstream is(line.substr(s));
        float a, b;
        if (!(is >> a >> b)) throw PcrError(PCR_ERR_SCENE, path + ":" + std::to_string(ln) + ": expected 'wavelength value'");
        pairs.emplace_back(a, b);
    }
    if (pairs.empty()) throw PcrError(PCR_ERR_SCENE, "no data samples in " + path);
    for (size_t i = 1; i < pairs.size(); i++)
        if (pairs[i].first <= pairs[i - 1].first) throw PcrError(PCR_ERR_SCENE, path + ": wavelengths must be strictly ascending");
    std::vector<float> out(kSpecN);
    for (int i = 0; i < kSpecN; i++) {
        float l = lambda_at(i);
        if (l <= pairs.front().first) { out[i] = pairs.front().second; continue; }
        if (l >= pairs.back().first) { out[i] = pairs.back().second; continue; }
        auto hi = std::upper_bound(pairs.begin(), pairs.end(), std::make_pair(l, 0.f),
                                   [](const auto& a, const auto& b) { return a.first < b.first; });
        auto lo = hi - 1;
        float t = (l - lo->first) / (hi->first - lo->first);
        out[i] = lo->second + t * (hi->second - lo->second);
    }
    return out;
}

struct ObjData {
    std::vector<float> v, vn;
    std::vector<std::array<int, 6>> faces;  // v0 v1 v2 n0 n1 n2 (n = -1 when absent)
};

// strtod on the OBJ number fields: blanks (newline included, as strtod's
// isspace) are skipped, then std::from_chars reads the number (correctly
// rounded, as strtod); the rare forms from_chars does not take (hex,
// out-of-range values) go to strtod itself.  No number: 0, pointer unmoved.
inline double scan_double(const char*& q, const char* end)
{
    const char* s = q;
    while (s < end && (*s == ' ' || *s == '\t' || *s == '\r' || *s == '\n' || *s == '\v' || *s == '\f')) s++;
    const char* num = s;
    if (num < end && *num == '+') {
        num++;
        if (num < end && (*num == '+' || *num == '-')) return 0.0;
    }
    const bool hex = end - num >= 2 && num[0] == '0' && (num[1] == 'x' || num[1] == 'X');
    double v = 0.0;
    const auto r = hex ? std::from_chars_result{num, std::errc::invalid_argument} : std::from_chars(num, end, v);
    if (r.ec == std::errc()) {
        q = r.ptr;
        return v;
    }
    if (r.ec == std::errc::invalid_argument && !hex) return 0.0;
    char* e;
    v = std::strtod(q, &e);   // the buffer is NUL-terminated
    q = e;
    return v;
}

// atoi over one face token's characters
inline int scan_int(const char* s, const char* end)
{
    bool neg = false;
    if (s < end && (*s == '+' || *s == '-')) neg = *s++ == '-';
    long long v = 0;
    while (s < end && *s >= '0' && *s <= '9') v = v * 10 + (*s++ - '0');
    return (int)(neg ? -v : v);
}

struct ObjChunk {
    std::vector<std::array<int, 6>> faces;
    std::string error;   // first error in this chunk
};

// One contiguous range of lines; nv / nn = vertices / normals defined
// before it.  Vertices and normals go straight to their final positions.
void parse_obj_lines(const char* p, const char* end, int nv, int nn, float* v, float* vn, ObjChunk& out,
                     const std::string& path)
{
    std::vector<std::pair<int, int>> idx;
    while (p < end) {
        const char* eol = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
        if (!eol) eol = end;
        const size_t len = (size_t)(eol - p);
        if (len >= 2 && p[0] == 'v' && p[1] == ' ') {
            const char* q = p + 2;
            for (int k = 0; k < 3; k++) v[(size_t)nv * 3 + k] = (float)scan_double(q, end);
            nv++;
        } else if (len >= 3 && p[0] == 'v' && p[1] == 'n' && p[2] == ' ') {
            const char* q = p + 3;
            for (int k = 0; k < 3; k++) vn[(size_t)nn * 3 + k] = (float)scan_double(q, end);
            nn++;
        } else if (len >= 2 && p[0] == 'f' && p[1] == ' ') {
            idx.clear();
            const char* q = p + 2;
            while (q < eol) {
                while (q < eol && (*q == ' ' || *q == '\t' || *q == '\r')) q++;
                if (q >= eol) break;
                const char* t0 = q;   // one token: v, v/t, v//n or v/t/n
                while (q < eol && *q != ' ' && *q != '\t' && *q != '\r') q++;
                int vi = scan_int(t0, q), ni = 0;
                const char* s1 = static_cast<const char*>(std::memchr(t0, '/', (size_t)(q - t0)));
                if (s1) {
                    const char* s2 = static_cast<const char*>(std::memchr(s1 + 1, '/', (size_t)(q - s1 - 1)));
                    if (s2 && s2 + 1 < q) ni = scan_int(s2 + 1, q);
                }
                vi = vi > 0 ? vi - 1 : nv + vi;
                ni = ni > 0 ? ni - 1 : (ni < 0 ? nn + ni : -1);
                if (vi < 0 || vi >= nv) {
                    out.error = "Failed to parse OBJ " + path + ": vertex index out of range";
                    return;
                }
                idx.emplace_back(vi, ni);
            }
            for (size_t k = 1; k + 1 < idx.size(); k++)
                out.faces.push_back({idx[0].first, idx[k].first, idx[k + 1].first, idx[0].second, idx[k].second,
                                     idx[k + 1].second});
        }
        p = eol + 1;
    }
}

// Wavefront OBJ subset the reference's loader reads (v, vn, f with v,
// v/t, v//n, v/t/n tokens, fans of polygons).  The file is read by several
// threads at once and cut into ranges of whole lines; a first parallel pass counts the v / vn
// lines of each range, so the second (also parallel) pass knows how many
// vertices precede every line (relative indices, range checks) and where
// its vertices go.  Faces are concatenated in file order and the first
// error in file order is reported, as a sequential reader would.
ObjData load_obj(const std::string& path)
{
    const int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) throw PcrError(PCR_ERR_SCENE, "Mesh file not found: " + path);
    struct stat sb;
    if (::fstat(fd, &sb) != 0) {
        ::close(fd);
        throw PcrError(PCR_ERR_SCENE, "Failed to read OBJ " + path);
    }
    const size_t fsize = (size_t)std::max<off_t>(sb.st_size, 0);
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int parts = fsize < (1u << 20) ? 1 : std::min(64, 2 * hw);
    auto run = [&](int n, auto&& fn) {
        if (n == 1) { fn(0); return; }
        std::vector<std::thread> th;
        const int nt = std::min(n, hw);
        for (int t = 0; t < nt; t++)
            th.emplace_back([&, t] { for (int k = t; k < n; k += nt) fn(k); });
        for (auto& x : th) x.join();
    };
    // the file in `parts` ranges read concurrently, then a newline and a NUL
    std::unique_ptr<char[]> buf(new char[fsize + 2]);
    std::vector<int> read_ok(parts, 1);
    run(parts, [&](int k) {
        size_t o = fsize * (size_t)k / (size_t)parts;
        const size_t e = fsize * (size_t)(k + 1) / (size_t)parts;
        while (o < e) {
            const ssize_t r = ::pread(fd, buf.get() + o, e - o, (off_t)o);
            if (r <= 0) { read_ok[k] = 0; return; }
            o += (size_t)r;
        }
    });
    ::close(fd);
    for (int ok : read_ok)
        if (!ok) throw PcrError(PCR_ERR_SCENE, "Failed to read OBJ " + path);
    buf[fsize] = '\n';
    buf[fsize + 1] = '\0';
    const char* const b0 = buf.get();
    const char* const end = b0 + fsize + 1;
    const size_t bsize = fsize + 1;
    // range starts on line boundaries
    std::vector<const char*> cut(parts + 1, end);
    cut[0] = b0;
    for (int k = 1; k < parts; k++) {
        const char* t = b0 + bsize * (size_t)k / (size_t)parts;
        if (t < cut[k - 1]) t = cut[k - 1];
        const char* nl = static_cast<const char*>(std::memchr(t, '\n', (size_t)(end - t)));
        cut[k] = nl ? nl + 1 : end;
    }
    std::vector<int> cv(parts, 0), cn(parts, 0);
    auto count = [&](int k) {
        for (const char* p = cut[k]; p < cut[k + 1];) {
            const char* eol = static_cast<const char*>(std::memchr(p, '\n', (size_t)(cut[k + 1] - p)));
            if (!eol) eol = cut[k + 1];
            const size_t len = (size_t)(eol - p);
            if (len >= 2 && p[0] == 'v' && p[1] == ' ') cv[k]++;
            else if (len >= 3 && p[0] == 'v' && p[1] == 'n' && p[2] == ' ') cn[k]++;
            p = eol + 1;
        }
    };
    run(parts, count);
    std::vector<int> v0(parts + 1, 0), n0(parts + 1, 0);
    for (int k = 0; k < parts; k++) {
        v0[k + 1] = v0[k] + cv[k];
        n0[k + 1] = n0[k] + cn[k];
    }
    ObjData d;
    d.v.resize((size_t)v0[parts] * 3);
    d.vn.resize((size_t)n0[parts] * 3);
    std::vector<ObjChunk> ch(parts);
    run(parts, [&](int k) { parse_obj_lines(cut[k], cut[k + 1], v0[k], n0[k], d.v.data(), d.vn.data(), ch[k], path); });
    size_t nf = 0;
    for (const auto& c : ch) {
        if (!c.error.empty()) throw PcrError(PCR_ERR_SCENE, c.error);
        nf += c.faces.size();
    }
    d.faces.reserve(nf);
    for (const auto& c : ch) d.faces.insert(d.faces.end(), c.faces.begin(), c.faces.end());
    return d;
}

// MeshLoader rotateXYZ / transform (code/Scenes/MeshLoader.cpp:89-136)
void rotate_xyz(float v[3], const float rd[3])
{
    const float kPi = 3.14159265358979323846f;
    float rx = rd[0] * (kPi / 180.f), ry = rd[1] * (kPi / 180.f), rz = rd[2] * (kPi / 180.f);
    if (rx != 0.f) { float c = std::cos(rx), s = std::sin(rx); float y = v[1] * c - v[2] * s, z = v[1] * s + v[2] * c; v[1] = y; v[2] = z; }
    if (ry != 0.f) { float c = std::cos(ry), s = std::sin(ry); float x = v[0] * c + v[2] * s, z = -v[0] * s + v[2] * c; v[0] = x; v[2] = z; }
    if (rz != 0.f) { float c = std::cos(rz), s = std::sin(rz); float x = v[0] * c - v[1] * s, y = v[0] * s + v[1] * c; v[0] = x; v[1] = y; }
}

void vec3_of(const JVal* j, const std::string& what, float out[3])
{
    if (!j || j->kind != JVal::Arr || j->arr.size() != 3)
        throw PcrError(PCR_ERR_SCENE, what + ": expected [x, y, z] array of 3 numbers");
    for (int k = 0; k < 3; k++) {
        if (j->arr[k].kind != JVal::Num) throw PcrError(PCR_ERR_SCENE, what + ": expected numbers");
        out[k] = j->arr[k].as_float();
    }
}

std::string req_str(const JVal& p, const char* key, const std::string& where)
{
    const JVal* v = p.get(key);
    if (!v || v->kind != JVal::Str) throw PcrError(PCR_ERR_SCENE, where + " missing string \"" + key + "\"");
    return v->str;
}
}  // namespace

// ============================================================ scene assembly
HostScene load_scene_json(const std::string& path, const std::string& data_root, const std::vector<float>* lut,
                          bool with_bvh)
{
    const std::string text = read_file(path);
    JParser P(text, path);
    JVal j = P.value();
    if (j.kind != JVal::Obj) throw PcrError(PCR_ERR_SCENE, path + ": top level must be an object");
    const JVal* sch = j.get("schema");
    if (!sch) throw PcrError(PCR_ERR_SCENE, path + ": missing required \"schema\" field");
    if (sch->kind != JVal::Str) throw PcrError(PCR_ERR_SCENE, path + ": \"schema\" must be a string like \"1.0\"");
    int major = 0, minor = 0;
    if (std::sscanf(sch->str.c_str(), "%d.%d", &major, &minor) != 2)
        throw PcrError(PCR_ERR_SCENE, path + ": malformed schema \"" + sch->str + "\" (expected major.minor)");
    if (major != 1)
        throw PcrError(PCR_ERR_SCENE, path + ": schema major version " + std::to_string(major) + " is not supported by this binary (expected 1.x)");
    HostScene S;
    S.name = req_str(j, "name", path + ": (root)");
    S.version = req_str(j, "version", path + ": (root)");
    if (const JVal* cam = j.get("camera")) {
        if (cam->kind != JVal::Obj) throw PcrError(PCR_ERR_SCENE, path + ": \"camera\" must be an object");
        if (const JVal* p = cam->get("position")) vec3_of(p, "camera.position", S.cam);
        if (const JVal* f = cam->get("fov")) {
            if (f->kind != JVal::Num) throw PcrError(PCR_ERR_SCENE, path + ": camera.fov must be a number");
            S.fov = f->as_float();
        }
    }
    const std::string root = data_root.empty() ? std::string(".") : data_root;
    std::map<std::string, int> name_to_idx;
    const JVal* mats = j.get("materials");
    if (!mats || mats->kind != JVal::Obj) throw PcrError(PCR_ERR_SCENE, path + ": missing or non-object \"materials\" map");
    for (const auto& kv : mats->obj) {
        const std::string& name = kv.first;
        const JVal& m = kv.second;
        if (m.kind != JVal::Obj) throw PcrError(PCR_ERR_SCENE, path + ": material \"" + name + "\" must be an object");
        pcr_material M{};
        M.ior = 1.5f;
        if (const JVal* a = m.get("albedo")) vec3_of(a, "materials." + name + ".albedo", M.albedo);
        if (const JVal* e = m.get("emissive")) vec3_of(e, "materials." + name + ".emissive", M.emissive);
        if (const JVal* s = m.get("albedo_spd")) {
            if (s->kind != JVal::Str) throw PcrError(PCR_ERR_SCENE, path + ": materials." + name + ".albedo_spd must be a string");
            auto tab = load_spd(root + "/spd/" + s->str + ".spd");
            std::copy(tab.begin(), tab.end(), M.tab_albedo);
            M.use_tab_albedo = 1;
            if (!m.get("albedo")) {
                float xyz[3], rgb[3];
                spectrum_to_xyz(M.tab_albedo, xyz);
                xyz_to_srgb(xyz, rgb);
                for (int k = 0; k < 3; k++) M.albedo[k] = std::max(0.f, rgb[k]);
            }
        }
        if (const JVal* s = m.get("emissive_spd")) {
            if (s->kind != JVal::Str) throw PcrError(PCR_ERR_SCENE, path + ": materials." + name + ".emissive_spd must be a string");
            auto tab = load_spd(root + "/spd/" + s->str + ".spd");
            if (const JVal* c = m.get("emissive_scale")) {
                if (c->kind != JVal::Num) throw PcrError(PCR_ERR_SCENE, path + ": materials." + name + ".emissive_scale must be a number");
                float sc = c->as_float();
                for (auto& x : tab) x *= sc;
            }
            std::copy(tab.begin(), tab.end(), M.tab_emissive);
            M.use_tab_emissive = 1;
            if (!m.get("emissive")) {
                float xyz[3], rgb[3];
                spectrum_to_xyz(M.tab_emissive, xyz);
                xyz_to_srgb(xyz, rgb);
                for (int k = 0; k < 3; k++) M.emissive[k] = std::max(0.f, rgb[k]);
            }
        }
        auto flag = [&](const char* key, int32_t& out) {
            if (const JVal* f = m.get(key)) {
                if (f->kind != JVal::Bool) throw PcrError(PCR_ERR_SCENE, path + ": materials." + name + "." + key + " must be a boolean");
                out = f->b ? 1 : 0;
            }
        };
        flag("metallic", M.metallic);
        flag("transparent", M.transparent);
        auto num = [&](const char* key, float& out) {
            if (const JVal* f = m.get(key)) {
                if (f->kind != JVal::Num) throw PcrError(PCR_ERR_SCENE, path + ": materials." + name + "." + key + " must be a number");
                out = f->as_float();
            }
        };
        num("ior", M.ior);
        num("cauchyB", M.cauchy_b);
        if (M.metallic && M.transparent)
            throw PcrError(PCR_ERR_SCENE, path + ": materials." + name + " cannot be both metallic and transparent");
        name_to_idx[name] = (int)S.materials.size();
        S.materials.push_back(M);
    }
    if (S.materials.empty()) throw PcrError(PCR_ERR_SCENE, path + ": \"materials\" map is empty");
    auto mat_of = [&](const JVal& p, const std::string& where) {
        std::string ref = req_str(p, "material", path + ": " + where);
        auto it = name_to_idx.find(ref);
        if (it == name_to_idx.end()) throw PcrError(PCR_ERR_SCENE, path + ": " + where + ".material references unknown material \"" + ref + "\"");
        return it->second;
    };

    const JVal* prims = j.get("primitives");
    if (!prims || prims->kind != JVal::Arr) throw PcrError(PCR_ERR_SCENE, path + ": missing or non-array \"primitives\"");
    std::vector<pcr_plane> walls, light_planes;
    std::vector<std::vector<pcr_triangle>> tri_lights;
    std::vector<int> light_kind;  // order of lights: 0 plane (index into light_planes), 1 tri set
    std::vector<int> light_ref;
    const std::string scene_dir = path.find('/') == std::string::npos ? "." : path.substr(0, path.rfind('/'));
    for (size_t i = 0; i < prims->arr.size(); i++) {
        const JVal& p = prims->arr[i];
        const std::string where = "primitives[" + std::to_string(i) + "]";
        if (p.kind != JVal::Obj) throw PcrError(PCR_ERR_SCENE, path + ": " + where + " must be an object");
        const std::string type = req_str(p, "type", path + ": " + where);
        const JVal* lf = p.get("light");
        const bool is_light = lf && lf->kind == JVal::Bool && lf->b;
        if (type == "sphere") {
            if (is_light) throw PcrError(PCR_ERR_SCENE, path + ": " + where + ": light flag is only valid on plane, triangle, or mesh primitives");
            pcr_sphere s{};
            vec3_of(p.get("center"), where + ".center", s.center);
            const JVal* r = p.get("radius");
            if (!r || r->kind != JVal::Num) throw PcrError(PCR_ERR_SCENE, path + ": " + where + " sphere needs center [x,y,z] and numeric radius");
            s.radius = r->as_float();
            s.mat = mat_of(p, where);
            S.spheres.push_back(s);
        } else if (type == "plane") {
            float o[3], u[3], v[3];
            vec3_of(p.get("origin"), where + ".origin", o);
            vec3_of(p.get("u"), where + ".u", u);
            vec3_of(p.get("v"), where + ".v", v);
            pcr_plane pl = make_plane(o, u, v, mat_of(p, where));
            if (is_light) { light_kind.push_back(0); light_ref.push_back((int)light_planes.size()); light_planes.push_back(pl); }
            else walls.push_back(pl);
        } else if (type == "triangle") {
            float a[3], b[3], c[3];
            vec3_of(p.get("v0"), where + ".v0", a);
            vec3_of(p.get("v1"), where + ".v1", b);
            vec3_of(p.get("v2"), where + ".v2", c);
            int mi = mat_of(p, where);
            int nn = (p.get("n0") ? 1 : 0) + (p.get("n1") ? 1 : 0) + (p.get("n2") ? 1 : 0);
            pcr_triangle t;
            if (nn == 0) t = make_triangle(a, b, c, nullptr, nullptr, nullptr, mi);
            else if (nn != 3) throw PcrError(PCR_ERR_SCENE, path + ": " + where + " triangle normals require all of n0, n1, n2 or none");
            else {
                float n0[3], n1[3], n2[3];
                vec3_of(p.get("n0"), where + ".n0", n0);
                vec3_of(p.get("n1"), where + ".n1", n1);
                vec3_of(p.get("n2"), where + ".n2", n2);
                t = make_triangle(a, b, c, n0, n1, n2, mi);
            }
            if (is_light) { light_kind.push_back(1); light_ref.push_back((int)tri_lights.size()); tri_lights.push_back({t}); }
            S.triangles.push_back(t);
        } else if (type == "mesh") {
            const std::string file = req_str(p, "file", path + ": " + where);
            float pos[3] = {0, 0, 0}, rot[3] = {0, 0, 0}, sc[3] = {1, 1, 1};
            if (const JVal* v = p.get("position")) vec3_of(v, where + ".position", pos);
            if (const JVal* v = p.get("rotation")) vec3_of(v, where + ".rotation", rot);
            if (const JVal* v = p.get("scale")) {
                if (v->kind == JVal::Num) sc[0] = sc[1] = sc[2] = v->as_float();
                else vec3_of(v, where + ".scale", sc);
            }
            bool smooth = true;
            if (const JVal* v = p.get("smooth")) {
                if (v->kind != JVal::Bool) throw PcrError(PCR_ERR_SCENE, path + ": " + where + ".smooth must be a boolean");
                smooth = v->b;
            }
            int mi;
            if (const JVal* m = p.get("material"); m && m->kind == JVal::Str) {
                auto it = name_to_idx.find(m->str);
                if (it == name_to_idx.end()) throw PcrError(PCR_ERR_SCENE, "Mesh material override '" + m->str + "' not in registry");
                mi = it->second;
            } else {
                auto it = name_to_idx.find("__pcr_mesh_fallback_grey");
                if (it == name_to_idx.end()) {
                    pcr_material fb{};
                    fb.albedo[0] = fb.albedo[1] = fb.albedo[2] = 0.7f;
                    fb.ior = 1.5f;
                    mi = (int)S.materials.size();
                    name_to_idx["__pcr_mesh_fallback_grey"] = mi;
                    S.materials.push_back(fb);
                } else {
                    mi = it->second;
                }
            }
            ObjData od = load_obj(scene_dir + "/" + file);
            const int nv = (int)od.v.size() / 3, nn = (int)od.vn.size() / 3, nf = (int)od.faces.size();
            for (const auto& f : od.faces)
                for (int k = 3; k < 6; k++)
                    if (f[k] >= nn) throw PcrError(PCR_ERR_SCENE, "Failed to parse OBJ " + file + ": normal index out of range");
            // per-vertex, per-normal and per-face work is independent: split
            // over host threads (same arithmetic per element)
            const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
            auto par = [&](int n, auto&& fn) {
                const int parts = n < (1 << 16) ? 1 : std::min(16, hw);
                if (parts == 1) fn(0, 0, n);
                else parallel_chunks(0, n, parts, fn);
            };
            std::vector<float> tv(od.v.size()), tn(od.vn.size());
            par(nv, [&](int, int lo, int hi) {
                for (int k = lo; k < hi; k++) {
                    float v[3] = {od.v[k * 3] * sc[0], od.v[k * 3 + 1] * sc[1], od.v[k * 3 + 2] * sc[2]};
                    rotate_xyz(v, rot);
                    tv[k * 3] = v[0] + pos[0]; tv[k * 3 + 1] = v[1] + pos[1]; tv[k * 3 + 2] = v[2] + pos[2];
                }
            });
            par(nn, [&](int, int lo, int hi) {
                for (int k = lo; k < hi; k++) {
                    float v[3] = {od.vn[k * 3], od.vn[k * 3 + 1], od.vn[k * 3 + 2]};
                    rotate_xyz(v, rot);
                    float m = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                    tn[k * 3] = v[0] / m; tn[k * 3 + 1] = v[1] / m; tn[k * 3 + 2] = v[2] / m;
                }
            });
            const size_t begin = S.triangles.size();
            S.triangles.resize(begin + (size_t)nf);
            par(nf, [&](int, int lo, int hi) {
                for (int k = lo; k < hi; k++) {
                    const auto& f = od.faces[k];
                    const bool have_n = f[3] >= 0 && f[4] >= 0 && f[5] >= 0 && smooth;
                    S.triangles[begin + k] =
                        have_n ? make_triangle(&tv[f[0] * 3], &tv[f[1] * 3], &tv[f[2] * 3], &tn[f[3] * 3], &tn[f[4] * 3],
                                               &tn[f[5] * 3], mi)
                               : make_triangle(&tv[f[0] * 3], &tv[f[1] * 3], &tv[f[2] * 3], nullptr, nullptr, nullptr, mi);
                }
            });
            if (is_light) {
                light_kind.push_back(1);
                light_ref.push_back((int)tri_lights.size());
                tri_lights.emplace_back(S.triangles.begin() + begin, S.triangles.end());
            }
        } else {
            throw PcrError(PCR_ERR_SCENE, path + ": " + where + ": unknown primitive type \"" + type + "\" (expected sphere, plane, triangle, or mesh)");
        }
    }
    if (light_kind.empty()) throw PcrError(PCR_ERR_SCENE, path + ": at least one primitive must have \"light\": true; found none");
    // lights in declaration order; renderer planes: light planes then walls
    for (size_t k = 0; k < light_kind.size(); k++) {
        pcr_light L{};
        L.kind = light_kind[k];
        if (L.kind == 0) {
            L.plane = light_planes[light_ref[k]];
            L.total_area = L.plane.area;
        } else {
            const auto& tl = tri_lights[light_ref[k]];
            L.tri_offset = (int)S.light_tris.size();
            L.tri_count = (int)tl.size();
            float acc = 0.f;
            for (const auto& t : tl) {
                float e1[3] = {t.v1[0] - t.v0[0], t.v1[1] - t.v0[1], t.v1[2] - t.v0[2]};
                float e2[3] = {t.v2[0] - t.v0[0], t.v2[1] - t.v0[1], t.v2[2] - t.v0[2]}, c[3];
                cross3(e1, e2, c);
                acc += 0.5f * std::sqrt(dot3(c, c));
                S.light_cum.push_back(acc);
                S.light_tris.push_back(t);
            }
            L.total_area = acc;
        }
        S.lights.push_back(L);
    }
    S.planes = light_planes;
    S.planes.insert(S.planes.end(), walls.begin(), walls.end());
    S.triangle_ids.resize(S.triangles.size());
    for (size_t i = 0; i < S.triangles.size(); i++) S.triangle_ids[i] = (int32_t)i;
    if (with_bvh) S.bvh = build_bvh(S.triangles, &S.triangle_ids);
    for (auto& m : S.materials) populate_material(m, lut);
    return S;
}

pcr_scene_desc HostScene::desc() const
{
    pcr_scene_desc d{};
    d.name = name.c_str();
    d.version = version.c_str();
    std::memcpy(d.cam_pos, cam, sizeof(cam));
    d.fov = fov;
    d.n_materials = (int32_t)materials.size();
    d.materials = materials.data();
    d.n_spheres = (int32_t)spheres.size();
    d.spheres = spheres.data();
    d.n_planes = (int32_t)planes.size();
    d.planes = planes.data();
    d.n_triangles = (int32_t)triangles.size();
    d.triangles = triangles.data();
    d.n_bvh_nodes = (int32_t)bvh.size();
    d.bvh_nodes = bvh.data();
    d.n_lights = (int32_t)lights.size();
    d.lights = lights.data();
    d.light_triangles = light_tris.data();
    d.light_cum_area = light_cum.data();
    d.triangle_ids = triangle_ids.data();
    return d;
}

}  // namespace pcr
