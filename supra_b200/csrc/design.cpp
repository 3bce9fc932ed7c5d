// Host-side design helpers of the product library. The arithmetic (types and order of every
// operation) follows SUPRA's host code so that LUTs, filter taps and scan-conversion tables are
// bit-identical to what the reference computes; compiled with -ffp-contract=off.
#include "design.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace sb {

namespace {

// Window formula, Beamformer/WindowFunction.h:121-138, evaluated in float.
float windowFormula(int type, float r, float p) {
    const float twoPi = 2 * static_cast<float>(M_PI);
    if (type == SB_WINDOW_RECTANGULAR) return 1.0f;
    if (type == SB_WINDOW_HANN) return (1 - p) * (0.5f - 0.5f * std::cos(twoPi * ((r + 1) * 0.5f))) + p;
    if (type == SB_WINDOW_HAMMING) return (1 - p) * (0.54f - 0.46f * std::cos(twoPi * ((r + 1) * 0.5f))) + p;
    if (type == SB_WINDOW_GAUSS)
        return static_cast<float>(1.0 / (p * std::sqrt(2.0 * M_PI)) * std::exp((-1.0 / 2.0) * (r / p) * (r / p)));
    return 0;
}

// Modified Bessel function of the first kind, order 0: the 9-term series FirFilterFactory uses
// (SupraLib/utilities/FirFilterFactory.h:216-228), templated on the evaluation type.
template <typename T> T besselI0(T x) {
    static const int fact[9] = {1, 2, 6, 24, 120, 720, 5040, 40320, 362880};
    T acc = 0.0;
    for (int k = 1; k < 10; k++) {
        T xp = std::pow(x / static_cast<T>(2.0), static_cast<T>(k));
        acc += std::pow(xp / static_cast<T>(fact[k - 1]), static_cast<T>(2.0));
    }
    return static_cast<T>(1.0) + acc;
}

}  // namespace

std::vector<float> windowLut(int type, float param, size_t n) {
    std::vector<float> lut(n);
    float peak = std::numeric_limits<float>::min();
    for (size_t i = 0; i < n; i++) {
        lut[i] = windowFormula(type, (static_cast<float>(i) / (n - 1)) * 2 - 1, param);
        peak = std::max(peak, lut[i]);
    }
    for (float& v : lut) v /= peak;
    return lut;
}

std::vector<float> firDesign(size_t length, int type, int window, double fs, double frequency, double bandwidth) {
    const float w0 = static_cast<float>(2 * M_PI * frequency / fs);
    const float wb = static_cast<float>(2 * M_PI * bandwidth / fs);
    const int mid = (static_cast<int>(length) - 1) / 2;
    std::vector<float> taps(length);
    for (int n = 0; n < static_cast<int>(length); n++) {
        const int k = n - mid;
        float h;
        if (type == 3) {  // Hilbert transformer: 2/(pi k) on odd k
            h = (k % 2 == 0) ? 0.0f : static_cast<float>(2.0 / (M_PI * k));
        } else if (type == 1) {  // high-pass
            h = (n == mid) ? static_cast<float>(1 - w0 / M_PI)
                           : static_cast<float>(-w0 / M_PI * std::sin(w0 * k) / (w0 * k));
        } else if (type == 2) {  // band-pass; the modulating cosine's phase is (w0 n - mid) as in the reference
            h = (n == mid) ? static_cast<float>(2.0 * wb / M_PI)
                           : static_cast<float>(2.0 * std::cos(w0 * n - mid) * wb / M_PI * std::sin(wb * k) / (wb * k));
        } else {  // low-pass
            h = (n == mid) ? static_cast<float>(w0 / M_PI) : static_cast<float>(w0 / M_PI * std::sin(w0 * k) / (w0 * k));
        }
        taps[n] = h;
    }
    const size_t maxN = length - 1;
    const float beta = 4.0f;
    for (int n = 0; n < static_cast<int>(length); n++) {
        float w = 1.0f;
        if (window == 1) w = static_cast<float>(0.50 - 0.50 * std::cos(2 * M_PI * n / maxN));
        else if (window == 2) w = static_cast<float>(0.54 - 0.46 * std::cos(2 * M_PI * n / maxN));
        else if (window == 3) {
            double arg = beta * std::sqrt(1.0 - std::pow(2 * (static_cast<float>(n) - maxN / 2) / maxN, 2.0));
            w = static_cast<float>(besselI0<double>(arg) / besselI0<float>(beta));
        }
        taps[n] *= w;
    }
    if (type == 2) {  // unit gain at the centre frequency
        float re = 0, im = 0;
        for (int k = 0; k < static_cast<int>(length); k++) {
            re += taps[k] * std::cos(w0 * static_cast<float>(k));
            im += taps[k] * std::sin(w0 * static_cast<float>(k));
        }
        const float g = std::sqrt(re * re + im * im);
        for (float& v : taps) v /= g;
    }
    return taps;
}

// ---------------------------------------------------------------------------------- scan tables
namespace {

struct D3 {
    double x, y, z;
};
inline D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 scale(double s, D3 a) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double len3(D3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

D3 slerp(D3 a, D3 b, double t) {  // great-circle interpolation of unit directions (SupraLib/vec.h:424-445)
    const double eps = 2.2204e-16;
    double om = std::acos(dot3(a, b));
    if (om < eps || t < eps) return a;
    if (1.0 - t < eps) return b;
    return add(scale(std::sin((1.0 - t) * om) / std::sin(om), a), scale(std::sin(t * om) / std::sin(om), b));
}

// Perpendicular from x onto the line (p, dir).
inline D3 perpendicular(D3 p, D3 dir, D3 x) {
    D3 v = sub(x, p);
    return sub(v, scale(dot3(dir, v), dir));
}

inline D3 origin(const sb_scanline_rx& s) { return {s.position[0], s.position[1], s.position[2]}; }
inline D3 heading(const sb_scanline_rx& s) { return {s.direction[0], s.direction[1], s.direction[2]}; }
inline D3 at(const sb_scanline_rx& s, double depth) { return add(origin(s), scale(depth, heading(s))); }

// Scanline parameter (t between line a and line b, distance d along it) of a point, found by the
// reference's iterative bracketing (Beamformer/ScanConverter.cu:840-894; <= 1000 steps, 1e-5 mm).
void locate2D(D3 a, D3 b, D3 da, D3 db, D3 x, double& tOut, double& dOut) {
    double tLo = 0, tHi = 1;
    D3 cLo = perpendicular(a, da, x), cHi = perpendicular(b, db, x);
    double dLo = len3(cLo), dHi = len3(cHi);
    if (cHi.x == 0 && cHi.y == 0 && cHi.z == 0) { tOut = tHi; dOut = len3(sub(x, b)); return; }
    if (cLo.x == 0 && cLo.y == 0 && cLo.z == 0) { tOut = tLo; dOut = len3(sub(x, a)); return; }
    double gap = 1e10;
    double t = (tHi - tLo) / 2 + tLo;
    D3 base{0, 0, 0};
    for (size_t it = 0; it < 1000 && gap > 1e-5; it++) {
        t = (1 - dHi / (dHi + dLo)) * tHi + (1 - dLo / (dHi + dLo)) * tLo;
        base = add(scale(1 - t, a), scale(t, b));
        D3 c = perpendicular(base, slerp(da, db, t), x);
        gap = len3(c);
        if (dot3(cLo, c) < 0) { tHi = t; cHi = c; dHi = gap; }
        else { tLo = t; cLo = c; dLo = gap; }
    }
    tOut = t;
    dOut = len3(sub(x, base));
}

inline double edge(double ax, double ay, double bx, double by, double px, double py) {
    return (bx - ax) * (py - ay) - (by - ay) * (px - ax);
}
inline bool inTriangle(double ax, double ay, double bx, double by, double cx, double cy, double px, double py) {
    return edge(bx, by, cx, cy, px, py) >= 0 && edge(cx, cy, ax, ay, px, py) >= 0 && edge(ax, ay, bx, by, px, py) >= 0;
}

}  // namespace

void scanGeometry(const sb_scanline_rx* lines, uint32_t lx, uint32_t ly, double depth, double resolution,
                  ScanTables& t) {
    const double big = std::numeric_limits<double>::max();
    double mn[3] = {big, big, big}, mx[3] = {-big, -big, -big};
    for (uint32_t y = 0; y < ly; y++)
        for (uint32_t x = 0; x < lx; x++)
            for (double dd : {0.0, depth}) {
                D3 p = at(lines[x + y * lx], dd);
                double v[3] = {p.x, p.y, p.z};
                for (int i = 0; i < 3; i++) {
                    mn[i] = std::min(mn[i], v[i]);
                    mx[i] = std::max(mx[i], v[i]);
                }
            }
    for (int i = 0; i < 3; i++) {
        t.bbMin[i] = mn[i];
        size_t n = static_cast<size_t>(std::ceil((mx[i] - mn[i]) / resolution)) + 1;
        t.size[i] = static_cast<uint32_t>(std::max(n, size_t(1)));
    }
}

void scanTables2D(const sb_scanline_rx* lines, uint32_t lx, uint32_t ly, uint32_t numSamples, double depth,
                  double resolution, ScanTables& t) {
    scanGeometry(lines, lx, ly, depth, resolution, t);
    const size_t W = t.size[0], H = t.size[1];
    const size_t n = W * H * t.size[2];
    t.mask.assign(n, 0);
    t.sampleIdx.assign(n, 0);
    t.weightX.assign(n, 0.0f);
    t.weightY.assign(n, 0.0f);
    t.weightZ.assign(n, 0.0f);
    const double step = depth / (numSamples - 1);
    const uint32_t nLines = lx * ly;
    const double ox = t.bbMin[0], oy = t.bbMin[1];
    // Quads in increasing order; a pixel on an edge shared by two quads keeps the later quad's values.
    for (uint32_t y = 0; y < ly; y++) {
        for (uint32_t x = 0; x + 1 < lx; x++) {
            const sb_scanline_rx& L0 = lines[x + y * lx];
            const sb_scanline_rx& L1 = lines[x + 1 + y * lx];
            D3 s0 = at(L0, 0.0), s1 = at(L1, 0.0), e0 = at(L0, depth), e1 = at(L1, depth);
            double loX = std::min(std::min(std::min(s0.x, s1.x), e0.x), e1.x);
            double loY = std::min(std::min(std::min(s0.y, s1.y), e0.y), e1.y);
            double hiX = std::max(std::max(std::max(s0.x, s1.x), e0.x), e1.x);
            double hiY = std::max(std::max(std::max(s0.y, s1.y), e0.y), e1.y);
            size_t px0 = static_cast<size_t>(std::floor((loX - ox) / resolution));
            size_t py0 = static_cast<size_t>(std::floor((loY - oy) / resolution));
            size_t px1 = static_cast<size_t>(std::ceil((hiX - ox) / resolution));
            size_t py1 = static_cast<size_t>(std::ceil((hiY - oy) / resolution));
            for (size_t px = px0; px <= px1; px++) {
                for (size_t py = py0; py <= py1; py++) {
                    double qx = static_cast<double>(px) * resolution + ox;
                    double qy = static_cast<double>(py) * resolution + oy;
                    bool inside = inTriangle(e1.x, e1.y, e0.x, e0.y, s0.x, s0.y, qx, qy) ||
                                  inTriangle(s0.x, s0.y, s1.x, s1.y, e1.x, e1.y, qx, qy);
                    if (!inside || px >= W || py >= H) continue;
                    double tt, dd;
                    locate2D(origin(L0), origin(L1), heading(L0), heading(L1), D3{qx, qy, 0.0}, tt, dd);
                    const size_t i = px + py * W;
                    uint32_t row = static_cast<uint32_t>(std::floor(dd / step));
                    t.mask[i] = 1;
                    t.sampleIdx[i] = static_cast<uint32_t>(row * nLines + x + y * lx);
                    t.weightX[i] = static_cast<float>(tt);
                    t.weightY[i] = static_cast<float>(dd - (row * step));  // in mm, as the reference stores it
                }
            }
        }
    }
}

}  // namespace sb
