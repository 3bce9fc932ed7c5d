// ================================================================================================
// supra_b200 ORACLE (part 2) — test infrastructure only: scan conversion tables and gathers,
// minimum-variance beamforming, adjoint DAS reference gradient. See supra_oracle.cpp for the rules.
// ================================================================================================
#include "supra_b200.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace {

constexpr double kEps = 2.2204e-16;          // M_EPS, SL/utilities/utility.h:43
constexpr int kMaxIter = 1000;               // ScanConverter::m_mappingMaxIterations, BF/ScanConverter.h:30
constexpr double kDistThreshold = 1e-5;      // ScanConverter::m_mappingDistanceThreshold, BF/ScanConverter.h:31
constexpr double kTetThreshold = 1e-9;       // ScanConverterInternals::m_tetrahedronTestDistanceThreshold, BF/ScanConverter.cu:45

// ------------------------------------------------------------------ small vector algebra (SL/vec.h)
template <typename T> struct V3 { T x, y, z; };
template <typename T> struct V2 { T x, y; };
template <typename T> V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> V3<T> operator*(T s, V3<T> a) { return {a.x * s, a.y * s, a.z * s}; }   // vec.h:316
template <typename T> V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <typename T> T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }  // vec.h:361
template <typename T> T norm(V3<T> a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }  // vec.h:349
template <typename T> V3<T> normalize(V3<T> a) { return a / norm(a); }
template <typename T> V3<T> cross(V3<T> a, V3<T> b) {  // vec.h:367
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// slerp3, SL/vec.h:424-445
template <typename T> V3<T> slerp3(V3<T> a, V3<T> b, T t) {
    T omega = std::acos(dot(a, b));
    if (omega < kEps) return a;
    if (t < kEps) return a;
    if (static_cast<T>(1.0) - t < kEps) return b;
    return (std::sin((static_cast<T>(1.0) - t) * omega) / std::sin(omega)) * a + (std::sin(t * omega) / std::sin(omega)) * b;
}

V3<double> pointOf(const sb_scanline_rx& s, double depth) {  // ScanlineRxParameters3D::getPoint, SL/USImageProperties.h:73-76
    V3<double> p{s.position[0], s.position[1], s.position[2]};
    V3<double> d{s.direction[0], s.direction[1], s.direction[2]};
    return p + depth * d;
}
V3<double> posOf(const sb_scanline_rx& s) { return {s.position[0], s.position[1], s.position[2]}; }
V3<double> dirOf(const sb_scanline_rx& s) { return {s.direction[0], s.direction[1], s.direction[2]}; }

// ------------------------------------------------------------------------- 2D helpers (double)
double bary2(V2<double> a, V2<double> b, V2<double> c) {  // ScanConverter::barycentricCoordinate2D, BF/ScanConverter.cu:818-821
    return (b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x);
}
bool insideTriangle(V2<double> a, V2<double> b, V2<double> c, V2<double> p) {  // :823-831
    double w0 = bary2(b, c, p), w1 = bary2(c, a, p), w2 = bary2(a, b, p);
    return w0 >= 0 && w1 >= 0 && w2 >= 0;
}
V3<double> pointLineConnection(V3<double> a, V3<double> da, V3<double> x) {  // :833-838
    V3<double> conn = x - a;
    return conn - dot(da, conn) * da;
}
// ScanConverter::mapToParameters2D, BF/ScanConverter.cu:840-894
V2<double> mapToParameters2D(V3<double> a, V3<double> b, V3<double> da, V3<double> db, V3<double> x) {
    double lowT = 0, highT = 1;
    V3<double> lowConn = pointLineConnection(a, da, x);
    V3<double> highConn = pointLineConnection(b, db, x);
    double lowDist = norm(lowConn), highDist = norm(highConn);
    if (highConn.x == 0 && highConn.y == 0 && highConn.z == 0) return {highT, norm(x - b)};
    if (lowConn.x == 0 && lowConn.y == 0 && lowConn.z == 0) return {lowT, norm(x - a)};
    double dist = 1e10;
    double t = (highT - lowT) / 2 + lowT;
    V3<double> lineBase{0, 0, 0};
    for (size_t it = 0; it < static_cast<size_t>(kMaxIter) && dist > kDistThreshold; it++) {
        t = (1 - highDist / (highDist + lowDist)) * highT + (1 - lowDist / (highDist + lowDist)) * lowT;
        lineBase = (1 - t) * a + t * b;
        V3<double> lineDir = slerp3(da, db, t);
        V3<double> conn = pointLineConnection(lineBase, lineDir, x);
        dist = norm(conn);
        if (dot(lowConn, conn) < 0) { highT = t; highConn = conn; highDist = dist; }
        else { lowT = t; lowConn = conn; lowDist = dist; }
    }
    return {t, norm(x - lineBase)};
}

// ------------------------------------------------------------------------- 3D helpers (float)
float bary3(V3<float> a, V3<float> b, V3<float> c, V3<float> p) {  // BF/ScanConverter.cu:149-174
    const float axby = a.x * b.y, cypz = c.y * p.z, axbz = a.x * b.z, czpy = c.z * p.y;
    const float aybx = a.y * b.x, cxpz = c.x * p.z, aybz = a.y * b.z, czpx = c.z * p.x;
    const float azbx = a.z * b.x, cxpy = c.x * p.y, azby = a.z * b.y, cypx = c.y * p.x;
    return (axby - aybx) * (c.z - p.z) + (aybz - azby) * (c.x - p.x) + (azbx - axbz) * (c.y - p.y) +
           (cypz - czpy) * (a.x - b.x) - (cxpz - czpx) * (a.y - b.y) + (cxpy - cypx) * (a.z - b.z);
}
bool insideTet(V3<float> a, V3<float> b, V3<float> c, V3<float> d, V3<float> p) {  // :131-146
    float w0 = bary3(a, b, c, d), w1 = bary3(p, b, c, d), w2 = bary3(a, p, c, d), w3 = bary3(a, b, p, d),
          w4 = bary3(a, b, c, p);
    return w0 > 0 && w1 >= -kTetThreshold && w2 >= -kTetThreshold && w3 >= -kTetThreshold && w4 >= -kTetThreshold;
}
V3<float> pointPlaneConnection(V3<float> a, V3<float> na, V3<float> x) { return dot(na, (x - a)) * na; }  // :176-180

// ScanConverterInternals::mapToParameters3D, BF/ScanConverter.cu:182-275 (Tf = float)
bool mapToParameters3D(V3<float> a, V3<float> ax, V3<float> ay, V3<float> axy, V3<float> da, V3<float> dax,
                       V3<float> day, V3<float> daxy, V3<float> x, V3<float>& out) {
    V3<float> normalXLow = normalize(cross(da, (ay + day) - a));
    V3<float> normalYLow = normalize(cross((ax + dax) - a, da));
    V3<float> normalXHigh = normalize(cross(dax, (axy + daxy) - ax));
    V3<float> normalYHigh = normalize(cross((axy + daxy) - ay, day));
    V2<float> lowT{0, 0}, highT{1, 1};
    V3<float> lowConnX = pointPlaneConnection(a, normalXLow, x);
    V3<float> highConnX = pointPlaneConnection(ax, normalXHigh, x);
    V3<float> lowConnY = pointPlaneConnection(a, normalYLow, x);
    V3<float> highConnY = pointPlaneConnection(ay, normalYHigh, x);
    V2<float> lowDist{norm(lowConnX), norm(lowConnY)};
    V2<float> highDist{norm(highConnX), norm(highConnY)};
    if (dot(lowConnX, highConnX) > 0 || dot(lowConnY, highConnY) > 0) return false;
    V2<float> dist{1e10f, 1e10f};
    V2<float> t{(highT.x - lowT.x) / 2 + lowT.x, (highT.y - lowT.y) / 2 + lowT.y};
    V3<float> pbX1{0, 0, 0}, pbY1{0, 0, 0}, pbX2{0, 0, 0}, pbY2{0, 0, 0};
    for (int it = 0; it < kMaxIter && (dist.x > kDistThreshold || dist.y > kDistThreshold); it++) {
        V2<float> sum{highDist.x + lowDist.x, highDist.y + lowDist.y};
        t = {(1 - highDist.x / sum.x) * highT.x + (1 - lowDist.x / sum.x) * lowT.x,
             (1 - highDist.y / sum.y) * highT.y + (1 - lowDist.y / sum.y) * lowT.y};
        pbX1 = (1 - t.x) * a + t.x * ax;
        pbX2 = (1 - t.x) * ay + t.x * axy;
        pbY1 = (1 - t.y) * a + t.y * ay;
        pbY2 = (1 - t.y) * ax + t.y * axy;
        V3<float> dir = slerp3(slerp3(da, dax, t.x), slerp3(day, daxy, t.x), t.y);
        V3<float> nx = normalize(cross(dir, pbX2 - pbX1));
        V3<float> ny = normalize(cross(pbY2 - pbY1, dir));
        V3<float> connX = pointPlaneConnection(pbX1, nx, x);
        V3<float> connY = pointPlaneConnection(pbY1, ny, x);
        dist = {norm(connX), norm(connY)};
        if (dot(highConnX, connX) > kEps) { highT.x = t.x; highConnX = connX; highDist.x = dist.x; }
        else if (dot(lowConnX, connX) > kEps) { lowT.x = t.x; lowConnX = connX; lowDist.x = dist.x; }
        if (dot(highConnY, connY) > kEps) { highT.y = t.y; highConnY = connY; highDist.y = dist.y; }
        else if (dot(lowConnY, connY) > kEps) { lowT.y = t.y; lowConnY = connY; lowDist.y = dist.y; }
    }
    V3<float> lineBase = (1 - t.y) * pbX1 + t.y * pbX2;
    out = {t.x, t.y, norm(x - lineBase)};
    return true;
}

V3<float> toF(V3<double> v) { return {static_cast<float>(v.x), static_cast<float>(v.y), static_cast<float>(v.z)}; }

}  // namespace

extern "C" {

// Scan-conversion tables, ScanConverter::updateInternals, BF/ScanConverter.cu:513-815.
// scanlines: [layout_x * layout_y], index x + y * layout_x. If any table pointer is NULL only the
// image size is returned. The 2D build is serial (quirk Q7: on a shared scanline edge the quad with
// the higher index wins); the 3D build visits quads in the reference's launch order.
int orc_scan_tables(const sb_scanline_rx* lines, uint32_t lx, uint32_t ly, uint32_t numSamples, double depth,
                    double resolution, uint32_t* sizeOut, double* bbMinOut, uint8_t* mask, uint32_t* sampleIdx,
                    float* weightX, float* weightY, float* weightZ) {
    auto L = [&](size_t x, size_t y) -> const sb_scanline_rx& { return lines[x + y * lx]; };
    double startDepth = 0, endDepth = depth;
    V3<double> bbMin{std::numeric_limits<double>::max(), std::numeric_limits<double>::max(), std::numeric_limits<double>::max()};
    V3<double> bbMax{-std::numeric_limits<double>::max(), -std::numeric_limits<double>::max(), -std::numeric_limits<double>::max()};
    for (size_t y = 0; y < ly; y++)
        for (size_t x = 0; x < lx; x++) {
            V3<double> p1 = pointOf(L(x, y), startDepth), p2 = pointOf(L(x, y), endDepth);
            bbMin = {std::min(bbMin.x, p1.x), std::min(bbMin.y, p1.y), std::min(bbMin.z, p1.z)};
            bbMax = {std::max(bbMax.x, p1.x), std::max(bbMax.y, p1.y), std::max(bbMax.z, p1.z)};
            bbMin = {std::min(bbMin.x, p2.x), std::min(bbMin.y, p2.y), std::min(bbMin.z, p2.z)};
            bbMax = {std::max(bbMax.x, p2.x), std::max(bbMax.y, p2.y), std::max(bbMax.z, p2.z)};
        }
    size_t W = static_cast<size_t>(std::ceil((bbMax.x - bbMin.x) / resolution)) + 1;
    size_t H = static_cast<size_t>(std::ceil((bbMax.y - bbMin.y) / resolution)) + 1;
    size_t D = static_cast<size_t>(std::ceil((bbMax.z - bbMin.z) / resolution)) + 1;
    W = std::max(W, size_t(1)); H = std::max(H, size_t(1)); D = std::max(D, size_t(1));
    sizeOut[0] = static_cast<uint32_t>(W); sizeOut[1] = static_cast<uint32_t>(H); sizeOut[2] = static_cast<uint32_t>(D);
    if (bbMinOut) { bbMinOut[0] = bbMin.x; bbMinOut[1] = bbMin.y; bbMinOut[2] = bbMin.z; }
    if (!mask || !sampleIdx || !weightX || !weightY || !weightZ) return 0;
    size_t numel = W * H * D;
    std::fill(mask, mask + numel, 0);
    std::fill(sampleIdx, sampleIdx + numel, 0u);
    std::fill(weightX, weightX + numel, 0.0f);
    std::fill(weightY, weightY + numel, 0.0f);
    std::fill(weightZ, weightZ + numel, 0.0f);
    double sampleDistance = depth / (numSamples - 1);  // USImageProperties::getSampleDistance, SL/USImageProperties.cpp:326-329
    uint32_t numScanlines = lx * ly;
    bool is2D = (lx == 1 || ly == 1);
    if (is2D) {
        V2<double> bb2{bbMin.x, bbMin.y};
        for (size_t y = 0; y < ly; y++) {
            for (int x = 0; x < static_cast<int>(lx) - 1; x++) {
                V3<double> s3 = pointOf(L(x, y), startDepth), sN3 = pointOf(L(x + 1, y), startDepth);
                V3<double> e3 = pointOf(L(x, y), endDepth), eN3 = pointOf(L(x + 1, y), endDepth);
                V2<double> start{s3.x, s3.y}, startN{sN3.x, sN3.y}, end{e3.x, e3.y}, endN{eN3.x, eN3.y};
                V2<double> qMin{std::min(std::min(std::min(start.x, startN.x), end.x), endN.x),
                                std::min(std::min(std::min(start.y, startN.y), end.y), endN.y)};
                V2<double> qMax{std::max(std::max(std::max(start.x, startN.x), end.x), endN.x),
                                std::max(std::max(std::max(start.y, startN.y), end.y), endN.y)};
                size_t pminx = static_cast<size_t>(std::floor((qMin.x - bb2.x) / resolution));
                size_t pminy = static_cast<size_t>(std::floor((qMin.y - bb2.y) / resolution));
                size_t pmaxx = static_cast<size_t>(std::ceil((qMax.x - bb2.x) / resolution));
                size_t pmaxy = static_cast<size_t>(std::ceil((qMax.y - bb2.y) / resolution));
                for (size_t px = pminx; px <= pmaxx; px++) {
                    for (size_t py = pminy; py <= pmaxy; py++) {
                        V2<double> pos{static_cast<double>(px) * resolution + bb2.x, static_cast<double>(py) * resolution + bb2.y};
                        if (insideTriangle(endN, end, start, pos) || insideTriangle(start, startN, endN, pos)) {
                            size_t idx = px + py * W;
                            if (px >= W || py >= H) continue;
                            mask[idx] = 1;
                            V2<double> p = mapToParameters2D(posOf(L(x, y)), posOf(L(x + 1, y)), dirOf(L(x, y)),
                                                             dirOf(L(x + 1, y)), {pos.x, pos.y, 0.0});
                            double t = p.x, d = p.y;
                            uint32_t sis = static_cast<uint32_t>(std::floor(d / sampleDistance));
                            float wY = static_cast<float>(d - (sis * sampleDistance));  // quirk Q5: in mm
                            float wX = static_cast<float>(t);
                            uint32_t si = static_cast<uint32_t>(sis * numScanlines + x + y * lx);
                            sampleIdx[idx] = si;
                            weightX[idx] = wX;
                            weightY[idx] = wY;
                        }
                    }
                }
            }
        }
    } else {
        for (int y = 0; y < static_cast<int>(ly) - 1; y++) {
            for (int x = 0; x < static_cast<int>(lx) - 1; x++) {
                V3<double> s1 = pointOf(L(x, y), startDepth), e1 = pointOf(L(x, y), endDepth);
                V3<double> s2 = pointOf(L(x + 1, y), startDepth), e2 = pointOf(L(x + 1, y), endDepth);
                V3<double> s3 = pointOf(L(x, y + 1), startDepth), e3 = pointOf(L(x, y + 1), endDepth);
                V3<double> s4 = pointOf(L(x + 1, y + 1), startDepth), e4 = pointOf(L(x + 1, y + 1), endDepth);
                auto vmin = [](V3<double> a, V3<double> b) { return V3<double>{std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; };
                auto vmax = [](V3<double> a, V3<double> b) { return V3<double>{std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; };
                V3<double> tMin = vmin(vmin(vmin(s1, s2), vmin(s3, s4)), vmin(vmin(e1, e2), vmin(e3, e4)));
                V3<double> tMax = vmax(vmax(vmax(s1, s2), vmax(s3, s4)), vmax(vmax(e1, e2), vmax(e3, e4)));
                int vminx = static_cast<int>(static_cast<size_t>(std::floor((tMin.x - bbMin.x) / resolution)));
                int vminy = static_cast<int>(static_cast<size_t>(std::floor((tMin.y - bbMin.y) / resolution)));
                int vminz = static_cast<int>(static_cast<size_t>(std::floor((tMin.z - bbMin.z) / resolution)));
                int vmaxx = static_cast<int>(static_cast<size_t>(std::ceil((tMax.x - bbMin.x) / resolution)));
                int vmaxy = static_cast<int>(static_cast<size_t>(std::ceil((tMax.y - bbMin.y) / resolution)));
                int vmaxz = static_cast<int>(static_cast<size_t>(std::ceil((tMax.z - bbMin.z) / resolution)));
                V3<float> fs1 = toF(s1), fs2 = toF(s2), fs3 = toF(s3), fs4 = toF(s4);
                V3<float> fe1 = toF(e1), fe2 = toF(e2), fe3 = toF(e3), fe4 = toF(e4);
                V3<float> p1 = toF(posOf(L(x, y))), p2 = toF(posOf(L(x + 1, y))), p3 = toF(posOf(L(x, y + 1))),
                          p4 = toF(posOf(L(x + 1, y + 1)));
                V3<float> d1 = toF(dirOf(L(x, y))), d2 = toF(dirOf(L(x + 1, y))), d3 = toF(dirOf(L(x, y + 1))),
                          d4 = toF(dirOf(L(x + 1, y + 1)));
                float res = static_cast<float>(resolution);
                V3<float> fbb = toF(bbMin);
                float sd = static_cast<float>(sampleDistance);
                for (int vz = vminz; vz <= vmaxz; vz++)
                    for (int vy = vminy; vy <= vmaxy; vy++)
                        for (int vx = vminx; vx <= vmaxx; vx++) {
                            // computeParameterBB3D, BF/ScanConverter.cu:277-347, then computeParametersVoxel3D :50-124
                            V3<float> vp{static_cast<float>(vx) * res + fbb.x, static_cast<float>(vy) * res + fbb.y,
                                         static_cast<float>(vz) * res + fbb.z};
                            if (insideTet(fs1, fs2, fs3, fe1, vp) || insideTet(fs2, fs4, fs3, fe4, vp) ||
                                insideTet(fs2, fe1, fe2, fe4, vp) || insideTet(fs3, fe3, fe1, fe4, vp) ||
                                insideTet(fs2, fs3, fe1, fe4, vp)) {
                                V3<float> prm;
                                if (mapToParameters3D(p1, p2, p3, p4, d1, d2, d3, d4, vp, prm)) {
                                    if (vx < 0 || vy < 0 || vz < 0 || static_cast<size_t>(vx) >= W ||
                                        static_cast<size_t>(vy) >= H || static_cast<size_t>(vz) >= D)
                                        continue;
                                    size_t vi = vx + vy * W + vz * W * H;
                                    mask[vi] = 1;
                                    float d = prm.z + 0;
                                    uint32_t sis = static_cast<uint32_t>(std::floor(d / sd));
                                    float wY = d / sd - sis;
                                    sampleIdx[vi] = static_cast<uint32_t>(sis * lx * ly + x + y * lx);
                                    weightX[vi] = prm.x;
                                    weightY[vi] = wY;
                                    weightZ[vi] = prm.y;
                                }
                            }
                        }
            }
        }
    }
    return 0;
}

// scanConvert2D / scanConvert3D, BF/ScanConverter.cu:349-428. in: FP32 [numSamples][lx*ly].
// The 2D gather of the reference has no bounds check; reads past the input are taken as 0 here.
int orc_scan_apply(const float* in, uint32_t lx, uint32_t ly, uint32_t numSamples, const uint32_t* size,
                   const uint8_t* mask, const uint32_t* sampleIdx, const float* wXs, const float* wYs,
                   const float* wZs, void* out, int outDtype) {
    uint32_t W = size[0], H = size[1], D = size[2];
    uint32_t numScanlines = lx * ly;
    size_t inN = static_cast<size_t>(numScanlines) * numSamples;
    auto rd = [&](size_t i) -> float { return i < inN ? in[i] : 0.0f; };
    bool is2D = (lx == 1 || ly == 1);
    for (uint32_t z = 0; z < D; z++)
        for (uint32_t y = 0; y < H; y++)
            for (uint32_t x = 0; x < W; x++) {
                size_t p = x + static_cast<size_t>(y) * W + static_cast<size_t>(z) * W * H;
                float val = 0;
                if (mask[p]) {
                    uint32_t s = sampleIdx[p];
                    float wX = wXs[p], wY = wYs[p];
                    if (is2D) {
                        val = (1 - wY) * ((1 - wX) * rd(s) + wX * rd(s + 1)) +
                              wY * ((1 - wX) * rd(s + numScanlines) + wX * rd(s + 1 + numScanlines));
                    } else {
                        float wZ = wZs[p];
                        if (s + 1 + lx + numScanlines < numSamples * numScanlines) {
                            val = (1 - wY) * ((1 - wZ) * ((1 - wX) * in[s] + wX * in[s + 1]) +
                                              wZ * ((1 - wX) * in[s + lx] + wX * in[s + 1 + lx])) +
                                  wY * ((1 - wZ) * ((1 - wX) * in[s + numScanlines] + wX * in[s + 1 + numScanlines]) +
                                        wZ * ((1 - wX) * in[s + lx + numScanlines] + wX * in[s + 1 + lx + numScanlines]));
                        }
                    }
                }
                if (outDtype == SB_UINT8) static_cast<uint8_t*>(out)[p] = static_cast<uint8_t>(std::min(std::max(val, 0.0f), 255.0f));
                else if (outDtype == SB_INT16) static_cast<int16_t*>(out)[p] = static_cast<int16_t>(std::min(std::max(val, -32767.0f), 32767.0f));
                else static_cast<float*>(out)[p] = val;
            }
    return 0;
}

// ------------------------------------------------------------------------------------ MV
// RxBeamformerMV::performRxBeamforming, BF/RxBeamformerMV.cu:382-622 with the kernels :60-378.
// Real data (iscomplex = 0) follows the reference: aperture from the first/last nonzero channel of
// the centre sample (:80-110), subarrays of size min(L, aperture), spatial covariance summed over the
// active subarrays (:152-195), temporal smoothing over +-T samples truncated at the edges of the
// 2000-sample processing blocks (:197-228), diagonal loading trace/size (:239-276, scaled by
// loadingScale), unused diagonal set to the loading and unused off-diagonals 0 (:278-306),
// a = R^-1 1, y = numChannels * sum_v (sum_k x_k[v]) a_v / (sum a * nActive^p) (:308-378),
// |y| > 1e7 or NaN -> 0. Sizes and masks are taken at each sample's own depth (for depths >= 2000
// the reference reads them at depth - 2000 from out-of-range buffers, quirk Q4).
// precision 32: covariance and weighting in float, solve in double. 64: everything double.
// Complex data (iscomplex = 1, interleaved): R = sum x x^H, y = sum_v conj(a_v) xbar_v / (Re sum a ...).
}  // extern "C"

// solveBlockwisePCGJacobi (BF/RxBeamformerMVpcg.cu:450-546) in working precision W on the leading
// sz x sz block of R (row-major, pitch L), right-hand side 1; the solution goes to a[0..sz).
template <typename W>
void pcgSolve(const std::vector<std::complex<double>>& R, uint32_t L, uint32_t sz, uint32_t maxIt, double thr,
              std::vector<std::complex<double>>& a) {
    std::vector<W> x(sz, W(1)), r(sz), d(sz), q(sz), t(sz), sv(sz), A(static_cast<size_t>(sz) * sz);
    for (uint32_t i = 0; i < sz; i++)
        for (uint32_t j = 0; j < sz; j++) A[i * sz + j] = static_cast<W>(R[i * L + j].real());
    auto matvec = [&](const std::vector<W>& v, std::vector<W>& o) {
        for (uint32_t i = 0; i < sz; i++) {
            W acc = 0;
            for (uint32_t j = 0; j < sz; j++) acc += A[i * sz + j] * v[j];
            o[i] = acc;
        }
    };
    auto dot = [&](const std::vector<W>& u, const std::vector<W>& w) {
        W acc = 0;
        for (uint32_t i = 0; i < sz; i++) acc += u[i] * w[i];
        return acc;
    };
    matvec(x, t);
    for (uint32_t i = 0; i < sz; i++) {
        r[i] = W(-1) * t[i] + W(1);
        d[i] = r[i] / A[i * sz + i];
    }
    W deltaNew = dot(r, d);
    W residualNorm = W(2) * static_cast<W>(thr);
    for (uint32_t it = 0; it < maxIt && static_cast<double>(deltaNew) > 1e-30 && residualNorm > static_cast<W>(thr); it++) {
        matvec(d, q);
        const W alpha = deltaNew / dot(d, q);
        for (uint32_t i = 0; i < sz; i++) x[i] = alpha * d[i] + x[i];
        matvec(x, t);
        for (uint32_t i = 0; i < sz; i++) r[i] = W(-1) * t[i] + W(1);
        residualNorm = std::sqrt(dot(r, r));
        for (uint32_t i = 0; i < sz; i++) sv[i] = r[i] / A[i * sz + i];
        const W deltaOld = deltaNew;
        deltaNew = dot(r, sv);
        const W beta = deltaNew / deltaOld;
        for (uint32_t i = 0; i < sz; i++) d[i] = beta * d[i] + sv[i];
    }
    for (uint32_t i = 0; i < sz; i++) a[i] = std::complex<double>(static_cast<double>(x[i]), 0.0);
}

extern "C" {

// solver 0: Cholesky (RxBeamformerMV). solver 1: RxBeamformerMVpcg's Jacobi-PCG (BF/RxBeamformerMVpcg.cu:
// 450-546): on the sz x sz loaded system R a = 1 from a = 1, residual r = b - R a recomputed every
// iteration (reinitialisation frequency 1), stop after maxIt iterations, when r.s <= 1e-30 or when
// |r| <= pcgThr; sums in order, in float (precision 32) or double (64). Real data only.
static int mvImpl(const float* raw, int iscomplex, float* outF, double* outD, uint32_t nRx, uint32_t nCh, uint32_t nS,
                  uint32_t L, uint32_t T, double scalingPower, float loadingScale, int precision, uint32_t blockSize,
                  int nthreads, int solver, uint32_t maxIt, double pcgThr) {
    if (L == 0) L = nCh / 2;
    if (L > nCh || L == 0) return -1;
    if (blockSize == 0) blockSize = 2000;
    const uint32_t numSub = nCh - L + 1;
    typedef std::complex<double> cd;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int line = 0; line < static_cast<int>(nRx); line++) {
        auto X = [&](uint32_t s, uint32_t ch) -> cd {
            size_t i = s + static_cast<size_t>(ch) * nS + static_cast<size_t>(line) * nCh * nS;
            if (iscomplex) return cd(raw[2 * i], raw[2 * i + 1]);
            return cd(raw[i], 0.0);
        };
        // per-sample aperture
        std::vector<uint32_t> first(nS), size(nS);
        std::vector<uint8_t> masks(static_cast<size_t>(nS) * numSub);
        std::vector<uint32_t> offs(static_cast<size_t>(nS) * numSub);
        for (uint32_t s = 0; s < nS; s++) {
            uint32_t f = 0, l = 0;
            for (uint32_t ch = 0; ch < nCh; ch++) if (X(s, ch) != cd(0, 0)) { f = ch; break; }
            for (int32_t ch = static_cast<int32_t>(nCh) - 1; ch >= 0; ch--) if (X(s, ch) != cd(0, 0)) { l = ch; break; }
            uint32_t sz = std::min(L, l - f + 1);
            size[s] = sz;
            first[s] = f;
            for (uint32_t k = 0; k < numSub; k++) {
                bool m = (f + k + sz - 1) <= l;
                uint32_t o = std::min(std::max(f + k, 0u), nCh - sz + 1);
                offs[s * numSub + k] = o;
                if (k > 1) m = m && (o != offs[s * numSub + k - 1]);
                masks[s * numSub + k] = m;
            }
        }
        std::vector<cd> Rraw(static_cast<size_t>(nS) * L * L, cd(0, 0));
        for (uint32_t s = 0; s < nS; s++) {
            uint32_t sz = size[s];
            for (uint32_t r = 0; r < sz; r++)
                for (uint32_t c = 0; c < sz; c++) {
                    if (precision == 32 && !iscomplex) {
                        float acc = 0;
                        for (uint32_t k = 0; k < numSub; k++)
                            if (masks[s * numSub + k]) {
                                uint32_t o = offs[s * numSub + k];
                                acc += static_cast<float>(X(s, o + c).real()) * static_cast<float>(X(s, o + r).real());
                            }
                        Rraw[(static_cast<size_t>(s) * L + r) * L + c] = cd(acc, 0);
                    } else {
                        cd acc(0, 0);
                        for (uint32_t k = 0; k < numSub; k++)
                            if (masks[s * numSub + k]) {
                                uint32_t o = offs[s * numSub + k];
                                acc += X(s, o + r) * std::conj(X(s, o + c));
                            }
                        Rraw[(static_cast<size_t>(s) * L + r) * L + c] = acc;
                    }
                }
        }
        for (uint32_t s = 0; s < nS; s++) {
            uint32_t sz = size[s];
            uint32_t b0 = (s / blockSize) * blockSize;
            uint32_t b1 = std::min(nS, b0 + blockSize) - 1;
            int firstT = std::max(static_cast<int>(b0), static_cast<int>(s) - static_cast<int>(T));
            int lastT = std::min(static_cast<int>(b1), static_cast<int>(s) + static_cast<int>(T));
            std::vector<cd> R(static_cast<size_t>(L) * L, cd(0, 0));
            for (uint32_t r = 0; r < sz; r++)
                for (uint32_t c = 0; c < sz; c++) {
                    if (precision == 32 && !iscomplex) {
                        float acc = 0;
                        for (int t = firstT; t <= lastT; t++) acc += static_cast<float>(Rraw[(static_cast<size_t>(t) * L + r) * L + c].real());
                        R[r * L + c] = cd(acc, 0);
                    } else {
                        cd acc(0, 0);
                        for (int t = firstT; t <= lastT; t++) acc += Rraw[(static_cast<size_t>(t) * L + r) * L + c];
                        R[r * L + c] = acc;
                    }
                }
            double trace = 0;
            if (precision == 32 && !iscomplex) {
                float tr = 0;
                for (uint32_t i = 0; i < sz; i++) tr += static_cast<float>(R[i * L + i].real());
                float loading = (1.0f / static_cast<float>(sz)) * tr * loadingScale;
                for (uint32_t i = 0; i < sz; i++) R[i * L + i] = cd(static_cast<float>(R[i * L + i].real()) + loading, 0);
                for (uint32_t i = sz; i < L; i++) R[i * L + i] = cd(loading, 0);
                trace = tr;
            } else {
                for (uint32_t i = 0; i < sz; i++) trace += R[i * L + i].real();
                double loading = (1.0 / sz) * trace * loadingScale;
                for (uint32_t i = 0; i < sz; i++) R[i * L + i] += loading;
                for (uint32_t i = sz; i < L; i++) R[i * L + i] = cd(loading, 0);
            }
            cd y(0, 0);
            if (solver == 1 && trace > 0 && std::isfinite(trace)) {
                std::vector<cd> a(L, cd(0, 0));
                if (precision == 32) pcgSolve<float>(R, L, sz, maxIt, pcgThr, a);
                else pcgSolve<double>(R, L, sz, maxIt, pcgThr, a);
                int nActive = 0;
                for (uint32_t k = 0; k < numSub; k++) nActive += masks[s * numSub + k] != 0;
                if (precision == 32) {
                    float ws = 0.0f;
                    for (uint32_t v = 0; v < sz; v++) ws += static_cast<float>(a[v].real()) * 1.0f;
                    ws = 1.0f / (ws * std::pow(static_cast<float>(nActive), static_cast<float>(scalingPower)));
                    float bs = 0.0f;
                    for (uint32_t v = 0; v < sz; v++) {
                        float sm = 0.0f;
                        for (uint32_t k = 0; k < numSub; k++)
                            if (masks[s * numSub + k]) sm += static_cast<float>(X(s, offs[s * numSub + k] + v).real());
                        bs += sm * static_cast<float>(a[v].real()) * ws;
                    }
                    y = cd(bs, 0);
                } else {
                    double asum = 0;
                    for (uint32_t v = 0; v < sz; v++) asum += a[v].real();
                    double ws = 1.0 / (asum * std::pow(static_cast<double>(nActive), scalingPower));
                    double bs = 0;
                    for (uint32_t v = 0; v < sz; v++) {
                        double sm = 0;
                        for (uint32_t k = 0; k < numSub; k++)
                            if (masks[s * numSub + k]) sm += X(s, offs[s * numSub + k] + v).real();
                        bs += sm * a[v].real() * ws;
                    }
                    y = cd(bs, 0);
                }
            } else if (solver == 0 && trace > 0 && std::isfinite(trace)) {
                // Cholesky R = G G^H (double), a = R^-1 1
                std::vector<cd> G(static_cast<size_t>(L) * L, cd(0, 0));
                bool ok = true;
                for (uint32_t j = 0; j < L && ok; j++) {
                    double dsum = R[j * L + j].real();
                    for (uint32_t k = 0; k < j; k++) dsum -= std::norm(G[j * L + k]);
                    if (!(dsum > 0)) { ok = false; break; }
                    double gjj = std::sqrt(dsum);
                    G[j * L + j] = gjj;
                    for (uint32_t i = j + 1; i < L; i++) {
                        cd v = R[i * L + j];
                        for (uint32_t k = 0; k < j; k++) v -= G[i * L + k] * std::conj(G[j * L + k]);
                        G[i * L + j] = v / gjj;
                    }
                }
                if (ok) {
                    std::vector<cd> z(L), a(L);
                    for (uint32_t i = 0; i < L; i++) {
                        cd v(1, 0);
                        for (uint32_t k = 0; k < i; k++) v -= G[i * L + k] * z[k];
                        z[i] = v / G[i * L + i].real();
                    }
                    for (int i = static_cast<int>(L) - 1; i >= 0; i--) {
                        cd v = z[i];
                        for (uint32_t k = i + 1; k < L; k++) v -= std::conj(G[k * L + i]) * a[k];
                        a[i] = v / G[i * L + i].real();
                    }
                    int nActive = 0;
                    for (uint32_t k = 0; k < numSub; k++) nActive += masks[s * numSub + k] != 0;
                    if (precision == 32 && !iscomplex) {
                        float ws = 0.0f;
                        for (uint32_t v = 0; v < sz; v++) ws += static_cast<float>(a[v].real()) * 1.0f;
                        ws = 1.0f / (ws * std::pow(static_cast<float>(nActive), static_cast<float>(scalingPower)));
                        float bs = 0.0f;
                        for (uint32_t v = 0; v < sz; v++) {
                            float sm = 0.0f;
                            for (uint32_t k = 0; k < numSub; k++)
                                if (masks[s * numSub + k]) sm += static_cast<float>(X(s, offs[s * numSub + k] + v).real());
                            bs += sm * static_cast<float>(a[v].real()) * ws;
                        }
                        y = cd(bs, 0);
                    } else {
                        cd asum(0, 0);
                        for (uint32_t v = 0; v < sz; v++) asum += a[v];
                        double ws = 1.0 / (asum.real() * std::pow(static_cast<double>(nActive), scalingPower));
                        for (uint32_t v = 0; v < sz; v++) {
                            cd sm(0, 0);
                            for (uint32_t k = 0; k < numSub; k++)
                                if (masks[s * numSub + k]) sm += X(s, offs[s * numSub + k] + v);
                            y += sm * std::conj(a[v]) * ws;
                        }
                    }
                }
            }
            if (std::abs(y) > 1e7 || std::isnan(y.real()) || std::isnan(y.imag())) y = cd(0, 0);
            y *= static_cast<double>(nCh);
            size_t o = static_cast<size_t>(line) + static_cast<size_t>(s) * nRx;
            if (outF) {
                if (iscomplex) { outF[2 * o] = static_cast<float>(y.real()); outF[2 * o + 1] = static_cast<float>(y.imag()); }
                else outF[o] = static_cast<float>(y.real());
            }
            if (outD) {
                if (iscomplex) { outD[2 * o] = y.real(); outD[2 * o + 1] = y.imag(); }
                else outD[o] = y.real();
            }
        }
    }
    return 0;
}

int orc_mv(const float* raw, int iscomplex, float* outF, double* outD, uint32_t nRx, uint32_t nCh, uint32_t nS,
           uint32_t L, uint32_t T, double scalingPower, float loadingScale, int precision, uint32_t blockSize,
           int nthreads) {
    return mvImpl(raw, iscomplex, outF, outD, nRx, nCh, nS, L, T, scalingPower, loadingScale, precision, blockSize,
                  nthreads, 0, 0, 0.0);
}

// RxBeamformerMVpcg::performRxBeamforming (BF/RxBeamformerMVpcg.cu:622-800): real data, no sample
// blocks; maxIt 0 means the subarray size (:649).
int orc_mv_pcg(const float* raw, float* outF, double* outD, uint32_t nRx, uint32_t nCh, uint32_t nS, uint32_t L,
               uint32_t T, double scalingPower, float loadingScale, uint32_t maxIt, double thr, int precision,
               int nthreads) {
    const uint32_t Ls = L == 0 ? nCh / 2 : L;
    return mvImpl(raw, 0, outF, outD, nRx, nCh, nS, L, T, scalingPower, loadingScale, precision, nS, nthreads, 1,
                  maxIt == 0 ? Ls : maxIt, thr);
}

}  // extern "C"
