// Scan conversion: table construction (2D on the host, 3D on the device in one launch), the
// table-driven bilinear / trilinear gathers, and the envelope -> log -> scan chain.
//   ScanConverter::updateInternals  Beamformer/ScanConverter.cu:513-815
//   scanConvert2D / scanConvert3D   Beamformer/ScanConverter.cu:349-428
#include <array>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "design.h"
#include "envelope.cuh"

struct sb_scan_plan {
    uint32_t lx, ly, numSamples;
    double depth, resolution;
    uint32_t size[3];
    bool is2D;
    uint8_t* dMask = nullptr;
    uint32_t* dSampleIdx = nullptr;
    float* dWX = nullptr;
    float* dWY = nullptr;
    float* dWZ = nullptr;
    float* dLog = nullptr;  // sb_env_log_scan_run's log-compressed envelope [numSamples][lx * ly]
};

namespace sb {
namespace {

// ----------------------------------------------------------------- 3D tables, single launch
struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3add(F3 a, F3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ F3 f3sub(F3 a, F3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ F3 f3mul(float s, F3 a) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
__device__ __forceinline__ float f3dot(F3 a, F3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float f3len(F3 a) { return __fsqrt_rn(f3dot(a, a)); }
__device__ __forceinline__ F3 f3unit(F3 a) {
    float n = f3len(a);
    return {__fdiv_rn(a.x, n), __fdiv_rn(a.y, n), __fdiv_rn(a.z, n)};
}
__device__ __forceinline__ F3 f3cross(F3 a, F3 b) {
    return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
__device__ F3 f3slerp(F3 a, F3 b, float t) {
    const double eps = 2.2204e-16;
    float om = acosf(f3dot(a, b));
    if (om < eps || t < eps) return a;
    if (__fsub_rn(1.0f, t) < eps) return b;
    float s = sinf(om);
    return f3add(f3mul(__fdiv_rn(sinf(__fmul_rn(__fsub_rn(1.0f, t), om)), s), a), f3mul(__fdiv_rn(sinf(__fmul_rn(t, om)), s), b));
}
// 4x4 determinant with a row of ones, as the reference expands it (ScanConverter.cu:149-174)
__device__ float det4(F3 a, F3 b, F3 c, F3 p) {
    const float axby = __fmul_rn(a.x, b.y), cypz = __fmul_rn(c.y, p.z), axbz = __fmul_rn(a.x, b.z), czpy = __fmul_rn(c.z, p.y);
    const float aybx = __fmul_rn(a.y, b.x), cxpz = __fmul_rn(c.x, p.z), aybz = __fmul_rn(a.y, b.z), czpx = __fmul_rn(c.z, p.x);
    const float azbx = __fmul_rn(a.z, b.x), cxpy = __fmul_rn(c.x, p.y), azby = __fmul_rn(a.z, b.y), cypx = __fmul_rn(c.y, p.x);
    float r = __fmul_rn(__fsub_rn(axby, aybx), __fsub_rn(c.z, p.z));
    r = __fadd_rn(r, __fmul_rn(__fsub_rn(aybz, azby), __fsub_rn(c.x, p.x)));
    r = __fadd_rn(r, __fmul_rn(__fsub_rn(azbx, axbz), __fsub_rn(c.y, p.y)));
    r = __fadd_rn(r, __fmul_rn(__fsub_rn(cypz, czpy), __fsub_rn(a.x, b.x)));
    r = __fsub_rn(r, __fmul_rn(__fsub_rn(cxpz, czpx), __fsub_rn(a.y, b.y)));
    r = __fadd_rn(r, __fmul_rn(__fsub_rn(cxpy, cypx), __fsub_rn(a.z, b.z)));
    return r;
}
__device__ bool inTet(F3 a, F3 b, F3 c, F3 d, F3 p) {
    const double th = 1e-9;
    return det4(a, b, c, d) > 0 && det4(p, b, c, d) >= -th && det4(a, p, c, d) >= -th && det4(a, b, p, d) >= -th &&
           det4(a, b, c, p) >= -th;
}
__device__ F3 planeConn(F3 a, F3 n, F3 x) { return f3mul(f3dot(n, f3sub(x, a)), n); }

// ScanConverterInternals::mapToParameters3D (ScanConverter.cu:182-275) in float.
__device__ bool locate3D(F3 a, F3 ax, F3 ay, F3 axy, F3 da, F3 dax, F3 day, F3 daxy, F3 x, F3& res) {
    const double eps = 2.2204e-16;
    F3 nXLo = f3unit(f3cross(da, f3sub(f3add(ay, day), a)));
    F3 nYLo = f3unit(f3cross(f3sub(f3add(ax, dax), a), da));
    F3 nXHi = f3unit(f3cross(dax, f3sub(f3add(axy, daxy), ax)));
    F3 nYHi = f3unit(f3cross(f3sub(f3add(axy, daxy), ay), day));
    float loTx = 0, loTy = 0, hiTx = 1, hiTy = 1;
    F3 loCX = planeConn(a, nXLo, x), hiCX = planeConn(ax, nXHi, x);
    F3 loCY = planeConn(a, nYLo, x), hiCY = planeConn(ay, nYHi, x);
    float loDx = f3len(loCX), loDy = f3len(loCY), hiDx = f3len(hiCX), hiDy = f3len(hiCY);
    if (f3dot(loCX, hiCX) > 0 || f3dot(loCY, hiCY) > 0) return false;
    float gx = 1e10f, gy = 1e10f;
    float tx = __fadd_rn(__fdiv_rn(__fsub_rn(hiTx, loTx), 2.0f), loTx), ty = __fadd_rn(__fdiv_rn(__fsub_rn(hiTy, loTy), 2.0f), loTy);
    F3 bX1{0, 0, 0}, bX2{0, 0, 0}, bY1{0, 0, 0}, bY2{0, 0, 0};
    for (int it = 0; it < 1000 && (gx > 1e-5 || gy > 1e-5); it++) {
        float sx = __fadd_rn(hiDx, loDx), sy = __fadd_rn(hiDy, loDy);
        tx = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(hiDx, sx)), hiTx), __fmul_rn(__fsub_rn(1.0f, __fdiv_rn(loDx, sx)), loTx));
        ty = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(hiDy, sy)), hiTy), __fmul_rn(__fsub_rn(1.0f, __fdiv_rn(loDy, sy)), loTy));
        bX1 = f3add(f3mul(__fsub_rn(1.0f, tx), a), f3mul(tx, ax));
        bX2 = f3add(f3mul(__fsub_rn(1.0f, tx), ay), f3mul(tx, axy));
        bY1 = f3add(f3mul(__fsub_rn(1.0f, ty), a), f3mul(ty, ay));
        bY2 = f3add(f3mul(__fsub_rn(1.0f, ty), ax), f3mul(ty, axy));
        F3 dir = f3slerp(f3slerp(da, dax, tx), f3slerp(day, daxy, tx), ty);
        F3 nx = f3unit(f3cross(dir, f3sub(bX2, bX1)));
        F3 ny = f3unit(f3cross(f3sub(bY2, bY1), dir));
        F3 cX = planeConn(bX1, nx, x), cY = planeConn(bY1, ny, x);
        gx = f3len(cX);
        gy = f3len(cY);
        if (f3dot(hiCX, cX) > eps) { hiTx = tx; hiCX = cX; hiDx = gx; }
        else if (f3dot(loCX, cX) > eps) { loTx = tx; loCX = cX; loDx = gx; }
        if (f3dot(hiCY, cY) > eps) { hiTy = ty; hiCY = cY; hiDy = gy; }
        else if (f3dot(loCY, cY) > eps) { loTy = ty; loCY = cY; loDy = gy; }
    }
    F3 base = f3add(f3mul(__fsub_rn(1.0f, ty), bX1), f3mul(ty, bX2));
    res = {tx, ty, f3len(f3sub(x, base))};
    return true;
}

struct Quad {
    F3 s[4], e[4], p[4], d[4];   // start/end points, origins, directions of the 4 scanlines (float)
    int vmin[3], vmax[3];        // voxel bounding box
};

// Every voxel searches the quads from the last launched to the first and takes the first that
// claims it (inside one of its 5 tetrahedra and mapped): the result the reference's sequence of
// per-quad launches leaves behind.
__global__ void scan3DTablesKernel(const Quad* quads, int numQuads, int qlx, uint32_t W, uint32_t H, uint32_t D, F3 bb,
                                   float res, float sampleDistance, uint32_t lx, uint32_t ly, uint8_t* mask,
                                   uint32_t* sampleIdx, float* wX, float* wY, float* wZ) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= static_cast<size_t>(W) * H * D) return;
    const int vx = static_cast<int>(i % W), vy = static_cast<int>((i / W) % H), vz = static_cast<int>(i / (static_cast<size_t>(W) * H));
    const F3 pos{__fadd_rn(__fmul_rn(static_cast<float>(vx), res), bb.x), __fadd_rn(__fmul_rn(static_cast<float>(vy), res), bb.y),
                 __fadd_rn(__fmul_rn(static_cast<float>(vz), res), bb.z)};
    mask[i] = 0;
    sampleIdx[i] = 0;
    wX[i] = 0.0f;
    wY[i] = 0.0f;
    wZ[i] = 0.0f;
    for (int q = numQuads - 1; q >= 0; q--) {
        const Quad& Q = quads[q];
        if (vx < Q.vmin[0] || vx > Q.vmax[0] || vy < Q.vmin[1] || vy > Q.vmax[1] || vz < Q.vmin[2] || vz > Q.vmax[2]) continue;
        const F3 *s = Q.s, *e = Q.e;
        if (!(inTet(s[0], s[1], s[2], e[0], pos) || inTet(s[1], s[3], s[2], e[3], pos) || inTet(s[1], e[0], e[1], e[3], pos) ||
              inTet(s[2], e[2], e[0], e[3], pos) || inTet(s[1], s[2], e[0], e[3], pos)))
            continue;
        F3 prm;
        if (!locate3D(Q.p[0], Q.p[1], Q.p[2], Q.p[3], Q.d[0], Q.d[1], Q.d[2], Q.d[3], pos, prm)) continue;
        const int qx = q % qlx, qy = q / qlx;
        const float dd = __fadd_rn(prm.z, 0.0f);
        const uint32_t row = static_cast<uint32_t>(floorf(__fdiv_rn(dd, sampleDistance)));
        mask[i] = 1;
        sampleIdx[i] = static_cast<uint32_t>(row * lx * ly + qx + qy * lx);
        wX[i] = prm.x;
        wY[i] = __fsub_rn(__fdiv_rn(dd, sampleDistance), static_cast<float>(row));
        wZ[i] = prm.y;
        return;
    }
}

// ----------------------------------------------------------------- gathers
template <typename IN> __device__ __forceinline__ float rd(const IN* in, size_t i, size_t n) {
    return i < n ? toFloat(in[i]) : 0.0f;
}

struct ScanArgs {
    uint32_t W, H, D, lx, ly, nS;
    const uint8_t* mask;
    const uint32_t* sIdx;
    const float *wX, *wY, *wZ;
};

// bilinear (2D) / trilinear (3D) table gather (ScanConverter.cu:349-428). The 2D reference does
// not bound its reads; reads past the input are taken as 0 here.
template <typename IN, bool IS2D>
__device__ __forceinline__ float scanPixel(const IN* __restrict__ in, const ScanArgs& a, uint32_t m, uint32_t s,
                                           float wx, float wy, float wz) {
    if (!m) return 0.0f;
    const uint32_t L = a.lx * a.ly;
    const size_t inN = static_cast<size_t>(L) * a.nS;
    const float ux = __fsub_rn(1.0f, wx), uy = __fsub_rn(1.0f, wy);
    if (IS2D)
        return __fadd_rn(__fmul_rn(uy, __fadd_rn(__fmul_rn(ux, rd(in, s, inN)), __fmul_rn(wx, rd(in, s + 1, inN)))),
                         __fmul_rn(wy, __fadd_rn(__fmul_rn(ux, rd(in, s + L, inN)), __fmul_rn(wx, rd(in, s + 1 + L, inN)))));
    if (!(static_cast<size_t>(s) + 1 + a.lx + L < inN)) return 0.0f;
    const float uz = __fsub_rn(1.0f, wz);
    auto bl = [&](size_t b) {
        return __fadd_rn(__fmul_rn(uz, __fadd_rn(__fmul_rn(ux, toFloat(in[b])), __fmul_rn(wx, toFloat(in[b + 1])))),
                         __fmul_rn(wz, __fadd_rn(__fmul_rn(ux, toFloat(in[b + a.lx])), __fmul_rn(wx, toFloat(in[b + 1 + a.lx])))));
    };
    return __fadd_rn(__fmul_rn(uy, bl(s)), __fmul_rn(wy, bl(static_cast<size_t>(s) + L)));
}

template <typename OUT> struct Out4;
template <> struct Out4<uint8_t> {
    static __device__ __forceinline__ void put(uint8_t* o, float a, float b, float c, float d) {
        *reinterpret_cast<uchar4*>(o) = make_uchar4(clampCast<uint8_t>(a), clampCast<uint8_t>(b), clampCast<uint8_t>(c),
                                                    clampCast<uint8_t>(d));
    }
};
template <> struct Out4<int16_t> {
    static __device__ __forceinline__ void put(int16_t* o, float a, float b, float c, float d) {
        *reinterpret_cast<short4*>(o) = make_short4(clampCast<int16_t>(a), clampCast<int16_t>(b), clampCast<int16_t>(c),
                                                    clampCast<int16_t>(d));
    }
};
template <> struct Out4<float> {
    static __device__ __forceinline__ void put(float* o, float a, float b, float c, float d) {
        *reinterpret_cast<float4*>(o) = make_float4(clampCast<float>(a), clampCast<float>(b), clampCast<float>(c),
                                                    clampCast<float>(d));
    }
};

// Eight consecutive output pixels per thread, as two groups of four: each group's table entries as
// one 4-byte and two (3D: three) 16-byte loads and one vector store (the output is aligned to four
// elements; the tables are device allocations). VEC = false: one pixel per thread, for an output
// that is not.
template <typename IN, typename OUT, bool IS2D, bool VEC>
__global__ void __launch_bounds__(256) scanKernel(const IN* __restrict__ in, OUT* __restrict__ out, ScanArgs a) {
    const size_t n = static_cast<size_t>(a.W) * a.H * a.D;
    const size_t g = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (!VEC) {
        if (g < n)
            out[g] = clampCast<OUT>(scanPixel<IN, IS2D>(in, a, a.mask[g], a.sIdx[g], a.wX[g], a.wY[g], IS2D ? 0.0f : a.wZ[g]));
        return;
    }
    // two groups of four pixels: both groups' table loads, then all their gathers, are in flight together
    const size_t i0 = 8 * g;
    if (i0 >= n) return;
    if (i0 + 8 <= n) {
        uchar4 m[2];
        uint4 si[2];
        float4 wx[2], wy[2], wz[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const size_t b = i0 + 4 * h;
            m[h] = __ldg(reinterpret_cast<const uchar4*>(a.mask + b));
            si[h] = __ldg(reinterpret_cast<const uint4*>(a.sIdx + b));
            wx[h] = __ldg(reinterpret_cast<const float4*>(a.wX + b));
            wy[h] = __ldg(reinterpret_cast<const float4*>(a.wY + b));
            wz[h] = IS2D ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : __ldg(reinterpret_cast<const float4*>(a.wZ + b));
        }
#pragma unroll
        for (int h = 0; h < 2; h++)
            Out4<OUT>::put(out + i0 + 4 * h, scanPixel<IN, IS2D>(in, a, m[h].x, si[h].x, wx[h].x, wy[h].x, wz[h].x),
                           scanPixel<IN, IS2D>(in, a, m[h].y, si[h].y, wx[h].y, wy[h].y, wz[h].y),
                           scanPixel<IN, IS2D>(in, a, m[h].z, si[h].z, wx[h].z, wy[h].z, wz[h].z),
                           scanPixel<IN, IS2D>(in, a, m[h].w, si[h].w, wx[h].w, wy[h].w, wz[h].w));
        return;
    }
    for (size_t i = i0; i < n; i++)
        out[i] = clampCast<OUT>(scanPixel<IN, IS2D>(in, a, a.mask[i], a.sIdx[i], a.wX[i], a.wY[i], IS2D ? 0.0f : a.wZ[i]));
}

template <typename IN, typename OUT>
int launchScan(bool is2D, const ScanArgs& a, const IN* in, OUT* out, cudaStream_t st) {
    const size_t n = static_cast<size_t>(a.W) * a.H * a.D;
    const bool vec = reinterpret_cast<uintptr_t>(out) % (4 * sizeof(OUT)) == 0;
    const unsigned blocks = static_cast<unsigned>(((vec ? (n + 7) / 8 : n) + 255) / 256);
    if (vec) {
        if (is2D) scanKernel<IN, OUT, true, true><<<blocks, 256, 0, st>>>(in, out, a);
        else scanKernel<IN, OUT, false, true><<<blocks, 256, 0, st>>>(in, out, a);
    } else {
        if (is2D) scanKernel<IN, OUT, true, false><<<blocks, 256, 0, st>>>(in, out, a);
        else scanKernel<IN, OUT, false, false><<<blocks, 256, 0, st>>>(in, out, a);
    }
    SB_CHECK_LAUNCH("scanKernel");
    return SB_OK;
}

ScanArgs scanArgs(const sb_scan_plan* p) {
    ScanArgs a;
    a.W = p->size[0];
    a.H = p->size[1];
    a.D = p->size[2];
    a.lx = p->lx;
    a.ly = p->ly;
    a.nS = p->numSamples;
    a.mask = p->dMask;
    a.sIdx = p->dSampleIdx;
    a.wX = p->dWX;
    a.wY = p->dWY;
    a.wZ = p->dWZ;
    return a;
}

F3 toF3(double x, double y, double z) { return {static_cast<float>(x), static_cast<float>(y), static_cast<float>(z)}; }

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" {

int sb_scan_plan_create(const sb_scanline_rx* lines, uint32_t lx, uint32_t ly, uint32_t numSamples, double depth,
                        double resolution, sb_scan_plan** plan) {
    SB_REQUIRE(lines && plan, "sb_scan_plan_create: null argument");
    *plan = nullptr;
    SB_REQUIRE(lx >= 1 && ly >= 1 && numSamples >= 2 && depth > 0 && resolution > 0, "sb_scan_plan_create: bad sizes");
    const bool is2D = (lx == 1 || ly == 1);
    SB_REQUIRE(is2D ? (lx * ly > 1) : true, "sb_scan_plan_create: need at least two scanlines");
    SB_REQUIRE(is2D ? ly == 1 : true, "sb_scan_plan_create: 2D layouts must be scanlines along x");
    ScanTables t;
    if (is2D) scanTables2D(lines, lx, ly, numSamples, depth, resolution, t);
    else scanGeometry(lines, lx, ly, depth, resolution, t);
    const size_t n = static_cast<size_t>(t.size[0]) * t.size[1] * t.size[2];
    SB_REQUIRE(n <= (size_t(1) << 31), "sb_scan_plan_create: image of %zu voxels too large", n);
    sb_scan_plan* p = new sb_scan_plan();
    p->lx = lx;
    p->ly = ly;
    p->numSamples = numSamples;
    p->depth = depth;
    p->resolution = resolution;
    p->is2D = is2D;
    for (int i = 0; i < 3; i++) p->size[i] = t.size[i];
    cudaError_t e = cudaMalloc(&p->dMask, n);
    if (e == cudaSuccess) e = cudaMalloc(&p->dSampleIdx, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&p->dWX, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&p->dWY, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&p->dWZ, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&p->dLog, static_cast<size_t>(numSamples) * lx * ly * sizeof(float));
    if (e != cudaSuccess) {
        sb_scan_plan_destroy(p);
        return cudaFail(e, "sb_scan_plan_create: cudaMalloc");
    }
    if (is2D) {
        e = cudaMemcpy(p->dMask, t.mask.data(), n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(p->dSampleIdx, t.sampleIdx.data(), n * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(p->dWX, t.weightX.data(), n * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(p->dWY, t.weightY.data(), n * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(p->dWZ, t.weightZ.data(), n * 4, cudaMemcpyHostToDevice);
    } else {
        // per-quad data in the reference's launch order (ScanConverter.cu:746-809)
        std::vector<Quad> quads;
        auto L = [&](uint32_t x, uint32_t y) -> const sb_scanline_rx& { return lines[x + y * lx]; };
        auto pt = [](const sb_scanline_rx& s, double d) {
            return std::array<double, 3>{s.position[0] + d * s.direction[0], s.position[1] + d * s.direction[1],
                                         s.position[2] + d * s.direction[2]};
        };
        for (uint32_t y = 0; y + 1 < ly; y++)
            for (uint32_t x = 0; x + 1 < lx; x++) {
                const sb_scanline_rx* q4[4] = {&L(x, y), &L(x + 1, y), &L(x, y + 1), &L(x + 1, y + 1)};
                Quad Q;
                double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
                for (int c = 0; c < 4; c++) {
                    auto s = pt(*q4[c], 0.0), ee = pt(*q4[c], depth);
                    Q.s[c] = toF3(s[0], s[1], s[2]);
                    Q.e[c] = toF3(ee[0], ee[1], ee[2]);
                    Q.p[c] = toF3(q4[c]->position[0], q4[c]->position[1], q4[c]->position[2]);
                    Q.d[c] = toF3(q4[c]->direction[0], q4[c]->direction[1], q4[c]->direction[2]);
                    for (int k = 0; k < 3; k++) {
                        mn[k] = std::min(mn[k], std::min(s[k], ee[k]));
                        mx[k] = std::max(mx[k], std::max(s[k], ee[k]));
                    }
                }
                for (int k = 0; k < 3; k++) {
                    Q.vmin[k] = static_cast<int>(static_cast<size_t>(std::floor((mn[k] - t.bbMin[k]) / resolution)));
                    Q.vmax[k] = static_cast<int>(static_cast<size_t>(std::ceil((mx[k] - t.bbMin[k]) / resolution)));
                }
                quads.push_back(Q);
            }
        Quad* dQ = nullptr;
        e = cudaMalloc(&dQ, quads.size() * sizeof(Quad));
        if (e == cudaSuccess) e = cudaMemcpy(dQ, quads.data(), quads.size() * sizeof(Quad), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            F3 bb = toF3(t.bbMin[0], t.bbMin[1], t.bbMin[2]);
            scan3DTablesKernel<<<static_cast<unsigned>((n + 127) / 128), 128>>>(
                dQ, static_cast<int>(quads.size()), static_cast<int>(lx - 1), t.size[0], t.size[1], t.size[2], bb,
                static_cast<float>(resolution), static_cast<float>(depth / (numSamples - 1)), lx, ly, p->dMask,
                p->dSampleIdx, p->dWX, p->dWY, p->dWZ);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaDeviceSynchronize();
        }
        cudaFree(dQ);
    }
    if (e != cudaSuccess) {
        sb_scan_plan_destroy(p);
        return cudaFail(e, "sb_scan_plan_create: tables");
    }
    *plan = p;
    return SB_OK;
}

int sb_scan_plan_destroy(sb_scan_plan* p) {
    if (!p) return SB_OK;
    cudaFree(p->dMask);
    cudaFree(p->dSampleIdx);
    cudaFree(p->dWX);
    cudaFree(p->dWY);
    cudaFree(p->dWZ);
    cudaFree(p->dLog);
    delete p;
    return SB_OK;
}

int sb_scan_tables_2d_host(const sb_scanline_rx* lines, uint32_t lx, uint32_t numSamples, double depth,
                           double resolution, uint32_t size_xyz[3], uint8_t* mask, uint32_t* sampleIdx, float* wX,
                           float* wY) {
    SB_REQUIRE(lines && size_xyz, "sb_scan_tables_2d_host: null argument");
    SB_REQUIRE(lx >= 2 && numSamples >= 2 && depth > 0 && resolution > 0, "sb_scan_tables_2d_host: bad sizes");
    ScanTables t;
    if (!(mask && sampleIdx && wX && wY)) {
        scanGeometry(lines, lx, 1, depth, resolution, t);
        for (int i = 0; i < 3; i++) size_xyz[i] = t.size[i];
        return SB_OK;
    }
    scanTables2D(lines, lx, 1, numSamples, depth, resolution, t);
    for (int i = 0; i < 3; i++) size_xyz[i] = t.size[i];
    std::copy(t.mask.begin(), t.mask.end(), mask);
    std::copy(t.sampleIdx.begin(), t.sampleIdx.end(), sampleIdx);
    std::copy(t.weightX.begin(), t.weightX.end(), wX);
    std::copy(t.weightY.begin(), t.weightY.end(), wY);
    return SB_OK;
}

int sb_scan_image_size(const sb_scan_plan* p, uint32_t size_xyz[3]) {
    SB_REQUIRE(p && size_xyz, "sb_scan_image_size: null argument");
    for (int i = 0; i < 3; i++) size_xyz[i] = p->size[i];
    return SB_OK;
}

int sb_scan_copy_tables(const sb_scan_plan* p, uint8_t* mask, uint32_t* sampleIdx, float* wX, float* wY, float* wZ) {
    SB_REQUIRE(p, "sb_scan_copy_tables: null plan");
    const size_t n = static_cast<size_t>(p->size[0]) * p->size[1] * p->size[2];
    if (mask) SB_CUDA(cudaMemcpy(mask, p->dMask, n, cudaMemcpyDeviceToHost));
    if (sampleIdx) SB_CUDA(cudaMemcpy(sampleIdx, p->dSampleIdx, n * 4, cudaMemcpyDeviceToHost));
    if (wX) SB_CUDA(cudaMemcpy(wX, p->dWX, n * 4, cudaMemcpyDeviceToHost));
    if (wY) SB_CUDA(cudaMemcpy(wY, p->dWY, n * 4, cudaMemcpyDeviceToHost));
    if (wZ) SB_CUDA(cudaMemcpy(wZ, p->dWZ, n * 4, cudaMemcpyDeviceToHost));
    return SB_OK;
}

int sb_scan_run(const sb_scan_plan* p, const void* in, int in_dtype, void* out, int out_dtype, sb_stream stream) {
    SB_REQUIRE(p && in && out, "sb_scan_run: null argument");
    const ScanArgs a = scanArgs(p);
    cudaStream_t st = S(stream);
#define SB_SCAN(INT, OUTT) return launchScan<INT, OUTT>(p->is2D, a, static_cast<const INT*>(in), static_cast<OUTT*>(out), st)
    if (in_dtype == SB_FLOAT32 && out_dtype == SB_UINT8) SB_SCAN(float, uint8_t);
    if (in_dtype == SB_FLOAT32 && out_dtype == SB_FLOAT32) SB_SCAN(float, float);
    if (in_dtype == SB_FLOAT32 && out_dtype == SB_INT16) SB_SCAN(float, int16_t);
    if (in_dtype == SB_UINT8 && out_dtype == SB_UINT8) SB_SCAN(uint8_t, uint8_t);
    if (in_dtype == SB_UINT8 && out_dtype == SB_FLOAT32) SB_SCAN(uint8_t, float);
    if (in_dtype == SB_INT16 && out_dtype == SB_INT16) SB_SCAN(int16_t, int16_t);
    if (in_dtype == SB_INT16 && out_dtype == SB_FLOAT32) SB_SCAN(int16_t, float);
    if (in_dtype == SB_INT16 && out_dtype == SB_UINT8) SB_SCAN(int16_t, uint8_t);
#undef SB_SCAN
    return fail(SB_ERR_UNSUPPORTED, "sb_scan_run: %d -> %d unsupported", in_dtype, out_dtype);
}

// HilbertFirEnvelope -> LogCompressor (float) -> ScanConverter. The envelope and its log are
// computed once per input sample, by the tiled envelope kernel, into the plan's float image
// (numSamples x lines: 1 MB for a 2048 x 128 frame, which stays in L2); the table gather reads it
// from there. HBM traffic: the RF in, the tables and the image out.
int sb_env_log_scan_run(const sb_hilbert_plan* hilbert, const sb_scan_plan* scan, const float* rf, void* out,
                        int out_dtype, double dynamic_range_db, double gain, double in_max, sb_stream stream) {
    SB_REQUIRE(hilbert && scan && rf && out, "sb_env_log_scan_run: null argument");
    SB_REQUIRE(in_max > 0 && dynamic_range_db > 0, "sb_env_log_scan_run: inMax and dynamic range must be > 0");
    SB_REQUIRE(out_dtype == SB_UINT8 || out_dtype == SB_FLOAT32, "sb_env_log_scan_run: out dtype %d", out_dtype);
    float inScale, k;
    logConstants(dynamic_range_db, gain, in_max, SB_FLOAT32, inScale, k);
    cudaStream_t st = S(stream);
    const int nL = static_cast<int>(scan->lx * scan->ly), nS = static_cast<int>(scan->numSamples);
    const int r = launchHilbert(hilbert, rf, SB_FLOAT32, scan->dLog, nS, nL, true, inScale, k, st);
    if (r != SB_OK) return r;
    const ScanArgs a = scanArgs(scan);
    if (out_dtype == SB_UINT8) return launchScan<float, uint8_t>(scan->is2D, a, scan->dLog, static_cast<uint8_t*>(out), st);
    return launchScan<float, float>(scan->is2D, a, scan->dLog, static_cast<float*>(out), st);
}

}  // extern "C"
