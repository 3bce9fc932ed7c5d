// Minimum-variance (Capon) receive beamforming on raw-delayed channel data.
//
// Replaces RxBeamformerMV::performRxBeamforming (Beamformer/RxBeamformerMV.cu:382-622) and its
// kernels (:80-378): per (scanline, sample) the active aperture is taken from the first and last
// nonzero channel (:44-110), the spatially smoothed covariance over the K active subarrays of
// length sz = min(L, aperture) is summed over +-T samples clipped to the reference's 2000-sample
// processing blocks (:152-228), loaded with trace/sz on the diagonal (:239-306), solved for
// a = R^-1 1 and applied as y = numChannels * sum_v xbar_v a_v / (sum_v a_v * K^p) (:308-378), with
// |y| > 1e7 or NaN written as 0.
//
// B200 design: one warp per pixel, no cuBLAS, no host synchronisation.
//  * The covariance R = sum_k y_k y_k^H of the Hankel subarray vectors y_k = x[f+k .. f+k+L-1] is
//    Toeplitz-recursive along its diagonals: R[r][c] = R[r-1][c-1] + x[f+K-1+r] x*[f+K-1+c]
//    - x[f+r-1] x*[f+c-1]. Lane d owns the circulant diagonal d (entries (r, (r+d) mod L)), so one
//    sample's covariance costs K + 2(L-1) complex MACs per lane instead of K*L.
//  * For L <= 32 a warp walks a run of consecutive samples and keeps the temporal window sum in
//    registers, adding the entering sample's covariance and subtracting the leaving one. The sum is
//    kept as an unevaluated pair (hi, lo) updated by TwoSum (Knuth), so a bright echo that leaves the
//    window cancels to O(eps^2) instead of leaving O(eps) of its energy behind. For L in (32, 64]
//    (real data) every sample's window is summed directly.
//    The window's TwoSum updates of complex entries run on (re, im) pairs in packed adds
//    (__fadd2_rn, and s - h as the exact __ffma2_rn(h, -1, s)).
//  * The loaded matrix is transposed through shared memory into one row per lane and factored by an
//    FP32 Crout Cholesky R = G G^H (broadcast reads of the finished rows). Complex matrices with one
//    row per lane are kept in two planes (real and imaginary parts), so that the inner products over
//    pairs of columns run as packed FMAs with natural operands (solveRegsCplx). Only forward substitutions
//    are needed: with z = G^-1 1 and w = G^-1 xbar, sum_v a_v = z^H z and sum_v xbar_v a*_v = w^T z*.
//  * Condition estimate (max G_ii / min G_ii)^2. Systems above the threshold (or whose FP32
//    factorisation breaks down) are appended to a queue that a second kernel re-solves in FP64
//    (covariance, factorisation and substitutions), so FP64 runs only for those systems.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "common.cuh"

namespace sb {
namespace {

constexpr uint32_t kMvBlock = 2000;  // RxBeamformerMV.cu:390 sampleBlockSize
constexpr uint32_t kMvRun = 25;      // consecutive samples per warp; divides kMvBlock (25: the c3 warps fill 8.9 waves of 148 SMs x 8 warps)
constexpr int kMvMaxWarps = 8;
constexpr size_t kMvSmemBudget = 220 * 1024;
constexpr uint32_t kFull = 0xffffffffu;

template <class T> struct V {
    T re, im;
};

template <bool C> struct Elem;
template <> struct Elem<false> {
    float re;
};
template <> struct __align__(8) Elem<true> {
    float re, im;
};

template <bool C, class T> __device__ __forceinline__ V<T> vz() { return V<T>{T(0), T(0)}; }

template <bool C, class T> __device__ __forceinline__ V<T> ld(const Elem<C>& e) {
    V<T> v;
    v.re = T(e.re);
    if constexpr (C) v.im = T(e.im);
    else v.im = T(0);
    return v;
}

template <bool C, class T, class S> __device__ __forceinline__ V<T> ldG(const S& e) {
    V<T> v;
    v.re = T(e.re);
    if constexpr (C) v.im = T(e.im);
    else v.im = T(0);
    return v;
}

// acc += a * conj(b)
template <bool C, class T> __device__ __forceinline__ void macConj(V<T>& acc, const V<T>& a, const V<T>& b) {
    acc.re = fma(a.re, b.re, acc.re);
    if constexpr (C) {
        acc.re = fma(a.im, b.im, acc.re);
        acc.im = fma(a.im, b.re, acc.im);
        acc.im = fma(-a.re, b.im, acc.im);
    }
}
// acc -= a * conj(b)
template <bool C, class T> __device__ __forceinline__ void mscConj(V<T>& acc, const V<T>& a, const V<T>& b) {
    acc.re = fma(-a.re, b.re, acc.re);
    if constexpr (C) {
        acc.re = fma(-a.im, b.im, acc.re);
        acc.im = fma(-a.im, b.re, acc.im);
        acc.im = fma(a.re, b.im, acc.im);
    }
}
// acc -= a * b
template <bool C, class T> __device__ __forceinline__ void msc(V<T>& acc, const V<T>& a, const V<T>& b) {
    acc.re = fma(-a.re, b.re, acc.re);
    if constexpr (C) {
        acc.re = fma(a.im, b.im, acc.re);
        acc.im = fma(-a.re, b.im, acc.im);
        acc.im = fma(-a.im, b.re, acc.im);
    }
}

template <bool C, class T> __device__ __forceinline__ V<T> shflV(const V<T>& v, int src) {
    V<T> o;
    o.re = __shfl_sync(kFull, v.re, src);
    if constexpr (C) o.im = __shfl_sync(kFull, v.im, src);
    else o.im = T(0);
    return o;
}

template <class T> __device__ __forceinline__ T warpSum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Error-free sum (Knuth's TwoSum): hi + b = s + e exactly; the error is accumulated into lo.
__device__ __forceinline__ void twoSumAdd(float& hi, float& lo, float b) {
    const float s = __fadd_rn(hi, b);
    const float bb = __fsub_rn(s, hi);
    const float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    hi = s;
    lo = __fadd_rn(lo, e);
}

struct MvCounters {
    unsigned long long systems;
    unsigned long long fp64Systems;
    unsigned int queued;
    unsigned int maxCondBits;  // float bits of the largest condition estimate (non-negative)
};

struct MvArgs {
    const void* in;
    void* out;
    uint32_t nRx, nCh, nS, L, T;
    uint32_t ringSlots, ringPitch, runsPerLine, runsPerBlock, numItems;
    uint32_t blockLen;  // temporal windows are clipped to blocks of this many samples
    float power, loadScale, thr;
    int pcg;            // solve by Jacobi-PCG (RxBeamformerMVpcg) instead of Cholesky
    int pcgMaxIt;
    float pcgThr;
    uint32_t* queue;
    MvCounters* counters;
};

struct SampleMeta {
    int f, K, sz, pad;
};

template <class In> __device__ __forceinline__ Elem<false> readIn(const In* p) {
    Elem<false> e;
    e.re = static_cast<float>(__ldg(p));
    return e;
}
__device__ __forceinline__ Elem<true> readInC(const float2* p) {
    const float2 v = __ldg(p);
    Elem<true> e;
    e.re = v.x;
    e.im = v.y;
    return e;
}

// Stages sample t of one scanline ([nCh][nS] at xl) into a ring slot and derives the aperture
// (first / last nonzero channel, computeSubArrayMasks RxBeamformerMV.cu:80-110): sz = min(L, l-f+1)
// and the K = l - sz - f + 2 active subarrays start at f, f+1, ..., f+K-1.
template <bool C, class In>
__device__ __forceinline__ SampleMeta loadSample(const MvArgs& a, const In* xl, uint32_t t, Elem<C>* slot, int lane) {
    int first = -1, last = -1;
    for (uint32_t c0 = 0; c0 < a.ringPitch; c0 += 32) {
        const uint32_t ch = c0 + lane;
        Elem<C> v;
        v.re = 0.0f;
        if constexpr (C) v.im = 0.0f;
        if (ch < a.nCh) {
            if constexpr (C) v = readInC(reinterpret_cast<const float2*>(xl) + static_cast<size_t>(ch) * a.nS + t);
            else v = readIn(xl + static_cast<size_t>(ch) * a.nS + t);
        }
        slot[ch] = v;
        bool nz = v.re != 0.0f;
        if constexpr (C) nz = nz || v.im != 0.0f;
        const uint32_t m = __ballot_sync(kFull, nz);
        if (m) {
            if (first < 0) first = static_cast<int>(c0) + __ffs(m) - 1;
            last = static_cast<int>(c0) + 31 - __clz(m);
        }
    }
    SampleMeta md;
    md.f = first < 0 ? 0 : first;
    const int l = last < 0 ? 0 : last;
    md.sz = min(static_cast<int>(a.L), l - md.f + 1);
    md.K = l - md.sz - md.f + 2;
    md.pad = 0;
    __syncwarp();
    return md;
}

// Adds sign * (covariance of one sample) to the register accumulators of this lane's circulant
// diagonals d = lane + 32q. Entry r of diagonal d is R[r][(r + d) mod L]. The first row of the
// sample's covariance (D0[d] = R[0][d], a K-term sum) is computed when `fresh` and stored in d0,
// otherwise read back from d0: a sample enters and later leaves the window with identical values.
template <bool C, int NR, bool COMP, class T>
__device__ __forceinline__ void addCov(const Elem<C>* xv, SampleMeta m, V<T>* d0, bool fresh, int L, int lane, T sign,
                                       V<T> (&hi)[NR][32 * NR], V<T> (&lo)[NR][32 * NR]) {
    const int f = m.f, K = m.K;
    V<T> D0[NR];
    if (fresh) {
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const int d = lane + 32 * q;
            const int dd = d < L ? d : 0;
            V<T> a0 = vz<C, T>(), a1 = vz<C, T>(), a2 = vz<C, T>(), a3 = vz<C, T>();
            int k = 0;
            for (; k + 3 < K; k += 4) {
                macConj<C, T>(a0, ld<C, T>(xv[f + k]), ld<C, T>(xv[f + k + dd]));
                macConj<C, T>(a1, ld<C, T>(xv[f + k + 1]), ld<C, T>(xv[f + k + 1 + dd]));
                macConj<C, T>(a2, ld<C, T>(xv[f + k + 2]), ld<C, T>(xv[f + k + 2 + dd]));
                macConj<C, T>(a3, ld<C, T>(xv[f + k + 3]), ld<C, T>(xv[f + k + 3 + dd]));
            }
            for (; k < K; k++) macConj<C, T>(a0, ld<C, T>(xv[f + k]), ld<C, T>(xv[f + k + dd]));
            D0[q].re = (a0.re + a1.re) + (a2.re + a3.re);
            D0[q].im = (a0.im + a1.im) + (a2.im + a3.im);
            d0[d] = D0[q];
        }
        __syncwarp();
    } else {
#pragma unroll
        for (int q = 0; q < NR; q++) D0[q] = d0[lane + 32 * q];
    }
    // Start of the lower segment of diagonal d (entry (L-d, 0)) = conj(D0 of diagonal L-d).
    V<T> E0[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) {
        const int d = lane + 32 * q;
        const int src = (d > 0 && d < L) ? L - d : 0;
        const V<T> v = d0[src];
        E0[q].re = v.re;
        E0[q].im = -v.im;
    }
#pragma unroll
    for (int q = 0; q < NR; q++) {
        const int d = lane + 32 * q;
        const bool act = d < L;
        const int de = act ? d : 0;
        V<T> cur = D0[q];
#pragma unroll
        for (int r = 0; r < 32 * NR; r++) {
            if (r >= L) break;
            if (r > 0) {
                int c = r + de;
                if (c >= L) c -= L;
                const int cm1 = c > 0 ? c - 1 : 0;
                V<T> delta = vz<C, T>();
                macConj<C, T>(delta, ld<C, T>(xv[f + r - 1 + K]), ld<C, T>(xv[f + cm1 + K]));
                mscConj<C, T>(delta, ld<C, T>(xv[f + r - 1]), ld<C, T>(xv[f + cm1]));
                V<T> nxt;
                nxt.re = cur.re + delta.re;
                nxt.im = cur.im + delta.im;
                cur = c == 0 ? E0[q] : nxt;
            }
            if (act) {
                if constexpr (COMP && C && std::is_same<T, float>::value) {
                    // TwoSum of the real and imaginary parts in packed adds (s - h etc. as fma(h, -1, s))
                    const float2 m1 = make_float2(-1.0f, -1.0f);
                    const float2 h = make_float2(hi[q][r].re, hi[q][r].im);
                    const float2 b = make_float2(sign * cur.re, sign * cur.im);
                    const float2 s2 = __fadd2_rn(h, b);
                    const float2 bb = __ffma2_rn(h, m1, s2);
                    const float2 e = __fadd2_rn(__ffma2_rn(__ffma2_rn(bb, m1, s2), m1, h), __ffma2_rn(bb, m1, b));
                    const float2 l = __fadd2_rn(make_float2(lo[q][r].re, lo[q][r].im), e);
                    hi[q][r].re = s2.x;
                    hi[q][r].im = s2.y;
                    lo[q][r].re = l.x;
                    lo[q][r].im = l.y;
                } else if constexpr (COMP) {
                    twoSumAdd(hi[q][r].re, lo[q][r].re, sign * cur.re);
                    if constexpr (C) twoSumAdd(hi[q][r].im, lo[q][r].im, sign * cur.im);
                } else {
                    hi[q][r].re += sign * cur.re;
                    if constexpr (C) hi[q][r].im += sign * cur.im;
                }
            }
        }
    }
}

// Result of one system: y (before the numChannels factor) and whether it is valid.
template <class T> struct MvOut {
    V<T> y;
    bool ok;
    T cond;
};

// Crout Cholesky of the loaded L x L matrix in Gs (row pitch GP; entries outside the sz x sz block
// replaced by the loading on the diagonal and 0 elsewhere), one row per lane (rows lane + 32q) in
// registers. The forward substitutions z = G^-1 1 and w = G^-1 xbar advance one column behind the
// factorisation inside the same loop, which gives the scheduler two independent chains.
template <bool C, int NR, class T, class GE>
__device__ __forceinline__ MvOut<T> solveRegs(GE* Gs, int GP, int L, int sz, T loading, int lane, const V<T> (&xbar)[NR],
                                              T power, int K) {
    V<T> g[NR][32 * NR];
    MvOut<T> res;
    res.ok = true;
    res.y = vz<C, T>();
    T gmin = T(INFINITY), gmax = T(0);
    V<T> az[NR], aw[NR], zf[NR], wf[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) {
        az[q] = vz<C, T>();
        az[q].re = T(1);
        aw[q] = xbar[q];
        zf[q] = vz<C, T>();
        wf[q] = vz<C, T>();
    }
#pragma unroll
    for (int j = 0; j < 32 * NR; j++) {
        if (j >= L) break;
        V<T> acc[NR], acc2[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const int i = lane + 32 * q;
            V<T> a = vz<C, T>();
            if (i < sz && j < sz) a = ldG<C, T>(Gs[i * GP + j]);
            if (i == j) a.re += loading;
            acc[q] = a;
            acc2[q] = vz<C, T>();
        }
#pragma unroll
        for (int k = 0; k + 1 < j; k += 2) {
            // rows have an even pitch: entries (j, k) and (j, k + 1) are one aligned pair
            V<T> gjk, gjk1;
            if constexpr (C) {
                const float4 p = *reinterpret_cast<const float4*>(&Gs[j * GP + k]);
                gjk = V<T>{p.x, p.y};
                gjk1 = V<T>{p.z, p.w};
            } else {
                const float2 p = *reinterpret_cast<const float2*>(&Gs[j * GP + k]);
                gjk = V<T>{p.x, T(0)};
                gjk1 = V<T>{p.y, T(0)};
            }
#pragma unroll
            for (int q = 0; q < NR; q++) {
                mscConj<C, T>(acc[q], g[q][k], gjk);
                mscConj<C, T>(acc2[q], g[q][k + 1], gjk1);
            }
        }
        if (j & 1) {
            const V<T> gjk = ldG<C, T>(Gs[j * GP + j - 1]);
#pragma unroll
            for (int q = 0; q < NR; q++) mscConj<C, T>(acc[q], g[q][j - 1], gjk);
        }
#pragma unroll
        for (int q = 0; q < NR; q++) {
            acc[q].re += acc2[q].re;
            acc[q].im += acc2[q].im;
        }
        const T djj = __shfl_sync(kFull, acc[j >> 5].re, j & 31);
        if (!(djj > T(0))) {  // warp-uniform: the factorisation broke down
            res.ok = false;
            return res;
        }
        const T inv = rsqrtf(djj);  // MUFU reciprocal square root (about 2 ulp)
        const T gjj = djj * inv;
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const int i = lane + 32 * q;
            V<T> v = vz<C, T>();
            if (i > j) {
                v.re = acc[q].re * inv;
                v.im = acc[q].im * inv;
            } else if (i == j) {
                v.re = gjj;
            }
            g[q][j] = v;
            if (i < L) {
                Gs[i * GP + j].re = v.re;
                if constexpr (C) Gs[i * GP + j].im = v.im;
            }
        }
        __syncwarp();
        if (j < sz) {
            gmin = min(gmin, gjj);
            gmax = max(gmax, gjj);
            // forward substitution step j: row j is final, column j of G is known to every lane
            V<T> zk = shflV<C, T>(az[j >> 5], j & 31);
            V<T> wk = shflV<C, T>(aw[j >> 5], j & 31);
            zk.re *= inv;
            zk.im *= inv;
            wk.re *= inv;
            wk.im *= inv;
#pragma unroll
            for (int q = 0; q < NR; q++) {
                const int i = lane + 32 * q;
                if (i == j) {
                    zf[q] = zk;
                    wf[q] = wk;
                }
                if (i > j) {
                    msc<C, T>(az[q], g[q][j], zk);
                    msc<C, T>(aw[q], g[q][j], wk);
                }
            }
        }
    }
    T zz = T(0);
    V<T> zw = vz<C, T>();
#pragma unroll
    for (int q = 0; q < NR; q++) {
        zz += zf[q].re * zf[q].re + zf[q].im * zf[q].im;
        macConj<C, T>(zw, wf[q], zf[q]);
    }
    zz = warpSum(zz);
    zw.re = warpSum(zw.re);
    if constexpr (C) zw.im = warpSum(zw.im);
    const T scale = T(1) / (zz * pow(static_cast<T>(K), power));
    res.y.re = zw.re * scale;
    res.y.im = zw.im * scale;
    res.cond = gmin > T(0) ? (gmax / gmin) * (gmax / gmin) : T(INFINITY);
    return res;
}

// The Cholesky and forward substitutions of solveRegs for complex data with one row per lane (L <= 32),
// the loaded matrix kept in two planes of floats (real parts at re, imaginary parts at im, row pitch
// GP). The inner products of column j run over pairs of columns (k, k + 1) in packed FMAs: each lane
// keeps its row of G negated, in pairs, so that every product is a natural packed operand:
//   re(A - sum g conj(b)) = A.re + sum (-g.re) b.re + sum (-g.im) b.im
//   im(A - sum g conj(b)) = (A.im + sum (-g.im) b.re) - sum (-g.re) b.im
// with b = G[j][k] read from the planes as pairs of floats.
__device__ __forceinline__ MvOut<float> solveRegsCplx(float* Gre, float* Gim, int GP, int L, int sz, float loading,
                                                      int lane, const V<float> (&xbar)[1], float power, int K) {
    float2 nr[16], ni[16];  // -G[lane][2m], -G[lane][2m + 1]: real and imaginary parts
    MvOut<float> res;
    res.ok = true;
    res.y = vz<true, float>();
    float gmin = INFINITY, gmax = 0.0f;
    V<float> az = vz<true, float>(), aw = xbar[0], zf = vz<true, float>(), wf = vz<true, float>();
    az.re = 1.0f;
    const int i = lane;
#pragma unroll
    for (int j = 0; j < 32; j++) {
        if (j >= L) break;
        float are = 0.0f, aim = 0.0f;
        if (i < sz && j < sz) {
            are = Gre[i * GP + j];
            aim = Gim[i * GP + j];
        }
        if (i == j) are += loading;
        float2 accR = make_float2(are, 0.0f), accIp = make_float2(aim, 0.0f), accIn = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int k = 0; k + 1 < j; k += 2) {
            // entries (j, k) and (j, k + 1): rows have an even pitch, so each plane's pair is aligned
            const float2 bR = *reinterpret_cast<const float2*>(&Gre[j * GP + k]);
            const float2 bI = *reinterpret_cast<const float2*>(&Gim[j * GP + k]);
            accR = __ffma2_rn(nr[k / 2], bR, accR);
            accR = __ffma2_rn(ni[k / 2], bI, accR);
            accIp = __ffma2_rn(ni[k / 2], bR, accIp);
            accIn = __ffma2_rn(nr[k / 2], bI, accIn);
        }
        if (j & 1) {
            const float bre = Gre[j * GP + j - 1], bim = Gim[j * GP + j - 1];
            accR.x = fmaf(nr[(j - 1) / 2].x, bre, accR.x);
            accR.x = fmaf(ni[(j - 1) / 2].x, bim, accR.x);
            accIp.x = fmaf(ni[(j - 1) / 2].x, bre, accIp.x);
            accIn.x = fmaf(nr[(j - 1) / 2].x, bim, accIn.x);
        }
        const float accRe = accR.x + accR.y;
        const float accIm = (accIp.x + accIp.y) - (accIn.x + accIn.y);
        const float djj = __shfl_sync(kFull, accRe, j & 31);
        if (!(djj > 0.0f)) {  // warp-uniform: the factorisation broke down
            res.ok = false;
            return res;
        }
        const float inv = rsqrtf(djj);  // MUFU reciprocal square root (about 2 ulp)
        const float gjj = djj * inv;
        float vre = 0.0f, vim = 0.0f;
        if (i > j) {
            vre = accRe * inv;
            vim = accIm * inv;
        } else if (i == j) {
            vre = gjj;
        }
        if (j & 1) {
            nr[j / 2].y = -vre;
            ni[j / 2].y = -vim;
        } else {
            nr[j / 2].x = -vre;
            ni[j / 2].x = -vim;
        }
        if (i < L) {
            Gre[i * GP + j] = vre;
            Gim[i * GP + j] = vim;
        }
        __syncwarp();
        if (j < sz) {
            gmin = fminf(gmin, gjj);
            gmax = fmaxf(gmax, gjj);
            V<float> zk = shflV<true, float>(az, j & 31);
            V<float> wk = shflV<true, float>(aw, j & 31);
            zk.re *= inv;
            zk.im *= inv;
            wk.re *= inv;
            wk.im *= inv;
            if (i == j) {
                zf = zk;
                wf = wk;
            }
            if (i > j) {
                const V<float> g{vre, vim};
                msc<true, float>(az, g, zk);
                msc<true, float>(aw, g, wk);
            }
        }
    }
    float zz = zf.re * zf.re + zf.im * zf.im;
    V<float> zw = vz<true, float>();
    macConj<true, float>(zw, wf, zf);
    zz = warpSum(zz);
    zw.re = warpSum(zw.re);
    zw.im = warpSum(zw.im);
    const float scale = 1.0f / (zz * pow(static_cast<float>(K), power));
    res.y.re = zw.re * scale;
    res.y.im = zw.im * scale;
    res.cond = gmin > 0.0f ? (gmax / gmin) * (gmax / gmin) : INFINITY;
    return res;
}

// RxBeamformerMVpcg (Beamformer/RxBeamformerMVpcg.cu:450-546, 548-620) on the sz x sz loaded system
// R a = 1, real data: Jacobi-preconditioned conjugate gradients from x = 1 with the residual
// recomputed from x every iteration (reinitialisation frequency 1), stopping after maxIt iterations,
// when r.s <= 1e-30 or when |r| <= thr; then y = sum_v xbar_v a_v / (sum_v a_v * K^p). Row i of R
// sits in registers of lane i % 32 (q = i / 32); R v broadcasts v_j from its lane.
template <int NR, class GE>
__device__ __forceinline__ MvOut<float> solvePcgRegs(const GE* Gs, int GP, float* vbuf, int sz, float loading, int lane,
                                                     const V<float> (&xbar)[NR], float power, int K, int maxIt, float thr) {
    // R stays in the shared-memory tile (rows of pitch GP, read as aligned pairs); the covariance
    // accumulators of the sliding window are live across the solve, so R is not copied to registers
    float dg[NR];
    bool valid[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) {
        const int i = lane + 32 * q;
        valid[q] = i < sz;
        dg[q] = valid[q] ? Gs[i * GP + i].re + loading : 1.0f;
    }
    // o = R v on the sz x sz block. The loop runs over whole groups of four columns (a warp-uniform
    // trip count, no per-column branch): the vectors are zero on rows >= sz, so the columns past sz
    // (finite window sums of the tile) contribute nothing. Four independent accumulators per row.
    // v is staged in the warp's vector buffer (32 NR floats) and read as 16-byte broadcasts: one
    // shared-memory read per four columns instead of four shuffles (the SM's shuffle unit is shared
    // by all its warps; the two products per iteration would otherwise issue 16 NR shuffles per row group)
    const int jmax = (sz + 3) & ~3;
    auto matvec = [&](const float (&v)[NR], float (&o)[NR]) {
        float p4[NR][4];
#pragma unroll
        for (int q = 0; q < NR; q++)
#pragma unroll
            for (int c = 0; c < 4; c++) p4[q][c] = 0.0f;
        __syncwarp();  // the previous product's reads of vbuf are done
#pragma unroll
        for (int q = 0; q < NR; q++) vbuf[lane + 32 * q] = v[q];
        __syncwarp();
        for (int j = 0; j < jmax; j += 4) {
            const float4 vv = *reinterpret_cast<const float4*>(vbuf + j);
            const float vj[4] = {vv.x, vv.y, vv.z, vv.w};
#pragma unroll
            for (int q = 0; q < NR; q++) {
                const GE* row = &Gs[(valid[q] ? lane + 32 * q : 0) * GP + j];
                const float2 a0 = *reinterpret_cast<const float2*>(row);
                const float2 a1 = *reinterpret_cast<const float2*>(row + 2);
                p4[q][0] = fmaf(a0.x, vj[0], p4[q][0]);
                p4[q][1] = fmaf(a0.y, vj[1], p4[q][1]);
                p4[q][2] = fmaf(a1.x, vj[2], p4[q][2]);
                p4[q][3] = fmaf(a1.y, vj[3], p4[q][3]);
            }
        }
#pragma unroll
        for (int q = 0; q < NR; q++)
            o[q] = valid[q] ? fmaf(loading, v[q], (p4[q][0] + p4[q][1]) + (p4[q][2] + p4[q][3])) : 0.0f;
    };
    auto dot = [&](const float (&u)[NR], const float (&w)[NR]) {
        float acc = 0.0f;
#pragma unroll
        for (int q = 0; q < NR; q++) acc = fmaf(u[q], w[q], acc);
        return warpSum(acc);
    };
    float x[NR], r[NR], d[NR], t[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) x[q] = valid[q] ? 1.0f : 0.0f;
    matvec(x, t);
#pragma unroll
    for (int q = 0; q < NR; q++) {
        r[q] = valid[q] ? fmaf(-1.0f, t[q], 1.0f) : 0.0f;
        d[q] = r[q] / dg[q];
    }
    float deltaNew = dot(r, d);
    float residualNorm = 2.0f * thr;
    for (int it = 0; it < maxIt && static_cast<double>(deltaNew) > 1e-30 && residualNorm > thr; it++) {
        matvec(d, t);  // q = A d
        const float alpha = deltaNew / dot(d, t);
#pragma unroll
        for (int q = 0; q < NR; q++) x[q] = fmaf(alpha, d[q], x[q]);
        matvec(x, t);  // r = b - A x
#pragma unroll
        for (int q = 0; q < NR; q++) r[q] = valid[q] ? fmaf(-1.0f, t[q], 1.0f) : 0.0f;
        float sv[NR];
        float rr = 0.0f, rs = 0.0f;
#pragma unroll
        for (int q = 0; q < NR; q++) {
            sv[q] = r[q] / dg[q];
            rr = fmaf(r[q], r[q], rr);
            rs = fmaf(r[q], sv[q], rs);
        }
        // the two reductions interleaved (independent shuffle chains)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            rr += __shfl_xor_sync(kFull, rr, o);
            rs += __shfl_xor_sync(kFull, rs, o);
        }
        residualNorm = sqrtf(rr);
        const float deltaOld = deltaNew;
        deltaNew = rs;
        const float beta = deltaNew / deltaOld;
#pragma unroll
        for (int q = 0; q < NR; q++) d[q] = fmaf(beta, d[q], sv[q]);
    }
    float asum = 0.0f, y = 0.0f;
#pragma unroll
    for (int q = 0; q < NR; q++) asum += x[q];
    asum = warpSum(asum);
    const float ws = 1.0f / (asum * powf(static_cast<float>(K), power));
#pragma unroll
    for (int q = 0; q < NR; q++) y += xbar[q].re * x[q] * ws;
    MvOut<float> res;
    res.ok = true;
    res.y = V<float>{warpSum(y), 0.0f};
    res.cond = 0.0f;
    return res;
}

// Same factorisation and substitutions in FP64 with the rows kept in shared memory (used only for
// the queued systems).
template <bool C, int NR>
__device__ MvOut<double> solveSmem64(V<double>* Gs, int GP, int L, int sz, double loading, int lane,
                                     const V<double> (&xbar)[NR], double power, int K) {
    MvOut<double> res;
    res.ok = true;
    res.y = vz<C, double>();
    res.cond = 0.0;
    // apply the loading and the unused-block rule in place
    for (int idx = lane; idx < L * L; idx += 32) {
        const int i = idx / L, j = idx % L;
        V<double>& e = Gs[i * GP + j];
        if (!(i < sz && j < sz)) e = vz<C, double>();
        if (i == j) e.re += loading;
    }
    __syncwarp();
    for (int j = 0; j < L; j++) {
        V<double> acc[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const int i = lane + 32 * q;
            acc[q] = i < L ? Gs[i * GP + j] : vz<C, double>();
            if (i >= j && i < L)
                for (int k = 0; k < j; k++) mscConj<C, double>(acc[q], Gs[i * GP + k], Gs[j * GP + k]);
        }
        const double djj = __shfl_sync(kFull, acc[j >> 5].re, j & 31);
        if (!(djj > 0.0)) {
            res.ok = false;
            return res;
        }
        const double gjj = sqrt(djj);
        __syncwarp();
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const int i = lane + 32 * q;
            if (i < L) {
                V<double> v = vz<C, double>();
                if (i > j) {
                    v.re = acc[q].re / gjj;
                    v.im = acc[q].im / gjj;
                } else if (i == j) {
                    v.re = gjj;
                }
                Gs[i * GP + j] = v;
            }
        }
        __syncwarp();
    }
    V<double> az[NR], aw[NR], zf[NR], wf[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) {
        az[q] = vz<C, double>();
        az[q].re = 1.0;
        aw[q] = xbar[q];
        zf[q] = vz<C, double>();
        wf[q] = vz<C, double>();
    }
    for (int k = 0; k < sz; k++) {
        const double gkk = Gs[k * GP + k].re;
        V<double> zk = shflV<C, double>(k >= 32 ? az[NR - 1] : az[0], k & 31);
        V<double> wk = shflV<C, double>(k >= 32 ? aw[NR - 1] : aw[0], k & 31);
        zk.re /= gkk;
        zk.im /= gkk;
        wk.re /= gkk;
        wk.im /= gkk;
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const int i = lane + 32 * q;
            if (i == k) {
                zf[q] = zk;
                wf[q] = wk;
            }
            if (i > k && i < L) {
                const V<double> gik = Gs[i * GP + k];
                msc<C, double>(az[q], gik, zk);
                msc<C, double>(aw[q], gik, wk);
            }
        }
    }
    double zz = 0.0;
    V<double> zw = vz<C, double>();
#pragma unroll
    for (int q = 0; q < NR; q++) {
        zz += zf[q].re * zf[q].re + zf[q].im * zf[q].im;
        macConj<C, double>(zw, wf[q], zf[q]);
    }
    zz = warpSum(zz);
    zw.re = warpSum(zw.re);
    if constexpr (C) zw.im = warpSum(zw.im);
    const double scale = 1.0 / (zz * pow(static_cast<double>(K), power));
    res.y.re = zw.re * scale;
    res.y.im = zw.im * scale;
    return res;
}

template <class Out> __device__ __forceinline__ void storeOut(Out* out, size_t idx, float re, float im);
template <> __device__ __forceinline__ void storeOut<float>(float* out, size_t idx, float re, float) {
    out[idx] = clampCast<float>(re);
}
template <> __device__ __forceinline__ void storeOut<int16_t>(int16_t* out, size_t idx, float re, float) {
    out[idx] = clampCast<int16_t>(re);
}
template <> __device__ __forceinline__ void storeOut<float2>(float2* out, size_t idx, float re, float im) {
    out[idx] = make_float2(re, im);
}

// |y| > 1e7 or NaN -> 0, then times numChannels (RxBeamformerMV.cu:366-375).
template <bool C, class T> __device__ __forceinline__ V<T> finishY(V<T> y, uint32_t nCh) {
    const T mag = C ? sqrt(y.re * y.re + y.im * y.im) : abs(y.re);
    if (mag > T(1e7) || isnan(y.re) || isnan(y.im)) y = vz<C, T>();
    y.re *= static_cast<T>(nCh);
    y.im *= static_cast<T>(nCh);
    return y;
}

__device__ __forceinline__ void atomicMaxFloatBits(unsigned int* addr, float v) {
    if (!(v >= 0.0f)) v = FLT_MAX;  // NaN / infinite estimates count as the largest
    atomicMax(addr, __float_as_uint(fminf(v, FLT_MAX)));
}

__host__ __device__ constexpr size_t alignUp(size_t v, size_t a) { return (v + a - 1) / a * a; }

template <bool C, int NR> struct MvLayout {
    static constexpr int GR = 32 * NR;
    static constexpr int GP = 32 * NR + 2;  // even: pairs (k, k+1) of a row are 2-element aligned
    __host__ __device__ static size_t ringBytes(uint32_t slots, uint32_t pitch) {
        return alignUp(static_cast<size_t>(slots) * pitch * sizeof(Elem<C>), 16);
    }
    __host__ __device__ static size_t metaBytes(uint32_t slots) { return alignUp(slots * sizeof(SampleMeta), 16); }
    __host__ __device__ static size_t d0Bytes(uint32_t slots) {
        return alignUp(static_cast<size_t>(slots) * GR * sizeof(V<float>), 16);
    }
    __host__ __device__ static size_t gBytes() { return alignUp(static_cast<size_t>(GR) * GP * sizeof(Elem<C>), 16); }
    // the PCG solve's search vector (real data only), read back as 16-byte broadcasts
    __host__ __device__ static size_t vecBytes() { return C ? 0 : alignUp(static_cast<size_t>(GR) * sizeof(float), 16); }
    __host__ __device__ static size_t perWarp(uint32_t slots, uint32_t pitch) {
        return ringBytes(slots, pitch) + metaBytes(slots) + d0Bytes(slots) + gBytes() + vecBytes();
    }
};

__device__ __forceinline__ void cpAsync4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpAsync8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Starts the copy of sample t of one scanline into its ring slot (FP32 / complex input: cp.async,
// no registers held; int16 input is converted, so it is loaded synchronously in sampleMeta).
template <bool C, class In>
__device__ __forceinline__ void issueSample(const MvArgs& a, const In* xl, uint32_t t, Elem<C>* slot, int lane) {
    if constexpr (!std::is_same<In, int16_t>::value) {
        for (uint32_t ch = lane; ch < a.nCh; ch += 32) {
            const In* src = xl + static_cast<size_t>(ch) * a.nS + t;
            if constexpr (C) cpAsync8(&slot[ch], src);
            else cpAsync4(&slot[ch], src);
        }
        cpAsyncCommit();
    }
}

// Completes sample t in its slot and derives the aperture (first / last nonzero channel,
// computeSubArrayMasks RxBeamformerMV.cu:80-110): sz = min(L, l-f+1), and the K = l - sz - f + 2
// active subarrays start at f, f+1, ..., f+K-1. Channels past nCh are zero padding.
template <bool C, class In>
__device__ __forceinline__ SampleMeta sampleMeta(const MvArgs& a, const In* xl, uint32_t t, Elem<C>* slot, int lane) {
    if constexpr (std::is_same<In, int16_t>::value) {
        for (uint32_t ch = lane; ch < a.nCh; ch += 32) slot[ch].re = static_cast<float>(__ldg(xl + static_cast<size_t>(ch) * a.nS + t));
    } else {
        cpAsyncWaitAll();
    }
    __syncwarp();
    int first = -1, last = -1;
    for (uint32_t c0 = 0; c0 < a.nCh; c0 += 32) {
        const uint32_t ch = c0 + lane;
        bool nz = false;
        if (ch < a.nCh) {
            const Elem<C> v = slot[ch];
            nz = v.re != 0.0f;
            if constexpr (C) nz = nz || v.im != 0.0f;
        }
        const uint32_t m = __ballot_sync(kFull, nz);
        if (m) {
            if (first < 0) first = static_cast<int>(c0) + __ffs(m) - 1;
            last = static_cast<int>(c0) + 31 - __clz(m);
        }
    }
    SampleMeta md;
    md.f = first < 0 ? 0 : first;
    const int l = last < 0 ? 0 : last;
    md.sz = min(static_cast<int>(a.L), l - md.f + 1);
    md.K = l - md.sz - md.f + 2;
    md.pad = 0;
    return md;
}

// One warp per run of consecutive samples of one scanline inside one 2000-sample block.
// LT != 0 fixes the subarray length at compile time (L = LT), which folds the per-entry range checks
// of the unrolled loops. Real data with one row per lane runs two CTAs per SM (128 registers, a few
// spilled; both CTAs' shared memory fits): PCG solve 5.07 -> 4.70 ms, Cholesky 2.31 -> 2.28 ms on
// c0's 2000-depth raw-delayed data, bit-identical. Complex data and two rows per lane keep the whole
// register file (their window state alone is 128 registers).
template <bool C, int NR, bool SLIDE, int LT, class In, class Out>
__global__ void __launch_bounds__(32 * kMvMaxWarps, (C || NR > 1) ? 1 : 2) mvKernel(MvArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    using L_ = MvLayout<C, NR>;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t item = blockIdx.x * (blockDim.x >> 5) + warp;
    if (item >= a.numItems) return;
    const uint32_t line = item / a.runsPerLine, run = item % a.runsPerLine;
    const uint32_t blk = run / a.runsPerBlock, j = run % a.runsPerBlock;
    const uint32_t b0 = blk * a.blockLen;
    const uint32_t bEnd = min(a.nS, b0 + a.blockLen);  // exclusive
    const uint32_t sA = b0 + j * kMvRun;
    if (sA >= bEnd) return;
    const uint32_t sB = min(sA + kMvRun, bEnd);
    const int L = LT ? LT : static_cast<int>(a.L), T = static_cast<int>(a.T);
    const uint32_t R = a.ringSlots;

    unsigned char* base = smem + static_cast<size_t>(warp) * L_::perWarp(R, a.ringPitch);
    Elem<C>* ring = reinterpret_cast<Elem<C>*>(base);
    SampleMeta* meta = reinterpret_cast<SampleMeta*>(base + L_::ringBytes(R, a.ringPitch));
    V<float>* d0c = reinterpret_cast<V<float>*>(base + L_::ringBytes(R, a.ringPitch) + L_::metaBytes(R));
    Elem<C>* Gs = reinterpret_cast<Elem<C>*>(base + L_::ringBytes(R, a.ringPitch) + L_::metaBytes(R) + L_::d0Bytes(R));
    float* vbuf = reinterpret_cast<float*>(base + L_::ringBytes(R, a.ringPitch) + L_::metaBytes(R) + L_::d0Bytes(R) +
                                           L_::gBytes());
    const In* xl = static_cast<const In*>(a.in) + static_cast<size_t>(line) * a.nCh * a.nS;
    Out* out = static_cast<Out*>(a.out);

    // zero padding past nCh in every slot (written once; copies only touch channels < nCh)
    for (uint32_t i = lane; i < R * (a.ringPitch - a.nCh); i += 32) {
        const uint32_t sl = i / (a.ringPitch - a.nCh), ch = a.nCh + i % (a.ringPitch - a.nCh);
        ring[static_cast<size_t>(sl) * a.ringPitch + ch].re = 0.0f;
        if constexpr (C) ring[static_cast<size_t>(sl) * a.ringPitch + ch].im = 0.0f;
    }
    // the transposed window sums fill rows and columns < L of Gs; the rest stays 0 (the PCG products
    // run over whole groups of four columns)
    for (uint32_t i = lane; i < static_cast<uint32_t>(32 * NR) * L_::GP; i += 32) {
        Gs[i].re = 0.0f;
        if constexpr (C) Gs[i].im = 0.0f;
    }
    auto slotOf = [&](uint32_t t) -> Elem<C>* { return ring + static_cast<size_t>(t % R) * a.ringPitch; };
    auto complete = [&](uint32_t t) {
        const SampleMeta m = sampleMeta<C, In>(a, xl, t, slotOf(t), lane);
        if (lane == 0) meta[t % R] = m;
        __syncwarp();
    };

    V<float> hi[NR][32 * NR], lo[NR][32 * NR];
    // the first sample's window, then the sample that enters at the second step
    const uint32_t w0 = static_cast<uint32_t>(max(static_cast<int>(b0), static_cast<int>(sA) - T));
    const uint32_t w1 = min(bEnd - 1, sA + a.T);
    for (uint32_t t = w0; t <= w1; t++) {
        issueSample<C, In>(a, xl, t, slotOf(t), lane);
        complete(t);
    }
    if (sA + 1 < sB && w1 + 1 <= bEnd - 1) issueSample<C, In>(a, xl, w1 + 1, slotOf(w1 + 1), lane);

    unsigned long long systems = 0;
    float condMax = 0.0f;
    for (uint32_t s = sA; s < sB; s++) {
        const uint32_t t0 = static_cast<uint32_t>(max(static_cast<int>(b0), static_cast<int>(s) - T));
        const uint32_t t1 = min(bEnd - 1, s + a.T);
        const bool hasNew = s > sA && s + a.T <= bEnd - 1;
        if (hasNew) complete(s + a.T);
        bool fullWindow = true;
        if constexpr (SLIDE) fullWindow = s == sA;
        const bool hasOld = !fullWindow && static_cast<int>(s) - T - 1 >= static_cast<int>(b0);
        if (fullWindow) {
#pragma unroll
            for (int q = 0; q < NR; q++)
#pragma unroll
                for (int r = 0; r < 32 * NR; r++) {
                    hi[q][r] = vz<C, float>();
                    lo[q][r] = vz<C, float>();
                }
        }
        // one call site for the covariance updates: the whole window, or the entering and leaving sample
        const int nJobs = fullWindow ? static_cast<int>(t1 - t0 + 1) : static_cast<int>(hasNew) + static_cast<int>(hasOld);
        for (int jb = 0; jb < nJobs; jb++) {
            uint32_t t;
            float sign = 1.0f;
            bool fresh = true;
            if (fullWindow) t = t0 + jb;
            else if (jb == 0 && hasNew) t = s + a.T;
            else {
                t = s - a.T - 1;
                sign = -1.0f;
                fresh = false;
            }
            addCov<C, NR, SLIDE, float>(slotOf(t), meta[t % R], d0c + static_cast<size_t>(t % R) * L_::GR, fresh, L,
                                        lane, sign, hi, lo);
        }
        // prefetch the sample entering at the next step; its slot held sample s - T - 1, whose
        // subtraction above was the last use
        __syncwarp();
        if (s > sA && s + 1 < sB && s + a.T + 1 <= bEnd - 1)
            issueSample<C, In>(a, xl, s + a.T + 1, slotOf(s + a.T + 1), lane);
        // transpose the window sum into rows
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const int d = lane + 32 * q;
            if (d < L) {
#pragma unroll
                for (int r = 0; r < 32 * NR; r++) {
                    if (r >= L) break;
                    int c = r + d;
                    if (c >= L) c -= L;
                    if constexpr (C) {  // complex: real and imaginary planes
                        float* pl = reinterpret_cast<float*>(Gs);
                        pl[r * L_::GP + c] = hi[q][r].re + lo[q][r].re;
                        pl[L_::GR * L_::GP + r * L_::GP + c] = hi[q][r].im + lo[q][r].im;
                    } else {
                        Gs[r * L_::GP + c].re = hi[q][r].re + lo[q][r].re;
                    }
                }
            }
        }
        __syncwarp();
        const SampleMeta ms = meta[s % R];
        const Elem<C>* xs = slotOf(s);
        // trace of the sz x sz block and the loading (RxBeamformerMV.cu:239-276)
        float tr = 0.0f;
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const int i = lane + 32 * q;
            if (i < ms.sz) tr += C ? reinterpret_cast<const float*>(Gs)[i * L_::GP + i] : Gs[i * L_::GP + i].re;
        }
        tr = warpSum(tr);
        const float loading = (1.0f / static_cast<float>(ms.sz)) * tr * a.loadScale;
        // xbar_v = sum over the active subarrays of x[f + k + v]
        V<float> xbar[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const int i = lane + 32 * q;
            const int ii = i < ms.sz ? i : 0;
            V<float> acc0 = vz<C, float>(), acc1 = vz<C, float>();
            int k = 0;
            for (; k + 1 < ms.K; k += 2) {
                const V<float> v0 = ld<C, float>(xs[ms.f + k + ii]), v1 = ld<C, float>(xs[ms.f + k + 1 + ii]);
                acc0.re += v0.re;
                acc0.im += v0.im;
                acc1.re += v1.re;
                acc1.im += v1.im;
            }
            if (k < ms.K) {
                const V<float> v0 = ld<C, float>(xs[ms.f + k + ii]);
                acc0.re += v0.re;
                acc0.im += v0.im;
            }
            acc0.re += acc1.re;
            acc0.im += acc1.im;
            xbar[q] = i < ms.sz ? acc0 : vz<C, float>();
        }
        V<float> y = vz<C, float>();
        bool write = true;
        if (!C && a.pcg) {
            if constexpr (!C) {
                if (tr > 0.0f && isfinite(tr))
                    y = solvePcgRegs<NR, Elem<C>>(Gs, L_::GP, vbuf, ms.sz, loading, lane, xbar, a.power, ms.K, a.pcgMaxIt,
                                                  a.pcgThr).y;
            }
        } else if (tr > 0.0f && isfinite(tr)) {
            MvOut<float> r;
            if constexpr (C && NR == 1) {
                float* pl = reinterpret_cast<float*>(Gs);
                r = solveRegsCplx(pl, pl + L_::GR * L_::GP, L_::GP, L, ms.sz, loading, lane, xbar, a.power, ms.K);
            } else {
                r = solveRegs<C, NR, float, Elem<C>>(Gs, L_::GP, L, ms.sz, loading, lane, xbar, a.power, ms.K);
            }
            const float cond = r.ok ? r.cond : INFINITY;
            condMax = fmaxf(condMax, fminf(cond, FLT_MAX));
            if (a.thr > 0.0f && (!r.ok || cond > a.thr)) {
                write = false;
                if (lane == 0) {
                    const unsigned int qi = atomicAdd(&a.counters->queued, 1u);
                    a.queue[qi] = line * a.nS + s;
                }
            } else if (r.ok) {
                y = r.y;
            }
        }
        __syncwarp();
        if (write && lane == 0) {
            y = finishY<C, float>(y, a.nCh);
            storeOut<Out>(out, static_cast<size_t>(s) * a.nRx + line, y.re, y.im);
        }
        systems++;
    }
    if (lane == 0) {
        atomicAdd(&a.counters->systems, systems);
        atomicMaxFloatBits(&a.counters->maxCondBits, condMax);
    }
}

// FP64 re-solve of the queued systems: one warp per system, covariance accumulated in FP64 in
// shared memory, Cholesky and substitutions in FP64.
template <bool C, int NR, class In, class Out>
__global__ void __launch_bounds__(128) mvFp64Kernel(MvArgs a, uint32_t window) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int GP = 32 * NR + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int warpsPerCta = blockDim.x >> 5;
    const size_t ringBytes = alignUp(static_cast<size_t>(window) * a.ringPitch * sizeof(Elem<C>), 16);
    const size_t metaBytes = alignUp(window * sizeof(SampleMeta), 16);
    const size_t gBytes = static_cast<size_t>(32 * NR) * GP * sizeof(V<double>);
    unsigned char* base = smem + static_cast<size_t>(warp) * (ringBytes + metaBytes + gBytes);
    Elem<C>* ring = reinterpret_cast<Elem<C>*>(base);
    V<double>* Gs = reinterpret_cast<V<double>*>(base + ringBytes + metaBytes);
    const int L = static_cast<int>(a.L);
    const unsigned int nq = *reinterpret_cast<volatile unsigned int*>(&a.counters->queued);
    Out* out = static_cast<Out*>(a.out);
    for (unsigned int qi = blockIdx.x * warpsPerCta + warp; qi < nq; qi += gridDim.x * warpsPerCta) {
        const uint32_t id = a.queue[qi];
        const uint32_t line = id / a.nS, s = id % a.nS;
        const uint32_t b0 = (s / a.blockLen) * a.blockLen;
        const uint32_t bEnd = min(a.nS, b0 + a.blockLen);
        const uint32_t t0 = static_cast<uint32_t>(max(static_cast<int>(b0), static_cast<int>(s) - static_cast<int>(a.T)));
        const uint32_t t1 = min(bEnd - 1, s + a.T);
        const In* xl = static_cast<const In*>(a.in) + static_cast<size_t>(line) * a.nCh * a.nS;
        for (int idx = lane; idx < 32 * NR * GP; idx += 32) Gs[idx] = vz<C, double>();
        __syncwarp();
        SampleMeta ms{};
        for (uint32_t t = t0; t <= t1; t++) {
            Elem<C>* xv = ring + static_cast<size_t>(t - t0) * a.ringPitch;
            const SampleMeta m = loadSample<C, In>(a, xl, t, xv, lane);
            if (t == s) ms = m;
            // direct covariance: lane owns columns c = lane + 32q; R[r][c] += x[f+k+r] x*[f+k+c]
            for (int k = 0; k < m.K; k++) {
#pragma unroll
                for (int q = 0; q < NR; q++) {
                    const int c = lane + 32 * q;
                    if (c >= L) continue;
                    const V<double> xc = ld<C, double>(xv[m.f + k + c]);
                    for (int r = 0; r < L; r++) macConj<C, double>(Gs[r * GP + c], ld<C, double>(xv[m.f + k + r]), xc);
                }
            }
            __syncwarp();
        }
        const Elem<C>* xs = ring + static_cast<size_t>(s - t0) * a.ringPitch;
        double tr = 0.0;
        for (int i = lane; i < ms.sz; i += 32) tr += Gs[i * GP + i].re;
        tr = warpSum(tr);
        const double loading = (1.0 / ms.sz) * tr * static_cast<double>(a.loadScale);
        V<double> xbar[NR];
#pragma unroll
        for (int q = 0; q < NR; q++) {
            const int i = lane + 32 * q;
            V<double> acc = vz<C, double>();
            if (i < ms.sz)
                for (int k = 0; k < ms.K; k++) {
                    const V<double> v = ld<C, double>(xs[ms.f + k + i]);
                    acc.re += v.re;
                    acc.im += v.im;
                }
            xbar[q] = acc;
        }
        V<double> y = vz<C, double>();
        if (tr > 0.0 && isfinite(tr)) {
            const MvOut<double> r = solveSmem64<C, NR>(Gs, GP, L, ms.sz, loading, lane, xbar, static_cast<double>(a.power), ms.K);
            if (r.ok) y = r.y;
        }
        if (lane == 0) {
            y = finishY<C, double>(y, a.nCh);
            storeOut<Out>(out, static_cast<size_t>(s) * a.nRx + line, static_cast<float>(y.re), static_cast<float>(y.im));
            atomicAdd(&a.counters->fp64Systems, 1ull);
        }
        __syncwarp();
    }
}

template <bool C, int NR, class In, class Out>
int launchMv(MvArgs& a, cudaStream_t st) {
    using L_ = MvLayout<C, NR>;
    const size_t perWarp = L_::perWarp(a.ringSlots, a.ringPitch);
    const int warps = static_cast<int>(std::min<size_t>(kMvMaxWarps, kMvSmemBudget / perWarp));
    if (warps < 1)
        return fail(SB_ERR_UNSUPPORTED, "sb_mv_run: %u channels with temporal smoothing %u need %zu bytes of shared memory per warp",
                    a.nCh, a.T, perWarp);
    const size_t smemBytes = perWarp * warps;
    constexpr bool SLIDE = NR == 1;
    // L = 32 (one row per lane) is specialised; for two rows per lane the folded variant exceeds the
    // register file, so it keeps the runtime length
    auto kern = (NR == 1 && a.L == 32u) ? mvKernel<C, NR, SLIDE, NR == 1 ? 32 : 0, In, Out>
                                         : mvKernel<C, NR, SLIDE, 0, In, Out>;
    SB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smemBytes)));
    const uint32_t grid = (a.numItems + warps - 1) / warps;
    kern<<<grid, 32 * warps, smemBytes, st>>>(a);
    SB_CHECK_LAUNCH("mvKernel");
    if (a.thr > 0.0f) {
        const uint32_t window = 2 * a.T + 1;
        const size_t per64 = alignUp(static_cast<size_t>(window) * a.ringPitch * sizeof(Elem<C>), 16) +
                             alignUp(window * sizeof(SampleMeta), 16) +
                             static_cast<size_t>(32 * NR) * (32 * NR + 1) * sizeof(V<double>);
        const int w64 = static_cast<int>(std::min<size_t>(4, kMvSmemBudget / per64));
        if (w64 < 1) return fail(SB_ERR_UNSUPPORTED, "sb_mv_run: FP64 re-solve needs %zu bytes of shared memory", per64);
        auto k64 = mvFp64Kernel<C, NR, In, Out>;
        SB_CUDA(cudaFuncSetAttribute(k64, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(per64 * w64)));
        k64<<<2 * smCount(), 32 * w64, per64 * w64, st>>>(a, window);
        SB_CHECK_LAUNCH("mvFp64Kernel");
    }
    return SB_OK;
}

template <bool C, class In, class Out> int dispatchNR(MvArgs& a, cudaStream_t st) {
    if (a.L <= 32) return launchMv<C, 1, In, Out>(a, st);
    if constexpr (!C) return launchMv<C, 2, In, Out>(a, st);
    return fail(SB_ERR_UNSUPPORTED, "sb_mv_run: complex data supports subarrays of at most 32 channels (got %u)", a.L);
}

}  // namespace
}  // namespace sb

using namespace sb;

namespace {

// Shared body of sb_mv_run and sb_mv_pcg_run: blockLen clips the temporal windows, pcgMaxIt > 0
// selects the PCG solve.
int mvRun(const void* raw_delayed, int in_dtype, void* out, int out_dtype, uint32_t num_scanlines,
          uint32_t num_channels, uint32_t num_samples, uint32_t subarray_size, uint32_t temporal_smoothing,
          double subarray_scaling_power, int compute_means, float loading_scale, float fp64_threshold,
          sb_mv_stats* stats_host, sb_stream stream, uint32_t blockLen, int pcgMaxIt, float pcgThr) {
    SB_REQUIRE(raw_delayed && out, "sb_mv_run: null pointer");
    SB_REQUIRE(num_scanlines > 0 && num_channels > 0 && num_samples > 0, "sb_mv_run: empty input");
    if (compute_means)
        return fail(SB_ERR_UNSUPPORTED,
                    "sb_mv_run: computeMeans is not supported (the reference indexes its mean buffers out of range)");
    const uint32_t L = subarray_size == 0 ? num_channels / 2 : subarray_size;
    SB_REQUIRE(L >= 1 && L <= num_channels, "sb_mv_run: subarray size %u out of range for %u channels", L, num_channels);
    if (L > 64) return fail(SB_ERR_UNSUPPORTED, "sb_mv_run: subarrays of at most 64 channels are supported (got %u)", L);
    SB_REQUIRE(temporal_smoothing <= 64, "sb_mv_run: temporal smoothing %u > 64", temporal_smoothing);
    SB_REQUIRE(static_cast<uint64_t>(num_scanlines) * num_samples < (1ull << 32), "sb_mv_run: too many samples");
    const bool cplx = in_dtype == SB_COMPLEX64;
    if (cplx) SB_REQUIRE(out_dtype == SB_COMPLEX64, "sb_mv_run: complex input needs SB_COMPLEX64 output");
    else {
        SB_REQUIRE(in_dtype == SB_FLOAT32 || in_dtype == SB_INT16, "sb_mv_run: input dtype must be float32, int16 or complex64");
        SB_REQUIRE(out_dtype == SB_FLOAT32 || out_dtype == SB_INT16, "sb_mv_run: real input needs float32 or int16 output");
    }
    cudaStream_t st = S(stream);
    MvArgs a{};
    a.in = raw_delayed;
    a.out = out;
    a.nRx = num_scanlines;
    a.nCh = num_channels;
    a.nS = num_samples;
    a.L = L;
    a.T = temporal_smoothing;
    a.ringSlots = 2 * temporal_smoothing + 2;
    // channel reads reach index nCh - 1 + L - 1 (apertures narrower than L); padding is zero
    a.ringPitch = (num_channels + (L <= 32 ? 32 : 64) + 31) / 32 * 32;
    a.blockLen = blockLen;
    a.runsPerBlock = (blockLen + kMvRun - 1) / kMvRun;
    const uint32_t nBlocks = (num_samples + blockLen - 1) / blockLen;
    a.runsPerLine = nBlocks * a.runsPerBlock;
    a.numItems = num_scanlines * a.runsPerLine;
    a.power = static_cast<float>(subarray_scaling_power);
    a.loadScale = loading_scale;
    a.thr = fp64_threshold;
    a.pcg = pcgMaxIt > 0 ? 1 : 0;
    a.pcgMaxIt = pcgMaxIt;
    a.pcgThr = pcgThr;

    // scratch: counters, and the FP64 queue when the re-solve is enabled
    const size_t qBytes = fp64_threshold > 0.0f ? static_cast<size_t>(num_scanlines) * num_samples * sizeof(uint32_t) : 0;
    void* scratch = nullptr;
    SB_CUDA(cudaMallocAsync(&scratch, sizeof(MvCounters) + qBytes, st));
    a.counters = static_cast<MvCounters*>(scratch);
    a.queue = qBytes ? reinterpret_cast<uint32_t*>(static_cast<char*>(scratch) + sizeof(MvCounters)) : nullptr;
    int rc = SB_OK;
    if (cudaMemsetAsync(a.counters, 0, sizeof(MvCounters), st) != cudaSuccess) rc = cudaFail(cudaGetLastError(), "cudaMemsetAsync");
    if (rc == SB_OK) {
        if (cplx) rc = dispatchNR<true, float2, float2>(a, st);
        else if (in_dtype == SB_FLOAT32 && out_dtype == SB_FLOAT32) rc = dispatchNR<false, float, float>(a, st);
        else if (in_dtype == SB_FLOAT32) rc = dispatchNR<false, float, int16_t>(a, st);
        else if (out_dtype == SB_FLOAT32) rc = dispatchNR<false, int16_t, float>(a, st);
        else rc = dispatchNR<false, int16_t, int16_t>(a, st);
    }
    if (rc == SB_OK && stats_host) {
        MvCounters c{};
        if (cudaMemcpyAsync(&c, a.counters, sizeof(c), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = cudaFail(cudaGetLastError(), "sb_mv_run stats");
        else {
            stats_host->systems = c.systems;
            stats_host->fp64_systems = c.fp64Systems;
            float m;
            std::memcpy(&m, &c.maxCondBits, sizeof(m));
            stats_host->max_condition_estimate = m;
        }
    }
    cudaFreeAsync(scratch, st);
    return rc;
}

}  // namespace

extern "C" int sb_mv_run(const void* raw_delayed, int in_dtype, void* out, int out_dtype, uint32_t num_scanlines,
                         uint32_t num_channels, uint32_t num_samples, uint32_t subarray_size, uint32_t temporal_smoothing,
                         double subarray_scaling_power, int compute_means, float loading_scale, float fp64_threshold,
                         sb_mv_stats* stats_host, sb_stream stream) {
    return mvRun(raw_delayed, in_dtype, out, out_dtype, num_scanlines, num_channels, num_samples, subarray_size,
                 temporal_smoothing, subarray_scaling_power, compute_means, loading_scale, fp64_threshold, stats_host,
                 stream, kMvBlock, 0, 0.0f);
}

extern "C" int sb_mv_pcg_run(const void* raw_delayed, int in_dtype, void* out, int out_dtype, uint32_t num_scanlines,
                             uint32_t num_channels, uint32_t num_samples, uint32_t subarray_size,
                             uint32_t temporal_smoothing, uint32_t max_iterations_override, double convergence_threshold,
                             double subarray_scaling_power, int compute_means, float loading_scale, sb_stream stream) {
    SB_REQUIRE(in_dtype != SB_COMPLEX64, "sb_mv_pcg_run: the PCG solve takes real data (float32 or int16)");
    SB_REQUIRE(convergence_threshold >= 0.0, "sb_mv_pcg_run: negative convergence threshold");
    const uint32_t L = subarray_size == 0 ? num_channels / 2 : subarray_size;
    // RxBeamformerMVpcg.cu:649: maxIterations = subArraySize unless overridden
    const uint32_t maxIt = max_iterations_override == 0 ? L : max_iterations_override;
    SB_REQUIRE(maxIt >= 1 && maxIt <= 100000, "sb_mv_pcg_run: iteration count %u out of range", maxIt);
    // no sample blocks: the PCG reference smooths over +-T clipped only at the record ends
    return mvRun(raw_delayed, in_dtype, out, out_dtype, num_scanlines, num_channels, num_samples, subarray_size,
                 temporal_smoothing, subarray_scaling_power, compute_means, loading_scale, 0.0f, nullptr, stream,
                 std::max<uint32_t>(num_samples, 1), static_cast<int>(maxIt), static_cast<float>(convergence_threshold));
}
