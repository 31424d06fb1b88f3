// gx_device.cuh -- device building blocks shared by the askAdam and MCMC
// kernels: acquisition protocol, Philox4x32-10, elementwise losses (with the
// Rician log-Bessel terms) and the per-voxel forward models with their
// tangent (dS/dtheta) accumulation.  All reference citations are paths in
// kschan0214/gacelle.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define GX_HD __host__ __device__ __forceinline__
#else
#define GX_HD inline
#endif

namespace gx {

constexpr int kMaxTE = 64;
constexpr int kPairTE = 16;  // echoes of the pair variant of the persistent TV kernel
constexpr int kMaxFA = 16;
constexpr int kMaxShell = 64;
constexpr int kMaxParam = 6;  // fitted parameters + noise
constexpr int kMaxMeas = 128;

enum ModelId { kR2S = 1, kR1R2S = 2, kNEXI = 3, kNEXI2 = 4 };
constexpr int kRiceNodes = 34;  // mybesseli trapezoid nodes (NEXI/gpuNEXIrice.m:752)
enum LossId { kL1 = 0, kL2 = 1, kHuber = 2, kMSE = 3, kGauss = 4, kRician = 5 };
enum OptId { kAdam = 0, kSGDM = 1, kRMSProp = 2 };

// Acquisition protocol, passed by value as a kernel parameter (constant
// bank): every thread of a warp reads the same element, which the constant
// cache broadcasts.
struct DevProtocol {
    int model;   // ModelId; NEXI with lmax = 2 is kNEXI2
    int nm;      // measurements
    int np;      // fitted parameters (without noise)
    int n_te, n_fa, n_shell, nx;
    float tr;    // [s]
    float h;     // NEXI node spacing 1/(nx-1)
    float te[kMaxTE];
    float te_l2e[kMaxTE];   // te * log2(e): exp(-te R2*) = 2^(-te_l2e R2*)
    // the first kPairTE of te and -te_l2e duplicated into (x, x) pairs: 64-bit
    // operands of the two-voxel pair instructions
    float2 te_pair[kPairTE];
    float2 nl2e_pair[kPairTE];
    float fa_rad[kMaxFA];
    float bval[kMaxShell];
    float delta[kMaxShell];
    float lb[kMaxParam], ub[kMaxParam];
    // NEXI Rician mean (gpuNEXIrice): interior nodes t_i = i pi / 33, i = 1..32,
    // of the 34-node Bessel trapezoids: cos(t_i) - 1 and sin(t_i)^2
    int rice;
    float rice_cm1[kRiceNodes - 2];
    float rice_s2[kRiceNodes - 2];
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11).  Counter words are
// (a, b, c, tag); the key is the 64-bit seed.
// ---------------------------------------------------------------------------
struct U4 { uint32_t x, y, z, w; };

GX_HD U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed) {
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return U4{c0, c1, c2, c3};
}

// Uniform on (0,1) from 23 random bits: exactly representable in FP32.
GX_HD float u01(uint32_t x) { return ((float)(x >> 9) + 0.5f) * (1.0f / 8388608.0f); }
GX_HD uint32_t rand_below(uint32_t x, uint32_t n) { return (uint32_t)(((uint64_t)x * n) >> 32); }

enum RngTag : uint32_t { kTagAdamInit = 1, kTagGwInit = 2, kTagGwMove = 3, kTagGwPerm = 4,
                         kTagGwRbPart = 5, kTagMhMove = 6, kTagGwGPerm = 7, kTagGwGRbPart = 8,
                         kTagGwGMove = 9, kTagGwGInit = 10 };
// flag bits above the tag: red-black move, global warm-up step; the
// repetition index sits in bits 16-31
constexpr uint32_t kTagRedBlack = 1u << 8;
constexpr uint32_t kTagWarmup = 1u << 9;

#if defined(__CUDACC__)
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, float& n0, float& n1) {
    float u1 = u01(a), u2 = u01(b);
    float r = sqrtf(-2.0f * logf(u1));
    float s, c;
    sincospif(2.0f * u2, &s, &c);
    n0 = r * c;
    n1 = r * s;
}
#endif

// ---------------------------------------------------------------------------
// Rician log-likelihood terms.  I0 and I1 from the polynomial approximations
// of Abramowitz & Stegun 9.8.1-9.8.4 (|x| < 3.75: series in (x/3.75)^2;
// |x| >= 3.75: x^(1/2) e^(-x) I_nu(x) as a polynomial in 3.75/x).  For the
// large-argument branch 1 - I1/I0 is evaluated as (P0 - P1)/P0 with the
// coefficient differences taken exactly, so the gradient term does not cancel.
// log_i0e = log(exp(-|x|) I0(x));  omr = 1 - I1(x)/I0(x).
// ---------------------------------------------------------------------------
GX_HD void rician_terms(float x, float& log_i0e, float& omr) {
    float ax = fabsf(x);
    float r;  // 1 - I1(|x|)/I0(|x|)
    if (ax < 3.75f) {
        float t = ax * (1.0f / 3.75f);
        float t2 = t * t;
        float i0 = 1.0f + t2 * (3.5156229f + t2 * (3.0899424f + t2 * (1.2067492f +
                   t2 * (0.2659732f + t2 * (0.0360768f + t2 * 0.0045813f)))));
        float i1x = 0.5f + t2 * (0.87890594f + t2 * (0.51498869f + t2 * (0.15084934f +
                    t2 * (0.02658733f + t2 * (0.00301532f + t2 * 0.00032411f)))));
        log_i0e = logf(i0) - ax;
        r = 1.0f - ax * i1x / i0;
    } else {
        float u = 3.75f / ax;
        float p0 = 0.39894228f + u * (0.01328592f + u * (0.00225319f + u * (-0.00157565f +
                   u * (0.00916281f + u * (-0.02057706f + u * (0.02635537f +
                   u * (-0.01647633f + u * 0.00392377f)))))));
        float d = u * (0.05316616f + u * (0.00587337f + u * (-0.00321366f + u * (0.01947836f +
                  u * (-0.04340673f + u * (0.05530849f + u * (-0.03435287f +
                  u * 0.00812436f)))))));
        log_i0e = logf(p0) - 0.5f * logf(ax);
        r = d / p0;
    }
    omr = x >= 0.0f ? r : 2.0f - r;  // I1 is odd: 1 - R(-a) = 1 + R(a)
}

// Per-voxel constants of the likelihood losses.
struct LossAux {
    float inv_s2;     // 1/sigma^2
    float gauss_c;    // 0.5*log(2*pi*sigma^2)
};

GX_HD LossAux make_loss_aux(float sigma) {
    LossAux a;
    a.inv_s2 = 1.0f / (sigma * sigma);
    a.gauss_c = 0.5f * logf(6.283185307179586f * sigma * sigma);
    return a;
}

// Elementwise loss value and derivative with respect to the prediction s
// (utils/askadam.m:86-95 for l1/l2/huber/mse with Reduction="none").
template <int LOSS>
GX_HD float loss_elem(float s, float y, float w, const LossAux& a, float mse_scale,
                      float hd, float& d) {
    float r = s - y;
    if (LOSS == kL1) {
        d = w * (float)((r > 0.0f) - (r < 0.0f));
        return w * fabsf(r);
    } else if (LOSS == kL2) {
        d = 2.0f * w * r;
        return w * r * r;
    } else if (LOSS == kHuber) {
        float ar = fabsf(r);
        if (ar <= hd) {
            d = w * r;
            return w * 0.5f * r * r;
        }
        d = w * hd * (float)((r > 0.0f) - (r < 0.0f));
        return w * (hd * ar - 0.5f * hd * hd);
    } else if (LOSS == kMSE) {
        d = 2.0f * mse_scale * r;
        return mse_scale * r * r;
    } else if (LOSS == kGauss) {
        d = w * r * a.inv_s2;
        return w * (0.5f * r * r * a.inv_s2 + a.gauss_c);
    } else {  // kRician: (y-s)^2/(2 s2) - log(i0e(y s / s2)) - log(y / s2)
        float x = y * s * a.inv_s2;
        float lg, omr;
        rician_terms(x, lg, omr);
        float c = y > 0.0f ? -logf(y * a.inv_s2) : 0.0f;
        d = w * (r * a.inv_s2 + y * a.inv_s2 * omr);
        return w * (0.5f * r * r * a.inv_s2 - lg + c);
    }
}

#if defined(__CUDACC__)

// ---------------------------------------------------------------------------
// FP32 operations with explicit rounding (to nearest, subnormals flushed), on
// scalars and on packed pairs (PTX f32x2: one instruction for two lanes of a
// 64-bit register pair).  The optimiser, the parameter transform and the
// R2*/MSE sums are written with these in every kernel, so that a kernel that
// updates two voxels per thread with pair instructions produces bit for bit
// what the one-voxel-per-thread kernels produce.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float add1(float a, float b) {
    float d;
    asm("add.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float sub1(float a, float b) {
    float d;
    asm("sub.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float mul1(float a, float b) {
    float d;
    asm("mul.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float fma1(float a, float b, float c) {
    float d;
    asm("fma.rn.ftz.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
// 2^x and 1/x by the PTX approximations (ex2.approx, rcp.approx), subnormals
// flushed; exp(x) = 2^(x log2 e) and a / b = a * (1/b) are built on them.
__device__ __forceinline__ float ex2_ftz(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kLog2e = 1.4426950408889634f;

__device__ __forceinline__ unsigned long long pk2(float2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long r) {
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    unsigned long long d;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)));
    return upk2(d);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)));
    return upk2(d);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    unsigned long long d;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)));
    return upk2(d);
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    unsigned long long d;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)), "l"(pk2(c)));
    return upk2(d);
}
__device__ __forceinline__ float2 bcast2(float a) { return make_float2(a, a); }

// Accumulates loss and d(loss)/d(theta) over the measurements of one voxel.
// set_nan_inf_zero (utils/askadam.m:80): a non-finite prediction becomes 0
// and carries no gradient.
// Models whose signal can be non-finite inside the parameter bounds (NEXI:
// fa -> 1 makes the exchange rate r2 = r1 fa/(1-fa) overflow).
template <int NP> struct MayBeNonFinite { static constexpr bool value = NP >= 4; };

// MSE accumulation: per measurement one FMA for sum r^2 and one per parameter
// for sum r dS/dtheta; mse_finish applies mse_scale (loss) and 2 mse_scale
// (gradient) once per voxel.  The residual output keeps its per-measurement
// value mse_scale r^2.  An accumulator's finish() must follow the model.
template <int NP>
__device__ __forceinline__ void mse_add(float r, const float (&dS)[NP], bool bad, float& total, float (&g)[NP],
                                        float* res, int ri, float mse_scale) {
    total = __fmaf_rn(r, r, total);
    if (res) res[ri] = mse_scale * r * r;
    if (!bad) {
#pragma unroll
        for (int k = 0; k < NP; ++k) g[k] = __fmaf_rn(r, dS[k], g[k]);
    }
}

template <int NP>
__device__ __forceinline__ void mse_finish(float& total, float (&g)[NP], float mse_scale) {
    total = mul1(total, mse_scale);
    const float s2 = mul1(2.0f, mse_scale);
#pragma unroll
    for (int k = 0; k < NP; ++k) g[k] = mul1(g[k], s2);
}

template <int LOSS, int NP>
struct LossAcc {
    static constexpr bool kMse = LOSS == kMSE;
    float total;
    float g[NP];
    const float* y;   // measurement m at y[m*ys]
    int ys;
    const float* w;   // nullptr: unit weights
    int ws;
    LossAux aux;
    float mse_scale, hd;
    float* res;       // nullptr or residual output at res[m*rs]
    int rs;

    __device__ __forceinline__ void add(int m, float S, const float (&dS)[NP]) {
        bool bad = MayBeNonFinite<NP>::value ? !isfinite(S) : false;
        float s = bad ? 0.0f : S;
        if constexpr (LOSS == kMSE) {
            mse_add(s - y[m * ys], dS, bad, total, g, res, m * rs, mse_scale);
            return;
        }
        float ww = w ? w[m * ws] : 1.0f;
        float d;
        float l = loss_elem<LOSS>(s, y[m * ys], ww, aux, mse_scale, hd, d);
        total += l;
        if (res) res[m * rs] = l;
        if (!bad) {
#pragma unroll
            for (int k = 0; k < NP; ++k) g[k] += d * dS[k];
        }
    }
    __device__ __forceinline__ void finish() {
        if constexpr (LOSS == kMSE) mse_finish(total, g, mse_scale);
    }
    __device__ __forceinline__ float meas(int m) const { return y[m * ys]; }
};

template <int MODEL> struct ModelNP;
template <> struct ModelNP<kR2S> { static constexpr int value = 2; };
template <> struct ModelNP<kR1R2S> { static constexpr int value = 3; };
template <> struct ModelNP<kNEXI> { static constexpr int value = 4; };
template <> struct ModelNP<kNEXI2> { static constexpr int value = 5; };

// One echo of the mono-exponential model, S = M0 exp(-TE R2*), and its
// derivatives with respect to (M0, R2*) (R2star/gpuR2starMapping.m:427-434).
__device__ __forceinline__ void r2s_echo(float te, float te_l2e, float M0, float R2, float& S, float (&dS)[2]) {
    const float E = ex2_ftz(mul1(-te_l2e, R2));  // exp(-te R2*), as in the fused R2*/MSE sums
    S = M0 * E;
    dS[0] = E;
    dS[1] = -te * S;
}

// LossAcc whose measurements are loaded into registers before the model runs
// (load()), so that all of a voxel's loads are in flight together instead of
// one per measurement; add() must be called with compile-time indices m
// (an unrolled loop, model_r2s_unrolled).  Same loss arithmetic as LossAcc.
template <int LOSS, int NP, int MAXM>
struct PrefLossAcc {
    static constexpr bool kMse = LOSS == kMSE;
    float total;
    float g[NP];
    float yv[MAXM];
    const float* w;   // nullptr: unit weights
    int ws;
    LossAux aux;
    float mse_scale, hd;
    float* res;       // nullptr or residual output at res[m*rs]
    int rs;

    __device__ __forceinline__ void load(const float* y, int ys, int nm) {
#pragma unroll
        for (int m = 0; m < MAXM; ++m) yv[m] = m < nm ? y[(size_t)m * ys] : 0.0f;  // global or shared
    }
    // measurements in echo quads: quad j of the voxel (measurements 4j..4j+3,
    // zero-padded) at q[j*qs], so that a warp reads 512 contiguous bytes
    // per quad
    __device__ __forceinline__ void load_quads(const float4* q, size_t qs) {
        static_assert(MAXM % 4 == 0, "whole quads");
#pragma unroll
        for (int j = 0; j < MAXM / 4; ++j) {
            const float4 t = __ldcg(q + j * qs);
            yv[4 * j] = t.x;
            yv[4 * j + 1] = t.y;
            yv[4 * j + 2] = t.z;
            yv[4 * j + 3] = t.w;
        }
    }
    __device__ __forceinline__ void add(int m, float S, const float (&dS)[NP]) {
        bool bad = MayBeNonFinite<NP>::value ? !isfinite(S) : false;
        float s = bad ? 0.0f : S;
        if constexpr (LOSS == kMSE) {
            mse_add(s - yv[m], dS, bad, total, g, res, m * rs, mse_scale);
            return;
        }
        float ww = w ? w[m * ws] : 1.0f;
        float d;
        float l = loss_elem<LOSS>(s, yv[m], ww, aux, mse_scale, hd, d);
        total += l;
        if (res) res[m * rs] = l;
        if (!bad) {
#pragma unroll
            for (int k = 0; k < NP; ++k) g[k] += d * dS[k];
        }
    }
    __device__ __forceinline__ void finish() {
        if constexpr (LOSS == kMSE) mse_finish(total, g, mse_scale);
    }
    __device__ __forceinline__ float meas(int m) const { return yv[m]; }
};

// Accumulators that take the fused R2*/MSE echo path (kMse true).
template <class A, class = void> struct AccMse { static constexpr bool value = false; };
template <class A> struct AccMse<A, decltype(void(A::kMse))> { static constexpr bool value = A::kMse; };

// Per-voxel model inputs besides theta.
struct VoxAux {
    float b1;                 // R1R2*: flip-angle scaling
    const float* sa;          // R1R2*: sin(b1*FA_f) at sa[f*fs]
    const float* ca;          // R1R2*: cos(b1*FA_f)
    int fs;
    float sigma = 1.0f;       // NEXI Rician mean: noise sigma (normalised by b0)
};

// Rician mean of a noise-free signal S (myriceM1 / myL12 / mybesseli,
// NEXI/gpuNEXIrice.m:726-755): M1 = max(sigma sqrt(pi/2) L(x), S) with
// x = max(-S^2 / (2 sigma^2), -170) and L(x) = exp(x/2) ((1-x) I0(-x/2) -
// x I1(-x/2)), the I_nu being 34-node trapezoids over t in [0, pi].  With
// z = -x/2 the factor exp(x/2) is folded into the integrands,
// exp(z (cos t - 1)), so nothing overflows in FP32.  dM1/dS differentiates
// the discretised function, as autodiff does: dL/dx = -T0/2 - 3 T1/2 -
// x V / 2 with T_nu the scaled trapezoids and V that of sin^2 t.
__device__ __forceinline__ float rice_mean(const DevProtocol& P, float S, float sigma, float& dM1) {
    const float s2i = 1.0f / (sigma * sigma);
    const float xr = -0.5f * S * S * s2i;
    const bool clamped = xr < -170.0f;
    const float x = clamped ? -170.0f : xr;
    const float z = -0.5f * x;
    const float eend = __expf(-2.0f * z);   // t = pi: cos t - 1 = -2
    float T0 = 0.5f * (1.0f + eend), T1 = 0.5f * (1.0f - eend), V = 0.0f;
#pragma unroll 8
    for (int i = 0; i < kRiceNodes - 2; ++i) {
        const float c1 = P.rice_cm1[i];
        const float e = __expf(z * c1);
        T0 += e;
        T1 = fmaf(e, c1 + 1.0f, T1);
        V = fmaf(e, P.rice_s2[i], V);
    }
    const float hn = 1.0f / (float)(kRiceNodes - 1);  // trapezoid step / pi
    T0 *= hn;
    T1 *= hn;
    V *= hn;
    const float k = 1.2533141373155003f * sigma;  // sqrt(pi/2) sigma
    const float M = k * ((1.0f - x) * T0 - x * T1);
    if (M > S) {
        const float dL = -0.5f * T0 - 1.5f * T1 - 0.5f * x * V;
        dM1 = clamped ? 0.0f : k * dL * (-S * s2i);
        return M;
    }
    dM1 = 1.0f;
    return S;
}

// One echo of R2*/MSE, fused: E = exp(-te R2*) = 2^(-(te log2 e) R2*),
// r = M0 E - y, and with q = r E the sums sum r^2, sum q (dS/dM0 = E) and
// sum te q (dS/dR2* = -te M0 E, the factor -M0 applied once per voxel).
// Explicit roundings, so that every kernel evaluates it identically.
struct R2sMseSums {
    float sse = 0.0f, g0 = 0.0f, g1 = 0.0f;
    __device__ __forceinline__ float echo(float te, float te_l2e, float M0, float R2, float y) {
        const float E = ex2_ftz(mul1(-te_l2e, R2));
        const float r = fma1(M0, E, -y);
        sse = fma1(r, r, sse);
        const float q = mul1(r, E);
        g0 = add1(g0, q);
        g1 = fma1(te, q, g1);
        return r;
    }
    template <class Acc>
    __device__ __forceinline__ void store(float M0, Acc& acc) const {
        acc.total = add1(acc.total, sse);
        acc.g[0] = add1(acc.g[0], g0);
        acc.g[1] = fma1(-M0, g1, acc.g[1]);
    }
};

// S = M0 exp(-TE R2*)  (R2star/gpuR2starMapping.m:427-434)
template <class Acc>
__device__ __forceinline__ void model_r2s(const DevProtocol& P, const float* th, Acc& acc) {
    float M0 = th[0], R2 = th[1];
    if constexpr (AccMse<Acc>::value) {
        R2sMseSums u;
        if (acc.res) {
            for (int m = 0; m < P.nm; ++m) {
                const float r = u.echo(P.te[m], P.te_l2e[m], M0, R2, acc.meas(m));
                acc.res[m * acc.rs] = acc.mse_scale * r * r;
            }
        } else {
#pragma unroll 4
            for (int m = 0; m < P.nm; ++m) u.echo(P.te[m], P.te_l2e[m], M0, R2, acc.meas(m));
        }
        u.store(M0, acc);
    } else {
        for (int m = 0; m < P.nm; ++m) {
            float S, dS[2];
            r2s_echo(P.te[m], P.te_l2e[m], M0, R2, S, dS);
            acc.add(m, S, dS);
        }
    }
}

// model_r2s with the echo loop unrolled to a compile-time bound (nm <= MAXM),
// so that an accumulator holding the voxel's measurements in registers
// (PrefLossAcc) is indexed by constants.  Same arithmetic per echo.
template <int MAXM, class Acc>
__device__ __forceinline__ void model_r2s_unrolled(const DevProtocol& P, int nm, const float* th, Acc& acc) {
    float M0 = th[0], R2 = th[1];
    if constexpr (AccMse<Acc>::value) {
        R2sMseSums u;
#pragma unroll
        for (int m = 0; m < MAXM; ++m)
            if (m < nm) {
                const float r = u.echo(P.te[m], P.te_l2e[m], M0, R2, acc.meas(m));
                if (acc.res) acc.res[m * acc.rs] = acc.mse_scale * r * r;
            }
        u.store(M0, acc);
    } else {
#pragma unroll
        for (int m = 0; m < MAXM; ++m) {
            if (m < nm) {
                float S, dS[2];
                r2s_echo(P.te[m], P.te_l2e[m], M0, R2, S, dS);
                acc.add(m, S, dS);
            }
        }
    }
}

// R1-R2*/MSE, fused (up to NFA flip angles; exactly NFA when EXACT): exp(-te
// R2*) once per echo time, shared by the flip angles (2^x with te log2 e, as
// for R2*), r = (A M0) E2 - y, and per flip angle f the sums sum q and sum
// te q with q = r E2, so that dS/dM0 = A E2, dS/dR1 = M0 E2 dA/dR1 and dS/dR2*
// = -te A M0 E2 are applied once per voxel.  Explicit roundings; echo times
// outer, flip angles inner.  RES: the residual output is written.  NTE > 0:
// exactly NTE echo times, the loop unrolled (the echo constants become
// constant-bank operands, no loop control); 0: any number.
template <int NFA, bool EXACT, bool RES, int NTE, class Acc>
__device__ __forceinline__ void r1r2s_mse_sums(const DevProtocol& P, float R2, int nfa, const float (&AM0)[NFA],
                                               float& sse, float (&Sq)[NFA], float (&Stq)[NFA], Acc& acc) {
    const int nte = NTE > 0 ? NTE : P.n_te;
    constexpr int UNROLL = NTE > 0 ? NTE : 2;
#pragma unroll UNROLL
    for (int t = 0; t < nte; ++t) {
        const float te = P.te[t];
        const float E2 = ex2_ftz(mul1(-P.te_l2e[t], R2));
#pragma unroll
        for (int f = 0; f < NFA; ++f)
            if (EXACT || f < nfa) {
                const int m = t + f * nte;
                const float r = fma1(AM0[f], E2, -acc.meas(m));
                sse = fma1(r, r, sse);
                if (RES) acc.res[m * acc.rs] = acc.mse_scale * r * r;
                const float q = mul1(r, E2);
                Sq[f] = add1(Sq[f], q);
                Stq[f] = fma1(te, q, Stq[f]);
            }
    }
}

template <int NFA, bool EXACT, int NTE, class Acc>
__device__ __forceinline__ void r1r2s_mse(const DevProtocol& P, float M0, float R1, float R2, const VoxAux& va,
                                          Acc& acc) {
    const float E1 = __expf(-P.tr * R1);
    const int nfa = EXACT ? NFA : P.n_fa;
    float A[NFA], dA[NFA], AM0[NFA], Sq[NFA], Stq[NFA];
#pragma unroll
    for (int f = 0; f < NFA; ++f) {
        A[f] = dA[f] = AM0[f] = 0.0f;
        if (EXACT || f < nfa) {
            const float sa = va.sa[f * va.fs], ca = va.ca[f * va.fs];
            const float inv = 1.0f / (1.0f - ca * E1);
            A[f] = sa * (1.0f - E1) * inv;
            dA[f] = sa * (ca - 1.0f) * inv * inv * (-P.tr * E1);
            AM0[f] = mul1(A[f], M0);
        }
        Sq[f] = 0.0f;
        Stq[f] = 0.0f;
    }
    float sse = 0.0f;
    if (acc.res) r1r2s_mse_sums<NFA, EXACT, true, NTE>(P, R2, nfa, AM0, sse, Sq, Stq, acc);
    else r1r2s_mse_sums<NFA, EXACT, false, NTE>(P, R2, nfa, AM0, sse, Sq, Stq, acc);
    float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f;
#pragma unroll
    for (int f = 0; f < NFA; ++f)
        if (EXACT || f < nfa) {
            g0 = fma1(A[f], Sq[f], g0);
            g1 = fma1(dA[f], Sq[f], g1);
            g2 = fma1(A[f], Stq[f], g2);
        }
    acc.total = add1(acc.total, sse);
    acc.g[0] = add1(acc.g[0], g0);
    acc.g[1] = fma1(M0, g1, acc.g[1]);
    acc.g[2] = fma1(-M0, g2, acc.g[2]);
}

// S = M0 sin(a)(1-E1)/(1-cos(a)E1) exp(-TE R2*), E1 = exp(-TR R1), a = b1*FA;
// measurement index TE fastest then FA (R1R2s/gpuJointR1R2starMapping.m:375-422,513-525).
// UNROLL (the register-capped fused kernel): the two-angle, 12-echo protocol
// with its echo loop unrolled.
template <bool UNROLL, class Acc>
__device__ __forceinline__ void model_r1r2s(const DevProtocol& P, const float* th,
                                            const VoxAux& va, Acc& acc) {
    float M0 = th[0], R1 = th[1], R2 = th[2];
    if constexpr (AccMse<Acc>::value) {
        if (P.n_fa == 2) {
            if (UNROLL && P.n_te == 12) r1r2s_mse<2, true, 12>(P, M0, R1, R2, va, acc);
            else r1r2s_mse<2, true, 0>(P, M0, R1, R2, va, acc);
            return;
        }
        if (P.n_fa <= 4) {
            r1r2s_mse<4, false, 0>(P, M0, R1, R2, va, acc);
            return;
        }
    }
    float E1 = __expf(-P.tr * R1);
    for (int f = 0; f < P.n_fa; ++f) {
        float sa = va.sa[f * va.fs], ca = va.ca[f * va.fs];
        float inv = 1.0f / (1.0f - ca * E1);
        float A = sa * (1.0f - E1) * inv;
        float dA = sa * (ca - 1.0f) * inv * inv * (-P.tr * E1);
        for (int t = 0; t < P.n_te; ++t) {
            float te = P.te[t];
            float E2 = __expf(-te * R2);
            float B = M0 * E2;
            float S = A * B;
            float dS[3] = {A * E2, B * dA, -te * S};
            acc.add(t + f * P.n_te, S, dS);
        }
    }
}

// NEXI narrow-pulse Karger model (NEXI/gpuNEXI.m:902-996, M at :1090-1097):
// per shell j, S_j = trapz_x M(x) over x = linspace(0,1,nx); lmax = 2 adds
// Sl2_j = p2 |trapz_x M (3x^2-1)/2|; finally min(S,1).  The tangent sums per
// node are reduced to the five intermediate partials (f, d1, d2, r1, r2) and
// chained to (fa, Da, De, ra) once per shell.
template <bool LMAX2, class Acc, int NP>
__device__ __forceinline__ void model_nexi_impl(const DevProtocol& P, const float* th, const VoxAux& va,
                                                Acc& acc) {
    const float EPS = 1e-8f;
    float fa_in = th[0];
    float f = fmaxf(fa_in, EPS);
    float Da = th[1], De = th[2], ra = th[3];
    float gate = fa_in > EPS ? 1.0f : 0.0f;  // d max(fa,eps)/d fa
    float omf = 1.0f - f;
    // gpuNEXIrice guards re = ra fa / max(1 - fa, eps) (NEXI/gpuNEXIrice.m:684)
    const bool rice = P.rice != 0;
    float omg = rice ? fmaxf(omf, EPS) : omf;
    float rf = f / omg;
    int nx = P.nx;
    float h = P.h;
    int nsh = P.n_shell;
    for (int j = 0; j < nsh; ++j) {
        float b = P.bval[j], D = P.delta[j];
        float d2 = b * De;
        float r1 = D * ra;
        float r2 = r1 * rf;
        float base = r1 - r2 - d2;
        float c1 = r1 + r2 + d2;
        float q4 = 4.0f * r1 * r2;
        float bDa = b * Da;
        float fd2 = omf * d2;
        // nodes in pairs (i, i+1) on the two lanes of pair instructions, an
        // odd node count padded with a node of weight 0; per lane the
        // operations of a node at a time (ptxas may fuse a pair multiply
        // into the following pair add; this is the model's only form, so
        // every path rounds alike), the sums kept per lane and folded at
        // the end
        const float2 z2 = make_float2(0.f, 0.f), half = bcast2(0.5f), one = bcast2(1.0f), two = bcast2(2.0f);
        const float2 bDa2 = bcast2(bDa), base2 = bcast2(base), q42 = bcast2(q4), c12 = bcast2(c1);
        const float2 f2 = bcast2(f), fd22 = bcast2(fd2), d22 = bcast2(d2), omf2 = bcast2(omf);
        const float2 r2x4 = bcast2(4.0f * r2), r1x4 = bcast2(4.0f * r1);
        float2 S0p = z2, Sfp = z2, Sd1p = z2, Sd2p = z2, Sr1p = z2, Sr2p = z2;
        float2 T0p = z2, Tfp = z2, Td1p = z2, Td2p = z2, Tr1p = z2, Tr2p = z2;
        // node indices (i, i+1) carried as exact floats (integers below 2^24),
        // so the loop converts no integer to float: conversions share the
        // SFU's issue rate with the rsqrt and the exponentials of the node
        float2 fi = make_float2(0.0f, 1.0f);
        for (int i = 0; i < nx; i += 2, fi = add2(fi, two)) {
            const float2 x = mul2(fi, bcast2(h));
            const float2 x2 = mul2(x, x);
            const float2 d1 = mul2(bDa2, x2);
            const float2 s = add2(base2, d1);
            const float2 Q = fma2(s, s, q42);
            const float2 rs = make_float2(rsqrtf(Q.x), rsqrtf(Q.y));
            const float2 l2raw = mul2(mul2(half, Q), rs);
            const bool ax = l2raw.x > EPS, ay = l2raw.y > EPS;
            const float2 l2 = make_float2(ax ? l2raw.x : EPS, ay ? l2raw.y : EPS);
            const float2 rs2 = mul2(two, rs);
            const float2 inv_l2 = make_float2(ax ? rs2.x : 1.0f / EPS, ay ? rs2.y : 1.0f / EPS);
            const float2 l1 = mul2(half, add2(c12, d1));
            const float2 lm = sub2(l1, l2), lp = add2(l1, l2);
            const float2 N = sub2(fma2(f2, d1, fd22), lm);
            const float2 Pp = mul2(mul2(half, N), inv_l2);
            const float2 em = make_float2(__expf(-lm.x), __expf(-lm.y));
            const float2 ep = make_float2(__expf(-lp.x), __expf(-lp.y));
            const float2 omP = sub2(one, Pp);
            const float2 M = fma2(Pp, ep, mul2(omP, em));
            // reverse sweep with Mbar = 1
            const float2 Ppb = sub2(ep, em);
            const float2 lpb = mul2(make_float2(-Pp.x, -Pp.y), ep);
            float2 lmb = mul2(make_float2(-omP.x, -omP.y), em);
            const float2 Nb = mul2(mul2(half, Ppb), inv_l2);
            float2 l2b = mul2(mul2(make_float2(-Ppb.x, -Ppb.y), Pp), inv_l2);
            lmb = sub2(lmb, Nb);
            const float2 l1b = add2(lpb, lmb);
            l2b = add2(l2b, sub2(lpb, lmb));
            const float2 Qbr = mul2(mul2(bcast2(0.125f), l2b), inv_l2);
            const float2 Qb = make_float2(ax ? Qbr.x : 0.0f, ay ? Qbr.y : 0.0f);
            const float2 sb = mul2(mul2(two, s), Qb);
            const float2 hl1 = mul2(half, l1b);
            const float2 fb = mul2(Nb, sub2(d1, d22));
            const float2 d1b = add2(add2(mul2(Nb, f2), sb), hl1);
            const float2 d2b = add2(sub2(mul2(Nb, omf2), sb), hl1);
            const float2 r1b = add2(add2(mul2(r2x4, Qb), sb), hl1);
            const float2 r2b = add2(sub2(mul2(r1x4, Qb), sb), hl1);
            const float2 wt = make_float2((i == 0 || i == nx - 1) ? 0.5f : 1.0f,
                                          i + 1 >= nx ? 0.0f : (i + 1 == nx - 1 ? 0.5f : 1.0f));
            S0p = fma2(wt, M, S0p);
            Sfp = fma2(wt, fb, Sfp);
            Sd1p = fma2(mul2(wt, x2), d1b, Sd1p);
            Sd2p = fma2(wt, d2b, Sd2p);
            Sr1p = fma2(wt, r1b, Sr1p);
            Sr2p = fma2(wt, r2b, Sr2p);
            if (LMAX2) {
                const float2 p2w = mul2(wt, fma2(bcast2(1.5f), x2, bcast2(-0.5f)));
                T0p = fma2(p2w, M, T0p);
                Tfp = fma2(p2w, fb, Tfp);
                Td1p = fma2(mul2(p2w, x2), d1b, Td1p);
                Td2p = fma2(p2w, d2b, Td2p);
                Tr1p = fma2(p2w, r1b, Tr1p);
                Tr2p = fma2(p2w, r2b, Tr2p);
            }
        }
        const float S0 = S0p.x + S0p.y, Sf = Sfp.x + Sfp.y, Sd1 = Sd1p.x + Sd1p.y, Sd2 = Sd2p.x + Sd2p.y;
        const float Sr1 = Sr1p.x + Sr1p.y, Sr2 = Sr2p.x + Sr2p.y;
        const float T0 = T0p.x + T0p.y, Tf = Tfp.x + Tfp.y, Td1 = Td1p.x + Td1p.y, Td2 = Td2p.x + Td2p.y;
        const float Tr1 = Tr1p.x + Tr1p.y, Tr2 = Tr2p.x + Tr2p.y;
        float r2_f = rice ? (omf > EPS ? r1 / (omf * omf) : r1 / EPS) : r1 / (omf * omf);
        {
            float S = S0 * h;
            float dS[NP];
            dS[0] = gate * h * (Sf + Sr2 * r2_f);
            dS[1] = h * Sd1 * b;
            dS[2] = h * Sd2 * b;
            dS[3] = h * (Sr1 + Sr2 * rf) * D;
            if (NP > 4) dS[NP - 1] = 0.0f;
            if (rice) {  // Rician floor correction (NEXI/gpuNEXIrice.m:653)
                float dM1;
                S = rice_mean(P, S, va.sigma, dM1);
#pragma unroll
                for (int k = 0; k < NP; ++k) dS[k] *= dM1;
            }
            if (S > 1.0f) {  // min(S,1), NEXI/gpuNEXI.m:928
                S = 1.0f;
#pragma unroll
                for (int k = 0; k < NP; ++k) dS[k] = 0.0f;
            }
            acc.add(j, S, dS);
        }
        if (LMAX2) {
            float p2 = th[NP - 1];
            float T = T0 * h;
            float sg = (float)((T > 0.0f) - (T < 0.0f));
            float S = p2 * fabsf(T);
            float dS[NP];
            dS[0] = gate * p2 * sg * h * (Tf + Tr2 * r2_f);
            dS[1] = p2 * sg * h * Td1 * b;
            dS[2] = p2 * sg * h * Td2 * b;
            dS[3] = p2 * sg * h * (Tr1 + Tr2 * rf) * D;
            dS[NP - 1] = fabsf(T);
            if (S > 1.0f) {
                S = 1.0f;
#pragma unroll
                for (int k = 0; k < NP; ++k) dS[k] = 0.0f;
            }
            acc.add(nsh + j, S, dS);
        }
    }
}

// UNROLL: unrolled protocol loops where a caller's register budget allows
// (the fused kernel of the joint R1-R2* model).
template <int MODEL, bool UNROLL = false, class Acc>
__device__ __forceinline__ void model_eval(const DevProtocol& P, const float* th, const VoxAux& va,
                                           Acc& acc) {
    if constexpr (MODEL == kR2S) model_r2s(P, th, acc);
    else if constexpr (MODEL == kR1R2S) model_r1r2s<UNROLL>(P, th, va, acc);
    else if constexpr (MODEL == kNEXI) model_nexi_impl<false, Acc, 4>(P, th, va, acc);
    else model_nexi_impl<true, Acc, 5>(P, th, va, acc);
}

// Forward-only accumulation (no derivatives): used by gx_forward and MCMC.
template <int NP>
struct SignalSink {
    float* out;   // out[m*os]
    int os;
    __device__ __forceinline__ void add(int m, float S, const float (&)[NP]) { out[m * os] = S; }
};

// Sum of weighted squared residuals, accumulated in FP64 (MCMC logP).
template <int NP>
struct SosSink {
    const float* y;
    int ys;
    const float* w;
    int ws;
    double sos;
    __device__ __forceinline__ void add(int m, float S, const float (&)[NP]) {
        float r = S - y[m * ys];
        float ww = w ? w[m * ws] : 1.0f;
        sos += (double)(ww * r * r);
    }
};

// Copies the protocol into shared memory so that the per-measurement loops
// read it with shared-memory broadcasts instead of indexed parameter loads.
__device__ __forceinline__ void stage_protocol(const DevProtocol& P, DevProtocol* s_P) {
    const int* src = reinterpret_cast<const int*>(&P);
    int* dst = reinterpret_cast<int*>(s_P);
    for (int i = threadIdx.x; i < (int)(sizeof(DevProtocol) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
}

// unscale_parameters (utils/askadam.m:1063-1075) and its derivative: the
// logistic s = 1 / (1 + exp(-z)) with exp(-z) = 2^(-z log2 e) and the fast
// reciprocal; theta = lb + (ub-lb) s, dtheta/dz = (ub-lb) s (1-s).
__device__ __forceinline__ float unscale(int transform, float lb, float ub, float z, float& dth) {
    if (transform == 0) {
        const float s = rcp_ftz(add1(1.0f, ex2_ftz(mul1(z, -kLog2e))));
        const float d = sub1(ub, lb);
        dth = mul1(mul1(d, s), sub1(1.0f, s));
        return fma1(d, s, lb);
    }
    float zc = fminf(fmaxf(z, 0.0f), 1.0f);  // set_boundary01 before evaluation
    dth = (z >= 0.0f && z <= 1.0f) ? (ub - lb) : 0.0f;
    return zc * (ub - lb) + lb;
}

// Anisotropic TV at one masked voxel (utils/spatial_total_variation.m:45-66):
// c = theta at the voxel, f[d] / b[d] = theta at the forward / backward
// neighbour along axis d (periodic), mb[d] = backward neighbour inside the
// mask, iv[d] = 1/voxel size.  cost = sum_d |f_d - c| iv_d;
// d cost_total / d c = sum_d (-sgn(f_d - c) + mb_d sgn(c - b_d)) iv_d.
// One function for every one-voxel kernel (tv_terms2m restates it for two
// voxels) so that all paths round identically.
// sign(x) in {-1, 0, +1} (0 for +-0), as compare-and-select.
__device__ __forceinline__ float sgn0(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

__device__ __forceinline__ void tv_terms(float c, const float* f, const float* b, const bool* mb,
                                         const float* iv, int nd, float& cost, float& grad) {
    float cs = 0.0f, gr = 0.0f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d < nd) {
            const float df = sub1(f[d], c);
            cs = fma1(fabsf(df), iv[d], cs);  // fused, as the two-voxel form
            const float t = -sgn0(df) + (mb[d] ? sgn0(sub1(c, b[d])) : 0.0f);  // small integers: exact
            gr = add1(gr, mul1(t, iv[d]));
        }
    }
    cost = cs;
    grad = gr;
}

// Surface TV of one vertex (gpuNEXI.surface_total_variation, NEXI/gpuNEXI.m:
// 1165-1254): its cost sum_j |q_j|, q_j = (theta_v - theta_nb_j) / len_j over
// the neighbour slots j (G: the parameter on the vertex grid, 0 off the mask;
// a non-finite q_j is dropped), and the derivative of the whole regulariser
// with respect to theta_v: every masked neighbour also holds the edge back to
// v (mesh adjacency is symmetric, with the same length), hence
// sum_j (1 + mask(nb_j)) sgn(q_j) / len_j.  A padding slot names v itself.
__device__ __forceinline__ void surf_tv_terms(float c, const float* G, const unsigned char* mk, const int* nb,
                                              const float* len, int maxnb, size_t stride, float& cost,
                                              float& grad) {
    float cs = 0.0f, gr = 0.0f;
    for (int j = 0; j < maxnb; ++j) {
        const int q = nb[(size_t)j * stride];
        const float l = len[(size_t)j * stride];
        const float t = __fdiv_rn(sub1(c, G[q]), l);
        if (!isfinite(t)) continue;
        cs = add1(cs, fabsf(t));
        gr = add1(gr, __fdiv_rn(mul1(mk[q] ? 2.0f : 1.0f, sgn0(t)), l));
    }
    cost = cs;
    grad = gr;
}

// Prior-distribution regulariser of one parameter (gpuNEXI.prior_distribution_normal,
// NEXI/gpuNEXI.m:1256-1307): z = (theta - mu) / sd; a finite z adds |z| to the
// cost and sgn(z) / sd to d cost / d theta, a non-finite one nothing.
__device__ __forceinline__ void prior_terms(float th, float mu, float sd, float& cost, float& grad) {
    const float z = __fdiv_rn(sub1(th, mu), sd);
    const bool ok = isfinite(z);
    cost = ok ? fabsf(z) : 0.0f;
    grad = ok ? __fdiv_rn(sgn0(z), sd) : 0.0f;
}

// Saturated product (PTX mul.sat: the result clamped to [0, 1], NaN to 0).
__device__ __forceinline__ float mul_sat1(float a, float b) {
    float d;
    asm("mul.rn.ftz.sat.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}

// Backward-neighbour mask word of a voxel: byte d (d = 0, 1, 2 for x, y, z)
// is kMaskByte when the backward neighbour along d lies inside the mask, else
// 0; byte 3 holds the periodic-wrap flags (bit 0-2 last x/y/z plane, 3-5
// first).  Broadcasting byte d to all four bytes gives the float kSignScale
// (bits 0x7F7F7F7F, about 3.4e38) or 0.
constexpr unsigned int kMaskByte = 0x7Fu;
__device__ __forceinline__ float mask_scale(unsigned int w, int d) {
    return __int_as_float((int)__byte_perm(w, 0u, (unsigned int)d * 0x1111u));
}

// tv_terms for two voxels on the lanes of pair instructions, with the signs
// as saturated products and the mask as a scale (w0 / w1: the two voxels'
// mask words).  With subnormals flushed every nonzero x has |x| >= 2^-126,
// so sat(x K) - sat(-x K) = sgn0(x) exactly for K >= 2^127 (and 0 for x = 0
// or NaN), and sat(x 0) = 0 drops a backward term outside the mask;
// -|df| = df (-sgn0(df)) exactly.  Every lane result equals tv_terms' bit
// for bit: the costs add |df| iv by the same fused multiply-add, and the
// gradient terms are small integers times iv (exact products), so the fused
// multiply-add rounds as the separate multiply and add.
// ivp / nivp: the inverse voxel sizes and their negatives as (x, x) pairs.
__device__ __forceinline__ void tv_terms2m(float2 c, const float (&f0)[3], const float (&b0)[3],
                                           const float (&f1)[3], const float (&b1)[3], unsigned int w0,
                                           unsigned int w1, const float2* ivp, const float2* nivp, int nd,
                                           float2& cost, float2& grad) {
    const float K = __int_as_float(0x7F7F7F7F);
    float2 cs = make_float2(0.0f, 0.0f), gr = cs;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d < nd) {
            const float2 ivd = ivp[d];
            const float2 df = sub2(make_float2(f0[d], f1[d]), c);
            const float2 snf = sub2(make_float2(mul_sat1(-df.x, K), mul_sat1(-df.y, K)),
                                    make_float2(mul_sat1(df.x, K), mul_sat1(df.y, K)));  // -sgn0(df)
            cs = fma2(mul2(df, snf), nivp[d], cs);                                      // + |df| iv
            const float2 cb = sub2(c, make_float2(b0[d], b1[d]));
            const float k0 = mask_scale(w0, d), k1 = mask_scale(w1, d);
            const float2 sb = sub2(make_float2(mul_sat1(cb.x, k0), mul_sat1(cb.y, k1)),
                                   make_float2(mul_sat1(-cb.x, k0), mul_sat1(-cb.y, k1)));  // mb sgn0(cb)
            gr = fma2(add2(snf, sb), ivd, gr);
        }
    }
    cost = cs;
    grad = gr;
}

// Optimiser step of one parameter (adamupdate / sgdmupdate / rmspropupdate,
// called from utils/askadam.m:673-691).  sc = per-epoch schedule:
// Adam (lr_e/(1-b1^e), 1/(1-b2^e)); others (lr_e, 0).  The square root is
// the approximate one (fast_sqrt0) and the Adam quotient a * rcp(b).
struct OptConst {
    int optimiser;
    float beta1, beta2, eps, momentum, rms_decay, rms_eps;
};

// sqrt(x), x >= 0, by the PTX approximate square root (sqrt.approx,
// subnormals flushed); the optimisers' second moments are never negative
__device__ __forceinline__ float fast_sqrt0(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Adam: m1 = b1 m1 + (1-b1) g, m2 = b2 m2 + ((1-b2) g) g,
// z -= (lr_e m1) / (sqrt(m2 / (1-b2^e)) + eps), the last step as one fused
// multiply-add z + (-(lr_e m1)) (1 / (...)).  (ptxas contracts an FP32x2
// multiply followed by a subtraction into a fused multiply-add even with an
// explicit .rn rounding, so the two-voxel form is fused; every form is
// written fused so that all kernels round alike.)
__device__ __forceinline__ void opt_step(const OptConst& o, float2 sc, float& z, float& m1, float& m2, float g) {
    if (o.optimiser == kAdam) {
        m1 = fma1(o.beta1, m1, mul1(sub1(1.0f, o.beta1), g));
        m2 = fma1(o.beta2, m2, mul1(mul1(sub1(1.0f, o.beta2), g), g));
        z = fma1(mul1(-sc.x, m1), rcp_ftz(add1(fast_sqrt0(mul1(m2, sc.y)), o.eps)), z);
    } else if (o.optimiser == kSGDM) {
        m1 = o.momentum * m1 - sc.x * g;
        z += m1;
    } else {
        m2 = o.rms_decay * m2 + (1.0f - o.rms_decay) * g * g;
        z -= __fdividef(sc.x * g, fast_sqrt0(m2) + o.rms_eps);
    }
}

// The constants of the pair transform and optimiser as (x, x) pairs, so that
// the pair instructions take them as kernel-parameter operands.
struct PairConsts {
    float2 nl2e;      // -log2(e)
    float2 one;
    float2 rng[2];    // ub - lb of the two parameters
    float2 lb[2];
    float2 b1, omb1, b2, omb2, eps;  // Adam: beta1, 1 - beta1, beta2, 1 - beta2, epsilon
    float2 mse, s2;   // mse_scale, 2 mse_scale
    float2 iv[3];     // inverse voxel sizes
    float2 niv[3];    // their negatives
};

// The sigmoid transform of a pair of voxels with its constants from
// PairConsts (on each lane bit for bit unscale's operations).
__device__ __forceinline__ float2 unscale_sig2c(const PairConsts& k, int i, float2 z, float2& dth) {
    const float2 e = mul2(z, k.nl2e);
    const float2 den = add2(k.one, make_float2(ex2_ftz(e.x), ex2_ftz(e.y)));
    const float2 s = make_float2(rcp_ftz(den.x), rcp_ftz(den.y));
    dth = mul2(mul2(k.rng[i], s), sub2(k.one, s));
    return fma2(k.rng[i], s, k.lb[i]);
}

// The Adam step of opt_step on a pair of voxels, with its constants from
// PairConsts and the epoch's schedule as pairs nscx = (-sc.x, -sc.x),
// scy = (sc.y, sc.y) (on each lane bit for bit opt_step's operations).
__device__ __forceinline__ void adam_step2c(const PairConsts& k, float2 nscx, float2 scy, float2& z, float2& m1,
                                            float2& m2, float2 g) {
    m1 = fma2(k.b1, m1, mul2(k.omb1, g));
    m2 = fma2(k.b2, m2, mul2(mul2(k.omb2, g), g));
    const float2 v = mul2(m2, scy);
    const float2 den = add2(make_float2(fast_sqrt0(v.x), fast_sqrt0(v.y)), k.eps);
    z = fma2(mul2(nscx, m1), make_float2(rcp_ftz(den.x), rcp_ftz(den.y)), z);
}

#endif  // __CUDACC__

}  // namespace gx
