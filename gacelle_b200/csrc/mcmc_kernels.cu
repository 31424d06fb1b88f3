// mcmc_kernels.cu -- Metropolis-Hastings and Goodman-Weare ensemble MCMC.
//
// Goodman-Weare: a block holds VPB voxels; each voxel's ensemble lives in
// shared memory and one thread advances one walker (simultaneous update) or
// one walker of each half (red-black).  Proposals use counter-based Philox
// keyed by (voxel, walker, step, repetition), the partner draws are shared by
// all voxels as in the reference, the likelihood is accumulated in FP64 and
// kept samples are folded into FP64 running sums on the fly (optionally
// written out as the full posterior).  Reference: utils/mcmc.m
// (metropolis_hastings :82-190, goodman_weare :192-383, find_partner
// :797-803, res2out :806-862), utils/logP_Gaussian.m.
#include "gx_internal.h"

namespace gx {

constexpr int kMaxWalker = 256;

// find_partner (mcmc.m:797-803): a uniform random derangement of the W
// walkers (Fisher-Yates, fixed points rejected), from the Philox stream
// (step, attempt, draw/4, tag).
__device__ void derangement_dev(uint64_t seed, int k, uint32_t tag, int W, int* out) {
    int perm[kMaxWalker];
    bool ok = false;
    for (uint32_t attempt = 0; attempt < 4096 && !ok; ++attempt) {
        for (int i = 0; i < W; ++i) perm[i] = i;
        U4 u{0, 0, 0, 0};
        for (int i = W - 1, d = 0; i >= 1; --i, ++d) {
            if ((d & 3) == 0) u = philox((uint32_t)k, attempt, (uint32_t)(d >> 2), tag, seed);
            uint32_t r = (d & 3) == 0 ? u.x : (d & 3) == 1 ? u.y : (d & 3) == 2 ? u.z : u.w;
            int j = (int)rand_below(r, (uint32_t)(i + 1));
            int t = perm[i]; perm[i] = perm[j]; perm[j] = t;
        }
        ok = true;
        for (int i = 0; i < W; ++i) ok = ok && perm[i] != i;
    }
    for (int i = 0; i < W; ++i) out[i] = ok ? perm[i] : (i + 1) % W;
}

// Red-black anchors (mcmc.m:328-329): the a-th active walker of half `half`
// anchors on frozen(randi(numel(frozen))); written as absolute walker indices.
__device__ void rb_anchors_dev(uint64_t seed, int k, uint32_t tag, int W, int* out) {
    int h = W / 2;
    for (int half = 0; half < 2; ++half) {
        int na = half == 0 ? h : W - h, nf = half == 0 ? W - h : h, f0 = half == 0 ? h : 0;
        int a0 = half == 0 ? 0 : h;
        U4 u{0, 0, 0, 0};
        for (int a = 0; a < na; ++a) {
            if ((a & 3) == 0) u = philox((uint32_t)k, (uint32_t)half, (uint32_t)(a >> 2), tag, seed);
            uint32_t r = (a & 3) == 0 ? u.x : (a & 3) == 1 ? u.y : (a & 3) == 2 ? u.z : u.w;
            out[a0 + a] = f0 + (int)rand_below(r, (uint32_t)nf);
        }
    }
}

// Partner tables [rep][nsteps][W]: simultaneous -> one derangement per step,
// red-black -> the anchors of both halves.  Rows past `iteration` are the
// global warm-up steps 1..(nsteps - iteration).  global_block selects the
// global block's streams (goodman_weare_wglobal_constant).
__global__ void gw_partner_kernel(McmcParams p, int* partner, int nsteps, int global_block) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= p.repetition * nsteps) return;
    int rr = idx / nsteps, kk = idx % nsteps + 1;
    int k = kk <= p.iteration ? kk : kk - p.iteration;
    uint32_t bits = ((uint32_t)rr << 16) | (kk > p.iteration ? kTagWarmup : 0u);
    int* out = partner + (size_t)idx * p.nwalker;
    if (p.update == 0) derangement_dev(p.seed, k, (global_block ? kTagGwGPerm : kTagGwPerm) | bits, p.nwalker, out);
    else rb_anchors_dev(p.seed, k, (global_block ? kTagGwGRbPart : kTagGwRbPart) | bits, p.nwalker, out);
}

// logP_Gaussian (utils/logP_Gaussian.m:18-20) of the model's parameters and
// the noise sigma (the last of the NV variables, a compile-time index so that
// the caller's parameter vector stays in registers); y / w with strides.
template <int MODEL, int NV>
__device__ __forceinline__ double log_prob_t(int nm, const DevProtocol& P, const float (&x)[NV], const float* y,
                                             int ys, const float* w, int ws, const VoxAux& va) {
    constexpr int NP = ModelNP<MODEL>::value;
    static_assert(NV == NP + 1, "the variables are the model's parameters and the noise sigma");
    SosSink<NP> sink{y, ys, w, ws, 0.0};
    model_eval<MODEL>(P, x, va, sink);
    const double noise = (double)x[NV - 1];
    const double n2 = noise * noise;
    return -sink.sos / (2.0 * n2) - 0.5 * nm * log(6.283185307179586 * n2);
}

__device__ __forceinline__ int kept_index(const McmcParams& p, int k) {
    if (k <= p.nburnin) return -1;
    int j = k - p.nburnin + 1;
    if (j % p.thinning) return -1;
    int c = j / p.thinning - (p.thinning == 1 ? 1 : 0) - 1;
    return c < p.ns ? c : -1;
}

// Walker start (mcmc.m:267-275): x0 + (ub-lb)*startRange*randn, clamped; the
// normal draws of walker w of voxel v come four at a time from the Philox
// stream (v, w, j, kTagGwInit).
template <int NV>
__device__ __forceinline__ void gw_walker_start(const McmcParams& p, int v, int w, float (&x)[NV]) {
    float nrm[(NV + 3) / 4 * 4];
#pragma unroll
    for (int j = 0; j * 4 < NV; ++j) {
        U4 u = philox((uint32_t)v, (uint32_t)w, (uint32_t)j, kTagGwInit, p.seed);
        box_muller(u.x, u.y, nrm[4 * j], nrm[4 * j + 1]);
        box_muller(u.z, u.w, nrm[4 * j + 2], nrm[4 * j + 3]);
    }
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        float val = p.x0[(size_t)q * p.nvox + v] + (p.ub[q] - p.lb[q]) * p.start_range * nrm[q];
        x[q] = fminf(fmaxf(val, p.lb[q]), p.ub[q]);
    }
}

// Goodman-Weare, steps [k0, k1] of repetition rr.  State between launches:
// xstate [nvar][nvox][W], lpstate [nvox][W].  NV = parameters + noise, fixed
// at compile time, and RB (red-black: a thread owns a walker of each half)
// keep every per-walker vector in registers; the running sums of the kept
// samples live in shared memory (each thread its own walkers' slots) and are
// folded into the per-voxel sums at the end of the launch.
template <int MODEL, int NV, bool RB>
__global__ void __launch_bounds__(1024, 1)
gw_kernel(McmcParams p, int rr, int k0, int k1, int init, float* xstate, double* lpstate, double* sum,
          double* sumsq) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ DevProtocol s_P;
    stage_protocol(p.P, &s_P);
    const int W = p.nwalker, nm = p.nm;
    const int h = W / 2;
    const int tpv = RB ? (W - h) : W;
    const int vpb = blockDim.x / tpv;
    const int vl = threadIdx.x / tpv, a = threadIdx.x % tpv;
    const int v = blockIdx.x * vpb + vl;
    const bool in_block = vl < vpb;
    const bool live = in_block && v < p.nvox;
    double* ssum = reinterpret_cast<double*>(smem_raw);           // [2][vpb][W][NV] kept-sample sums
    float* xs = reinterpret_cast<float*>(ssum + 2 * vpb * W * NV); // [vpb][W][NV]
    float* ys = xs + vpb * W * NV;                                // [vpb][nm]
    float* ws = ys + vpb * nm;                                    // [vpb][nm]
    float* xv = xs + (in_block ? vl : 0) * W * NV;
    double* sv1 = ssum + (in_block ? vl : 0) * W * NV;
    double* sv2 = sv1 + vpb * W * NV;
    const float* yv = ys + (in_block ? vl : 0) * nm;
    const float* wv = p.weights ? ws + (in_block ? vl : 0) * nm : nullptr;
    if (live)
        for (int m = a; m < nm; m += tpv) {
            ys[vl * nm + m] = p.data[(size_t)m * p.nvox + v];
            if (p.weights) ws[vl * nm + m] = p.weights[(size_t)m * p.nvox + v];
        }
    float b1 = (live && p.b1) ? p.b1[v] : 1.0f;
    float sa[MODEL == kR1R2S ? kMaxFA : 1], ca[MODEL == kR1R2S ? kMaxFA : 1];
    if (MODEL == kR1R2S)
        for (int f = 0; f < p.P.n_fa; ++f) sincosf(b1 * p.P.fa_rad[f], &sa[f], &ca[f]);
    VoxAux va{b1, sa, ca, 1};

    // walkers owned by this thread: slot 0 (simultaneous: walker a; red-black:
    // walker a of the first half, if any) and, red-black, slot 1 (walker h + a)
    const int wown0 = RB ? (a < h ? a : -1) : a, wown1 = RB ? h + a : -1;
    const bool own0 = live && wown0 >= 0 && wown0 < W, own1 = RB && live && wown1 >= 0 && wown1 < W;
    float x0s[NV], x1s[RB ? NV : 1];
    double lp0 = 0.0, lp1 = 0.0;
#pragma unroll
    for (int q = 0; q < NV; ++q) x0s[q] = 0.0f;
#pragma unroll
    for (int q = 0; q < (RB ? NV : 1); ++q) x1s[q] = 0.0f;
    if (own0)
#pragma unroll
        for (int q = 0; q < NV; ++q) { sv1[wown0 * NV + q] = 0.0; sv2[wown0 * NV + q] = 0.0; }
    if (own1)
#pragma unroll
        for (int q = 0; q < NV; ++q) { sv1[wown1 * NV + q] = 0.0; sv2[wown1 * NV + q] = 0.0; }
    __syncthreads();
    if (own0) {
        if (init) gw_walker_start<NV>(p, v, wown0, x0s);
        else
#pragma unroll
            for (int q = 0; q < NV; ++q) x0s[q] = xstate[((size_t)q * p.nvox + v) * W + wown0];
#pragma unroll
        for (int q = 0; q < NV; ++q) xv[wown0 * NV + q] = x0s[q];
    }
    if constexpr (RB) {
        if (own1) {
            if (init) gw_walker_start<NV>(p, v, wown1, x1s);
            else
#pragma unroll
                for (int q = 0; q < NV; ++q) x1s[q] = xstate[((size_t)q * p.nvox + v) * W + wown1];
#pragma unroll
            for (int q = 0; q < NV; ++q) xv[wown1 * NV + q] = x1s[q];
        }
    }
    __syncthreads();
    if (own0) lp0 = init ? log_prob_t<MODEL, NV>(nm, s_P, x0s, yv, 1, wv, 1, va) : lpstate[(size_t)v * W + wown0];
    if constexpr (RB)
        if (own1) lp1 = init ? log_prob_t<MODEL, NV>(nm, s_P, x1s, yv, 1, wv, 1, va) : lpstate[(size_t)v * W + wown1];
    unsigned int nacc = 0;
    const float amin1 = p.a - 1.0f;

    // stretch proposal of walker w (state xw, log-likelihood lpw) about its
    // partner: xn and its log-likelihood lpp, and whether it is accepted
    auto propose = [&](int w, int k, uint32_t flags, const float (&xw)[NV], double lpw, float (&xn)[NV],
                       double& lpp) -> bool {
        const int* pt = p.partner + ((size_t)rr * p.iteration + (k - 1)) * W;
        const int q = pt[w];
        U4 u = philox((uint32_t)v, (uint32_t)w, (uint32_t)k, kTagGwMove | ((uint32_t)rr << 16) | flags, p.seed);
        float t = amin1 * u01(u.x) + 1.0f;
        float zz = t * t / p.a;
        bool oob = false;
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            float xq = xv[q * NV + j];
            float xp = xq + (xw[j] - xq) * zz;
            oob |= (xp < p.lb[j]) || (xp > p.ub[j]);
            xn[j] = fminf(fmaxf(xp, p.lb[j]), p.ub[j]);
        }
        lpp = log_prob_t<MODEL, NV>(nm, s_P, xn, yv, 1, wv, 1, va);
        double lr = (double)(NV - 1) * (double)logf(zz) + (lpp - lpw);
        return !oob && lr > (double)logf(u01(u.y));
    };
    auto commit = [&](int w, const float (&xn)[NV], double lpp, float (&xw)[NV], double& lpw) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            xw[j] = xn[j];
            xv[w * NV + j] = xn[j];
        }
        lpw = lpp;
        ++nacc;
    };
    auto keep = [&](int w, int c, const float (&xw)[NV]) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double d = (double)xw[j] - (double)p.shift[(size_t)j * p.nvox + v];
            sv1[w * NV + j] += d;
            sv2[w * NV + j] += d * d;
            if (p.posterior)
                p.posterior[((((size_t)j * p.repetition + rr) * p.ns + c) * W + w) * p.nvox + v] = xw[j];
        }
    };

    for (int k = k0; k <= k1; ++k) {
        if constexpr (!RB) {
            float xn[NV];
            double lpp = 0.0;
            const bool acc = own0 && propose(wown0, k, 0u, x0s, lp0, xn, lpp);
            __syncthreads();  // every walker has read the old ensemble
            if (acc) commit(wown0, xn, lpp, x0s, lp0);
            __syncthreads();
        } else {
            // the active half moves about anchors in the frozen half
            if (own0) {
                float xn[NV];
                double lpp = 0.0;
                if (propose(wown0, k, 1u << 8, x0s, lp0, xn, lpp)) commit(wown0, xn, lpp, x0s, lp0);
            }
            __syncthreads();  // the moved half is visible before the other half anchors on it
            if (own1) {
                float xn[NV];
                double lpp = 0.0;
                if (propose(wown1, k, 1u << 8, x1s, lp1, xn, lpp)) commit(wown1, xn, lpp, x1s, lp1);
            }
            __syncthreads();
        }
        const int c = kept_index(p, k);
        if (c >= 0) {
            if (own0) keep(wown0, c, x0s);
            if constexpr (RB)
                if (own1) keep(wown1, c, x1s);
        }
    }
    // persist walker state, fold the kept-sample sums of this launch
    if (own0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) xstate[((size_t)q * p.nvox + v) * W + wown0] = x0s[q];
        lpstate[(size_t)v * W + wown0] = lp0;
    }
    if constexpr (RB) {
        if (own1) {
#pragma unroll
            for (int q = 0; q < NV; ++q) xstate[((size_t)q * p.nvox + v) * W + wown1] = x1s[q];
            lpstate[(size_t)v * W + wown1] = lp1;
        }
    }
    if (live) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double t1 = own0 ? sv1[wown0 * NV + j] : 0.0, t2 = own0 ? sv2[wown0 * NV + j] : 0.0;
            if (own1) { t1 += sv1[wown1 * NV + j]; t2 += sv2[wown1 * NV + j]; }
            if (t1 != 0.0) atomicAdd(&sum[(size_t)j * p.nvox + v], t1);
            if (t2 != 0.0) atomicAdd(&sumsq[(size_t)j * p.nvox + v], t2);
        }
    }
    unsigned int wsum = nacc;
    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(p.n_acc, (unsigned long long)wsum);
}

// Metropolis-Hastings, one thread per voxel (mcmc.m:144-167).  NV =
// parameters + noise at compile time (the state in registers); the voxel's
// measurements are read from [nm][nvox] with coalesced loads.
template <int MODEL, int NV>
__global__ void mh_kernel(McmcParams p, int rr, int k0, int k1, int init, float* xstate,
                          double* lpstate, double* sum, double* sumsq) {
    __shared__ DevProtocol s_P;
    stage_protocol(p.P, &s_P);
    __syncthreads();
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    bool live = v < p.nvox;
    const int nm = p.nm;
    const float* yv = p.data + (live ? v : 0);
    const float* wv = p.weights ? p.weights + (live ? v : 0) : nullptr;
    float b1 = (live && p.b1) ? p.b1[v] : 1.0f;
    float sa[MODEL == kR1R2S ? kMaxFA : 1], ca[MODEL == kR1R2S ? kMaxFA : 1];
    if (MODEL == kR1R2S)
        for (int f = 0; f < p.P.n_fa; ++f) sincosf(b1 * p.P.fa_rad[f], &sa[f], &ca[f]);
    VoxAux va{b1, sa, ca, 1};
    float x[NV];
    double lp = 0.0;
    double s1[NV], s2[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) { s1[q] = 0.0; s2[q] = 0.0; x[q] = 0.0f; }
    unsigned int nacc = 0;
    if (live) {
        if (init) {
#pragma unroll
            for (int q = 0; q < NV; ++q)
                x[q] = fminf(fmaxf(p.x0[(size_t)q * p.nvox + v], p.lb[q]), p.ub[q]);
            lp = log_prob_t<MODEL, NV>(nm, s_P, x, yv, p.nvox, wv, p.nvox, va);
        } else {
#pragma unroll
            for (int q = 0; q < NV; ++q) x[q] = xstate[(size_t)q * p.nvox + v];
            lp = lpstate[v];
        }
        for (int k = k0; k <= k1; ++k) {
            float nrm[(NV + 3) / 4 * 4];
            uint32_t tag = kTagMhMove | ((uint32_t)rr << 16);
#pragma unroll
            for (int j = 0; j * 4 < NV; ++j) {
                U4 u = philox((uint32_t)v, (uint32_t)k, (uint32_t)j, tag, p.seed);
                box_muller(u.x, u.y, nrm[4 * j], nrm[4 * j + 1]);
                box_muller(u.z, u.w, nrm[4 * j + 2], nrm[4 * j + 3]);
            }
            U4 ua = philox((uint32_t)v, (uint32_t)k, 8u, tag, p.seed);
            float xp[NV];
            bool oob = false;
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                float t = x[q] + p.xstep[q] * nrm[q];
                oob |= (t < p.lb[q]) || (t > p.ub[q]);
                xp[q] = fminf(fmaxf(t, p.lb[q]), p.ub[q]);
            }
            double lpp = log_prob_t<MODEL, NV>(nm, s_P, xp, yv, p.nvox, wv, p.nvox, va);
            if (!oob && (lpp - lp) > (double)logf(u01(ua.x))) {
#pragma unroll
                for (int q = 0; q < NV; ++q) x[q] = xp[q];
                lp = lpp;
                ++nacc;
            }
            int c = kept_index(p, k);
            if (c >= 0)
#pragma unroll
                for (int j = 0; j < NV; ++j) {
                    double d = (double)x[j] - (double)p.shift[(size_t)j * p.nvox + v];
                    s1[j] += d;
                    s2[j] += d * d;
                    if (p.posterior)
                        p.posterior[(((size_t)j * p.repetition + rr) * p.ns + c) * p.nvox + v] = x[j];
                }
        }
#pragma unroll
        for (int q = 0; q < NV; ++q) xstate[(size_t)q * p.nvox + v] = x[q];
        lpstate[v] = lp;
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            sum[(size_t)j * p.nvox + v] += s1[j];
            sumsq[(size_t)j * p.nvox + v] += s2[j];
        }
    }
    unsigned int wsum = nacc;
    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(p.n_acc, (unsigned long long)wsum);
}

// ---------------------------------------------------------------------------
// goodman_weare_wglobal_constant (mcmc.m:385-578) and gw_global_block
// (:581-626).  One iteration = a local stretch move per (voxel, walker) with
// the walker's globals held (z^(NND-1)), then a global stretch move per walker
// with the locals held (z^(NGlobal-1)), accepted on the log-likelihood
// difference summed over all voxels in FP64.  The voxel sum is a grid-wide
// dependency, so an iteration is two launches (four with red-black):
//   gwg_step_kernel    apply the previous global decision to the cached logP,
//                      local block, kept local samples, and the logP of the
//                      global proposal with per-CTA partial sums;
//   gwg_accept_kernel  one CTA per walker: partial sums in a fixed order,
//                      accept / reject, kept global samples.
// The step kernel's first CTA publishes each global proposal (with its
// stretch factor, acceptance uniform and bounds flag); the accept kernel reads
// it, so no CTA reads a global value another CTA of the same launch updates.
// ---------------------------------------------------------------------------
enum GwgFlags { kGwgInit = 1, kGwgApply = 2, kGwgLocal = 4, kGwgEval = 8 };

// Row of the global partner table and the Philox tag bits of one global block.
__device__ __forceinline__ int gwg_row(const McmcParams& p, int rr, int k, int warm) {
    return rr * p.nsteps_g + (warm ? p.iteration + k - 1 : k - 1);
}

__device__ __forceinline__ bool gwg_active(int half, int w, int W) {
    return half < 0 || (half == 0 ? w < W / 2 : w >= W / 2);
}

// Global proposal of walker w: g(anchor) + (g(w) - g(anchor)) * z, clamped;
// g(walker, q) = g[walker * nvar + q].  Returns true when out of bounds.
__device__ bool gwg_proposal(const McmcParams& p, int rr, int k, int warm, int w, const float* g, float* out,
                             float& zz, float& lu) {
    const int q0 = p.gpartner[(size_t)gwg_row(p, rr, k, warm) * p.nwalker + w];
    uint32_t tag = kTagGwGMove | ((uint32_t)rr << 16) | (warm ? kTagWarmup : 0u) | (p.update ? kTagRedBlack : 0u);
    U4 u = philox((uint32_t)w, (uint32_t)k, 0u, tag, p.seed);
    float t = (p.a - 1.0f) * u01(u.x) + 1.0f;
    zz = t * t / p.a;
    lu = logf(u01(u.y));
    bool oob = false;
    const int nvar = p.nvar;
    for (int q = 0; q < nvar; ++q) {
        if (!p.is_global[q]) { out[q] = 0.0f; continue; }
        float gq = g[q0 * nvar + q];
        float val = gq + (g[w * nvar + q] - gq) * zz;
        oob |= (val < p.lb[q]) || (val > p.ub[q]);
        out[q] = fminf(fmaxf(val, p.lb[q]), p.ub[q]);
    }
    return oob;
}

// Start value of global q for walker w: uniform over [lb, ub] (mcmc.m:488).
__device__ __forceinline__ float gwg_global_init(const McmcParams& p, int w, int q) {
    U4 u = philox((uint32_t)w, (uint32_t)(q >> 2), 0u, kTagGwGInit, p.seed);
    uint32_t r = (q & 3) == 0 ? u.x : (q & 3) == 1 ? u.y : (q & 3) == 2 ? u.z : u.w;
    return p.lb[q] + (p.ub[q] - p.lb[q]) * u01(r);
}

// One thread per (voxel, walker); blockDim = vpb * W.  NV = parameters +
// noise at compile time (per-thread vectors in registers).
template <int MODEL, int NV>
__global__ void gwg_step_kernel(McmcParams p, int rr, int k, int warm, int flags, int half, float* xstate,
                                double* lpstate) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ DevProtocol s_P;
    stage_protocol(p.P, &s_P);
    constexpr int nvar = NV;
    const int W = p.nwalker, nm = p.nm, h = W / 2;
    const int vpb = blockDim.x / W;
    const int vl = threadIdx.x / W, w = threadIdx.x % W;
    const int v = blockIdx.x * vpb + vl;
    const bool live = v < p.nvox;
    double* s_red = reinterpret_cast<double*>(smem_raw);          // [vpb][W]
    float* xs = reinterpret_cast<float*>(s_red + vpb * W);         // [vpb][W][nvar] locals
    float* s_g = xs + vpb * W * nvar;                              // [W][nvar] globals
    float* s_gp = s_g + W * nvar;                                  // [W][nvar] global proposals
    float* ys = s_gp + W * nvar;                                   // [vpb][nm]
    float* ws = ys + vpb * nm;                                     // [vpb][nm]
    float* xv = xs + vl * W * nvar;
    const float* yv = ys + vl * nm;
    const float* wv = p.weights ? ws + vl * nm : nullptr;
    if (live)
        for (int m = w; m < nm; m += W) {
            ys[vl * nm + m] = p.data[(size_t)m * p.nvox + v];
            if (p.weights) ws[vl * nm + m] = p.weights[(size_t)m * p.nvox + v];
        }
    for (int i = threadIdx.x; i < W * nvar; i += blockDim.x) {
        int ww = i / nvar, q = i % nvar;
        float gv = 0.0f;
        if (p.is_global[q]) gv = (flags & kGwgInit) ? gwg_global_init(p, ww, q) : p.gstate[(size_t)q * W + ww];
        s_g[i] = gv;
        if ((flags & kGwgInit) && blockIdx.x == 0 && p.is_global[q]) p.gstate[(size_t)q * W + ww] = gv;
    }
    float b1 = (live && p.b1) ? p.b1[v] : 1.0f;
    float sa[MODEL == kR1R2S ? kMaxFA : 1], ca[MODEL == kR1R2S ? kMaxFA : 1];
    if (MODEL == kR1R2S)
        for (int f = 0; f < p.P.n_fa; ++f) sincosf(b1 * p.P.fa_rad[f], &sa[f], &ca[f]);
    VoxAux va{b1, sa, ca, 1};
    float x[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) x[q] = 0.0f;
    if (live) {
        if (flags & kGwgInit) {
            // locals: x0 + (ub-lb)*startRange*randn, clamped (mcmc.m:483-484), goodman_weare's stream
            float xi[NV];
            gw_walker_start<NV>(p, v, w, xi);
#pragma unroll
            for (int q = 0; q < NV; ++q)
                if (!p.is_global[q]) x[q] = xi[q];
        } else {
#pragma unroll
            for (int q = 0; q < NV; ++q)
                if (!p.is_global[q]) x[q] = xstate[((size_t)q * p.nvox + v) * W + w];
        }
#pragma unroll
        for (int q = 0; q < NV; ++q) xv[w * NV + q] = x[q];
    }
    __syncthreads();
    // parameter vector of (this voxel, walker ww) with globals gsrc
    auto compose = [&](const float (&loc)[NV], const float* gsrc, float (&out)[NV]) {
#pragma unroll
        for (int q = 0; q < NV; ++q) out[q] = p.is_global[q] ? gsrc[q] : loc[q];
    };
    double lp = 0.0;
    if (live) {
        if (flags & kGwgInit) {
            float xx[NV];
            compose(x, s_g + w * nvar, xx);
            lp = log_prob_t<MODEL, NV>(nm, s_P, xx, yv, 1, wv, 1, va);
        } else {
            lp = lpstate[(size_t)v * W + w];
            if ((flags & kGwgApply) && p.gacc[w]) lp = p.lpg[(size_t)v * W + w];
        }
    }
    unsigned int nacc = 0;
    if (flags & kGwgLocal) {
        const int* pt = p.partner + ((size_t)rr * p.iteration + (k - 1)) * W;
        const float expo = (float)(p.nnd - 1);
        for (int s = 0; s < (p.update == 0 ? 1 : 2); ++s) {
            const bool act = live && (p.update == 0 || (s == 0 ? w < h : w >= h));
            float xn[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) xn[q] = 0.0f;
            bool acc = false;
            double lpp = 0.0;
            if (act) {
                int q0 = pt[w];
                uint32_t tag = kTagGwMove | ((uint32_t)rr << 16) | (p.update ? kTagRedBlack : 0u);
                U4 u = philox((uint32_t)v, (uint32_t)w, (uint32_t)k, tag, p.seed);
                float t = (p.a - 1.0f) * u01(u.x) + 1.0f;
                float zz = t * t / p.a;
                bool oob = false;
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    if (p.is_global[q]) { xn[q] = 0.0f; continue; }
                    float xq = xv[q0 * nvar + q];
                    float xp = xq + (xv[w * nvar + q] - xq) * zz;
                    oob |= (xp < p.lb[q]) || (xp > p.ub[q]);
                    xn[q] = fminf(fmaxf(xp, p.lb[q]), p.ub[q]);
                }
                float xx[NV];
                compose(xn, s_g + w * nvar, xx);
                lpp = log_prob_t<MODEL, NV>(nm, s_P, xx, yv, 1, wv, 1, va);
                double lr = (double)expo * (double)logf(zz) + (lpp - lp);
                acc = !oob && lr > (double)logf(u01(u.y));
            }
            __syncthreads();  // the (half-)ensemble was read before any walker moves
            if (act && acc) {
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    x[q] = xn[q];
                    xv[w * NV + q] = xn[q];
                }
                lp = lpp;
                ++nacc;
            }
            __syncthreads();
        }
        // kept local samples: per voxel, summed over walkers in order (no atomics)
        int c = warm ? -1 : kept_index(p, k);
        if (c >= 0 && live) {
            for (int q = w; q < nvar; q += W) {
                if (p.is_global[q]) continue;
                double sh = (double)p.shift[(size_t)q * p.nvox + v], s1 = 0.0, s2 = 0.0;
                for (int ww = 0; ww < W; ++ww) {
                    double d = (double)xv[ww * nvar + q] - sh;
                    s1 += d;
                    s2 += d * d;
                }
                p.sum[(size_t)q * p.nvox + v] += s1;
                p.sumsq[(size_t)q * p.nvox + v] += s2;
            }
            if (p.posterior)
#pragma unroll
                for (int q = 0; q < NV; ++q)
                    if (!p.is_global[q])
                        p.posterior[((((size_t)q * p.repetition + rr) * p.ns + c) * W + w) * p.nvox + v] = x[q];
        }
    }
    if (flags & kGwgEval) {
        for (int ww = threadIdx.x; ww < W; ww += blockDim.x) {
            if (!gwg_active(half, ww, W)) continue;
            float zz, lu;
            bool oob = gwg_proposal(p, rr, k, warm, ww, s_g, s_gp + ww * nvar, zz, lu);
            if (blockIdx.x == 0) {  // published for the accept kernel
                for (int q = 0; q < nvar; ++q) p.gprop[(size_t)q * W + ww] = s_gp[ww * nvar + q];
                p.gzz[ww] = zz;
                p.glu[ww] = lu;
                p.goob[ww] = oob ? 1 : 0;
            }
        }
        __syncthreads();
        const bool act = gwg_active(half, w, W);
        double d = 0.0;
        if (live && act) {
            float xx[NV];
            compose(x, s_gp + w * nvar, xx);
            double lpg = log_prob_t<MODEL, NV>(nm, s_P, xx, yv, 1, wv, 1, va);
            p.lpg[(size_t)v * W + w] = lpg;
            d = lpg - lp;
        }
        s_red[vl * W + w] = d;
        __syncthreads();
        if (vl == 0 && act) {
            double t = 0.0;
            for (int j = 0; j < vpb; ++j) t += s_red[j * W + w];
            p.partial[(size_t)w * gridDim.x + blockIdx.x] = t;
        }
    }
    if (live) {
#pragma unroll
        for (int q = 0; q < NV; ++q)
            if (!p.is_global[q]) xstate[((size_t)q * p.nvox + v) * W + w] = x[q];
        lpstate[(size_t)v * W + w] = lp;
    }
    unsigned int wsum = nacc;
    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(p.n_acc, (unsigned long long)wsum);
}

// One CTA per walker (grid = W).  c >= 0: record the kept global sample c.
__global__ void gwg_accept_kernel(McmcParams p, int rr, int k, int warm, int half, int c, int nparts) {
    __shared__ double red[256];
    __shared__ float s_g[kMaxParam];
    const int w = blockIdx.x, W = p.nwalker;
    const bool act = gwg_active(half, w, W);
    double t = 0.0;
    if (act)
        for (int i = threadIdx.x; i < nparts; i += blockDim.x) t += p.partial[(size_t)w * nparts + i];
    red[threadIdx.x] = t;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        int acc = 0;
        float gp[kMaxParam];
        if (act) {
            // the proposal the step kernel evaluated (mcmc.m:598-603)
            for (int q = 0; q < p.nvar; ++q) gp[q] = p.gprop[(size_t)q * W + w];
            double lr = (double)(p.ng - 1) * (double)logf(p.gzz[w]) + red[0];
            acc = !p.goob[w] && lr > (double)p.glu[w];
            if (acc) {
                for (int q = 0; q < p.nvar; ++q)
                    if (p.is_global[q]) p.gstate[(size_t)q * W + w] = gp[q];
                atomicAdd(p.n_gacc, 1ull);
            }
        }
        p.gacc[w] = acc;
        for (int q = 0; q < p.nvar; ++q) s_g[q] = p.gstate[(size_t)q * W + w];
        if (c >= 0)
            for (int q = 0; q < p.nvar; ++q)
                if (p.is_global[q]) {
                    double d = (double)s_g[q] - (double)p.shift[(size_t)q * p.nvox];
                    p.gsum[(size_t)q * W + w] += d;
                    p.gsumsq[(size_t)q * W + w] += d * d;
                }
    }
    __syncthreads();
    if (c >= 0 && p.posterior)
        for (int q = 0; q < p.nvar; ++q)
            if (p.is_global[q])
                for (int v = threadIdx.x; v < p.nvox; v += blockDim.x)
                    p.posterior[((((size_t)q * p.repetition + rr) * p.ns + c) * W + w) * p.nvox + v] = s_g[q];
}

// mean / std of the global parameters over W * ns * rep samples (unfilled
// slots count as zeros, as for the locals), repeated for every voxel.
__global__ void gwg_finalize_kernel(McmcParams p, int missing, float* mean, float* stdv) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= p.nvox) return;
    const int W = p.nwalker;
    double N = (double)W * p.ns * p.repetition;
    for (int q = 0; q < p.nvar; ++q) {
        if (!p.is_global[q]) continue;
        double sh = (double)p.shift[(size_t)q * p.nvox];
        double s1 = 0.0, s2 = 0.0;
        for (int w = 0; w < W; ++w) {
            s1 += p.gsum[(size_t)q * W + w];
            s2 += p.gsumsq[(size_t)q * W + w];
        }
        double nz = (double)missing * W * p.repetition;
        s1 += nz * (-sh);
        s2 += nz * sh * sh;
        double md = s1 / N;
        double var = N > 1.0 ? (s2 - s1 * md) / (N - 1.0) : 0.0;
        if (mean) mean[(size_t)q * p.nvox + v] = (float)(sh + md);
        if (stdv) stdv[(size_t)q * p.nvox + v] = (float)sqrt(fmax(var, 0.0));
    }
}

// shift = clamp(x0): the running sums are taken about the start value.
__global__ void mcmc_shift_kernel(McmcParams p) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= p.nvox) return;
    for (int q = 0; q < p.nvar; ++q)
        p.shift[(size_t)q * p.nvox + v] = fminf(fmaxf(p.x0[(size_t)q * p.nvox + v], p.lb[q]), p.ub[q]);
}

// mean / std (N-1) over W*ns*rep samples; slots the reference preallocates
// but never fills stay zero and are counted (res2out, mcmc.m:806-862).
__global__ void mcmc_finalize_kernel(McmcParams p, int missing, float* mean, float* stdv) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= p.nvox) return;
    int W = p.algorithm == 1 ? p.nwalker : 1;
    double N = (double)W * p.ns * p.repetition;
    for (int q = 0; q < p.nvar; ++q) {
        size_t i = (size_t)q * p.nvox + v;
        double sh = (double)p.shift[i];
        double s1 = p.sum[i], s2 = p.sumsq[i];
        double nz = (double)missing * W * p.repetition;
        s1 += nz * (-sh);
        s2 += nz * sh * sh;
        double md = s1 / N;
        double var = N > 1.0 ? (s2 - s1 * md) / (N - 1.0) : 0.0;
        if (mean) mean[i] = (float)(sh + md);
        if (stdv) stdv[i] = (float)sqrt(fmax(var, 0.0));
    }
}

cudaError_t launch_mcmc_partners(const McmcParams& p, int* partner, cudaStream_t s) {
    int n = p.repetition * p.iteration;
    int block = 128;
    gw_partner_kernel<<<(n + block - 1) / block, block, 0, s>>>(p, partner, p.iteration, 0);
    ++g_kernel_launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || p.ng == 0) return e;
    n = p.repetition * p.nsteps_g;
    gw_partner_kernel<<<(n + block - 1) / block, block, 0, s>>>(p, const_cast<int*>(p.gpartner), p.nsteps_g, 1);
    ++g_kernel_launches;
    return cudaGetLastError();
}

// Goodman-Weare launch shape for a block hint (threads): whole voxels of
// tpv threads (one walker, or one walker of each half) per CTA.
static void gw_shape(const McmcParams& p, int block_hint, int* vpb, int* block, size_t* smem) {
    const int W = p.nwalker, h = W / 2;
    const int tpv = p.update == 0 ? W : W - h;
    const int target = block_hint > 0 ? block_hint : 128;
    *vpb = target / tpv > 0 ? target / tpv : 1;
    *block = *vpb * tpv;
    *smem = sizeof(double) * 2 * (size_t)(*vpb) * W * p.nvar +
            sizeof(float) * ((size_t)(*vpb) * W * p.nvar + 2 * (size_t)(*vpb) * p.nm);
}

// Steps [k0, k1] of repetition rr as one launch (init: the walkers start at k0 == 1).
template <int MODEL>
static cudaError_t mcmc_launch_steps(const McmcParams& p, int block_hint, int rr, int k0, int k1, float* xstate,
                                     double* lpstate, double* sum, double* sumsq, cudaStream_t s) {
    constexpr int NV = ModelNP<MODEL>::value + 1;  // the model's parameters and the noise sigma
    if (p.nvar != NV) return cudaErrorInvalidValue;
    if (p.algorithm == 1) {
        int vpb, block;
        size_t smem;
        gw_shape(p, block_hint, &vpb, &block, &smem);
        const int nb = (p.nvox + vpb - 1) / vpb;
        auto k = p.update == 0 ? gw_kernel<MODEL, NV, false> : gw_kernel<MODEL, NV, true>;
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        k<<<nb, block, smem, s>>>(p, rr, k0, k1, k0 == 1 ? 1 : 0, xstate, lpstate, sum, sumsq);
    } else {
        const int block = block_hint > 0 ? block_hint : 128;
        const int nb = (p.nvox + block - 1) / block;
        mh_kernel<MODEL, NV><<<nb, block, 0, s>>>(p, rr, k0, k1, k0 == 1 ? 1 : 0, xstate, lpstate, sum, sumsq);
    }
    ++g_kernel_launches;
    return cudaGetLastError();
}

template <int MODEL>
static cudaError_t mcmc_run_model(const McmcParams& p, int block_hint, cudaStream_t s,
                                  float* xstate, double* lpstate) {
    const int chunk = 250;  // steps per launch: bounded kernel duration
    for (int rr = 0; rr < p.repetition; ++rr)
        for (int k0 = 1; k0 <= p.iteration; k0 += chunk) {
            int k1 = k0 + chunk - 1 < p.iteration ? k0 + chunk - 1 : p.iteration;
            cudaError_t e = mcmc_launch_steps<MODEL>(p, block_hint, rr, k0, k1, xstate, lpstate, p.sum, p.sumsq, s);
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

int mcmc_block_candidates(const McmcParams& p, int* out, int maxn) {
    int n = 0;
    if (p.algorithm == 1) {
        const int W = p.nwalker, tpv = p.update == 0 ? W : W - W / 2;
        for (int vpb = 1; vpb <= 32 && n < maxn; vpb *= 2) {
            const int block = vpb * tpv;
            if (block > 1024) break;
            if (block < 32 && vpb < 32) continue;  // at least one warp
            out[n++] = block;
        }
    } else {
        for (int b = 64; b <= 512 && n < maxn; b *= 2) out[n++] = b;
    }
    return n;
}

cudaError_t launch_mcmc_trial(const McmcParams& p, int model, int block_hint, int k1, float* xstate,
                              double* lpstate, double* sum, double* sumsq, cudaStream_t s) {
    switch (model) {
    case kR2S: return mcmc_launch_steps<kR2S>(p, block_hint, 0, 1, k1, xstate, lpstate, sum, sumsq, s);
    case kR1R2S: return mcmc_launch_steps<kR1R2S>(p, block_hint, 0, 1, k1, xstate, lpstate, sum, sumsq, s);
    case kNEXI: return mcmc_launch_steps<kNEXI>(p, block_hint, 0, 1, k1, xstate, lpstate, sum, sumsq, s);
    default: return mcmc_launch_steps<kNEXI2>(p, block_hint, 0, 1, k1, xstate, lpstate, sum, sumsq, s);
    }
}

int kept_index_host(const McmcParams& p, int k) {
    if (k <= p.nburnin) return -1;
    int j = k - p.nburnin + 1;
    if (j % p.thinning) return -1;
    int c = j / p.thinning - (p.thinning == 1 ? 1 : 0) - 1;
    return c < p.ns ? c : -1;
}

void gwg_launch_shape(const McmcParams& p, int block_hint, int* vpb, int* block, int* nblocks, size_t* smem) {
    const int W = p.nwalker;
    int target = block_hint > 0 ? block_hint : 256;
    *vpb = target / W > 0 ? target / W : 1;
    *block = *vpb * W;
    *nblocks = (p.nvox + *vpb - 1) / *vpb;
    *smem = sizeof(double) * (size_t)(*vpb) * W +
            sizeof(float) * ((size_t)(*vpb) * W * p.nvar + 2 * (size_t)W * p.nvar + 2 * (size_t)(*vpb) * p.nm);
}

template <int MODEL>
static cudaError_t mcmc_run_global(const McmcParams& p, int block_hint, cudaStream_t s, float* xstate,
                                   double* lpstate) {
    if (p.nvar != ModelNP<MODEL>::value + 1) return cudaErrorInvalidValue;
    int vpb, block, nb;
    size_t smem;
    gwg_launch_shape(p, block_hint, &vpb, &block, &nb, &smem);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(gwg_step_kernel<MODEL, ModelNP<MODEL>::value + 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    auto A = [&](int rr, int k, int warm, int flags, int half) {
        gwg_step_kernel<MODEL, ModelNP<MODEL>::value + 1><<<nb, block, smem, s>>>(p, rr, k, warm, flags, half,
                                                                                  xstate, lpstate);
        ++g_kernel_launches;
    };
    auto B = [&](int rr, int k, int warm, int half, int c) {
        gwg_accept_kernel<<<p.nwalker, 256, 0, s>>>(p, rr, k, warm, half, c, nb);
        ++g_kernel_launches;
    };
    for (int rr = 0; rr < p.repetition; ++rr) {
        bool first = true;
        for (int kw = 1; kw <= p.global_warmup; ++kw) {
            int f = (first ? kGwgInit : kGwgApply) | kGwgEval;
            first = false;
            if (p.update == 0) {
                A(rr, kw, 1, f, -1);
                B(rr, kw, 1, -1, -1);
            } else {
                A(rr, kw, 1, f, 0);
                B(rr, kw, 1, 0, -1);
                A(rr, kw, 1, kGwgApply | kGwgEval, 1);
                B(rr, kw, 1, 1, -1);
            }
        }
        for (int k = 1; k <= p.iteration; ++k) {
            int f = (first ? kGwgInit : kGwgApply) | kGwgLocal | kGwgEval;
            first = false;
            int c = kept_index_host(p, k);
            if (p.update == 0) {
                A(rr, k, 0, f, -1);
                B(rr, k, 0, -1, c);
            } else {
                A(rr, k, 0, f, 0);
                B(rr, k, 0, 0, -1);
                A(rr, k, 0, kGwgApply | kGwgEval, 1);
                B(rr, k, 0, 1, c);
            }
            if ((k & 63) == 0) {
                cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) return e;
            }
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_mcmc(const McmcParams& p, int model, int block, cudaStream_t s) {
    // walker state between chunked launches
    size_t W = p.algorithm == 1 ? (size_t)p.nwalker : 1;
    float* xstate = nullptr;
    double* lpstate = nullptr;
    cudaError_t e = cudaMallocAsync(&xstate, sizeof(float) * p.nvar * p.nvox * W, s);
    if (e != cudaSuccess) return e;
    e = cudaMallocAsync(&lpstate, sizeof(double) * p.nvox * W, s);
    if (e != cudaSuccess) { cudaFreeAsync(xstate, s); return e; }
    mcmc_shift_kernel<<<(p.nvox + 127) / 128, 128, 0, s>>>(p);
    ++g_kernel_launches;
    if (p.ng > 0) {
        switch (model) {
        case kR2S: e = mcmc_run_global<kR2S>(p, block, s, xstate, lpstate); break;
        case kR1R2S: e = mcmc_run_global<kR1R2S>(p, block, s, xstate, lpstate); break;
        case kNEXI: e = mcmc_run_global<kNEXI>(p, block, s, xstate, lpstate); break;
        default: e = mcmc_run_global<kNEXI2>(p, block, s, xstate, lpstate); break;
        }
        cudaFreeAsync(xstate, s);
        cudaFreeAsync(lpstate, s);
        return e;
    }
    switch (model) {
    case kR2S: e = mcmc_run_model<kR2S>(p, block, s, xstate, lpstate); break;
    case kR1R2S: e = mcmc_run_model<kR1R2S>(p, block, s, xstate, lpstate); break;
    case kNEXI: e = mcmc_run_model<kNEXI>(p, block, s, xstate, lpstate); break;
    default: e = mcmc_run_model<kNEXI2>(p, block, s, xstate, lpstate); break;
    }
    cudaFreeAsync(xstate, s);
    cudaFreeAsync(lpstate, s);
    return e;
}

int mcmc_missing_slots(const McmcParams& p) {
    // kept = #k in (nburnin, iteration] with (k - nburnin + 1) % thinning == 0
    int kept = 0;
    for (int k = p.nburnin + 1; k <= p.iteration; ++k)
        if ((k - p.nburnin + 1) % p.thinning == 0) ++kept;
    int missing = p.ns - kept;
    return missing < 0 ? 0 : missing;
}

cudaError_t launch_mcmc_finalize(const McmcParams& p, float* mean, float* stdv, cudaStream_t s) {
    const int missing = mcmc_missing_slots(p);
    mcmc_finalize_kernel<<<(p.nvox + 127) / 128, 128, 0, s>>>(p, missing, mean, stdv);
    ++g_kernel_launches;
    if (p.ng > 0) {
        gwg_finalize_kernel<<<(p.nvox + 127) / 128, 128, 0, s>>>(p, missing, mean, stdv);
        ++g_kernel_launches;
    }
    return cudaGetLastError();
}

}  // namespace gx
