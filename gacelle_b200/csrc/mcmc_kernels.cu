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

// Partner table: simultaneous -> one derangement per (rep, step) (find_partner);
// red-black -> absolute index of the frozen-half anchor of every active walker
// (frozen(randi(numel(frozen),1,na)), mcmc.m:328-329).
__global__ void gw_partner_kernel(McmcParams p, int* partner) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= p.repetition * p.iteration) return;
    int rr = idx / p.iteration, k = idx % p.iteration + 1;
    int W = p.nwalker;
    int* out = partner + (size_t)idx * W;
    if (p.update == 0) {
        int perm[kMaxWalker];
        bool ok = false;
        for (uint32_t attempt = 0; attempt < 4096 && !ok; ++attempt) {
            for (int i = 0; i < W; ++i) perm[i] = i;
            U4 u{0, 0, 0, 0};
            for (int i = W - 1, d = 0; i >= 1; --i, ++d) {
                if ((d & 3) == 0)
                    u = philox((uint32_t)k, attempt, (uint32_t)(d >> 2), kTagGwPerm | ((uint32_t)rr << 16), p.seed);
                uint32_t r = (d & 3) == 0 ? u.x : (d & 3) == 1 ? u.y : (d & 3) == 2 ? u.z : u.w;
                int j = (int)rand_below(r, (uint32_t)(i + 1));
                int t = perm[i]; perm[i] = perm[j]; perm[j] = t;
            }
            ok = true;
            for (int i = 0; i < W; ++i) ok = ok && perm[i] != i;
        }
        for (int i = 0; i < W; ++i) out[i] = ok ? perm[i] : (i + 1) % W;
    } else {
        int h = W / 2;
        for (int half = 0; half < 2; ++half) {
            int na = half == 0 ? h : W - h, nf = half == 0 ? W - h : h, f0 = half == 0 ? h : 0;
            int a0 = half == 0 ? 0 : h;
            U4 u{0, 0, 0, 0};
            for (int a = 0; a < na; ++a) {
                if ((a & 3) == 0)
                    u = philox((uint32_t)k, (uint32_t)half, (uint32_t)(a >> 2), kTagGwRbPart | ((uint32_t)rr << 16), p.seed);
                uint32_t r = (a & 3) == 0 ? u.x : (a & 3) == 1 ? u.y : (a & 3) == 2 ? u.z : u.w;
                out[a0 + a] = f0 + (int)rand_below(r, (uint32_t)nf);
            }
        }
    }
}

template <int MODEL>
__device__ __forceinline__ double log_prob(const McmcParams& p, const DevProtocol& P, const float* x,
                                           const float* y, const float* w, const VoxAux& va) {
    constexpr int NP = ModelNP<MODEL>::value;
    SosSink<NP> sink{y, 1, w, 1, 0.0};
    model_eval<MODEL>(P, x, va, sink);
    double noise = (double)x[p.nvar - 1];
    double n2 = noise * noise;
    return -sink.sos / (2.0 * n2) - 0.5 * p.nm * log(6.283185307179586 * n2);
}

__device__ __forceinline__ int kept_index(const McmcParams& p, int k) {
    if (k <= p.nburnin) return -1;
    int j = k - p.nburnin + 1;
    if (j % p.thinning) return -1;
    int c = j / p.thinning - (p.thinning == 1 ? 1 : 0) - 1;
    return c < p.ns ? c : -1;
}

// Goodman-Weare, steps [k0, k1] of repetition rr.  State between launches:
// xstate [nvar][nvox][W], lpstate [nvox][W].
template <int MODEL>
__global__ void gw_kernel(McmcParams p, int rr, int k0, int k1, int init, float* xstate,
                          double* lpstate, double* sum, double* sumsq) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ DevProtocol s_P;
    stage_protocol(p.P, &s_P);
    const int W = p.nwalker, nvar = p.nvar, nm = p.nm;
    const int h = W / 2;
    const int tpv = p.update == 0 ? W : (W - h);
    const int vpb = blockDim.x / tpv;
    const int vl = threadIdx.x / tpv, a = threadIdx.x % tpv;
    const int v = blockIdx.x * vpb + vl;
    const bool in_block = vl < vpb;
    const bool live = in_block && v < p.nvox;
    float* xs = reinterpret_cast<float*>(smem_raw);               // [vpb][W][nvar]
    float* ys = xs + vpb * W * nvar;                              // [vpb][nm]
    float* ws = ys + vpb * nm;                                    // [vpb][nm]
    float* xv = xs + (in_block ? vl : 0) * W * nvar;
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

    // walkers owned by this thread
    int wown[2];
    int nown;
    if (p.update == 0) { wown[0] = a; nown = 1; }
    else { wown[0] = a < h ? a : -1; wown[1] = h + a; nown = 2; }
    float x[2][kMaxParam];
    double lp[2];
    double s1[kMaxParam], s2[kMaxParam];
    for (int q = 0; q < kMaxParam; ++q) { s1[q] = 0.0; s2[q] = 0.0; }
    __syncthreads();
    for (int o = 0; o < nown; ++o) {
        int w = wown[o];
        if (!live || w < 0 || w >= W) continue;
        if (init) {
            // walker start: x0 + (ub-lb)*startRange*randn, clamped (mcmc.m:267-275)
            float nrm[8];
            for (int j = 0; j * 4 < nvar; ++j) {
                U4 u = philox((uint32_t)v, (uint32_t)w, (uint32_t)j, kTagGwInit, p.seed);
                float n0, n1, n2, n3;
                box_muller(u.x, u.y, n0, n1);
                box_muller(u.z, u.w, n2, n3);
                nrm[4 * j] = n0; nrm[4 * j + 1] = n1; nrm[4 * j + 2] = n2; nrm[4 * j + 3] = n3;
            }
            for (int q = 0; q < nvar; ++q) {
                float val = p.x0[(size_t)q * p.nvox + v] + (p.ub[q] - p.lb[q]) * p.start_range * nrm[q];
                x[o][q] = fminf(fmaxf(val, p.lb[q]), p.ub[q]);
            }
        } else {
            for (int q = 0; q < nvar; ++q) x[o][q] = xstate[((size_t)q * p.nvox + v) * W + w];
        }
        for (int q = 0; q < nvar; ++q) xv[w * nvar + q] = x[o][q];
    }
    __syncthreads();
    for (int o = 0; o < nown; ++o) {
        int w = wown[o];
        if (!live || w < 0 || w >= W) continue;
        lp[o] = init ? log_prob<MODEL>(p, s_P, x[o], yv, wv, va) : lpstate[(size_t)v * W + w];
    }
    if (!init && live)
        for (int q = 0; q < nvar; ++q) {
            s1[q] = 0.0;
            s2[q] = 0.0;
        }
    unsigned int nacc = 0;
    const float amin1 = p.a - 1.0f;

    for (int k = k0; k <= k1; ++k) {
        const int* pt = p.partner + ((size_t)rr * p.iteration + (k - 1)) * W;
        if (p.update == 0) {
            float xn[kMaxParam];
            bool acc = false;
            double lpp = 0.0;
            int w = wown[0];
            if (live) {
                int q = pt[w];
                U4 u = philox((uint32_t)v, (uint32_t)w, (uint32_t)k, kTagGwMove | ((uint32_t)rr << 16), p.seed);
                float t = amin1 * u01(u.x) + 1.0f;
                float zz = t * t / p.a;
                bool oob = false;
                for (int j = 0; j < nvar; ++j) {
                    float xq = xv[q * nvar + j];
                    float xp = xq + (xv[w * nvar + j] - xq) * zz;
                    oob |= (xp < p.lb[j]) || (xp > p.ub[j]);
                    xn[j] = fminf(fmaxf(xp, p.lb[j]), p.ub[j]);
                }
                lpp = log_prob<MODEL>(p, s_P, xn, yv, wv, va);
                double lr = (double)(nvar - 1) * (double)logf(zz) + (lpp - lp[0]);
                acc = !oob && lr > (double)logf(u01(u.y));
            }
            __syncthreads();  // every walker has read the old ensemble
            if (live && acc) {
                for (int j = 0; j < nvar; ++j) {
                    x[0][j] = xn[j];
                    xv[w * nvar + j] = xn[j];
                }
                lp[0] = lpp;
                ++nacc;
            }
            __syncthreads();
        } else {
            for (int s = 0; s < 2; ++s) {
                int o = s;  // slot 0: first half, slot 1: second half
                int w = wown[o];
                bool act = live && w >= 0 && w < W;
                if (act) {
                    int q = pt[w];
                    U4 u = philox((uint32_t)v, (uint32_t)w, (uint32_t)k,
                                  kTagGwMove | ((uint32_t)rr << 16) | (1u << 8), p.seed);
                    float t = amin1 * u01(u.x) + 1.0f;
                    float zz = t * t / p.a;
                    float xn[kMaxParam];
                    bool oob = false;
                    for (int j = 0; j < nvar; ++j) {
                        float xq = xv[q * nvar + j];
                        float xp = xq + (x[o][j] - xq) * zz;
                        oob |= (xp < p.lb[j]) || (xp > p.ub[j]);
                        xn[j] = fminf(fmaxf(xp, p.lb[j]), p.ub[j]);
                    }
                    double lpp = log_prob<MODEL>(p, s_P, xn, yv, wv, va);
                    double lr = (double)(nvar - 1) * (double)logf(zz) + (lpp - lp[o]);
                    if (!oob && lr > (double)logf(u01(u.y))) {
                        for (int j = 0; j < nvar; ++j) {
                            x[o][j] = xn[j];
                            xv[w * nvar + j] = xn[j];
                        }
                        lp[o] = lpp;
                        ++nacc;
                    }
                }
                __syncthreads();  // the moved half is visible before the other half anchors on it
            }
        }
        int c = kept_index(p, k);
        if (c >= 0 && live) {
            for (int o = 0; o < nown; ++o) {
                int w = wown[o];
                if (w < 0 || w >= W) continue;
                for (int j = 0; j < nvar; ++j) {
                    double d = (double)x[o][j] - (double)p.shift[(size_t)j * p.nvox + v];
                    s1[j] += d;
                    s2[j] += d * d;
                    if (p.posterior)
                        p.posterior[((((size_t)j * p.repetition + rr) * p.ns + c) * W + w) * p.nvox + v] = x[o][j];
                }
            }
        }
    }
    // persist walker state, fold the kept-sample sums of this launch
    if (live) {
        for (int o = 0; o < nown; ++o) {
            int w = wown[o];
            if (w < 0 || w >= W) continue;
            for (int q = 0; q < nvar; ++q) xstate[((size_t)q * p.nvox + v) * W + w] = x[o][q];
            lpstate[(size_t)v * W + w] = lp[o];
        }
        for (int j = 0; j < nvar; ++j) {
            if (s1[j] != 0.0) atomicAdd(&sum[(size_t)j * p.nvox + v], s1[j]);
            if (s2[j] != 0.0) atomicAdd(&sumsq[(size_t)j * p.nvox + v], s2[j]);
        }
    }
    unsigned int wsum = nacc;
    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(p.n_acc, (unsigned long long)wsum);
}

// Metropolis-Hastings, one thread per voxel (mcmc.m:144-167).
template <int MODEL>
__global__ void mh_kernel(McmcParams p, int rr, int k0, int k1, int init, float* xstate,
                          double* lpstate, double* sum, double* sumsq) {
    __shared__ DevProtocol s_P;
    stage_protocol(p.P, &s_P);
    __syncthreads();
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    bool live = v < p.nvox;
    const int nvar = p.nvar, nm = p.nm;
    float yv[kMaxMeas], wv[kMaxMeas];
    if (live)
        for (int m = 0; m < nm; ++m) {
            yv[m] = p.data[(size_t)m * p.nvox + v];
            wv[m] = p.weights ? p.weights[(size_t)m * p.nvox + v] : 1.0f;
        }
    float b1 = (live && p.b1) ? p.b1[v] : 1.0f;
    float sa[MODEL == kR1R2S ? kMaxFA : 1], ca[MODEL == kR1R2S ? kMaxFA : 1];
    if (MODEL == kR1R2S)
        for (int f = 0; f < p.P.n_fa; ++f) sincosf(b1 * p.P.fa_rad[f], &sa[f], &ca[f]);
    VoxAux va{b1, sa, ca, 1};
    float x[kMaxParam];
    double lp = 0.0;
    double s1[kMaxParam], s2[kMaxParam];
    for (int q = 0; q < kMaxParam; ++q) { s1[q] = 0.0; s2[q] = 0.0; x[q] = 0.0f; }
    unsigned int nacc = 0;
    if (live) {
        if (init) {
            for (int q = 0; q < nvar; ++q)
                x[q] = fminf(fmaxf(p.x0[(size_t)q * p.nvox + v], p.lb[q]), p.ub[q]);
            lp = log_prob<MODEL>(p, s_P, x, yv, wv, va);
        } else {
            for (int q = 0; q < nvar; ++q) x[q] = xstate[(size_t)q * p.nvox + v];
            lp = lpstate[v];
        }
        for (int k = k0; k <= k1; ++k) {
            float nrm[8];
            uint32_t tag = kTagMhMove | ((uint32_t)rr << 16);
            for (int j = 0; j * 4 < nvar; ++j) {
                U4 u = philox((uint32_t)v, (uint32_t)k, (uint32_t)j, tag, p.seed);
                float n0, n1, n2, n3;
                box_muller(u.x, u.y, n0, n1);
                box_muller(u.z, u.w, n2, n3);
                nrm[4 * j] = n0; nrm[4 * j + 1] = n1; nrm[4 * j + 2] = n2; nrm[4 * j + 3] = n3;
            }
            U4 ua = philox((uint32_t)v, (uint32_t)k, 8u, tag, p.seed);
            float xp[kMaxParam];
            bool oob = false;
            for (int q = 0; q < nvar; ++q) {
                float t = x[q] + p.xstep[q] * nrm[q];
                oob |= (t < p.lb[q]) || (t > p.ub[q]);
                xp[q] = fminf(fmaxf(t, p.lb[q]), p.ub[q]);
            }
            double lpp = log_prob<MODEL>(p, s_P, xp, yv, wv, va);
            if (!oob && (lpp - lp) > (double)logf(u01(ua.x))) {
                for (int q = 0; q < nvar; ++q) x[q] = xp[q];
                lp = lpp;
                ++nacc;
            }
            int c = kept_index(p, k);
            if (c >= 0)
                for (int j = 0; j < nvar; ++j) {
                    double d = (double)x[j] - (double)p.shift[(size_t)j * p.nvox + v];
                    s1[j] += d;
                    s2[j] += d * d;
                    if (p.posterior)
                        p.posterior[(((size_t)j * p.repetition + rr) * p.ns + c) * p.nvox + v] = x[j];
                }
        }
        for (int q = 0; q < nvar; ++q) xstate[(size_t)q * p.nvox + v] = x[q];
        lpstate[v] = lp;
        for (int j = 0; j < nvar; ++j) {
            sum[(size_t)j * p.nvox + v] += s1[j];
            sumsq[(size_t)j * p.nvox + v] += s2[j];
        }
    }
    unsigned int wsum = nacc;
    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(p.n_acc, (unsigned long long)wsum);
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
    gw_partner_kernel<<<(n + block - 1) / block, block, 0, s>>>(p, partner);
    ++g_kernel_launches;
    return cudaGetLastError();
}

template <int MODEL>
static cudaError_t mcmc_run_model(const McmcParams& p, int block_hint, cudaStream_t s,
                                  float* xstate, double* lpstate) {
    const int chunk = 250;  // steps per launch: bounded kernel duration
    if (p.algorithm == 1) {
        int W = p.nwalker, h = W / 2;
        int tpv = p.update == 0 ? W : W - h;
        int target = block_hint > 0 ? block_hint : 128;
        int vpb = target / tpv > 0 ? target / tpv : 1;
        int block = vpb * tpv;
        size_t smem = sizeof(float) * ((size_t)vpb * W * p.nvar + 2 * (size_t)vpb * p.nm);
        int nb = (p.nvox + vpb - 1) / vpb;
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(gw_kernel<MODEL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        for (int rr = 0; rr < p.repetition; ++rr)
            for (int k0 = 1; k0 <= p.iteration; k0 += chunk) {
                int k1 = k0 + chunk - 1 < p.iteration ? k0 + chunk - 1 : p.iteration;
                gw_kernel<MODEL><<<nb, block, smem, s>>>(p, rr, k0, k1, k0 == 1 ? 1 : 0, xstate, lpstate, p.sum, p.sumsq);
                ++g_kernel_launches;
                cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) return e;
            }
    } else {
        int block = block_hint > 0 ? block_hint : 128;
        int nb = (p.nvox + block - 1) / block;
        for (int rr = 0; rr < p.repetition; ++rr)
            for (int k0 = 1; k0 <= p.iteration; k0 += chunk) {
                int k1 = k0 + chunk - 1 < p.iteration ? k0 + chunk - 1 : p.iteration;
                mh_kernel<MODEL><<<nb, block, 0, s>>>(p, rr, k0, k1, k0 == 1 ? 1 : 0, xstate, lpstate, p.sum, p.sumsq);
                ++g_kernel_launches;
                cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) return e;
            }
    }
    return cudaSuccess;
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

cudaError_t launch_mcmc_finalize(const McmcParams& p, float* mean, float* stdv, cudaStream_t s) {
    // kept = #k in (nburnin, iteration] with (k - nburnin + 1) % thinning == 0
    int kept = 0;
    for (int k = p.nburnin + 1; k <= p.iteration; ++k)
        if ((k - p.nburnin + 1) % p.thinning == 0) ++kept;
    int missing = p.ns - kept;
    if (missing < 0) missing = 0;
    mcmc_finalize_kernel<<<(p.nvox + 127) / 128, 128, 0, s>>>(p, missing, mean, stdv);
    ++g_kernel_launches;
    return cudaGetLastError();
}

}  // namespace gx
