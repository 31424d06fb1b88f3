// askadam_kernels.cu -- askAdam on B200.
//
// Fused path
//   fused_kernel   one thread per voxel runs a whole range of epochs with the
//                  parameters and Adam moments in registers and the voxel's
//                  measurements staged once in shared memory: forward model,
//                  loss, hand-written adjoint, sigmoid chain rule and the
//                  optimiser update are one pass per epoch.  Per-epoch loss
//                  (and stopping statistics) are block-reduced and added in
//                  FP64 to a per-volume history; state is checkpointed every
//                  ckpt_every epochs so the host can rebuild the minimum-loss
//                  and stopping-epoch states by replay.
//   tv_step_kernel the same evaluation plus the anisotropic TV term for one
//                  epoch; the regularised maps travel between epochs in a
//                  double-buffered full grid (zeros outside the mask).
// Plain path (the op-by-op drop-in): unscale, forward, loss, adjoint, TV,
//                  z-gradient and optimiser kernels, one launch each per epoch.
//
// Reference: utils/askadam.m (model_gradient :23-117, optimisation :121-365,
// initialise_parameter :368-412, update_parameters :673-691,
// unscale_parameters :1063-1075), utils/spatial_total_variation.m.
#include <climits>

#include "gx_internal.h"

namespace gx {

long long g_kernel_launches = 0;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-reduce NQ per-thread values and add them in FP64 to dst[0..NQ).
// q[0] is scaled by scale0.  s_red holds 2*32*NQ doubles; alternating the
// half by epoch parity lets one __syncthreads per epoch suffice.
template <int NQ>
__device__ __forceinline__ void block_accumulate(const float (&q)[NQ], double* dst, double scale0,
                                                 double* s_red, int parity) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double* buf = s_red + parity * 32 * NQ;
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
        float s = warp_sum(q[k]);
        if (lane == 0) buf[warp * NQ + k] = (double)s;
    }
    __syncthreads();
    if (threadIdx.x < NQ) {
        double t = 0.0;
        for (int w = 0; w < nw; ++w) t += buf[w * NQ + threadIdx.x];
        if (threadIdx.x == 0) t *= scale0;
        if (t != 0.0) atomicAdd(dst + threadIdx.x, t);
    }
}

__device__ __forceinline__ OptConst opt_const(const AdamParams& a) {
    return OptConst{a.optimiser, a.beta1, a.beta2, a.eps, a.momentum, a.rms_decay, a.rms_eps};
}

__device__ __forceinline__ void opt_update(const AdamParams& a, float2 sc, float& z, float& m1,
                                           float& m2, float g) {
    opt_step(opt_const(a), sc, z, m1, m2, g);
}

__device__ __forceinline__ float voxel_sigma(const AdamParams& a, int v) {
    return a.sigma ? a.sigma[v] : a.sigma_default;
}

// Add the prior regulariser of voxel v to its physical-parameter gradient g
// and regularisation loss reg (in regmap order, like the TV terms).
template <int NP>
__device__ __forceinline__ void prior_voxel(const AdamParams& a, const DevVol& V, int v, const float (&th)[NP],
                                            float (&g)[NP], float& reg) {
    for (int r = 0; r < a.n_reg; ++r) {
        const int k = a.reg_param[r];
        const size_t i = (size_t)r * a.nvtot + v;
        float t = 0.0f;
#pragma unroll
        for (int kk = 0; kk < NP; ++kk)
            if (kk == k) t = th[kk];
        float cost, gr;
        prior_terms(t, a.prior_mu[i], a.prior_sd[i], cost, gr);
        reg = fma1(V.tv_scale[r], cost, reg);
#pragma unroll
        for (int kk = 0; kk < NP; ++kk)
            if (kk == k) g[kk] = fma1(V.tv_scale[r], gr, g[kk]);
    }
    if (v == V.off) reg = add1(reg, V.prior_off);
}

// ---------------------------------------------------------------------------
// State initialisation (initialise_parameter, utils/askadam.m:368-412).
// ---------------------------------------------------------------------------
__global__ void init_state_kernel(AdamParams a, const float* theta0, float randomness,
                                  uint64_t seed) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    int local = v - V.off;
    bool lin = a.transform == 1;
    for (int k = 0; k < a.np; ++k) {
        U4 u = philox((uint32_t)local, (uint32_t)k, 0u, kTagAdamInit, seed);
        float n0, n1;
        box_muller(u.x, u.y, n0, n1);
        float uni = u01(u.z);
        float lb = a.P.lb[k], ub = a.P.ub[k];
        float z;
        if (theta0) {
            float t0 = theta0[(size_t)k * a.nvtot + v];
            if (!lin) {
                float eb = 1e-4f * (ub - lb);
                float tc = fmaxf(fminf(t0, ub - eb), lb + eb);
                float nn = (tc - lb) / (ub - lb);
                z = (1.0f - randomness) * logf(nn / (1.0f - nn)) + randomness * n0;
            } else {
                z = (1.0f - randomness) * (t0 - lb) / (ub - lb) + randomness * uni;
            }
        } else {
            z = lin ? uni : randomness * n0;
        }
        if (lin) z = fminf(fmaxf(z, 0.0f), 1.0f);
        size_t i = (size_t)k * a.nvtot + v;
        a.z[i] = z;
        a.m1[i] = 0.0f;
        a.m2[i] = 0.0f;
        if (a.zprev) a.zprev[i] = z;
    }
}

// ---------------------------------------------------------------------------
// Fused multi-epoch kernel (no spatial coupling).
// ---------------------------------------------------------------------------
template <int MODEL, int LOSS, bool STATS>
__device__ __forceinline__ void fused_body(const AdamParams& a, int e_begin, int e_end, int update_last, int record) {
    constexpr int NP = ModelNP<MODEL>::value;
    constexpr int NQ = STATS ? kHistW : 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* s_red = reinterpret_cast<double*>(smem_raw);
    float* s_y = reinterpret_cast<float*>(s_red + 2 * 32 * NQ);
    const int B = blockDim.x, tid = threadIdx.x;
    const int v = blockIdx.x * B + tid;
    const int vol = a.blk_vol[blockIdx.x];
    const DevVol& V = a.vols[vol];
    const bool valid = (v - V.off) < V.nvox;
    const int nm = a.nm;
    float* s_w = s_y + nm * B;
    float* s_sa = a.weights ? s_w + nm * B : s_w;
    float* s_ca = s_sa + a.P.n_fa * B;
    __shared__ DevProtocol s_P;
    stage_protocol(a.P, &s_P);
    for (int m = 0; m < nm; ++m) s_y[m * B + tid] = a.data[(size_t)m * a.nvtot + v];
    if (a.weights)
        for (int m = 0; m < nm; ++m) s_w[m * B + tid] = a.weights[(size_t)m * a.nvtot + v];
    float b1 = a.b1 ? a.b1[v] : 1.0f;
    if (MODEL == kR1R2S)
        for (int f = 0; f < a.P.n_fa; ++f) sincosf(b1 * a.P.fa_rad[f], &s_sa[f * B + tid], &s_ca[f * B + tid]);
    VoxAux va{b1, s_sa + tid, s_ca + tid, B};
    va.sigma = voxel_sigma(a, v);
    LossAux aux = make_loss_aux(voxel_sigma(a, v));
    __syncthreads();

    float z[NP], m1[NP], m2[NP], zp[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        size_t i = (size_t)k * a.nvtot + v;
        z[k] = a.z[i];
        m1[k] = a.m1[i];
        m2[k] = a.m2[i];
        zp[k] = STATS ? a.zprev[i] : 0.0f;
    }
    const float normf = V.norm;
    const double normd = V.normd;
    const size_t slot = (size_t)3 * NP * a.nvtot;
    // the next checkpoint epoch (a multiple of ckpt_every), kept as a counter
    int next_ck = a.ckpt_every > 0 ? (e_begin + a.ckpt_every - 1) / a.ckpt_every * a.ckpt_every : INT_MAX;

    for (int e = e_begin; e <= e_end; ++e) {
        float th[NP], dth[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) th[k] = unscale(a.transform, a.P.lb[k], a.P.ub[k], z[k], dth[k]);
        LossAcc<LOSS, NP> acc;
        acc.total = 0.0f;
#pragma unroll
        for (int k = 0; k < NP; ++k) acc.g[k] = 0.0f;
        acc.y = s_y + tid; acc.ys = B;
        acc.w = a.weights ? s_w + tid : nullptr; acc.ws = B;
        acc.aux = aux; acc.mse_scale = a.mse_scale; acc.hd = a.huber_delta;
        acc.res = (a.res_out && e == e_end && valid) ? a.res_out + v : nullptr;
        acc.rs = a.nvtot;
        model_eval<MODEL, MODEL == kR1R2S>(s_P, th, va, acc);
        acc.finish();
        float gz[NP];
        float reg = 0.0f;
        if (a.prior_mu) {  // prior regulariser (the host records it through STATS)
            float gth[NP];
#pragma unroll
            for (int k = 0; k < NP; ++k) gth[k] = acc.g[k] * normf;
            if (valid) prior_voxel<NP>(a, V, v, th, gth, reg);
#pragma unroll
            for (int k = 0; k < NP; ++k) gz[k] = gth[k] * dth[k];
        } else {
#pragma unroll
            for (int k = 0; k < NP; ++k) gz[k] = acc.g[k] * normf * dth[k];
        }
        if (record) {
            float q[NQ];
            q[0] = valid ? acc.total : 0.0f;
            if (STATS) {
                float g2 = 0.f, z2 = 0.f, d2 = 0.f;
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    g2 += gz[k] * gz[k];
                    z2 += z[k] * z[k];
                    d2 += (z[k] - zp[k]) * (z[k] - zp[k]);
                }
                q[NQ > 1 ? 1 : 0] = reg;
                if (NQ > 4) {
                    q[2] = valid ? g2 : 0.f;
                    q[3] = valid ? z2 : 0.f;
                    q[4] = valid ? d2 : 0.f;
                }
            }
            block_accumulate<NQ>(q, a.hist + ((size_t)vol * (a.niter + 1) + e) * kHistW, normd,
                                 s_red, e & 1);
        }
        if (e <= update_last) {
            float2 sc = a.sched[e];
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                if (STATS) zp[k] = z[k];
                opt_update(a, sc, z[k], m1[k], m2[k], gz[k]);
            }
            if (e == next_ck) {
                next_ck += a.ckpt_every;
                float* c = a.ckpt + (size_t)(e / a.ckpt_every) * slot;
                if (valid)
#pragma unroll
                    for (int k = 0; k < NP; ++k) {
                        c[(size_t)k * a.nvtot + v] = z[k];
                        c[(size_t)(NP + k) * a.nvtot + v] = m1[k];
                        c[(size_t)(2 * NP + k) * a.nvtot + v] = m2[k];
                    }
            }
        }
    }
    if (valid) {
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            size_t i = (size_t)k * a.nvtot + v;
            a.z[i] = z[k];
            a.m1[i] = m1[k];
            a.m2[i] = m2[k];
            if (STATS) a.zprev[i] = zp[k];
        }
    }
}

template <int MODEL, int LOSS, bool STATS>
__global__ void fused_kernel(AdamParams a, int e_begin, int e_end, int update_last, int record) {
    fused_body<MODEL, LOSS, STATS>(a, e_begin, e_end, update_last, record);
}

// The joint R1-R2* model's fused kernel: the two-angle, 12-echo protocol with
// its echo loop unrolled, registers capped at 80 (unrolled and uncapped it
// takes 128 and loses half of the resident warps).
template <int LOSS, bool STATS>
__global__ void __maxnreg__(80) fused_kernel_r1r2s(AdamParams a, int e_begin, int e_end, int update_last,
                                                   int record) {
    fused_body<kR1R2S, LOSS, STATS>(a, e_begin, e_end, update_last, record);
}

template <int MODEL, int LOSS, bool STATS>
constexpr auto fused_kernel_fn() {
    if constexpr (MODEL == kR1R2S) return &fused_kernel_r1r2s<LOSS, STATS>;
    else return &fused_kernel<MODEL, LOSS, STATS>;
}

// ---------------------------------------------------------------------------
// One epoch with the spatial TV regulariser (utils/spatial_total_variation.m:
// periodic forward differences of the physical map, mask at the centre voxel,
// sum(|.|)/Nmask*lambda).  d cost / d theta(q) =
//   sum_d [ -mask(q) sgn(theta(q+e_d)-theta(q)) + mask(q-e_d) sgn(theta(q)-theta(q-e_d)) ] / vs_d
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sgnf(float x) { return (float)((x > 0.0f) - (x < 0.0f)); }

template <int MODEL, int LOSS, bool STATS>
__global__ void tv_step_kernel(AdamParams a, int e, int update, int record, int want_res) {
    constexpr int NP = ModelNP<MODEL>::value;
    constexpr int NQ = STATS ? kHistW : 2;
    __shared__ double s_red[2 * 32 * NQ];
    __shared__ DevProtocol s_P;
    stage_protocol(a.P, &s_P);
    __syncthreads();
    const int B = blockDim.x, tid = threadIdx.x;
    const int v = blockIdx.x * B + tid;
    const int vol = a.blk_vol[blockIdx.x];
    const DevVol& V = a.vols[vol];
    const bool valid = (v - V.off) < V.nvox;
    float z[NP], m1[NP], m2[NP], zp[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        size_t i = (size_t)k * a.nvtot + v;
        z[k] = a.z[i];
        m1[k] = a.m1[i];
        m2[k] = a.m2[i];
        zp[k] = STATS ? a.zprev[i] : 0.0f;
    }
    float b1 = a.b1 ? a.b1[v] : 1.0f;
    float sa[MODEL == kR1R2S ? kMaxFA : 1], ca[MODEL == kR1R2S ? kMaxFA : 1];
    if (MODEL == kR1R2S)
        for (int f = 0; f < a.P.n_fa; ++f) sincosf(b1 * a.P.fa_rad[f], &sa[f], &ca[f]);
    VoxAux va{b1, sa, ca, 1};
    va.sigma = voxel_sigma(a, v);
    float th[NP], dth[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) th[k] = unscale(a.transform, a.P.lb[k], a.P.ub[k], z[k], dth[k]);
    LossAcc<LOSS, NP> acc;
    acc.total = 0.0f;
#pragma unroll
    for (int k = 0; k < NP; ++k) acc.g[k] = 0.0f;
    acc.y = a.data + v; acc.ys = a.nvtot;
    acc.w = a.weights ? a.weights + v : nullptr; acc.ws = a.nvtot;
    acc.aux = make_loss_aux(voxel_sigma(a, v));
    acc.mse_scale = a.mse_scale; acc.hd = a.huber_delta;
    acc.res = (want_res && a.res_out && valid) ? a.res_out + v : nullptr;
    acc.rs = a.nvtot;
    model_eval<MODEL>(s_P, th, va, acc);
    acc.finish();
    float gth[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) gth[k] = acc.g[k] * V.norm;

    float reg = 0.0f;
    if (valid && a.surf_nb) {
        const unsigned char* mk = a.maskgrid + V.grid_off;
        for (int r = 0; r < a.n_reg; ++r) {
            const int k = a.reg_param[r];
            const float* G = a.grid_cur + (size_t)r * a.grid_total + V.grid_off;
            float c = 0.0f;
#pragma unroll
            for (int kk = 0; kk < NP; ++kk)
                if (kk == k) c = th[kk];
            float cost, gr;
            surf_tv_terms(c, G, mk, a.surf_nb + v, a.surf_len + v, a.surf_maxnb, a.nvtot, cost, gr);
            reg += V.tv_scale[r] * cost;
#pragma unroll
            for (int kk = 0; kk < NP; ++kk)
                if (kk == k) gth[kk] = fma1(V.tv_scale[r], gr, gth[kk]);
        }
    } else if (valid) {
        const int dx = V.dims[0], dy = V.dims[1], dz = V.dims[2];
        const int p = a.gidx[v];
        const int x = p % dx, yz = p / dx, y = yz % dy, zc = yz / dy;
        const int nd = a.tv_3d ? 3 : 2;
        const int sx = 1, sy = dx, sz = dx * dy;
        int fw[3] = {x + 1 < dx ? p + sx : p - x, y + 1 < dy ? p + sy : p - y * sy,
                     zc + 1 < dz ? p + sz : p - zc * sz};
        int bw[3] = {x > 0 ? p - sx : p + (dx - 1) * sx, y > 0 ? p - sy : p + (dy - 1) * sy,
                     zc > 0 ? p - sz : p + (dz - 1) * sz};
        const unsigned char* mk = a.maskgrid + V.grid_off;
        bool mb[3] = {mk[bw[0]] != 0, mk[bw[1]] != 0, mk[bw[2]] != 0};
        for (int r = 0; r < a.n_reg; ++r) {
            const int k = a.reg_param[r];
            const float* G = a.grid_cur + (size_t)r * a.grid_total + V.grid_off;
            float c = 0.0f;
#pragma unroll
            for (int kk = 0; kk < NP; ++kk)
                if (kk == k) c = th[kk];
            float f[3], b[3];
            for (int d = 0; d < nd; ++d) {
                f[d] = G[fw[d]];
                b[d] = G[bw[d]];
            }
            float cost, gr;
            tv_terms(c, f, b, mb, a.inv_vs, nd, cost, gr);
            reg += V.tv_scale[r] * cost;
#pragma unroll
            for (int kk = 0; kk < NP; ++kk)
                if (kk == k) gth[kk] = fma1(V.tv_scale[r], gr, gth[kk]);
        }
    }
    float gz[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) gz[k] = gth[k] * dth[k];
    if (record) {
        float q[NQ];
        q[0] = valid ? acc.total : 0.0f;
        q[1] = valid ? reg : 0.0f;
        if (STATS) {
            float g2 = 0.f, z2 = 0.f, d2 = 0.f;
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                g2 += gz[k] * gz[k];
                z2 += z[k] * z[k];
                d2 += (z[k] - zp[k]) * (z[k] - zp[k]);
            }
            if (NQ > 4) {
                q[2] = valid ? g2 : 0.f;
                q[3] = valid ? z2 : 0.f;
                q[4] = valid ? d2 : 0.f;
            }
        }
        block_accumulate<NQ>(q, a.hist + ((size_t)vol * (a.niter + 1) + e) * kHistW, V.normd,
                             s_red, 0);
    }
    if (update && valid) {
        float2 sc = a.sched[e];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            if (STATS) zp[k] = z[k];
            opt_update(a, sc, z[k], m1[k], m2[k], gz[k]);
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            size_t i = (size_t)k * a.nvtot + v;
            a.z[i] = z[k];
            a.m1[i] = m1[k];
            a.m2[i] = m2[k];
            if (STATS) a.zprev[i] = zp[k];
        }
        const int p = a.gidx[v];
        for (int r = 0; r < a.n_reg; ++r) {
            const int k = a.reg_param[r];
            float zk = 0.0f;
            float lb = a.P.lb[k], ub = a.P.ub[k];
#pragma unroll
            for (int kk = 0; kk < NP; ++kk)
                if (kk == k) zk = z[kk];
            float dd;
            a.grid_next[(size_t)r * a.grid_total + V.grid_off + p] = unscale(a.transform, lb, ub, zk, dd);
        }
        if (a.ckpt_every > 0 && (e % a.ckpt_every) == 0) {
            float* cp = a.ckpt + (size_t)(e / a.ckpt_every) * 3 * NP * a.nvtot;
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                cp[(size_t)k * a.nvtot + v] = z[k];
                cp[(size_t)(NP + k) * a.nvtot + v] = m1[k];
                cp[(size_t)(2 * NP + k) * a.nvtot + v] = m2[k];
            }
        }
    }
}

// Scatter the regularised maps of the current z into a TV grid.
// Mask grid of the TV regulariser from the work-list grid indices, with the
// input checks: an index outside its volume's grid sets bit 1 of err, an
// index seen twice sets bit 2; bad_vol receives the lowest offending volume.
// The byte mask is updated through 32-bit atomics on its aligned words.
__global__ void tv_mask_kernel(AdamParams a, unsigned char* mask, int* err, int* bad_vol) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    const int vol = a.blk_vol[blockIdx.x];
    const DevVol& V = a.vols[vol];
    if (v - V.off >= V.nvox) return;
    const int p = a.gidx[v];
    const long long gsz = (long long)V.dims[0] * V.dims[1] * V.dims[2];
    if (p < 0 || p >= gsz) {
        atomicOr(err, 1);
        atomicMin(bad_vol, vol);
        return;
    }
    for (int j = 0; a.surf_nb && j < a.surf_maxnb; ++j) {
        const int nb = a.surf_nb[(size_t)j * a.nvtot + v];
        if (nb < 0 || nb >= gsz) {
            atomicOr(err, 4);
            atomicMin(bad_vol, vol);
            return;
        }
    }
    const size_t q = (size_t)V.grid_off + (size_t)p;
    unsigned int* w = reinterpret_cast<unsigned int*>(mask + (q & ~(size_t)3));
    const unsigned int bit = 1u << (8 * (q & 3));
    if (atomicOr(w, bit) & bit) {
        atomicOr(err, 2);
        atomicMin(bad_vol, vol);
    }
}

__global__ void tv_scatter_kernel(AdamParams a, float* grid) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    if (v - V.off >= V.nvox) return;
    int p = a.gidx[v];
    for (int r = 0; r < a.n_reg; ++r) {
        int k = a.reg_param[r];
        float dd;
        grid[(size_t)r * a.grid_total + V.grid_off + p] =
            unscale(a.transform, a.P.lb[k], a.P.ub[k], a.z[(size_t)k * a.nvtot + v], dd);
    }
}

// theta = unscale(z) (askadam.m:312-326) and per-voxel mean residual (resloss).
__global__ void finalize_kernel(AdamParams a, const float* zsrc, float* theta_out, const float* res,
                                float* resloss) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    if (theta_out)
        for (int k = 0; k < a.np; ++k) {
            float dd;
            size_t i = (size_t)k * a.nvtot + v;
            theta_out[i] = unscale(a.transform, a.P.lb[k], a.P.ub[k], zsrc[i], dd);
        }
    if (res && resloss) {
        float s = 0.0f;
        for (int m = 0; m < a.nm; ++m) s += res[(size_t)m * a.nvtot + v];
        resloss[v] = s / (float)a.nm;
    }
}

// Copy (z, m1, m2) between the live state and a checkpoint slot.
__global__ void copy_state_kernel(AdamParams a, float* slot, const float* z_, const float* m1_,
                                  const float* m2_, int to_ckpt) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    for (int k = 0; k < a.np; ++k) {
        size_t i = (size_t)k * a.nvtot + v;
        size_t j0 = i, j1 = (size_t)(a.np + k) * a.nvtot + v, j2 = (size_t)(2 * a.np + k) * a.nvtot + v;
        if (to_ckpt) {
            slot[j0] = z_[i]; slot[j1] = m1_[i]; slot[j2] = m2_[i];
        } else {
            a.z[i] = slot[j0]; a.m1[i] = slot[j1]; a.m2[i] = slot[j2];
            if (a.zprev) a.zprev[i] = slot[j0];
        }
    }
}

// ---------------------------------------------------------------------------
// Plain path kernels.
// ---------------------------------------------------------------------------
__global__ void plain_unscale_kernel(AdamParams a, PlainBufs b) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    for (int k = 0; k < a.np; ++k) {
        size_t i = (size_t)k * a.nvtot + v;
        float d;
        b.theta[i] = unscale(a.transform, a.P.lb[k], a.P.ub[k], a.z[i], d);
        b.dth[i] = d;
    }
}

template <int MODEL>
__global__ void plain_forward_kernel(AdamParams a, PlainBufs b) {
    constexpr int NP = ModelNP<MODEL>::value;
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    float th[NP];
    for (int k = 0; k < NP; ++k) th[k] = b.theta[(size_t)k * a.nvtot + v];
    float b1 = a.b1 ? a.b1[v] : 1.0f;
    float sa[MODEL == kR1R2S ? kMaxFA : 1], ca[MODEL == kR1R2S ? kMaxFA : 1];
    if (MODEL == kR1R2S)
        for (int f = 0; f < a.P.n_fa; ++f) sincosf(b1 * a.P.fa_rad[f], &sa[f], &ca[f]);
    VoxAux va{b1, sa, ca, 1};
    va.sigma = voxel_sigma(a, v);
    SignalSink<NP> sink{b.signal + v, a.nvtot};
    model_eval<MODEL>(a.P, th, va, sink);
}

template <int LOSS>
__global__ void plain_loss_kernel(AdamParams a, PlainBufs b) {
    __shared__ double s_red[2 * 32];
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    bool valid = v < a.nvtot && (v - V.off) < V.nvox;
    float tot = 0.0f;
    if (v < a.nvtot) {
        LossAux aux = make_loss_aux(voxel_sigma(a, v));
        for (int m = 0; m < a.nm; ++m) {
            size_t i = (size_t)m * a.nvtot + v;
            float S = b.signal[i];
            bool bad = !isfinite(S);
            float s = bad ? 0.0f : S;
            float w = (a.weights ? a.weights[i] : 1.0f) * (b.r.vmod ? b.r.vmod[v] : 1.0f);
            float d;
            float l = loss_elem<LOSS>(s, a.data[i], w, aux, a.mse_scale, a.huber_delta, d);
            b.res[i] = l;
            b.dsig[i] = bad ? 0.0f : d * V.norm;
            tot += l;
        }
        if (b.r.vloss) b.r.vloss[v] = tot / (float)a.nm;  // mean(reshape(residuals, Nmeas, Nvol), 1)
    }
    float q[1] = {valid ? tot : 0.0f};
    block_accumulate<1>(q, b.acc, V.normd, s_red, 0);
}

// ---------------------------------------------------------------------------
// robustConvergence (utils/askadam.m:448-510, 530-581) on the op-by-op path.
// The medians enter only through "median > threshold", which needs no sort:
// with c = #{x <= t} among n values, an odd n gives median > t iff
// c < (n+1)/2; an even n (median = mean of the two middle values) gives true
// for c < n/2, false for c > n/2 and, for c = n/2, compares the mean of
// max{x <= t} and min{x > t} with t.  A NaN anywhere makes the median NaN.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned int ord_bits(float x) {
    unsigned int u = __float_as_uint(x);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord_float(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ bool median_above(int n, int n_le, unsigned int max_le, unsigned int min_gt, int n_nan, float t) {
    if (n_nan > 0 || n == 0) return false;
    if (n & 1) return n_le < (n + 1) / 2;
    int k = n / 2;
    if (n_le < k) return true;
    if (n_le > k) return false;
    return 0.5f * (ord_float(max_le) + ord_float(min_gt)) > t;
}

__global__ void robust_reset_kernel(AdamParams a, PlainBufs b) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    b.r.vmod[v] = 1.0f;
    b.r.flagcnt[v] = 0;
    b.r.mainmask[v] = 1;
    b.r.convmask[v] = 1;
}

// perVoxelLossInit and history = repmat(perVoxelLossInit, window, 1)
__global__ void robust_seed_kernel(AdamParams a, PlainBufs b, int window) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    float l = b.r.vloss[v];
    b.r.vinit[v] = l;
    for (int q = 0; q < window; ++q) b.r.ring[(size_t)q * a.nvtot + v] = l;
}

// History shift (the oldest row `slot` takes the current losses; `oldest` is
// the new oldest row), both improvements, and the statistics of each
// improvement around its population threshold.
__global__ void robust_check_kernel(AdamParams a, PlainBufs b, int slot, int oldest, RobustOpts ro) {
    __shared__ int s_cnt[3];
    __shared__ unsigned int s_ext[4];
    if (threadIdx.x < 3) s_cnt[threadIdx.x] = 0;
    if (threadIdx.x == 0) { s_ext[0] = 0u; s_ext[1] = 0xffffffffu; s_ext[2] = 0u; s_ext[3] = 0xffffffffu; }
    __syncthreads();
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    if (v < a.nvtot && (v - V.off) < V.nvox) {
        float cur = b.r.vloss[v];
        b.r.ring[(size_t)slot * a.nvtot + v] = cur;
        float old = b.r.ring[(size_t)oldest * a.nvtot + v];
        float ia = (old - cur) / (old + 1e-8f);
        float init = b.r.vinit[v];
        float ib = (init - cur) / (init + 1e-8f);
        b.r.imp_a[v] = ia;
        b.r.imp_b[v] = ib;
        if (isnan(ia) || isnan(ib)) atomicAdd(&s_cnt[2], 1);
        if (ia <= ro.pop_thres) { atomicAdd(&s_cnt[0], 1); atomicMax(&s_ext[0], ord_bits(ia)); }
        else if (!isnan(ia)) atomicMin(&s_ext[1], ord_bits(ia));
        if (ib <= ro.init_pop_thres) { atomicAdd(&s_cnt[1], 1); atomicMax(&s_ext[2], ord_bits(ib)); }
        else if (!isnan(ib)) atomicMin(&s_ext[3], ord_bits(ib));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        RobustStat* st = b.r.stat;
        if (s_cnt[0]) atomicAdd(&st->n_le_a, s_cnt[0]);
        if (s_cnt[1]) atomicAdd(&st->n_le_b, s_cnt[1]);
        if (s_cnt[2]) atomicAdd(&st->n_nan, s_cnt[2]);
        atomicMax(&st->max_le_a, s_ext[0]);
        atomicMin(&st->min_gt_a, s_ext[1]);
        atomicMax(&st->max_le_b, s_ext[2]);
        atomicMin(&st->min_gt_b, s_ext[3]);
    }
}

// Outlier flags, main mask and weight modulator (askadam.m:483-508).
__global__ void robust_flag_kernel(AdamParams a, PlainBufs b, RobustOpts ro, int nvox) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    if (v >= a.nvtot || (v - V.off) >= V.nvox) return;
    const RobustStat st = *b.r.stat;
    const bool med_a = median_above(nvox, st.n_le_a, st.max_le_a, st.min_gt_a, st.n_nan, ro.pop_thres);
    const bool med_b = median_above(nvox, st.n_le_b, st.max_le_b, st.min_gt_b, st.n_nan, ro.init_pop_thres);
    const bool fail_a = b.r.imp_a[v] < ro.voxel_thres && med_a;
    const bool fail_b = b.r.imp_b[v] < ro.init_thres && med_b;
    int c = b.r.flagcnt[v];
    c = (fail_a && fail_b) ? c + 1 : (c > 0 ? c - 1 : 0);
    b.r.flagcnt[v] = c;
    b.r.mainmask[v] = c == 0;
    b.r.vmod[v] = c == 0 ? 1.0f : ro.outlier_weight;
}

__global__ void robust_differs_kernel(AdamParams a, PlainBufs b) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    bool d = v < a.nvtot && (v - V.off) < V.nvox && b.r.mainmask[v] != b.r.convmask[v];
    if (__syncthreads_or(d) && threadIdx.x == 0) atomicOr(&b.r.stat->differs, 1);
}

// mainMask_conv = mainMask when it changed (askadam.m:559-562)
__global__ void robust_refresh_kernel(AdamParams a, PlainBufs b) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot || !b.r.stat->differs) return;
    b.r.convmask[v] = b.r.mainmask[v];
    if (v == 0) b.acc[7] = 1.0;
}

// mean(perVoxelLoss(mainMask_conv)) as sum and count into acc[5], acc[6]
__global__ void robust_conv_kernel(AdamParams a, PlainBufs b) {
    __shared__ double s_red[2 * 32 * 2];
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    bool in = v < a.nvtot && (v - V.off) < V.nvox && b.r.convmask[v];
    float q[2] = {in ? b.r.vloss[v] : 0.0f, in ? 1.0f : 0.0f};
    block_accumulate<2>(q, b.acc + 5, 1.0, s_red, 0);
}

template <int NP>
struct DsigAcc {
    const float* ds;
    int s;
    float g[NP];
    __device__ __forceinline__ void add(int m, float S, const float (&dS)[NP]) {
        float d = ds[m * s];
#pragma unroll
        for (int k = 0; k < NP; ++k) g[k] += d * dS[k];
    }
};

template <int MODEL>
__global__ void plain_adjoint_kernel(AdamParams a, PlainBufs b) {
    constexpr int NP = ModelNP<MODEL>::value;
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    float th[NP];
    for (int k = 0; k < NP; ++k) th[k] = b.theta[(size_t)k * a.nvtot + v];
    float b1 = a.b1 ? a.b1[v] : 1.0f;
    float sa[MODEL == kR1R2S ? kMaxFA : 1], ca[MODEL == kR1R2S ? kMaxFA : 1];
    if (MODEL == kR1R2S)
        for (int f = 0; f < a.P.n_fa; ++f) sincosf(b1 * a.P.fa_rad[f], &sa[f], &ca[f]);
    VoxAux va{b1, sa, ca, 1};
    va.sigma = voxel_sigma(a, v);
    DsigAcc<NP> acc;
    acc.ds = b.dsig + v;
    acc.s = a.nvtot;
    for (int k = 0; k < NP; ++k) acc.g[k] = 0.0f;
    model_eval<MODEL>(a.P, th, va, acc);
    for (int k = 0; k < NP; ++k) b.gth[(size_t)k * a.nvtot + v] = acc.g[k];
}

// Scatter theta of the regularised maps into the grid, then TV cost + grad.
__global__ void plain_scatter_kernel(AdamParams a, PlainBufs b, float* grid) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    if (v - V.off >= V.nvox) return;
    for (int r = 0; r < a.n_reg; ++r)
        grid[(size_t)r * a.grid_total + V.grid_off + a.gidx[v]] =
            b.theta[(size_t)a.reg_param[r] * a.nvtot + v];
}

__global__ void plain_tv_kernel(AdamParams a, PlainBufs b, const float* grid) {
    __shared__ double s_red[2 * 32];
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    bool valid = v < a.nvtot && (v - V.off) < V.nvox;
    float reg = 0.0f;
    if (valid && a.surf_nb) {
        const unsigned char* mk = a.maskgrid + V.grid_off;
        const int p = a.gidx[v];
        for (int r = 0; r < a.n_reg; ++r) {
            const float* G = grid + (size_t)r * a.grid_total + V.grid_off;
            float cost, gr;
            surf_tv_terms(G[p], G, mk, a.surf_nb + v, a.surf_len + v, a.surf_maxnb, a.nvtot, cost, gr);
            reg += V.tv_scale[r] * cost;
            float* gk = b.gth + (size_t)a.reg_param[r] * a.nvtot + v;
            *gk = fma1(V.tv_scale[r], gr, *gk);
        }
    } else if (valid) {
        const int dx = V.dims[0], dy = V.dims[1], dz = V.dims[2];
        const int p = a.gidx[v];
        const int x = p % dx, yz = p / dx, y = yz % dy, zc = yz / dy;
        const int nd = a.tv_3d ? 3 : 2;
        const int sy = dx, sz = dx * dy;
        int fw[3] = {x + 1 < dx ? p + 1 : p - x, y + 1 < dy ? p + sy : p - y * sy,
                     zc + 1 < dz ? p + sz : p - zc * sz};
        int bw[3] = {x > 0 ? p - 1 : p + (dx - 1), y > 0 ? p - sy : p + (dy - 1) * sy,
                     zc > 0 ? p - sz : p + (dz - 1) * sz};
        const unsigned char* mk = a.maskgrid + V.grid_off;
        bool mb[3] = {mk[bw[0]] != 0, mk[bw[1]] != 0, mk[bw[2]] != 0};
        for (int r = 0; r < a.n_reg; ++r) {
            const float* G = grid + (size_t)r * a.grid_total + V.grid_off;
            float c = G[p];
            float fv[3], bv[3];
            for (int d = 0; d < nd; ++d) {
                fv[d] = G[fw[d]];
                bv[d] = G[bw[d]];
            }
            float cost, gr;
            tv_terms(c, fv, bv, mb, a.inv_vs, nd, cost, gr);
            reg += V.tv_scale[r] * cost;
            float* gk = b.gth + (size_t)a.reg_param[r] * a.nvtot + v;
            *gk = fma1(V.tv_scale[r], gr, *gk);
        }
    }
    float q[1] = {reg};
    block_accumulate<1>(q, b.acc + 1, 1.0, s_red, 0);
}

// Prior regulariser of the op-by-op path: gth += its gradient, acc[1] += its loss.
__global__ void plain_prior_kernel(AdamParams a, PlainBufs b) {
    __shared__ double s_red[2 * 32];
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    bool valid = v < a.nvtot && (v - V.off) < V.nvox;
    float reg = 0.0f;
    if (valid) {
        for (int r = 0; r < a.n_reg; ++r) {
            const int k = a.reg_param[r];
            const size_t i = (size_t)r * a.nvtot + v;
            float cost, gr;
            prior_terms(b.theta[(size_t)k * a.nvtot + v], a.prior_mu[i], a.prior_sd[i], cost, gr);
            reg = fma1(V.tv_scale[r], cost, reg);
            float* gk = b.gth + (size_t)k * a.nvtot + v;
            *gk = fma1(V.tv_scale[r], gr, *gk);
        }
        if (v == V.off) reg = add1(reg, V.prior_off);
    }
    float q[1] = {reg};
    block_accumulate<1>(q, b.acc + 1, 1.0, s_red, 0);
}

template <bool STATS>
__global__ void plain_zgrad_kernel(AdamParams a, PlainBufs b) {
    __shared__ double s_red[2 * 32 * 3];
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    const DevVol& V = a.vols[a.blk_vol[blockIdx.x]];
    bool valid = v < a.nvtot && (v - V.off) < V.nvox;
    float g2 = 0.f, z2 = 0.f, d2 = 0.f;
    if (v < a.nvtot) {
        for (int k = 0; k < a.np; ++k) {
            size_t i = (size_t)k * a.nvtot + v;
            float g = b.gth[i] * b.dth[i];
            b.gz[i] = g;
            if (STATS) {
                float z = a.z[i];
                g2 += g * g;
                z2 += z * z;
                d2 += (z - a.zprev[i]) * (z - a.zprev[i]);
                a.zprev[i] = z;
            }
        }
    }
    if (STATS) {
        float q[3] = {valid ? g2 : 0.f, valid ? z2 : 0.f, valid ? d2 : 0.f};
        block_accumulate<3>(q, b.acc + 2, 1.0, s_red, 0);
    }
}

__global__ void plain_update_kernel(AdamParams a, PlainBufs b, int e) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nvtot) return;
    float2 sc = a.sched[e];
    for (int k = 0; k < a.np; ++k) {
        size_t i = (size_t)k * a.nvtot + v;
        float z = a.z[i], m1 = a.m1[i], m2 = a.m2[i];
        opt_update(a, sc, z, m1, m2, b.gz[i]);
        a.z[i] = z;
        a.m1[i] = m1;
        a.m2[i] = m2;
    }
}

template <int MODEL>
__global__ void forward_only_kernel(DevProtocol P, const float* theta, const float* b1_, int nvox,
                                    float* signal) {
    constexpr int NP = ModelNP<MODEL>::value;
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    float th[NP];
    for (int k = 0; k < NP; ++k) th[k] = theta[(size_t)k * nvox + v];
    float b1 = b1_ ? b1_[v] : 1.0f;
    float sa[MODEL == kR1R2S ? kMaxFA : 1], ca[MODEL == kR1R2S ? kMaxFA : 1];
    if (MODEL == kR1R2S)
        for (int f = 0; f < P.n_fa; ++f) sincosf(b1 * P.fa_rad[f], &sa[f], &ca[f]);
    VoxAux va{b1, sa, ca, 1};
    va.sigma = b1;  // the aux map: b1 (R1R2*) or sigma (NEXI Rician mean)
    SignalSink<NP> sink{signal + v, nvox};
    model_eval<MODEL>(P, th, va, sink);
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
#define GX_MODEL_SWITCH(model, F, ...)                      \
    switch (model) {                                        \
    case kR2S: F<kR2S, __VA_ARGS__>; break;                 \
    case kR1R2S: F<kR1R2S, __VA_ARGS__>; break;             \
    case kNEXI: F<kNEXI, __VA_ARGS__>; break;               \
    default: F<kNEXI2, __VA_ARGS__>; break;                 \
    }

template <int MODEL, int LOSS, bool STATS>
static cudaError_t fused_dispatch3(const AdamParams& a, int e_begin, int e_end, int update_last,
                                   bool record, int block, int nblocks, cudaStream_t s) {
    constexpr int NQ = STATS ? kHistW : 1;
    size_t smem = sizeof(double) * 2 * 32 * NQ +
                  sizeof(float) * (size_t)block * (a.nm * (a.weights ? 2 : 1) + 2 * a.P.n_fa);
    auto k = fused_kernel_fn<MODEL, LOSS, STATS>();
    if (smem > 48 * 1024) {
        cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
    }
    k<<<nblocks, block, smem, s>>>(a, e_begin, e_end, update_last, record ? 1 : 0);
    ++g_kernel_launches;
    return cudaGetLastError();
}

template <int MODEL, bool STATS>
static cudaError_t fused_dispatch2(const AdamParams& a, int loss, int e_begin, int e_end,
                                   int update_last, bool record, int block, int nblocks,
                                   cudaStream_t s) {
    switch (loss) {
    case kL1: return fused_dispatch3<MODEL, kL1, STATS>(a, e_begin, e_end, update_last, record, block, nblocks, s);
    case kL2: return fused_dispatch3<MODEL, kL2, STATS>(a, e_begin, e_end, update_last, record, block, nblocks, s);
    case kHuber: return fused_dispatch3<MODEL, kHuber, STATS>(a, e_begin, e_end, update_last, record, block, nblocks, s);
    case kMSE: return fused_dispatch3<MODEL, kMSE, STATS>(a, e_begin, e_end, update_last, record, block, nblocks, s);
    case kGauss: return fused_dispatch3<MODEL, kGauss, STATS>(a, e_begin, e_end, update_last, record, block, nblocks, s);
    default: return fused_dispatch3<MODEL, kRician, STATS>(a, e_begin, e_end, update_last, record, block, nblocks, s);
    }
}

// Largest launch block of fused_kernel<MODEL, LOSS, STATS> for this job:
// the kernel's thread limit and the dynamic shared memory it takes per block.
template <int MODEL, int LOSS, bool STATS>
static int fused_limit3(const AdamParams& a) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fused_kernel_fn<MODEL, LOSS, STATS>()) != cudaSuccess) return 0;
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return 0;
    constexpr int NQ = STATS ? kHistW : 1;
    const size_t per = sizeof(float) * (size_t)(a.nm * (a.weights ? 2 : 1) + 2 * a.P.n_fa);
    const size_t fixed = sizeof(double) * 2 * 32 * NQ + fa.sharedSizeBytes;
    int b = fa.maxThreadsPerBlock / 32 * 32;
    while (b > 0 && fixed + per * b > (size_t)optin) b -= 32;
    return b;
}

template <int MODEL, bool STATS>
static int fused_limit2(const AdamParams& a, int loss) {
    switch (loss) {
    case kL1: return fused_limit3<MODEL, kL1, STATS>(a);
    case kL2: return fused_limit3<MODEL, kL2, STATS>(a);
    case kHuber: return fused_limit3<MODEL, kHuber, STATS>(a);
    case kMSE: return fused_limit3<MODEL, kMSE, STATS>(a);
    case kGauss: return fused_limit3<MODEL, kGauss, STATS>(a);
    default: return fused_limit3<MODEL, kRician, STATS>(a);
    }
}

int fused_block_limit(const AdamParams& a, int model, int loss, bool stats) {
#define GX_L(M) return stats ? fused_limit2<M, true>(a, loss) : fused_limit2<M, false>(a, loss)
    switch (model) {
    case kR2S: GX_L(kR2S);
    case kR1R2S: GX_L(kR1R2S);
    case kNEXI: GX_L(kNEXI);
    default: GX_L(kNEXI2);
    }
#undef GX_L
}

cudaError_t launch_fused(const AdamParams& a, int model, int loss, bool stats, int e_begin,
                         int e_end, int update_last, bool record, int block, int nblocks,
                         cudaStream_t s) {
#define GX_F(M)                                                                                    \
    return stats ? fused_dispatch2<M, true>(a, loss, e_begin, e_end, update_last, record, block, nblocks, s) \
                 : fused_dispatch2<M, false>(a, loss, e_begin, e_end, update_last, record, block, nblocks, s)
    switch (model) {
    case kR2S: GX_F(kR2S);
    case kR1R2S: GX_F(kR1R2S);
    case kNEXI: GX_F(kNEXI);
    default: GX_F(kNEXI2);
    }
#undef GX_F
}

template <int MODEL, int LOSS, bool STATS>
static cudaError_t tv_dispatch3(const AdamParams& a, int e, bool update, bool record,
                                bool want_res, int block, int nblocks, cudaStream_t s) {
    tv_step_kernel<MODEL, LOSS, STATS><<<nblocks, block, 0, s>>>(a, e, update ? 1 : 0,
                                                                  record ? 1 : 0, want_res ? 1 : 0);
    ++g_kernel_launches;
    return cudaGetLastError();
}

template <int MODEL, bool STATS>
static cudaError_t tv_dispatch2(const AdamParams& a, int loss, int e, bool update, bool record,
                                bool want_res, int block, int nblocks, cudaStream_t s) {
    switch (loss) {
    case kL1: return tv_dispatch3<MODEL, kL1, STATS>(a, e, update, record, want_res, block, nblocks, s);
    case kL2: return tv_dispatch3<MODEL, kL2, STATS>(a, e, update, record, want_res, block, nblocks, s);
    case kHuber: return tv_dispatch3<MODEL, kHuber, STATS>(a, e, update, record, want_res, block, nblocks, s);
    case kMSE: return tv_dispatch3<MODEL, kMSE, STATS>(a, e, update, record, want_res, block, nblocks, s);
    case kGauss: return tv_dispatch3<MODEL, kGauss, STATS>(a, e, update, record, want_res, block, nblocks, s);
    default: return tv_dispatch3<MODEL, kRician, STATS>(a, e, update, record, want_res, block, nblocks, s);
    }
}

cudaError_t launch_tv_step(const AdamParams& a, int model, int loss, bool stats, int e,
                           bool update, bool record, bool want_res, int block, int nblocks,
                           cudaStream_t s) {
#define GX_T(M)                                                                                  \
    return stats ? tv_dispatch2<M, true>(a, loss, e, update, record, want_res, block, nblocks, s) \
                 : tv_dispatch2<M, false>(a, loss, e, update, record, want_res, block, nblocks, s)
    switch (model) {
    case kR2S: GX_T(kR2S);
    case kR1R2S: GX_T(kR1R2S);
    case kNEXI: GX_T(kNEXI);
    default: GX_T(kNEXI2);
    }
#undef GX_T
}

cudaError_t launch_init_state(const AdamParams& a, const float* theta0, double randomness,
                              uint64_t seed, int block, cudaStream_t s) {
    int nb = (a.nvtot + block - 1) / block;
    init_state_kernel<<<nb, block, 0, s>>>(a, theta0, (float)randomness, seed);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_tv_mask(const AdamParams& a, unsigned char* mask, int* err, int* bad_vol, int block,
                           int nblocks, cudaStream_t s) {
    tv_mask_kernel<<<nblocks, block, 0, s>>>(a, mask, err, bad_vol);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_tv_scatter(const AdamParams& a, float* grid, int block, int nblocks,
                              cudaStream_t s) {
    tv_scatter_kernel<<<nblocks, block, 0, s>>>(a, grid);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_finalize(const AdamParams& a, const float* zsrc, float* theta_out,
                            const float* res, float* resloss, int block, int nblocks,
                            cudaStream_t s) {
    finalize_kernel<<<nblocks, block, 0, s>>>(a, zsrc, theta_out, res, resloss);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_copy_state(const AdamParams& a, float* dst, const float* z_, const float* m1_,
                              const float* m2_, bool to_ckpt, int block, int nblocks,
                              cudaStream_t s) {
    copy_state_kernel<<<nblocks, block, 0, s>>>(a, dst, z_, m1_, m2_, to_ckpt ? 1 : 0);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_plain_unscale(const AdamParams& a, const PlainBufs& b, int block, int nblocks,
                                 cudaStream_t s) {
    plain_unscale_kernel<<<nblocks, block, 0, s>>>(a, b);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_plain_forward(const AdamParams& a, int model, const PlainBufs& b, int block,
                                 int nblocks, cudaStream_t s) {
    switch (model) {
    case kR2S: plain_forward_kernel<kR2S><<<nblocks, block, 0, s>>>(a, b); break;
    case kR1R2S: plain_forward_kernel<kR1R2S><<<nblocks, block, 0, s>>>(a, b); break;
    case kNEXI: plain_forward_kernel<kNEXI><<<nblocks, block, 0, s>>>(a, b); break;
    default: plain_forward_kernel<kNEXI2><<<nblocks, block, 0, s>>>(a, b); break;
    }
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_plain_loss(const AdamParams& a, int loss, const PlainBufs& b, int block,
                              int nblocks, cudaStream_t s) {
    switch (loss) {
    case kL1: plain_loss_kernel<kL1><<<nblocks, block, 0, s>>>(a, b); break;
    case kL2: plain_loss_kernel<kL2><<<nblocks, block, 0, s>>>(a, b); break;
    case kHuber: plain_loss_kernel<kHuber><<<nblocks, block, 0, s>>>(a, b); break;
    case kMSE: plain_loss_kernel<kMSE><<<nblocks, block, 0, s>>>(a, b); break;
    case kGauss: plain_loss_kernel<kGauss><<<nblocks, block, 0, s>>>(a, b); break;
    default: plain_loss_kernel<kRician><<<nblocks, block, 0, s>>>(a, b); break;
    }
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_plain_adjoint(const AdamParams& a, int model, const PlainBufs& b, int block,
                                 int nblocks, cudaStream_t s) {
    switch (model) {
    case kR2S: plain_adjoint_kernel<kR2S><<<nblocks, block, 0, s>>>(a, b); break;
    case kR1R2S: plain_adjoint_kernel<kR1R2S><<<nblocks, block, 0, s>>>(a, b); break;
    case kNEXI: plain_adjoint_kernel<kNEXI><<<nblocks, block, 0, s>>>(a, b); break;
    default: plain_adjoint_kernel<kNEXI2><<<nblocks, block, 0, s>>>(a, b); break;
    }
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_plain_tv(const AdamParams& a, const PlainBufs& b, float* grid, int block,
                            int nblocks, cudaStream_t s) {
    plain_scatter_kernel<<<nblocks, block, 0, s>>>(a, b, grid);
    plain_tv_kernel<<<nblocks, block, 0, s>>>(a, b, grid);
    g_kernel_launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_plain_prior(const AdamParams& a, const PlainBufs& b, int block, int nblocks, cudaStream_t s) {
    plain_prior_kernel<<<nblocks, block, 0, s>>>(a, b);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_plain_zgrad(const AdamParams& a, const PlainBufs& b, bool stats, int block,
                               int nblocks, cudaStream_t s) {
    if (stats) plain_zgrad_kernel<true><<<nblocks, block, 0, s>>>(a, b);
    else plain_zgrad_kernel<false><<<nblocks, block, 0, s>>>(a, b);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_plain_update(const AdamParams& a, const PlainBufs& b, int e, int block,
                                int nblocks, cudaStream_t s) {
    plain_update_kernel<<<nblocks, block, 0, s>>>(a, b, e);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_forward_only(const DevProtocol& P, int model, const float* theta,
                                const float* b1, int nvox, float* signal, cudaStream_t s) {
    const int block = 128;
    int nb = (nvox + block - 1) / block;
    if (nb == 0) return cudaSuccess;
    switch (model) {
    case kR2S: forward_only_kernel<kR2S><<<nb, block, 0, s>>>(P, theta, b1, nvox, signal); break;
    case kR1R2S: forward_only_kernel<kR1R2S><<<nb, block, 0, s>>>(P, theta, b1, nvox, signal); break;
    case kNEXI: forward_only_kernel<kNEXI><<<nb, block, 0, s>>>(P, theta, b1, nvox, signal); break;
    default: forward_only_kernel<kNEXI2><<<nb, block, 0, s>>>(P, theta, b1, nvox, signal); break;
    }
    ++g_kernel_launches;
    return cudaGetLastError();
}


cudaError_t launch_robust_reset(const AdamParams& a, const PlainBufs& b, int block, int nblocks, cudaStream_t s) {
    robust_reset_kernel<<<nblocks, block, 0, s>>>(a, b);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_robust_seed(const AdamParams& a, const PlainBufs& b, int window, int block, int nblocks,
                               cudaStream_t s) {
    robust_seed_kernel<<<nblocks, block, 0, s>>>(a, b, window);
    ++g_kernel_launches;
    return cudaGetLastError();
}

cudaError_t launch_robust_check(const AdamParams& a, const PlainBufs& b, int slot, int oldest,
                                const RobustOpts& ro, int nvox, int block, int nblocks, cudaStream_t s) {
    RobustStat init{0, 0, 0, 0u, 0xffffffffu, 0u, 0xffffffffu, 0};
    cudaError_t e = cudaMemcpyAsync(b.r.stat, &init, sizeof(init), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    robust_check_kernel<<<nblocks, block, 0, s>>>(a, b, slot, oldest, ro);
    robust_flag_kernel<<<nblocks, block, 0, s>>>(a, b, ro, nvox);
    g_kernel_launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_robust_window(const AdamParams& a, const PlainBufs& b, int block, int nblocks, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(&b.r.stat->differs, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    robust_differs_kernel<<<nblocks, block, 0, s>>>(a, b);
    robust_refresh_kernel<<<nblocks, block, 0, s>>>(a, b);
    g_kernel_launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_robust_conv(const AdamParams& a, const PlainBufs& b, int block, int nblocks, cudaStream_t s) {
    robust_conv_kernel<<<nblocks, block, 0, s>>>(a, b);
    ++g_kernel_launches;
    return cudaGetLastError();
}

}  // namespace gx
