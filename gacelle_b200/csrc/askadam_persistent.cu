// askadam_persistent.cu -- askAdam with spatial TV as one persistent,
// cooperative launch over a range of epochs (R2* model).
//
// Each CTA owns a contiguous slice of the voxel work-list for the whole
// launch: the slice's Adam state lives in shared memory (and its measurements
// too when they fit; otherwise they are read from L2, all of a voxel's echoes
// in flight together), and only the regularised parameter map travels between
// CTAs (the double-buffered full-grid TV map with a one-cell halo that holds
// the periodic neighbours, read through L2 with ld.global.cg since other CTAs
// wrote it in the same launch).  Each launch writes its start map from the
// staged state and passes one grid barrier before the first epoch, so it
// depends on no map left by another kernel.
//
// An epoch runs in two passes over the slice.  The fidelity pass (forward
// model, loss, adjoint) needs only the CTA's own voxels; the TV/update pass
// (TV subgradient from the neighbours' map values of the previous epoch,
// sigmoid chain rule, optimiser, new map value) needs every CTA's previous
// map.  The voxels are processed by worker warps that never wait for one
// another: a worker warp arrives on a shared-memory mbarrier (with its
// partial loss-history sums) after its map writes, runs its next fidelity
// pass, and waits only before its next TV/update pass.  The CTA's last warp
// is a barrier warp: it collects the worker arrivals, adds the epoch's loss
// history, runs the grid barrier and opens the next TV/update pass (a second
// mbarrier).  Every wait is bounded: if one expires the kernel raises an
// error flag that the host reports as GX_ETIMEOUT, and every CTA returns.
//
// The per-voxel arithmetic (forward model, loss, adjoint, TV subgradient,
// sigmoid chain rule, optimiser) rounds as tv_step_kernel does, so the two
// paths produce the same parameters (the two-voxel variant's TV signs come
// from saturated products, tv_terms2m, equal to tv_terms' bit for bit).  Reference: utils/askadam.m:23-117,
// 673-691; utils/spatial_total_variation.m:24-66.
#include <algorithm>

#include "gx_internal.h"

namespace gx {

namespace {

template <int V> struct IntC { static constexpr int value = V; };

__device__ __forceinline__ float warp_sum_p(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Loss with the kind chosen at run time (uniform across the launch).
struct RtLoss {
    int kind;
    __device__ __forceinline__ float operator()(float s, float y, float w, const LossAux& a, float ms, float hd,
                                                float& d) const {
        switch (kind) {
        case kL1: return loss_elem<kL1>(s, y, w, a, ms, hd, d);
        case kL2: return loss_elem<kL2>(s, y, w, a, ms, hd, d);
        case kHuber: return loss_elem<kHuber>(s, y, w, a, ms, hd, d);
        case kMSE: return loss_elem<kMSE>(s, y, w, a, ms, hd, d);
        case kGauss: return loss_elem<kGauss>(s, y, w, a, ms, hd, d);
        default: return loss_elem<kRician>(s, y, w, a, ms, hd, d);
        }
    }
};

// LossAcc equivalent whose loss kind is either fixed (LOSS >= 0) or run-time.
template <int LOSS, int NP>
struct PLossAcc {
    float total;
    float g[NP];
    const float* y;
    int ys;
    const float* w;
    int ws;
    LossAux aux;
    float mse_scale, hd;
    float* res;
    int rs;
    RtLoss rt;
    __device__ __forceinline__ void add(int m, float S, const float (&dS)[NP]) {
        bool bad = MayBeNonFinite<NP>::value ? !isfinite(S) : false;
        float s = bad ? 0.0f : S;
        if (LOSS == kMSE || (LOSS < 0 && rt.kind == kMSE)) {
            mse_add(s - y[m * ys], dS, bad, total, g, res, m * rs, mse_scale);
            return;
        }
        float ww = w ? w[m * ws] : 1.0f;
        float d;
        float l;
        if constexpr (LOSS >= 0) l = loss_elem<LOSS>(s, y[m * ys], ww, aux, mse_scale, hd, d);
        else l = rt(s, y[m * ys], ww, aux, mse_scale, hd, d);
        total += l;
        if (res) res[m * rs] = l;
        if (!bad) {
#pragma unroll
            for (int k = 0; k < NP; ++k) g[k] += d * dS[k];
        }
    }
    __device__ __forceinline__ void finish() {
        if (LOSS == kMSE || (LOSS < 0 && rt.kind == kMSE)) mse_finish(total, g, mse_scale);
    }
};

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier of a cooperative launch, run by one thread per CTA (the last
// lane of the CTA's barrier warp) on a counter that only grows (zeroed before
// the launch): after the CTA's writes are acquired at CTA scope, one
// release-add publishes them to the other CTAs, and the barrier of the k-th
// epoch boundary is open once the counter reaches (k+1) x #CTAs, so the last
// CTA's add itself opens it.  The wait is bounded; false once any CTA's wait
// has expired.
__device__ __forceinline__ void grid_arrive_one(PersistBarrier* gb) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&gb->count) : "memory");
}

__device__ __forceinline__ bool grid_wait_one(PersistBarrier* gb, unsigned int target, long long limit) {
    const long long t0 = clock64();
    while (ld_acquire_gpu(&gb->count) < target) {
        if (*(volatile int*)&gb->error) return false;
        if (clock64() - t0 > limit) {
            atomicExch(&gb->error, 1);
            return false;
        }
        __nanosleep(20);
    }
    return *(volatile int*)&gb->error == 0;
}

// Shared-memory mbarriers between the worker warps and the barrier warp:
// arrive has release and try_wait acquire semantics at CTA scope, and a
// thread waiting in try_wait is suspended, taking no issue slots from the
// warps that still work.
__device__ __forceinline__ unsigned int smem_u32(const void* p) {
    return (unsigned int)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned int count) {
    asm volatile("mbarrier.init.shared.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned int parity) {
    unsigned int done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Wait for the completion of the barrier's phase with the given parity
// (the barrier is never more than one phase ahead of the waiter).  Bounded
// by `limit` SM clock cycles: false, with the grid's error flag raised, once
// the wait has expired.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned int parity, PersistBarrier* gb,
                                          long long limit) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > limit) {
            atomicExch(&gb->error, 1);
            return false;
        }
    }
    return true;
}

// The persistent kernel's TV map of one volume, with a one-cell halo on
// every face: grid point (x, y, z) sits at P = (x+1) + (y+1) sy + (z+1) sz,
// and the halo cell beyond a face holds the value of the periodic neighbour
// (the voxel on the opposite face), so the six face neighbours of every grid
// point are at P +- 1, P +- sy, P +- sz (utils/spatial_total_variation.m:
// 55-66 wraps around with circshift).  A voxel on a face writes its new value
// also into the halo cell that mirrors it: on the last x plane at P - mx, on
// the first at P + mx (likewise y, z).  Layout L > 0: the strides are 2^L
// and 2^2L (dx + 2, dy + 2 <= 2^L), so the neighbour offsets are immediate
// operands of the loads (L = 7, 8, 9); L = 0: sy = dx + 2, sz = (dx + 2)(dy + 2).
struct HaloMap {
    int sy, sz;      // strides
    int mx, my, mz;  // mirror offsets dx, dy sy, dz sz
    bool tv3;
    template <int L>
    __device__ __forceinline__ void load(const float* G, int P, float (&f)[3], float (&b)[3]) const {
        const int ty = L > 0 ? 1 << L : sy, tz = L > 0 ? 1 << (2 * L) : sz;
        const float* g = G + P;
        f[0] = __ldcg(g + 1); b[0] = __ldcg(g - 1);
        f[1] = __ldcg(g + ty); b[1] = __ldcg(g - ty);
        if (tv3) { f[2] = __ldcg(g + tz); b[2] = __ldcg(g - tz); }
        else { f[2] = 0.0f; b[2] = 0.0f; }
    }
    // fl: the voxel's face flags (bits 0-2 last x/y/z plane, 3-5 first)
    __device__ __forceinline__ void mirror(float* G, int P, unsigned int fl, float v) const {
        if (fl & 1) G[P - mx] = v;
        if (fl & 8) G[P + mx] = v;
        if (fl & 2) G[P - my] = v;
        if (fl & 16) G[P + my] = v;
        if (tv3) {
            if (fl & 4) G[P - mz] = v;
            if (fl & 32) G[P + mz] = v;
        }
    }
};

}  // namespace

// MAXM > 0: the standard configuration (MSE, sigmoid transform, Adam, one
// regularised map) with the measurements prefetched into registers
// (nm <= MAXM), those options folded in at compile time and the residuals of
// the final evaluation written by a pass after the epoch loop; MAXM == 0: any
// loss, transform, optimiser and regulariser count, measurements read one at
// a time.
// Threads per CTA at most: the 32-echo variant and the pair variants (two
// voxels' measurements per thread) need more than 64 registers.
__host__ __device__ constexpr bool persist_pairs(int maxm, bool stats) { return maxm > 0 && maxm <= 16 && !stats; }
__host__ __device__ constexpr int persist_max_threads(int maxm, bool stats) {
    return (maxm > 16 || persist_pairs(maxm, stats)) ? 768 : kPersistMaxThreads;
}

// HOOK: the bound of the waits and the grid barrier's arrival count come from
// the launch arguments (the context's test hooks); otherwise they are the
// compile-time default, which keeps the wait loops of the timed kernel lean.
template <int LOSS, bool STATS, int MAXM, bool HOOK>
__global__ void __launch_bounds__(persist_max_threads(MAXM, STATS), 1)
tv_persistent_kernel(AdamParams a, PersistArgs p) {
    const long long wait_limit = HOOK ? p.spin_cycles : kBarrierSpinCycles;
    const unsigned int extra_arrivals = HOOK ? p.extra_arrivals : 0u;
    constexpr int NP = 2;  // R2*: M0, R2star
    constexpr int NS = STATS ? 4 : 3;  // z, m1, m2 [, z of the previous epoch]
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* s_red = reinterpret_cast<double*>(smem_raw);                     // [2][32][kHistW]
    float* s_st = reinterpret_cast<float*>(s_red + 2 * 32 * kHistW);         // [NS][NP][slice]
    // CACHE: the standard configuration without statistics keeps, from the
    // fidelity pass, the unregularised parameter's z-gradient and the
    // regularised one's fidelity gradient (in the space the previous-epoch z
    // takes when statistics are on), and from the update pass the regularised
    // parameter's theta and dtheta/dz, so that no pass evaluates a transform
    // another pass has evaluated; same operations, same order.
    // PAIR (up to 16 measurements, without statistics): two voxels per
    // thread, pair instructions, with the fidelity-pass cache (CACHE)
    constexpr bool PAIR = persist_pairs(MAXM, STATS);
    constexpr bool CACHE = PAIR;
    constexpr int NAUX = CACHE ? 4 : NP;
    float* s_gf = s_st + (size_t)NS * NP * p.slice;                          // [NAUX][slice] fidelity pass results
    int* s_p = reinterpret_cast<int*>(s_gf + (size_t)NAUX * p.slice);        // [slice] position in the haloed map
    unsigned int* s_w = reinterpret_cast<unsigned int*>(s_p + p.slice);      // [slice] mask words (mask_scale)
    float* s_y = reinterpret_cast<float*>(s_w + p.slice);                     // [nm][slice] if staged
    const int BT = blockDim.x, tid = threadIdx.x;
    const int base = blockIdx.x * p.slice;
    const int n = min(base + p.slice, a.nvtot) - base;  // voxels of this slice
    const int S = p.slice;
    // shared-memory position of slice voxel i: the pair variant stores the
    // voxel pair (64c + l, 64c + l + 32) of pair q = 32c + l at positions 2q,
    // 2q + 1, so that a pair is one 8-byte access
    auto sidx = [](int i) { return PAIR ? (i & ~63) | ((i & 31) << 1) | ((i >> 5) & 1) : i; };
    const DevVol& Vg = a.vols[a.blk_vol[base / p.pad_block]];  // a slice lies in one volume
    struct {
        int off, nvox;
        float norm;
        double normd;
        long long grid_off, hgrid_off;
    } V{Vg.off, Vg.nvox, Vg.norm, Vg.normd, Vg.grid_off, Vg.hgrid_off};
    const int nreal = V.off + V.nvox - base;  // slice voxels i < nreal are real (the padding follows)
    const float tvs0 = Vg.tv_scale[0], tvs1 = Vg.tv_scale[1];
    const int dx = Vg.dims[0], dy = Vg.dims[1], dz = Vg.dims[2];
    const int sy = dx, sz = dx * dy;
    const int wx = dx - 1, wy = (dy - 1) * dx, wz = (dz - 1) * dx * dy;  // wrap offsets
    const int hy = p.hlayout > 0 ? 1 << p.hlayout : dx + 2;
    const int hz = p.hlayout > 0 ? 1 << (2 * p.hlayout) : (dx + 2) * (dy + 2);
    const HaloMap hm{hy, hz, dx, dy * hy, dz * hz, a.tv_3d != 0};
    const unsigned char* mk = a.maskgrid + V.grid_off;
    // the map of the launch's first epoch: written below from the staged state
    float* const gstart = ((p.e_begin >= 1 && ((p.e_begin - 1) & 1)) ? p.grid1 : p.grid0) + V.hgrid_off;
    // stage the slice's state, TV neighbourhood (and measurements, if they fit)
    // once, and write the slice's values of the start map; a padding voxel
    // takes the map position of the volume's first voxel (so that its
    // neighbour loads stay inside the map), no mask and no map write
    for (int i = tid; i < n; i += BT) {
        const int v = base + i;
        int pp = 0;
        unsigned int w = 0;
        const bool real = (v - V.off) < V.nvox;
        if (a.n_reg > 0) {
            const int gp = a.gidx[real ? v : V.off];
            const int x = gp % dx, yz = gp / dx, y = yz % dy, zc = yz / dy;
            const unsigned int wrap = (x == dx - 1) | ((y == dy - 1) << 1) | ((zc == dz - 1) << 2) |
                                      ((x == 0) << 3) | ((y == 0) << 4) | ((zc == 0) << 5);
            const int bw0 = x > 0 ? gp - 1 : gp + wx;
            const int bw1 = y > 0 ? gp - sy : gp + wy;
            const int bw2 = zc > 0 ? gp - sz : gp + wz;
            w = wrap << 24;
            if (real)
                w |= (mk[bw0] ? kMaskByte : 0u) | (mk[bw1] ? kMaskByte << 8 : 0u) | (mk[bw2] ? kMaskByte << 16 : 0u);
            pp = (x + 1) + (y + 1) * hy + (zc + 1) * hz;
            if (real)
                for (int r = 0; r < min(a.n_reg, 2); ++r) {
                    const int k = a.reg_param[r];
                    float dd;
                    const float th = unscale(a.transform, a.P.lb[k], a.P.ub[k], a.z[(size_t)k * a.nvtot + v], dd);
                    float* G = gstart + (size_t)r * p.hgrid_total;
                    G[pp] = th;
                    hm.mirror(G, pp, wrap, th);
                }
        }
        const int j = sidx(i);
        s_p[j] = pp;
        s_w[j] = w;
        if constexpr (CACHE) {  // theta and dtheta/dz of the regularised parameter (see pass 2)
            const int k = a.reg_param[0];
            float dd;
            const float th = unscale(0, a.P.lb[k], a.P.ub[k], a.z[(size_t)k * a.nvtot + v], dd);
            s_gf[2 * S + j] = dd;
            s_gf[3 * S + j] = th;
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            size_t gi = (size_t)k * a.nvtot + base + i;
            s_st[(0 * NP + k) * S + j] = a.z[gi];
            s_st[(1 * NP + k) * S + j] = a.m1[gi];
            s_st[(2 * NP + k) * S + j] = a.m2[gi];
            if constexpr (STATS) s_st[(3 * NP + k) * S + j] = a.zprev ? a.zprev[gi] : 0.0f;
        }
        if (p.data_in_smem)
            for (int m = 0; m < a.nm; ++m) s_y[m * S + j] = a.data[(size_t)m * a.nvtot + base + i];
    }
    __shared__ DevProtocol s_P;
    stage_protocol(a.P, &s_P);
    // bar_arrive: one arrival per worker warp and epoch; bar_open: one per
    // epoch boundary (the grid barrier has passed, or s_err is set)
    __shared__ unsigned long long bar_arrive, bar_open;
    __shared__ int s_err;
    const int NWT = BT - 32;  // worker threads; the last warp is the barrier warp
    if (tid == 0) {
        mbar_init(&bar_arrive, (unsigned int)(NWT >> 5));
        mbar_init(&bar_open, 1u);
        s_err = 0;
    }
    __syncthreads();
    // every CTA's part of the start map before the first TV pass (the grid
    // barrier's first round; the epoch boundaries follow from the second)
    if (tid == BT - 1) {
        grid_arrive_one(p.barrier);
        if (!grid_wait_one(p.barrier, gridDim.x + extra_arrivals, wait_limit)) s_err = 1;
    }
    __syncthreads();
    if (s_err) return;
    constexpr bool STD = MAXM > 0;
    const bool tv3 = a.tv_3d != 0;
    const int nm = a.nm;
    const int transform = STD ? 0 : a.transform;
    const int nreg = STD ? 1 : min(a.n_reg, 2);  // R2*: at most two maps
    const OptConst oc{STD ? kAdam : a.optimiser, a.beta1, a.beta2, a.eps, a.momentum, a.rms_decay, a.rms_eps};
    const float ivx = a.inv_vs[0], ivy = a.inv_vs[1], ivz = a.inv_vs[2];

    if (tid >= NWT) {
        // barrier warp: history of each epoch, grid barrier between epochs
        const int lane = tid & 31, nw = NWT >> 5;
        constexpr int NQ = STATS ? kHistW : 2;  // without statistics columns 2-4 stay zero
        const int vol = a.blk_vol[base / p.pad_block];
        for (int e = p.e_begin; e <= p.e_end; ++e) {
            const unsigned int ph = (unsigned int)(e - p.e_begin) & 1u;
            if (!mbar_wait(&bar_arrive, ph, p.barrier, wait_limit)) {
                if (lane == 31) {
                    *(volatile int*)&s_err = 1;
                    mbar_arrive(&bar_open);
                }
                return;
            }
            // lane 31 publishes the CTA's maps and waits for the other CTAs
            // while lanes 0-4 add the epoch's loss history
            int ok = 1;
            if (e < p.e_end && lane == 31) {
                grid_arrive_one(p.barrier);
                ok = grid_wait_one(p.barrier, (unsigned int)(e - p.e_begin + 2) * gridDim.x + extra_arrivals,
                                   wait_limit);
                if (!ok) *(volatile int*)&s_err = 1;
            }
            if (p.record && a.hist && lane < NQ) {
                const double* buf = s_red + (e & 1) * 32 * kHistW;
                double t = 0.0;
                for (int w = 0; w < nw; ++w) t += buf[w * kHistW + lane];
                if (lane == 0) t *= V.normd;
                if (t != 0.0) atomicAdd(a.hist + ((size_t)vol * (a.niter + 1) + e) * kHistW + lane, t);
            }
            __syncwarp();  // the history buffer of epoch e is read before epoch e+1 opens
            if (e < p.e_end) {
                if (lane == 31) mbar_arrive(&bar_open);
                ok = __shfl_sync(0xffffffffu, ok, 31);
                if (!ok) return;
            }
        }
    } else
    for (int e = p.e_begin; e <= p.e_end; ++e) {
        const float* gcur = (e >= 1 && ((e - 1) & 1)) ? p.grid1 : p.grid0;  // epoch 0 reads the start map
        float* gnext = e & 1 ? p.grid1 : p.grid0;
        float q0 = 0.f, q1 = 0.f, q2 = 0.f, q3 = 0.f, q4 = 0.f;
        const bool upd = e <= p.update_last;
        const float2 sc = upd ? a.sched[e] : float2{0.f, 0.f};
        if constexpr (PAIR) {
        // two voxels per thread and pass: pair q takes voxels i0 = 64 (q / 32)
        // + q % 32 and i1 = i0 + 32 of the slice (a warp covers 64
        // consecutive voxels, and each of its per-voxel accesses 32
        // consecutive ones); the parameter, gradient and optimiser arithmetic
        // in pair instructions, lane .x on voxel i0 and .y on voxel i1; the
        // regularised parameter kr is a compile-time constant of the epoch's
        // code (false: a wait has failed, the kernel returns)
        auto pair_epoch = [&](auto KR, auto HLC) -> bool {
        constexpr int kr = decltype(KR)::value, HL = decltype(HLC)::value;
        const int npair = n >> 1;  // n is a multiple of 64 in pair mode
        // shared memory: pair q at float2 position q; global: voxels v0, v0+32
        auto ld2 = [](const float* b, int q) { return reinterpret_cast<const float2*>(b)[q]; };
        auto st2 = [](float* b, int q, float2 x) { reinterpret_cast<float2*>(b)[q] = x; };
        auto st2g = [](float* b, int v0, float2 x) {
            b[v0] = x.x;
            b[v0 + 32] = x.y;
        };
        // pass 1: data fidelity of the slice (own voxels only)
        for (int q = tid; q < npair; q += NWT) {
            const int i0 = ((q >> 5) << 6) + (q & 31), v0 = base + i0;
            const bool ok0 = i0 < nreal, ok1 = i0 + 32 < nreal;
            float2 y[MAXM];  // measurement m of both voxels
            if (p.data_quads) {
                // chunk-interleaved pair quads: quad j of pair u at
                // ((u / 32) (MAXM / 2) + j) 32 + u % 32 (constant offsets)
                const float4* pq = p.data_quads + (size_t)((base >> 6) + (q >> 5)) * (MAXM / 2) * 32 + (q & 31);
#pragma unroll
                for (int j = 0; j < MAXM / 2; ++j) {
                    const float4 t = __ldcg(pq + j * 32);
                    y[2 * j] = make_float2(t.x, t.y);
                    y[2 * j + 1] = make_float2(t.z, t.w);
                }
            } else {
#pragma unroll
                for (int m = 0; m < MAXM; ++m)
                    y[m] = m >= nm ? make_float2(0.f, 0.f)
                           : p.data_in_smem ? ld2(s_y + (size_t)m * S, q)
                                            : make_float2(a.data[(size_t)m * a.nvtot + v0],
                                                          a.data[(size_t)m * a.nvtot + v0 + 32]);
            }
            float2 th[NP], dth[NP];
#pragma unroll
            for (int k = 0; k < NP; ++k)
                if (k == kr) {  // written by the previous update (or the staging)
                    th[k] = ld2(s_gf + 3 * S, q);
                    dth[k] = ld2(s_gf + 2 * S, q);
                } else {
                    th[k] = unscale_sig2c(p.k, k, ld2(s_st + k * S, q), dth[k]);
                }
            // R2sMseSums on both lanes with the residual negated, y - M0 E:
            // every partial sum is the exact negative of the scalar one
            float2 sse = make_float2(0.f, 0.f), g0n = sse, g1n = sse;
            const float2 nM0 = make_float2(-th[0].x, -th[0].y), R2 = th[1];
            auto echo = [&](int m) {
                const float2 x = mul2(a.P.nl2e_pair[m], R2);
                const float2 E = make_float2(ex2_ftz(x.x), ex2_ftz(x.y));
                const float2 rn = fma2(nM0, E, y[m]);
                sse = fma2(rn, rn, sse);
                const float2 qn = mul2(rn, E);
                g0n = add2(g0n, qn);
                g1n = fma2(a.P.te_pair[m], qn, g1n);
            };
            if (nm == MAXM) {  // the full protocol: no per-echo test
#pragma unroll
                for (int m = 0; m < MAXM; ++m) echo(m);
            } else {
#pragma unroll
                for (int m = 0; m < MAXM; ++m)
                    if (m < nm) echo(m);
            }
            const float2 zero = make_float2(0.f, 0.f);
            const float2 tot = mul2(add2(zero, sse), p.k.mse);
            float2 g[NP];
            g[0] = mul2(sub2(zero, g0n), p.k.s2);
            g[1] = mul2(fma2(th[0], g1n, zero), p.k.s2);
            const float2 nrm = bcast2(V.norm);
            const float2 gr = mul2(kr == 0 ? g[0] : g[1], nrm), gn = mul2(kr == 0 ? g[1] : g[0], nrm);
            st2(s_gf + 0 * S, q, mul2(gn, kr == 0 ? dth[1] : dth[0]));
            st2(s_gf + 1 * S, q, gr);
            if (ok0) q0 += tot.x;
            if (ok1) q0 += tot.y;
        }
        // every CTA's map of the previous epoch (written before its arrival)
        if (e > p.e_begin)
            if (!mbar_wait(&bar_open, (unsigned int)(e - 1 - p.e_begin) & 1u, p.barrier, wait_limit) ||
                *(volatile int*)&s_err)
                return false;
        const bool ckpt = upd && a.ckpt_every > 0 && (e % a.ckpt_every) == 0;
        float* cp = ckpt ? a.ckpt + (size_t)(e / a.ckpt_every) * 3 * NP * a.nvtot : nullptr;
        const float* G = gcur + V.hgrid_off;
        float* Gn = gnext + V.hgrid_off;
        const float2 nscx = bcast2(-sc.x), scy = bcast2(sc.y);
        // pass 2: TV subgradient, chain rule, optimiser, new map values
        for (int q = tid; q < npair; q += NWT) {
            const int i0 = ((q >> 5) << 6) + (q & 31), v0 = base + i0;
            const bool ok0 = i0 < nreal, ok1 = i0 + 32 < nreal;
            const float2 gn = ld2(s_gf + 0 * S, q);
            float2 grf = ld2(s_gf + 1 * S, q);
            const float2 dthr = ld2(s_gf + 2 * S, q);
            const float2 c = ld2(s_gf + 3 * S, q);
            const int2 pp = reinterpret_cast<const int2*>(s_p)[q];
            const int p0 = pp.x, p1 = pp.y;
            const uint2 w01 = reinterpret_cast<const uint2*>(s_w)[q];
            // every voxel loads (a padding voxel at a valid position), only
            // real voxels add their terms
            float f0[3], b0[3], f1[3], b1[3];
            hm.load<HL>(G, p0, f0, b0);
            hm.load<HL>(G, p1, f1, b1);
            float2 cost, gt;
            tv_terms2m(c, f0, b0, f1, b1, w01.x, w01.y, p.k.iv, p.k.niv, tv3 ? 3 : 2, cost, gt);
            if (ok0) {
                q1 = __fmaf_rn(tvs0, cost.x, q1);
                grf.x = fma1(tvs0, gt.x, grf.x);
            }
            if (ok1) {
                q1 = __fmaf_rn(tvs0, cost.y, q1);
                grf.y = fma1(tvs0, gt.y, grf.y);
            }
            if (upd) {
                const float2 gzr = mul2(grf, dthr);
                const float2 gz[NP] = {kr == 0 ? gzr : gn, kr == 0 ? gn : gzr};
                float2 zr = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    float* pz = s_st + (0 * NP + k) * S;
                    float* p1s = s_st + (1 * NP + k) * S;
                    float* p2s = s_st + (2 * NP + k) * S;
                    float2 zz = ld2(pz, q), mm1 = ld2(p1s, q), mm2 = ld2(p2s, q);
                    adam_step2c(p.k, nscx, scy, zz, mm1, mm2, gz[k]);
                    st2(pz, q, zz);
                    st2(p1s, q, mm1);
                    st2(p2s, q, mm2);
                    if (k == kr) zr = zz;
                    if (ckpt) {  // padding voxels included: never read back
                        st2g(cp + (size_t)k * a.nvtot, v0, zz);
                        st2g(cp + (size_t)(NP + k) * a.nvtot, v0, mm1);
                        st2g(cp + (size_t)(2 * NP + k) * a.nvtot, v0, mm2);
                    }
                }
                float2 dd;
                const float2 thr = unscale_sig2c(p.k, kr, zr, dd);
                // the new map value and its dtheta/dz serve the next
                // fidelity pass too (the same transform of the same z)
                st2(s_gf + 2 * S, q, dd);
                st2(s_gf + 3 * S, q, thr);
                if (ok0) Gn[p0] = thr.x;
                if (ok1) Gn[p1] = thr.y;
                const unsigned int fw0 = ok0 ? w01.x >> 24 : 0u, fw1 = ok1 ? w01.y >> 24 : 0u;
                if (fw0 | fw1) {  // voxels on a face of the volume: the halo copies
                    hm.mirror(Gn, p0, fw0, thr.x);
                    hm.mirror(Gn, p1, fw1, thr.y);
                }
            }
        }
        return true;
        };
        bool go;
        if (p.hlayout == 7) go = a.reg_param[0] == 0 ? pair_epoch(IntC<0>{}, IntC<7>{}) : pair_epoch(IntC<1>{}, IntC<7>{});
        else if (p.hlayout == 8) go = a.reg_param[0] == 0 ? pair_epoch(IntC<0>{}, IntC<8>{}) : pair_epoch(IntC<1>{}, IntC<8>{});
        else if (p.hlayout == 9) go = a.reg_param[0] == 0 ? pair_epoch(IntC<0>{}, IntC<9>{}) : pair_epoch(IntC<1>{}, IntC<9>{});
        else go = a.reg_param[0] == 0 ? pair_epoch(IntC<0>{}, IntC<0>{}) : pair_epoch(IntC<1>{}, IntC<0>{});
        if (!go) return;
        } else {
        // pass 1: data fidelity of the slice (own voxels only)
        for (int i = tid; i < n; i += NWT) {
            const int v = base + i;
            const bool ok = (v - V.off) < V.nvox;
            const float* yb = p.data_in_smem ? s_y + i : a.data + v;
            const int ys = p.data_in_smem ? S : a.nvtot;
            PrefLossAcc<LOSS, NP, (MAXM > 0 ? MAXM : 4)> pacc;
            if constexpr (MAXM > 0) {  // the measurement loads first: in flight during the transform
                if (p.data_quads) pacc.load_quads(p.data_quads + v, (size_t)a.nvtot);
                else pacc.load(yb, ys, nm);
            }
            float th[NP], dth[NP];
#pragma unroll
            for (int k = 0; k < NP; ++k)
                th[k] = unscale(transform, a.P.lb[k], a.P.ub[k], s_st[(0 * NP + k) * S + i], dth[k]);
            float tot, g0, g1;
            if constexpr (MAXM > 0) {
                auto& acc = pacc;
                acc.total = 0.0f;
                acc.g[0] = acc.g[1] = 0.0f;
                acc.w = a.weights ? a.weights + v : nullptr;
                acc.ws = a.nvtot;
                acc.aux = make_loss_aux(a.sigma ? a.sigma[v] : a.sigma_default);
                acc.mse_scale = a.mse_scale;
                acc.hd = a.huber_delta;
                acc.res = nullptr;  // residuals: pass after the epoch loop
                acc.rs = a.nvtot;
                model_r2s_unrolled<MAXM>(a.P, nm, th, acc);  // echo constants as constant-bank operands
                acc.finish();
                tot = acc.total;
                g0 = acc.g[0];
                g1 = acc.g[1];
            } else {
                PLossAcc<LOSS, NP> acc;
                acc.total = 0.0f;
                acc.g[0] = acc.g[1] = 0.0f;
                acc.y = yb;
                acc.ys = ys;
                acc.w = a.weights ? a.weights + v : nullptr;
                acc.ws = a.nvtot;
                acc.aux = make_loss_aux(a.sigma ? a.sigma[v] : a.sigma_default);
                acc.mse_scale = a.mse_scale;
                acc.hd = a.huber_delta;
                acc.res = (p.want_res && a.res_out && e == p.e_end && ok) ? a.res_out + v : nullptr;
                acc.rs = a.nvtot;
                acc.rt.kind = p.loss;
                VoxAux va{1.0f, nullptr, nullptr, 1};
                model_eval<kR2S>(s_P, th, va, acc);
                acc.finish();
                tot = acc.total;
                g0 = acc.g[0];
                g1 = acc.g[1];
            }
            s_gf[0 * S + i] = g0 * V.norm;
            s_gf[1 * S + i] = g1 * V.norm;
            if (ok) q0 += tot;
        }
        // every CTA's map of the previous epoch (written before its arrival)
        if (e > p.e_begin)
            if (!mbar_wait(&bar_open, (unsigned int)(e - 1 - p.e_begin) & 1u, p.barrier, wait_limit) ||
                *(volatile int*)&s_err)
                return;
        // pass 2: TV subgradient, chain rule, optimiser, new map values
        for (int i = tid; i < n; i += NWT) {
            const int v = base + i;
            const bool ok = (v - V.off) < V.nvox;
            float z[NP], th[NP], dth[NP], gth[NP];
            float gz[NP];
            float reg = 0.0f;
            const int pidx = s_p[i];
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                z[k] = s_st[(0 * NP + k) * S + i];
                th[k] = unscale(transform, a.P.lb[k], a.P.ub[k], z[k], dth[k]);
                gth[k] = s_gf[k * S + i];
            }
            if (ok && nreg > 0) {
                const unsigned int w = s_w[i];
                const unsigned int fl = w >> 24;
                const bool mb[3] = {(w & 1u) != 0, (w & 0x100u) != 0, (w & 0x10000u) != 0};
                const float iv[3] = {ivx, ivy, ivz};
                for (int r = 0; r < nreg; ++r) {
                    const int k = a.reg_param[r];
                    const float c = k == 0 ? th[0] : th[1];
                    float f[3], b[3];
                    hm.load<0>(gcur + (size_t)r * p.hgrid_total + V.hgrid_off, pidx, f, b);
                    float cost, gr;
                    tv_terms(c, f, b, mb, iv, tv3 ? 3 : 2, cost, gr);
                    const float tvs = r == 0 ? tvs0 : tvs1;
                    reg += tvs * cost;
                    if (k == 0) gth[0] = fma1(tvs, gr, gth[0]);
                    else gth[1] = fma1(tvs, gr, gth[1]);
                }
            }
#pragma unroll
            for (int k = 0; k < NP; ++k) gz[k] = gth[k] * dth[k];
            if (ok) {
                q1 += reg;
                if constexpr (STATS) {
#pragma unroll
                    for (int k = 0; k < NP; ++k) {
                        float zpk = s_st[(3 * NP + k) * S + i];
                        q2 += gz[k] * gz[k];
                        q3 += z[k] * z[k];
                        q4 += (z[k] - zpk) * (z[k] - zpk);
                    }
                }
            }
            if (upd && ok) {
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    float zz = z[k];
                    float mm1 = s_st[(1 * NP + k) * S + i], mm2 = s_st[(2 * NP + k) * S + i];
                    if constexpr (STATS) s_st[(3 * NP + k) * S + i] = zz;
                    opt_step(oc, sc, zz, mm1, mm2, gz[k]);
                    z[k] = zz;
                    s_st[(0 * NP + k) * S + i] = zz;
                    s_st[(1 * NP + k) * S + i] = mm1;
                    s_st[(2 * NP + k) * S + i] = mm2;
                    if (a.ckpt_every > 0 && (e % a.ckpt_every) == 0) {
                        float* cp = a.ckpt + (size_t)(e / a.ckpt_every) * 3 * NP * a.nvtot;
                        cp[(size_t)k * a.nvtot + v] = zz;
                        cp[(size_t)(NP + k) * a.nvtot + v] = mm1;
                        cp[(size_t)(2 * NP + k) * a.nvtot + v] = mm2;
                    }
                }
                for (int r = 0; r < nreg; ++r) {
                    const int k = a.reg_param[r];
                    float dd;
                    const float th = unscale(transform, a.P.lb[k], a.P.ub[k], k == 0 ? z[0] : z[1], dd);
                    float* Gn = gnext + (size_t)r * p.hgrid_total + V.hgrid_off;
                    Gn[pidx] = th;
                    const unsigned int fl = s_w[i] >> 24;
                    if (fl) hm.mirror(Gn, pidx, fl, th);
                }
            }
        }
        }
        // arrival: this warp's map writes and partial history sums
        const int lane = tid & 31, warp = tid >> 5;
        if (p.record && a.hist) {
            double* buf = s_red + (e & 1) * 32 * kHistW;
            float q[kHistW] = {q0, q1, q2, q3, q4};
            constexpr int NQ = STATS ? kHistW : 2;
#pragma unroll
            for (int k = 0; k < NQ; ++k) {
                float sum = warp_sum_p(q[k]);
                if (lane == 0) buf[warp * kHistW + k] = (double)sum;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&bar_arrive);
    }
    __syncthreads();
    if constexpr (STD) {
        // residuals of the final evaluation; the launch ends with an epoch
        // without update (host-checked), so the state is the evaluated one
        if (p.want_res && a.res_out) {
            for (int i = tid; i < n; i += BT) {
                const int v = base + i;
                if ((v - V.off) >= V.nvox) continue;
                float th[NP], dth[NP];
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    th[k] = unscale(transform, a.P.lb[k], a.P.ub[k], s_st[(0 * NP + k) * S + sidx(i)], dth[k]);
                PLossAcc<LOSS, NP> acc;
                acc.total = 0.0f;
                acc.g[0] = acc.g[1] = 0.0f;
                acc.y = p.data_in_smem ? s_y + sidx(i) : a.data + v;
                acc.ys = p.data_in_smem ? S : a.nvtot;
                acc.w = a.weights ? a.weights + v : nullptr;
                acc.ws = a.nvtot;
                acc.aux = make_loss_aux(a.sigma ? a.sigma[v] : a.sigma_default);
                acc.mse_scale = a.mse_scale;
                acc.hd = a.huber_delta;
                acc.res = a.res_out + v;
                acc.rs = a.nvtot;
                acc.rt.kind = p.loss;
                VoxAux va{1.0f, nullptr, nullptr, 1};
                model_eval<kR2S>(s_P, th, va, acc);
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < n; i += BT) {
        const int v = base + i;
        if ((v - V.off) >= V.nvox) continue;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            size_t gi = (size_t)k * a.nvtot + v;
            const int j = sidx(i);
            a.z[gi] = s_st[(0 * NP + k) * S + j];
            a.m1[gi] = s_st[(1 * NP + k) * S + j];
            a.m2[gi] = s_st[(2 * NP + k) * S + j];
            if constexpr (STATS)
                if (a.zprev) a.zprev[gi] = s_st[(3 * NP + k) * S + j];
        }
    }
}

namespace {

// Variants: MSE with up to 8, 12, 16 or 32 echoes (measurements prefetched
// into registers; the smallest bound that holds the protocol), and any loss /
// echo count with the loss chosen at run time.
// The pair variant covers a slice in chunks of 64 voxels (pairs i, i+32).
bool pair_layout_ok(int nvtot, int slice) { return nvtot % 64 == 0 && slice % 64 == 0; }

int persist_variant(const AdamParams& a, int loss, bool res_after_loop) {
    const bool std_cfg = loss == kMSE && a.transform == 0 && a.optimiser == kAdam && a.n_reg == 1 && res_after_loop;
    if (std_cfg && a.nm <= 8) return 8;
    if (std_cfg && a.nm <= 12) return 12;
    if (std_cfg && a.nm <= 16) return 16;
    if (std_cfg && a.nm <= 32) return 32;
    return 0;
}

template <int LOSS, int MAXM>
cudaError_t launch_persist_t(const AdamParams& a, PersistArgs p, int bt, int nblocks, size_t smem,
                             cudaStream_t s) {
    const bool hook = p.spin_cycles != kBarrierSpinCycles || p.extra_arrivals != 0;
    auto k = p.stats ? (hook ? tv_persistent_kernel<LOSS, true, MAXM, true> : tv_persistent_kernel<LOSS, true, MAXM, false>)
                     : (hook ? tv_persistent_kernel<LOSS, false, MAXM, true> : tv_persistent_kernel<LOSS, false, MAXM, false>);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void* args[] = {const_cast<void*>(static_cast<const void*>(&a)), static_cast<void*>(&p)};
    e = cudaLaunchCooperativeKernel((const void*)k, dim3(nblocks), dim3(bt), args, smem, s);
    ++g_kernel_launches;
    return e;
}

template <int LOSS, int MAXM>
int occupancy_t(int bt, size_t smem) {
    int nb = 0, nb2 = 0;
    auto k0 = tv_persistent_kernel<LOSS, false, MAXM, false>;
    auto k1 = tv_persistent_kernel<LOSS, true, MAXM, false>;
    if (cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k0, bt, smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, k1, bt, smem) != cudaSuccess) return 0;
    return nb < nb2 ? nb : nb2;
}

int occupancy_v(int variant, int bt, size_t smem) {
    if (variant == 8) return occupancy_t<kMSE, 8>(bt, smem);
    if (variant == 12) return occupancy_t<kMSE, 12>(bt, smem);
    if (variant == 16) return occupancy_t<kMSE, 16>(bt, smem);
    if (variant == 32) return occupancy_t<kMSE, 32>(bt, smem);
    return occupancy_t<-1, 0>(bt, smem);
}

}  // namespace

// Plan a persistent launch: one CTA per SM, slice = ceil(nvtot / #SM) voxels
// (rounded to whole warps, or with several volumes to a padding block so that
// a slice never straddles two volumes), the slice's Adam state in shared
// memory (and its measurements too when they fit), up to kPersistMaxThreads
// threads (worker warps and a barrier warp).  Returns false when the problem
// does not fit, in which case the caller uses the per-epoch kernel.
bool plan_persistent(const AdamParams& a, int model, int loss, bool stats, int pad_block, const int* vol_npad,
                     int nvol, PersistPlan* plan) {
    if (model != kR2S) return false;
    int dev = 0, nsm = 0, smem_optin = 0, coop = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return false;
    // one volume: slices of 64 voxels (the pair variant's chunks); several:
    // of padding blocks, so that every volume starts on a slice boundary
    const int gran = nvol == 1 ? 64 : pad_block;
    int slice = (a.nvtot + nsm - 1) / nsm;
    slice = (slice + gran - 1) / gran * gran;
    {
        long long acc = 0;
        for (int i = 0; i < nvol; ++i) {  // every volume starts on a slice boundary
            if (acc % slice) return false;
            acc += vol_npad[i];
        }
    }
    const bool stats_any = true;  // size for the larger (statistics) variant
    const int NS = stats_any ? 4 : 3;
    size_t red = sizeof(double) * 2 * 32 * kHistW;
    size_t state = sizeof(float) * (size_t)(NS + 1) * 2 * slice + sizeof(int) * slice +
                   sizeof(unsigned int) * slice;  // + fidelity gradient [2][slice], mask words
    size_t data = sizeof(float) * (size_t)a.nm * slice;
    const size_t budget = (size_t)smem_optin - 2048;  // static shared memory (staged protocol) and slack
    if (red + state > budget) return false;
    int in_smem = red + state + data <= budget ? 1 : 0;
    size_t smem = red + state + (in_smem ? data : 0);
    // worker threads: as many as fit beside the barrier warp, spread so that
    // the last pass over the slice is full (every worker warp reaches the
    // grid barrier after the same number of voxels)
    const int variant = persist_variant(a, loss, true);
    const bool pairs = persist_pairs(variant, stats) && pair_layout_ok(a.nvtot, slice);  // two voxels per thread
    const int units = pairs ? slice / 2 : slice;
    // every variant that may run with this thread count must allow it
    const int maxw = std::min(persist_max_threads(variant, stats), persist_max_threads(variant, !stats)) - 32;
    int passes = (units + maxw - 1) / maxw;
    int bt = ((units + passes - 1) / passes + 31) / 32 * 32 + 32;
    int nb = occupancy_v(variant, bt, smem);
    if (variant != 0) nb = std::min(nb, occupancy_v(0, bt, smem));
    if (nb < 1) return false;
    plan->slice = slice;
    plan->vpt = 0;
    plan->threads = bt;
    plan->ctas = (a.nvtot + slice - 1) / slice;
    if (plan->ctas > nb * nsm) return false;
    plan->smem = smem;
    plan->data_in_smem = in_smem;
    plan->quad_width = (!in_smem && variant > 0) ? variant : 0;
    plan->quad_pairs = pairs ? 1 : 0;
    return true;
}

cudaError_t launch_tv_persistent(const AdamParams& a, const PersistPlan& plan, PersistArgs p, cudaStream_t s) {
    p.slice = plan.slice;
    // the pair variant's constants, rounded as the kernels round them (FP32)
    auto pr = [](float x) { return make_float2(x, x); };
    p.k.nl2e = pr(-kLog2e);
    p.k.one = pr(1.0f);
    for (int i = 0; i < 2; ++i) {
        p.k.rng[i] = pr(a.P.ub[i] - a.P.lb[i]);
        p.k.lb[i] = pr(a.P.lb[i]);
    }
    p.k.b1 = pr(a.beta1);
    p.k.omb1 = pr(1.0f - a.beta1);
    p.k.b2 = pr(a.beta2);
    p.k.omb2 = pr(1.0f - a.beta2);
    p.k.eps = pr(a.eps);
    p.k.mse = pr(a.mse_scale);
    p.k.s2 = pr(2.0f * a.mse_scale);
    for (int d = 0; d < 3; ++d) {
        p.k.iv[d] = pr(a.inv_vs[d]);
        p.k.niv[d] = pr(-a.inv_vs[d]);
    }
    p.data_in_smem = plan.data_in_smem;
    // the register-prefetch variants write residuals after their epoch loop,
    // which needs a launch whose last epoch is not followed by an update
    const int variant = persist_variant(a, p.loss, !p.want_res || p.e_end > p.update_last);
    // the pair variant needs slices and a work-list of whole 64-voxel chunks;
    // otherwise the run-time variant takes the launch
    int var = variant;
    if (persist_pairs(var, p.stats != 0) && !pair_layout_ok(a.nvtot, plan.slice)) var = 0;
    const int pairs = persist_pairs(var, p.stats != 0) ? 1 : 0;
    if (var != plan.quad_width || pairs != plan.quad_pairs) p.data_quads = nullptr;  // read [nm][nvtot]
    if (var == 8) return launch_persist_t<kMSE, 8>(a, p, plan.threads, plan.ctas, plan.smem, s);
    if (var == 12) return launch_persist_t<kMSE, 12>(a, p, plan.threads, plan.ctas, plan.smem, s);
    if (var == 16) return launch_persist_t<kMSE, 16>(a, p, plan.threads, plan.ctas, plan.smem, s);
    if (var == 32) return launch_persist_t<kMSE, 32>(a, p, plan.threads, plan.ctas, plan.smem, s);
    return launch_persist_t<-1, 0>(a, p, plan.threads, plan.ctas, plan.smem, s);
}

namespace {

__global__ void echo_quads_kernel(const float* data, int nm, int nvtot, int width, float4* out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvtot) return;
    for (int j = 0; j < width / 4; ++j) {
        float t[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int m = 4 * j + c;
            t[c] = m < nm ? data[(size_t)m * nvtot + v] : 0.0f;
        }
        out[(size_t)j * nvtot + v] = make_float4(t[0], t[1], t[2], t[3]);
    }
}

// Pair quads: with the voxel pairs (u0, u0 + 32), u0 = 64 (u / 32) + u % 32,
// quad j of pair u = (y_2j(u0), y_2j(u0+32), y_2j+1(u0), y_2j+1(u0+32)) at
// out[((u / 32) (width / 2) + j) 32 + u % 32]: the width / 2 quads of 32
// consecutive pairs lie together, 512 bytes apart.
__global__ void pair_quads_kernel(const float* data, int nm, int nvtot, int width, float4* out) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int npair = nvtot >> 1;
    if (u >= npair) return;
    const int u0 = ((u >> 5) << 6) + (u & 31);
    float4* o = out + (size_t)(u >> 5) * (width / 2) * 32 + (u & 31);
    for (int j = 0; j < width / 2; ++j) {
        const int m0 = 2 * j, m1 = 2 * j + 1;
        const float* r0 = data + (size_t)m0 * nvtot + u0;
        const float* r1 = data + (size_t)m1 * nvtot + u0;
        o[j * 32] = make_float4(m0 < nm ? r0[0] : 0.f, m0 < nm ? r0[32] : 0.f, m1 < nm ? r1[0] : 0.f,
                                m1 < nm ? r1[32] : 0.f);
    }
}

}  // namespace

cudaError_t launch_echo_quads(const float* data, int nm, int nvtot, int width, bool pairs, float4* out,
                              cudaStream_t s) {
    if (width % 4 != 0 || nm > width || (pairs ? nvtot % 64 : nvtot % 2)) return cudaErrorInvalidValue;
    if (pairs) pair_quads_kernel<<<(nvtot / 2 + 255) / 256, 256, 0, s>>>(data, nm, nvtot, width, out);
    else echo_quads_kernel<<<(nvtot + 255) / 256, 256, 0, s>>>(data, nm, nvtot, width, out);
    ++g_kernel_launches;
    return cudaGetLastError();
}

}  // namespace gx
