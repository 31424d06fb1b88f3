// posterior_stats.cu -- posterior median, inter-quartile range and mode per
// voxel and parameter, computed on the device from the kept samples
// (mcmc.res2out, utils/mcmc.m:806-862), so that a run whose posterior does
// not fit a host round trip (200k voxels x 64 walkers x 400 samples x 5
// parameters is 102 GB) still returns these summaries.
//
// One CTA per (voxel, parameter): the N = rep x ns x W samples of the
// segment (stride nvox in the posterior [nvar][rep][ns][W][nvox]) are staged
// in shared memory as order-preserving 32-bit keys when they fit, otherwise
// re-read from HBM on every pass.  Order statistics come from a radix select
// that resolves the bits below the segment's common prefix (min and max key)
// eight at a time, for up to three ranks at once (the lower neighbours of
// the median and of the 25th and 75th percentiles), with warp-aggregated
// shared-memory histogram updates; a last pass finds each rank's upper
// neighbour.  The mode is the most populated of the Nbin - 1 bins between
// linspace(lb - 1e-8, ub + 1e-8, Nbin) (the lowest bin wins a tie), its
// value the bin centre.
//
// MATLAB semantics restated: median of an even count = mean of the two middle
// values; iqr = prctile(x, 75) - prctile(x, 25) with prctile's midpoint rule
// (sorted value i sits at percentile 100 (i - 0.5) / N, linear interpolation
// in between, clamped outside); discretize puts x in bin k when
// edges(k) <= x < edges(k+1), the last bin closed, values outside the edges
// are NaN and ignored by mode; linspace(d1, d2, n) = d1 + ((0:n-1) (d2 - d1)) / (n - 1)
// with the last element d2.
#include <cfloat>

#include "gx_internal.h"

namespace gx {

namespace {

constexpr int kStatThreads = 512;
constexpr int kMaxTargets = 3;

__device__ __forceinline__ uint32_t f2key(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float key2f(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Histogram increment with the lanes of a warp that hit the same bin merged
// into one shared-memory atomic (posterior samples crowd into few bins).
__device__ __forceinline__ void hist_add(unsigned int* hist, int bin, bool active) {
    const unsigned int am = __ballot_sync(0xffffffffu, active);
    if (!active) return;
    const unsigned int peers = __match_any_sync(am, bin);
    const int lane = threadIdx.x & 31;
    if (lane == __ffs(peers) - 1) atomicAdd(hist + bin, (unsigned int)__popc(peers));
}

struct BlockScratch {
    unsigned int hist[kMaxTargets][256];
    uint32_t red_u[2][kStatThreads / 32];
    unsigned int red_i[kStatThreads / 32];
    uint32_t prefix[kMaxTargets];
    unsigned int rank[kMaxTargets];   // rank still to find within the current prefix
    unsigned int below[kMaxTargets];  // elements below the current prefix range
    unsigned int eq[kMaxTargets];     // elements equal to the selected key
    uint32_t next[kMaxTargets];       // upper neighbour
    uint32_t kmin, kmax;
};

template <bool STAGED>
__device__ __forceinline__ uint32_t key_at(const uint32_t* keys, const float* seg, size_t stride, int i) {
    if constexpr (STAGED) return keys[i];
    else return f2key(__ldg(seg + (size_t)i * stride));
}

}  // namespace

// grid (nvox, nvar); post [nvar][N][nvox] with N = rep * ns * W.
template <bool STAGED>
__global__ void __launch_bounds__(kStatThreads)
posterior_stats_kernel(const float* __restrict__ post, int nvox, int N, int nbin, const double* __restrict__ lbub,
                       float* median, float* iqr, float* mode) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ BlockScratch S;
    const int v = blockIdx.x, q = blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kStatThreads / 32;
    const size_t stride = (size_t)nvox;
    const float* seg = post + (size_t)q * N * stride + v;
    uint32_t* keys = reinterpret_cast<uint32_t*>(smem_raw);           // [N] when staged
    unsigned int* mhist = reinterpret_cast<unsigned int*>(smem_raw + (STAGED ? sizeof(uint32_t) * (size_t)N : 0));
    const bool want_ord = median || iqr;

    // stage the keys and find the segment's smallest and largest key
    uint32_t lo = 0xffffffffu, hi = 0u;
    for (int i = tid; i < N; i += kStatThreads) {
        const uint32_t k = f2key(__ldg(seg + (size_t)i * stride));
        if constexpr (STAGED) keys[i] = k;
        lo = min(lo, k);
        hi = max(hi, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) { S.red_u[0][warp] = lo; S.red_u[1][warp] = hi; }
    __syncthreads();
    if (tid == 0) {
        uint32_t a = S.red_u[0][0], b = S.red_u[1][0];
        for (int w = 1; w < NW; ++w) { a = min(a, S.red_u[0][w]); b = max(b, S.red_u[1][w]); }
        S.kmin = a;
        S.kmax = b;
    }
    __syncthreads();
    const uint32_t kmin = S.kmin, kmax = S.kmax;

    if (want_ord) {
        // ranks (0-based) of the lower neighbours: median, 25th, 75th percentile
        double pos[kMaxTargets];
        pos[0] = 0.5 * (double)(N - 1);                      // median: (N-1)/2
        pos[1] = (double)N * 0.25 - 0.5;                     // prctile midpoint rule
        pos[2] = (double)N * 0.75 - 0.5;
        int nt = iqr ? 3 : 1;
        if (tid < kMaxTargets) {
            double pc = fmin(fmax(pos[tid], 0.0), (double)(N - 1));
            S.rank[tid] = (unsigned int)floor(pc);
            S.below[tid] = 0;
            S.prefix[tid] = 0;
        }
        // radix select over the bits below the common prefix of kmin and kmax
        const uint32_t diff = kmin ^ kmax;
        int hb = diff ? 32 - __clz(diff) : 0;   // bits [0, hb) differ somewhere
        if (tid < kMaxTargets) S.prefix[tid] = hb >= 32 ? 0u : (kmin & ~((1u << hb) - 1u));
        __syncthreads();
        while (hb > 0) {
            const int w = hb < 8 ? hb : 8;
            const int lob = hb - w;
            const uint32_t mask = hb >= 32 ? 0u : ~((1u << hb) - 1u);
            const uint32_t dmask = (1u << w) - 1u;
            for (int i = tid; i < nt * 256; i += kStatThreads) (&S.hist[0][0])[i] = 0u;
            __syncthreads();
            uint32_t pf[kMaxTargets];
#pragma unroll
            for (int t = 0; t < kMaxTargets; ++t) pf[t] = S.prefix[t];
            const int nfull = (N + kStatThreads - 1) / kStatThreads;
            for (int it = 0; it < nfull; ++it) {
                const int i = it * kStatThreads + tid;
                const bool in = i < N;
                const uint32_t k = in ? key_at<STAGED>(keys, seg, stride, i) : 0u;
                const int d = (int)((k >> lob) & dmask);
#pragma unroll
                for (int t = 0; t < kMaxTargets; ++t)
                    if (t < nt) hist_add(S.hist[t], d, in && ((k ^ pf[t]) & mask) == 0u);
            }
            __syncthreads();
            // one warp per target: find the digit whose cumulative count passes the rank
            if (warp < nt) {
                const int t = warp;
                const unsigned int* h = S.hist[t];
                unsigned int c[8], s = 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) { c[j] = h[lane * 8 + j]; s += c[j]; }
                unsigned int incl = s;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned int n = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += n;
                }
                const unsigned int r = S.rank[t];
                const unsigned int found = __ballot_sync(0xffffffffu, incl > r);
                const int fl = __ffs(found) - 1;   // first lane whose range passes the rank
                if (lane == fl) {
                    unsigned int acc = incl - s;
                    int j = 0;
                    while (acc + c[j] <= r) { acc += c[j]; ++j; }
                    const uint32_t dsel = (uint32_t)(lane * 8 + j);
                    S.prefix[t] = (S.prefix[t] & mask) | (dsel << lob);
                    S.rank[t] = r - acc;
                    S.below[t] += acc;
                    S.eq[t] = c[j];
                }
            }
            __syncthreads();
            hb = lob;
        }
        if (tid < kMaxTargets) {
            if (kmin == kmax) S.eq[tid] = (unsigned int)N;   // no pass ran: every key equals kmin
            S.next[tid] = 0xffffffffu;
        }
        __syncthreads();
        // upper neighbours: the selected key again while equal keys remain, else
        // the smallest key above it
        uint32_t sel[kMaxTargets], nx[kMaxTargets];
        bool need_any = false;
#pragma unroll
        for (int t = 0; t < kMaxTargets; ++t) {
            sel[t] = S.prefix[t];
            nx[t] = 0xffffffffu;
            // rank + 1 still among the equal keys?
            const unsigned int r1 = (unsigned int)floor(fmin(fmax(pos[t], 0.0), (double)(N - 1))) + 1u;
            if (t < nt && r1 < (unsigned int)N && r1 >= S.below[t] + S.eq[t]) need_any = true;
        }
        if (need_any) {
            for (int i = tid; i < N; i += kStatThreads) {
                const uint32_t k = key_at<STAGED>(keys, seg, stride, i);
#pragma unroll
                for (int t = 0; t < kMaxTargets; ++t)
                    if (k > sel[t]) nx[t] = min(nx[t], k);
            }
#pragma unroll
            for (int t = 0; t < kMaxTargets; ++t) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) nx[t] = min(nx[t], __shfl_xor_sync(0xffffffffu, nx[t], o));
                if (lane == 0) atomicMin(&S.next[t], nx[t]);
            }
        }
        __syncthreads();
        if (tid == 0) {
            double xs[kMaxTargets], xn[kMaxTargets];
            for (int t = 0; t < nt; ++t) {
                const unsigned int r = (unsigned int)floor(fmin(fmax(pos[t], 0.0), (double)(N - 1)));
                xs[t] = (double)key2f(sel[t]);
                const bool same = r + 1u < S.below[t] + S.eq[t] || r + 1u >= (unsigned int)N;
                xn[t] = same ? xs[t] : (double)key2f(S.next[t]);
            }
            const size_t o = (size_t)q * nvox + v;
            if (median) {
                // odd N: pos is a whole rank; even N: mean of the two middle values
                median[o] = (N & 1) ? (float)xs[0] : (float)(0.5 * (xs[0] + xn[0]));
            }
            if (iqr) {
                double pr[2];
                for (int j = 0; j < 2; ++j) {
                    const double p = pos[1 + j];
                    if (p <= 0.0) pr[j] = xs[1 + j];                 // below the first sample's percentile
                    else if (p >= (double)(N - 1)) pr[j] = xs[1 + j]; // above the last one's
                    else {
                        const double f = p - floor(p);
                        pr[j] = xs[1 + j] + f * (xn[1 + j] - xs[1 + j]);
                    }
                }
                iqr[o] = (float)(pr[1] - pr[0]);
            }
        }
    }

    if (mode) {
        // discretize(x, linspace(lb - 1e-8, ub + 1e-8, nbin)), then the most
        // populated bin (lowest index on ties) and its centre
        const double d1 = lbub[2 * q] - 1e-8, d2 = lbub[2 * q + 1] + 1e-8;
        const int n1 = nbin - 1;           // bins
        auto edge = [&](int k) { return k >= n1 ? d2 : d1 + ((double)k * (d2 - d1)) / (double)n1; };
        const double inv = (double)n1 / (d2 - d1);
        for (int i = tid; i < n1; i += kStatThreads) mhist[i] = 0u;
        __syncthreads();
        const int nfull = (N + kStatThreads - 1) / kStatThreads;
        for (int it = 0; it < nfull; ++it) {
            const int i = it * kStatThreads + tid;
            bool in = i < N;
            int b = 0;
            if (in) {
                const double x = (double)key2f(key_at<STAGED>(keys, seg, stride, i));
                if (x < d1 || x > d2 || !(d2 > d1)) in = false;  // NaN under discretize: ignored by mode
                else {
                    b = (int)floor((x - d1) * inv);
                    b = min(max(b, 0), n1 - 1);
                    while (b > 0 && x < edge(b)) --b;
                    while (b < n1 - 1 && x >= edge(b + 1)) ++b;
                }
            }
            hist_add(mhist, b, in);
        }
        __syncthreads();
        // argmax, lowest bin on ties: pack (count, n1 - bin)
        unsigned long long best = 0ull;
        for (int i = tid; i < n1; i += kStatThreads) {
            const unsigned long long c = ((unsigned long long)mhist[i] << 32) | (unsigned int)(n1 - i);
            best = c > best ? c : best;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
            best = t > best ? t : best;
        }
        __shared__ unsigned long long s_best[NW];
        if (lane == 0) s_best[warp] = best;
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < NW; ++w) best = s_best[w] > best ? s_best[w] : best;
            best = s_best[0] > best ? s_best[0] : best;
            const unsigned int cnt = (unsigned int)(best >> 32);
            const int b = n1 - (int)(best & 0xffffffffu);
            mode[(size_t)q * nvox + v] = cnt == 0 ? __int_as_float(0x7fc00000) : (float)((edge(b) + edge(b + 1)) / 2.0);
        }
    }
}

// Shared memory of the staged variant: keys plus the mode histogram.
size_t posterior_stats_smem(int N, int nbin, bool staged) {
    return (staged ? sizeof(uint32_t) * (size_t)N : 0) + sizeof(unsigned int) * (size_t)(nbin > 1 ? nbin : 2);
}

cudaError_t launch_posterior_stats(const float* post, int nvar, int nvox, int N, int nbin, const double* lbub,
                                   float* median, float* iqr, float* mode, cudaStream_t s) {
    if (nvar < 1 || nvox < 1 || N < 1) return cudaErrorInvalidValue;
    if (mode && nbin < 2) return cudaErrorInvalidValue;
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    const size_t budget = (size_t)optin - sizeof(BlockScratch) - 1024;
    const bool staged = posterior_stats_smem(N, nbin, true) <= budget;
    const size_t smem = posterior_stats_smem(N, nbin, staged);
    if (smem > budget) return cudaErrorInvalidValue;  // Nbin too large for the histogram
    auto k = staged ? posterior_stats_kernel<true> : posterior_stats_kernel<false>;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<dim3(nvox, nvar), kStatThreads, smem, s>>>(post, nvox, N, nbin, lbub, median, iqr, mode);
    ++g_kernel_launches;
    return cudaGetLastError();
}

}  // namespace gx
