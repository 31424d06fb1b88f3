// dictionary.cu -- dictionary matching for likelihood starting points
// (gpuNEXI.likelihood, NEXI/gpuNEXI.m:813-836): for every voxel the first
// dictionary entry j minimising
//     sse_j = sum_m wt_m (S0_m - c_j S_jm)^2,   c_j = (S0 . S_j) / (S_j . S_j).
//
// Expanded per (voxel i, entry j):  sse = A_i - 2 c B_ij + c^2 C_j with
// D_ij = S0_i . S_j, B_ij = sum_m wt_m S0_im S_jm, A_i = sum_m wt_m S0_im^2,
// E_j = S_j . S_j, C_j = sum_m wt_m S_jm^2 and c = D_ij / E_j (unit weights:
// sse = A_i - D_ij^2 / E_j).  The pair terms are the dot products of a
// [nvox x nm] x [nm x ndict] product, computed here as a register-tiled GEMM
// over dictionary tiles with a running argmin in the epilogue, so the score
// matrix is never stored.  The products accumulate in FP64: for a good match
// sse / A is ~1e-3, so the expanded form loses about three digits to
// cancellation, which FP32 (or TF32 tensor-core) accumulation cannot afford
// for an exact decision; with K = nm ~ 24 the epilogue also costs as much as
// the products, so the CUDA-core FP64 pipe is the right unit here.
#include "gx_internal.h"

namespace gx {

namespace {

constexpr int kTile = 64;   // voxels and entries per CTA tile
constexpr int kThreads = 256;

// Per entry: 1 / (S_j . S_j) and sum_m wt_m S_jm^2 (double).
__global__ void dict_entry_kernel(const float* dict, int ndict, int nm, const float* wt, double* invE,
                                  double* C) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ndict) return;
    double e = 0.0, c = 0.0;
    for (int m = 0; m < nm; ++m) {
        double s = (double)dict[(size_t)m * ndict + j];
        e = fma(s, s, e);
        c = fma(wt ? (double)wt[m] * s : s, s, c);
    }
    invE[j] = 1.0 / e;   // E = 0: inf, and the pair scores NaN, which never wins
    C[j] = c;
}

// Lexicographic (sse, j): smaller sse, then smaller j (MATLAB min's first index).
__device__ __forceinline__ bool better(double s1, int j1, double s0, int j0) {
    return s1 < s0 || (s1 == s0 && j1 < j0);
}

template <bool WEIGHTED>
__global__ void __launch_bounds__(kThreads)
dict_match_kernel(const float* signals, int nvox, const float* dict, int ndict, int nm, const float* wt,
                  const double* invE, const double* Cj, int* best, float* best_sse) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sv = reinterpret_cast<double*>(smem_raw);      // [nm][64] voxel signals
    double* sd = sv + (size_t)nm * kTile;                  // [nm][64] dictionary tile
    double* sw = sd + (size_t)nm * kTile;                  // [nm][64] wt * voxel signals (weighted)
    __shared__ double s_A[kTile], s_ie[kTile], s_c[kTile];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int i0 = blockIdx.x * kTile;
    for (int q = tid; q < nm * kTile; q += kThreads) {
        int m = q / kTile, v = q % kTile;
        double x = (i0 + v < nvox) ? (double)signals[(size_t)m * nvox + i0 + v] : 0.0;
        sv[q] = x;
        if (WEIGHTED) sw[q] = (double)wt[m] * x;
    }
    __syncthreads();
    if (tid < kTile) {
        double a = 0.0;
        for (int m = 0; m < nm; ++m) a = fma(WEIGHTED ? sw[m * kTile + tid] : sv[m * kTile + tid], sv[m * kTile + tid], a);
        s_A[tid] = a;
    }
    double bs[4];
    int bj[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) { bs[a] = INFINITY; bj[a] = 0x7fffffff; }

    for (int j0 = 0; j0 < ndict; j0 += kTile) {
        __syncthreads();  // the previous tile is consumed
        for (int q = tid; q < nm * kTile; q += kThreads) {
            int m = q / kTile, e = q % kTile;
            sd[q] = (j0 + e < ndict) ? (double)dict[(size_t)m * ndict + j0 + e] : 0.0;
        }
        if (tid < kTile) {
            bool ok = j0 + tid < ndict;
            s_ie[tid] = ok ? invE[j0 + tid] : 0.0;
            s_c[tid] = ok ? Cj[j0 + tid] : 0.0;
        }
        __syncthreads();
        double D[4][4], B[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) { D[a][b] = 0.0; B[a][b] = 0.0; }
        for (int m = 0; m < nm; ++m) {
            double x[4], y[4], xw[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                x[a] = sv[m * kTile + ty + 16 * a];
                if (WEIGHTED) xw[a] = sw[m * kTile + ty + 16 * a];
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) y[b] = sd[m * kTile + tx + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    D[a][b] = fma(x[a], y[b], D[a][b]);
                    if (WEIGHTED) B[a][b] = fma(xw[a], y[b], B[a][b]);
                }
        }
        // epilogue: entries in increasing j per thread, strict improvement
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int e = tx + 16 * b, j = j0 + e;
            if (j >= ndict) continue;
            const double ie = s_ie[e], cc = s_c[e];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double c = D[a][b] * ie;
                const double sse = WEIGHTED ? s_A[ty + 16 * a] - c * (2.0 * B[a][b] - c * cc)
                                            : s_A[ty + 16 * a] - c * D[a][b];
                if (sse < bs[a]) { bs[a] = sse; bj[a] = j; }
            }
        }
    }
    // fold the 16 threads that share each voxel (lanes with equal ty)
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        double s = bs[a];
        int j = bj[a];
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            double s2 = __shfl_xor_sync(0xffffffffu, s, o);
            int j2 = __shfl_xor_sync(0xffffffffu, j, o);
            if (better(s2, j2, s, j)) { s = s2; j = j2; }
        }
        const int i = i0 + ty + 16 * a;
        if (tx == 0 && i < nvox) {
            best[i] = j == 0x7fffffff ? -1 : j;
            if (best_sse) best_sse[i] = (float)s;
        }
    }
}

}  // namespace

size_t dict_match_smem(int nm, bool weighted) {
    return sizeof(double) * (size_t)nm * kTile * (weighted ? 3 : 2);
}

cudaError_t launch_dictionary_match(const float* signals, int nvox, const float* dict, int ndict, int nm,
                                    const float* wt, double* invE, double* Cj, int* best, float* best_sse,
                                    cudaStream_t s) {
    dict_entry_kernel<<<(ndict + 255) / 256, 256, 0, s>>>(dict, ndict, nm, wt, invE, Cj);
    ++g_kernel_launches;
    const bool weighted = wt != nullptr;
    const size_t smem = dict_match_smem(nm, weighted);
    auto k = weighted ? dict_match_kernel<true> : dict_match_kernel<false>;
    // the kernel also holds static shared arrays, so opt in for every size
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<(nvox + kTile - 1) / kTile, kThreads, smem, s>>>(signals, nvox, dict, ndict, nm, wt, invE, Cj, best,
                                                          best_sse);
    ++g_kernel_launches;
    return cudaGetLastError();
}

}  // namespace gx
