// noalloc.cu -- gx_askadam_noalloc: the fused askAdam fit of one volume
// without allocating any memory.
//
// Who needs it: programs that cannot call cudaMalloc once they are running,
// for example a host application that hands all device memory to its own
// allocator and forbids other allocations (a MATLAB MEX gateway working on
// MATLAB's own gpuArray memory), a reconstruction pipeline that reserves its
// memory at start-up and must not allocate (or fail with out-of-memory)
// while it streams data, or an embedding that must keep its device footprint
// fixed.  They pass device pointers for the measurements, the start point and
// the result; the engine's working memory comes from one fixed array below.
//
// The working memory is a file-scope __device__ array of kScratchBytes
// (32 MiB).  Every GPU on which the library is loaded holds it until the
// process exits.  All calls on a device share it and it keeps the contents of
// the last call; this function clears what must start at zero (the loss
// history) and rewrites everything else before use.  Two calls whose GPU work
// overlaps (different streams or host threads on the same device) race on it.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "gx_internal.h"

using namespace gx;

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

gx_status cuda_fail(cudaError_t e, const char* what) {
    char msg[512];
    snprintf(msg, sizeof(msg), "gx_askadam_noalloc: %s: %s", what, cudaGetErrorString(e));
    return internal_fail(e == cudaErrorMemoryAllocation ? GX_ENOMEM : GX_ECUDA, msg);
}

// The device address of g_scratch on the current device.  In host code the
// name g_scratch is only a host-side handle, not a device address, so it is
// resolved with cudaGetSymbolAddress once per device, with that device current.
gx_status scratch_address(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return internal_fail(GX_EUNSUPPORTED, "gx_askadam_noalloc: device index too large");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_scratch)");
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[dev];
    return GX_OK;
}

#define NA_CK(call)                                    \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// Byte offsets of the working arrays inside the fixed array for nvox voxels
// (padded to whole blocks of B), nm measurements, np parameters and N
// iterations; `total` is the bytes the layout needs.
struct Layout {
    size_t nvtot, nblocks;
    size_t vol, blk, sched, hist, data, th, z, m1, m2, total;
};

Layout layout(size_t nvox, int B, int nm, int np, int N) {
    Layout L;
    L.nvtot = (nvox + B - 1) / B * B;
    L.nblocks = L.nvtot / B;
    size_t off = 0;
    L.vol = off;   off += align256(sizeof(DevVol));
    L.blk = off;   off += align256(sizeof(int) * L.nblocks);
    L.sched = off; off += align256(sizeof(float2) * ((size_t)N + 1));
    L.hist = off;  off += align256(sizeof(double) * ((size_t)N + 1) * kHistW);
    L.data = off;  off += align256(sizeof(float) * nm * L.nvtot);
    L.th = off;    off += align256(sizeof(float) * np * L.nvtot);
    L.z = off;     off += align256(sizeof(float) * np * L.nvtot);
    L.m1 = off;    off += align256(sizeof(float) * np * L.nvtot);
    L.m2 = off;    off += align256(sizeof(float) * np * L.nvtot);
    L.total = off;
    return L;
}

// The largest voxel count whose layout fits the fixed array (0 if none does):
// the layout grows with nvox, so a binary search over the same function
// gives a figure that a retry is certain to pass.
size_t max_voxels(int B, int nm, int np, int N) {
    if (layout(1, B, nm, np, N).total > kScratchBytes) return 0;
    size_t lo = 1, hi = kScratchBytes / sizeof(float) + 1;  // layout(hi) cannot fit
    while (hi - lo > 1) {
        const size_t mid = lo + (hi - lo) / 2;
        if (layout(mid, B, nm, np, N).total <= kScratchBytes) lo = mid;
        else hi = mid;
    }
    return lo;
}

}  // namespace

extern "C" gx_status gx_askadam_noalloc(const gx_model* model, const float* data, const float* theta0,
                                        int32_t nvox, const gx_askadam_opts* o, void* cuda_stream,
                                        float* theta_out, double* final_loss) {
    if (!model || !data || !theta0 || !o || !theta_out)
        return internal_fail(GX_EINVAL, "gx_askadam_noalloc: NULL argument");
    if (nvox < 1) return internal_fail(GX_EINVAL, "gx_askadam_noalloc: nvox must be >= 1");
    if (o->n_reg > 0 && o->lambda[0] > 0)
        return internal_fail(GX_EUNSUPPORTED, "gx_askadam_noalloc: regularisation (TV or prior) needs gx_askadam");
    if (o->path != GX_PATH_FUSED) return internal_fail(GX_EUNSUPPORTED, "gx_askadam_noalloc: fused path only");
    if (o->robust_convergence)
        return internal_fail(GX_EUNSUPPORTED, "gx_askadam_noalloc: robustConvergence runs on gx_askadam's "
                                              "op-by-op path; this entry point has the fused path only");
    if (internal_can_stop(o))
        return internal_fail(GX_EUNSUPPORTED, "gx_askadam_noalloc: runs every iteration; disable the stopping "
                                              "criteria (tol, patienceConvergence, step/grad tolerances)");
    DevProtocol P;
    int np = 0, nm = 0, id = 0;
    gx_status st = internal_model(model, o->lb, o->ub, &P, &np, &nm, &id);
    if (st != GX_OK) return st;
    st = internal_validate_opts(o, np);  // iteration, bounds, loss / optimiser / transform kinds
    if (st != GX_OK) return st;
    if (o->loss == GX_LOSS_GAUSS_LOGP || o->loss == GX_LOSS_RICIAN_LOGP)
        if (!(o->sigma > 0)) return internal_fail(GX_EINVAL, "gx_askadam_noalloc: likelihood loss needs sigma > 0");
    const int B = o->block_size > 0 ? o->block_size : 128;
    if (B % 32 || B > 1024) return internal_fail(GX_EINVAL, "gx_askadam_noalloc: bad block_size");
    const int N = o->iteration;

    // layout of the fixed working memory
    const Layout Lo = layout((size_t)nvox, B, nm, np, N);
    const size_t nvtot = Lo.nvtot, nblocks = Lo.nblocks;
    const size_t off_vol = Lo.vol, off_blk = Lo.blk, off_sched = Lo.sched, off_hist = Lo.hist;
    const size_t off_data = Lo.data, off_th = Lo.th, off_z = Lo.z, off_m1 = Lo.m1, off_m2 = Lo.m2;
    if (Lo.total > kScratchBytes) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "gx_askadam_noalloc: %d voxels x %d iterations need %zu bytes of working memory; the fixed "
                 "array holds %zu (at most %zu voxels at this iteration count)",
                 nvox, N, Lo.total, kScratchBytes, max_voxels(B, nm, np, N));
        return internal_fail(GX_EINVAL, msg);
    }
    unsigned char* base = nullptr;
    st = scratch_address(&base);
    if (st != GX_OK) return st;
    cudaStream_t s = (cudaStream_t)cuda_stream;

    DevVol vol;
    memset(&vol, 0, sizeof(vol));
    vol.off = 0;
    vol.nvox = nvox;
    vol.npad = (int)nvtot;
    vol.normd = 1.0 / ((double)nm * (double)nvox);
    vol.norm = (float)vol.normd;
    vol.dims[0] = nvox; vol.dims[1] = 1; vol.dims[2] = 1;
    NA_CK(cudaMemcpyAsync(base + off_vol, &vol, sizeof(vol), cudaMemcpyHostToDevice, s));
    NA_CK(cudaMemsetAsync(base + off_blk, 0, sizeof(int) * nblocks, s));
    // optimiser schedule, written through a small host buffer on the stack
    float2 chunk[256];
    for (int e0 = 0; e0 <= N; e0 += 256) {
        int n = (N + 1 - e0) < 256 ? (N + 1 - e0) : 256;
        for (int i = 0; i < n; ++i) {
            int e = e0 + i;
            chunk[i] = float2{0.f, 0.f};
            if (e >= 1) {
                double lr = o->initial_learn_rate / (1.0 + o->decay_rate * (e - 1));
                if (o->optimiser == GX_OPT_ADAM)
                    chunk[i] = float2{(float)(lr / (1.0 - std::pow(o->beta1, (double)e))),
                                      (float)(1.0 / (1.0 - std::pow(o->beta2, (double)e)))};
                else
                    chunk[i] = float2{(float)lr, 0.f};
            }
        }
        // a copy from pageable host memory has staged its source when the call
        // returns, so the stack buffer can be refilled at once
        NA_CK(cudaMemcpyAsync(base + off_sched + sizeof(float2) * e0, chunk, sizeof(float2) * n,
                              cudaMemcpyHostToDevice, s));
    }
    NA_CK(cudaMemsetAsync(base + off_hist, 0, sizeof(double) * ((size_t)N + 1) * kHistW, s));
    float* d_data = reinterpret_cast<float*>(base + off_data);
    float* d_th = reinterpret_cast<float*>(base + off_th);
    NA_CK(cudaMemsetAsync(d_data, 0, sizeof(float) * nm * nvtot, s));
    NA_CK(cudaMemsetAsync(d_th, 0, sizeof(float) * np * nvtot, s));
    NA_CK(cudaMemcpy2DAsync(d_data, sizeof(float) * nvtot, data, sizeof(float) * nvox, sizeof(float) * nvox, nm,
                            cudaMemcpyDeviceToDevice, s));
    NA_CK(cudaMemcpy2DAsync(d_th, sizeof(float) * nvtot, theta0, sizeof(float) * nvox, sizeof(float) * nvox, np,
                            cudaMemcpyDeviceToDevice, s));

    AdamParams a;
    memset(&a, 0, sizeof(a));
    a.P = P;
    a.nm = nm;
    a.np = np;
    a.nvtot = (int)nvtot;
    a.data = d_data;
    a.sigma_default = (float)o->sigma;
    a.z = reinterpret_cast<float*>(base + off_z);
    a.m1 = reinterpret_cast<float*>(base + off_m1);
    a.m2 = reinterpret_cast<float*>(base + off_m2);
    a.blk_vol = reinterpret_cast<const int*>(base + off_blk);
    a.vols = reinterpret_cast<const DevVol*>(base + off_vol);
    a.nvol = 1;
    a.niter = N;
    a.sched = reinterpret_cast<const float2*>(base + off_sched);
    a.optimiser = o->optimiser;
    a.transform = o->transform;
    a.beta1 = (float)o->beta1; a.beta2 = (float)o->beta2; a.eps = (float)o->epsilon;
    a.momentum = (float)o->momentum; a.rms_decay = (float)o->rms_decay; a.rms_eps = (float)o->rms_epsilon;
    a.mse_scale = (float)o->mse_scale;
    a.huber_delta = (float)o->huber_delta;
    a.hist = reinterpret_cast<double*>(base + off_hist);

    NA_CK(launch_init_state(a, d_th, o->randomness, o->seed, B, s));
    if (N == 0) NA_CK(launch_fused(a, id, o->loss, false, 0, 0, -1, true, B, (int)nblocks, s));
    else NA_CK(launch_fused(a, id, o->loss, false, 1, N, N - 1, true, B, (int)nblocks, s));
    NA_CK(launch_finalize(a, a.z, d_th, nullptr, nullptr, B, (int)nblocks, s));
    NA_CK(cudaMemcpy2DAsync(theta_out, sizeof(float) * nvox, d_th, sizeof(float) * nvtot, sizeof(float) * nvox, np,
                            cudaMemcpyDeviceToDevice, s));
    double h[kHistW];
    NA_CK(cudaMemcpyAsync(h, base + off_hist + sizeof(double) * (size_t)N * kHistW, sizeof(h),
                          cudaMemcpyDeviceToHost, s));
    NA_CK(cudaStreamSynchronize(s));
    if (final_loss) *final_loss = h[0] + h[1];
    return GX_OK;
}
