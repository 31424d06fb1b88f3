// gx_internal.h -- declarations shared between the kernel translation units
// and the host runtime (capi.cu).  Not part of the public C-ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gx_device.cuh"

namespace gx {

constexpr int kHistW = 5;  // per-epoch record: fidelity, reg, |g|^2, |z|^2, |dz|^2
constexpr int kMaxReg = 8;

// Per-volume entry of the voxel work-list.  Volumes are concatenated in the
// SoA arrays, each padded to a multiple of the block size so that a block
// never straddles two volumes.
struct DevVol {
    int off;            // first (padded) voxel index of the volume
    int nvox;           // real voxels
    int npad;           // padded voxels
    float norm;         // 1 / (nm * nvox): askadam mean (utils/askadam.m:96)
    double normd;
    int dims[3];        // TV grid
    long long grid_off; // offset of the volume's grid in the TV grid buffers
    long long hgrid_off; // offset of the volume's haloed map in the persistent kernel's map buffers
    float tv_scale[kMaxReg];  // lambda_k / Nmask (spatial_total_variation.m:40; also the prior's)
    float prior_off;    // prior regulariser loss of the grid points outside the mask
};

// Parameters shared by the askAdam kernels (passed by value).
struct AdamParams {
    DevProtocol P;
    int nm, np, nvtot;            // nvtot: padded voxel count, array stride
    const float* data;            // [nm][nvtot]
    const float* weights;         // [nm][nvtot] or nullptr
    const float* b1;              // [nvtot] or nullptr
    const float* sigma;           // [nvtot] or nullptr
    float sigma_default;
    float* z; float* m1; float* m2; float* zprev;  // [np][nvtot]
    const int* blk_vol;           // block -> volume
    const DevVol* vols;
    int nvol;
    int niter;
    const float2* sched;          // [niter+1]: (lr_e/(1-b1^e), 1/(1-b2^e)) or (lr_e, 0)
    int optimiser, transform;
    float beta1, beta2, eps, momentum, rms_decay, rms_eps;
    float mse_scale, huber_delta;
    double* hist;                 // [nvol][niter+1][kHistW] or nullptr
    float* ckpt;                  // checkpoint slots, each 3*np*nvtot floats
    int ckpt_every;
    float* res_out;               // [nm][nvtot] or nullptr
    // TV
    int n_reg;
    int reg_param[kMaxReg];
    int tv_3d;
    float inv_vs[3];
    const int* gidx;              // [nvtot] grid index within the volume's grid
    const unsigned char* maskgrid;
    const float* grid_cur;        // [n_reg][grid total]
    float* grid_next;
    long long grid_total;
    // prior-distribution regulariser (instead of TV): [n_reg][nvtot], or nullptr
    const float* prior_mu;
    const float* prior_sd;
    // surface TV (instead of the grid stencil): [surf_maxnb][nvtot] neighbour
    // grid indices and edge lengths, or nullptr
    const int* surf_nb;
    const float* surf_len;
    int surf_maxnb;
};

// Kernel launchers (askadam_kernels.cu).  Return cudaError_t of the launch.
cudaError_t launch_init_state(const AdamParams& a, const float* theta0, double randomness,
                              uint64_t seed, int block, cudaStream_t s);
cudaError_t launch_fused(const AdamParams& a, int model, int loss, bool stats, int e_begin,
                         int e_end, int update_last, bool record, int block, int nblocks,
                         cudaStream_t s);
// Largest launch block (multiple of 32) the fused kernel variant of this job
// accepts: its thread limit and its per-block shared memory; 0 on error.
int fused_block_limit(const AdamParams& a, int model, int loss, bool stats);
cudaError_t launch_tv_step(const AdamParams& a, int model, int loss, bool stats, int e,
                           bool update, bool record, bool want_res, int block, int nblocks,
                           cudaStream_t s);
cudaError_t launch_tv_mask(const AdamParams& a, unsigned char* mask, int* err, int* bad_vol, int block,
                           int nblocks, cudaStream_t s);
cudaError_t launch_tv_scatter(const AdamParams& a, float* grid, int block, int nblocks,
                              cudaStream_t s);
cudaError_t launch_finalize(const AdamParams& a, const float* zsrc, float* theta_out,
                            const float* res, float* resloss, int block, int nblocks,
                            cudaStream_t s);
cudaError_t launch_copy_state(const AdamParams& a, float* dst, const float* z_, const float* m1_,
                              const float* m2_, bool to_ckpt, int block, int nblocks,
                              cudaStream_t s);

// Plain (unfused) path: one kernel per reference operation.
// robustConvergence state of the op-by-op path (utils/askadam.m:221-241,
// 448-510); all arrays [nvtot] unless noted, NULL when the option is off.
struct RobustStat {
    int n_le_a, n_le_b, n_nan;          // counts of improvements <= the population thresholds
    unsigned int max_le_a, min_gt_a;    // order-preserving bits of the neighbours of each threshold
    unsigned int max_le_b, min_gt_b;
    int differs;                        // main mask differs from the convergence mask
};
struct RobustBufs {
    float* vmod = nullptr;               // weight modulator (1 or outlierWeight)
    float* vloss = nullptr;              // per-voxel mean residual of the current evaluation
    float* vinit = nullptr;              // ... of the starting point (perVoxelLossInit)
    float* ring = nullptr;               // [window][nvtot] loss history of the last checks
    float* imp_a = nullptr;              // improvement over the history window
    float* imp_b = nullptr;              // improvement since the start
    int* flagcnt = nullptr;              // outlierFlagCount
    unsigned char* mainmask = nullptr;   // unflagged voxels
    unsigned char* convmask = nullptr;   // voxel set of the convergence signal (mainMask_conv)
    RobustStat* stat = nullptr;
};

struct PlainBufs {
    float* theta;    // [np][nvtot]
    float* dth;      // [np][nvtot] dtheta/dz
    float* signal;   // [nm][nvtot]
    float* dsig;     // [nm][nvtot] d loss / d signal (normalised)
    float* res;      // [nm][nvtot]
    float* gth;      // [np][nvtot]
    float* gz;       // [np][nvtot]
    double* acc;     // [8] per-iteration sums; robustConvergence uses [5..7]
    RobustBufs r;
};
cudaError_t launch_plain_unscale(const AdamParams& a, const PlainBufs& b, int block, int nblocks, cudaStream_t s);
cudaError_t launch_plain_forward(const AdamParams& a, int model, const PlainBufs& b, int block,
                                 int nblocks, cudaStream_t s);
cudaError_t launch_plain_loss(const AdamParams& a, int loss, const PlainBufs& b, int block,
                              int nblocks, cudaStream_t s);
cudaError_t launch_plain_adjoint(const AdamParams& a, int model, const PlainBufs& b, int block,
                                 int nblocks, cudaStream_t s);
cudaError_t launch_plain_tv(const AdamParams& a, const PlainBufs& b, float* grid, int block,
                            int nblocks, cudaStream_t s);
cudaError_t launch_plain_prior(const AdamParams& a, const PlainBufs& b, int block, int nblocks, cudaStream_t s);
cudaError_t launch_plain_zgrad(const AdamParams& a, const PlainBufs& b, bool stats, int block,
                               int nblocks, cudaStream_t s);
cudaError_t launch_plain_update(const AdamParams& a, const PlainBufs& b, int e, int block,
                                int nblocks, cudaStream_t s);
// robustConvergence on the op-by-op path (one volume view per call).
struct RobustOpts {
    float outlier_weight, voxel_thres, pop_thres, init_thres, init_pop_thres;
};
cudaError_t launch_robust_reset(const AdamParams& a, const PlainBufs& b, int block, int nblocks, cudaStream_t s);
cudaError_t launch_robust_seed(const AdamParams& a, const PlainBufs& b, int window, int block, int nblocks,
                               cudaStream_t s);
cudaError_t launch_robust_check(const AdamParams& a, const PlainBufs& b, int slot, int oldest,
                                const RobustOpts& ro, int nvox, int block, int nblocks, cudaStream_t s);
cudaError_t launch_robust_window(const AdamParams& a, const PlainBufs& b, int block, int nblocks, cudaStream_t s);
cudaError_t launch_robust_conv(const AdamParams& a, const PlainBufs& b, int block, int nblocks, cudaStream_t s);

// Dictionary matching (dictionary.cu): invE, Cj are [ndict] double scratch.
size_t dict_match_smem(int nm, bool weighted);
cudaError_t launch_dictionary_match(const float* signals, int nvox, const float* dict, int ndict, int nm,
                                    const float* wt, double* invE, double* Cj, int* best, float* best_sse,
                                    cudaStream_t s);

// Forward only (gx_forward).
cudaError_t launch_forward_only(const DevProtocol& P, int model, const float* theta,
                                const float* b1, int nvox, float* signal, cudaStream_t s);

// MCMC (mcmc_kernels.cu).
struct McmcParams {
    DevProtocol P;
    int nm, nvar, nvox;
    const float* data;     // [nm][nvox]
    const float* weights;  // [nm][nvox] or nullptr
    const float* b1;
    const float* x0;       // [nvar][nvox]
    float lb[kMaxParam], ub[kMaxParam], xstep[kMaxParam];
    int algorithm, nwalker, iteration, thinning, nburnin, ns, repetition, update;
    float a;               // stretch scale
    float start_range;
    uint64_t seed;
    const int* partner;    // simultaneous: [rep][iteration][W]; redblack: [rep][iteration][W]
    double* sum;           // [nvar][nvox] shifted sums
    double* sumsq;
    float* shift;          // [nvar][nvox]
    float* posterior;      // [nvar][rep][ns][W][nvox] or nullptr
    unsigned long long* n_acc;
    // goodman_weare_wglobal_constant (ng > 0): parameters shared by all voxels
    int is_global[kMaxParam];
    int ng, nnd, global_warmup;
    int nsteps_g;          // rows per repetition of gpartner: iteration + global_warmup
    float* gstate;         // [nvar][W] current global values (global rows used)
    int* gacc;             // [W] last global block's decision
    double* lpg;           // [nvox][W] logP at the global proposal
    double* partial;       // [W][nblocks] per-CTA sums of logP(proposal) - logP(current)
    double* gsum;          // [nvar][W] kept global samples, shifted
    double* gsumsq;
    const int* gpartner;   // [rep][nsteps_g][W] global-block anchors
    float* gprop;          // [nvar][W] global proposal of the current block
    float* gzz;            // [W] its stretch factor
    float* glu;            // [W] log of its acceptance uniform
    int* goob;             // [W] proposal outside the bounds
    unsigned long long* n_gacc;
};
cudaError_t launch_mcmc_partners(const McmcParams& p, int* partner, cudaStream_t s);
// goodman_weare_wglobal_constant launch shape: voxels per CTA, threads, CTAs
// (= rows of the partial-sum table) and dynamic shared memory.
void gwg_launch_shape(const McmcParams& p, int block_hint, int* vpb, int* block, int* nblocks, size_t* smem);
cudaError_t launch_mcmc(const McmcParams& p, int model, int block, cudaStream_t s);
// Launch shapes the MCMC autotuner tries (threads per block), and one trial
// launch of steps 1..k1 from the start into scratch state and sums.
int mcmc_block_candidates(const McmcParams& p, int* out, int maxn);
cudaError_t launch_mcmc_trial(const McmcParams& p, int model, int block_hint, int k1, float* xstate,
                              double* lpstate, double* sum, double* sumsq, cudaStream_t s);
cudaError_t launch_mcmc_finalize(const McmcParams& p, float* mean, float* stdv, cudaStream_t s);
// Kept slots the reference preallocates but never fills: numel(Nburnin+1:thinning:iteration)
// minus the steps k with mod(k - Nburnin + 1, thinning) == 0.
int mcmc_missing_slots(const McmcParams& p);
// Posterior median / iqr / mode (posterior_stats.cu) of post [nvar][N][nvox],
// N = rep * ns * W; lbub [nvar][2] (lb, ub) on the device; outputs
// [nvar][nvox] or nullptr.
cudaError_t launch_posterior_stats(const float* post, int nvar, int nvox, int N, int nbin, const double* lbub,
                                   float* median, float* iqr, float* mode, cudaStream_t s);

extern long long g_kernel_launches;  // launches of this library's kernels (process-wide)

// Persistent cooperative TV kernel (askadam_persistent.cu).
constexpr int kPersistMaxThreads = 1024;
// default bound of the persistent kernel's waits: about 2 s at B200 clocks
constexpr long long kBarrierSpinCycles = 4000000000LL;

struct PersistBarrier {
    unsigned int count;  // CTA arrivals since the launch (zeroed before it)
    int error;           // a bounded wait expired
    int pad[2];
};

struct PersistArgs {
    int e_begin, e_end, update_last;
    int record, want_res, stats, loss;
    // TV maps of the persistent kernel (input of even / odd epochs): per
    // volume (dx+2) x (dy+2) x (dz+2) with a one-cell halo on every face that
    // holds the periodic neighbour's value, so that every neighbour load has
    // a fixed offset; [n_reg][hgrid_total], zero outside the mask
    float* grid0;
    float* grid1;
    long long hgrid_total;
    int hlayout;             // L = 7, 8, 9: strides 2^L, 2^2L; 0: (dx+2), (dx+2)(dy+2) per volume
    PersistBarrier* barrier; // zeroed before the launch
    int slice;               // voxels per CTA
    int data_in_smem;
    int pad_block;           // block size of the work-list padding (blk_vol granularity)
    const float4* data_quads; // echo quads of the measurements (launch_echo_quads layout), or nullptr
    long long spin_cycles;   // bound of every wait, SM clock cycles (kBarrierSpinCycles unless a test sets it)
    unsigned int extra_arrivals; // 0; a test's count of arrivals the grid barrier waits for beyond the grid's
    PairConsts k;            // constants of the two-voxel variant (filled by launch_tv_persistent)
};

struct PersistPlan {
    int slice, vpt, threads, ctas, data_in_smem;
    int quad_width;          // > 0: the launch reads echo quads, this many measurements wide
    int quad_pairs;          // the quads are pair quads (two voxels per thread)
    size_t smem;
};

bool plan_persistent(const AdamParams& a, int model, int loss, bool stats, int pad_block, const int* vol_npad,
                     int nvol, PersistPlan* plan);
cudaError_t launch_tv_persistent(const AdamParams& a, const PersistPlan& plan, PersistArgs p, cudaStream_t s);
// Echo quads out[j][v] = (data[4j][v], .., data[4j+3][v]), or with pairs
// (voxels u0 = 64 (u / 32) + u % 32 and u0 + 32) quad j of pair u =
// (data[2j][u0], data[2j][u0+32], data[2j+1][u0], data[2j+1][u0+32]) at
// out[((u / 32) (width / 2) + j) 32 + u % 32]; 0 for nm <= m < width
// (width % 4 == 0; nvtot even, with pairs a multiple of 64)
cudaError_t launch_echo_quads(const float* data, int nm, int nvtot, int width, bool pairs, float4* out,
                              cudaStream_t s);

}  // namespace gx

// Helpers defined in capi.cu for the other translation units.
#include "../../include/gacelle_b200.h"
namespace gx {
gx_status internal_fail(gx_status s, const char* msg);
gx_status internal_model(const gx_model* m, const double* lb, const double* ub, DevProtocol* P,
                         int* np, int* nm, int* id);
bool internal_can_stop(const gx_askadam_opts* o);
// iteration count, bounds and the loss / optimiser / transform enumerations
gx_status internal_validate_opts(const gx_askadam_opts* o, int np);

}  // namespace gx
