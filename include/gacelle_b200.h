/*
 * gacelle_b200.h -- C-ABI of libgacelle_b200.so, the B200 (sm_100a) engine
 * for GACELLE's voxel-parallel solvers askAdam and MCMC.
 *
 * The entry points replace the MATLAB calls that the reference's built-in
 * model classes make (kschan0214/gacelle, paths relative to its root):
 *
 *   gx_askadam  <- askadam().optimisation(data, mask, weights, pars0, fitting,
 *                                         @model.FWD, ...)      utils/askadam.m:121-365
 *                  dispatched from R2star/gpuR2starMapping.m:237,
 *                  R1R2s/gpuJointR1R2starMapping.m:272, NEXI/gpuNEXI.m:435
 *   gx_mcmc     <- mcmc().optimisation(data, mask, weights, pars0, fitting,
 *                                      @model.FWD, ...)         utils/mcmc.m:18-80
 *                  (metropolis_hastings :82-190, goodman_weare :192-383)
 *                  dispatched from R2star/gpuR2starMapping.m:243,
 *                  R1R2s/gpuJointR1R2starMapping.m:279, NEXI/gpuNEXI.m:440
 *   gx_forward  <- model.FWD(pars, ...)  R2star/gpuR2starMapping.m:321-363,
 *                  R1R2s/gpuJointR1R2starMapping.m:375-422, NEXI/gpuNEXI.m:902-930
 *   gx_model_gradient <- askadam.model_gradient (utils/askadam.m:23-117), one
 *                  evaluation of loss and its gradient (dlfeval/dlgradient).
 *
 * Conventions
 *  - Plain C types only; no CUDA or C++ types cross the boundary.
 *  - Arrays are structure-of-arrays, voxel fastest: element (k, v) of a
 *    [K][nvox] array lives at index k*nvox + v.  This is MATLAB's
 *    [Nvox, K] column-major layout, i.e. utils.vectorise_NDto2D output
 *    before the transpose in utils.reshape_ND2GD (utils/utils.m:157-238).
 *  - mem == GX_MEM_HOST: every array pointer in the call (inputs and
 *    outputs) is host memory; the engine stages copies itself.
 *    mem == GX_MEM_DEVICE: every array pointer is device memory of the
 *    context's device (scalars in result structs are still written to the
 *    host struct).
 *  - Every call returns a gx_status; on failure gx_last_error() holds a
 *    thread-local message.  Calls on one context are serialised; calls are
 *    synchronous at return, like the reference's blocking optimisation().
 *  - There is no CPU fallback: without a usable CUDA device every compute
 *    entry point returns GX_ECUDA.
 */
#ifndef GACELLE_B200_H
#define GACELLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GX_ABI_VERSION 6

typedef enum {
    GX_OK = 0,
    GX_EINVAL = 1,       /* bad argument, shape or option */
    GX_ENOMEM = 2,       /* device or pinned-host allocation failed */
    GX_ECUDA = 3,        /* CUDA runtime error or no device */
    GX_EUNSUPPORTED = 4, /* option the engine does not implement */
    GX_ETIMEOUT = 5,     /* a bounded device wait expired */
    GX_ENUMERIC = 6,     /* non-finite loss; partial result returned */
    GX_ECANCELLED = 7    /* host cancel flag was set */
} gx_status;

/* Built-in forward models (the reference's model classes). */
typedef enum {
    GX_MODEL_R2S = 1,   /* gpuR2starMapping: M0, R2star */
    GX_MODEL_R1R2S = 2, /* gpuJointR1R2starMapping: M0, R1, R2star */
    GX_MODEL_NEXI = 3,  /* gpuNEXI: fa, Da, De, ra [, p2 if lmax = 2] */
    GX_MODEL_NEXI_RICE = 4 /* gpuNEXIrice: fa, Da, De, ra; lmax 0; Rician mean of the NEXI
                            * signal for the per-voxel noise sigma (gx_volume.sigma, or
                            * gx_askadam_opts.sigma; gx_forward's aux map) */
} gx_model_kind;

typedef enum {
    GX_LOSS_L1 = 0,          /* w*|s-y|            (l1loss)        */
    GX_LOSS_L2 = 1,          /* w*(s-y)^2          (l2loss)        */
    GX_LOSS_HUBER = 2,       /* huber, transition point huber_delta */
    GX_LOSS_MSE = 3,         /* mse_scale*(s-y)^2, weights ignored */
    GX_LOSS_GAUSS_LOGP = 4,  /* Gaussian negative log-likelihood   */
    GX_LOSS_RICIAN_LOGP = 5  /* Rician negative log-likelihood     */
} gx_loss;

typedef enum { GX_OPT_ADAM = 0, GX_OPT_SGDM = 1, GX_OPT_RMSPROP = 2 } gx_optimiser;
typedef enum { GX_TRANSFORM_SIGMOID = 0, GX_TRANSFORM_LINEAR = 1 } gx_transform;
typedef enum { GX_CONV_EMA = 0, GX_CONV_LINEAR = 1 } gx_conv_model;
typedef enum { GX_PATH_FUSED = 0, GX_PATH_PLAIN = 1 } gx_path;
typedef enum {
    GX_STOP_NONE = 0, GX_STOP_CONVERGENCE = 1, GX_STOP_TOL = 2, GX_STOP_STEP = 3,
    GX_STOP_GRAD = 4
} gx_stop_reason;
typedef enum { GX_MCMC_MH = 0, GX_MCMC_ENSEMBLE = 1 } gx_mcmc_algorithm;
typedef enum { GX_GW_SIMULTANEOUS = 0, GX_GW_REDBLACK = 1 } gx_gw_update;
typedef enum { GX_MEM_HOST = 0, GX_MEM_DEVICE = 1 } gx_memory;
/* The regulariser of the lambda / regmap entries: the spatial TV of
 * utils/spatial_total_variation.m; gpuNEXI.prior_distribution_normal
 * (NEXI/gpuNEXI.m:1256-1307, fitting.regularisationType 'prior'); or
 * gpuNEXI.surface_total_variation (NEXI/gpuNEXI.m:1165-1254, fitting.dataType
 * 'surface' with TV) over the mesh neighbours in gx_volume. */
typedef enum { GX_REG_TV = 0, GX_REG_PRIOR = 1, GX_REG_SURFACE_TV = 2 } gx_reg_type;

typedef struct gx_context gx_context;

/* Model and acquisition protocol (constructor arguments of the model class). */
typedef struct {
    int32_t kind;               /* gx_model_kind */
    int32_t lmax;               /* NEXI: 0 or 2 */
    int32_t nx;                 /* NEXI: powder-average trapezoid nodes (14 = reference) */
    int32_t n_te;               /* R2*, R1R2*: echo times [s] */
    const double* te;
    int32_t n_fa;               /* R1R2*: nominal flip angles [deg] */
    const double* fa_deg;
    double tr;                  /* R1R2*: repetition time [s] */
    int32_t n_shell;            /* NEXI: b-values [ms/um^2] and Delta [ms] per shell */
    const double* bval;
    const double* big_delta;
} gx_model;

/* One masked volume.  nmeas/nparam follow from the model (gx_model_sizes). */
typedef struct {
    int32_t dims[3];            /* grid size, x fastest (TV only; else {nvox,1,1}) */
    int32_t nvox;               /* masked voxels */
    const int32_t* grid_index;  /* [nvox] column-major linear grid index; NULL = 0..nvox-1 */
    const float* data;          /* [nmeas][nvox] */
    const float* weights;       /* [nmeas][nvox] or NULL (= 1) */
    const float* theta0;        /* [nparam][nvox] starting point, physical units, or NULL */
    const float* b1;            /* R1R2*: [nvox] B1 scaling of the flip angle, or NULL (= 1) */
    const float* sigma;         /* GAUSS/RICIAN loss: [nvox] noise sigma, or NULL (= opts sigma) */
    /* GX_REG_PRIOR: mean and SD of each regmap parameter, [n_reg][nvox] in
     * regmap order (required then, ignored otherwise).  The regulariser adds
     * lambda_r / nvox * |(theta - mu) / sd| over the voxels whose z-score is
     * finite, plus prior_offset: the part of the reference's loss from grid
     * points outside the mask, where the parameter image is 0 (a constant
     * with no gradient; 0 when the caller has no grid). */
    const float* prior_mu;
    const float* prior_sd;
    double prior_offset;
    /* GX_REG_SURFACE_TV: the vertices of the grid (dims, grid_index as for TV)
     * and, per voxel, its mesh neighbours as [max_neighbours][nvox] grid
     * indices with the edge lengths; a vertex with fewer neighbours repeats its
     * own index.  The regulariser adds lambda_r / nvox * sum |theta_v -
     * theta_nb| / length over the voxels' slots (theta = 0 off the mask,
     * non-finite quotients dropped); the adjacency must be symmetric with equal
     * lengths both ways, as a triangle mesh gives. */
    int32_t max_neighbours;
    const int32_t* neighbours;
    const float* edge_length;
} gx_volume;

/* askAdam options: the `fitting` struct after askadam.check_set_default_basic
 * (utils/askadam.m:735-878). */
typedef struct {
    int32_t iteration;
    double initial_learn_rate, decay_rate;
    int32_t optimiser;          /* gx_optimiser */
    double beta1, beta2, epsilon;          /* adamupdate */
    double momentum;                       /* sgdmupdate */
    double rms_decay, rms_epsilon;         /* rmspropupdate */
    int32_t loss;               /* gx_loss */
    double mse_scale;           /* 0.5: MATLAB mse is half mean squared error */
    double huber_delta;         /* 1 */
    double sigma;               /* noise sigma for GAUSS/RICIAN when volume sigma is NULL */
    int32_t transform;          /* gx_transform */
    double randomness;
    uint64_t seed;
    const double* lb;           /* [nparam] */
    const double* ub;           /* [nparam] */
    double tol, convergence_value;
    int32_t convergence_window;
    double patience_convergence; /* may be +Inf */
    int32_t convergence_model;  /* gx_conv_model */
    double ema_decay;
    double step_tol, grad_tol, patience_step, patience_grad;
    int32_t n_reg;              /* regularised parameters (TV or prior, per reg_type) */
    int32_t reg_param[8];       /* parameter index of each regmap entry */
    double lambda[8];
    int32_t tv_3d;              /* 0 = '2D', 1 = '3D' */
    double voxel_size[3];
    int32_t path;               /* gx_path */
    int32_t chunk;              /* fused path: iterations per launch if stopping may trigger; 0 = auto */
    /* threads per block; 0 = the default (128), or on the fused path without
     * TV the block chosen by the project's autotuner: the first call of a key
     * (model, loss, measurement count, variant, optimiser, transform, voxel-
     * count class) times 64 / 128 / 256 / 512 threads (and 32 for work-lists
     * of at most 64 x 148 voxels) on a few epochs of its own data and the
     * fastest is kept for the process; GACELLE_B200_AUTOTUNE=0
     * turns tuning off */
    int32_t block_size;
    /* robustConvergence (update_outlier_mask, utils/askadam.m:448-510, and the
     * main-population convergence signal of :530-581): every
     * weight_update_interval epochs, voxels that improve less than
     * outlier_voxel_thres over the last outlier_check_window checks and less
     * than outlier_init_thres since the start, while the population's median
     * improvements exceed outlier_pop_thres / outlier_init_pop_thres, are
     * flagged and their weights scaled by outlier_weight (the mse loss ignores
     * weights, as in the reference); convergence is judged on the mean loss of
     * the unflagged voxels.  The engine runs it on the op-by-op path, which
     * reads the loss back every epoch as the reference's loop does.
     * outlier_min_flag_duration is accepted and, as in the reference, unused. */
    int32_t robust_convergence;
    double outlier_weight;
    int32_t weight_update_interval, outlier_check_window, outlier_min_flag_duration;
    double outlier_voxel_thres, outlier_pop_thres, outlier_init_thres, outlier_init_pop_thres;
    int32_t reg_type;           /* gx_reg_type of the n_reg / reg_param / lambda entries */
} gx_askadam_opts;

/* Per-volume askAdam output (out.final / out.min of utils/askadam.m:345-362).
 * Array outputs are caller-allocated; any may be NULL except final_theta. */
typedef struct {
    float* final_theta;         /* [nparam][nvox] */
    float* min_theta;           /* [nparam][nvox] */
    float* final_residual;      /* [nmeas][nvox] elementwise loss */
    float* min_residual;
    float* final_resloss;       /* [nvox] mean residual per voxel */
    float* min_resloss;
    double* loss_history;       /* [iteration+1], host memory even for GX_MEM_DEVICE */
    double final_loss, final_loss_fidelity, final_loss_reg;
    double min_loss, min_loss_fidelity, min_loss_reg;
    int32_t final_niteration, min_niteration, stop_reason;
} gx_askadam_result;

/* MCMC options: the `fitting` struct after mcmc.check_set_default_basic
 * (utils/mcmc.m:633-679).  Parameters are the model's plus noise (last). */
typedef struct {
    int32_t algorithm;          /* gx_mcmc_algorithm */
    int32_t iteration, thinning;
    double burnin;              /* < 1: fraction of iteration; >= 1: count */
    int32_t repetition;
    int32_t nwalker;
    double step_size;           /* Goodman-Weare stretch scale a */
    double start_range;
    int32_t ensemble_update;    /* gx_gw_update */
    const double* x_step;       /* MH proposal step [nvar] */
    const double* lb;           /* [nvar] */
    const double* ub;           /* [nvar] */
    uint64_t seed;
    int32_t block_size;         /* threads per block (Goodman-Weare: a multiple of the walkers of one
                                 * update); 0 = chosen by the autotuner (MH and Goodman-Weare without
                                 * global parameters: trial steps per block shape, cached per key) */
    /* goodman_weare_wglobal_constant (utils/mcmc.m:385-626), chosen by the
     * reference when a start field has one value for all voxels: nonzero
     * entries mark parameters shared by all voxels of a volume (one value per
     * walker; their start is drawn uniformly over [lb, ub]).  Needs the
     * ensemble algorithm and at least one local and one global parameter.
     * NULL: every parameter is per voxel. */
    const int32_t* is_global;   /* [nvar] or NULL */
    int32_t global_warmup;      /* global-only iterations before the joint loop */
    int32_t nbin;               /* mode: edges linspace(lb - 1e-8, ub + 1e-8, nbin); 0 = 1001 */
} gx_mcmc_opts;

typedef struct {
    float* mean;                /* [nvar][nvox] posterior mean */
    float* std;                 /* [nvar][nvox] posterior standard deviation (N-1) */
    float* posterior;           /* [nvar][rep][ns][nwalker][nvox] or NULL */
    int64_t n_accepted, n_proposals;
    int32_t ns;                 /* kept samples per walker and repetition */
    /* global block of goodman_weare_wglobal_constant (walker moves); the
     * statistics and posterior of a global parameter repeat its value for
     * every voxel */
    int64_t n_global_accepted, n_global_proposals;
    /* res2out's order and histogram summaries (utils/mcmc.m:806-862), each
     * [nvar][nvox] or NULL, computed on the device from the kept samples (the
     * posterior need not be returned): median (mean of the two middle values
     * for an even count), iqr (prctile midpoint rule), mode (centre of the most
     * populated of the nbin - 1 bins, the lowest on ties; samples outside the
     * edges ignored, NaN when none is inside) */
    float* median;
    float* iqr;
    float* mode;
} gx_mcmc_result;

/* Device-side timing of the last compute call on a context (CUDA events on
 * the context's stream). */
typedef struct {
    double total_ms;            /* whole call, first to last device operation */
    double main_kernel_ms;      /* summed duration of the main (hot) kernel launches */
    int32_t main_launches;      /* number of main-kernel launches timed */
    int64_t kernel_launches;    /* launches of this library's kernels in the call */
    int64_t h2d_bytes, d2h_bytes;
    int32_t tv_path;            /* askAdam with TV: GX_TV_* flags of the main pass, else 0 */
    int32_t block_size;         /* threads per block of the main kernel's launches */
    int32_t autotuned;          /* 1: the autotuner ran its trials in this call (block_size 0,
                                 * first call of its key in the process) */
    double aux_kernel_ms;       /* summed duration of the post-processing kernels (MCMC: the
                                 * posterior median / iqr / mode) */
} gx_timing;

/* gx_timing.tv_path flags */
#define GX_TV_PERSISTENT 1      /* all epochs of a launch in one cooperative kernel */
#define GX_TV_PAIRS 2           /* two voxels per thread (FP32x2 pair instructions) */
#define GX_TV_DATA_SMEM 4       /* measurements staged in shared memory */
#define GX_TV_DATA_QUADS 8      /* measurements read from L2 as echo / pair quads */

const char* gx_version(void);
int32_t gx_abi_version(void);
const char* gx_last_error(void);
/* sizeof() of a public struct by name ("gx_model", "gx_volume", ...), for
 * binding checks; 0 for an unknown name. */
size_t gx_struct_size(const char* name);

gx_status gx_context_create(int32_t device, gx_context** out);
gx_status gx_context_destroy(gx_context* ctx);
/* Run the context's work on an external cudaStream_t.  NULL selects the
 * context's own non-blocking stream (the initial one); the CUDA default
 * streams are selected by their handles cudaStreamLegacy (0x1) and
 * cudaStreamPerThread (0x2). */
gx_status gx_context_set_stream(gx_context* ctx, void* cuda_stream);
gx_status gx_last_timing(gx_context* ctx, gx_timing* out);
/* Host-side cancel flag polled between launches; nonzero stops the call
 * with GX_ECANCELLED.  NULL clears it. */
gx_status gx_set_cancel_flag(gx_context* ctx, volatile int32_t* flag);

/* Fault injection for tests of the error paths (the reference's counterparts
 * are its error() identifiers and the out-of-memory catch of
 * utils/utils.m:698-706).  The settings hold for the context's following
 * calls until cleared (NULL or all zero). */
typedef struct {
    /* > 0: the n-th device workspace request of every following call fails as
     * an allocation failure would (GX_ENOMEM), without touching the device. */
    int32_t fail_alloc_at;
    /* > 0: bound, in SM clock cycles, of every wait in the persistent TV
     * kernel (default about 2 s). */
    int64_t wait_limit_cycles;
    /* > 0: the persistent kernel's grid barrier waits for this many arrivals
     * more than the grid makes, so its bounded wait runs out: every CTA then
     * returns and the call reports GX_ETIMEOUT, with the context usable. */
    int32_t barrier_extra_arrivals;
} gx_test_hooks;
gx_status gx_context_set_test_hooks(gx_context* ctx, const gx_test_hooks* hooks);

gx_status gx_model_sizes(const gx_model* model, int32_t* nparam, int32_t* nmeas);

/* model.FWD (R2star/gpuR2starMapping.m:321-363, R1R2s/gpuJointR1R2starMapping.m:375-422,
 * NEXI/gpuNEXI.m:902-930, NEXI/gpuNEXIrice.m:635-662).  aux [nvox]: b1 for
 * R1R2* (NULL: 1), the noise sigma for GX_MODEL_NEXI_RICE (required). */
gx_status gx_forward(gx_context* ctx, const gx_model* model, int32_t mem, const float* theta,
                     const float* aux, int32_t nvox, float* signal);

gx_status gx_model_gradient(gx_context* ctx, const gx_model* model, int32_t mem,
                            const gx_volume* vol, const gx_askadam_opts* opts,
                            const float* theta, float* gtheta, float* residual,
                            double* loss, double* loss_fidelity, double* loss_reg);

gx_status gx_askadam(gx_context* ctx, const gx_model* model, int32_t mem, const gx_volume* vols,
                     int32_t nvol, const gx_askadam_opts* opts, gx_askadam_result* results);

gx_status gx_mcmc(gx_context* ctx, const gx_model* model, int32_t mem, const gx_volume* vols,
                  int32_t nvol, const gx_mcmc_opts* opts, gx_mcmc_result* results);

/* Dictionary starting points (gpuNEXI.likelihood, NEXI/gpuNEXI.m:813-836,
 * called by estimate_prior :675-760 for start = 'likelihood'): for each voxel
 * the index of the first dictionary entry j minimising
 * sum_m wt_m (S0_m - c S_jm)^2 with c = (S0 . S_j) / (S_j . S_j).
 * signals [nm][nvox] and dict [nm][ndict] (voxel / entry fastest), wt [nm]
 * or NULL (ones); best [nvox] (-1 when no entry scores, e.g. all-zero
 * entries), best_sse [nvox] or NULL.  Host or device pointers per mem. */
gx_status gx_dictionary_match(gx_context* ctx, int32_t mem, const float* signals, int32_t nvox,
                              const float* dict, int32_t ndict, int32_t nm, const float* wt,
                              int32_t* best, float* best_sse);

/* No counterpart in the reference.  The fused askAdam fit of one volume
 * (final parameters only, every iteration run, no TV) for callers that cannot
 * allocate device memory while they run: applications whose framework owns
 * all device memory through its own allocator, or pipelines that reserve
 * their memory up front and must not allocate or hit out-of-memory later.
 * data [nmeas][nvox], theta0 [nparam][nvox] and theta_out [nparam][nvox] are
 * device pointers of the current device; the work is queued on cuda_stream
 * (NULL: the default stream) and finished at return; final_loss (host,
 * nullable) receives the last epoch's loss.  Working memory is a fixed 32 MiB
 * device array inside the library (held by every GPU that loads it until the
 * process exits); problems that do not fit are rejected with GX_EINVAL and the
 * maximum voxel count in gx_last_error().  The first call on a device looks up
 * that array's device address.  Calls share the array, so calls whose GPU
 * work overlaps race; stopping criteria must be disabled (GX_EUNSUPPORTED). */
gx_status gx_askadam_noalloc(const gx_model* model, const float* data, const float* theta0,
                             int32_t nvox, const gx_askadam_opts* opts, void* cuda_stream,
                             float* theta_out, double* final_loss);

#ifdef __cplusplus
}
#endif
#endif
