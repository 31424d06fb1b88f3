/*
 * oracle.h -- FP64 CPU restatement of GACELLE's askAdam / MCMC hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * engine (libgacelle_b200.so) and the timed CPU baseline in bench.py.  It is
 * never linked into, loaded by, or called from the product path.
 *
 * PARITY UNPINNED: the reference (kschan0214/gacelle) is MATLAB and relies on
 * closed MathWorks toolboxes (dlarray/dlgradient/adamupdate/mse, gpuArray,
 * arrayfun); it ships no tests, golden vectors or fixtures, and no MATLAB or
 * Octave exists on this machine or the GPU machine.  The restatement below is
 * pinned instead by (1) the reference source formulas cited per function,
 * (2) central finite differences and float64 autograd of the hand-written
 * adjoints, (3) the reference's own source-stated quadrature accuracies
 * (NEXI Nx=14 NRMSE < 0.05%, NEXI/gpuNEXI.m:950; Bessel Nx=34 NRMSE < 0.05%,
 * utils/gacelle_besseli.m:5), and (4) the Philox4x32-10 known-answer vectors
 * of Salmon et al. (SC'11).
 */
#ifndef GACELLE_ORACLE_H
#define GACELLE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_MODEL_R2S = 1, ORC_MODEL_R1R2S = 2, ORC_MODEL_NEXI = 3,
       ORC_MODEL_NEXI_RICE = 4 /* gpuNEXIrice: Rician mean of the lmax-0 NEXI signal */ };
enum { ORC_LOSS_L1 = 0, ORC_LOSS_L2 = 1, ORC_LOSS_HUBER = 2, ORC_LOSS_MSE = 3,
       ORC_LOSS_GAUSS = 4, ORC_LOSS_RICIAN = 5 };
enum { ORC_OPT_ADAM = 0, ORC_OPT_SGDM = 1, ORC_OPT_RMSPROP = 2 };
enum { ORC_TRANSFORM_SIGMOID = 0, ORC_TRANSFORM_LINEAR = 1 };
enum { ORC_CONV_EMA = 0, ORC_CONV_LINEAR = 1 };
enum { ORC_STOP_NONE = 0, ORC_STOP_CONVERGENCE = 1, ORC_STOP_TOL = 2,
       ORC_STOP_STEP = 3, ORC_STOP_GRAD = 4 };
enum { ORC_GW_SIMULTANEOUS = 0, ORC_GW_REDBLACK = 1 };

/* Acquisition protocol and model choice. */
typedef struct {
    int model;              /* ORC_MODEL_* */
    int lmax;               /* NEXI: 0 or 2 */
    int nx;                 /* NEXI: trapezoid nodes over x = cos(theta) in [0,1] */
    int n_te;               /* R2*, R1R2*: echo times [s] */
    const double* te;
    int n_fa;               /* R1R2*: nominal flip angles [deg] */
    const double* fa_deg;
    double tr;              /* R1R2*: repetition time [s] */
    int n_shell;            /* NEXI: b [ms/um^2] and Delta [ms] per shell */
    const double* bval;
    const double* delta;
} orc_model;

int orc_nparams(const orc_model* m);     /* askAdam parameter count (no noise) */
int orc_nmeas(const orc_model* m);

/* Single-voxel forward model, including the FWD-level post-processing of
 * the reference (NEXI min(S,1)).  theta[np] -> s[nm]. */
/* aux: per-voxel model input, b1 (R1R2*) or the noise sigma (NEXI Rician mean). */
void orc_forward_voxel(const orc_model* m, const double* theta, double b1, double* s);
/* Vector-Jacobian product of orc_forward_voxel: thetabar[np] += J^T sbar. */
void orc_vjp_voxel(const orc_model* m, const double* theta, double b1,
                   const double* sbar, double* thetabar);
/* Batched forward: theta [np][nvox], b1 [nvox] or NULL, s [nm][nvox]. */
void orc_forward(const orc_model* m, const double* theta, const double* b1,
                 int nvox, double* s);

/* Elementwise loss and its derivative with respect to the prediction s. */
double orc_loss_value(int loss, double s, double y, double w, double sigma,
                      double mse_scale, double huber_delta);
double orc_loss_deriv(int loss, double s, double y, double w, double sigma,
                      double mse_scale, double huber_delta);

/* Exponentially scaled modified Bessel functions of the first kind,
 * i0e(x) = exp(-|x|) I0(x), i1e(x) = exp(-|x|) I1(x). */
double orc_i0e(double x);
double orc_i1e(double x);
/* The reference's 34-node trapezoid Bessel integral (utils/gacelle_besseli.m:3-8). */
double orc_besseli_trapz(int nu, double z, int nx);

/* Philox4x32-10. */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double orc_u01(uint32_t x);

typedef struct {
    int iteration;
    double lr, decay;
    int optimiser;
    double beta1, beta2, eps, momentum, rms_decay, rms_eps;
    int loss;
    double mse_scale, huber_delta, sigma;
    int transform;
    double randomness;
    uint64_t seed;
    const double* lb;            /* [np] */
    const double* ub;            /* [np] */
    double tol, conv_value;
    int conv_window;
    double patience_conv;
    int conv_model;
    double ema_decay;
    double step_tol, grad_tol;
    double patience_step, patience_grad;
    int n_reg;
    int reg_param[8];
    double lambda[8];
    int tv_3d;
    double voxel_size[3];
    int nthreads;
    int state_f32;               /* round z, m, v to float after every update (FP32-storage emulation) */
    /* robustConvergence (utils/askadam.m:448-510, 530-581) */
    int robust;
    double outlier_weight;
    int weight_update_interval, outlier_check_window;
    double outlier_voxel_thres, outlier_pop_thres, outlier_init_thres, outlier_init_pop_thres;
    int reg_type;                /* 0: spatial TV; 1: prior_distribution_normal (NEXI/gpuNEXI.m:1256-1307);
                                  * 2: surface_total_variation (NEXI/gpuNEXI.m:1165-1254) */
} orc_adam_opts;

typedef struct {
    int dims[3];
    int nvox;
    const int* grid_index;       /* [nvox] column-major linear index, or NULL */
    const double* data;          /* [nm][nvox] voxel fastest */
    const double* weights;       /* [nm][nvox] or NULL */
    const double* theta0;        /* [np][nvox] or NULL */
    const double* b1;            /* [nvox] or NULL */
    const double* sigma;         /* [nvox] or NULL */
    double norm_nvox;            /* voxel count used by the mean; 0 -> nvox */
    const double* prior_mu;      /* [n_reg][nvox] prior mean (reg_type 1) */
    const double* prior_sd;      /* [n_reg][nvox] prior SD */
    double prior_offset;         /* prior loss of the grid points outside the mask */
    int max_neighbours;          /* reg_type 2 (surface TV): mesh neighbours per voxel */
    const int* neighbours;       /* [max_neighbours][nvox] grid indices */
    const double* edge_length;   /* [max_neighbours][nvox] */
} orc_volume;

typedef struct {
    double* final_theta;         /* [np][nvox] */
    double* min_theta;           /* [np][nvox] or NULL */
    double* final_residual;      /* [nm][nvox] or NULL */
    double* min_residual;        /* [nm][nvox] or NULL */
    double* loss_history;        /* [iteration+1] or NULL */
    double final_loss, final_fid, final_reg;
    double min_loss, min_fid, min_reg;
    int final_niter, min_niter, stop_reason;
    unsigned char* ever_flagged; /* [nvox] or NULL: robustConvergence flagged the voxel at some check */
} orc_adam_result;

int orc_askadam(const orc_model* m, const orc_volume* vol, const orc_adam_opts* o,
                orc_adam_result* r);

/* One evaluation of askadam.model_gradient at physical parameters theta:
 * returns loss, fidelity, reg; gtheta [np][nvox] gradient wrt theta. */
double orc_model_gradient(const orc_model* m, const orc_volume* vol, const orc_adam_opts* o,
                          const double* theta, double* gtheta, double* residual,
                          double* fid, double* reg);

typedef struct {
    int algorithm;               /* 0 MH, 1 ensemble (Goodman-Weare) */
    int iteration, thinning;
    double burnin;
    int repetition;
    int nwalker;
    double step_size;            /* GW stretch scale a */
    double start_range;
    int ensemble_update;         /* ORC_GW_* */
    const double* x_step;        /* MH proposal step [nvar] */
    const double* lb;            /* [nvar] */
    const double* ub;            /* [nvar] */
    uint64_t seed;
    int nthreads;
    const int* is_global;        /* [nvar] or NULL: nonzero = shared by all voxels
                                  * (goodman_weare_wglobal_constant) */
    int global_warmup;           /* global-only iterations before the joint loop */
} orc_mcmc_opts;

typedef struct {
    double* mean;                /* [nvar][nvox] */
    double* std;                 /* [nvar][nvox] */
    float* posterior;            /* [nvar][nvox][nwalker][ns][rep] or NULL */
    long long n_accepted, n_proposals;
    int ns;
} orc_mcmc_result;

/* nvar = orc_nparams + 1 (noise last).  x0 [nvar][nvox].  With is_global
 * set (ensemble only), mean/std/posterior of a global parameter hold its value
 * for every voxel; returns -2 when there is no local or no global parameter. */
int orc_mcmc(const orc_model* m, const orc_volume* vol, const double* x0,
             const orc_mcmc_opts* o, orc_mcmc_result* r);
int orc_mcmc_nsamples(int iteration, double burnin, int thinning);
/* Derangement shared by all voxels at GW step k (mcmc.m:797-803). */
void orc_gw_partner(uint64_t seed, int step, int rep, int nwalker, int* partner);

/* likelihood (NEXI/gpuNEXI.m:813-836): for each voxel i the first dictionary
 * entry j minimising sum_m wt_m (S0_im - c S_jm)^2, c = (S0_i . S_j) / (S_j . S_j).
 * signals [nm][nvox], dict [nm][ndict] (measurement-major), wt [nm] or NULL. */
void orc_dictionary_match(const double* signals, int nvox, const double* dict, int ndict, int nm,
                          const double* wt, int* best, double* best_sse);

/* 3-D anisotropic TV (utils/spatial_total_variation.m:24-66) on a full grid. */
double orc_tv_cost(const int dims[3], const unsigned char* mask, const double* img,
                   int tv_3d, const double vs[3]);
void orc_tv_grad(const int dims[3], const unsigned char* mask, const double* img,
                 int tv_3d, const double vs[3], double* grad);

#ifdef __cplusplus
}
#endif
#endif
