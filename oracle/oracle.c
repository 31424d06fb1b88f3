/*
 * oracle.c -- FP64 CPU restatement of GACELLE's askAdam / MCMC hot path.
 *
 * TEST INFRASTRUCTURE ONLY (checker and CPU baseline).  Never part of the
 * product path.  PARITY UNPINNED against MATLAB runs (no MATLAB exists here
 * and the reference ships no golden vectors); pinned by the source formulas
 * cited per function, finite differences, float64 autograd, the reference's
 * stated quadrature accuracies and the Philox known-answer vectors.
 *
 * All reference citations are paths inside kschan0214/gacelle.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EPS 1e-8 /* askadam.epsilon (utils/askadam.m:14), utils.epsilon */

/* ------------------------------------------------------------------------ */
/* Philox4x32-10, Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as  */
/* easy as 1, 2, 3", SC'11.                                                  */
/* ------------------------------------------------------------------------ */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Uniform on the open interval (0,1); 23 random bits so that the value is
 * exactly representable in FP32 (the device computes the same number). */
double orc_u01(uint32_t x) { return ((double)(x >> 9) + 0.5) * (1.0 / 8388608.0); }

static uint32_t rand_below(uint32_t x, uint32_t n) { return (uint32_t)(((uint64_t)x * n) >> 32); }

/* Random-stream tags (4th counter word, low byte). */
enum { TAG_ADAM_INIT = 1, TAG_GW_INIT = 2, TAG_GW_MOVE = 3, TAG_GW_PERM = 4,
       TAG_GW_RBPART = 5, TAG_MH_MOVE = 6, TAG_GW_GPERM = 7, TAG_GW_GRBPART = 8,
       TAG_GW_GMOVE = 9, TAG_GW_GINIT = 10 };
/* flag bits above the tag: red-black move (1<<8), global warm-up step (1<<9);
 * the repetition index sits in bits 16-31 */
#define TAG_RB (1u << 8)
#define TAG_WARM (1u << 9)

static void philox_call(uint64_t seed, uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                        uint32_t out[4]) {
    uint32_t ctr[4] = {a, b, c, d};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    orc_philox(ctr, key, out);
}

/* Box-Muller pair from two uniforms. */
static void box_muller(uint32_t a, uint32_t b, double* n0, double* n1) {
    double u1 = orc_u01(a), u2 = orc_u01(b);
    double r = sqrt(-2.0 * log(u1));
    double ang = 2.0 * M_PI * u2;
    *n0 = r * cos(ang);
    *n1 = r * sin(ang);
}

/* ------------------------------------------------------------------------ */
/* Models                                                                    */
/* ------------------------------------------------------------------------ */
int orc_nparams(const orc_model* m) {
    switch (m->model) {
    case ORC_MODEL_R2S: return 2;   /* M0, R2star   (R2star/gpuR2starMapping.m:24) */
    case ORC_MODEL_R1R2S: return 3; /* M0, R1, R2star (R1R2s/gpuJointR1R2starMapping.m:25) */
    case ORC_MODEL_NEXI: return m->lmax == 2 ? 5 : 4; /* fa, Da, De, ra[, p2] (NEXI/gpuNEXI.m:28,125-133) */
    case ORC_MODEL_NEXI_RICE: return 4;                /* fa, Da, De, ra (NEXI/gpuNEXIrice.m:15,74-84) */
    }
    return 0;
}

int orc_nmeas(const orc_model* m) {
    switch (m->model) {
    case ORC_MODEL_R2S: return m->n_te;
    case ORC_MODEL_R1R2S: return m->n_te * m->n_fa;
    case ORC_MODEL_NEXI: return m->n_shell * (m->lmax / 2 + 1);
    case ORC_MODEL_NEXI_RICE: return m->n_shell;
    }
    return 0;
}

/* S = M0 exp(-TE R2*)   (R2star/gpuR2starMapping.m:427-434) */
static void r2s_fwd(const orc_model* m, const double* th, double* s) {
    for (int t = 0; t < m->n_te; ++t) s[t] = th[0] * exp(-m->te[t] * th[1]);
}

static void r2s_vjp(const orc_model* m, const double* th, const double* sb, double* tb) {
    for (int t = 0; t < m->n_te; ++t) {
        double e = exp(-m->te[t] * th[1]);
        tb[0] += sb[t] * e;
        tb[1] += sb[t] * (-m->te[t] * th[0] * e);
    }
}

/* S = M0 sin(a)(1-E1)/(1-cos(a)E1) exp(-TE R2*), E1 = exp(-TR R1), a = b1*FA,
 * TE fastest then FA   (R1R2s/gpuJointR1R2starMapping.m:375-422,513-525) */
static void r1r2s_fwd(const orc_model* m, const double* th, double b1, double* s) {
    double M0 = th[0], R1 = th[1], R2 = th[2];
    double E1 = exp(-m->tr * R1);
    for (int f = 0; f < m->n_fa; ++f) {
        double a = b1 * m->fa_deg[f] * (M_PI / 180.0);
        double A = sin(a) * (1.0 - E1) / (1.0 - cos(a) * E1);
        for (int t = 0; t < m->n_te; ++t) s[t + f * m->n_te] = M0 * A * exp(-m->te[t] * R2);
    }
}

static void r1r2s_vjp(const orc_model* m, const double* th, double b1, const double* sb,
                      double* tb) {
    double M0 = th[0], R1 = th[1], R2 = th[2];
    double E1 = exp(-m->tr * R1);
    for (int f = 0; f < m->n_fa; ++f) {
        double a = b1 * m->fa_deg[f] * (M_PI / 180.0);
        double sa = sin(a), ca = cos(a);
        double den = 1.0 - ca * E1;
        double A = sa * (1.0 - E1) / den;
        double dA_dE1 = sa * (ca - 1.0) / (den * den);
        double dA_dR1 = dA_dE1 * (-m->tr * E1);
        for (int t = 0; t < m->n_te; ++t) {
            double g = sb[t + f * m->n_te];
            double E2 = exp(-m->te[t] * R2);
            tb[0] += g * A * E2;
            tb[1] += g * M0 * E2 * dA_dR1;
            tb[2] += g * (-m->te[t] * M0 * A * E2);
        }
    }
}

/* NEXI node value M(x) (NEXI/gpuNEXI.m:1090-1097) and its partials with
 * respect to (f, d1, d2, r1, r2). */
typedef struct { double M, df, dd1, dd2, dr1, dr2; } nexi_node;

static nexi_node nexi_node_eval(double f, double d1, double d2, double r1, double r2) {
    nexi_node n;
    double sdiff = r1 - r2 + d1 - d2;
    double Q = sdiff * sdiff + 4.0 * r1 * r2;
    double l2raw = sqrt(Q) / 2.0;
    int active = l2raw > ORC_EPS;
    double l2 = active ? l2raw : ORC_EPS;
    double l1 = (r1 + r2 + d1 + d2) / 2.0;
    double lm = l1 - l2, lp = l1 + l2;
    double N = f * d1 + (1.0 - f) * d2 - lm;
    double Pp = N / (l2 * 2.0);
    double ep = exp(-lp), em = exp(-lm);
    n.M = Pp * ep + (1.0 - Pp) * em;
    /* reverse sweep with Mbar = 1 */
    double Ppb = ep - em;
    double lpb = -Pp * ep;
    double lmb = -(1.0 - Pp) * em;
    double Nb = Ppb / (2.0 * l2);
    double l2b = -Ppb * Pp / l2;
    double fb = Nb * (d1 - d2);
    double d1b = Nb * f;
    double d2b = Nb * (1.0 - f);
    lmb += -Nb;
    double l1b = lpb + lmb;
    l2b += lpb - lmb;
    double r1b = 0.0, r2b = 0.0;
    if (active) {
        double Qb = l2b / (8.0 * l2raw);
        double sb = 2.0 * sdiff * Qb;
        r1b += 4.0 * r2 * Qb + sb;
        r2b += 4.0 * r1 * Qb - sb;
        d1b += sb;
        d2b -= sb;
    }
    r1b += 0.5 * l1b; r2b += 0.5 * l1b; d1b += 0.5 * l1b; d2b += 0.5 * l1b;
    n.df = fb; n.dd1 = d1b; n.dd2 = d2b; n.dr1 = r1b; n.dr2 = r2b;
    return n;
}

/* Trapezoid weights of utils/gacelle_trapz.m:53-56 on x = linspace(0,1,nx). */
static double trapz_w(int i, int nx) {
    double h = 1.0 / (nx - 1);
    return (i == 0 || i == nx - 1) ? 0.5 * h : h;
}

/* Per-shell raw (pre-min) signals: Sl0[j], and Sl2 integral T[j] when lmax=2
 * (NEXI/gpuNEXI.m:932-996). */
static void nexi_raw(const orc_model* m, const double* th, double* sl0, double* T2) {
    double fa = fmax(th[0], ORC_EPS), Da = th[1], De = th[2], ra = th[3];
    int nx = m->nx;
    for (int j = 0; j < m->n_shell; ++j) {
        double b = m->bval[j], D = m->delta[j];
        double Daj = b * Da, Dej = b * De, r1 = D * ra, r2 = r1 * fa / (1.0 - fa);
        double s0 = 0.0, s2 = 0.0;
        for (int i = 0; i < nx; ++i) {
            double x = (double)i / (nx - 1);
            nexi_node n = nexi_node_eval(fa, Daj * x * x, Dej, r1, r2);
            double w = trapz_w(i, nx);
            s0 += w * n.M;
            s2 += w * n.M * (3.0 * x * x - 1.0) / 2.0;
        }
        sl0[j] = s0;
        if (T2) T2[j] = s2;
    }
}

static void nexi_fwd(const orc_model* m, const double* th, double* s) {
    int ns = m->n_shell;
    double T2[256];
    nexi_raw(m, th, s, m->lmax == 2 ? T2 : NULL);
    if (m->lmax == 2)
        for (int j = 0; j < ns; ++j) s[ns + j] = th[4] * fabs(T2[j]);
    int nm = orc_nmeas(m);
    for (int k = 0; k < nm; ++k) s[k] = fmin(s[k], 1.0); /* NEXI/gpuNEXI.m:928 */
}

static void nexi_vjp(const orc_model* m, const double* th, const double* sb_in, double* tb) {
    int ns = m->n_shell, nx = m->nx;
    double sl0[256], T2[256], sb[512];
    nexi_raw(m, th, sl0, m->lmax == 2 ? T2 : NULL);
    for (int j = 0; j < ns; ++j) sb[j] = sl0[j] <= 1.0 ? sb_in[j] : 0.0;
    if (m->lmax == 2)
        for (int j = 0; j < ns; ++j) sb[ns + j] = th[4] * fabs(T2[j]) <= 1.0 ? sb_in[ns + j] : 0.0;
    double fa = fmax(th[0], ORC_EPS), Da = th[1], De = th[2], ra = th[3];
    double fb = 0, Dab = 0, Deb = 0, rab = 0;
    for (int j = 0; j < ns; ++j) {
        double b = m->bval[j], D = m->delta[j];
        double Dej = b * De, r1 = D * ra, r2 = r1 * fa / (1.0 - fa);
        double sgn2 = 0.0;
        if (m->lmax == 2) {
            tb[4] += sb[ns + j] * fabs(T2[j]);
            sgn2 = (T2[j] > 0) - (T2[j] < 0);
        }
        for (int i = 0; i < nx; ++i) {
            double x = (double)i / (nx - 1);
            double w = trapz_w(i, nx);
            double Mb = sb[j] * w;
            if (m->lmax == 2) Mb += sb[ns + j] * th[4] * sgn2 * w * (3.0 * x * x - 1.0) / 2.0;
            if (Mb == 0.0) continue;
            nexi_node n = nexi_node_eval(fa, b * Da * x * x, Dej, r1, r2);
            double r2_r1 = fa / (1.0 - fa);
            double r2_f = r1 / ((1.0 - fa) * (1.0 - fa));
            fb += Mb * (n.df + n.dr2 * r2_f);
            Dab += Mb * n.dd1 * b * x * x;
            Deb += Mb * n.dd2 * b;
            rab += Mb * (n.dr1 + n.dr2 * r2_r1) * D;
        }
    }
    if (th[0] > ORC_EPS) tb[0] += fb; /* fa = max(fa, eps), NEXI/gpuNEXI.m:905 */
    tb[1] += Dab;
    tb[2] += Deb;
    tb[3] += rab;
}

/* gpuNEXIrice.FWD (NEXI/gpuNEXIrice.m:635-662): Sl0 with fa = max(fa, eps)
 * and re = ra fa / max(1 - fa, eps) (:665-688), then the Rician mean
 * myriceM1 (:726-737), then min(s, 1). */
static void nexi_rice_raw(const orc_model* m, const double* th, double* sl0) {
    double fa = fmax(th[0], ORC_EPS), Da = th[1], De = th[2], ra = th[3];
    int nx = m->nx;
    for (int j = 0; j < m->n_shell; ++j) {
        double b = m->bval[j], D = m->delta[j];
        double r1 = D * ra, r2 = r1 * fa / fmax(1.0 - fa, ORC_EPS);
        double s0 = 0.0;
        for (int i = 0; i < nx; ++i) {
            double x = (double)i / (nx - 1);
            s0 += trapz_w(i, nx) * nexi_node_eval(fa, b * Da * x * x, b * De, r1, r2).M;
        }
        sl0[j] = s0;
    }
}

/* myL12 (NEXI/gpuNEXIrice.m:739-744) with mybesseli (:751-755):
 * L(x) = exp(x/2) ((1 - x) I0(-x/2) - x I1(-x/2)), x clamped at -170, the
 * I_nu as 34-node trapezoids of (1/pi) int_0^pi exp(z cos t) cos(nu t) dt.
 * dLdx differentiates that discretised function (what autodiff sees):
 * dL/dx = L/2 + exp(x/2) (-T0 - T1 - (1-x)/2 T1 + x/2 U1),  U1 = the
 * trapezoid of cos^2 t exp(z cos t) / pi, T_nu = the I_nu trapezoids. */
static double rice_L12(double xin, double* dLdx) {
    int clamped = xin < -170.0;
    double x = clamped ? -170.0 : xin;
    double z = -x / 2.0;
    double T0 = orc_besseli_trapz(0, z, 34), T1 = orc_besseli_trapz(1, z, 34);
    double h = M_PI / 33.0, U1 = 0.0;
    for (int i = 0; i < 34; ++i) {
        double t = i * h, w = (i == 0 || i == 33) ? 0.5 * h : h;
        U1 += w * cos(t) * cos(t) * exp(z * cos(t));
    }
    U1 /= M_PI;
    double e = exp(x / 2.0);
    double L = e * ((1.0 - x) * T0 - x * T1);
    if (dLdx) *dLdx = clamped ? 0.0 : 0.5 * L + e * (-T0 - T1 - 0.5 * (1.0 - x) * T1 + 0.5 * x * U1);
    return L;
}

/* M1 = max(sigma sqrt(pi/2) L12(-nu^2 / (2 sigma^2)), nu) and dM1/dnu. */
static double rice_M1(double nu, double sigma, double* dM1) {
    double dL;
    double x = -nu * nu / (2.0 * sigma * sigma);
    double M = sigma * sqrt(M_PI / 2.0) * rice_L12(x, &dL);
    if (M > nu) {
        *dM1 = sigma * sqrt(M_PI / 2.0) * dL * (-nu / (sigma * sigma));
        return M;
    }
    *dM1 = 1.0;
    return nu;
}

static void nexi_rice_fwd(const orc_model* m, const double* th, double sigma, double* s) {
    nexi_rice_raw(m, th, s);
    for (int j = 0; j < m->n_shell; ++j) {
        double d;
        s[j] = fmin(rice_M1(s[j], sigma, &d), 1.0);
    }
}

static void nexi_rice_vjp(const orc_model* m, const double* th, double sigma, const double* sb_in,
                          double* tb) {
    int ns = m->n_shell, nx = m->nx;
    double sl0[256], sb[256];
    nexi_rice_raw(m, th, sl0);
    for (int j = 0; j < ns; ++j) {
        double d, M1 = rice_M1(sl0[j], sigma, &d);
        sb[j] = M1 <= 1.0 ? sb_in[j] * d : 0.0;
    }
    double fa = fmax(th[0], ORC_EPS), Da = th[1], De = th[2], ra = th[3];
    double omf = fmax(1.0 - fa, ORC_EPS);
    /* d(fa / max(1-fa, eps)) / d fa */
    double rfd = 1.0 - fa > ORC_EPS ? 1.0 / ((1.0 - fa) * (1.0 - fa)) : 1.0 / ORC_EPS;
    double fb = 0, Dab = 0, Deb = 0, rab = 0;
    for (int j = 0; j < ns; ++j) {
        double b = m->bval[j], D = m->delta[j];
        double r1 = D * ra, r2 = r1 * fa / omf;
        for (int i = 0; i < nx; ++i) {
            double x = (double)i / (nx - 1);
            double Mb = sb[j] * trapz_w(i, nx);
            if (Mb == 0.0) continue;
            nexi_node n = nexi_node_eval(fa, b * Da * x * x, b * De, r1, r2);
            fb += Mb * (n.df + n.dr2 * r1 * rfd);
            Dab += Mb * n.dd1 * b * x * x;
            Deb += Mb * n.dd2 * b;
            rab += Mb * (n.dr1 + n.dr2 * fa / omf) * D;
        }
    }
    if (th[0] > ORC_EPS) tb[0] += fb;
    tb[1] += Dab;
    tb[2] += Deb;
    tb[3] += rab;
}

void orc_forward_voxel(const orc_model* m, const double* th, double b1, double* s) {
    switch (m->model) {
    case ORC_MODEL_R2S: r2s_fwd(m, th, s); break;
    case ORC_MODEL_R1R2S: r1r2s_fwd(m, th, b1, s); break;
    case ORC_MODEL_NEXI: nexi_fwd(m, th, s); break;
    case ORC_MODEL_NEXI_RICE: nexi_rice_fwd(m, th, b1, s); break;
    }
}

void orc_vjp_voxel(const orc_model* m, const double* th, double b1, const double* sb,
                   double* tb) {
    switch (m->model) {
    case ORC_MODEL_R2S: r2s_vjp(m, th, sb, tb); break;
    case ORC_MODEL_R1R2S: r1r2s_vjp(m, th, b1, sb, tb); break;
    case ORC_MODEL_NEXI: nexi_vjp(m, th, sb, tb); break;
    case ORC_MODEL_NEXI_RICE: nexi_rice_vjp(m, th, b1, sb, tb); break;
    }
}

void orc_forward(const orc_model* m, const double* theta, const double* b1, int nvox, double* s) {
    int np = orc_nparams(m), nm = orc_nmeas(m);
#pragma omp parallel for schedule(static)
    for (int v = 0; v < nvox; ++v) {
        double th[8], sv[512];
        for (int k = 0; k < np; ++k) th[k] = theta[(size_t)k * nvox + v];
        orc_forward_voxel(m, th, b1 ? b1[v] : 1.0, sv);
        for (int k = 0; k < nm; ++k) s[(size_t)k * nvox + v] = sv[k];
    }
}

/* ------------------------------------------------------------------------ */
/* Bessel functions (DLMF 10.25.2 power series; 10.40.1 asymptotic series)  */
/* ------------------------------------------------------------------------ */
static double bessel_scaled(int nu, double x) {
    double ax = fabs(x);
    double v;
    if (ax < 30.0) {
        double t = ax * ax / 4.0, term = (nu == 0) ? 1.0 : ax / 2.0, sum = 0.0;
        for (int k = 0; k < 500; ++k) {
            sum += term;
            term *= t / ((k + 1.0) * (k + 1.0 + nu));
            if (term < 1e-18 * sum) break;
        }
        v = sum * exp(-ax);
    } else {
        double mu = 4.0 * nu * nu, sum = 1.0, prod = 1.0;
        for (int k = 1; k < 40; ++k) {
            double f = (2.0 * k - 1.0);
            prod *= -(mu - f * f) / (k * 8.0 * ax);
            sum += prod;
            if (fabs(prod) < 1e-18) break;
        }
        v = sum / sqrt(2.0 * M_PI * ax);
    }
    if (nu == 1 && x < 0) v = -v;
    return v;
}

double orc_i0e(double x) { return bessel_scaled(0, x); }
double orc_i1e(double x) { return bessel_scaled(1, x); }

/* I_nu(z) = 1/pi * trapz(theta, exp(z cos theta) cos(nu theta)), theta in [0,pi]
 * (utils/gacelle_besseli.m:3-8). */
double orc_besseli_trapz(int nu, double z, int nx) {
    double h = M_PI / (nx - 1), s = 0.0;
    for (int i = 0; i < nx; ++i) {
        double th = i * h;
        double w = (i == 0 || i == nx - 1) ? 0.5 * h : h;
        s += w * exp(z * cos(th)) * cos(nu * th);
    }
    return s / M_PI;
}

/* ------------------------------------------------------------------------ */
/* Elementwise losses (utils/askadam.m:86-95; MATLAB l1loss/l2loss/huber/mse */
/* with Reduction="none"), plus Gaussian and Rician negative log-likelihoods */
/* ------------------------------------------------------------------------ */
static double sgn(double x) { return (x > 0) - (x < 0); }

double orc_loss_value(int loss, double s, double y, double w, double sigma, double mse_scale,
                      double hd) {
    double r = s - y;
    switch (loss) {
    case ORC_LOSS_L1: return w * fabs(r);
    case ORC_LOSS_L2: return w * r * r;
    case ORC_LOSS_HUBER: {
        double a = fabs(r);
        return w * (a <= hd ? 0.5 * r * r : hd * a - 0.5 * hd * hd);
    }
    case ORC_LOSS_MSE: return mse_scale * r * r; /* weights ignored, askadam.m:93-94 */
    case ORC_LOSS_GAUSS: {
        double s2 = sigma * sigma;
        return w * (r * r / (2.0 * s2) + 0.5 * log(2.0 * M_PI * s2));
    }
    case ORC_LOSS_RICIAN: {
        double s2 = sigma * sigma;
        double x = y * s / s2, ax = fabs(x);
        double logI0 = ax + log(orc_i0e(ax));
        double c = y > 0 ? -log(y / s2) : 0.0;
        return w * ((y * y + s * s) / (2.0 * s2) - logI0 + c);
    }
    }
    return 0.0;
}

double orc_loss_deriv(int loss, double s, double y, double w, double sigma, double mse_scale,
                      double hd) {
    double r = s - y;
    switch (loss) {
    case ORC_LOSS_L1: return w * sgn(r);
    case ORC_LOSS_L2: return 2.0 * w * r;
    case ORC_LOSS_HUBER: return fabs(r) <= hd ? w * r : w * hd * sgn(r);
    case ORC_LOSS_MSE: return 2.0 * mse_scale * r;
    case ORC_LOSS_GAUSS: return w * r / (sigma * sigma);
    case ORC_LOSS_RICIAN: {
        double s2 = sigma * sigma;
        double x = y * s / s2;
        double ratio = orc_i1e(x) / orc_i0e(x);
        return w * (s / s2 - (y / s2) * ratio);
    }
    }
    return 0.0;
}

/* ------------------------------------------------------------------------ */
/* Spatial TV (utils/spatial_total_variation.m:24-66): periodic forward     */
/* differences, mask applied at the centre voxel only.                      */
/* ------------------------------------------------------------------------ */
static size_t lin(const int d[3], int x, int y, int z) {
    return (size_t)x + (size_t)d[0] * ((size_t)y + (size_t)d[1] * z);
}

double orc_tv_cost(const int d[3], const unsigned char* mask, const double* img, int tv_3d,
                   const double vs[3]) {
    double cost = 0.0;
    int nd = tv_3d ? 3 : 2;
    for (int z = 0; z < d[2]; ++z)
        for (int y = 0; y < d[1]; ++y)
            for (int x = 0; x < d[0]; ++x) {
                size_t p = lin(d, x, y, z);
                if (!mask[p]) continue;
                double c = img[p];
                double nb[3] = {img[lin(d, (x + 1) % d[0], y, z)], img[lin(d, x, (y + 1) % d[1], z)],
                                img[lin(d, x, y, (z + 1) % d[2])]};
                for (int k = 0; k < nd; ++k) cost += fabs((nb[k] - c) / vs[k]);
            }
    return cost;
}

void orc_tv_grad(const int d[3], const unsigned char* mask, const double* img, int tv_3d,
                 const double vs[3], double* g) {
    int nd = tv_3d ? 3 : 2;
    for (int z = 0; z < d[2]; ++z)
        for (int y = 0; y < d[1]; ++y)
            for (int x = 0; x < d[0]; ++x) {
                size_t q = lin(d, x, y, z);
                double c = img[q], acc = 0.0;
                size_t fw[3] = {lin(d, (x + 1) % d[0], y, z), lin(d, x, (y + 1) % d[1], z),
                                lin(d, x, y, (z + 1) % d[2])};
                size_t bw[3] = {lin(d, (x + d[0] - 1) % d[0], y, z),
                                lin(d, x, (y + d[1] - 1) % d[1], z),
                                lin(d, x, y, (z + d[2] - 1) % d[2])};
                for (int k = 0; k < nd; ++k) {
                    if (mask[q]) acc -= sgn(img[fw[k]] - c) / vs[k];
                    if (mask[bw[k]]) acc += sgn(c - img[bw[k]]) / vs[k];
                }
                g[q] = acc;
            }
}

/* ------------------------------------------------------------------------ */
/* askAdam                                                                   */
/* ------------------------------------------------------------------------ */
static double sigmoid(double z) { return 1.0 / (1.0 + exp(-z)); }

/* unscale_parameters (utils/askadam.m:1063-1075) */
static double unscale(const orc_adam_opts* o, int k, double z) {
    if (o->transform == ORC_TRANSFORM_SIGMOID) return o->lb[k] + (o->ub[k] - o->lb[k]) * sigmoid(z);
    return z * (o->ub[k] - o->lb[k]) + o->lb[k];
}

static double dunscale(const orc_adam_opts* o, int k, double z) {
    if (o->transform == ORC_TRANSFORM_SIGMOID) {
        double s = sigmoid(z);
        return (o->ub[k] - o->lb[k]) * s * (1.0 - s);
    }
    return o->ub[k] - o->lb[k];
}

typedef struct {
    const orc_model* m;
    const orc_volume* vol;
    const orc_adam_opts* o;
    int np, nm, nv;
    double norm;           /* 1 / (nm * Nv) */
    unsigned char* mask;   /* full-grid mask for TV */
    double* grid;          /* full-grid image scratch */
    double* grid_g;
    size_t ngrid;
    const double* wmod;    /* [nv] robustConvergence weight modulator, or NULL */
    double* vloss;         /* [nv] per-voxel mean residual of the last evaluation, or NULL */
} adam_ctx;

/* askadam.model_gradient (utils/askadam.m:23-117) at parameters z (linear
 * mode: already clamped).  Returns total loss; gz [np][nv] gradient w.r.t. z. */
static double eval_z(adam_ctx* c, const double* z, double* gz, double* res, double* fid_out,
                     double* reg_out, double* gtheta_out) {
    const orc_adam_opts* o = c->o;
    const orc_volume* vol = c->vol;
    int np = c->np, nm = c->nm, nv = c->nv;
    double fid = 0.0;
    double* theta = (double*)malloc(sizeof(double) * (size_t)np * nv);
    double* gth = (double*)calloc((size_t)np * nv, sizeof(double));
    double* lfv = (double*)malloc(sizeof(double) * (size_t)(nv > 0 ? nv : 1));  /* per-voxel loss */
    for (size_t i = 0; i < (size_t)np * nv; ++i) theta[i] = unscale(o, (int)(i / nv), z[i]);
#pragma omp parallel for schedule(static) num_threads(o->nthreads > 0 ? o->nthreads : 1)
    for (int v = 0; v < nv; ++v) {
        double th[8], s[512], sb[512], tb[8] = {0};
        for (int k = 0; k < np; ++k) th[k] = theta[(size_t)k * nv + v];
        double sig = vol->sigma ? vol->sigma[v] : o->sigma;
        double b1 = c->m->model == ORC_MODEL_NEXI_RICE ? sig : (vol->b1 ? vol->b1[v] : 1.0);
        orc_forward_voxel(c->m, th, b1, s);
        double lf = 0.0;
        for (int k = 0; k < nm; ++k) {
            int bad = !isfinite(s[k]);
            double sk = bad ? 0.0 : s[k]; /* utils.set_nan_inf_zero, askadam.m:80 */
            double y = vol->data[(size_t)k * nv + v];
            double w = (vol->weights ? vol->weights[(size_t)k * nv + v] : 1.0) * (c->wmod ? c->wmod[v] : 1.0);
            double rv = orc_loss_value(o->loss, sk, y, w, sig, o->mse_scale, o->huber_delta);
            if (res) res[(size_t)k * nv + v] = rv;
            lf += rv;
            sb[k] = bad ? 0.0 : orc_loss_deriv(o->loss, sk, y, w, sig, o->mse_scale, o->huber_delta) * c->norm;
        }
        lfv[v] = lf;
        orc_vjp_voxel(c->m, th, b1, sb, tb);
        for (int k = 0; k < np; ++k) gth[(size_t)k * nv + v] = tb[k];
    }
    /* summed in voxel order: the same state always gives the same loss,
     * whatever the thread count */
    for (int v = 0; v < nv; ++v) fid += lfv[v];
    if (c->vloss)
        for (int v = 0; v < nv; ++v) c->vloss[v] = lfv[v] / nm;  /* mean(reshape(residuals, Nmeas, Nvol), 1) */
    free(lfv);
    fid *= c->norm;
    double reg = 0.0;
    if (o->n_reg > 0 && o->lambda[0] > 0 && o->reg_type == 1) {
        /* prior_distribution_normal (NEXI/gpuNEXI.m:1296-1303): lambda / Nmask *
         * sum |(theta - mu) / sigma| over the finite z-scores; the gradient of a
         * finite one is lambda / Nmask * sgn(z) / sigma */
        double nmask = (double)nv;
        for (int r = 0; r < o->n_reg; ++r) {
            int k = o->reg_param[r];
            double sr = 0.0;
            for (int v = 0; v < nv; ++v) {
                double sd = vol->prior_sd[(size_t)r * nv + v];
                double zs = (theta[(size_t)k * nv + v] - vol->prior_mu[(size_t)r * nv + v]) / sd;
                if (!isfinite(zs)) continue;
                sr += fabs(zs);
                double sg = zs > 0 ? 1.0 : (zs < 0 ? -1.0 : 0.0);
                gth[(size_t)k * nv + v] += o->lambda[r] / nmask * sg / sd;
            }
            reg += sr / nmask * o->lambda[r];
        }
        reg += vol->prior_offset;
    } else if (o->n_reg > 0 && o->lambda[0] > 0 && o->reg_type == 2) {
        /* surface_total_variation (NEXI/gpuNEXI.m:1236-1251): theta on the vertex
         * grid (0 off the mask), (theta_v - theta_nb) / length per neighbour slot
         * of every masked vertex, non-finite entries zeroed, sum |.| / Nmask *
         * lambda.  The gradient is the exact adjoint, scattered to both ends. */
        double nmask = (double)nv;
        int* inv = (int*)malloc(sizeof(int) * c->ngrid);
        for (size_t q = 0; q < c->ngrid; ++q) inv[q] = -1;
        for (int v = 0; v < nv; ++v) inv[vol->grid_index[v]] = v;
        for (int r = 0; r < o->n_reg; ++r) {
            int k = o->reg_param[r];
            memset(c->grid, 0, sizeof(double) * c->ngrid);
            for (int v = 0; v < nv; ++v) c->grid[vol->grid_index[v]] = theta[(size_t)k * nv + v];
            double sr = 0.0;
            for (int v = 0; v < nv; ++v)
                for (int j = 0; j < vol->max_neighbours; ++j) {
                    int q = vol->neighbours[(size_t)j * nv + v];
                    double len = vol->edge_length[(size_t)j * nv + v];
                    double t = (c->grid[vol->grid_index[v]] - c->grid[q]) / len;
                    if (!isfinite(t)) continue;
                    sr += fabs(t);
                    double d = (t > 0 ? 1.0 : (t < 0 ? -1.0 : 0.0)) / len * o->lambda[r] / nmask;
                    gth[(size_t)k * nv + v] += d;
                    if (inv[q] >= 0) gth[(size_t)k * nv + inv[q]] -= d;
                }
            reg += sr / nmask * o->lambda[r];
        }
        free(inv);
    } else if (o->n_reg > 0 && o->lambda[0] > 0) { /* spatial_total_variation.m:29 */
        double nmask = (double)nv;
        for (int r = 0; r < o->n_reg; ++r) {
            int k = o->reg_param[r];
            memset(c->grid, 0, sizeof(double) * c->ngrid);
            for (int v = 0; v < nv; ++v) c->grid[vol->grid_index[v]] = theta[(size_t)k * nv + v];
            double cost = orc_tv_cost(vol->dims, c->mask, c->grid, o->tv_3d, o->voxel_size);
            reg += cost / nmask * o->lambda[r];
            orc_tv_grad(vol->dims, c->mask, c->grid, o->tv_3d, o->voxel_size, c->grid_g);
            for (int v = 0; v < nv; ++v)
                gth[(size_t)k * nv + v] += o->lambda[r] / nmask * c->grid_g[vol->grid_index[v]];
        }
    }
    for (size_t i = 0; i < (size_t)np * nv; ++i) {
        int k = (int)(i / nv);
        gz[i] = gth[i] * dunscale(o, k, z[i]);
    }
    if (gtheta_out) memcpy(gtheta_out, gth, sizeof(double) * (size_t)np * nv);
    free(theta);
    free(gth);
    if (fid_out) *fid_out = fid;
    if (reg_out) *reg_out = reg;
    return fid + reg;
}

static int setup_ctx(adam_ctx* c, const orc_model* m, const orc_volume* vol,
                     const orc_adam_opts* o) {
    c->m = m; c->vol = vol; c->o = o;
    c->np = orc_nparams(m); c->nm = orc_nmeas(m); c->nv = vol->nvox;
    double nn = vol->norm_nvox > 0 ? vol->norm_nvox : (double)vol->nvox;
    c->norm = 1.0 / ((double)c->nm * nn);
    c->mask = NULL; c->grid = NULL; c->grid_g = NULL; c->ngrid = 0;
    c->wmod = NULL; c->vloss = NULL;
    if (o->n_reg > 0 && o->lambda[0] > 0 && o->reg_type == 1) {
        if (!vol->prior_mu || !vol->prior_sd) return -1;
    } else if (o->n_reg > 0 && o->lambda[0] > 0) {
        if (o->reg_type == 2 && (!vol->neighbours || !vol->edge_length)) return -1;
        if (!vol->grid_index) return -1;
        c->ngrid = (size_t)vol->dims[0] * vol->dims[1] * vol->dims[2];
        c->mask = (unsigned char*)calloc(c->ngrid, 1);
        c->grid = (double*)calloc(c->ngrid, sizeof(double));
        c->grid_g = (double*)calloc(c->ngrid, sizeof(double));
        for (int v = 0; v < vol->nvox; ++v) c->mask[vol->grid_index[v]] = 1;
    }
    return 0;
}

static void free_ctx(adam_ctx* c) { free(c->mask); free(c->grid); free(c->grid_g); }

double orc_model_gradient(const orc_model* m, const orc_volume* vol, const orc_adam_opts* o,
                          const double* theta, double* gtheta, double* residual, double* fid,
                          double* reg) {
    adam_ctx c;
    if (setup_ctx(&c, m, vol, o)) return NAN;
    /* evaluate with an identity-like transform by passing z such that unscale(z) = theta:
     * use the linear map directly. */
    orc_adam_opts lin = *o;
    lin.transform = ORC_TRANSFORM_LINEAR;
    c.o = &lin;
    size_t n = (size_t)c.np * c.nv;
    double* z = (double*)malloc(sizeof(double) * n);
    double* gz = (double*)malloc(sizeof(double) * n);
    for (size_t i = 0; i < n; ++i) {
        int k = (int)(i / c.nv);
        z[i] = (theta[i] - o->lb[k]) / (o->ub[k] - o->lb[k]);
    }
    double L = eval_z(&c, z, gz, residual, fid, reg, gtheta);
    free(z); free(gz); free_ctx(&c);
    return L;
}

static double clamp01(double z) { return z < 0 ? 0 : (z > 1 ? 1 : z); }

static int cmp_double(const void* a, const void* b) {
    double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

/* median of n values (NaN if any is NaN; even n: mean of the two middle ones) */
static double median_d(const double* x, int n) {
    double* t = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        if (isnan(x[i])) { free(t); return NAN; }
        t[i] = x[i];
    }
    qsort(t, (size_t)n, sizeof(double), cmp_double);
    double med = n == 0 ? NAN : (n & 1) ? t[n / 2] : 0.5 * (t[n / 2 - 1] + t[n / 2]);
    free(t);
    return med;
}

int orc_askadam(const orc_model* m, const orc_volume* vol, const orc_adam_opts* o,
                orc_adam_result* r) {
    adam_ctx c;
    if (setup_ctx(&c, m, vol, o)) return -1;
    int np = c.np, nm = c.nm, nv = c.nv;
    size_t n = (size_t)np * nv;
    double* z = (double*)malloc(sizeof(double) * n);
    double* zc = (double*)calloc(n, sizeof(double));
    double* zmin = (double*)malloc(sizeof(double) * n);
    double* zprev = (double*)malloc(sizeof(double) * n);
    double* g = (double*)malloc(sizeof(double) * n);
    double* m1 = (double*)calloc(n, sizeof(double));
    double* m2 = (double*)calloc(n, sizeof(double));
    double* res = (double*)malloc(sizeof(double) * (size_t)nm * nv);
    double* resmin = (double*)malloc(sizeof(double) * (size_t)nm * nv);
    int lin_mode = o->transform == ORC_TRANSFORM_LINEAR;

    /* initialise_parameter (utils/askadam.m:368-412) */
    for (int k = 0; k < np; ++k)
        for (int v = 0; v < nv; ++v) {
            uint32_t u[4];
            philox_call(o->seed, (uint32_t)v, (uint32_t)k, 0u, TAG_ADAM_INIT, u);
            double nrm, dummy;
            box_muller(u[0], u[1], &nrm, &dummy);
            double uni = orc_u01(u[2]);
            double zz;
            if (vol->theta0) {
                double t0 = vol->theta0[(size_t)k * nv + v];
                if (!lin_mode) {
                    double eb = 1e-4 * (o->ub[k] - o->lb[k]);
                    double tc = fmax(fmin(t0, o->ub[k] - eb), o->lb[k] + eb);
                    double nn = (tc - o->lb[k]) / (o->ub[k] - o->lb[k]);
                    zz = (1.0 - o->randomness) * log(nn / (1.0 - nn)) + o->randomness * nrm;
                } else {
                    zz = (1.0 - o->randomness) * (t0 - o->lb[k]) / (o->ub[k] - o->lb[k]) +
                         o->randomness * uni;
                }
            } else {
                zz = lin_mode ? uni : o->randomness * nrm;
            }
            if (lin_mode) zz = clamp01(zz); /* set_boundary01, askadam.m:185 */
            z[(size_t)k * nv + v] = o->state_f32 ? (double)(float)zz : zz;
        }

#define EVAL(resbuf, fidp, regp)                                                           \
    ({                                                                                     \
        for (size_t i_ = 0; i_ < n; ++i_) zc[i_] = lin_mode ? clamp01(z[i_]) : z[i_];      \
        double L_ = eval_z(&c, zc, g, resbuf, fidp, regp, NULL);                           \
        if (lin_mode)                                                                      \
            for (size_t i_ = 0; i_ < n; ++i_)                                              \
                if (z[i_] < 0.0 || z[i_] > 1.0) g[i_] = 0.0;                               \
        L_;                                                                                \
    })

    /* robustConvergence state (utils/askadam.m:221-241) */
    int RW = o->outlier_check_window > 0 ? o->outlier_check_window : 1;
    double *wmod = NULL, *vloss = NULL, *vinit = NULL, *vhist = NULL, *impA = NULL, *impB = NULL;
    int *flagcnt = NULL;
    unsigned char *mainmask = NULL, *convmask = NULL;
    int reprime = 0;
    if (o->robust) {
        wmod = (double*)malloc(sizeof(double) * nv);
        vloss = (double*)malloc(sizeof(double) * nv);
        vinit = (double*)malloc(sizeof(double) * nv);
        vhist = (double*)malloc(sizeof(double) * (size_t)RW * nv);
        impA = (double*)malloc(sizeof(double) * nv);
        impB = (double*)malloc(sizeof(double) * nv);
        flagcnt = (int*)calloc(nv, sizeof(int));
        mainmask = (unsigned char*)malloc(nv);
        convmask = (unsigned char*)malloc(nv);
        for (int v = 0; v < nv; ++v) { wmod[v] = 1.0; mainmask[v] = 1; convmask[v] = 1; }
        c.wmod = wmod;
        c.vloss = vloss;
    }

    double fid, reg;
    double loss = EVAL(res, &fid, &reg);
    if (r->loss_history) r->loss_history[0] = loss;
    if (o->robust) { /* perVoxelLossInit, history = repmat(init, outlierCheckWindow, 1) */
        memcpy(vinit, vloss, sizeof(double) * nv);
        for (int q = 0; q < RW; ++q) memcpy(vhist + (size_t)q * nv, vloss, sizeof(double) * nv);
    }
    double minLoss = loss, minFid = fid, minReg = reg;
    memcpy(zmin, z, sizeof(double) * n);
    memcpy(resmin, res, sizeof(double) * (size_t)nm * nv);
    int minIter = 0, epoch = 0, stop = ORC_STOP_NONE;
    double ema = loss;
    int W = o->conv_window > 0 ? o->conv_window : 1;
    double* buf = (double*)malloc(sizeof(double) * W);
    for (int i = 0; i < W; ++i) buf[i] = 1.0;
    double ewic = 0, ewis = 0, ewig = 0;
    memcpy(zprev, z, sizeof(double) * n);

    for (int e = 1; e <= o->iteration; ++e) {
        epoch = e;
        loss = EVAL(res, &fid, &reg);
        if (r->loss_history) r->loss_history[e] = loss;
        if (minLoss > loss) { /* update_min_loss, askadam.m:433-446 */
            minLoss = loss; minFid = fid; minReg = reg;
            memcpy(zmin, z, sizeof(double) * n);
            memcpy(resmin, res, sizeof(double) * (size_t)nm * nv);
            minIter = e;
        }
        double loss_conv = loss;
        if (o->robust) {
            /* update_outlier_mask (askadam.m:448-510): the new weights apply
             * from the next evaluation */
            if (o->weight_update_interval > 0 && e % o->weight_update_interval == 0) {
                memmove(vhist, vhist + nv, sizeof(double) * (size_t)(RW - 1) * nv);
                memcpy(vhist + (size_t)(RW - 1) * nv, vloss, sizeof(double) * nv);
                for (int v = 0; v < nv; ++v) {
                    impA[v] = (vhist[v] - vloss[v]) / (vhist[v] + 1e-8);
                    impB[v] = (vinit[v] - vloss[v]) / (vinit[v] + 1e-8);
                }
                double medA = median_d(impA, nv), medB = median_d(impB, nv);
                for (int v = 0; v < nv; ++v) {
                    int failA = impA[v] < o->outlier_voxel_thres && medA > o->outlier_pop_thres;
                    int failB = impB[v] < o->outlier_init_thres && medB > o->outlier_init_pop_thres;
                    if (failA && failB) flagcnt[v] += 1;
                    else flagcnt[v] = flagcnt[v] > 0 ? flagcnt[v] - 1 : 0;
                    mainmask[v] = flagcnt[v] == 0;
                    wmod[v] = mainmask[v] ? 1.0 : o->outlier_weight;
                    if (!mainmask[v] && r->ever_flagged) r->ever_flagged[v] = 1;
                }
            }
            /* main-population loss with the mask frozen between window
             * boundaries (askadam.m:530-563) */
            if (e % (o->conv_window > 0 ? o->conv_window : 1) == 0 && memcmp(mainmask, convmask, nv) != 0) {
                memcpy(convmask, mainmask, nv);
                reprime = o->conv_window;
            }
            double sl = 0.0;
            int cnt = 0;
            for (int v = 0; v < nv; ++v)
                if (convmask[v]) { sl += vloss[v]; ++cnt; }
            loss_conv = sl / cnt;
        }
        /* update_convergence_signals, askadam.m:512-632 */
        double conv;
        if (o->conv_model == ORC_CONV_EMA) {
            double en = o->ema_decay * ema + (1.0 - o->ema_decay) * loss_conv;
            conv = fabs(en - ema) / (fabs(ema) + 1e-8);
            ema = en;
        } else {
            for (int i = 0; i < W - 1; ++i) buf[i] = buf[i + 1];
            buf[W - 1] = loss_conv;
            double xm = (W + 1) / 2.0, ym = 0, sxy = 0, sxx = 0;
            for (int i = 0; i < W; ++i) ym += buf[i];
            ym /= W;
            for (int i = 0; i < W; ++i) {
                sxy += (i + 1 - xm) * (buf[i] - ym);
                sxx += (i + 1 - xm) * (i + 1 - xm);
            }
            conv = sxx > 0 ? -(sxy / sxx) : 0.0;
        }
        if (reprime > 0) { reprime -= 1; ewic = 0; }
        else if (conv > o->conv_value || e <= o->conv_window) ewic = 0;
        else if (!o->robust && (minLoss - loss) > o->conv_value) ewic = 0;
        else ewic += 1;
        if (o->step_tol > 0) {
            double num = 0, den = 0;
            for (size_t i = 0; i < n; ++i) {
                double dd = z[i] - zprev[i];
                num += dd * dd;
                den += z[i] * z[i];
            }
            double sn = sqrt(num) / (1.0 + sqrt(den));
            memcpy(zprev, z, sizeof(double) * n);
            ewis = sn < o->step_tol ? ewis + 1 : 0;
        }
        if (o->grad_tol > 0) {
            double gn = 0;
            for (size_t i = 0; i < n; ++i) gn += g[i] * g[i];
            gn = sqrt(gn);
            ewig = gn < o->grad_tol ? ewig + 1 : 0;
        }
        /* check_stopping, askadam.m:634-671 */
        if (ewic > o->patience_conv) { stop = ORC_STOP_CONVERGENCE; break; }
        if (loss < o->tol) { stop = ORC_STOP_TOL; break; }
        if (o->step_tol > 0 && ewis > o->patience_step) { stop = ORC_STOP_STEP; break; }
        if (o->grad_tol > 0 && ewig > o->patience_grad) { stop = ORC_STOP_GRAD; break; }
        /* update_parameters, askadam.m:673-691 */
        double lr = o->lr / (1.0 + o->decay * (e - 1));
        if (e < o->iteration) {
            double bc1 = 1.0 - pow(o->beta1, e), bc2 = 1.0 - pow(o->beta2, e);
            for (size_t i = 0; i < n; ++i) {
                double gi = g[i];
                if (o->optimiser == ORC_OPT_ADAM) {
                    m1[i] = o->beta1 * m1[i] + (1.0 - o->beta1) * gi;
                    m2[i] = o->beta2 * m2[i] + (1.0 - o->beta2) * gi * gi;
                    z[i] -= lr * (m1[i] / bc1) / (sqrt(m2[i] / bc2) + o->eps);
                } else if (o->optimiser == ORC_OPT_SGDM) {
                    m1[i] = o->momentum * m1[i] - lr * gi;
                    z[i] += m1[i];
                } else {
                    m2[i] = o->rms_decay * m2[i] + (1.0 - o->rms_decay) * gi * gi;
                    z[i] -= lr * gi / (sqrt(m2[i]) + o->rms_eps);
                }
                if (o->state_f32) {
                    z[i] = (float)z[i];
                    m1[i] = (float)m1[i];
                    m2[i] = (float)m2[i];
                }
            }
        }
    }
    /* finalisation (askadam.m:312-362) */
    for (size_t i = 0; i < n; ++i) {
        int k = (int)(i / nv);
        double zf = lin_mode ? clamp01(z[i]) : z[i];
        double zm = lin_mode ? clamp01(zmin[i]) : zmin[i];
        r->final_theta[i] = unscale(o, k, zf);
        if (r->min_theta) r->min_theta[i] = unscale(o, k, zm);
    }
    if (r->final_residual) memcpy(r->final_residual, res, sizeof(double) * (size_t)nm * nv);
    if (r->min_residual) memcpy(r->min_residual, resmin, sizeof(double) * (size_t)nm * nv);
    r->final_loss = loss; r->final_fid = fid; r->final_reg = reg;
    r->min_loss = minLoss; r->min_fid = minFid; r->min_reg = minReg;
    r->final_niter = epoch; r->min_niter = minIter; r->stop_reason = stop;
#undef EVAL
    free(z); free(zc); free(zmin); free(zprev); free(g); free(m1); free(m2);
    free(res); free(resmin); free(buf);
    free(wmod); free(vloss); free(vinit); free(vhist); free(impA); free(impB);
    free(flagcnt); free(mainmask); free(convmask);
    free_ctx(&c);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* MCMC (utils/mcmc.m)                                                       */
/* ------------------------------------------------------------------------ */
int orc_mcmc_nsamples(int iteration, double burnin, int thinning) {
    int nb = burnin < 1 ? (int)floor(iteration * burnin) : (int)burnin; /* mcmc.m:788-794 */
    if (nb + 1 > iteration) return 0;
    return (iteration - nb - 1) / thinning + 1; /* numel(Nburnin+1:thinning:iteration) */
}

static int nburnin(const orc_mcmc_opts* o) {
    return o->burnin < 1 ? (int)floor(o->iteration * o->burnin) : (int)o->burnin;
}

/* find_partner (mcmc.m:797-803): uniform random derangement, one per step,
 * shared by all voxels.  Fisher-Yates with rejection of fixed points. */
static void derangement(uint64_t seed, int step, uint32_t tag, int W, int* p) {
    for (uint32_t attempt = 0; attempt < 4096; ++attempt) {
        for (int i = 0; i < W; ++i) p[i] = i;
        uint32_t u[4];
        for (int i = W - 1, d = 0; i >= 1; --i, ++d) {
            if ((d & 3) == 0)
                philox_call(seed, (uint32_t)step, attempt, (uint32_t)(d >> 2), tag, u);
            int j = (int)rand_below(u[d & 3], (uint32_t)(i + 1));
            int t = p[i]; p[i] = p[j]; p[j] = t;
        }
        int fixed = 0;
        for (int i = 0; i < W; ++i) fixed |= (p[i] == i);
        if (!fixed) return;
    }
    for (int i = 0; i < W; ++i) p[i] = (i + 1) % W; /* unreachable in practice */
}

void orc_gw_partner(uint64_t seed, int step, int rep, int W, int* p) {
    derangement(seed, step, TAG_GW_PERM | ((uint32_t)rep << 16), W, p);
}

/* Red-black anchor draw (mcmc.m:328-329): for half-step s, the partner of
 * the a-th active walker is frozen[randi(numel(frozen))], shared by voxels. */
static void rb_partner_tag(uint64_t seed, int step, uint32_t tag, int half, int na, int nf, int* out) {
    uint32_t u[4];
    for (int a = 0; a < na; ++a) {
        if ((a & 3) == 0) philox_call(seed, (uint32_t)step, (uint32_t)half, (uint32_t)(a >> 2), tag, u);
        out[a] = (int)rand_below(u[a & 3], (uint32_t)nf);
    }
}

static void rb_partner(uint64_t seed, int step, int rep, int half, int na, int nf, int* out) {
    rb_partner_tag(seed, step, TAG_GW_RBPART | ((uint32_t)rep << 16), half, na, nf, out);
}

typedef struct {
    const orc_model* m;
    const orc_volume* vol;
    int nm, np, nvar;
} mc_ctx;

/* logP_Gaussian(sum w (FWD - y)^2, noise, Nm)  (utils/logP_Gaussian.m:18-20) */
static double logp(const mc_ctx* c, int v, const double* x) {
    double s[512];
    double b1 = c->vol->b1 ? c->vol->b1[v] : 1.0;
    orc_forward_voxel(c->m, x, b1, s);
    double sos = 0.0;
    int nv = c->vol->nvox;
    for (int k = 0; k < c->nm; ++k) {
        double w = c->vol->weights ? c->vol->weights[(size_t)k * nv + v] : 1.0;
        double r = s[k] - c->vol->data[(size_t)k * nv + v];
        sos += w * r * r;
    }
    double noise = x[c->nvar - 1];
    return -sos / (2.0 * noise * noise) - c->nm / 2.0 * log(2.0 * M_PI * noise * noise);
}

static int mcmc_gw_global(const orc_model* m, const orc_volume* vol, const double* x0,
                          const orc_mcmc_opts* o, orc_mcmc_result* r);

int orc_mcmc(const orc_model* m, const orc_volume* vol, const double* x0,
             const orc_mcmc_opts* o, orc_mcmc_result* r) {
    if (o->is_global) {
        int any = 0;
        for (int p = 0; p < orc_nparams(m) + 1; ++p) any |= o->is_global[p] != 0;
        if (any) return o->algorithm == 1 ? mcmc_gw_global(m, vol, x0, o, r) : -1;
    }
    mc_ctx c = {m, vol, orc_nmeas(m), orc_nparams(m), orc_nparams(m) + 1};
    int nvar = c.nvar, nv = vol->nvox;
    int W = o->algorithm == 1 ? o->nwalker : 1;
    int nb = nburnin(o);
    int ns = orc_mcmc_nsamples(o->iteration, o->burnin, o->thinning);
    r->ns = ns;
    int rep = o->repetition;
    double nsample = (double)W * ns * rep;
    long long acc_total = 0, prop_total = 0;
    int* perm = NULL;
    int* rbp = NULL;
    int h = W / 2;
    if (o->algorithm == 1 && o->ensemble_update == ORC_GW_SIMULTANEOUS) {
        perm = (int*)malloc(sizeof(int) * (size_t)rep * o->iteration * W);
        for (int rr = 0; rr < rep; ++rr)
            for (int k = 1; k <= o->iteration; ++k)
                orc_gw_partner(o->seed, k, rr, W, perm + ((size_t)rr * o->iteration + (k - 1)) * W);
    }
    if (o->algorithm == 1 && o->ensemble_update == ORC_GW_REDBLACK) {
        rbp = (int*)malloc(sizeof(int) * (size_t)rep * o->iteration * W);
        for (int rr = 0; rr < rep; ++rr)
            for (int k = 1; k <= o->iteration; ++k) {
                int* base = rbp + ((size_t)rr * o->iteration + (k - 1)) * W;
                rb_partner(o->seed, k, rr, 0, h, W - h, base);
                rb_partner(o->seed, k, rr, 1, W - h, h, base + h);
            }
    }

#pragma omp parallel for schedule(dynamic, 4) reduction(+ : acc_total, prop_total) num_threads(o->nthreads > 0 ? o->nthreads : 1)
    for (int v = 0; v < nv; ++v) {
        double xi[64 * 8], lpi[64], x[64 * 8], xo[64 * 8], lp[64];
        double sum[8] = {0}, sumsq[8] = {0}, shift[8];
        /* starting points (mcmc.m:125-129, 267-275) */
        for (int w = 0; w < W; ++w) {
            double nrm[8];
            if (o->algorithm == 1) {
                for (int j = 0; j * 4 < nvar; ++j) {
                    uint32_t u[4];
                    philox_call(o->seed, (uint32_t)v, (uint32_t)w, (uint32_t)j, TAG_GW_INIT, u);
                    double a, b, cc, d;
                    box_muller(u[0], u[1], &a, &b);
                    box_muller(u[2], u[3], &cc, &d);
                    double q[4] = {a, b, cc, d};
                    for (int t = 0; t < 4 && 4 * j + t < nvar; ++t) nrm[4 * j + t] = q[t];
                }
            }
            for (int p = 0; p < nvar; ++p) {
                double val = x0[(size_t)p * nv + v];
                if (o->algorithm == 1) val += (o->ub[p] - o->lb[p]) * o->start_range * nrm[p];
                val = fmin(fmax(val, o->lb[p]), o->ub[p]);
                xi[w * nvar + p] = val;
            }
            lpi[w] = logp(&c, v, xi + w * nvar);
        }
        /* running sums are taken about the clamped start value */
        for (int p = 0; p < nvar; ++p) shift[p] = fmin(fmax(x0[(size_t)p * nv + v], o->lb[p]), o->ub[p]);
        long long acc = 0, prop = 0;
        for (int rr = 0; rr < rep; ++rr) {
            memcpy(x, xi, sizeof(double) * W * nvar);
            memcpy(lp, lpi, sizeof(double) * W);
            int counter = 0;
            for (int k = 1; k <= o->iteration; ++k) {
                if (o->algorithm == 0) {
                    /* metropolis_hastings, mcmc.m:144-167 */
                    double nrm[8], xp[8];
                    for (int j = 0; j * 4 < nvar; ++j) {
                        uint32_t u[4];
                        philox_call(o->seed, (uint32_t)v, (uint32_t)k, (uint32_t)j,
                                    TAG_MH_MOVE | ((uint32_t)rr << 16), u);
                        double a, b, cc, d;
                        box_muller(u[0], u[1], &a, &b);
                        box_muller(u[2], u[3], &cc, &d);
                        double q[4] = {a, b, cc, d};
                        for (int t = 0; t < 4 && 4 * j + t < nvar; ++t) nrm[4 * j + t] = q[t];
                    }
                    uint32_t ua[4];
                    philox_call(o->seed, (uint32_t)v, (uint32_t)k, 8u, TAG_MH_MOVE | ((uint32_t)rr << 16), ua);
                    int oob = 0;
                    for (int p = 0; p < nvar; ++p) {
                        xp[p] = x[p] + o->x_step[p] * nrm[p];
                        oob |= (xp[p] < o->lb[p]) || (xp[p] > o->ub[p]);
                        xp[p] = fmin(fmax(xp[p], o->lb[p]), o->ub[p]);
                    }
                    double lpp = logp(&c, v, xp);
                    ++prop;
                    if (!oob && (lpp - lp[0]) > log(orc_u01(ua[0]))) {
                        memcpy(x, xp, sizeof(double) * nvar);
                        lp[0] = lpp;
                        ++acc;
                    }
                } else if (o->ensemble_update == ORC_GW_SIMULTANEOUS) {
                    /* goodman_weare simultaneous, mcmc.m:290-318 */
                    const int* pt = perm + ((size_t)rr * o->iteration + (k - 1)) * W;
                    memcpy(xo, x, sizeof(double) * W * nvar);
                    for (int w = 0; w < W; ++w) {
                        uint32_t u[4];
                        philox_call(o->seed, (uint32_t)v, (uint32_t)w, (uint32_t)k,
                                    TAG_GW_MOVE | ((uint32_t)rr << 16), u);
                        double a = o->step_size;
                        double t = (a - 1.0) * orc_u01(u[0]) + 1.0;
                        double zz = t * t / a;
                        double xp[8];
                        int oob = 0;
                        for (int p = 0; p < nvar; ++p) {
                            double xq = xo[pt[w] * nvar + p];
                            xp[p] = xq + (xo[w * nvar + p] - xq) * zz;
                            oob |= (xp[p] < o->lb[p]) || (xp[p] > o->ub[p]);
                            xp[p] = fmin(fmax(xp[p], o->lb[p]), o->ub[p]);
                        }
                        double lpp = logp(&c, v, xp);
                        ++prop;
                        double lr = (nvar - 1) * log(zz) + (lpp - lp[w]);
                        if (!oob && lr > log(orc_u01(u[1]))) {
                            memcpy(x + w * nvar, xp, sizeof(double) * nvar);
                            lp[w] = lpp;
                            ++acc;
                        }
                    }
                } else {
                    /* goodman_weare red-black, mcmc.m:321-357 */
                    const int* pb = rbp + ((size_t)rr * o->iteration + (k - 1)) * W;
                    for (int s = 0; s < 2; ++s) {
                        int a0 = s == 0 ? 0 : h, na = s == 0 ? h : W - h;
                        int f0 = s == 0 ? h : 0;
                        for (int ai = 0; ai < na; ++ai) {
                            int w = a0 + ai;
                            int q = f0 + pb[(s == 0 ? 0 : h) + ai];
                            uint32_t u[4];
                            philox_call(o->seed, (uint32_t)v, (uint32_t)w, (uint32_t)k,
                                        TAG_GW_MOVE | ((uint32_t)rr << 16) | (1u << 8), u);
                            double a = o->step_size;
                            double t = (a - 1.0) * orc_u01(u[0]) + 1.0;
                            double zz = t * t / a;
                            double xp[8];
                            int oob = 0;
                            for (int p = 0; p < nvar; ++p) {
                                double xq = x[q * nvar + p];
                                xp[p] = xq + (x[w * nvar + p] - xq) * zz;
                                oob |= (xp[p] < o->lb[p]) || (xp[p] > o->ub[p]);
                                xp[p] = fmin(fmax(xp[p], o->lb[p]), o->ub[p]);
                            }
                            double lpp = logp(&c, v, xp);
                            ++prop;
                            double lr = (nvar - 1) * log(zz) + (lpp - lp[w]);
                            if (!oob && lr > log(orc_u01(u[1]))) {
                                memcpy(xo + w * nvar, xp, sizeof(double) * nvar);
                                lp[w] = lpp;
                                ++acc;
                            } else {
                                memcpy(xo + w * nvar, x + w * nvar, sizeof(double) * nvar);
                            }
                        }
                        /* the active half is written back only after the whole half-step */
                        for (int ai = 0; ai < na; ++ai)
                            memcpy(x + (a0 + ai) * nvar, xo + (a0 + ai) * nvar, sizeof(double) * nvar);
                    }
                }
                /* burn-in / thinning (mcmc.m:172-175, 363-366) */
                if (k > nb && (k - nb + 1) % o->thinning == 0 && counter < ns) {
                    for (int w = 0; w < W; ++w)
                        for (int p = 0; p < nvar; ++p) {
                            double val = x[w * nvar + p];
                            double d = val - shift[p];
                            sum[p] += d;
                            sumsq[p] += d * d;
                            if (r->posterior) {
                                size_t idx = (size_t)v + (size_t)nv * (w + (size_t)W * (counter + (size_t)ns * rr));
                                r->posterior[(size_t)p * nv * W * ns * rep + idx] = (float)val;
                            }
                        }
                    ++counter;
                }
            }
            /* unfilled sample slots stay zero in the reference's preallocated array */
            int missing = ns - counter;
            for (int p = 0; p < nvar; ++p) {
                double d = 0.0 - shift[p];
                sum[p] += (double)missing * W * d;
                sumsq[p] += (double)missing * W * d * d;
            }
        }
        for (int p = 0; p < nvar; ++p) {
            double mean_d = sum[p] / nsample;
            double var = nsample > 1 ? (sumsq[p] - sum[p] * mean_d) / (nsample - 1.0) : 0.0;
            if (r->mean) r->mean[(size_t)p * nv + v] = shift[p] + mean_d;
            if (r->std) r->std[(size_t)p * nv + v] = sqrt(fmax(var, 0.0));
        }
        acc_total += acc;
        prop_total += prop;
    }
    r->n_accepted = acc_total;
    r->n_proposals = prop_total;
    free(perm);
    free(rbp);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* goodman_weare_wglobal_constant (utils/mcmc.m:385-578) with gw_global_block */
/* (:581-626): parameters split into local (per voxel) and global (shared by */
/* all voxels, one value per walker).  Each iteration is a local stretch move */
/* with the globals held (exponent z^(NND-1)), then a global stretch move with */
/* the locals held, accepted on the log-likelihood difference summed over all */
/* voxels in double (exponent z^(NGlobal-1)).  Locals start at x0 +          */
/* (ub-lb)*startRange*randn (clamped), globals uniformly over their bounds;   */
/* every repetition restarts from those walkers; globalWarmup global-only     */
/* iterations precede the joint loop.  The voxel sum runs in voxel order.     */
/* ------------------------------------------------------------------------ */
typedef struct {
    const mc_ctx* c;
    const orc_mcmc_opts* o;
    int nv, W, nvar, ng, nnd;
    const int* isg;
    double* x;     /* [nv][W][nvar] local slots used */
    double* g;     /* [W][nvar] global slots used */
    double* lp;    /* [nv][W] cached logP at the current state */
    double* lpg;   /* [nv][W] logP of the global proposal */
} gwg_state;

static double gwg_logp(const gwg_state* S, int v, int w, const double* gw) {
    double xx[8];
    for (int p = 0; p < S->nvar; ++p)
        xx[p] = S->isg[p] ? gw[p] : S->x[((size_t)v * S->W + w) * S->nvar + p];
    return logp(S->c, v, xx);
}

/* One global block (gw_global_block): the walkers of `act` (na of them)
 * propose around anchors `anc`; returns accepted count. */
static long long gwg_global_sub(gwg_state* S, int k, uint32_t tagbits, const int* act, const int* anc, int na) {
    const orc_mcmc_opts* o = S->o;
    int W = S->W, nvar = S->nvar, nv = S->nv;
    double* gp = (double*)malloc(sizeof(double) * (size_t)na * nvar);
    int* oob = (int*)calloc((size_t)na, sizeof(int));
    double* zz = (double*)malloc(sizeof(double) * (size_t)na);
    double* lu = (double*)malloc(sizeof(double) * (size_t)na);
    for (int i = 0; i < na; ++i) {
        int w = act[i], q = anc[i];
        uint32_t u[4];
        philox_call(o->seed, (uint32_t)w, (uint32_t)k, 0u, TAG_GW_GMOVE | tagbits, u);
        double a = o->step_size;
        double t = (a - 1.0) * orc_u01(u[0]) + 1.0;
        zz[i] = t * t / a;
        lu[i] = log(orc_u01(u[1]));
        for (int p = 0; p < nvar; ++p) {
            if (!S->isg[p]) { gp[(size_t)i * nvar + p] = 0.0; continue; }
            double gq = S->g[(size_t)q * nvar + p];
            double val = gq + (S->g[(size_t)w * nvar + p] - gq) * zz[i];
            oob[i] |= (val < o->lb[p]) || (val > o->ub[p]);
            gp[(size_t)i * nvar + p] = fmin(fmax(val, o->lb[p]), o->ub[p]);
        }
    }
#pragma omp parallel for schedule(static) num_threads(o->nthreads > 0 ? o->nthreads : 1)
    for (int v = 0; v < nv; ++v)
        for (int i = 0; i < na; ++i)
            S->lpg[(size_t)v * W + act[i]] = gwg_logp(S, v, act[i], gp + (size_t)i * nvar);
    long long nacc = 0;
    for (int i = 0; i < na; ++i) {
        int w = act[i];
        double d = 0.0;
        for (int v = 0; v < nv; ++v) d += S->lpg[(size_t)v * W + w] - S->lp[(size_t)v * W + w];
        double lr = (S->ng - 1) * log(zz[i]) + d;
        if (!oob[i] && lr > lu[i]) {
            ++nacc;
            for (int p = 0; p < nvar; ++p)
                if (S->isg[p]) S->g[(size_t)w * nvar + p] = gp[(size_t)i * nvar + p];
            for (int v = 0; v < nv; ++v) S->lp[(size_t)v * W + w] = S->lpg[(size_t)v * W + w];
        }
    }
    free(gp); free(oob); free(zz); free(lu);
    return nacc;
}

static void gwg_global_block(gwg_state* S, int k, int rr, int warm) {
    const orc_mcmc_opts* o = S->o;
    int W = S->W;
    uint32_t bits = ((uint32_t)rr << 16) | (warm ? TAG_WARM : 0u);
    int act[256], anc[256];
    if (o->ensemble_update == ORC_GW_SIMULTANEOUS) {
        int pt[256];
        derangement(o->seed, k, TAG_GW_GPERM | bits, W, pt);
        for (int w = 0; w < W; ++w) { act[w] = w; anc[w] = pt[w]; }
        gwg_global_sub(S, k, bits, act, anc, W);
    } else {
        int h = W / 2;
        for (int s = 0; s < 2; ++s) {
            int a0 = s == 0 ? 0 : h, na = s == 0 ? h : W - h, f0 = s == 0 ? h : 0, nf = s == 0 ? W - h : h;
            int pb[256];
            rb_partner_tag(o->seed, k, TAG_GW_GRBPART | bits, s, na, nf, pb);
            for (int i = 0; i < na; ++i) { act[i] = a0 + i; anc[i] = f0 + pb[i]; }
            gwg_global_sub(S, k, bits | TAG_RB, act, anc, na);
        }
    }
}

static int mcmc_gw_global(const orc_model* m, const orc_volume* vol, const double* x0,
                          const orc_mcmc_opts* o, orc_mcmc_result* r) {
    mc_ctx c = {m, vol, orc_nmeas(m), orc_nparams(m), orc_nparams(m) + 1};
    int nvar = c.nvar, nv = vol->nvox, W = o->nwalker, rep = o->repetition;
    int nb = nburnin(o);
    int ns = orc_mcmc_nsamples(o->iteration, o->burnin, o->thinning);
    r->ns = ns;
    int ng = 0;
    for (int p = 0; p < nvar; ++p) ng += o->is_global[p] != 0;
    if (ng == 0 || ng == nvar) return -2;
    gwg_state S = {&c, o, nv, W, nvar, ng, nvar - ng, o->is_global, NULL, NULL, NULL, NULL};
    size_t nx = (size_t)nv * W * nvar;
    double* xi = (double*)malloc(sizeof(double) * nx);
    double* gi = (double*)calloc((size_t)W * nvar, sizeof(double));
    double* lpi = (double*)malloc(sizeof(double) * (size_t)nv * W);
    S.x = (double*)malloc(sizeof(double) * nx);
    S.g = (double*)malloc(sizeof(double) * (size_t)W * nvar);
    S.lp = (double*)malloc(sizeof(double) * (size_t)nv * W);
    S.lpg = (double*)malloc(sizeof(double) * (size_t)nv * W);
    double* sum = (double*)calloc((size_t)nvar * nv, sizeof(double));
    double* sumsq = (double*)calloc((size_t)nvar * nv, sizeof(double));
    double* shift = (double*)malloc(sizeof(double) * (size_t)nvar * nv);
    for (int p = 0; p < nvar; ++p)
        for (int v = 0; v < nv; ++v)
            shift[(size_t)p * nv + v] = fmin(fmax(x0[(size_t)p * nv + (o->is_global[p] ? 0 : v)], o->lb[p]), o->ub[p]);
    /* walker start: locals as in goodman_weare (same stream), globals uniform */
    for (int v = 0; v < nv; ++v)
        for (int w = 0; w < W; ++w) {
            double nrm[8];
            for (int j = 0; j * 4 < nvar; ++j) {
                uint32_t u[4];
                philox_call(o->seed, (uint32_t)v, (uint32_t)w, (uint32_t)j, TAG_GW_INIT, u);
                double a, b, cc, d;
                box_muller(u[0], u[1], &a, &b);
                box_muller(u[2], u[3], &cc, &d);
                double q[4] = {a, b, cc, d};
                for (int t = 0; t < 4 && 4 * j + t < nvar; ++t) nrm[4 * j + t] = q[t];
            }
            for (int p = 0; p < nvar; ++p) {
                double val = 0.0;
                if (!o->is_global[p]) {
                    val = x0[(size_t)p * nv + v] + (o->ub[p] - o->lb[p]) * o->start_range * nrm[p];
                    val = fmin(fmax(val, o->lb[p]), o->ub[p]);
                }
                xi[((size_t)v * W + w) * nvar + p] = val;
            }
        }
    for (int w = 0; w < W; ++w)
        for (int p = 0; p < nvar; ++p)
            if (o->is_global[p]) {
                uint32_t u[4];
                philox_call(o->seed, (uint32_t)w, (uint32_t)(p >> 2), 0u, TAG_GW_GINIT, u);
                gi[(size_t)w * nvar + p] = o->lb[p] + (o->ub[p] - o->lb[p]) * orc_u01(u[p & 3]);
            }
    memcpy(S.x, xi, sizeof(double) * nx);
    memcpy(S.g, gi, sizeof(double) * (size_t)W * nvar);
#pragma omp parallel for schedule(static) num_threads(o->nthreads > 0 ? o->nthreads : 1)
    for (int v = 0; v < nv; ++v)
        for (int w = 0; w < W; ++w) lpi[(size_t)v * W + w] = gwg_logp(&S, v, w, gi + (size_t)w * nvar);

    long long acc_total = 0, prop_total = 0;
    int h = W / 2;
    int* pt = (int*)malloc(sizeof(int) * (size_t)W);
    for (int rr = 0; rr < rep; ++rr) {
        memcpy(S.x, xi, sizeof(double) * nx);
        memcpy(S.g, gi, sizeof(double) * (size_t)W * nvar);
        memcpy(S.lp, lpi, sizeof(double) * (size_t)nv * W);
        for (int kw = 1; kw <= o->global_warmup; ++kw) gwg_global_block(&S, kw, rr, 1);
        int counter = 0;
        for (int k = 1; k <= o->iteration; ++k) {
            /* LOCAL block, globals held (mcmc.m:515-553) */
            if (o->ensemble_update == ORC_GW_SIMULTANEOUS) {
                orc_gw_partner(o->seed, k, rr, W, pt);
            }
            long long acc = 0;
#pragma omp parallel for schedule(static) reduction(+ : acc) num_threads(o->nthreads > 0 ? o->nthreads : 1)
            for (int v = 0; v < nv; ++v) {
                double* xv = S.x + (size_t)v * W * nvar;
                double xo[256 * 8];
                if (o->ensemble_update == ORC_GW_SIMULTANEOUS) {
                    memcpy(xo, xv, sizeof(double) * W * nvar);
                    for (int w = 0; w < W; ++w) {
                        uint32_t u[4];
                        philox_call(o->seed, (uint32_t)v, (uint32_t)w, (uint32_t)k, TAG_GW_MOVE | ((uint32_t)rr << 16), u);
                        double a = o->step_size, t = (a - 1.0) * orc_u01(u[0]) + 1.0, zz = t * t / a;
                        double xp[8];
                        int oob = 0;
                        for (int p = 0; p < nvar; ++p) {
                            if (o->is_global[p]) { xp[p] = S.g[(size_t)w * nvar + p]; continue; }
                            double xq = xo[pt[w] * nvar + p];
                            double val = xq + (xo[w * nvar + p] - xq) * zz;
                            oob |= (val < o->lb[p]) || (val > o->ub[p]);
                            xp[p] = fmin(fmax(val, o->lb[p]), o->ub[p]);
                        }
                        double lpp = logp(&c, v, xp);
                        double lr = (S.nnd - 1) * log(zz) + (lpp - S.lp[(size_t)v * W + w]);
                        if (!oob && lr > log(orc_u01(u[1]))) {
                            for (int p = 0; p < nvar; ++p)
                                if (!o->is_global[p]) xv[w * nvar + p] = xp[p];
                            S.lp[(size_t)v * W + w] = lpp;
                            ++acc;
                        }
                    }
                } else {
                    int pb[256];
                    for (int s = 0; s < 2; ++s) {
                        int a0 = s == 0 ? 0 : h, na = s == 0 ? h : W - h, f0 = s == 0 ? h : 0, nf = s == 0 ? W - h : h;
                        rb_partner(o->seed, k, rr, s, na, nf, pb);
                        for (int i = 0; i < na; ++i) {
                            int w = a0 + i, q = f0 + pb[i];
                            uint32_t u[4];
                            philox_call(o->seed, (uint32_t)v, (uint32_t)w, (uint32_t)k,
                                        TAG_GW_MOVE | ((uint32_t)rr << 16) | TAG_RB, u);
                            double a = o->step_size, t = (a - 1.0) * orc_u01(u[0]) + 1.0, zz = t * t / a;
                            double xp[8];
                            int oob = 0;
                            for (int p = 0; p < nvar; ++p) {
                                if (o->is_global[p]) { xp[p] = S.g[(size_t)w * nvar + p]; continue; }
                                double xq = xv[q * nvar + p];
                                double val = xq + (xv[w * nvar + p] - xq) * zz;
                                oob |= (val < o->lb[p]) || (val > o->ub[p]);
                                xp[p] = fmin(fmax(val, o->lb[p]), o->ub[p]);
                            }
                            double lpp = logp(&c, v, xp);
                            double lr = (S.nnd - 1) * log(zz) + (lpp - S.lp[(size_t)v * W + w]);
                            if (!oob && lr > log(orc_u01(u[1]))) {
                                for (int p = 0; p < nvar; ++p) xo[w * nvar + p] = o->is_global[p] ? 0.0 : xp[p];
                                S.lp[(size_t)v * W + w] = lpp;
                                ++acc;
                            } else {
                                memcpy(xo + w * nvar, xv + w * nvar, sizeof(double) * nvar);
                            }
                        }
                        for (int i = 0; i < na; ++i)
                            memcpy(xv + (a0 + i) * nvar, xo + (a0 + i) * nvar, sizeof(double) * nvar);
                    }
                }
            }
            acc_total += acc;
            prop_total += (long long)nv * W;
            /* GLOBAL block, locals held (mcmc.m:555-558, 581-626) */
            gwg_global_block(&S, k, rr, 0);
            /* thinning / burn-in (mcmc.m:560-565) */
            if (k > nb && (k - nb + 1) % o->thinning == 0 && counter < ns) {
                for (int v = 0; v < nv; ++v)
                    for (int w = 0; w < W; ++w)
                        for (int p = 0; p < nvar; ++p) {
                            double val = o->is_global[p] ? S.g[(size_t)w * nvar + p]
                                                         : S.x[((size_t)v * W + w) * nvar + p];
                            double d = val - shift[(size_t)p * nv + v];
                            sum[(size_t)p * nv + v] += d;
                            sumsq[(size_t)p * nv + v] += d * d;
                            if (r->posterior) {
                                size_t idx = (size_t)v + (size_t)nv * (w + (size_t)W * (counter + (size_t)ns * rr));
                                r->posterior[(size_t)p * nv * W * ns * rep + idx] = (float)val;
                            }
                        }
                ++counter;
            }
        }
        int missing = ns - counter;
        for (int p = 0; p < nvar; ++p)
            for (int v = 0; v < nv; ++v) {
                double d = 0.0 - shift[(size_t)p * nv + v];
                sum[(size_t)p * nv + v] += (double)missing * W * d;
                sumsq[(size_t)p * nv + v] += (double)missing * W * d * d;
            }
    }
    double nsample = (double)W * ns * rep;
    for (int p = 0; p < nvar; ++p)
        for (int v = 0; v < nv; ++v) {
            size_t i = (size_t)p * nv + v;
            double md = sum[i] / nsample;
            double var = nsample > 1 ? (sumsq[i] - sum[i] * md) / (nsample - 1.0) : 0.0;
            if (r->mean) r->mean[i] = shift[i] + md;
            if (r->std) r->std[i] = sqrt(fmax(var, 0.0));
        }
    r->n_accepted = acc_total;
    r->n_proposals = prop_total;
    free(xi); free(gi); free(lpi); free(S.x); free(S.g); free(S.lp); free(S.lpg);
    free(sum); free(sumsq); free(shift); free(pt);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Dictionary starting points, gpuNEXI.likelihood (NEXI/gpuNEXI.m:813-836):  */
/* sse = sum(wt .* (S0i - (S0i'*S) ./ dot(S,S) .* S).^2) in the direct form; */
/* [sse_new, best_index] = min(sse) keeps the first minimum; NaN never wins. */
/* ------------------------------------------------------------------------ */
void orc_dictionary_match(const double* signals, int nvox, const double* dict, int ndict, int nm,
                          const double* wt, int* best, double* best_sse) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nvox; ++i) {
        double bs = INFINITY;
        int bj = -1;
        for (int j = 0; j < ndict; ++j) {
            double d = 0.0, e = 0.0;
            for (int m = 0; m < nm; ++m) {
                double sj = dict[(size_t)m * ndict + j];
                d += signals[(size_t)m * nvox + i] * sj;
                e += sj * sj;
            }
            double c = d / e, sse = 0.0;
            for (int m = 0; m < nm; ++m) {
                double r = signals[(size_t)m * nvox + i] - c * dict[(size_t)m * ndict + j];
                sse += (wt ? wt[m] : 1.0) * r * r;
            }
            if (sse < bs) { bs = sse; bj = j; }
        }
        best[i] = bj;
        if (best_sse) best_sse[i] = bs;
    }
}
