/*
 * oracle_ecyl.c -- FP64 CPU restatement of e_cyl_iso (2.5-D elastic FDTD in
 * cylindrical coordinates r, z with azimuthal mode n, CPML).
 *
 * TEST INFRASTRUCTURE ONLY (see seismod_oracle.h).  Every cell is visited by
 * a plain loop over the padded grid (nx2 = nx + np radial columns, the PML
 * only past r = (nx-1) dr; nz2 = nz + 2 np rows, index i*nz2 + j), and
 * every update keeps the reference's order of floating-point operations
 * (built without FMA contraction) so that it follows the reference to a few
 * ulp.  Where each update is taken from:
 *   materials          e_cyl_iso.c:363-441
 *   CPML coefficients  pml.c:2107-2185 (compute_cpml_cyl)
 *   vr  update_vr_cyl  propagate.c:2706-2812, n > 0 update_vr_cyl_n :3312-3477
 *   vt  update_vt_cyl  propagate.c:2815-2905, n > 0 update_vt_cyl_n :3479-3585
 *   vz  update_vz_cyl  propagate.c:2908-2996, n > 0 update_vz_cyl_n :3587-3693
 *   trr ttt tzz        propagate.c:2999-3133, n > 0 update_taa_cyl_n :3695-3845
 *   trz update_trz_cyl propagate.c:3136-3212 (also for n > 0: e_cyl_iso.c:643)
 *   trt update_trt_cyl propagate.c:3215-3246, n > 0 update_trt_cyl_n :3958-4008
 *   ttz update_ttz_cyl propagate.c:3249-3309, n > 0 update_ttz_cyl_n :4010-4088
 *   div, curl          propagate.c:4090-4118
 *   sources            src.c:186-236 (forces, Kurkjian)
 *
 * Memory variables.  The reference keeps each CPML memory variable in a
 * compact array walked in loop order.  Here each one is addressed by its cell:
 * z-side variables in an nx2 x (2 np + 1) strip, slot zs(j) = j below the
 * interior and np + (j - (nz + np - 1)) above it; r-side variables in an
 * (np + 1) x nz2 strip, slot i - (nx - 1) for the half-node updates and
 * i - nx for the node updates.  Every cell owns its own variable in both.
 */
#include "seismod_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { ZV_TRZ, ZV_TTZ, ZV_TZZ, ZV_VZ, ZV_VR, ZV_VT, NZV };   /* z-side memory variables */
enum {
    RV_DTRR, RV_TRR1, RV_TRT1, RV_TTT1,    /* vr (node) */
    RV_TRT2, RV_DTRT, RV_TTT2,             /* vt (half node) */
    RV_DTRZ, RV_TRZ, RV_TTZ,               /* vz (half node) */
    RV_DVR, RV_VR1, RV_VT1,                /* trr ttt tzz (half node) */
    RV_DVZ,                                /* trz (node) */
    RV_DVT, RV_VR2, RV_VT2,                /* trt (node) */
    RV_VZ,                                 /* ttz (half node) */
    NRV
};

struct orc_ecyl {
    size_t nx, nz, np, nx2, nz2;
    int n;
    double dx, dz, dt;
    double *f[9];           /* vr vt vz trr ttt tzz trz trt ttz */
    double *m[8];           /* lij l2mij mu mui muj bi bj bij */
    double *c[15];          /* ik_r ik_z ikh_z b_r c_r b_z c_z bh_z ch_z | ikH_r ikH_z bH_r cH_r bH_z cH_z */
    double *zm[NZV], *rm[NRV];
};

enum { C_IKR, C_IKZ, C_IKHZ, C_BR, C_CR, C_BZ, C_CZ, C_BHZ, C_CHZ,
       C_IKHR_E, C_IKHZ_E, C_BHR_E, C_CHR_E, C_BHZ_E, C_CHZ_E };

/* ======================================================================
 * set-up
 * ====================================================================== */

static double harm2(double a, double b)
{
    if (a == 0.0 && b == 0.0) return 0.0;
    return 2. * a * b / (a + b);
}

double orc_ecyl_materials(size_t nx2, size_t nz2, const double *vp, const double *vs,
                          const double *rho, double *lij, double *l2mij, double *mu,
                          double *mui, double *muj, double *bi, double *bj, double *bij)
{
    /* e_cyl_iso.c:363-441: lambda, lambda + 2 mu and 1/rho at the cell;
     * mu averaged harmonically in z (muj), in r (mui) and over the four
     * surrounding cells (mu); 1/rho of arithmetic means in z (bj) and r (bi) */
    const size_t N = nx2 * nz2;
    double *m0 = malloc(N * sizeof *m0);
    double vpmax = 0.0;
    for (size_t k = 0; k < N; ++k) {
        vpmax = vp[k] > vpmax ? vp[k] : vpmax;
        lij[k] = rho[k] * (vp[k] * vp[k] - 2. * vs[k] * vs[k]);
        m0[k] = rho[k] * vs[k] * vs[k];
        l2mij[k] = lij[k] + 2.0 * m0[k];
        bij[k] = 1. / rho[k];
    }
    for (size_t i = 0; i < nx2; ++i) {
        const size_t r = i * nz2;
        muj[r] = m0[r];
        bj[r] = bij[r];
        for (size_t j = 1; j < nz2; ++j) {
            muj[r + j] = harm2(m0[r + j], m0[r + j - 1]);
            bj[r + j] = 1. / ((rho[r + j] + rho[r + j - 1]) / 2.0);
        }
    }
    for (size_t j = 0; j < nz2; ++j) {
        mui[j] = m0[j];
        bi[j] = 1. / rho[j];
        for (size_t i = 1; i < nx2; ++i) {
            const size_t k = i * nz2 + j, w = k - nz2;
            mui[k] = harm2(m0[k], m0[w]);
            bi[k] = 1. / ((rho[k] + rho[w]) / 2.0);
        }
    }
    mu[0] = m0[0];
    for (size_t j = 1; j < nz2; ++j) mu[j] = harm2(m0[j], m0[j - 1]);
    for (size_t i = 1; i < nx2; ++i) {
        const size_t r = i * nz2;
        mu[r] = harm2(m0[r], m0[r - nz2]);
        for (size_t j = 1; j < nz2; ++j) {
            const double a = m0[r + j], b = m0[r + j - 1], c = m0[r - nz2 + j],
                         d = m0[r - nz2 + j - 1];
            /* zero when any two of the four are zero (each triple product
             * vanishes), else the four-point harmonic mean */
            if (b * c * d == 0.0 && a * c * d == 0.0 && a * b * d == 0.0 && a * b * c == 0.0)
                mu[r + j] = 0.0;
            else
                mu[r + j] = 4. * a * b * c * d / (b * c * d + a * c * d + a * b * d + a * b * c);
        }
    }
    free(m0);
    return vpmax;
}

void orc_ecyl_cpml(size_t np, double dx, double dz, double dt, double order, double vmax,
                   double Rc, double kappa_max, double alpha_max, int absorb,
                   double *const *c)
{
    /* pml.c:2107-2185 compute_cpml_cyl.  As there, the z half-node kappa
     * uses dx / Lx and the end-of-grid alpha uses alpha_max / (np + 1). */
    const double Lx = np * dx, Lz = np * dz;
    const double d0x = -(order + 1.) * vmax * log(Rc) / (2. * Lx);
    const double d0z = -(order + 1.) * vmax * log(Rc) / (2. * Lz);
    const double da = alpha_max / np, da2 = alpha_max / (np + 1);
    for (size_t n = 0; n < np; ++n) {
        if (!absorb) {
            c[C_IKR][n] = c[C_IKZ][n] = c[C_IKHZ][n] = 1.;
            c[C_BR][n] = c[C_CR][n] = c[C_BZ][n] = c[C_CZ][n] = c[C_BHZ][n] = c[C_CHZ][n] = 0.;
            continue;
        }
        const double kr = 1. + (kappa_max - 1.) * pow(((np - n) * dx / Lx), order);
        const double kz = 1. + (kappa_max - 1.) * pow(((np - n) * dz / Lz), order);
        const double khz = 1. + (kappa_max - 1.) * pow(((np - n - 0.5) * dx / Lx), order);
        c[C_IKR][n] = 1. / kr;
        c[C_IKZ][n] = 1. / kz;
        c[C_IKHZ][n] = 1. / khz;
        const double d_x = d0x * pow(((np - n) * dx / Lx), order), a_x = n * da;
        c[C_BR][n] = exp(-(d_x / kr + a_x) * dt);
        c[C_CR][n] = d_x * (c[C_BR][n] - 1.) / (kr * (d_x + kr * a_x));
        const double d_z = d0z * pow(((np - n) * dz / Lz), order), a_z = n * da;
        const double dh_z = d0z * pow(((np - n - 0.5) * dz / Lz), order), ah_z = (n + 0.5) * da;
        c[C_BZ][n] = exp(-(d_z / kz + a_z) * dt);
        c[C_CZ][n] = d_z * (c[C_BZ][n] - 1.) / (kz * (d_z + kz * a_z));
        c[C_BHZ][n] = exp(-(dh_z / khz + ah_z) * dt);
        c[C_CHZ][n] = dh_z * (c[C_BHZ][n] - 1.) / (khz * (dh_z + khz * ah_z));
    }
    for (size_t n = 0; n < np + 1; ++n) {
        if (!absorb) {
            c[C_IKHR_E][n] = c[C_IKHZ_E][n] = 1.;
            c[C_BHR_E][n] = c[C_CHR_E][n] = c[C_BHZ_E][n] = c[C_CHZ_E][n] = 0.;
            continue;
        }
        const double kHr = 1. + (kappa_max - 1.) * pow(((n + 0.5) * dx / Lx), order);
        const double kHz = 1. + (kappa_max - 1.) * pow(((n + 0.5) * dz / Lz), order);
        c[C_IKHR_E][n] = 1. / kHr;
        c[C_IKHZ_E][n] = 1. / kHz;
        const double dHx = d0x * pow(((n + 0.5) * dx / Lx), order), aHx = (np - n - 0.5) * da2;
        c[C_BHR_E][n] = exp(-(dHx / kHr + aHx) * dt);
        c[C_CHR_E][n] = dHx * (c[C_BHR_E][n] - 1.) / (kHr * (dHx + kHr * aHx));
        const double dHz = d0z * pow(((n + 0.5) * dz / Lz), order), aHz = (np - n - 0.5) * da2;
        c[C_BHZ_E][n] = exp(-(dHz / kHz + aHz) * dt);
        c[C_CHZ_E][n] = dHz * (c[C_BHZ_E][n] - 1.) / (kHz * (dHz + kHz * aHz));
    }
}

size_t orc_ecyl_kurkjian(double A, double f, double dt, double lij_at_src, double x_src,
                         double dx, double dz, int n, size_t maxlen, double *fct)
{
    /* src.c:202-228: a Ricker of peak 1 scaled by A times
     * lambda / (2 pi) eps_m 2 / (dx^2 dz) (x / dx)^n, eps_m = 1 (n = 0) or 2 */
    const double pi = 4.0 * atan(1.0), pi2 = pi * pi;
    const double eps = n > 0 ? 2.0 : 1.0;
    const double term = lij_at_src / (2. * pi) * eps * 2. / (dx * dx * dz) * pow(x_src / dx, n);
    const double tcut = 1.0 / f;
    size_t len = (size_t)ceil(tcut * 2.0 / dt);
    if (len > maxlen) len = maxlen;
    double amax = 0.0;
    for (size_t i = 0; i < len; ++i) {
        const double time = i * dt - tcut;
        const double K = pi2 * f * f * time * time;
        fct[i] = 2. * pi2 * f * f * (1.0 - 2.0 * K) * exp(-K);
        amax = amax > fabs(fct[i]) ? amax : fabs(fct[i]);
    }
    for (size_t i = 0; i < len; ++i) fct[i] *= A / amax * term;
    return len;
}

orc_ecyl *orc_ecyl_new(size_t nx, size_t nz, size_t np, int n, double dx, double dz, double dt,
                       const double *const *mat, const double *const *coef)
{
    orc_ecyl *o = calloc(1, sizeof *o);
    o->nx = nx;
    o->nz = nz;
    o->np = np;
    o->nx2 = nx + np;
    o->nz2 = nz + 2 * np;
    o->n = n;
    o->dx = dx;
    o->dz = dz;
    o->dt = dt;
    const size_t N = o->nx2 * o->nz2;
    for (int k = 0; k < 9; ++k) o->f[k] = calloc(N, sizeof(double));
    for (int k = 0; k < 8; ++k) {
        o->m[k] = malloc(N * sizeof(double));
        memcpy(o->m[k], mat[k], N * sizeof(double));
    }
    for (int k = 0; k < 15; ++k) {
        const size_t len = k < 9 ? np : np + 1;
        o->c[k] = malloc(len * sizeof(double));
        memcpy(o->c[k], coef[k], len * sizeof(double));
    }
    for (int k = 0; k < NZV; ++k) o->zm[k] = calloc(o->nx2 * (2 * np + 1), sizeof(double));
    for (int k = 0; k < NRV; ++k) o->rm[k] = calloc((np + 1) * o->nz2, sizeof(double));
    return o;
}

void orc_ecyl_free(orc_ecyl *o)
{
    if (!o) return;
    for (int k = 0; k < 9; ++k) free(o->f[k]);
    for (int k = 0; k < 8; ++k) free(o->m[k]);
    for (int k = 0; k < 15; ++k) free(o->c[k]);
    for (int k = 0; k < NZV; ++k) free(o->zm[k]);
    for (int k = 0; k < NRV; ++k) free(o->rm[k]);
    free(o);
}

/* ======================================================================
 * the step
 * ====================================================================== */

#define F(k, i, j) (o->f[k][(i) * o->nz2 + (j)])
#define M(k, i, j) (o->m[k][(i) * o->nz2 + (j)])
enum { VR, VT, VZ, TRR, TTT, TZZ, TRZ, TRT, TTZ };
enum { LIJ, L2M, MU, MUI, MUJ, BI, BJ, BIJ };

/* CPML filter of a derivative d: psi = b psi + c d, returns ik d + psi */
static double cpml(double *psi, double b, double c, double ik, double d)
{
    *psi = b * *psi + c * d;
    return ik * d + *psi;
}

static double *zvar(orc_ecyl *o, int v, size_t i, size_t j)
{
    const size_t np = o->np;
    const size_t s = j < np ? j : np + (j - (o->nz + np - 1));
    return &o->zm[v][i * (2 * np + 1) + s];
}

static double *rvar(orc_ecyl *o, int v, size_t slot, size_t j)
{
    return &o->rm[v][slot * o->nz2 + j];
}

/* z filter of the "half node" kind (vr, vt, taa): rows [0, np) with the
 * h coefficients, rows [nz+np-1, nz2-1) with the H coefficients */
static double zfilt_half(orc_ecyl *o, int v, size_t i, size_t j, double d)
{
    const size_t np = o->np, top = o->nz + np - 1;
    if (j < np) return cpml(zvar(o, v, i, j), o->c[C_BHZ][j], o->c[C_CHZ][j], o->c[C_IKHZ][j], d);
    if (j >= top) {
        const size_t jj = j - top;
        return cpml(zvar(o, v, i, j), o->c[C_BHZ_E][jj], o->c[C_CHZ_E][jj], o->c[C_IKHZ_E][jj], d);
    }
    return d;
}

/* z filter of the "node" kind (vz, ttz): rows [1, np) with the node
 * coefficients, rows [nz+np, nz2) with them mirrored */
static double zfilt_node(orc_ecyl *o, int v, size_t i, size_t j, double d)
{
    const size_t np = o->np, top = o->nz + np;
    if (j < np) return cpml(zvar(o, v, i, j), o->c[C_BZ][j], o->c[C_CZ][j], o->c[C_IKZ][j], d);
    if (j >= top) {
        const size_t k = np - 1 - (j - top);
        return cpml(zvar(o, v, i, j), o->c[C_BZ][k], o->c[C_CZ][k], o->c[C_IKZ][k], d);
    }
    return d;
}

/* z filter of trz: rows [1, np) with the h coefficients, rows [nz+np, nz2)
 * with the H coefficients */
static double zfilt_trz(orc_ecyl *o, size_t i, size_t j, double d)
{
    const size_t np = o->np, top = o->nz + np;
    if (j < np) return cpml(zvar(o, ZV_VR, i, j), o->c[C_BHZ][j], o->c[C_CHZ][j], o->c[C_IKHZ][j], d);
    if (j >= top) {
        const size_t jj = j - top;
        return cpml(zvar(o, ZV_VR, i, j), o->c[C_BHZ_E][jj], o->c[C_CHZ_E][jj], o->c[C_IKHZ_E][jj], d);
    }
    return d;
}

/* the value one row below (i, j) in the flat array, as the reference reads
 * it: with no PML (np = 0, the abs 0 case) the vz, trz and ttz loops start
 * at row 0 and read row -1, which is the last row of column i-1; at the
 * axis (i = 0) that read lands before the array and is taken as zero */
static double below(const orc_ecyl *o, int k, size_t i, size_t j)
{
    const size_t q = i * o->nz2 + j;
    return q == 0 ? 0.0 : o->f[k][q - 1];
}

/* first row the vz, trz and ttz updates touch: 1, or 0 without a PML */
static size_t jfirst(const orc_ecyl *o) { return o->np ? 1 : 0; }

static int zpml_half(const orc_ecyl *o, size_t j) { return j < o->np || j >= o->nz + o->np - 1; }
static int zpml_node(const orc_ecyl *o, size_t j) { return j < o->np || j >= o->nz + o->np; }

/* r filters: node kind (i >= nx, mirrored node coefficients) and half-node
 * kind (i >= nx-1, the H coefficients) */
static double rfilt_node(orc_ecyl *o, int v, size_t i, size_t j, double d)
{
    const size_t ii = i - o->nx, k = o->np - 1 - ii;
    return cpml(rvar(o, v, ii, j), o->c[C_BR][k], o->c[C_CR][k], o->c[C_IKR][k], d);
}
static double rfilt_half(orc_ecyl *o, int v, size_t i, size_t j, double d)
{
    const size_t ii = i - (o->nx - 1);
    return cpml(rvar(o, v, ii, j), o->c[C_BHR_E][ii], o->c[C_CHR_E][ii], o->c[C_IKHR_E][ii], d);
}

static void ecyl_vr(orc_ecyl *o)
{
    const double dx = o->dx, dz = o->dz;
    const int n = o->n;
    const size_t i0 = (n % 2) ? 0 : 1;
    for (size_t i = i0; i < o->nx2; ++i) {
        for (size_t j = 0; j + 1 < o->nz2; ++j) {
            double ddz = (F(TRZ, i, j + 1) - F(TRZ, i, j)) / dz;
            if (zpml_half(o, j)) ddz = zfilt_half(o, ZV_TRZ, i, j, ddz);
            double s;
            if (i == 0) {
                /* odd n, on the axis: trr is antisymmetric across it */
                s = (F(TRR, i, j) - -F(TRR, i, j)) / dx + ddz;
            } else if (i < o->nx) {
                const double a = (F(TRR, i, j) - F(TRR, i - 1, j)) / dx;
                const double b = (F(TRR, i, j) + F(TRR, i - 1, j)) / (2. * i * dx);
                const double c = (F(TTT, i, j) + F(TTT, i - 1, j)) / (2. * i * dx);
                s = n > 0 ? a + b + n * F(TRT, i, j) / (i * dx) - c + ddz : a + b - c + ddz;
            } else {
                const double a = rfilt_node(o, RV_DTRR, i, j, (F(TRR, i, j) - F(TRR, i - 1, j)) / dx);
                const double b = rfilt_node(o, RV_TRR1, i, j,
                                            (F(TRR, i, j) + F(TRR, i - 1, j)) / (2. * i * dx));
                const double c = rfilt_node(o, RV_TTT1, i, j,
                                            (F(TTT, i, j) + F(TTT, i - 1, j)) / (2. * i * dx));
                if (n > 0) {
                    const double d2 = rfilt_node(o, RV_TRT1, i, j, F(TRT, i, j) / (i * dx));
                    s = a + b + n * d2 - c + ddz;
                } else {
                    s = a + b - c + ddz;
                }
            }
            F(VR, i, j) += o->dt * M(BJ, i, j) * s;
        }
    }
}

static void ecyl_vt(orc_ecyl *o)
{
    const double dx = o->dx, dz = o->dz;
    const int n = o->n;
    for (size_t i = 0; i + 1 < o->nx2; ++i) {
        for (size_t j = 0; j + 1 < o->nz2; ++j) {
            double ddz = (F(TTZ, i, j + 1) - F(TTZ, i, j)) / dz;
            if (zpml_half(o, j)) ddz = zfilt_half(o, ZV_TTZ, i, j, ddz);
            const double a = (F(TRT, i + 1, j) + F(TRT, i, j)) / ((i + 0.5) * dx);
            const double b = (F(TRT, i + 1, j) - F(TRT, i, j)) / dx;
            double s;
            if (i + 1 < o->nx) {
                s = n > 0 ? a + b - n * F(TTT, i, j) / ((i + 0.5) * dx) + ddz : a + b + ddz;
            } else {
                const double fa = rfilt_half(o, RV_TRT2, i, j, a);
                const double fb = rfilt_half(o, RV_DTRT, i, j, b);
                if (n > 0) {
                    const double d2 = rfilt_half(o, RV_TTT2, i, j, F(TTT, i, j) / ((i + 0.5) * dx));
                    s = fa + fb - n * d2 + ddz;
                } else {
                    s = fa + fb + ddz;
                }
            }
            F(VT, i, j) += o->dt * M(BIJ, i, j) * s;
        }
    }
}

static void ecyl_vz(orc_ecyl *o)
{
    const double dx = o->dx, dz = o->dz;
    const int n = o->n;
    for (size_t i = 0; i + 1 < o->nx2; ++i) {
        for (size_t j = jfirst(o); j < o->nz2; ++j) {
            double ddz = (F(TZZ, i, j) - below(o, TZZ, i, j)) / dz;
            if (zpml_node(o, j)) ddz = zfilt_node(o, ZV_TZZ, i, j, ddz);
            const double a = (F(TRZ, i + 1, j) - F(TRZ, i, j)) / dx;
            const double b = (F(TRZ, i + 1, j) + F(TRZ, i, j)) / (2. * (i + 0.5) * dx);
            double s;
            if (i + 1 < o->nx) {
                s = n > 0 ? ddz + a + b + n * F(TTZ, i, j) / ((i + 0.5) * dx) : ddz + a + b;
            } else {
                const double fa = rfilt_half(o, RV_DTRZ, i, j, a);
                const double fb = rfilt_half(o, RV_TRZ, i, j, b);
                if (n > 0) {
                    const double d2 = rfilt_half(o, RV_TTZ, i, j, F(TTZ, i, j) / ((i + 0.5) * dx));
                    s = ddz + fa + fb + n * d2;
                } else {
                    s = ddz + fa + fb;
                }
            }
            F(VZ, i, j) += o->dt * M(BI, i, j) * s;
        }
    }
}

static void ecyl_taa(orc_ecyl *o)
{
    const double dx = o->dx, dz = o->dz, dt = o->dt;
    const int n = o->n;
    for (size_t i = 0; i + 1 < o->nx2; ++i) {
        for (size_t j = 0; j + 1 < o->nz2; ++j) {
            double dvrdr = (F(VR, i + 1, j) - F(VR, i, j)) / dx;
            double vrr = (F(VR, i + 1, j) + F(VR, i, j)) / (2. * (i + 0.5) * dx);
            double vtr = n > 0 ? F(VT, i, j) / ((i + 0.5) * dx) : 0.0;
            double dvzdz = (F(VZ, i, j + 1) - F(VZ, i, j)) / dz;
            if (i + 1 >= o->nx) {
                dvrdr = rfilt_half(o, RV_DVR, i, j, dvrdr);
                vrr = rfilt_half(o, RV_VR1, i, j, vrr);
                if (n > 0) vtr = rfilt_half(o, RV_VT1, i, j, vtr);
            }
            if (zpml_half(o, j)) dvzdz = zfilt_half(o, ZV_VZ, i, j, dvzdz);
            const double l2m = M(L2M, i, j), l = M(LIJ, i, j);
            if (n > 0) {
                F(TRR, i, j) += dt * l2m * dvrdr + dt * l * (vrr + n * vtr + dvzdz);
                F(TTT, i, j) += dt * l2m * (vrr + n * vtr) + dt * l * (dvrdr + dvzdz);
                F(TZZ, i, j) += dt * l2m * dvzdz + dt * l * (dvrdr + vrr + n * vtr);
            } else {
                F(TRR, i, j) += dt * l2m * dvrdr + dt * l * (vrr + dvzdz);
                F(TTT, i, j) += dt * l2m * vrr + dt * l * (dvrdr + dvzdz);
                F(TZZ, i, j) += dt * l2m * dvzdz + dt * l * (dvrdr + vrr);
            }
        }
    }
}

static void ecyl_trz(orc_ecyl *o)
{
    const double dx = o->dx, dz = o->dz;
    for (size_t i = 1; i < o->nx2; ++i) {
        for (size_t j = jfirst(o); j < o->nz2; ++j) {
            double ddz = (F(VR, i, j) - below(o, VR, i, j)) / dz;
            if (zpml_node(o, j)) ddz = zfilt_trz(o, i, j, ddz);
            double ddr = (F(VZ, i, j) - F(VZ, i - 1, j)) / dx;
            if (i >= o->nx) {
                const size_t ii = i - o->nx;
                ddr = cpml(rvar(o, RV_DVZ, ii, j), o->c[C_BHR_E][ii], o->c[C_CHR_E][ii],
                           o->c[C_IKHR_E][ii], ddr);
            }
            F(TRZ, i, j) += o->dt * M(MU, i, j) * (ddz + ddr);
        }
    }
}

static void ecyl_trt(orc_ecyl *o)
{
    const double dx = o->dx;
    const int n = o->n;
    const size_t i0 = (n % 2) ? 0 : 1;
    for (size_t i = i0; i < o->nx2; ++i) {
        for (size_t j = 0; j < o->nz2; ++j) {
            double s;
            if (i == 0) {
                s = (F(VT, i, j) - -F(VT, i, j)) / dx;   /* odd n, on the axis */
            } else if (i < o->nx) {
                const double a = (F(VT, i, j) - F(VT, i - 1, j)) / dx;
                const double c = (F(VT, i, j) + F(VT, i - 1, j)) / (2. * i * dx);
                s = n > 0 ? a - n * F(VR, i, j) / (i * dx) - c : a - c;
            } else {
                const double a = rfilt_node(o, RV_DVT, i, j, (F(VT, i, j) - F(VT, i - 1, j)) / dx);
                const double c = rfilt_node(o, RV_VT2, i, j,
                                            (F(VT, i, j) + F(VT, i - 1, j)) / (2. * i * dx));
                if (n > 0) {
                    const double b = rfilt_node(o, RV_VR2, i, j, F(VR, i, j) / (i * dx));
                    s = a - n * b - c;
                } else {
                    s = a - c;
                }
            }
            F(TRT, i, j) += o->dt * M(MUJ, i, j) * s;
        }
    }
}

static void ecyl_ttz(orc_ecyl *o)
{
    const double dx = o->dx, dz = o->dz, dt = o->dt;
    const int n = o->n;
    for (size_t i = 0; i + 1 < o->nx2; ++i) {
        for (size_t j = jfirst(o); j < o->nz2; ++j) {
            const int zp = zpml_node(o, j);
            const double diff = F(VT, i, j) - below(o, VT, i, j);
            const double mui = M(MUI, i, j);
            if (n == 0) {
                /* interior rows: dt mui (vt_j - vt_j-1) / dz, divided last */
                if (zp)
                    F(TTZ, i, j) += dt * mui * zfilt_node(o, ZV_VT, i, j, diff / dz);
                else
                    F(TTZ, i, j) += dt * mui * diff / dz;
                continue;
            }
            const double ddz = zp ? zfilt_node(o, ZV_VT, i, j, diff / dz) : diff / dz;
            double s;
            if (i + 1 < o->nx) {
                s = ddz - n * F(VZ, i, j) / ((i + 0.5) * dx);
            } else {
                const double vzr = rfilt_half(o, RV_VZ, i, j, F(VZ, i, j) / ((i + 0.5) * dx));
                s = ddz - n * vzr;
            }
            F(TTZ, i, j) += dt * mui * s;
        }
    }
}

void orc_ecyl_velocity(orc_ecyl *o)
{
    ecyl_vr(o);
    ecyl_vt(o);
    ecyl_vz(o);
}

void orc_ecyl_stress(orc_ecyl *o)
{
    ecyl_taa(o);
    ecyl_trz(o);
    ecyl_trt(o);
    ecyl_ttz(o);
}

void orc_ecyl_force(orc_ecyl *o, size_t index, int type, double value)
{
    /* src.c:186-199: dt b value into vr (Fr, Bulk), vt (Ftheta), vz (Fz, Bulk) */
    if (type == ORC_C_SRC_FR || type == ORC_C_SRC_BULK)
        o->f[VR][index] += o->dt * o->m[BJ][index] * value;
    if (type == ORC_C_SRC_FT) o->f[VT][index] += o->dt * o->m[BIJ][index] * value;
    if (type == ORC_C_SRC_FZ || type == ORC_C_SRC_BULK)
        o->f[VZ][index] += o->dt * o->m[BI][index] * value;
}

void orc_ecyl_kurkjian_add(orc_ecyl *o, size_t index, double value)
{
    /* src.c:231-236 */
    o->f[TRR][index] += o->dt * value;
    o->f[TZZ][index] += o->dt * value;
}

void orc_ecyl_get(const orc_ecyl *o, int field, double *out)
{
    memcpy(out, o->f[field], o->nx2 * o->nz2 * sizeof(double));
}

void orc_ecyl_set(orc_ecyl *o, int field, const double *in)
{
    memcpy(o->f[field], in, o->nx2 * o->nz2 * sizeof(double));
}

double orc_ecyl_probe(const orc_ecyl *o, int comp, size_t index)
{
    if (comp < ORC_C_DIV) return o->f[comp][index];
    const size_t i = index / o->nz2, j = index % o->nz2;
    const double dx = o->dx, dz = o->dz;
    if (comp == ORC_C_DIV) {
        /* propagate.c:4090-4100 (the radial term is not divided by dr there) */
        if (i + 1 >= o->nx2 || j + 1 >= o->nz2) return 0.0;
        return ((i + 1) * F(VR, i + 1, j) - i * F(VR, i, j)) / (i + 0.5) +
               o->n * F(VT, i, j) / ((i + 0.5) * dx) + (F(VZ, i, j + 1) - F(VZ, i, j)) / dz;
    }
    /* curl, propagate.c:4102-4118 */
    if (j == 0) return 0.0;
    if (i == 0) {
        if (!(o->n % 2)) return 0.0;
        return (F(VR, i, j) - F(VR, i, j - 1)) / dz - (F(VZ, i, j) - -F(VZ, i, j)) / dx;
    }
    return (F(VR, i, j) - F(VR, i, j - 1)) / dz - (F(VZ, i, j) - F(VZ, i - 1, j)) / dx;
}
