/*
 * seismod_oracle.c -- FP64 CPU restatement of the seismod FDTD hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see seismod_oracle.h).  Written for clarity, not
 * speed: every cell is visited by a plain loop, and every update keeps the
 * reference's order of floating-point operations so that, built without
 * FMA contraction, it agrees with the reference bit for bit or to a few ulp.
 */
#include "seismod_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ======================================================================
 * loops over independent planes split across host threads (the a_iso_3d
 * sweeps at full grid sizes).  Every cell is still computed by the same
 * expression in the same order, so the results do not depend on the
 * thread count.  ORC_THREADS sets the count (default: online cores, <= 64).
 * ====================================================================== */

typedef void (*orc_range_fn)(void *ctx, size_t lo, size_t hi);

struct orc_job {
    orc_range_fn fn;
    void *ctx;
    size_t lo, hi;
};

static void *orc_job_run(void *p)
{
    struct orc_job *j = p;
    j->fn(j->ctx, j->lo, j->hi);
    return NULL;
}

static int orc_threads(void)
{
    const char *e = getenv("ORC_THREADS");
    long n = e ? atol(e) : sysconf(_SC_NPROCESSORS_ONLN);
    if (n < 1) n = 1;
    if (n > 64) n = 64;
    return (int)n;
}

static void orc_parallel(size_t n, orc_range_fn fn, void *ctx)
{
    int nt = orc_threads();
    if ((size_t)nt > n) nt = (int)n;
    if (nt <= 1) {
        fn(ctx, 0, n);
        return;
    }
    pthread_t th[64];
    struct orc_job jobs[64];
    int started[64];
    for (int t = 0; t < nt; ++t) {
        jobs[t].fn = fn;
        jobs[t].ctx = ctx;
        jobs[t].lo = n * (size_t)t / (size_t)nt;
        jobs[t].hi = n * (size_t)(t + 1) / (size_t)nt;
        started[t] = t > 0 && pthread_create(&th[t], NULL, orc_job_run, &jobs[t]) == 0;
        if (t > 0 && !started[t]) fn(ctx, jobs[t].lo, jobs[t].hi);
    }
    fn(ctx, jobs[0].lo, jobs[0].hi);
    for (int t = 1; t < nt; ++t)
        if (started[t]) pthread_join(th[t], NULL);
}

/* ======================================================================
 * shared set-up
 * ====================================================================== */

size_t orc_src_len(double f, double dt0, double fac)
{
    /* src.c:47-48: length = ceil(2 tcut / dt), tcut = 1/f */
    double dt = fac * dt0;
    double tcut = 1.0 / f;
    return (size_t)ceil(tcut * 2.0 / dt);
}

void orc_src_fct(size_t n, const double *A, const double *f, double dt0, double fac,
                 size_t maxlen, double *fct, size_t *len)
{
    /* src.c:43-65.  Each pass n computes wavelet n, measures the peak of
     * wavelet 0 over len[n] samples and rescales wavelet 0 by A[n]/peak.
     * With one source this normalises its peak to A.  The reference reads
     * wavelet 0 past its end when len[n] > len[0]; this restatement stops at
     * the shorter length instead. */
    const double pi = 4.0 * atan(1.0);
    const double pi2 = pi * pi;
    double dt = fac * dt0;
    for (size_t s = 0; s < n; ++s) {
        double tcut = 1.0 / f[s];
        len[s] = (size_t)ceil(tcut * 2.0 / dt);
        if (len[s] > maxlen) len[s] = maxlen;
        double *w = fct + s * maxlen;
        double amax = 0.0;
        for (size_t i = 0; i < len[s]; ++i) {
            double time = i * dt - tcut;
            double K = pi2 * f[s] * f[s] * time * time;
            w[i] = A[s] * 2. * pi2 * f[s] * f[s] * (1.0 - 2.0 * K) * exp(-K);
            if (i < len[0]) {
                double a0 = fabs(fct[i]);
                amax = amax > a0 ? amax : a0;
            }
        }
        for (size_t i = 0; i < len[0]; ++i) fct[i] *= A[s] / amax;
    }
}

size_t orc_nsteps(double duration, double dt)
{
    size_t nsteps = (size_t)(duration / dt);
    if (nsteps * dt < duration) nsteps++;
    return nsteps;
}

int orc_sample(size_t it, double dt, double t0, double rdt)
{
    double t = dt * (it + 1);
    double dt2 = t - t0 + 1.e-15;
    double rem = fmod(1.e6 * dt2, 1.e6 * rdt);
    return (fabs(dt2) < 0.99 * dt) || (t > t0 && rdt > 0.0 && fabs(rem) < 1.e-8);
}

/* ======================================================================
 * e_iso
 * ====================================================================== */

double orc_eiso_materials(size_t nx, size_t nz, const double *vp, const double *vs,
                          const double *rho, double *la, double *mu, double *l2m,
                          double *b, double *bm)
{
    /* e_iso.c:423-462: nodal lambda, mu, lambda+2mu, 1/rho; mu averaged
     * along z, lambda and lambda+2mu along x, 1/rho over the 4 corners of
     * the vz node; the last row/column fall back to 2-point or nodal. */
    size_t n = nx * nz;
    double *lat = malloc(n * sizeof(double));
    double *mut = malloc(n * sizeof(double));
    double *l2t = malloc(n * sizeof(double));
    double vpmax = 0.0;
    for (size_t q = 0; q < n; ++q) {
        vpmax = vp[q] > vpmax ? vp[q] : vpmax;
        lat[q] = rho[q] * (vp[q] * vp[q] - 2. * vs[q] * vs[q]);
        mut[q] = rho[q] * vs[q] * vs[q];
        l2t[q] = lat[q] + 2. * mut[q];
        b[q] = 1. / rho[q];
    }
    for (size_t i = 0; i < nx; ++i) {
        for (size_t j = 0; j + 1 < nz; ++j)
            mu[i * nz + j] = (mut[i * nz + j] + mut[i * nz + j + 1]) / 2.0;
        mu[i * nz + nz - 1] = mut[i * nz + nz - 1];
    }
    for (size_t j = 0; j < nz; ++j) {
        for (size_t i = 0; i + 1 < nx; ++i) {
            la[i * nz + j] = (lat[i * nz + j] + lat[(i + 1) * nz + j]) / 2.0;
            l2m[i * nz + j] = (l2t[i * nz + j] + l2t[(i + 1) * nz + j]) / 2.0;
        }
        la[(nx - 1) * nz + j] = lat[(nx - 1) * nz + j];
        l2m[(nx - 1) * nz + j] = l2t[(nx - 1) * nz + j];
    }
    for (size_t i = 0; i + 1 < nx; ++i) {
        for (size_t j = 0; j + 1 < nz; ++j)
            bm[i * nz + j] = (b[i * nz + j] + b[(i + 1) * nz + j] +
                              b[i * nz + j + 1] + b[(i + 1) * nz + j + 1]) / 4.0;
        bm[i * nz + nz - 1] = (b[i * nz + nz - 1] + b[(i + 1) * nz + nz - 1]) / 2.0;
    }
    for (size_t j = 0; j + 1 < nz; ++j)
        bm[(nx - 1) * nz + j] = (b[(nx - 1) * nz + j] + b[(nx - 1) * nz + j + 1]) / 2.0;
    bm[nx * nz - 1] = b[nx * nz - 1];
    free(lat);
    free(mut);
    free(l2t);
    return vpmax;
}

void orc_eiso_profiles(size_t np, double h, size_t ncell, const double *vp,
                       double *d, double *dh, double *dH)
{
    /* e_iso.c:486-500: d0 = ln(1/R) 3/2 vbar / (np h), R = 1e-3, order 2,
     * vbar = MEAN of vp over the interior. */
    double vbar = 0.0;
    for (size_t q = 0; q < ncell; ++q) vbar += vp[q];
    vbar /= (double)ncell;
    double R = 0.001;
    double delta = np * h;
    double d0 = log(1. / R) * 3. / 2. * vbar / delta;
    for (size_t n = 0; n < np; ++n) {
        d[n] = d0 * pow(((np - n) * h / delta), 2);
        dh[n] = d0 * pow((((np - n) * h - h / 2.) / delta), 2);
    }
    for (size_t n = 0; n < np + 1; ++n)
        dH[n] = d0 * pow((((np - n) * h + h / 2.) / delta), 2);
}

static void bfp_round_rows(double *f, size_t nrows, size_t n, int B);
static void bfp_round_cols(double *f, size_t nrows, size_t n, int B);
static void bfp_round_strided(double *v, size_t stride, size_t n);

struct orc_eiso {
    size_t nx, nz, np, NX, NZ;
    double h, dt;
    const double *mat[5];      /* b, bm, la, l2m, mu: interior, i*nz+j */
    double *d, *dh, *dH;
    double *f[5], *fx[5], *fz[5];
    int bfp_block;             /* 0: FP64 storage; else block floating point */
    int bfp_axis;              /* blocks along X (0) or Z (1) */
    /* rectangles of cells the block storage keeps exact (source patches) */
    int npatch;
    long patch[16][4];         /* first X, first Z, rows, columns */
};

enum { M_B = 0, M_BM = 1, M_LA = 2, M_L2M = 3, M_MU = 4 };

orc_eiso *orc_eiso_new(size_t nx, size_t nz, size_t np, double h, double dt,
                       const double *la, const double *mu, const double *l2m,
                       const double *b, const double *bm,
                       const double *d, const double *dh, const double *dH)
{
    orc_eiso *o = calloc(1, sizeof(*o));
    o->nx = nx; o->nz = nz; o->np = np;
    o->NX = nx + 2 * np; o->NZ = nz + 2 * np;
    o->h = h; o->dt = dt;
    size_t n = nx * nz;
    double *m = malloc(5 * n * sizeof(double));
    memcpy(m + 0 * n, b, n * sizeof(double));
    memcpy(m + 1 * n, bm, n * sizeof(double));
    memcpy(m + 2 * n, la, n * sizeof(double));
    memcpy(m + 3 * n, l2m, n * sizeof(double));
    memcpy(m + 4 * n, mu, n * sizeof(double));
    for (int k = 0; k < 5; ++k) o->mat[k] = m + k * n;
    o->d = malloc((3 * np + 1) * sizeof(double));
    o->dh = o->d + np;
    o->dH = o->d + 2 * np;
    memcpy(o->d, d, np * sizeof(double));
    memcpy(o->dh, dh, np * sizeof(double));
    memcpy(o->dH, dH, (np + 1) * sizeof(double));
    size_t N = o->NX * o->NZ;
    for (int k = 0; k < 5; ++k) {
        o->f[k] = calloc(N, sizeof(double));
        o->fx[k] = calloc(N, sizeof(double));
        o->fz[k] = calloc(N, sizeof(double));
    }
    return o;
}

void orc_eiso_free(orc_eiso *o)
{
    if (!o) return;
    free((void *)o->mat[0]);
    free(o->d);
    for (int k = 0; k < 5; ++k) { free(o->f[k]); free(o->fx[k]); free(o->fz[k]); }
    free(o);
}

/* a cell of a rectangle the block storage keeps exact */
static int e_in_patch(const orc_eiso *o, long X, long Z)
{
    for (int q = 0; q < o->npatch; ++q) {
        const long *p = o->patch[q];
        if (X >= p[0] && X < p[0] + p[2] && Z >= p[1] && Z < p[1] + p[3]) return 1;
    }
    return 0;
}

static int e_interior(const orc_eiso *o, long X, long Z)
{
    return X >= (long)o->np && X < (long)(o->np + o->nx) &&
           Z >= (long)o->np && Z < (long)(o->np + o->nz);
}

/* value a neighbour read sees: the total inside, x part + z part in the
 * frame (pml.c reads "q_x[..] + q_z[..]"), zero beyond the outer edge
 * (the "= 0." terms of pml.c, e.g. pml.c:50,76,488,545). */
static double e_val(const orc_eiso *o, int k, long X, long Z)
{
    if (X < 0 || Z < 0 || X >= (long)o->NX || Z >= (long)o->NZ) return 0.0;
    size_t q = (size_t)X * o->NZ + (size_t)Z;
    /* block storage keeps the frame's totals as stored (rounded) values */
    if (e_interior(o, X, Z) || o->bfp_block) return o->f[k][q];
    return o->fx[k][q] + o->fz[k][q];
}

/* damping at a node (half = 0) or half node (half = 1) along one axis with
 * n interior nodes; returns -1 inside (undamped).  pml.c uses d[i] / dh[i]
 * on the start side and d[np-1-i] / dH[np-1-i] on the end side. */
static double e_damp(const orc_eiso *o, long P, size_t n, int half)
{
    long np = (long)o->np;
    if (P < np) return half ? o->dh[P] : o->d[P];
    if (P >= np + (long)n) {
        long i = P - np - (long)n;
        return half ? o->dH[np - 1 - i] : o->d[np - 1 - i];
    }
    return -1.0;
}

/* split-part update.  Damped (pml.c, e.g. :66-70):
 *   q = ((q*c2) + mat*delta/h) * c1,  c1 = 2dt/(2+dt d), c2 = (2-dt d)/(2dt)
 * Undamped, along the strip (pml.c, e.g. :117): q += dt*mat*delta/h. */
static double e_upd(const orc_eiso *o, double q, double damp, double mat, double delta)
{
    double dt = o->dt, h = o->h;
    if (damp < 0.0) return q + dt * mat * delta / h;
    double c1 = (2. * dt) / (2. + dt * damp);
    double c2 = (2. - dt * damp) / (2. * dt);
    q *= c2;
    q += mat * delta / h;
    q *= c1;
    return q;
}

/* material seen by a cell: the interior value, edge-replicated into the
 * frame (pml.c uses b[0], b[j], b[i*nz], b[nz-1], ...).  For lambda and
 * lambda+2mu in the lower-right corner pml.c:1044-1084 indexes
 * [nx*nx-1]; that is kept where it is inside the array (nx <= nz) and
 * replaced by the intended [nx*nz-1] where it is not. */
static double e_mat(const orc_eiso *o, int m, long X, long Z)
{
    long np = (long)o->np, nx = (long)o->nx, nz = (long)o->nz;
    long i = X - np, j = Z - np;
    if ((m == M_LA || m == M_L2M) && i >= nx && j >= nz) {
        size_t q = (size_t)(nx * nx - 1);
        if (q >= (size_t)(nx * nz)) q = (size_t)(nx * nz - 1);
        return o->mat[m][q];
    }
    i = i < 0 ? 0 : (i >= nx ? nx - 1 : i);
    j = j < 0 ? 0 : (j >= nz ? nz - 1 : j);
    return o->mat[m][i * nz + j];
}

void orc_eiso_velocity(orc_eiso *o)
{
    double dt = o->dt, h = o->h;
    for (long X = 0; X < (long)o->NX; ++X) {
        for (long Z = 0; Z < (long)o->NZ; ++Z) {
            size_t q = (size_t)X * o->NZ + (size_t)Z;
            /* vx at (X, Z): backward x difference of txx, backward z of txz */
            double ax = e_val(o, ORC_TXX, X, Z) - e_val(o, ORC_TXX, X - 1, Z);
            double az = e_val(o, ORC_TXZ, X, Z) - e_val(o, ORC_TXZ, X, Z - 1);
            /* vz at (X+1/2, Z+1/2): forward x of txz, forward z of tzz */
            double bx = e_val(o, ORC_TXZ, X + 1, Z) - e_val(o, ORC_TXZ, X, Z);
            double bz = e_val(o, ORC_TZZ, X, Z + 1) - e_val(o, ORC_TZZ, X, Z);
            if (e_interior(o, X, Z)) {
                /* propagate.c:2546-2548, 2560-2563 */
                size_t c = (size_t)(X - o->np) * o->nz + (size_t)(Z - o->np);
                double d1 = ax / h, d2 = az / h;
                o->f[ORC_VX][q] += dt * o->mat[M_B][c] * (d1 + d2);
                d1 = bx / h; d2 = bz / h;
                o->f[ORC_VZ][q] += dt * o->mat[M_BM][c] * (d1 + d2);
            } else {
                double b = e_mat(o, M_B, X, Z), bm = e_mat(o, M_BM, X, Z);
                o->fx[ORC_VX][q] = e_upd(o, o->fx[ORC_VX][q], e_damp(o, X, o->nx, 0), b, ax);
                o->fz[ORC_VX][q] = e_upd(o, o->fz[ORC_VX][q], e_damp(o, Z, o->nz, 0), b, az);
                o->fx[ORC_VZ][q] = e_upd(o, o->fx[ORC_VZ][q], e_damp(o, X, o->nx, 1), bm, bx);
                o->fz[ORC_VZ][q] = e_upd(o, o->fz[ORC_VZ][q], e_damp(o, Z, o->nz, 1), bm, bz);
                o->f[ORC_VX][q] = o->fx[ORC_VX][q] + o->fz[ORC_VX][q];
                o->f[ORC_VZ][q] = o->fx[ORC_VZ][q] + o->fz[ORC_VZ][q];
            }
        }
    }
}

void orc_eiso_stress(orc_eiso *o)
{
    double dt = o->dt, h = o->h;
    for (long X = 0; X < (long)o->NX; ++X) {
        for (long Z = 0; Z < (long)o->NZ; ++Z) {
            size_t q = (size_t)X * o->NZ + (size_t)Z;
            /* txx, tzz at (X+1/2, Z): forward x of vx, backward z of vz */
            double ax = e_val(o, ORC_VX, X + 1, Z) - e_val(o, ORC_VX, X, Z);
            double az = e_val(o, ORC_VZ, X, Z) - e_val(o, ORC_VZ, X, Z - 1);
            /* txz at (X, Z+1/2): forward z of vx, backward x of vz */
            double bz = e_val(o, ORC_VX, X, Z + 1) - e_val(o, ORC_VX, X, Z);
            double bx = e_val(o, ORC_VZ, X, Z) - e_val(o, ORC_VZ, X - 1, Z);
            if (e_interior(o, X, Z)) {
                /* propagate.c:2605-2611, 2645-2648 */
                size_t c = (size_t)(X - o->np) * o->nz + (size_t)(Z - o->np);
                double la = o->mat[M_LA][c], l2m = o->mat[M_L2M][c], mu = o->mat[M_MU][c];
                double dvx_x = dt * ax / h, dvz_z = dt * az / h;
                o->f[ORC_TXX][q] += l2m * dvx_x + la * dvz_z;
                o->f[ORC_TZZ][q] += l2m * dvz_z + la * dvx_x;
                double dvx_z = dt * bz / h, dvz_x = dt * bx / h;
                o->f[ORC_TXZ][q] += mu * (dvx_z + dvz_x);
            } else {
                double la = e_mat(o, M_LA, X, Z), l2m = e_mat(o, M_L2M, X, Z);
                double mu = e_mat(o, M_MU, X, Z);
                double dxh = e_damp(o, X, o->nx, 1), dzn = e_damp(o, Z, o->nz, 0);
                double dxn = e_damp(o, X, o->nx, 0), dzh = e_damp(o, Z, o->nz, 1);
                o->fx[ORC_TXX][q] = e_upd(o, o->fx[ORC_TXX][q], dxh, l2m, ax);
                o->fx[ORC_TZZ][q] = e_upd(o, o->fx[ORC_TZZ][q], dxh, la, ax);
                o->fz[ORC_TXX][q] = e_upd(o, o->fz[ORC_TXX][q], dzn, la, az);
                o->fz[ORC_TZZ][q] = e_upd(o, o->fz[ORC_TZZ][q], dzn, l2m, az);
                o->fx[ORC_TXZ][q] = e_upd(o, o->fx[ORC_TXZ][q], dxn, mu, bx);
                o->fz[ORC_TXZ][q] = e_upd(o, o->fz[ORC_TXZ][q], dzh, mu, bz);
                for (int k = ORC_TXX; k <= ORC_TXZ; ++k)
                    o->f[k][q] = o->fx[k][q] + o->fz[k][q];
            }
        }
    }
    /* block storage: the step stores its state rounded (velocities and
     * stresses, totals on the padded grid in blocks of B cells along Z;
     * the frame's split parts keep their precision, as the device keeps
     * them in FP32); the stress update above read the unrounded velocities */
    if (o->bfp_block && o->npatch == 0)
        for (int k = 0; k < 5; ++k) {
            if (o->bfp_axis == 0) bfp_round_cols(o->f[k], o->NX, o->NZ, o->bfp_block);
            else bfp_round_rows(o->f[k], o->NX, o->NZ, o->bfp_block);
        }
    if (o->bfp_block && o->npatch > 0) {   /* blocks along X, patches kept exact */
        size_t B = (size_t)o->bfp_block;
        for (int k = 0; k < 5; ++k)
            for (size_t x0 = 0; x0 < o->NX; x0 += B) {
                size_t nb = x0 + B < o->NX ? B : o->NX - x0;
                for (size_t Z = 0; Z < o->NZ; ++Z)
                    if (!e_in_patch(o, (long)x0, (long)Z))
                        bfp_round_strided(o->f[k] + x0 * o->NZ + Z, o->NZ, nb);
            }
    }
}

void orc_eiso_add_patch(orc_eiso *o, long X0, long Z0, long rows, long cols)
{
    if (o->npatch >= 16) return;
    long *p = o->patch[o->npatch++];
    p[0] = X0; p[1] = Z0; p[2] = rows; p[3] = cols;
}

void orc_eiso_set_bfp(orc_eiso *o, int block, int axis)
{
    o->bfp_block = block > 0 ? block : 0;
    o->bfp_axis = axis == 1 ? 1 : 0;
}

void orc_eiso_add_source(orc_eiso *o, size_t index, int type, double value)
{
    /* src.c:170-184; type ids follow structs.h:44 (SX=0, SZ=2, SXZ=4, BULK=6) */
    size_t i = index / o->nz, j = index % o->nz;
    size_t q = (i + o->np) * o->NZ + (j + o->np);
    if (type == 0 || type == 6) o->f[ORC_TXX][q] += value;
    if (type == 2 || type == 6) o->f[ORC_TZZ][q] += value;
    if (type == 4) o->f[ORC_TXZ][q] += value;
    if (o->bfp_block && !e_in_patch(o, (long)(q / o->NZ), (long)(q % o->NZ))) {
        /* the block of the source cell is stored again */
        size_t B = (size_t)o->bfp_block, Z = q % o->NZ, X = q / o->NZ;
        for (int k = ORC_TXX; k <= ORC_TXZ; ++k) {
            if (o->bfp_axis == 0) {
                size_t x0 = X / B * B, nb = x0 + B < o->NX ? B : o->NX - x0;
                bfp_round_strided(o->f[k] + x0 * o->NZ + Z, o->NZ, nb);
            } else {
                size_t z0 = Z / B * B;
                bfp_round_strided(o->f[k] + q - Z + z0, 1, z0 + B < o->NZ ? B : o->NZ - z0);
            }
        }
    }
}

void orc_eiso_get(const orc_eiso *o, int field, int part, double *out)
{
    size_t N = o->NX * o->NZ;
    for (size_t q = 0; q < N; ++q) {
        long X = (long)(q / o->NZ), Z = (long)(q % o->NZ);
        int in = e_interior(o, X, Z);
        if (part == ORC_TOTAL)
            out[q] = (in || o->bfp_block) ? o->f[field][q] : o->fx[field][q] + o->fz[field][q];
        else if (part == ORC_XPART) out[q] = in ? 0.0 : o->fx[field][q];
        else out[q] = in ? 0.0 : o->fz[field][q];
    }
}

void orc_eiso_set(orc_eiso *o, int field, int part, const double *in)
{
    size_t N = o->NX * o->NZ;
    double *dst = part == ORC_TOTAL ? o->f[field] : (part == ORC_XPART ? o->fx[field] : o->fz[field]);
    memcpy(dst, in, N * sizeof(double));
    /* block storage holds the frame's totals as stored values of their own */
    if (o->bfp_block && part == ORC_TOTAL) return;
    for (size_t q = 0; q < N; ++q) {
        long X = (long)(q / o->NZ), Z = (long)(q % o->NZ);
        if (!e_interior(o, X, Z)) o->f[field][q] = o->fx[field][q] + o->fz[field][q];
    }
}

double orc_eiso_probe(const orc_eiso *o, int field, size_t index)
{
    size_t i = index / o->nz, j = index % o->nz;
    return o->f[field][(i + o->np) * o->NZ + (j + o->np)];
}

/* ======================================================================
 * a_iso_3d
 * ====================================================================== */

void orc_a3d_pad_model(size_t nx, size_t ny, size_t nz, size_t np,
                       const double *vp_in, const double *rho_in,
                       double *vp_pad, double *rho_pad)
{
    /* io_utils.c:1050-1143: interior values at offset np on each axis, then
     * copied outwards from the nearest edge plane, z first, then y, then x. */
    size_t ny2 = ny + 2 * np, nz2 = nz + 2 * np, nx2 = nx + 2 * np;
    for (size_t i = 0; i < nx2; ++i)
        for (size_t j = 0; j < ny2; ++j)
            for (size_t k = 0; k < nz2; ++k) {
                size_t ii = i < np ? 0 : (i >= np + nx ? nx - 1 : i - np);
                size_t jj = j < np ? 0 : (j >= np + ny ? ny - 1 : j - np);
                size_t kk = k < np ? 0 : (k >= np + nz ? nz - 1 : k - np);
                size_t src = (ii * ny + jj) * nz + kk;
                size_t dst = (i * ny2 + j) * nz2 + k;
                vp_pad[dst] = vp_in[src];
                rho_pad[dst] = rho_in[src];
            }
}

double orc_a3d_cfl_vpmax(size_t nx, size_t nz, const double *vp_pad)
{
    /* a_iso_3d.c:368-374 scans ind = i*nz + j, i < nx, j < nz, of the padded
     * 3-D array (a 2-D sub-scan); kept as the reference has it. */
    double vpmax = 0.0;
    for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j < nz; ++j) {
            size_t ind = i * nz + j;
            vpmax = vp_pad[ind] > vpmax ? vp_pad[ind] : vpmax;
        }
    return vpmax;
}

void orc_a3d_cpml(size_t np, size_t nx2, size_t ny2, size_t nz2,
                  double dx, double dy, double dz, double dt,
                  double pml_order, double vmax, double Rc, double kappa_max,
                  int alpha_max_flag, double f0, double *const *coef)
{
    size_t n2[3] = {nx2, ny2, nz2};
    double h[3] = {dx, dy, dz};
    /* interior defaults a = 0, b = k = 1: a_iso_3d.c:525-548 */
    for (int ax = 0; ax < 3; ++ax) {
        double *a = coef[3 * ax + 0], *b = coef[3 * ax + 1], *k = coef[3 * ax + 2];
        double *a_h = coef[9 + 3 * ax + 0], *b_h = coef[9 + 3 * ax + 1], *k_h = coef[9 + 3 * ax + 2];
        for (size_t n = 0; n < n2[ax]; ++n) { a[n] = 0.0; b[n] = k[n] = 1.0; }
        for (size_t n = 0; n + 1 < n2[ax]; ++n) { a_h[n] = 0.0; b_h[n] = k_h[n] = 1.0; }
    }
    /* a_iso_3d.c:550-576 */
    const double pi = 4.0 * atan(1.0);
    double alpha_max = pi * f0;
    if (alpha_max_flag == 0) alpha_max = 0.0;
    double da = alpha_max / np;
    for (int ax = 0; ax < 3; ++ax) {
        double L = np * h[ax];
        double d0 = -(pml_order + 1.) * vmax * log(Rc) / (2. * L);
        double *a = coef[3 * ax + 0], *b = coef[3 * ax + 1], *k = coef[3 * ax + 2];
        double *a_h = coef[9 + 3 * ax + 0], *b_h = coef[9 + 3 * ax + 1], *k_h = coef[9 + 3 * ax + 2];
        size_t N2 = n2[ax];
        for (size_t n = 0; n < np; ++n) {
            k[n] = k[N2 - 1 - n] = 1. + (kappa_max - 1.) * pow(((np - n) * h[ax] / L), pml_order);
            k_h[n] = k_h[N2 - 2 - n] = 1. + (kappa_max - 1.) * pow(((np - n - 0.5) * h[ax] / L), pml_order);
            double alpha = n * da;
            double alpha_h = (n + 0.5) * da;
            double dd = d0 * pow(((np - n) * h[ax] / L), pml_order);
            double dd_h = d0 * pow(((np - n - 0.5) * h[ax] / L), pml_order);
            b[n] = b[N2 - 1 - n] = exp(-(dd / k[n] + alpha) * dt);
            b_h[n] = b_h[N2 - 2 - n] = exp(-(dd_h / k_h[n] + alpha_h) * dt);
            a[n] = a[N2 - 1 - n] = dd * (b[n] - 1.) / (k[n] * (dd + k[n] * alpha));
            a_h[n] = a_h[N2 - 2 - n] = dd_h * (b_h[n] - 1.) / (k_h[n] * (dd_h + k_h[n] * alpha_h));
        }
    }
}

struct orc_a3d {
    size_t nx2, ny2, nz2;
    double dx, dy, dz, dt;
    double *P, *vx, *vy, *vz;
    double *mPx, *mPy, *mPz, *mvx, *mvy, *mvz;
    double *irx, *iry, *irz, *K;
    double *coef[18];
    int bfp_block;   /* 0: FP64 storage; else block floating point, see below */
    int bfp_axis;    /* blocks along z (2) or y (1) */
};

orc_a3d *orc_a3d_new(size_t nx2, size_t ny2, size_t nz2, double dx, double dy, double dz,
                     double dt, const double *vp_pad, const double *rho_pad,
                     const double *const *coef)
{
    orc_a3d *o = calloc(1, sizeof(*o));
    o->nx2 = nx2; o->ny2 = ny2; o->nz2 = nz2;
    o->dx = dx; o->dy = dy; o->dz = dz; o->dt = dt;
    size_t N = nx2 * ny2 * nz2;
    double **arr[14] = {&o->P, &o->vx, &o->vy, &o->vz, &o->mPx, &o->mPy, &o->mPz,
                        &o->mvx, &o->mvy, &o->mvz, &o->irx, &o->iry, &o->irz, &o->K};
    for (int a = 0; a < 14; ++a) *arr[a] = calloc(N, sizeof(double));
    size_t n2[3] = {nx2, ny2, nz2};
    for (int c = 0; c < 18; ++c) {
        size_t len = c < 9 ? n2[c / 3] : n2[(c - 9) / 3] - 1;
        o->coef[c] = malloc(len * sizeof(double));
        memcpy(o->coef[c], coef[c], len * sizeof(double));
    }
    /* a_iso_3d.c:379-409: staggered buoyancy dt*2/(rho_a+rho_b); K*dt */
    for (size_t i = 0; i + 1 < nx2; ++i)
        for (size_t j = 0; j < ny2; ++j)
            for (size_t k = 0; k < nz2; ++k) {
                size_t a = (i * ny2 + j) * nz2 + k, b = ((i + 1) * ny2 + j) * nz2 + k;
                o->irx[a] = dt * 2. / (rho_pad[a] + rho_pad[b]);
            }
    for (size_t i = 0; i < nx2; ++i)
        for (size_t j = 0; j + 1 < ny2; ++j)
            for (size_t k = 0; k < nz2; ++k) {
                size_t a = (i * ny2 + j) * nz2 + k, b = (i * ny2 + j + 1) * nz2 + k;
                o->iry[a] = dt * 2. / (rho_pad[a] + rho_pad[b]);
            }
    for (size_t i = 0; i < nx2; ++i)
        for (size_t j = 0; j < ny2; ++j)
            for (size_t k = 0; k + 1 < nz2; ++k) {
                size_t a = (i * ny2 + j) * nz2 + k;
                o->irz[a] = dt * 2. / (rho_pad[a] + rho_pad[a + 1]);
            }
    for (size_t q = 0; q < N; ++q) o->K[q] = rho_pad[q] * vp_pad[q] * vp_pad[q] * dt;
    return o;
}

void orc_a3d_free(orc_a3d *o)
{
    if (!o) return;
    double *arr[14] = {o->P, o->vx, o->vy, o->vz, o->mPx, o->mPy, o->mPz,
                       o->mvx, o->mvy, o->mvz, o->irx, o->iry, o->irz, o->K};
    for (int a = 0; a < 14; ++a) free(arr[a]);
    for (int c = 0; c < 18; ++c) free(o->coef[c]);
    free(o);
}

/* a_iso_3d.c:605-617: vx on i < nx2-1 */
static void a3d_vx(void *ctx, size_t i0, size_t i1)
{
    orc_a3d *o = ctx;
    size_t ny2 = o->ny2, nz2 = o->nz2;
    const double *ax_h = o->coef[9], *bx_h = o->coef[10], *kx_h = o->coef[11];
    for (size_t i = i0; i < i1; ++i)
        for (size_t j = 0; j < ny2; ++j)
            for (size_t k = 0; k < nz2; ++k) {
                size_t a = (i * ny2 + j) * nz2 + k, b = ((i + 1) * ny2 + j) * nz2 + k;
                double g = (o->P[b] - o->P[a]) / o->dx;
                o->mPx[a] = bx_h[i] * o->mPx[a] + ax_h[i] * g;
                g = g / kx_h[i] + o->mPx[a];
                o->vx[a] -= o->irx[a] * g;
            }
}

/* a_iso_3d.c:620-634: vy on j < ny2-1 */
static void a3d_vy(void *ctx, size_t i0, size_t i1)
{
    orc_a3d *o = ctx;
    size_t ny2 = o->ny2, nz2 = o->nz2;
    const double *ay_h = o->coef[12], *by_h = o->coef[13], *ky_h = o->coef[14];
    for (size_t i = i0; i < i1; ++i)
        for (size_t j = 0; j + 1 < ny2; ++j)
            for (size_t k = 0; k < nz2; ++k) {
                size_t a = (i * ny2 + j) * nz2 + k, b = (i * ny2 + j + 1) * nz2 + k;
                double g = (o->P[b] - o->P[a]) / o->dy;
                o->mPy[a] = by_h[j] * o->mPy[a] + ay_h[j] * g;
                g = g / ky_h[j] + o->mPy[a];
                o->vy[a] -= o->iry[a] * g;
            }
}

/* a_iso_3d.c:637-651: vz on k < nz2-1 */
static void a3d_vz(void *ctx, size_t i0, size_t i1)
{
    orc_a3d *o = ctx;
    size_t ny2 = o->ny2, nz2 = o->nz2;
    const double *az_h = o->coef[15], *bz_h = o->coef[16], *kz_h = o->coef[17];
    for (size_t i = i0; i < i1; ++i)
        for (size_t j = 0; j < ny2; ++j)
            for (size_t k = 0; k + 1 < nz2; ++k) {
                size_t a = (i * ny2 + j) * nz2 + k;
                double g = (o->P[a + 1] - o->P[a]) / o->dz;
                o->mPz[a] = bz_h[k] * o->mPz[a] + az_h[k] * g;
                g = g / kz_h[k] + o->mPz[a];
                o->vz[a] -= o->irz[a] * g;
            }
}

/* a_iso_3d.c:659-683: i, j, k >= 1 (plane 0 is never updated) */
static void a3d_p(void *ctx, size_t i0, size_t i1)
{
    orc_a3d *o = ctx;
    size_t ny2 = o->ny2, nz2 = o->nz2;
    const double *ax = o->coef[0], *bx = o->coef[1], *kx = o->coef[2];
    const double *ay = o->coef[3], *by = o->coef[4], *ky = o->coef[5];
    const double *az = o->coef[6], *bz = o->coef[7], *kz = o->coef[8];
    for (size_t i = i0 > 1 ? i0 : 1; i < i1; ++i)
        for (size_t j = 1; j < ny2; ++j)
            for (size_t k = 1; k < nz2; ++k) {
                size_t a = (i * ny2 + j) * nz2 + k;
                size_t ax_ = ((i - 1) * ny2 + j) * nz2 + k;
                size_t ay_ = (i * ny2 + j - 1) * nz2 + k;
                double dvdx = (o->vx[a] - o->vx[ax_]) / o->dx;
                double dvdy = (o->vy[a] - o->vy[ay_]) / o->dy;
                double dvdz = (o->vz[a] - o->vz[a - 1]) / o->dz;
                o->mvx[a] = bx[i] * o->mvx[a] + ax[i] * dvdx;
                dvdx = dvdx / kx[i] + o->mvx[a];
                o->mvy[a] = by[j] * o->mvy[a] + ay[j] * dvdy;
                dvdy = dvdy / ky[j] + o->mvy[a];
                o->mvz[a] = bz[k] * o->mvz[a] + az[k] * dvdz;
                dvdz = dvdz / kz[k] + o->mvz[a];
                o->P[a] -= o->K[a] * (dvdx + dvdy + dvdz);
            }
}

/* ----------------------------------------------------------------------
 * Storage rounding (a checker mode with no counterpart in the reference):
 * the state a step leaves behind (P and the three velocities) is replaced
 * by the values 16-bit block floating point storage keeps, as the device's
 * block storage does: the pressure update of a step reads the velocities
 * that step computed, unrounded, and the state is rounded once when the
 * step stores it; a source added afterwards re-rounds the block of its cell.
 * A block is B consecutive z cells of one (i, j) row starting at a multiple
 * of B; its values share the exponent E of the block's largest magnitude M
 * (M in [2^(E-1), 2^E)), and each is kept as the integer
 * m = round_half_even(x 2^(15-E)), at most 32767 (15 bits and a sign),
 * i.e. x ~ m 2^(E-15); E is held in [-111, 114] as the device's 8-bit
 * exponent holds it.  The step arithmetic stays FP64, so the difference
 * from the plain oracle is the storage format's own error.  The CPML memory
 * variables keep FP64 (the device keeps them in FP32).
 * ---------------------------------------------------------------------- */
/* one block of n values at v[0], v[stride], ... */
static void bfp_round_strided(double *v, size_t stride, size_t n)
{
    double mx = 0.0;
    for (size_t k = 0; k < n; ++k) mx = fabs(v[k * stride]) > mx ? fabs(v[k * stride]) : mx;
    if (mx == 0.0 || !isfinite(mx)) return;
    int E;
    frexp(mx, &E);   /* mx in [2^(E-1), 2^E) */
    /* a block whose largest value would round up to 2^15 takes the next
     * exponent (the device compares the FP32 maximum with
     * 2^E (1 - 2^-16)); E is held in [-111, 114], the range of the
     * device's 8-bit exponent: tiny blocks keep the scale 2^126 */
    if (mx >= ldexp(1.0 - ldexp(1.0, -16), E)) E += 1;
    if (E < -111) E = -111;
    if (E > 114) E = 114;
    double sc = ldexp(1.0, 15 - E), isc = ldexp(1.0, E - 15);
    for (size_t k = 0; k < n; ++k) {
        double m = nearbyint(v[k * stride] * sc);
        if (m > 32767.0) m = 32767.0;
        v[k * stride] = m * isc;
    }
}

static void bfp_round_block(double *row, size_t k0, size_t k1)
{
    bfp_round_strided(row + k0, 1, k1 - k0);
}

/* blocks of B consecutive values along the fastest axis of rows of n */
static void bfp_round_rows(double *f, size_t nrows, size_t n, int B)
{
    for (size_t r = 0; r < nrows; ++r)
        for (size_t k0 = 0; k0 < n; k0 += (size_t)B)
            bfp_round_block(f + r * n, k0, k0 + (size_t)B < n ? k0 + (size_t)B : n);
}

/* blocks of B consecutive rows (stride n) at each position of the fastest
 * axis, in a plane of nrows rows of n */
static void bfp_round_cols(double *f, size_t nrows, size_t n, int B)
{
    for (size_t r0 = 0; r0 < nrows; r0 += (size_t)B) {
        size_t nb = r0 + (size_t)B < nrows ? (size_t)B : nrows - r0;
        for (size_t k = 0; k < n; ++k) bfp_round_strided(f + r0 * n + k, n, nb);
    }
}

struct bfp_job {
    double *f[3];
    size_t ny2, nz2;
    int B, axis;
};

static void bfp_planes(void *ctx, size_t i0, size_t i1)
{
    struct bfp_job *j = ctx;
    size_t plane = j->ny2 * j->nz2;
    for (int a = 0; a < 3; ++a) {
        if (!j->f[a]) continue;
        for (size_t i = i0; i < i1; ++i) {
            if (j->axis == 2) bfp_round_rows(j->f[a] + i * plane, j->ny2, j->nz2, j->B);
            else bfp_round_cols(j->f[a] + i * plane, j->ny2, j->nz2, j->B);
        }
    }
}

static void a3d_round(orc_a3d *o, double *f0, double *f1, double *f2)
{
    struct bfp_job j = {{f0, f1, f2}, o->ny2, o->nz2, o->bfp_block, o->bfp_axis};
    orc_parallel(o->nx2, bfp_planes, &j);
}

void orc_a3d_set_bfp(orc_a3d *o, int block, int axis)
{
    o->bfp_block = block > 0 ? block : 0;
    o->bfp_axis = axis == 1 ? 1 : 2;
}

void orc_a3d_velocity(orc_a3d *o)
{
    orc_parallel(o->nx2 - 1, a3d_vx, o);
    orc_parallel(o->nx2, a3d_vy, o);
    orc_parallel(o->nx2, a3d_vz, o);
}

void orc_a3d_pressure(orc_a3d *o)
{
    orc_parallel(o->nx2, a3d_p, o);
    if (o->bfp_block) {
        a3d_round(o, o->vx, o->vy, o->vz);
        a3d_round(o, o->P, NULL, NULL);
    }
}

void orc_a3d_add_source(orc_a3d *o, size_t index, double value)
{
    o->P[index] += value;
    if (o->bfp_block) {   /* the block of the source cell is stored again */
        size_t B = (size_t)o->bfp_block, k = index % o->nz2, ij = index / o->nz2;
        if (o->bfp_axis == 2) {
            size_t k0 = k / B * B;
            bfp_round_block(o->P + (index - k), k0, k0 + B < o->nz2 ? k0 + B : o->nz2);
        } else {
            size_t j = ij % o->ny2, j0 = j / B * B, nb = j0 + B < o->ny2 ? B : o->ny2 - j0;
            bfp_round_strided(o->P + (ij - j + j0) * o->nz2 + k, o->nz2, nb);
        }
    }
}

static double *a3d_field(const orc_a3d *o, int field)
{
    switch (field) {
    case ORC_A_VX: return o->vx;
    case ORC_A_VY: return o->vy;
    case ORC_A_VZ: return o->vz;
    default: return o->P;
    }
}

void orc_a3d_get(const orc_a3d *o, int field, double *out)
{
    memcpy(out, a3d_field(o, field), o->nx2 * o->ny2 * o->nz2 * sizeof(double));
}

void orc_a3d_set(orc_a3d *o, int field, const double *in)
{
    memcpy(a3d_field(o, field), in, o->nx2 * o->ny2 * o->nz2 * sizeof(double));
}

double orc_a3d_probe(const orc_a3d *o, int field, size_t index)
{
    return a3d_field(o, field)[index];
}

void orc_a3d_gather(const orc_a3d *o, size_t n, const int *field, const size_t *index,
                    double *out)
{
    for (size_t r = 0; r < n; ++r) out[r] = a3d_field(o, field[r])[index[r]];
}
