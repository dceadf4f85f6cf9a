/*
 * sm_setup.c -- host-side set-up of the e_iso / a_iso_3d paths, in FP64.
 *
 * These run once per shot before the time loop and must produce exactly the
 * numbers the reference feeds its loops: the same formulas in the same
 * order of operations, so results match bit for bit.
 */
#include "sm_host.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

size_t sm_ricker_length(double f, double dt, double fac)
{
    /* src.c:47-48 */
    double tcut = 1.0 / f;
    return (size_t)ceil(tcut * 2.0 / (fac * dt));
}

int sm_ricker(size_t n, const double *A, const double *f, double dt0, double fac,
              size_t stride, double *fct, size_t *length)
{
    if (n == 0) return SM_OK;
    if (!A || !f || !fct || !length || !(dt0 > 0.0) || !(fac > 0.0)) {
        return sm_fail(SM_EINVAL, "sm_ricker: bad argument");
    }
    const double pi = 4.0 * atan(1.0);
    const double pi2 = pi * pi;
    const double dt = fac * dt0;
    for (size_t s = 0; s < n; ++s) {
        if (!(f[s] > 0.0)) return sm_fail(SM_EINVAL, "sm_ricker: frequency must be > 0");
        if (sm_ricker_length(f[s], dt0, fac) > stride)
            return sm_fail(SM_EINVAL, "sm_ricker: stride shorter than the wavelet");
    }
    /* src.c:43-65.  Pass s writes wavelet s, takes the peak of wavelet 0 over
     * the first length[s] samples, and rescales wavelet 0 by A[s] / peak.
     * Where the reference would read wavelet 0 past its end (length[s] >
     * length[0]) the scan stops at length[0]. */
    for (size_t s = 0; s < n; ++s) {
        const double tcut = 1.0 / f[s];
        length[s] = sm_ricker_length(f[s], dt0, fac);
        double *w = fct + s * stride;
        double peak = 0.0;
        for (size_t i = 0; i < length[s]; ++i) {
            double time = i * dt - tcut;
            /* same left-to-right products as the reference */
            double K = pi2 * f[s] * f[s] * time * time;
            w[i] = A[s] * 2. * pi2 * f[s] * f[s] * (1.0 - 2.0 * K) * exp(-K);
            if (i < length[0]) {
                double a = fabs(fct[i]);
                if (a > peak) peak = a;
            }
        }
        for (size_t i = 0; i < length[0]; ++i) fct[i] *= A[s] / peak;
    }
    return SM_OK;
}

size_t sm_nsteps(double duration, double dt)
{
    size_t n = (size_t)(duration / dt);
    if (n * dt < duration) n++;
    return n;
}

int sm_sample_predicate(size_t it, double dt, double t0, double rdt)
{
    /* e_iso.c:643-658, a_iso_3d.c:700-719 */
    const double t = dt * (it + 1);
    const double dt2 = t - t0 + 1.e-15;
    const double rem = fmod(1.e6 * dt2, 1.e6 * rdt);
    return (fabs(dt2) < 0.99 * dt) || (t > t0 && rdt > 0.0 && fabs(rem) < 1.e-8);
}

int sm_eiso_materials(size_t nx, size_t nz, const double *vp, const double *vs,
                      const double *rho, double *la, double *mu, double *l2m,
                      double *b, double *bm, double *vpmax)
{
    if (nx < 2 || nz < 2 || !vp || !vs || !rho || !la || !mu || !l2m || !b || !bm)
        return sm_fail(SM_EINVAL, "sm_eiso_materials: bad argument (nx, nz >= 2)");
    const size_t n = nx * nz;
    /* nodal lambda, mu, lambda + 2 mu kept in the outputs' spare room:
     * la <- nodal lambda first, then averaged along x in place, column by
     * column from the front (each average reads i and i+1 before i+1 is
     * rewritten).  mu and l2m likewise. */
    double vmax = 0.0;
    for (size_t q = 0; q < n; ++q) {
        if (vp[q] > vmax) vmax = vp[q];
        double lam = rho[q] * (vp[q] * vp[q] - 2. * vs[q] * vs[q]);  /* e_iso.c:428 */
        double m = rho[q] * vs[q] * vs[q];                           /* :429 */
        la[q] = lam;
        mu[q] = m;
        l2m[q] = lam + 2. * m;                                       /* :430 */
        b[q] = 1. / rho[q];                                          /* :431 */
    }
    /* mu: average along z, last row nodal (e_iso.c:438-443) */
    for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j + 1 < nz; ++j)
            mu[i * nz + j] = (mu[i * nz + j] + mu[i * nz + j + 1]) / 2.0;
    /* lambda, lambda + 2 mu: average along x, last column nodal (:444-451) */
    for (size_t i = 0; i + 1 < nx; ++i)
        for (size_t j = 0; j < nz; ++j) {
            la[i * nz + j] = (la[i * nz + j] + la[(i + 1) * nz + j]) / 2.0;
            l2m[i * nz + j] = (l2m[i * nz + j] + l2m[(i + 1) * nz + j]) / 2.0;
        }
    /* 1/rho at the vz node: 4-point mean, 2-point on the last row/column,
     * nodal in the last corner (:452-462) */
    for (size_t i = 0; i + 1 < nx; ++i) {
        for (size_t j = 0; j + 1 < nz; ++j)
            bm[i * nz + j] = (b[i * nz + j] + b[(i + 1) * nz + j] +
                              b[i * nz + j + 1] + b[(i + 1) * nz + j + 1]) / 4.0;
        bm[i * nz + nz - 1] = (b[i * nz + nz - 1] + b[(i + 1) * nz + nz - 1]) / 2.0;
    }
    for (size_t j = 0; j + 1 < nz; ++j)
        bm[(nx - 1) * nz + j] = (b[(nx - 1) * nz + j] + b[(nx - 1) * nz + j + 1]) / 2.0;
    bm[n - 1] = b[n - 1];
    if (vpmax) *vpmax = vmax;
    return SM_OK;
}

int sm_eiso_profiles(size_t np, double h, size_t ncell, const double *vp,
                     double *d, double *dh, double *dH)
{
    if (np == 0 || ncell == 0 || !vp || !d || !dh || !dH || !(h > 0.0))
        return sm_fail(SM_EINVAL, "sm_eiso_profiles: bad argument");
    /* e_iso.c:486-500: d0 from the MEAN vp, R = 1e-3, quadratic profile */
    double vbar = 0.0;
    for (size_t q = 0; q < ncell; ++q) vbar += vp[q];
    vbar /= (double)ncell;
    const double R = 0.001;
    const double delta = np * h;
    const double d0 = log(1. / R) * 3. / 2. * vbar / delta;
    for (size_t n = 0; n < np; ++n) {
        d[n] = d0 * pow(((np - n) * h / delta), 2);
        dh[n] = d0 * pow((((np - n) * h - h / 2.) / delta), 2);
    }
    for (size_t n = 0; n < np + 1; ++n) dH[n] = d0 * pow((((np - n) * h + h / 2.) / delta), 2);
    return SM_OK;
}

/* one thread's share of sm_a3d_pad_model: padded x planes [i0, i1) */
struct a3d_pad_part {
    size_t nx, ny, nz, np, i0, i1;
    const double *vp, *rho;
    double *vp_pad, *rho_pad;
};

static void *a3d_pad_planes(void *arg)
{
    const struct a3d_pad_part *t = (const struct a3d_pad_part *)arg;
    const size_t nx = t->nx, ny = t->ny, nz = t->nz, np = t->np;
    const size_t ny2 = ny + 2 * np, nz2 = nz + 2 * np;
    for (size_t i = t->i0; i < t->i1; ++i) {
        size_t ii = i < np ? 0 : (i - np >= nx ? nx - 1 : i - np);
        for (size_t j = 0; j < ny2; ++j) {
            size_t jj = j < np ? 0 : (j - np >= ny ? ny - 1 : j - np);
            const double *sv = t->vp + (ii * ny + jj) * nz;
            const double *sr = t->rho + (ii * ny + jj) * nz;
            double *dv = t->vp_pad + (i * ny2 + j) * nz2;
            double *dr = t->rho_pad + (i * ny2 + j) * nz2;
            for (size_t k = 0; k < np; ++k) {
                dv[k] = sv[0];
                dr[k] = sr[0];
            }
            memcpy(dv + np, sv, nz * sizeof(double));
            memcpy(dr + np, sr, nz * sizeof(double));
            for (size_t k = np + nz; k < nz2; ++k) {
                dv[k] = sv[nz - 1];
                dr[k] = sr[nz - 1];
            }
        }
    }
    return NULL;
}

int sm_a3d_pad_model(size_t nx, size_t ny, size_t nz, size_t np,
                     const double *vp, const double *rho, double *vp_pad, double *rho_pad)
{
    if (!nx || !ny || !nz || !vp || !rho || !vp_pad || !rho_pad)
        return sm_fail(SM_EINVAL, "sm_a3d_pad_model: bad argument");
    /* io_utils.c:1096-1143: every padded node takes the value of the nearest
     * interior node (replication along z, then y, then x).  A pure copy, so
     * the x planes are split over host threads (the two padded volumes of a
     * 544^3 grid are 2.5 GB; one thread spends most of a second on them,
     * first-touch page faults included). */
    const size_t nx2 = nx + 2 * np, ny2 = ny + 2 * np, nz2 = nz + 2 * np;
    const size_t cells = nx2 * ny2 * nz2;
    size_t nt = sm_host_threads(cells, (size_t)1 << 20);
    if (nt > nx2) nt = nx2;
    struct a3d_pad_part part[SM_MAX_HOST_THREADS];
    for (size_t t = 0; t < nt; ++t)
        part[t] = (struct a3d_pad_part){nx, ny, nz, np, nx2 * t / nt, nx2 * (t + 1) / nt,
                                        vp, rho, vp_pad, rho_pad};
    sm_parallel(a3d_pad_planes, part, sizeof part[0], nt);
    return SM_OK;
}

double sm_a3d_cfl_vpmax(size_t nx, size_t nz, const double *vp_pad)
{
    /* a_iso_3d.c:368-374 scans index i*nz + j (i < nx, j < nz) of the padded
     * 3-D array; kept as is so the same inputs pass or fail the test */
    double v = 0.0;
    for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j < nz; ++j) {
            double a = vp_pad[i * nz + j];
            if (a > v) v = a;
        }
    return v;
}

double sm_a3d_cfl_vpmax_unpadded(size_t nx, size_t ny, size_t nz, size_t np, const double *vp)
{
    /* sm_a3d_cfl_vpmax on the padded model that sm_a3d_pad_model would
     * make: the same padded indices i*nz + j, each mapped to the interior
     * node whose value edge replication copies there */
    const size_t ny2 = ny + 2 * np, nz2 = nz + 2 * np;
    double v = 0.0;
    for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j < nz; ++j) {
            const size_t q = i * nz + j;
            const size_t x = q / (ny2 * nz2), y = q / nz2 % ny2, z = q % nz2;
            const size_t cx = x < np ? 0 : (x - np >= nx ? nx - 1 : x - np);
            const size_t cy = y < np ? 0 : (y - np >= ny ? ny - 1 : y - np);
            const size_t cz = z < np ? 0 : (z - np >= nz ? nz - 1 : z - np);
            const double a = vp[(cx * ny + cy) * nz + cz];
            if (a > v) v = a;
        }
    return v;
}

int sm_a3d_cpml(size_t np, size_t nx2, size_t ny2, size_t nz2,
                double dx, double dy, double dz, double dt,
                double pml_order, double vmax, double Rc, double kappa_max,
                int alpha_max_flag, double f0, double *const *coef)
{
    if (!coef) return sm_fail(SM_EINVAL, "sm_a3d_cpml: coef is NULL");
    const size_t n2[3] = {nx2, ny2, nz2};
    const double hh[3] = {dx, dy, dz};
    for (int c = 0; c < 18; ++c)
        if (!coef[c]) return sm_fail(SM_EINVAL, "sm_a3d_cpml: coefficient array is NULL");
    for (int a = 0; a < 3; ++a) {
        if (n2[a] < 2 * np + 2) return sm_fail(SM_EINVAL, "sm_a3d_cpml: grid smaller than the frame");
        double *A = coef[3 * a], *B = coef[3 * a + 1], *K = coef[3 * a + 2];
        double *Ah = coef[9 + 3 * a], *Bh = coef[9 + 3 * a + 1], *Kh = coef[9 + 3 * a + 2];
        /* a_iso_3d.c:525-548 */
        for (size_t n = 0; n < n2[a]; ++n) { A[n] = 0.0; B[n] = 1.0; K[n] = 1.0; }
        for (size_t n = 0; n + 1 < n2[a]; ++n) { Ah[n] = 0.0; Bh[n] = 1.0; Kh[n] = 1.0; }
    }
    if (np == 0) return SM_OK;
    /* a_iso_3d.c:550-576 */
    const double pi = 4.0 * atan(1.0);
    const double amax = alpha_max_flag == 0 ? 0.0 : pi * f0;
    const double da = amax / np;
    for (int a = 0; a < 3; ++a) {
        double *A = coef[3 * a], *B = coef[3 * a + 1], *K = coef[3 * a + 2];
        double *Ah = coef[9 + 3 * a], *Bh = coef[9 + 3 * a + 1], *Kh = coef[9 + 3 * a + 2];
        const size_t N = n2[a];
        const double L = np * hh[a];
        const double d0 = -(pml_order + 1.) * vmax * log(Rc) / (2. * L);
        for (size_t n = 0; n < np; ++n) {
            double k = 1. + (kappa_max - 1.) * pow(((np - n) * hh[a] / L), pml_order);
            double kh = 1. + (kappa_max - 1.) * pow(((np - n - 0.5) * hh[a] / L), pml_order);
            double al = n * da, alh = (n + 0.5) * da;
            double dd = d0 * pow(((np - n) * hh[a] / L), pml_order);
            double ddh = d0 * pow(((np - n - 0.5) * hh[a] / L), pml_order);
            double b = exp(-(dd / k + al) * dt);
            double bh = exp(-(ddh / kh + alh) * dt);
            double c = dd * (b - 1.) / (k * (dd + k * al));
            double ch = ddh * (bh - 1.) / (kh * (ddh + kh * alh));
            K[n] = K[N - 1 - n] = k;
            Kh[n] = Kh[N - 2 - n] = kh;
            B[n] = B[N - 1 - n] = b;
            Bh[n] = Bh[N - 2 - n] = bh;
            A[n] = A[N - 1 - n] = c;
            Ah[n] = Ah[N - 2 - n] = ch;
        }
    }
    return SM_OK;
}

/* ======================================================================
 * e_cyl_iso (padded grid nx2 = nx + np radial columns, PML at the outer
 * radius only; nz2 = nz + 2 np rows; index i*nz2 + j)
 * ====================================================================== */

int sm_ecyl_pad_model(size_t nx, size_t nz, size_t np, const double *vp, const double *vs,
                      const double *rho, double *vp_pad, double *vs_pad, double *rho_pad)
{
    /* io_utils.c:993-1026: interior at rows np..np+nz-1; the PML rows copy
     * the first / last interior row of their column; the outer PML columns
     * copy column nx-1 */
    if (!vp || !vs || !rho || !vp_pad || !vs_pad || !rho_pad || nx == 0 || nz == 0)
        return sm_fail(SM_EINVAL, "sm_ecyl_pad_model: bad argument");
    const size_t nz2 = nz + 2 * np, nx2 = nx + np;
    const double *src[3] = {vp, vs, rho};
    double *dst[3] = {vp_pad, vs_pad, rho_pad};
    for (int k = 0; k < 3; ++k) {
        for (size_t i = 0; i < nx; ++i) {
            double *col = dst[k] + i * nz2;
            memcpy(col + np, src[k] + i * nz, nz * sizeof(double));
            for (size_t j = 0; j < np; ++j) {
                col[j] = col[np];
                col[np + nz + j] = col[np + nz - 1];
            }
        }
        for (size_t i = nx; i < nx2; ++i)
            memcpy(dst[k] + i * nz2, dst[k] + (nx - 1) * nz2, nz2 * sizeof(double));
    }
    return SM_OK;
}

static double ecyl_harm(double a, double b)
{
    return (a == 0.0 && b == 0.0) ? 0.0 : 2. * a * b / (a + b);
}

int sm_ecyl_materials(size_t nx2, size_t nz2, const double *vp, const double *vs,
                      const double *rho, double *const *mat, double *vpmax)
{
    /* e_cyl_iso.c:363-441; mat: lij l2mij mu mui muj bi bj bij */
    if (!vp || !vs || !rho || !mat || nx2 == 0 || nz2 == 0)
        return sm_fail(SM_EINVAL, "sm_ecyl_materials: bad argument");
    for (int k = 0; k < 8; ++k)
        if (!mat[k]) return sm_fail(SM_EINVAL, "sm_ecyl_materials: material %d is NULL", k);
    double *lij = mat[0], *l2m = mat[1], *mu = mat[2], *mui = mat[3], *muj = mat[4],
           *bi = mat[5], *bj = mat[6], *bij = mat[7];
    const size_t N = nx2 * nz2;
    double *m = malloc(N * sizeof *m);
    if (!m) return sm_fail(SM_ENOMEM, "sm_ecyl_materials: out of host memory");
    double vmax = 0.0;
    for (size_t k = 0; k < N; ++k) {
        if (vp[k] > vmax) vmax = vp[k];
        lij[k] = rho[k] * (vp[k] * vp[k] - 2. * vs[k] * vs[k]);
        m[k] = rho[k] * vs[k] * vs[k];
        l2m[k] = lij[k] + 2.0 * m[k];
        bij[k] = 1. / rho[k];
    }
    for (size_t i = 0; i < nx2; ++i) {   /* z averages */
        const size_t c = i * nz2;
        muj[c] = m[c];
        bj[c] = bij[c];
        for (size_t j = 1; j < nz2; ++j) {
            muj[c + j] = ecyl_harm(m[c + j], m[c + j - 1]);
            bj[c + j] = 1. / ((rho[c + j] + rho[c + j - 1]) / 2.0);
        }
    }
    for (size_t j = 0; j < nz2; ++j) {   /* r averages */
        mui[j] = m[j];
        bi[j] = 1. / rho[j];
        for (size_t i = 1; i < nx2; ++i) {
            const size_t q = i * nz2 + j;
            mui[q] = ecyl_harm(m[q], m[q - nz2]);
            bi[q] = 1. / ((rho[q] + rho[q - nz2]) / 2.0);
        }
    }
    mu[0] = m[0];
    for (size_t j = 1; j < nz2; ++j) mu[j] = ecyl_harm(m[j], m[j - 1]);
    for (size_t i = 1; i < nx2; ++i) {   /* four-point average */
        const size_t c = i * nz2;
        mu[c] = ecyl_harm(m[c], m[c - nz2]);
        for (size_t j = 1; j < nz2; ++j) {
            const double a = m[c + j], b = m[c + j - 1], e = m[c - nz2 + j], d = m[c - nz2 + j - 1];
            const int none = b * e * d == 0.0 && a * e * d == 0.0 && a * b * d == 0.0 &&
                             a * b * e == 0.0;
            mu[c + j] = none ? 0.0 : 4. * a * b * e * d / (b * e * d + a * e * d + a * b * d + a * b * e);
        }
    }
    free(m);
    if (vpmax) *vpmax = vmax;
    return SM_OK;
}

int sm_ecyl_cpml(size_t np, double dx, double dz, double dt, double order, double vmax,
                 double Rc, double kappa_max, double alpha_max, int absorb, double *const *c)
{
    /* pml.c:2107-2185 (compute_cpml_cyl); c: ik_r ik_z ikh_z b_r c_r b_z c_z
     * bh_z ch_z (np) then ikH_r ikH_z bH_r cH_r bH_z cH_z (np + 1) */
    if (!c) return sm_fail(SM_EINVAL, "sm_ecyl_cpml: NULL");
    for (int k = 0; k < 15; ++k)
        if (!c[k]) return sm_fail(SM_EINVAL, "sm_ecyl_cpml: array %d is NULL", k);
    const double Lx = np * dx, Lz = np * dz;
    const double d0x = -(order + 1.) * vmax * log(Rc) / (2. * Lx);
    const double d0z = -(order + 1.) * vmax * log(Rc) / (2. * Lz);
    const double da = alpha_max / np, da2 = alpha_max / (np + 1);
    for (size_t n = 0; n < np; ++n) {
        if (!absorb) {
            c[0][n] = c[1][n] = c[2][n] = 1.;
            c[3][n] = c[4][n] = c[5][n] = c[6][n] = c[7][n] = c[8][n] = 0.;
            continue;
        }
        const double kr = 1. + (kappa_max - 1.) * pow(((np - n) * dx / Lx), order);
        const double kz = 1. + (kappa_max - 1.) * pow(((np - n) * dz / Lz), order);
        /* the half-node z kappa uses dx / Lx, as pml.c:2126 does */
        const double khz = 1. + (kappa_max - 1.) * pow(((np - n - 0.5) * dx / Lx), order);
        c[0][n] = 1. / kr;
        c[1][n] = 1. / kz;
        c[2][n] = 1. / khz;
        const double dxn = d0x * pow(((np - n) * dx / Lx), order), axn = n * da;
        c[3][n] = exp(-(dxn / kr + axn) * dt);
        c[4][n] = dxn * (c[3][n] - 1.) / (kr * (dxn + kr * axn));
        const double dzn = d0z * pow(((np - n) * dz / Lz), order), azn = n * da;
        const double dzh = d0z * pow(((np - n - 0.5) * dz / Lz), order), azh = (n + 0.5) * da;
        c[5][n] = exp(-(dzn / kz + azn) * dt);
        c[6][n] = dzn * (c[5][n] - 1.) / (kz * (dzn + kz * azn));
        c[7][n] = exp(-(dzh / khz + azh) * dt);
        c[8][n] = dzh * (c[7][n] - 1.) / (khz * (dzh + khz * azh));
    }
    for (size_t n = 0; n <= np; ++n) {
        if (!absorb) {
            c[9][n] = c[10][n] = 1.;
            c[11][n] = c[12][n] = c[13][n] = c[14][n] = 0.;
            continue;
        }
        const double kr = 1. + (kappa_max - 1.) * pow(((n + 0.5) * dx / Lx), order);
        const double kz = 1. + (kappa_max - 1.) * pow(((n + 0.5) * dz / Lz), order);
        c[9][n] = 1. / kr;
        c[10][n] = 1. / kz;
        const double dxe = d0x * pow(((n + 0.5) * dx / Lx), order), axe = (np - n - 0.5) * da2;
        c[11][n] = exp(-(dxe / kr + axe) * dt);
        c[12][n] = dxe * (c[11][n] - 1.) / (kr * (dxe + kr * axe));
        const double dze = d0z * pow(((n + 0.5) * dz / Lz), order), aze = (np - n - 0.5) * da2;
        c[13][n] = exp(-(dze / kz + aze) * dt);
        c[14][n] = dze * (c[13][n] - 1.) / (kz * (dze + kz * aze));
    }
    return SM_OK;
}

size_t sm_ecyl_kurkjian(double A, double f, double dt, double lij_at_src, double r_src,
                        double dx, double dz, int n, size_t maxlen, double *fct)
{
    /* src.c:202-228: peak-1 Ricker times A lambda/(2 pi) eps 2/(dx^2 dz)
     * (r/dx)^n, eps = 2 for n > 0 */
    const double pi = 4.0 * atan(1.0), pi2 = pi * pi;
    const double eps = n > 0 ? 2.0 : 1.0;
    const double term = lij_at_src / (2. * pi) * eps * 2. / (dx * dx * dz) * pow(r_src / dx, n);
    const double tcut = 1.0 / f;
    size_t len = (size_t)ceil(tcut * 2.0 / dt);
    if (!fct) return len;
    if (len > maxlen) len = maxlen;
    double amax = 0.0;
    for (size_t i = 0; i < len; ++i) {
        const double t = i * dt - tcut;
        const double K = pi2 * f * f * t * t;
        fct[i] = 2. * pi2 * f * f * (1.0 - 2.0 * K) * exp(-K);
        if (fabs(fct[i]) > amax) amax = fabs(fct[i]);
    }
    for (size_t i = 0; i < len; ++i) fct[i] *= A / amax * term;
    return len;
}
