/*
 * sm_drivers.c -- the e_iso and a_iso_3d programs with their time loops on
 * the GPU: same arguments, same input files, same trace files.
 *
 * The set-up follows the reference drivers step by step (e_iso.c:342-587,
 * a_iso_3d/a_iso_3d.c:240-591) in FP64 through the library's host
 * functions; the loop (e_iso.c:589-670, a_iso_3d.c:593-741) runs through
 * the C ABI.  Differences: errors return a non-zero status with a message
 * instead of abort()/exit(); snapshot records are written in the reference's
 * text snapshot format (write_snapshot, io_utils.c:1775-1820) since netCDF
 * is not available here; the 8 outer points of a 9-point source template
 * take the centre's type (io_utils.c:1494-1535 leaves them unset).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sm_io.h"

static int report(int rc, const char *prog)
{
    if (rc != SM_OK) fprintf(stderr, "%s: %s\n", prog, sm_last_error());
    return rc;
}

/* trace records -> receiver arrays for the device (trace records only) */
typedef struct {
    size_t n;
    size_t *index, *recno;
    int *comp;
    double *t0, *rdt;
} rec_plan;

static void rec_plan_free(rec_plan *r)
{
    free(r->index); free(r->recno); free(r->comp); free(r->t0); free(r->rdt);
}

static int write_traces(const char *base, const rec_plan *rp, const double *vals, size_t ld,
                        const size_t *counts, double dt, size_t nsteps)
{
    return sm_write_trace_set(base, rp->n, rp->recno, rp->t0, rp->rdt, dt, nsteps, vals, ld,
                              counts);
}

/* Snapshot records: the steps at which each is taken, by the traces'
 * sampling test (e_iso.c:641-669, a_iso_3d.c:698-741), in step order. */
typedef struct {
    size_t it, rec;
} snap_ev;

static int snap_cmp(const void *a, const void *b)
{
    const snap_ev *x = a, *y = b;
    if (x->it != y->it) return x->it < y->it ? -1 : 1;
    return x->rec < y->rec ? -1 : (x->rec > y->rec);
}

static int snap_events(const sm_record *rec, size_t nrec, double dt, size_t nsteps, snap_ev **out,
                       size_t *n)
{
    size_t cap = 16;
    *n = 0;
    *out = malloc(cap * sizeof(snap_ev));
    if (!*out) return sm_fail(SM_ENOMEM, "out of host memory");
    for (size_t r = 0; r < nrec; ++r) {
        if (rec[r].is_trace) continue;
        for (size_t it = 0; it < nsteps; ++it) {
            if (!sm_sample_predicate(it, dt, rec[r].t0, rec[r].dt)) continue;
            if (*n == cap) {
                snap_ev *m = realloc(*out, 2 * cap * sizeof(snap_ev));
                if (!m) return sm_fail(SM_ENOMEM, "out of host memory");
                *out = m;
                cap *= 2;
            }
            (*out)[(*n)++] = (snap_ev){it, r};
        }
    }
    qsort(*out, *n, sizeof(snap_ev), snap_cmp);
    return SM_OK;
}

static void check_dt_trc(const sm_record *rec, size_t nrec, double dt)
{
    /* io_utils.c:3561-3575 */
    for (size_t n = 0; n < nrec; ++n)
        if (rec[n].is_trace) {
            double rem = fmod(1000000.0 * rec[n].dt, 1000000.0 * dt);
            if (rem > 1.e-9) {
                fprintf(stdout, "\n *** Warning ***\n");
                fprintf(stdout, "Time step of receiver %zu not a multiple of modeling time step\n", n + 1);
                fprintf(stdout, " *** Warning ***\n");
            }
        }
}

/* Ricker wavelets of every source (src.c:43-65); *fct is n x stride */
static int make_wavelets(const sm_source *s, size_t n, double dt, double **fct, size_t **len,
                         size_t *stride)
{
    double *A = malloc(n * sizeof(double)), *f = malloc(n * sizeof(double));
    size_t st = 0;
    for (size_t q = 0; q < n; ++q) {
        A[q] = s[q].A;
        f[q] = s[q].f;
        size_t l = sm_ricker_length(s[q].f, dt, 1.0);
        if (l > st) st = l;
    }
    *fct = calloc(n * (st ? st : 1), sizeof(double));
    *len = calloc(n, sizeof(size_t));
    int rc = sm_ricker(n, A, f, dt, 1.0, st, *fct, *len);
    free(A);
    free(f);
    *stride = st;
    return rc;
}

int sm_e_iso_main(int argc, char **argv)
{
    const char *prog = "e_iso_gpu";
    sm_params p;
    sm_grid g;
    double *vp = NULL, *vs = NULL, *rho = NULL, *la = NULL, *mu = NULL, *l2m = NULL, *b = NULL, *bm = NULL;
    double *d = NULL, *dh = NULL, *dH = NULL, *fct = NULL, *vals = NULL;
    size_t *len = NULL, *counts = NULL;
    sm_source *src = NULL;
    sm_record *rec = NULL;
    rec_plan rp = {0};
    sm_eiso_t h = NULL;
    size_t nsrc = 0, ntpl = 1, nrec = 0, stride = 0;
    int rc;

    sm_params_defaults(&p);
    if ((rc = sm_parse_args(argc, argv, &p, prog))) return report(rc, prog);
    const size_t npml = p.np;   /* e_iso.c:346: the frame is kept outside the grid */
    if (p.verbose) fprintf(stdout, "\n *** e_iso - Elastic wave propagation in 2D isotropic media (GPU) ***\n\n");
    if ((rc = sm_read_model_e(p.modelfile, &g, &vp, &vs, &rho))) goto out;
    if (g.dx != g.dz) { rc = sm_fail(SM_EINVAL, "grid cell size must be equal in X and Z"); goto out; }
    if (npml == 0) {
        rc = sm_fail(SM_EINVAL, "e_iso needs its PML (abs 1, nl >= 1): with none the reference "
                                "indexes outside its arrays (propagate.c:2519)");
        goto out;
    }
    const double h_ = g.dx, dt = p.dt;
    const size_t nx = g.nx, nz = g.nz, ncell = nx * nz;
    la = malloc(ncell * sizeof(double)); mu = malloc(ncell * sizeof(double));
    l2m = malloc(ncell * sizeof(double)); b = malloc(ncell * sizeof(double));
    bm = malloc(ncell * sizeof(double));
    double vpmax = 0.0;
    if ((rc = sm_eiso_materials(nx, nz, vp, vs, rho, la, mu, l2m, b, bm, &vpmax))) goto out;
    if (dt > h_ / (sqrt(2.0) * vpmax)) {   /* e_iso.c:476-479 */
        rc = sm_fail(SM_ECFL, "Time step too large (dt > h / (sqrt(2) vpmax))");
        goto out;
    }
    d = malloc(npml * sizeof(double)); dh = malloc(npml * sizeof(double));
    dH = malloc((npml + 1) * sizeof(double));
    if ((rc = sm_eiso_profiles(npml, h_, ncell, vp, d, dh, dH))) goto out;
    if ((rc = sm_read_sources(p.sourcefile, &g, 0, &src, &nsrc, &ntpl))) goto out;
    if ((rc = make_wavelets(src, nsrc, dt, &fct, &len, &stride))) goto out;
    if ((rc = sm_read_records(p.outputfile, &g, 0, &rec, &nrec))) goto out;
    check_dt_trc(rec, nrec, dt);
    const size_t nsteps = sm_nsteps(p.duration, dt);

    if ((rc = sm_eiso_create(0, nx, nz, npml, h_, dt, la, mu, l2m, b, bm, d, dh, dH, p.precision, 1, &h)))
        goto out;
    {   /* sources: add_src (src.c:170-184) acts on Sx, Sz, Sxz and Bulk only */
        size_t *idx = malloc(nsrc * sizeof(size_t)), *ln = malloc(nsrc * sizeof(size_t));
        int *ty = malloc(nsrc * sizeof(int));
        double *w = malloc(nsrc * (stride ? stride : 1) * sizeof(double));
        size_t m = 0;
        for (size_t q = 0; q < nsrc; ++q) {
            int t = src[q].type;
            if (t != SM_SRC_SX && t != SM_SRC_SZ && t != SM_SRC_SXZ && t != SM_SRC_BULK) continue;
            if (src[q].i < 0 || src[q].k < 0 || (size_t)src[q].i >= nx || (size_t)src[q].k >= nz) {
                free(idx); free(ln); free(ty); free(w);
                rc = sm_fail(SM_EINVAL, "source %zu lies outside the grid", q + 1);
                goto out;
            }
            idx[m] = (size_t)src[q].i * nz + (size_t)src[q].k;
            ty[m] = t;
            ln[m] = len[q];
            memcpy(w + m * stride, fct + q * stride, stride * sizeof(double));
            ++m;
        }
        rc = sm_eiso_set_sources(h, 0, m, idx, ty, w, ln, stride, dt);
        free(idx); free(ln); free(ty); free(w);
        if (rc) goto out;
    }
    rp.index = malloc((nrec ? nrec : 1) * sizeof(size_t)); rp.recno = malloc((nrec ? nrec : 1) * sizeof(size_t));
    rp.comp = malloc((nrec ? nrec : 1) * sizeof(int));
    rp.t0 = malloc((nrec ? nrec : 1) * sizeof(double)); rp.rdt = malloc((nrec ? nrec : 1) * sizeof(double));
    for (size_t n = 0; n < nrec; ++n) {
        if (!rec[n].is_trace) continue;   /* snapshots: written as the loop passes them */
        if (rec[n].i < 0 || rec[n].k < 0 || (size_t)rec[n].i >= nx || (size_t)rec[n].k >= nz) {
            rc = sm_fail(SM_EINVAL, "record %zu lies outside the grid", n + 1);
            goto out;
        }
        rp.index[rp.n] = (size_t)rec[n].i * nz + (size_t)rec[n].k;
        rp.comp[rp.n] = rec[n].comp;
        rp.t0[rp.n] = rec[n].t0;
        rp.rdt[rp.n] = rec[n].dt;
        rp.recno[rp.n] = n;
        rp.n++;
    }
    if ((rc = sm_eiso_set_receivers(h, 0, rp.n, rp.index, rp.comp, rp.t0, rp.rdt, nsteps))) goto out;
    if (p.verbose) fprintf(stdout, "Starting main loop (%zu iterations)\n", nsteps);
    {   /* the loop, stopping after each snapshot step (write_snapshot, io_utils.c:1775) */
        snap_ev *ev = NULL;
        size_t nev = 0, done = 0;
        const size_t NX = nx + 2 * npml, NZ = nz + 2 * npml;
        double *field = NULL;
        if ((rc = snap_events(rec, nrec, dt, nsteps, &ev, &nev))) { free(ev); goto out; }
        if (nev && !(field = malloc(NX * NZ * sizeof(double)))) {
            free(ev);
            rc = sm_fail(SM_ENOMEM, "out of host memory");
            goto out;
        }
        for (size_t e = 0; e < nev && !rc; ++e) {
            const size_t upto = ev[e].it + 1;
            if (upto > done) rc = sm_eiso_run(h, upto - done);
            done = upto;
            if (!rc) rc = sm_eiso_get_field(h, 0, rec[ev[e].rec].comp, SM_PART_TOTAL, field);
            if (!rc)
                rc = sm_write_snapshot(p.basename, ev[e].rec + 1, dt * (double)upto, field, NX, NZ,
                                       npml, g.dx, g.dz, g.x0, g.z0, p.plot_strips);
        }
        if (!rc && done < nsteps) rc = sm_eiso_run(h, nsteps - done);
        free(ev);
        free(field);
        if (rc) goto out;
    }
    counts = calloc(rp.n ? rp.n : 1, sizeof(size_t));
    if ((rc = sm_eiso_read_traces(h, 0, 0, rp.n, NULL, 0, counts))) goto out;
    size_t ld = 1;
    for (size_t r = 0; r < rp.n; ++r) ld = counts[r] > ld ? counts[r] : ld;
    vals = malloc(rp.n * ld * sizeof(double) + 1);
    if ((rc = sm_eiso_read_traces(h, 0, 0, rp.n, vals, ld, counts))) goto out;
    rc = write_traces(p.basename, &rp, vals, ld, counts, dt, nsteps);
    if (p.verbose) fprintf(stdout, "\nEnd of computation\n");
out:
    sm_eiso_destroy(h);
    free(vp); free(vs); free(rho); free(la); free(mu); free(l2m); free(b); free(bm);
    free(d); free(dh); free(dH); free(fct); free(len); free(src); free(rec); free(vals); free(counts);
    rec_plan_free(&rp);
    return report(rc, prog);
}

int sm_a_iso_3d_main(int argc, char **argv)
{
    const char *prog = "a_iso_3d_gpu";
    sm_params p;
    sm_grid g;
    double *vp = NULL, *rho = NULL, *fct = NULL, *vals = NULL;
    double *coef[18] = {0};
    size_t *len = NULL, *counts = NULL;
    sm_source *src = NULL;
    sm_record *rec = NULL;
    rec_plan rp = {0};
    sm_a3d_t h = NULL;
    size_t nsrc = 0, ntpl = 1, nrec = 0, stride = 0;
    int rc;

    sm_params_defaults(&p);
    if ((rc = sm_parse_args(argc, argv, &p, prog))) return report(rc, prog);
    if (p.verbose) fprintf(stdout, "\n *** a_iso_3d - Acoustic wave propagation in 3D isotropic media (GPU) ***\n\n");
    if ((rc = sm_read_model_a(p.modelfile, &g, &vp, &rho))) goto out;
    if (g.dx != g.dz) { rc = sm_fail(SM_EINVAL, "grid cell size must be equal in X and Z"); goto out; }
    const size_t np = p.np, nx2 = g.nx + 2 * np, ny2 = g.ny + 2 * np, nz2 = g.nz + 2 * np;
    const size_t n3 = nx2 * ny2 * nz2;
    const double dt = p.dt;
    /* the model stays unpadded on the host: the library replicates its edges
     * (io_utils.c:1096-1143) as it stages the materials */
    {   /* a_iso_3d.c:368-374 and 411-417 */
        double vpmax = sm_a3d_cfl_vpmax_unpadded(g.nx, g.ny, g.nz, np, vp);
        if (dt * vpmax * sqrt(1. / (g.dx * g.dx) + 1. / (g.dy * g.dy) + 1. / (g.dz * g.dz)) > 1.) {
            rc = sm_fail(SM_ECFL, "Time step too large");
            goto out;
        }
    }
    if ((rc = sm_read_sources(p.sourcefile, &g, 1, &src, &nsrc, &ntpl))) goto out;
    if ((rc = make_wavelets(src, nsrc, dt, &fct, &len, &stride))) goto out;
    if ((rc = sm_read_records(p.outputfile, &g, 1, &rec, &nrec))) goto out;
    check_dt_trc(rec, nrec, dt);
    {
        const size_t n2[3] = {nx2, ny2, nz2};
        for (int c = 0; c < 18; ++c) coef[c] = malloc((c < 9 ? n2[c / 3] : n2[(c - 9) / 3]) * sizeof(double));
        if ((rc = sm_a3d_cpml(np, nx2, ny2, nz2, g.dx, g.dy, g.dz, dt, p.pml_order, p.vmax, p.Rc,
                              p.kappa_max, p.alpha_max, src[0].f, coef)))
            goto out;
    }
    const size_t nsteps = sm_nsteps(p.duration, dt);
    if ((rc = sm_a3d_create_unpadded(0, g.nx, g.ny, g.nz, np, g.dx, g.dy, g.dz, dt, vp, rho,
                                     (const double *const *)coef, p.precision, &h)))
        goto out;
    {   /* a_iso_3d.c:689-693: P += dt fct 1e6 for every source type */
        size_t *idx = malloc(nsrc * sizeof(size_t));
        for (size_t q = 0; q < nsrc; ++q) {
            long i = src[q].i + (long)np, j = src[q].j + (long)np, k = src[q].k + (long)np;
            if (i < 0 || j < 0 || k < 0 || (size_t)i >= nx2 || (size_t)j >= ny2 || (size_t)k >= nz2) {
                free(idx);
                rc = sm_fail(SM_EINVAL, "source %zu lies outside the grid", q + 1);
                goto out;
            }
            idx[q] = ((size_t)i * ny2 + (size_t)j) * nz2 + (size_t)k;
        }
        rc = sm_a3d_set_sources(h, nsrc, idx, fct, len, stride, dt * 1.e6);
        free(idx);
        if (rc) goto out;
    }
    rp.index = malloc((nrec ? nrec : 1) * sizeof(size_t)); rp.recno = malloc((nrec ? nrec : 1) * sizeof(size_t));
    rp.comp = malloc((nrec ? nrec : 1) * sizeof(int));
    rp.t0 = malloc((nrec ? nrec : 1) * sizeof(double)); rp.rdt = malloc((nrec ? nrec : 1) * sizeof(double));
    for (size_t n = 0; n < nrec; ++n) {
        if (!rec[n].is_trace) continue;   /* snapshots: written as the loop passes them */
        long i = rec[n].i + (long)np, j = rec[n].j + (long)np, k = rec[n].k + (long)np;
        if (i < 0 || j < 0 || k < 0 || (size_t)i >= nx2 || (size_t)j >= ny2 || (size_t)k >= nz2) {
            rc = sm_fail(SM_EINVAL, "record %zu lies outside the grid", n + 1);
            goto out;
        }
        rp.index[rp.n] = ((size_t)i * ny2 + (size_t)j) * nz2 + (size_t)k;
        rp.comp[rp.n] = rec[n].comp;
        rp.t0[rp.n] = rec[n].t0;
        rp.rdt[rp.n] = rec[n].dt;
        rp.recno[rp.n] = n;
        rp.n++;
    }
    if ((rc = sm_a3d_set_receivers(h, rp.n, rp.index, rp.comp, rp.t0, rp.rdt, nsteps))) goto out;
    if (p.verbose) fprintf(stdout, "Starting main loop (%zu iterations)\n", nsteps);
    {   /* the loop, stopping after each snapshot step: the x-z plane through the
         * first source, at y index (y_src - y0) / dy of the padded grid as
         * a_iso_3d.c:722-730 takes it */
        snap_ev *ev = NULL;
        size_t nev = 0, done = 0;
        double *vol = NULL, *plane = NULL;
        if ((rc = snap_events(rec, nrec, dt, nsteps, &ev, &nev))) { free(ev); goto out; }
        const size_t iy = nsrc ? (size_t)((src[0].y - g.y0) / g.dy) : 0;
        if (nev && iy >= ny2) {
            free(ev);
            rc = sm_fail(SM_EINVAL, "snapshot plane y index %zu outside the grid", iy);
            goto out;
        }
        if (nev && (!(vol = malloc(n3 * sizeof(double))) || !(plane = malloc(nx2 * nz2 * sizeof(double))))) {
            free(ev); free(vol);
            rc = sm_fail(SM_ENOMEM, "out of host memory");
            goto out;
        }
        for (size_t e = 0; e < nev && !rc; ++e) {
            const size_t upto = ev[e].it + 1;
            if (upto > done) rc = sm_a3d_run(h, upto - done);
            done = upto;
            if (!rc) rc = sm_a3d_get_field(h, rec[ev[e].rec].comp, vol);
            if (rc) break;
            for (size_t i = 0; i < nx2; ++i)
                for (size_t k = 0; k < nz2; ++k) plane[i * nz2 + k] = vol[(i * ny2 + iy) * nz2 + k];
            rc = sm_write_snapshot(p.basename, ev[e].rec + 1, dt * (double)upto, plane, nx2, nz2,
                                   np, g.dx, g.dz, g.x0, g.z0, p.plot_strips);
        }
        if (!rc && done < nsteps) rc = sm_a3d_run(h, nsteps - done);
        free(ev); free(vol); free(plane);
        if (rc) goto out;
    }
    counts = calloc(rp.n ? rp.n : 1, sizeof(size_t));
    if ((rc = sm_a3d_read_traces(h, 0, rp.n, NULL, 0, counts))) goto out;
    size_t ld = 1;
    for (size_t r = 0; r < rp.n; ++r) ld = counts[r] > ld ? counts[r] : ld;
    vals = malloc(rp.n * ld * sizeof(double) + 1);
    if ((rc = sm_a3d_read_traces(h, 0, rp.n, vals, ld, counts))) goto out;
    if (p.segy) {   /* save_segy, io_utils.c:3269-3559 */
        sm_record *tr = malloc((rp.n ? rp.n : 1) * sizeof(sm_record));
        double *tt = malloc(rp.n * ld * sizeof(double) + 1);
        if (!tr || !tt) { free(tr); free(tt); rc = sm_fail(SM_ENOMEM, "out of host memory"); goto out; }
        for (size_t r = 0; r < rp.n; ++r) {   /* sample times: t = dt (it + 1), a_iso_3d.c:595 */
            tr[r] = rec[rp.recno[r]];
            size_t s = 0;
            for (size_t it = 0; it < nsteps && s < counts[r]; ++it)
                if (sm_sample_predicate(it, dt, rp.t0[r], rp.rdt[r])) tt[r * ld + s++] = dt * (it + 1);
        }
        rc = sm_write_segy(p.basename, &p, tr, rp.n, nsrc ? &src[0] : NULL, vals, tt, ld, counts);
        free(tr);
        free(tt);
    } else {
        rc = write_traces(p.basename, &rp, vals, ld, counts, dt, nsteps);
    }
    if (p.verbose) fprintf(stdout, "\nEnd of computation\n");
out:
    sm_a3d_destroy(h);
    free(vp); free(rho); free(fct); free(len); free(src); free(rec);
    free(vals); free(counts);
    for (int c = 0; c < 18; ++c) free(coef[c]);
    rec_plan_free(&rp);
    return report(rc, prog);
}

/* div or curl of particle velocity over the grid (compute_div_cyl,
 * compute_curl_cyl, propagate.c:4090-4118), cells it does not reach left zero */
static void ecyl_div_curl(int comp, int n, size_t nx2, size_t nz2, double dx, double dz,
                          const double *vr, const double *vt, const double *vz, double *out)
{
    for (size_t q = 0; q < nx2 * nz2; ++q) out[q] = 0.0;
    if (comp == SM_DIV) {
        for (size_t i = 0; i + 1 < nx2; ++i)
            for (size_t j = 0; j + 1 < nz2; ++j) {
                const size_t q = i * nz2 + j;
                out[q] = ((i + 1) * vr[q + nz2] - i * vr[q]) / (i + 0.5) +
                         n * vt[q] / ((i + 0.5) * dx) + (vz[q + 1] - vz[q]) / dz;
            }
        return;
    }
    if (n % 2)
        for (size_t j = 1; j < nz2; ++j)
            out[j] = (vr[j] - vr[j - 1]) / dz - (vz[j] - -vz[j]) / dx;
    for (size_t i = 1; i < nx2; ++i)
        for (size_t j = 1; j < nz2; ++j) {
            const size_t q = i * nz2 + j;
            out[q] = (vr[q] - vr[q - 1]) / dz - (vz[q] - vz[q - nz2]) / dx;
        }
}

int sm_e_cyl_iso_main(int argc, char **argv)
{
    /* e_cyl_iso.c:277-790: set-up in FP64 through the library's host
     * functions, the loop through the C ABI.  Differences from the
     * reference: force sources are added once per step (the OpenMP build of
     * the reference adds them once per thread, e_cyl_iso.c:612-637); the
     * 9-point source template is refused (io_utils.c:1513-1534 offsets its
     * radial indices by np, which the cylindrical grid does not have);
     * snapshot records are written in the text format of write_snapshot
     * (io_utils.c:1775-1820) with the cylindrical grid's radii, where the
     * reference writes netCDF (write_snapshot_nc, e_cyl_iso.c:781). */
    const char *prog = "e_cyl_iso_gpu";
    sm_params p;
    sm_grid g;
    double *vp = NULL, *vs = NULL, *rho = NULL, *pad[3] = {0}, *mat[8] = {0}, *coef[15] = {0};
    double *fct = NULL, *vals = NULL;
    size_t *len = NULL, *counts = NULL, *sidx = NULL;
    int *stype = NULL;
    sm_source *src = NULL;
    sm_record *rec = NULL;
    rec_plan rp = {0};
    sm_ecyl_t h = NULL;
    size_t nsrc = 0, ntpl = 1, nrec = 0, stride = 0;
    int rc;

    sm_params_defaults(&p);
    if ((rc = sm_parse_args(argc, argv, &p, prog))) return report(rc, prog);
    const size_t np = p.np;   /* 0 with abs 0 (io_utils.c:293) */
    const int n = p.azimuthal_mode;
    if (p.verbose)
        fprintf(stdout, "\n *** e_cyl_iso - Elastic wave propagation in 2.5D isotropic media in "
                        "cylindrical coordinates (GPU) ***\n\n");
    if (n < 0) { rc = sm_fail(SM_EINVAL, "azimuthal_mode must be >= 0"); goto out; }
    if ((rc = sm_read_model_ecyl(p.modelfile, &g, &vp, &vs, &rho))) goto out;
    const size_t nx = g.nx, nz = g.nz, nx2 = nx + np, nz2 = nz + 2 * np, N = nx2 * nz2;
    const double dt = p.dt;
    for (int k = 0; k < 3; ++k)
        if (!(pad[k] = malloc(N * sizeof(double)))) { rc = sm_fail(SM_ENOMEM, "out of host memory"); goto out; }
    for (int k = 0; k < 8; ++k)
        if (!(mat[k] = malloc(N * sizeof(double)))) { rc = sm_fail(SM_ENOMEM, "out of host memory"); goto out; }
    for (int k = 0; k < 15; ++k)
        if (!(coef[k] = malloc((np + 1) * sizeof(double)))) { rc = sm_fail(SM_ENOMEM, "out of host memory"); goto out; }
    if ((rc = sm_ecyl_pad_model(nx, nz, np, vp, vs, rho, pad[0], pad[1], pad[2]))) goto out;
    double vpmax = 0.0;
    if ((rc = sm_ecyl_materials(nx2, nz2, pad[0], pad[1], pad[2], mat, &vpmax))) goto out;
    if (dt > 0.5 * (g.dx + g.dz) / (sqrt(2.0) * vpmax)) {   /* e_cyl_iso.c:484-488 */
        rc = sm_fail(SM_ECFL, "Time step too large");
        goto out;
    }
    if ((rc = sm_read_sources(p.sourcefile, &g, 0, &src, &nsrc, &ntpl))) goto out;
    if (ntpl != 1) {
        rc = sm_fail(SM_EINVAL, "e_cyl_iso takes 1-point sources (the 9-point template of "
                                "io_utils.c:1513-1534 does not fit the cylindrical grid)");
        goto out;
    }
    sidx = malloc(nsrc * sizeof(size_t));
    stype = malloc(nsrc * sizeof(int));
    if (!sidx || !stype) { rc = sm_fail(SM_ENOMEM, "out of host memory"); goto out; }
    for (size_t q = 0; q < nsrc; ++q) {
        if (src[q].i < 0 || src[q].k < 0 || (size_t)src[q].i >= nx2 || (size_t)src[q].k + np >= nz2) {
            rc = sm_fail(SM_EINVAL, "source %zu lies outside the grid", q + 1);
            goto out;
        }
        sidx[q] = (size_t)src[q].i * nz2 + (size_t)src[q].k + np;   /* io_utils.c:1487-1492 */
        stype[q] = src[q].type;
    }
    if (src[0].type == SM_SRC_KURKJIAN) {   /* e_cyl_iso.c:497-502: the first source alone */
        stride = sm_ecyl_kurkjian(src[0].A, src[0].f, dt, 0.0, src[0].x, g.dx, g.dz, n, 0, NULL);
        fct = calloc(stride ? stride : 1, sizeof(double));
        len = calloc(1, sizeof(size_t));
        if (!fct || !len) { rc = sm_fail(SM_ENOMEM, "out of host memory"); goto out; }
        len[0] = sm_ecyl_kurkjian(src[0].A, src[0].f, dt, mat[0][sidx[0]], src[0].x, g.dx, g.dz,
                                  n, stride, fct);
        nsrc = 1;
    } else if ((rc = make_wavelets(src, nsrc, dt, &fct, &len, &stride))) {
        goto out;
    }
    {   /* CPML, e_cyl_iso.c:529-535 */
        const double pi = 4.0 * atan(1.0);
        const double alpha = p.alpha_max ? pi * src[0].f : 0.0;
        if ((rc = sm_ecyl_cpml(np, g.dx, g.dz, dt, p.pml_order, p.vmax, p.Rc, p.kappa_max, alpha,
                               p.iwipe, coef)))
            goto out;
    }
    if ((rc = sm_read_records(p.outputfile, &g, 0, &rec, &nrec))) goto out;
    check_dt_trc(rec, nrec, dt);
    const size_t nsteps = sm_nsteps(p.duration, dt);
    if ((rc = sm_ecyl_create(0, nx, nz, np, n, g.dx, g.dz, dt, (const double *const *)mat,
                             (const double *const *)coef, p.precision, &h)))
        goto out;
    if ((rc = sm_ecyl_set_sources(h, nsrc, sidx, stype, fct, len, stride))) goto out;
    rp.index = malloc((nrec ? nrec : 1) * sizeof(size_t)); rp.recno = malloc((nrec ? nrec : 1) * sizeof(size_t));
    rp.comp = malloc((nrec ? nrec : 1) * sizeof(int));
    rp.t0 = malloc((nrec ? nrec : 1) * sizeof(double)); rp.rdt = malloc((nrec ? nrec : 1) * sizeof(double));
    for (size_t r = 0; r < nrec; ++r) {
        if (!rec[r].is_trace) continue;   /* snapshots: written as the loop passes them */
        if (rec[r].i < 0 || rec[r].k < 0 || (size_t)rec[r].i >= nx2 || (size_t)rec[r].k + np >= nz2) {
            rc = sm_fail(SM_EINVAL, "record %zu lies outside the grid", r + 1);
            goto out;
        }
        rp.index[rp.n] = (size_t)rec[r].i * nz2 + (size_t)rec[r].k + np;   /* io_utils.c:1661-1666 */
        rp.comp[rp.n] = rec[r].comp;
        rp.t0[rp.n] = rec[r].t0;
        rp.rdt[rp.n] = rec[r].dt;
        rp.recno[rp.n] = r;
        rp.n++;
    }
    if ((rc = sm_ecyl_set_receivers(h, rp.n, rp.index, rp.comp, rp.t0, rp.rdt, nsteps))) goto out;
    if (p.verbose) fprintf(stdout, "Starting main loop (%zu iterations)\n", nsteps);
    {   /* the loop, stopping after each snapshot step (e_cyl_iso.c:768-785) */
        snap_ev *ev = NULL;
        size_t nev = 0, done = 0;
        double *field = NULL, *vr = NULL, *vt = NULL, *vz = NULL;
        if ((rc = snap_events(rec, nrec, dt, nsteps, &ev, &nev))) { free(ev); goto out; }
        if (nev && (!(field = calloc(N, sizeof(double))) || !(vr = malloc(N * sizeof(double))) ||
                    !(vt = malloc(N * sizeof(double))) || !(vz = malloc(N * sizeof(double))))) {
            free(ev); free(field); free(vr); free(vt);
            rc = sm_fail(SM_ENOMEM, "out of host memory");
            goto out;
        }
        for (size_t e = 0; e < nev && !rc; ++e) {
            const size_t upto = ev[e].it + 1;
            if (upto > done) rc = sm_ecyl_run(h, upto - done);
            done = upto;
            const int comp = rec[ev[e].rec].comp;
            if (!rc && comp != SM_DIV && comp != SM_CURL) rc = sm_ecyl_get_field(h, comp, field);
            if (!rc && (comp == SM_DIV || comp == SM_CURL)) {
                if (!(rc = sm_ecyl_get_field(h, SM_VR, vr)) && !(rc = sm_ecyl_get_field(h, SM_VT, vt)))
                    rc = sm_ecyl_get_field(h, SM_VZ, vz);
                if (!rc) ecyl_div_curl(comp, n, nx2, nz2, g.dx, g.dz, vr, vt, vz, field);
            }
            if (!rc)
                rc = sm_write_snapshot_cyl(p.basename, ev[e].rec + 1, dt * (double)upto, field, nx2,
                                           nz2, np, g.dx, g.dz, g.x0, g.z0, p.plot_strips);
        }
        if (!rc && done < nsteps) rc = sm_ecyl_run(h, nsteps - done);
        free(ev); free(field); free(vr); free(vt); free(vz);
        if (rc) goto out;
    }
    counts = calloc(rp.n ? rp.n : 1, sizeof(size_t));
    if ((rc = sm_ecyl_read_traces(h, 0, rp.n, NULL, 0, counts))) goto out;
    size_t ld = 1;
    for (size_t r = 0; r < rp.n; ++r) ld = counts[r] > ld ? counts[r] : ld;
    vals = malloc(rp.n * ld * sizeof(double) + 1);
    if ((rc = sm_ecyl_read_traces(h, 0, rp.n, vals, ld, counts))) goto out;
    rc = write_traces(p.basename, &rp, vals, ld, counts, dt, nsteps);
    if (p.verbose) fprintf(stdout, "\nEnd of computation\n");
out:
    sm_ecyl_destroy(h);
    free(vp); free(vs); free(rho);
    for (int k = 0; k < 3; ++k) free(pad[k]);
    for (int k = 0; k < 8; ++k) free(mat[k]);
    for (int k = 0; k < 15; ++k) free(coef[k]);
    free(fct); free(len); free(sidx); free(stype); free(src); free(rec); free(vals); free(counts);
    rec_plan_free(&rp);
    return report(rc, prog);
}
