/*
 * sm_io.h -- readers of the reference's input files and the trace writer,
 * for the drop-in programs (sm_drivers.c).  Same formats and semantics as
 * io_utils.c; failures return a status instead of exiting.
 */
#ifndef SM_IO_H
#define SM_IO_H

#include <stddef.h>
#include <stdio.h>

#include "sm_host.h"

#ifdef __cplusplus
extern "C" {
#endif

/* inputParams + abs_params, structs.h:49-60, 80-105 (the fields this path uses) */
typedef struct {
    double dt;           /* s (the file holds ms) */
    double duration;     /* s */
    char modelfile[256], sourcefile[256], outputfile[256], basename[256];
    int iwipe;           /* "abs" */
    size_t np;           /* "nl" */
    int segy, shotpt_no, simulate_cmp;
    double Rc, kappa_max, vmax, pml_order;
    int alpha_max;
    int verbose;
    int plot_strips;     /* "plstr": snapshots include the absorbing frame */
    int azimuthal_mode;  /* e_cyl_iso: "azimuthal_mode" n */
    int precision;       /* SM_FP32 by default; "-P" */
} sm_params;

typedef struct {
    size_t nx, ny, nz;   /* ny = 1 for 2-D models */
    double dx, dy, dz, x0, y0, z0;
} sm_grid;

typedef struct {
    int type;            /* enum sourceType numbering (SM_SRC_*) */
    double A, f, x, y, z;
    long i, j, k;        /* node indices (interior, before any padding) */
} sm_source;

typedef struct {
    int comp;            /* enum component numbering (SM_VX ...) */
    int is_trace;        /* 0: snapshot record */
    double x, y, z, t0, dt;
    long i, j, k;
} sm_record;

/* defaults of set_defaults / set_defaults_3d (io_utils.c:63-135) */
void sm_params_defaults(sm_params *p);
/* command line + parameter file, io_utils.c:156-294 ("-P" added) */
int sm_parse_args(int argc, char **argv, sm_params *p, const char *prog);
int sm_read_par(const char *path, sm_params *p);
/* model files: e_iso (io_utils.c:296-328, 892-947) and a_iso_3d
 * (io_utils.c:384-401, 1029-1153, interior values only: padding is done by
 * sm_a3d_pad_model).  A file that starts with "SEISMODB" is read as a binary
 * model instead (layout in sm_io.c).  Arrays are malloc'ed; the caller frees
 * them. */
int sm_read_model_e(const char *path, sm_grid *g, double **vp, double **vs, double **rho);
int sm_read_model_a(const char *path, sm_grid *g, double **vp, double **rho);
/* e_cyl_iso model (io_utils.c:949-991, keyword isotropic_elastic_cyl; rows
 * are z, r fastest, one row = a radial profile); interior nx*nz values,
 * index i*nz + j, padding by sm_ecyl_pad_model.  Binary files as e_iso. */
int sm_read_model_ecyl(const char *path, sm_grid *g, double **vp, double **vs, double **rho);
/* source and output files (io_utils.c:1432-1741); *src / *rec malloc'ed */
int sm_read_sources(const char *path, const sm_grid *g, int three_d, sm_source **src,
                    size_t *nsrc, size_t *ntemplate);
int sm_read_records(const char *path, const sm_grid *g, int three_d, sm_record **rec,
                    size_t *nrec);
/* trc/<base>/<base>_<n>.trc, "%le    %le" of t and 1e3 * v (io_utils.c:1744-1768) */
int sm_write_trace_file(const char *base, size_t n, const double *t, const double *v,
                        size_t ns);
/* every receiver's trace file of a run (receiver r: file recno[r] + 1, its
 * counts[r] samples vals[r * ld ...] at the times dt * (it + 1) of the steps
 * it < nsteps that sm_sample_predicate(it, dt, t0[r], rdt[r]) keeps), the
 * files split over host threads; the first failure in receiver order is
 * returned */
int sm_write_trace_set(const char *base, size_t nrec, const size_t *recno, const double *t0,
                       const double *rdt, double dt, size_t nsteps, const double *vals, size_t ld,
                       const size_t *counts);
/* segy/<base>.sgy with the layout save_segy writes (io_utils.c:3269-3559):
 * 3200-byte textual header, 400-byte binary header, per trace a 240-byte
 * header and its samples as IEEE float32, all in the host's byte order as the
 * reference writes them.  Sample i of a trace is the value at time i*dt_r
 * (dt_r the record's interval), as fill_data_segy (io_utils.c:1770-1773)
 * places it; but where that routine keeps round(duration/dt_r) samples, so
 * that the last one lands one past its array and sample 0 (t = 0, never
 * recorded) is left uninitialised, each trace here holds
 * round(duration/dt_r) + 1 samples and every sample not recorded is zero.
 * Pressure traces are written too (trace code 11, the SEG-Y code of a
 * pressure sensor); the reference leaves them out.
 * rec[r]: the record of trace r; v, t: ntr rows of ld recorded values and
 * their times; count[r] of them. */
/* ssh/<base>/<base>_<n>_<t>.ssh, the text snapshot of write_snapshot
 * (io_utils.c:1775-1820): "%le  %le  %le" of x, z and 1e3 * value per node,
 * x slow; the interior nodes, or every node of the padded nx2 x nz2 plane
 * when plot_strips.  data: the padded plane, index i*nz2 + k. */
int sm_write_snapshot(const char *base, size_t n, double t, const double *data, size_t nx2,
                      size_t nz2, size_t np, double dx, double dz, double x0, double z0,
                      int plot_strips);
/* the same for the cylindrical grid of e_cyl_iso (nx2 = nx + np: no
 * absorbing columns before the axis) */
int sm_write_snapshot_cyl(const char *base, size_t n, double t, const double *data, size_t nx2,
                          size_t nz2, size_t np, double dx, double dz, double x0, double z0,
                          int plot_strips);
int sm_write_segy(const char *base, const sm_params *p, const sm_record *rec, size_t ntr,
                  const sm_source *src0, const double *v, const double *t, size_t ld,
                  const size_t *count);

#ifdef __cplusplus
}
#endif
#endif
