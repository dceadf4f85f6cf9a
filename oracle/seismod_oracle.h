/*
 * seismod_oracle.h -- FP64 CPU restatement of the seismod FDTD hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA path: only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark load
 * it.  The product library never links or calls anything declared here.
 *
 * It restates, in our own padded-grid formulation, the algorithm of
 *   e_iso     (2D P-SV elastic, velocity-stress staggered grid, split-field
 *              PML; e_iso.c:423-670, propagate.c:2511-2670, pml.c:39-1403)
 *   a_iso_3d  (3D acoustic, velocity-pressure staggered grid, CPML;
 *              a_iso_3d/a_iso_3d.c:368-693)
 *   e_cyl_iso (2.5-D elastic in r, z with azimuthal mode n, CPML;
 *              e_cyl_iso.c:363-790, propagate.c:2706-4118, pml.c:2107-2185;
 *              oracle_ecyl.c)
 * plus the host-side set-up they share (src.c:43-65,170-184;
 * io_utils.c:892-947,1029-1153,1744-1768).
 *
 * Layout.  e_iso grids are held padded: NX = nx + 2*np columns (x, slow) by
 * NZ = nz + 2*np rows (z, fast), index X*NZ + Z.  Inside the interior
 * [np, np+nx) x [np, np+nz) a field is one total value; in the absorbing
 * frame it is the sum of an x part and a z part (Collino & Tsogka split).
 * a_iso_3d grids use the reference's own padded layout ((i*ny2+j)*nz2+k).
 *
 * Parity is pinned by the tests against the reference itself: the reference
 * update functions compiled from their own sources (oracle/_ref/libref_eiso.so)
 * and the reference programs oracle/_ref/e_iso and oracle/_ref/a_iso_3d.
 */
#ifndef SEISMOD_ORACLE_H
#define SEISMOD_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* field ids, e_iso */
enum { ORC_VX = 0, ORC_VZ = 1, ORC_TXX = 2, ORC_TZZ = 3, ORC_TXZ = 4 };
/* field ids, a_iso_3d */
enum { ORC_A_VX = 0, ORC_A_VY = 1, ORC_A_VZ = 2, ORC_A_P = 3 };
/* which part of an e_iso field: total, x split part, z split part */
enum { ORC_TOTAL = 0, ORC_XPART = 1, ORC_ZPART = 2 };

/* ---------------- shared host-side set-up ---------------- */

/* Ricker wavelets, src.c:43-65, including its normalisation order (every
 * pass rescales source 0).  fct is n*maxlen, row s holds len[s] samples. */
void orc_src_fct(size_t n, const double *A, const double *f, double dt, double fac,
                 size_t maxlen, double *fct, size_t *len);
/* number of samples compute_src_fct allocates for frequency f, src.c:48 */
size_t orc_src_len(double f, double dt, double fac);
/* time-step count, e_iso.c:575-576 / a_iso_3d.c:578-579 */
size_t orc_nsteps(double duration, double dt);
/* receiver sampling predicate at step it, e_iso.c:643-658 */
int orc_sample(size_t it, double dt, double t0, double rdt);

/* ---------------- e_iso ---------------- */

/* material set-up e_iso.c:423-462; returns max vp (the CFL input) */
double orc_eiso_materials(size_t nx, size_t nz, const double *vp, const double *vs,
                          const double *rho, double *la, double *mu, double *l2m,
                          double *b, double *bm);
/* PML profile e_iso.c:482-500 (d0 from the MEAN vp) */
void orc_eiso_profiles(size_t np, double h, size_t ncell, const double *vp,
                       double *d, double *dh, double *dH);

typedef struct orc_eiso orc_eiso;
orc_eiso *orc_eiso_new(size_t nx, size_t nz, size_t np, double h, double dt,
                       const double *la, const double *mu, const double *l2m,
                       const double *b, const double *bm,
                       const double *d, const double *dh, const double *dH);
void orc_eiso_free(orc_eiso *o);
void orc_eiso_velocity(orc_eiso *o);                 /* e_iso.c:597-615 */
void orc_eiso_stress(orc_eiso *o);                   /* e_iso.c:616-634 */
/* add_src, src.c:170-184: index is the interior index i*nz+j */
void orc_eiso_add_source(orc_eiso *o, size_t index, int type, double value);
/* copy a padded field (NX*NZ) out / in.  For ORC_TOTAL the PML cells hold
 * x part + z part.  ORC_XPART / ORC_ZPART are zero in the interior. */
void orc_eiso_get(const orc_eiso *o, int field, int part, double *out);
void orc_eiso_set(orc_eiso *o, int field, int part, const double *in);
/* interior value at i*nz+j (what a receiver reads), e_iso.c:646-661 */
/* storage-rounding checker mode: 0 = FP64 storage (default); B > 0 = the
 * state is rounded to 16-bit block floating point (blocks of B cells along
 * X or Z of the padded grid) when a step stores it (no counterpart in the
 * reference) */
void orc_eiso_set_bfp(orc_eiso *o, int block, int axis);   /* axis 0: X, 1: Z */
/* a rectangle of padded cells (first X, first Z, rows, columns) the block
 * storage keeps exact: the source patches of the device's block storage */
void orc_eiso_add_patch(orc_eiso *o, long X0, long Z0, long rows, long cols);
double orc_eiso_probe(const orc_eiso *o, int field, size_t index);

/* ---------------- a_iso_3d ---------------- */

/* model padding by edge replication, io_utils.c:1096-1143.  vp_in/rho_in
 * are nx*ny*nz interior values; the outputs are nx2*ny2*nz2. */
void orc_a3d_pad_model(size_t nx, size_t ny, size_t nz, size_t np,
                       const double *vp_in, const double *rho_in,
                       double *vp_pad, double *rho_pad);
/* the vp maximum a_iso_3d feeds its CFL test (a 2-D sub-scan of the padded
 * array, a_iso_3d.c:368-374) */
double orc_a3d_cfl_vpmax(size_t nx, size_t nz, const double *vp_pad);
/* CPML coefficients a_iso_3d.c:500-576.  Node arrays have n2 entries, half
 * node arrays n2-1, per axis.  coef is 18 pointers in the order
 * ax bx kx ay by ky az bz kz ax_h bx_h kx_h ay_h by_h ky_h az_h bz_h kz_h. */
void orc_a3d_cpml(size_t np, size_t nx2, size_t ny2, size_t nz2,
                  double dx, double dy, double dz, double dt,
                  double pml_order, double vmax, double Rc, double kappa_max,
                  int alpha_max_flag, double f0, double *const *coef);

typedef struct orc_a3d orc_a3d;
orc_a3d *orc_a3d_new(size_t nx2, size_t ny2, size_t nz2, double dx, double dy, double dz,
                     double dt, const double *vp_pad, const double *rho_pad,
                     const double *const *coef);
void orc_a3d_free(orc_a3d *o);
void orc_a3d_velocity(orc_a3d *o);                   /* a_iso_3d.c:601-652 */
void orc_a3d_pressure(orc_a3d *o);                   /* a_iso_3d.c:655-684 */
void orc_a3d_add_source(orc_a3d *o, size_t index, double value); /* :689-693 */
void orc_a3d_get(const orc_a3d *o, int field, double *out);
void orc_a3d_set(orc_a3d *o, int field, const double *in);
double orc_a3d_probe(const orc_a3d *o, int field, size_t index);
/* out[r] = field[r] at index[r], r < n */
void orc_a3d_gather(const orc_a3d *o, size_t n, const int *field, const size_t *index,
                    double *out);
/* storage-rounding checker mode: 0 = FP64 storage (default); B > 0 = every
 * stored value rounded to 16-bit block floating point with blocks of B
 * cells along y or z (no counterpart in the reference) */
void orc_a3d_set_bfp(orc_a3d *o, int block, int axis);     /* axis 1: y, 2: z */

/* ---------------- e_cyl_iso (oracle_ecyl.c) ---------------- */

/* padded grid nx2 = nx + np (PML at the outer radius only) by
 * nz2 = nz + 2 np, index i*nz2 + j.  Fields: */
enum { ORC_C_VR = 0, ORC_C_VT, ORC_C_VZ, ORC_C_TRR, ORC_C_TTT, ORC_C_TZZ, ORC_C_TRZ,
       ORC_C_TRT, ORC_C_TTZ, ORC_C_DIV, ORC_C_CURL };
/* source types, numbered as enum sourceType (structs.h:44) */
enum { ORC_C_SRC_BULK = 6, ORC_C_SRC_FR = 9, ORC_C_SRC_FT = 10, ORC_C_SRC_FZ = 11,
       ORC_C_SRC_KURKJIAN = 12 };
typedef struct orc_ecyl orc_ecyl;
/* e_cyl_iso.c:363-441 on the padded model; returns max vp */
double orc_ecyl_materials(size_t nx2, size_t nz2, const double *vp, const double *vs,
                          const double *rho, double *lij, double *l2mij, double *mu,
                          double *mui, double *muj, double *bi, double *bj, double *bij);
/* pml.c:2107-2185; c: 15 arrays ik_r ik_z ikh_z b_r c_r b_z c_z bh_z ch_z
 * (np values) then ikH_r ikH_z bH_r cH_r bH_z cH_z (np + 1 values) */
void orc_ecyl_cpml(size_t np, double dx, double dz, double dt, double order, double vmax,
                   double Rc, double kappa_max, double alpha_max, int absorb,
                   double *const *c);
/* src.c:202-228 compute_kurkjian; returns the sample count */
size_t orc_ecyl_kurkjian(double A, double f, double dt, double lij_at_src, double x_src,
                         double dx, double dz, int n, size_t maxlen, double *fct);
/* mat: lij l2mij mu mui muj bi bj bij (padded); coef as orc_ecyl_cpml */
orc_ecyl *orc_ecyl_new(size_t nx, size_t nz, size_t np, int n, double dx, double dz, double dt,
                       const double *const *mat, const double *const *coef);
void orc_ecyl_free(orc_ecyl *o);
void orc_ecyl_velocity(orc_ecyl *o);       /* vr, vt, vz */
void orc_ecyl_stress(orc_ecyl *o);         /* trr ttt tzz, trz, trt, ttz */
void orc_ecyl_force(orc_ecyl *o, size_t index, int type, double value);   /* src.c:186-199 */
void orc_ecyl_kurkjian_add(orc_ecyl *o, size_t index, double value);     /* src.c:231-236 */
void orc_ecyl_get(const orc_ecyl *o, int field, double *out);
void orc_ecyl_set(orc_ecyl *o, int field, const double *in);
double orc_ecyl_probe(const orc_ecyl *o, int comp, size_t index);         /* with div, curl */

#ifdef __cplusplus
}
#endif
#endif
