/*
 * seismod_gpu.h -- C ABI of the B200 (sm_100a) FDTD library.
 *
 * Drop-in for the time loops of two seismod programs:
 *
 *   e_iso     2D P-SV elastic, velocity-stress staggered grid, split-field
 *             PML (Collino & Tsogka 2001)
 *   a_iso_3d  3D acoustic, velocity-pressure staggered grid, CPML
 *
 * The reference has no library interface: its time loops call C functions on
 * raw double arrays from main().  Each entry point below names the reference
 * code it replaces (file:line in the seismod sources).  Every function returns
 * an int status (SM_OK = 0); none exits or aborts; sm_last_error() gives a
 * message for the last failure on the calling thread.  Handles are not
 * thread-safe: use one handle per thread, or serialise calls on it.
 *
 * All array arguments are host pointers.  Layouts are the reference's:
 *   e_iso     interior arrays nx*nz, index i*nz + j (x slow, z fast),
 *             e_iso.c:384-393
 *   a_iso_3d  padded arrays nx2*ny2*nz2, index (i*ny2 + j)*nz2 + k,
 *             a_iso_3d.c:317-335 (nx2 = nx + 2*np, io_utils.c:396-398)
 */
#ifndef SEISMOD_GPU_H
#define SEISMOD_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SM_ABI_VERSION 1

/* status codes */
#define SM_OK        0
#define SM_EINVAL    1   /* bad argument                                    */
#define SM_ENOMEM    2   /* device or host allocation failed                */
#define SM_ECUDA     3   /* CUDA runtime error                              */
#define SM_ECFL      4   /* time step violates the reference's CFL test     */
#define SM_EIO       5   /* file could not be opened / parsed               */
#define SM_ETIMEOUT  6   /* a bounded wait gave up                          */
#define SM_EBUSY     7   /* admission refused: not enough device memory     */
#define SM_ESTATE    8   /* call not valid in the handle's current state    */
#define SM_ENOTFOUND 9   /* unknown ticket / index                          */

/* storage precision of wavefields and PML/CPML memory variables.
 * FP32 and FP64 compute in their own type; FP16 and BF16 store 16-bit values
 * with one power-of-two scale per field and compute in FP32.  BFP16 (block
 * floating point) stores the wavefields as 16-bit integer mantissas sharing
 * one 8-bit exponent per block of cells (a_iso_3d: 4 consecutive y rows of a
 * z column; e_iso: 4 consecutive x rows of a z column), set from the block's
 * largest value at every store, and computes in FP32; the CPML memory
 * variables and split parts stay FP32, and e_iso keeps the 20 x 9 cells
 * around each source in FP32 as well.  The reference stores FP64
 * (a_iso_3d.c:319-335, e_iso.c:384-411); BFP16 is the reduced-storage form
 * whose trace error stays below 1e-3 of FP64 on the benchmark shots. */
#define SM_FP32 0
#define SM_FP64 1
#define SM_FP16 2
#define SM_BF16 3
#define SM_BFP16 4

/* source types, numbered as enum sourceType (structs.h:44) */
#define SM_SRC_SX   0
#define SM_SRC_SZ   2
#define SM_SRC_SXZ  4
#define SM_SRC_BULK 6
#define SM_SRC_FR   9    /* e_cyl_iso force sources */
#define SM_SRC_FT   10
#define SM_SRC_FZ   11
#define SM_SRC_KURKJIAN 12

/* record components, numbered as enum component (structs.h:45) */
#define SM_VX   0
#define SM_VY   1
#define SM_VZ   2
#define SM_TXX  5
#define SM_TZZ  6
#define SM_TXZ  7
#define SM_P    8
#define SM_DIV  11   /* e_cyl_iso: divergence of particle velocity */
#define SM_CURL 12   /* e_cyl_iso: curl of particle velocity */
#define SM_VR   13
#define SM_VT   14   /* v_theta */
#define SM_TRR  15
#define SM_TRT  16   /* tau_r theta */
#define SM_TRZ  17
#define SM_TTT  18   /* tau_theta theta */
#define SM_TTZ  19   /* tau_theta z */

/* which part of an e_iso field: the total, or the x / z split part that the
 * PML frame carries (pml.c keeps q_x and q_z, q = q_x + q_z) */
#define SM_PART_TOTAL 0
#define SM_PART_X     1
#define SM_PART_Z     2

/* pass as `shot` to apply a call to every shot of a batch */
#define SM_ALL_SHOTS ((size_t)-1)

const char *sm_last_error(void);
int sm_abi_version(void);
/* device count and the SM count / HBM size of one device */
int sm_device_info(int device, int *sm_count, size_t *hbm_bytes, size_t *hbm_free);

/* Cache of the handles' large device arrays (no counterpart in the
 * reference, whose programs allocate once per run).  Destroying an e_iso or
 * a_iso_3d handle gives its wavefield, memory-variable and material arrays
 * to a per-device cache, and creating a handle takes blocks of the same size
 * (rounded to 2 MiB) from it, so shot after shot runs without cudaMalloc /
 * cudaFree of the state.  At most `bytes` per device stay cached (32 GiB by
 * default); sm_pool_trim frees every cached block, and an allocation that
 * fails trims the cache and tries once more.  sm_pool_cached reports the
 * bytes held. */
int sm_pool_trim(int device, size_t *freed);
int sm_pool_set_limit(int device, size_t bytes);
int sm_pool_cached(int device, size_t *bytes);

/* ======================================================================
 * host-side set-up, FP64, identical in arithmetic to the reference
 * ====================================================================== */

/* Ricker wavelets of n sources, src.c:43-65 compute_src_fct (including its
 * normalisation order: every pass rescales wavelet 0).  Row s of fct (stride
 * doubles) receives length[s] samples.  sm_ricker_length gives the length
 * the reference allocates for one source. */
size_t sm_ricker_length(double f, double dt, double fac);
int sm_ricker(size_t n, const double *A, const double *f, double dt, double fac,
              size_t stride, double *fct, size_t *length);
/* time-step count, e_iso.c:575-576 */
size_t sm_nsteps(double duration, double dt);
/* receiver sampling predicate at step it, e_iso.c:643-658 */
int sm_sample_predicate(size_t it, double dt, double t0, double rdt);

/* e_iso material averaging e_iso.c:423-462 (returns max vp through vpmax)
 * and PML damping profiles e_iso.c:482-500 (d, dh: np values; dH: np+1) */
int sm_eiso_materials(size_t nx, size_t nz, const double *vp, const double *vs,
                      const double *rho, double *la, double *mu, double *l2m,
                      double *b, double *bm, double *vpmax);
int sm_eiso_profiles(size_t np, double h, size_t ncell, const double *vp,
                     double *d, double *dh, double *dH);

/* a_iso_3d model padding by edge replication (io_utils.c:1096-1143), the
 * vp maximum its CFL test uses (a_iso_3d.c:368-374) and its CPML
 * coefficients (a_iso_3d.c:500-576).  coef: 18 arrays in the order
 * ax bx kx ay by ky az bz kz (n2 values each) then ax_h ... kz_h (n2-1). */
int sm_a3d_pad_model(size_t nx, size_t ny, size_t nz, size_t np,
                     const double *vp, const double *rho, double *vp_pad, double *rho_pad);
double sm_a3d_cfl_vpmax(size_t nx, size_t nz, const double *vp_pad);
/* the same maximum from the unpadded nx x ny x nz model (no reference
 * counterpart: sm_a3d_cfl_vpmax of sm_a3d_pad_model's output, without it) */
double sm_a3d_cfl_vpmax_unpadded(size_t nx, size_t ny, size_t nz, size_t np, const double *vp);
int sm_a3d_cpml(size_t np, size_t nx2, size_t ny2, size_t nz2,
                double dx, double dy, double dz, double dt,
                double pml_order, double vmax, double Rc, double kappa_max,
                int alpha_max_flag, double f0, double *const *coef);

/* ======================================================================
 * e_iso on the device
 * ====================================================================== */

typedef struct sm_eiso *sm_eiso_t;

/* Replaces the allocations of e_iso.c:384-411 and the state the time loop
 * e_iso.c:589-670 updates.  la, mu, l2m, b, bm are the averaged materials
 * that update_vx/update_vz/update_txxzz/update_txz (propagate.c:2511-2670)
 * and pml_v/pml_t (pml.c:39,684) receive; d, dh, dH the PML profiles.
 * nshots independent shots share the model (batched launch).  npml >= 1
 * (the reference indexes [npml-1] and fails for npml = 0,
 * propagate.c:2519). */
int sm_eiso_create(int device, size_t nx, size_t nz, size_t npml, double h, double dt,
                   const double *la, const double *mu, const double *l2m,
                   const double *b, const double *bm,
                   const double *d, const double *dh, const double *dH,
                   int precision, size_t nshots, sm_eiso_t *out);

/* Sources of one shot (or SM_ALL_SHOTS), add_src src.c:170-184: at step it
 * every source with it < length[s] adds scale * fct[s*stride + it] to txx
 * (Sx, Bulk), tzz (Sz, Bulk) or txz (Sxz) at interior index[s] = i*nz + j.
 * The reference uses scale = dt.  Replaces the previous source set. */
int sm_eiso_set_sources(sm_eiso_t h, size_t shot, size_t nsrc, const size_t *index,
                        const int *type, const double *fct, const size_t *length,
                        size_t stride, double scale);

/* Trace records of one shot (or SM_ALL_SHOTS), e_iso.c:641-669: receiver r
 * reads component comp[r] (SM_VX or SM_VZ; SM_TXX/SM_TZZ/SM_TXZ also work)
 * at interior index[r] after every step it for which
 * sm_sample_predicate(it, dt, t0[r], rdt[r]) holds, for it < nsteps_max.
 * Resets the sample counters. */
int sm_eiso_set_receivers(sm_eiso_t h, size_t shot, size_t nrec, const size_t *index,
                          const int *comp, const double *t0, const double *rdt,
                          size_t nsteps_max);

/* Advance every shot by nsteps time steps (the body of e_iso.c:589-670).
 * Asynchronous: returns once the work is queued. */
int sm_eiso_run(sm_eiso_t h, size_t nsteps);
/* Advance n handles of possibly different grid sizes, shot counts and
 * sources together by nsteps steps each (the same loop, e_iso.c:589-670,
 * for several models at once): each step is one launch over the slabs of
 * all of them (up to 32 handles per launch), one for all their sources and
 * one for all their receivers.  Every handle ends bit for bit where
 * sm_eiso_run(handles[k], nsteps) would leave it.  Same device and
 * precision for all; the work is queued on handles[0]'s stream after the
 * work already queued on every handle's stream, and every handle's stream
 * waits for it.  Asynchronous like sm_eiso_run. */
int sm_eiso_group_run(sm_eiso_t const *handles, int n, size_t nsteps);
int sm_eiso_sync(sm_eiso_t h);
/* steps taken so far */
int sm_eiso_step_count(sm_eiso_t h, size_t *it);

/* Copy the samples taken so far: values (raw field values; the reference
 * writes 1e3*v, io_utils.c:1767) of receivers [rec0, rec0+nrec) into
 * out[r*ld + s]; counts[r] receives the number of samples.  Synchronises. */
int sm_eiso_read_traces(sm_eiso_t h, size_t shot, size_t rec0, size_t nrec,
                        double *out, size_t ld, size_t *counts);

/* Whole padded field (NX*NZ, NX = nx+2*npml, NZ = nz+2*npml, index X*NZ+Z)
 * of one shot: SM_PART_TOTAL, or a split part (zero inside the interior).
 * set_field loads a state (tests, restarts); for SM_PART_TOTAL it writes
 * interior cells only, PML totals follow from the parts. */
int sm_eiso_get_field(sm_eiso_t h, size_t shot, int comp, int part, double *out);
int sm_eiso_set_field(sm_eiso_t h, size_t shot, int comp, int part, const double *in);
/* zero all wavefields and counters of every shot (e_iso.c:565-572) */
int sm_eiso_reset(sm_eiso_t h);
int sm_eiso_destroy(sm_eiso_t h);
/* the cudaStream_t the handle launches on (for timing with CUDA events) */
int sm_eiso_stream(sm_eiso_t h, void **stream);
/* launch configuration of the step kernel (warps per CTA, register cap),
 * an index in [0, *nconfigs); results do not depend on it */
int sm_eiso_set_config(sm_eiso_t h, int config);
int sm_eiso_get_config(sm_eiso_t h, int *config, int *nconfigs);
/* Autotuner: times every launch configuration that fits for trial_steps
 * steps (<= 0: 32) from a zero state and keeps the fastest; with graphs set
 * (sm_eiso_set_graph) the trials replay them, their capture untimed.
 * Results are cached per (precision, grid, shots, device) for the process.
 * Call at step 0 (or after sm_eiso_reset); the handle is left reset.  Any
 * output pointer may be NULL. */
int sm_eiso_autotune(sm_eiso_t h, int trial_steps, int *config, double *ms_per_step);
/* Replay the time loop as CUDA graphs of `steps` steps (2, 4, 8 or 16; 0
 * launches every kernel from the host, the default).  Results are the same
 * either way.  Graphs are captured lazily and again after new sources,
 * receivers, configurations or 16-bit scales.  With per-kernel timing on
 * (sm_eiso_set_timing) the graphs are captured again with event nodes
 * around each update launch, and the host waits for every replay. */
int sm_eiso_set_graph(sm_eiso_t h, int steps);
/* Per-kernel timing.  With timing on, every launch of the wavefield update
 * kernel(s) is bracketed by CUDA events on the handle's stream;
 * sm_eiso_kernel_stats synchronises and returns their summed duration and
 * launch count since the last reset, plus the number of kernels of every
 * kind launched (update, sources, receivers). */
int sm_eiso_set_timing(sm_eiso_t h, int on);
int sm_eiso_kernel_stats(sm_eiso_t h, int reset, double *update_ms, size_t *update_launches,
                         size_t *all_launches);

/* ======================================================================
 * a_iso_3d on the device
 * ====================================================================== */

typedef struct sm_a3d *sm_a3d_t;

/* Replaces the allocations of a_iso_3d.c:317-355, the material set-up
 * a_iso_3d.c:379-409 and the state of the time loop a_iso_3d.c:593-741.
 * vp, rho: padded, edge-replicated model (as read_model_a leaves it);
 * coef: the 18 CPML arrays of sm_a3d_cpml.  Outside the np-node frame the
 * coefficients must be a = 0, b = k = 1 (the reference's defaults). */
int sm_a3d_create(int device, size_t nx2, size_t ny2, size_t nz2, size_t np,
                  double dx, double dy, double dz, double dt,
                  const double *vp, const double *rho, const double *const *coef,
                  int precision, sm_a3d_t *out);
/* sm_a3d_create from the unpadded nx x ny x nz model: the padded nodes take
 * the value of the nearest interior node (io_utils.c:1096-1143) as the
 * materials are staged, so no padded copy is made on the host.  The handle
 * equals sm_a3d_create's on sm_a3d_pad_model's output bit for bit; coef is
 * for the padded grid (nx + 2 np, ...).  No reference counterpart. */
int sm_a3d_create_unpadded(int device, size_t nx, size_t ny, size_t nz, size_t np,
                           double dx, double dy, double dz, double dt,
                           const double *vp, const double *rho, const double *const *coef,
                           int precision, sm_a3d_t *out);
/* a_iso_3d.c:689-693: P[index[s]] += scale * fct[s*stride + it] while
 * it < length[s]; the reference uses scale = dt * 1e6 for every source type */
int sm_a3d_set_sources(sm_a3d_t h, size_t nsrc, const size_t *index, const double *fct,
                       const size_t *length, size_t stride, double scale);
/* a_iso_3d.c:698-741; comp SM_VX, SM_VY, SM_VZ (SM_P also works) */
int sm_a3d_set_receivers(sm_a3d_t h, size_t nrec, const size_t *index, const int *comp,
                         const double *t0, const double *rdt, size_t nsteps_max);
int sm_a3d_run(sm_a3d_t h, size_t nsteps);
/* Advance n handles of possibly different grid sizes and sources together
 * by nsteps steps each (the same loop, a_iso_3d.c:593-741, for several
 * models at once): each step is one launch over the tiles of all of them
 * (up to 16 handles per launch), one for all their sources and one for all
 * their receivers.  Every handle ends bit for bit where
 * sm_a3d_run(handles[k], nsteps) would leave it.  Same device and precision
 * for all; the work is queued on handles[0]'s stream after the work already
 * queued on every handle's stream, and every handle's stream waits for it.
 * Asynchronous like sm_a3d_run. */
int sm_a3d_group_run(sm_a3d_t const *handles, int n, size_t nsteps);
int sm_a3d_sync(sm_a3d_t h);
int sm_a3d_step_count(sm_a3d_t h, size_t *it);
int sm_a3d_read_traces(sm_a3d_t h, size_t rec0, size_t nrec, double *out, size_t ld,
                       size_t *counts);
/* whole padded field nx2*ny2*nz2 */
int sm_a3d_get_field(sm_a3d_t h, int comp, double *out);
int sm_a3d_set_field(sm_a3d_t h, int comp, const double *in);
int sm_a3d_reset(sm_a3d_t h);
int sm_a3d_destroy(sm_a3d_t h);
int sm_a3d_stream(sm_a3d_t h, void **stream);
/* launch configuration of the fused step kernel (tile rows, pipeline
 * depth): index in [0, nconfigs).  Results do not depend on it. */
int sm_a3d_set_config(sm_a3d_t h, int config);
/* x planes each CTA marches through (<= 0: the library's choice) */
int sm_a3d_set_chunk(sm_a3d_t h, int chunk);
int sm_a3d_get_config(sm_a3d_t h, int *config, int *nconfigs);
/* autotuner (over configurations and x-chunk lengths; trial_steps <= 0: 32)
 * and CUDA-graph replay, as sm_eiso_autotune / sm_eiso_set_graph */
int sm_a3d_autotune(sm_a3d_t h, int trial_steps, int *config, int *chunk, double *ms_per_step);
int sm_a3d_set_graph(sm_a3d_t h, int steps);
int sm_a3d_set_timing(sm_a3d_t h, int on);
int sm_a3d_kernel_stats(sm_a3d_t h, int reset, double *update_ms, size_t *update_launches,
                        size_t *all_launches);

/* ======================================================================
 * e_cyl_iso on the device: 2.5-D elastic FDTD in cylindrical coordinates
 * (r, z) for azimuthal mode n, CPML at the outer radius and at both z ends
 * (e_cyl_iso.c, propagate.c:2706-4118, pml.c:1811-2185).  Padded arrays are
 * nx2*nz2 with nx2 = nx + np (no layer before the axis r = 0) and
 * nz2 = nz + 2*np, index i*nz2 + j.  With the .par "abs 0" the reference
 * uses np = 0 (io_utils.c:293).  FP32 or FP64 storage.
 * ====================================================================== */

typedef struct sm_ecyl *sm_ecyl_t;

/* model padding of read_model_e_cyl (io_utils.c:993-1026): interior nx*nz
 * (index i*nz + j) into nx2*nz2 */
int sm_ecyl_pad_model(size_t nx, size_t nz, size_t np, const double *vp, const double *vs,
                      const double *rho, double *vp_pad, double *vs_pad, double *rho_pad);
/* material averaging e_cyl_iso.c:363-441 on the padded model; mat: 8 arrays
 * lij l2mij mu mui muj bi bj bij (nx2*nz2 each); vpmax for the CFL test
 * dt <= (dx+dz)/2 / (sqrt(2) vpmax) (e_cyl_iso.c:484-488) */
int sm_ecyl_materials(size_t nx2, size_t nz2, const double *vp, const double *vs,
                      const double *rho, double *const *mat, double *vpmax);
/* CPML coefficients, pml.c:2107-2185 (compute_cpml_cyl): 15 arrays ik_r
 * ik_z ikh_z b_r c_r b_z c_z bh_z ch_z (np values) then ikH_r ikH_z bH_r cH_r
 * bH_z cH_z (np + 1 values); absorb = the .par "abs" flag; alpha_max =
 * pi f0, or 0 when the .par alpha_max is 0 (e_cyl_iso.c:532-535) */
int sm_ecyl_cpml(size_t np, double dx, double dz, double dt, double order, double vmax,
                 double Rc, double kappa_max, double alpha_max, int absorb, double *const *c);
/* Kurkjian source wavelet, src.c:202-228 (lij_at_src: lij at the source
 * node, r_src its radius); returns the sample count (fct may be NULL) */
size_t sm_ecyl_kurkjian(double A, double f, double dt, double lij_at_src, double r_src,
                        double dx, double dz, int n, size_t maxlen, double *fct);

/* Replaces the allocations of e_cyl_iso.c:341-360 and the state of its time
 * loop e_cyl_iso.c:605-790.  mat and coef as produced above. */
int sm_ecyl_create(int device, size_t nx, size_t nz, size_t np, int n, double dx, double dz,
                   double dt, const double *const *mat, const double *const *coef,
                   int precision, sm_ecyl_t *out);
/* Sources at padded index[s]: SM_SRC_FR / SM_SRC_FT / SM_SRC_FZ / SM_SRC_BULK
 * add dt*b*fct[s*stride + it] after the velocity update (add_force_src_cyl,
 * src.c:186-199; fct from sm_ricker); one SM_SRC_KURKJIAN adds
 * dt*fct[it] to trr and tzz after the stress update (add_kurkjian_src,
 * src.c:231-236; fct from sm_ecyl_kurkjian).  Other types add nothing, as in
 * the reference's cylindrical loop. */
int sm_ecyl_set_sources(sm_ecyl_t h, size_t nsrc, const size_t *index, const int *type,
                        const double *fct, const size_t *length, size_t stride);
/* Records at padded index[r] (e_cyl_iso.c:668-790): components SM_VR SM_VT
 * SM_VZ SM_TRR SM_TTT SM_TZZ SM_TRZ SM_TRT SM_TTZ, or SM_DIV / SM_CURL
 * (compute_div_cyl / compute_curl_cyl, propagate.c:4090-4118, evaluated at
 * the record's node), sampled by sm_sample_predicate for it < nsteps_max */
int sm_ecyl_set_receivers(sm_ecyl_t h, size_t nrec, const size_t *index, const int *comp,
                          const double *t0, const double *rdt, size_t nsteps_max);
/* nsteps steps of the loop e_cyl_iso.c:605-790 (mode 0 or n > 0 forms) */
int sm_ecyl_run(sm_ecyl_t h, size_t nsteps);
int sm_ecyl_sync(sm_ecyl_t h);
int sm_ecyl_reset(sm_ecyl_t h);
/* samples so far of records [rec0, rec0+nrec) into out[r*ld + s] (raw
 * values; the reference writes 1e3 * value); counts[r] gets their number */
int sm_ecyl_read_traces(sm_ecyl_t h, size_t rec0, size_t nrec, double *out, size_t ld,
                        size_t *counts);
/* a whole padded field (nx2*nz2) of component SM_VR ... SM_TTZ */
int sm_ecyl_get_field(sm_ecyl_t h, int comp, double *out);
int sm_ecyl_set_field(sm_ecyl_t h, int comp, const double *in);
int sm_ecyl_stream(sm_ecyl_t h, void **stream);
int sm_ecyl_set_timing(sm_ecyl_t h, int on);
/* update_ms: device time of the velocity + source + stress launches */
int sm_ecyl_kernel_stats(sm_ecyl_t h, int reset, double *update_ms, size_t *update_launches,
                         size_t *all_launches);
int sm_ecyl_destroy(sm_ecyl_t h);
/* device memory of a handle, bytes */
size_t sm_ecyl_device_bytes(size_t nx, size_t nz, size_t np, int precision);

/* ======================================================================
 * device memory a handle needs (estimate used for admission; no reference
 * counterpart).  nrec receivers per shot, nsteps_max samples at most.
 * ====================================================================== */
int sm_eiso_device_bytes(size_t nx, size_t nz, size_t npml, int precision, size_t nshots,
                         size_t nrec, size_t nsteps_max, size_t *bytes);
int sm_a3d_device_bytes(size_t nx2, size_t ny2, size_t nz2, size_t np, int precision,
                        size_t nrec, size_t nsteps_max, size_t *bytes);

/* ======================================================================
 * Serving: a request loop over many shots of different grids (no reference
 * counterpart; the reference runs one program per shot).
 *
 * A request carries everything sm_eiso_create / sm_a3d_create and the
 * source and receiver set-up take, plus its step count; submit copies it, so
 * the caller's arrays may be freed on return.  A worker thread admits queued
 * requests in arrival order while the sum of admitted requests' device
 * memory (sm_*_device_bytes) stays within the budget and fewer than
 * max_active run; each admitted request gets its own handle and CUDA stream,
 * and the worker feeds every running request slices of slice_steps steps
 * (at most two slices queued per request), so requests that arrive while
 * others run start as soon as memory and a slot free up, and their kernels
 * overlap on the device.  A finished request's traces are copied to the host
 * and its device memory released.  Results do not depend on what else runs:
 * each request's arithmetic is that of a handle of its own.
 * ====================================================================== */
typedef struct {
    size_t nx, nz, npml;
    double h, dt;
    const double *la, *mu, *l2m, *b, *bm;   /* nx*nz, as sm_eiso_create */
    const double *d, *dh, *dH;              /* npml */
    int precision;
    size_t nsrc;                            /* as sm_eiso_set_sources */
    const size_t *src_index;
    const int *src_type;
    const double *src_fct;
    const size_t *src_length;
    size_t src_stride;
    double src_scale;
    size_t nrec;                            /* as sm_eiso_set_receivers */
    const size_t *rec_index;
    const int *rec_comp;
    const double *rec_t0, *rec_dt;
    size_t nsteps;
} sm_eiso_request;

typedef struct {
    size_t nx2, ny2, nz2, np;
    double dx, dy, dz, dt;
    const double *vp, *rho;                 /* padded, as sm_a3d_create */
    const double *const *coef;              /* 18 arrays, as sm_a3d_cpml */
    int precision;
    size_t nsrc;                            /* as sm_a3d_set_sources */
    const size_t *src_index;
    const double *src_fct;
    const size_t *src_length;
    size_t src_stride;
    double src_scale;
    size_t nrec;                            /* as sm_a3d_set_receivers */
    const size_t *rec_index;
    const int *rec_comp;
    const double *rec_t0, *rec_dt;
    size_t nsteps;
} sm_a3d_request;

/* request states */
#define SM_REQ_QUEUED  0
#define SM_REQ_RUNNING 1
#define SM_REQ_DONE    2
#define SM_REQ_FAILED  3

typedef struct {
    size_t submitted, completed, failed, running, queued;
    double latency_p50, latency_p99, latency_mean, latency_max;   /* s, submit -> traces on host */
    double wait_p50, wait_p99;            /* s, submit -> admitted */
    double busy_s;                        /* first submit -> last completion */
    double shots_per_s;                   /* completed / busy_s */
    double gcell_per_s;                   /* completed cell updates / busy_s / 1e9 */
    size_t hbm_budget, hbm_peak;          /* bytes admitted at most at one time */
    size_t max_running;                   /* most requests running at one time */
} sm_server_stats;

typedef struct sm_server *sm_server_t;

/* hbm_budget: bytes requests may hold (0: free device memory at creation
 * minus 2 GiB); max_active: running requests at most (0: 64); slice_steps:
 * steps per slice (0: 64); graph_steps: CUDA-graph length for each request
 * (0 none; else as sm_eiso_set_graph). */
int sm_server_create(int device, size_t hbm_budget, int max_active, int slice_steps,
                     int graph_steps, sm_server_t *out);
/* on != 0: running requests of one program and precision take their
 * slices together, one sm_eiso_group_run or sm_a3d_group_run call (one
 * launch per step over all of their grids) instead of one run each; results
 * are the same bits.  Call before the first submission. */
int sm_server_set_group(sm_server_t s, int on);
/* SM_EBUSY when the request alone exceeds the budget */
int sm_server_submit_eiso(sm_server_t s, const sm_eiso_request *r, uint64_t *ticket);
int sm_server_submit_a3d(sm_server_t s, const sm_a3d_request *r, uint64_t *ticket);
/* block until the request is done (SM_OK), failed (its error), or timeout_s
 * passed (SM_ETIMEOUT; < 0 waits for good) */
int sm_server_wait(sm_server_t s, uint64_t ticket, double timeout_s);
/* wait for every submitted request */
int sm_server_drain(sm_server_t s, double timeout_s);
int sm_server_status(sm_server_t s, uint64_t ticket, int *state, double *latency_s);
/* traces of a finished request, layout as sm_eiso_read_traces */
int sm_server_traces(sm_server_t s, uint64_t ticket, size_t rec0, size_t nrec, double *out,
                     size_t ld, size_t *counts);
/* forget a finished request (its traces) */
int sm_server_release(sm_server_t s, uint64_t ticket);
int sm_server_get_stats(sm_server_t s, sm_server_stats *st);
/* stops the worker after the running requests' queued slices; queued
 * requests are dropped */
int sm_server_destroy(sm_server_t s);
/* sizeof the request and stats structs, for bindings that lay them out */
int sm_server_struct_sizes(size_t *eiso_request, size_t *a3d_request, size_t *stats);

/* One e_iso shot that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc: programs whose device
 * memory is all handed out by their own allocator, or code running where a
 * device allocation is not allowed or would stall the device.  The whole run
 * (state, materials, tables, traces) lives in one fixed array of 24 MiB
 * inside this library, which every GPU that loads the library holds until
 * the process exits; a shot that needs more is rejected with SM_EINVAL and a
 * message giving the bytes it needs (a 400 x 400 grid with 20 PML cells, 64
 * receivers and 1500 steps fits).  FP32 storage only; results equal
 * sm_eiso_create / sm_eiso_run / sm_eiso_read_traces on the same request.
 *   r:       the shot, as for sm_server_submit_eiso (nshots = 1)
 *   stream:  cudaStream_t to run on (NULL: the legacy default stream); the
 *            call synchronizes this stream (after the uploads and again at
 *            the end) and returns when the run is done and the traces are
 *            copied
 *   traces:  nrec rows of ld doubles (may be NULL to learn the counts),
 *            counts: samples per receiver (required when nrec > 0)
 * The first call on a device looks up the array's device address (once per
 * device); make that first call before any stream capture.  Every call uses
 * the same array and clears what must start at zero, so calls on one device
 * that overlap on the GPU (other threads, other streams) race: run them one
 * at a time per device. */
int sm_eiso_run_noalloc(int device, void *stream, const sm_eiso_request *r, double *traces,
                        size_t ld, size_t *counts);

/* ======================================================================
 * drop-in programs: the whole of e_iso / a_iso_3d main() on the device,
 * reading the reference's .par / model / source / output files and writing
 * its trc/<base>/<base>_<n>.trc files.  argv as the reference takes it
 * (io_utils.c:156-202: -p file.par, -v, -h); an added "-P fp32|fp64|bfp16|fp16|bf16"
 * picks the storage precision (default fp32).  Returns 0 on success.
 * ====================================================================== */
int sm_e_iso_main(int argc, char **argv);
int sm_a_iso_3d_main(int argc, char **argv);
int sm_e_cyl_iso_main(int argc, char **argv);

#ifdef __cplusplus
}
#endif
#endif /* SEISMOD_GPU_H */
