// sm_ecyl.cu -- e_cyl_iso (2.5-D elastic FDTD in cylindrical coordinates r, z
// with azimuthal mode n, CPML) on sm_100a.
//
// Grid.  The reference's padded grid: nx2 = nx + np radial columns (the
// absorbing layer only beyond r = (nx-1) dr; r = 0 is the axis) by
// nz2 = nz + 2 np rows; here each column is padded to `pitch` cells so rows
// start aligned.  Nine fields (vr vt vz trr ttt tzz trz trt ttz) are updated
// in place: one launch updates the three velocities from the stresses
// (e_cyl_iso.c:612-633), force sources follow (src.c:186-199), one launch
// updates the six stresses from the velocities (e_cyl_iso.c:640-662), then a
// Kurkjian source (src.c:231-236) and the receivers.  One thread owns one
// cell (i, j) and every component stored there; z is the fast index, so a
// warp reads and writes consecutive cells.
//
// Arithmetic.  Each update keeps the reference's expression and order of
// operations (propagate.c:2706-3309 for mode 0, :3312-4088 for n > 0); this
// file is compiled without FMA contraction, so the FP64 build follows the
// FP64 reference to the last bit where the reference is built the same way.
// The FP32 build multiplies by reciprocals of the grid lengths instead of
// dividing (ECylQ).
// Materials arrive multiplied by dt on the host in FP64 (the reference's
// dt*b*(...) evaluates dt*b first).
//
// CPML memory variables.  z-side variables live in nx2 x (2 np + 1) strips
// (slot j below the interior, np + j - (nz + np - 1) above it), r-side ones
// in (np + 1) x nz2 strips (slot i - (nx - 1) for half-node updates, i - nx
// for node updates): every cell owns its own variable.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "sm_common.cuh"

namespace sm {

enum { C_VR, C_VT, C_VZ, C_TRR, C_TTT, C_TZZ, C_TRZ, C_TRT, C_TTZ };
enum { CM_L, CM_L2M, CM_MU, CM_MUI, CM_MUJ, CM_BI, CM_BJ, CM_BIJ };
// coefficient arrays (np each, then np + 1 each)
enum { K_IKR, K_IKZ, K_IKHZ, K_BR, K_CR, K_BZ, K_CZ, K_BHZ, K_CHZ,
       K_IKHR_E, K_IKHZ_E, K_BHR_E, K_CHR_E, K_BHZ_E, K_CHZ_E };
enum { ZV_TRZ, ZV_TTZ, ZV_TZZ, ZV_VZ, ZV_VR, ZV_VT, NZV };
enum { RV_DTRR, RV_TRR1, RV_TRT1, RV_TTT1, RV_TRT2, RV_DTRT, RV_TTT2, RV_DTRZ, RV_TRZ, RV_TTZ,
       RV_DVR, RV_VR1, RV_VT1, RV_DVZ, RV_DVT, RV_VR2, RV_VT2, RV_VZ, NRV };

template <typename C>
struct ECylArgs {
    int nx, nz, np, nx2, nz2, pitch, n;
    C dx, dz, idx, idz;   // and 1/dx, 1/dz (FP32 path)
    const C *inv;         // FP32 path: per column 1/(2 i dx), 1/(i dx), 1/((i+1/2) dx), 1/(2 (i+1/2) dx)
    C *f[9];
    const C *m[8];    // dt * (lij l2mij mu mui muj bi bj bij)
    const C *k;       // the 15 coefficient arrays, back to back
    C *zm;            // NZV strips of nx2 * (2 np + 1)
    C *rm;            // NRV strips of (np + 1) * nz2
};

template <typename C>
struct ECylDev {
    const ECylArgs<C> &a;
    int i, j;
    __device__ C F(int k, int ii, int jj) const { return a.f[k][(long long)ii * a.pitch + jj]; }
    // a field this launch only reads, through the read-only cache path
    __device__ C G(int k, int ii, int jj) const { return __ldg(a.f[k] + (long long)ii * a.pitch + jj); }
    __device__ C M(int k) const { return __ldg(a.m[k] + (long long)i * a.pitch + j); }
    __device__ C K(int arr, int idx) const {
        const int np = a.np;
        const int off = arr < 9 ? arr * np : 9 * np + (arr - 9) * (np + 1);
        return a.k[off + idx];
    }
    // one row below, as the reference's flat index reads it: with no PML the
    // row -1 of column i is row nz2-1 of column i-1, and before the array
    // (i = 0) it is taken as zero
    __device__ C below(int k) const {
        if (j > 0) return G(k, i, j - 1);
        return i > 0 ? G(k, i - 1, a.nz2 - 1) : C(0);
    }
    __device__ C cpml(C *psi, C b, C c, C ik, C d) const {
        const C p = b * *psi + c * d;
        *psi = p;
        return ik * d + p;
    }
    __device__ C *zvar(int v) const {
        const int np = a.np;
        const int s = j < np ? j : np + (j - (a.nz + np - 1));
        return a.zm + ((long long)v * a.nx2 + i) * (2 * np + 1) + s;
    }
    __device__ C *rvar(int v, int slot) const {
        return a.rm + ((long long)v * (a.np + 1) + slot) * a.nz2 + j;
    }
    __device__ bool zhalf() const { return j < a.np || j >= a.nz + a.np - 1; }
    __device__ bool znode() const { return j < a.np || j >= a.nz + a.np; }
    // z filters: h/H coefficients (vr, vt, taa), node coefficients mirrored
    // above (vz, ttz), h/H with rows from 1 (trz)
    __device__ C zf_half(int v, C d) const {
        const int top = a.nz + a.np - 1;
        if (j < a.np) return cpml(zvar(v), K(K_BHZ, j), K(K_CHZ, j), K(K_IKHZ, j), d);
        const int jj = j - top;
        return cpml(zvar(v), K(K_BHZ_E, jj), K(K_CHZ_E, jj), K(K_IKHZ_E, jj), d);
    }
    __device__ C zf_node(int v, C d) const {
        const int top = a.nz + a.np;
        if (j < a.np) return cpml(zvar(v), K(K_BZ, j), K(K_CZ, j), K(K_IKZ, j), d);
        const int q = a.np - 1 - (j - top);
        return cpml(zvar(v), K(K_BZ, q), K(K_CZ, q), K(K_IKZ, q), d);
    }
    __device__ C zf_trz(C d) const {
        const int top = a.nz + a.np;
        if (j < a.np) return cpml(zvar(ZV_VR), K(K_BHZ, j), K(K_CHZ, j), K(K_IKHZ, j), d);
        const int jj = j - top;
        return cpml(zvar(ZV_VR), K(K_BHZ_E, jj), K(K_CHZ_E, jj), K(K_IKHZ_E, jj), d);
    }
    // r filters beyond the interior: node (i >= nx, mirrored node
    // coefficients) and half node (i >= nx-1, the H coefficients)
    __device__ C rf_node(int v, C d) const {
        const int ii = i - a.nx, q = a.np - 1 - ii;
        return cpml(rvar(v, ii), K(K_BR, q), K(K_CR, q), K(K_IKR, q), d);
    }
    __device__ C rf_half(int v, C d) const {
        const int ii = i - (a.nx - 1);
        return cpml(rvar(v, ii), K(K_BHR_E, ii), K(K_CHR_E, ii), K(K_IKHR_E, ii), d);
    }
};

// Quotients by the grid's lengths: dx, dz, 2 i dx, i dx, (i + 1/2) dx and
// 2 (i + 1/2) dx.  FP64 divides, as the reference does; FP32 multiplies by
// reciprocals formed in FP64 on the host (per column), which keeps the FP32
// path far from its own error bound and avoids the division routine.
template <typename C>
struct ECylQ {
    static constexpr bool exact = sizeof(C) == 8;
    C dx, dz, idx, idz;
    C r2i, ri, r5, r25;       // denominators of column i (exact path)
    C i2i, ii, i5, i25;       // their reciprocals (FP32 path)
    __device__ ECylQ(const ECylArgs<C> &a, int i) : dx(a.dx), dz(a.dz), idx(a.idx), idz(a.idz) {
        r2i = C(2.) * C(i) * dx;
        ri = C(i) * dx;
        r5 = (C(i) + C(0.5)) * dx;
        r25 = C(2.) * (C(i) + C(0.5)) * dx;
        if (!exact) {
            const long long s = a.nx2;
            i2i = a.inv[i];
            ii = a.inv[s + i];
            i5 = a.inv[2 * s + i];
            i25 = a.inv[3 * s + i];
        }
    }
    __device__ C x(C v) const { return exact ? v / dx : v * idx; }
    __device__ C z(C v) const { return exact ? v / dz : v * idz; }
    __device__ C twoi(C v) const { return exact ? v / r2i : v * i2i; }
    __device__ C i1(C v) const { return exact ? v / ri : v * ii; }
    __device__ C half(C v) const { return exact ? v / r5 : v * i5; }
    __device__ C twohalf(C v) const { return exact ? v / r25 : v * i25; }
};

// vr, vt, vz of cell (i, j): update_vr/vt/vz_cyl (mode 0) or *_cyl_n (n > 0)
template <typename C, bool NPOS>
__global__ void __launch_bounds__(256) ecyl_velocity_kernel(const ECylArgs<C> a) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= a.nz2) return;
    const ECylDev<C> d{a, i, j};
    const ECylQ<C> Q(a, i);
    const int n = a.n;
    const long long q = (long long)i * a.pitch + j;
    // vr: rows [0, nz2-1), columns from 1 (from 0 for odd n: the axis)
    if (j + 1 < a.nz2 && (i >= 1 || (NPOS && (n % 2)))) {
        C ddz = Q.z(d.G(C_TRZ, i, j + 1) - d.G(C_TRZ, i, j));
        if (d.zhalf()) ddz = d.zf_half(ZV_TRZ, ddz);
        C s;
        if (i == 0) {
            s = Q.x(d.G(C_TRR, i, j) - -d.G(C_TRR, i, j)) + ddz;
        } else if (i < a.nx) {
            const C A = Q.x(d.G(C_TRR, i, j) - d.G(C_TRR, i - 1, j));
            const C B = Q.twoi(d.G(C_TRR, i, j) + d.G(C_TRR, i - 1, j));
            const C D = Q.twoi(d.G(C_TTT, i, j) + d.G(C_TTT, i - 1, j));
            if (NPOS)
                s = A + B + Q.i1(C(n) * d.G(C_TRT, i, j)) - D + ddz;
            else
                s = A + B - D + ddz;
        } else {
            const C A = d.rf_node(RV_DTRR, Q.x(d.G(C_TRR, i, j) - d.G(C_TRR, i - 1, j)));
            const C B = d.rf_node(RV_TRR1, Q.twoi(d.G(C_TRR, i, j) + d.G(C_TRR, i - 1, j)));
            const C D = d.rf_node(RV_TTT1, Q.twoi(d.G(C_TTT, i, j) + d.G(C_TTT, i - 1, j)));
            if (NPOS) {
                const C E = d.rf_node(RV_TRT1, Q.i1(d.G(C_TRT, i, j)));
                s = A + B + C(n) * E - D + ddz;
            } else {
                s = A + B - D + ddz;
            }
        }
        a.f[C_VR][q] += d.M(CM_BJ) * s;
    }
    if (i + 1 < a.nx2) {
        // vt: rows [0, nz2-1)
        if (j + 1 < a.nz2) {
            C ddz = Q.z(d.G(C_TTZ, i, j + 1) - d.G(C_TTZ, i, j));
            if (d.zhalf()) ddz = d.zf_half(ZV_TTZ, ddz);
            const C A = Q.half(d.G(C_TRT, i + 1, j) + d.G(C_TRT, i, j));
            const C B = Q.x(d.G(C_TRT, i + 1, j) - d.G(C_TRT, i, j));
            C s;
            if (i + 1 < a.nx) {
                if (NPOS)
                    s = A + B - Q.half(C(n) * d.G(C_TTT, i, j)) + ddz;
                else
                    s = A + B + ddz;
            } else {
                const C fa = d.rf_half(RV_TRT2, A), fb = d.rf_half(RV_DTRT, B);
                if (NPOS) {
                    const C E = d.rf_half(RV_TTT2, Q.half(d.G(C_TTT, i, j)));
                    s = fa + fb - C(n) * E + ddz;
                } else {
                    s = fa + fb + ddz;
                }
            }
            a.f[C_VT][q] += d.M(CM_BIJ) * s;
        }
        // vz: rows from 1 (from 0 without a PML)
        if (j >= 1 || a.np == 0) {
            C ddz = Q.z(d.G(C_TZZ, i, j) - d.below(C_TZZ));
            if (d.znode()) ddz = d.zf_node(ZV_TZZ, ddz);
            const C A = Q.x(d.G(C_TRZ, i + 1, j) - d.G(C_TRZ, i, j));
            const C B = Q.twohalf(d.G(C_TRZ, i + 1, j) + d.G(C_TRZ, i, j));
            C s;
            if (i + 1 < a.nx) {
                if (NPOS)
                    s = ddz + A + B + Q.half(C(n) * d.G(C_TTZ, i, j));
                else
                    s = ddz + A + B;
            } else {
                const C fa = d.rf_half(RV_DTRZ, A), fb = d.rf_half(RV_TRZ, B);
                if (NPOS) {
                    const C E = d.rf_half(RV_TTZ, Q.half(d.G(C_TTZ, i, j)));
                    s = ddz + fa + fb + C(n) * E;
                } else {
                    s = ddz + fa + fb;
                }
            }
            a.f[C_VZ][q] += d.M(CM_BI) * s;
        }
    }
}

// trr ttt tzz, trz, trt, ttz of cell (i, j)
template <typename C, bool NPOS>
__global__ void __launch_bounds__(256) ecyl_stress_kernel(const ECylArgs<C> a) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= a.nz2) return;
    const ECylDev<C> d{a, i, j};
    const ECylQ<C> Q(a, i);
    const int n = a.n;
    const long long q = (long long)i * a.pitch + j;
    // trr, ttt, tzz: columns [0, nx2-1), rows [0, nz2-1)
    if (i + 1 < a.nx2 && j + 1 < a.nz2) {
        C dvrdr = Q.x(d.G(C_VR, i + 1, j) - d.G(C_VR, i, j));
        C vrr = Q.twohalf(d.G(C_VR, i + 1, j) + d.G(C_VR, i, j));
        C vtr = NPOS ? Q.half(d.G(C_VT, i, j)) : C(0);
        C dvzdz = Q.z(d.G(C_VZ, i, j + 1) - d.G(C_VZ, i, j));
        if (i + 1 >= a.nx) {
            dvrdr = d.rf_half(RV_DVR, dvrdr);
            vrr = d.rf_half(RV_VR1, vrr);
            if (NPOS) vtr = d.rf_half(RV_VT1, vtr);
        }
        if (d.zhalf()) dvzdz = d.zf_half(ZV_VZ, dvzdz);
        const C l2m = d.M(CM_L2M), l = d.M(CM_L);
        if (NPOS) {
            a.f[C_TRR][q] += l2m * dvrdr + l * (vrr + C(n) * vtr + dvzdz);
            a.f[C_TTT][q] += l2m * (vrr + C(n) * vtr) + l * (dvrdr + dvzdz);
            a.f[C_TZZ][q] += l2m * dvzdz + l * (dvrdr + vrr + C(n) * vtr);
        } else {
            a.f[C_TRR][q] += l2m * dvrdr + l * (vrr + dvzdz);
            a.f[C_TTT][q] += l2m * vrr + l * (dvrdr + dvzdz);
            a.f[C_TZZ][q] += l2m * dvzdz + l * (dvrdr + vrr);
        }
    }
    // trz (update_trz_cyl for every n): columns from 1, rows from 1
    if (i >= 1 && (j >= 1 || a.np == 0)) {
        C ddz = Q.z(d.G(C_VR, i, j) - d.below(C_VR));
        if (d.znode()) ddz = d.zf_trz(ddz);
        C ddr = Q.x(d.G(C_VZ, i, j) - d.G(C_VZ, i - 1, j));
        if (i >= a.nx) {
            const int ii = i - a.nx;
            ddr = d.cpml(d.rvar(RV_DVZ, ii), d.K(K_BHR_E, ii), d.K(K_CHR_E, ii),
                         d.K(K_IKHR_E, ii), ddr);
        }
        a.f[C_TRZ][q] += d.M(CM_MU) * (ddz + ddr);
    }
    // trt: columns from 1 (from 0 for odd n), every row
    if (i >= 1 || (NPOS && (n % 2))) {
        C s;
        if (i == 0) {
            s = Q.x(d.G(C_VT, i, j) - -d.G(C_VT, i, j));
        } else if (i < a.nx) {
            const C A = Q.x(d.G(C_VT, i, j) - d.G(C_VT, i - 1, j));
            const C D = Q.twoi(d.G(C_VT, i, j) + d.G(C_VT, i - 1, j));
            if (NPOS)
                s = A - Q.i1(C(n) * d.G(C_VR, i, j)) - D;
            else
                s = A - D;
        } else {
            const C A = d.rf_node(RV_DVT, Q.x(d.G(C_VT, i, j) - d.G(C_VT, i - 1, j)));
            const C D = d.rf_node(RV_VT2, Q.twoi(d.G(C_VT, i, j) + d.G(C_VT, i - 1, j)));
            if (NPOS) {
                const C B = d.rf_node(RV_VR2, Q.i1(d.G(C_VR, i, j)));
                s = A - C(n) * B - D;
            } else {
                s = A - D;
            }
        }
        a.f[C_TRT][q] += d.M(CM_MUJ) * s;
    }
    // ttz: columns [0, nx2-1), rows from 1 (from 0 without a PML)
    if (i + 1 < a.nx2 && (j >= 1 || a.np == 0)) {
        const C diff = d.G(C_VT, i, j) - d.below(C_VT);
        const C mui = d.M(CM_MUI);
        const bool zp = d.znode();
        if (!NPOS) {
            // interior rows: dt mui (vt_j - vt_j-1) / dz, the division last
            if (zp)
                a.f[C_TTZ][q] += mui * d.zf_node(ZV_VT, Q.z(diff));
            else
                a.f[C_TTZ][q] += Q.z(mui * diff);
        } else {
            const C ddz = zp ? d.zf_node(ZV_VT, Q.z(diff)) : Q.z(diff);
            C s;
            if (i + 1 < a.nx)
                s = ddz - Q.half(C(n) * d.G(C_VZ, i, j));
            else
                s = ddz - C(n) * d.rf_half(RV_VZ, Q.half(d.G(C_VZ, i, j)));
            a.f[C_TTZ][q] += mui * s;
        }
    }
}

struct ECylSrc {
    long long q;     // padded (pitched) cell
    int type;        // SM_SRC_FR / FT / FZ / BULK
    long long voff;  // first sample in vals
    int len;
};

// force sources after the velocity update (src.c:186-199): dt b * value,
// one thread walking them in the reference's order (two sources may share
// a cell)
template <typename C>
__global__ void ecyl_force_kernel(ECylArgs<C> a, const ECylSrc *src, int nsrc, const double *vals,
                                  long long it) {
    if (threadIdx.x) return;
    for (int k = 0; k < nsrc; ++k) {
        const ECylSrc s = src[k];
        if (it >= s.len) continue;
        const C v = static_cast<C>(vals[s.voff + it]);
        if (s.type == SM_SRC_FR || s.type == SM_SRC_BULK) a.f[C_VR][s.q] += a.m[CM_BJ][s.q] * v;
        if (s.type == SM_SRC_FT) a.f[C_VT][s.q] += a.m[CM_BIJ][s.q] * v;
        if (s.type == SM_SRC_FZ || s.type == SM_SRC_BULK) a.f[C_VZ][s.q] += a.m[CM_BI][s.q] * v;
    }
}

// Kurkjian source after the stress update (src.c:231-236): dt * value, as
// scaled on the host, into trr and tzz
template <typename C>
__global__ void ecyl_kurkjian_kernel(ECylArgs<C> a, long long q, const double *vals, int len,
                                     long long it) {
    if (threadIdx.x || it >= len) return;
    const C v = static_cast<C>(vals[it]);
    a.f[C_TRR][q] += v;
    a.f[C_TZZ][q] += v;
}

struct ECylRec {
    int i, j;
    int comp;        // SM_VR ... or SM_DIV / SM_CURL
    int group;
    long long out;
};

// a record's value; div and curl are formed in FP64 from the stored fields
// (their differences cancel, so FP32 arithmetic there would add error that
// the fields themselves do not carry)
template <typename C>
__device__ double ecyl_probe(const ECylArgs<C> &a, int comp, int i, int j) {
    auto F = [&](int k, int ii, int jj) -> double {
        return static_cast<double>(a.f[k][(long long)ii * a.pitch + jj]);
    };
    const double dx = static_cast<double>(a.dx), dz = static_cast<double>(a.dz);
    switch (comp) {
    case SM_VR: return F(C_VR, i, j);
    case SM_VT: return F(C_VT, i, j);
    case SM_VZ: return F(C_VZ, i, j);
    case SM_TRR: return F(C_TRR, i, j);
    case SM_TTT: return F(C_TTT, i, j);
    case SM_TZZ: return F(C_TZZ, i, j);
    case SM_TRZ: return F(C_TRZ, i, j);
    case SM_TRT: return F(C_TRT, i, j);
    case SM_TTZ: return F(C_TTZ, i, j);
    case SM_DIV: {
        // propagate.c:4090-4100, its radial term not divided by dr
        if (i + 1 >= a.nx2 || j + 1 >= a.nz2) return 0.0;
        return ((i + 1) * F(C_VR, i + 1, j) - i * F(C_VR, i, j)) / (i + 0.5) +
               a.n * F(C_VT, i, j) / ((i + 0.5) * dx) + (F(C_VZ, i, j + 1) - F(C_VZ, i, j)) / dz;
    }
    default: {   // curl, propagate.c:4102-4118
        if (j == 0) return 0.0;
        if (i == 0) {
            if (!(a.n % 2)) return 0.0;
            return (F(C_VR, i, j) - F(C_VR, i, j - 1)) / dz - (F(C_VZ, i, j) - -F(C_VZ, i, j)) / dx;
        }
        return (F(C_VR, i, j) - F(C_VR, i, j - 1)) / dz - (F(C_VZ, i, j) - F(C_VZ, i - 1, j)) / dx;
    }
    }
}

template <typename C>
__global__ void ecyl_gather_kernel(ECylArgs<C> a, const ECylRec *rec, int nrec,
                                   const int32_t *table, long long nsteps_max, double *traces,
                                   long long it) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec || it >= nsteps_max) return;
    const ECylRec e = rec[r];
    const int32_t slot = table[(long long)e.group * nsteps_max + it];
    if (slot < 0) return;
    traces[e.out + slot] = ecyl_probe<C>(a, e.comp, e.i, e.j);
}

}  // namespace sm

using namespace sm;

struct sm_ecyl {
    int device = 0;
    int precision = SM_FP32;
    int nx = 0, nz = 0, np = 0, nx2 = 0, nz2 = 0, pitch = 0, n = 0;
    double dx = 0, dz = 0, dt = 0;
    size_t it = 0;
    size_t elem = 4;
    cudaStream_t stream = nullptr;
    DevBuf fields, mats, coef, zm, rm, inv;
    size_t fstride = 0;   // elements between fields
    // sources
    std::vector<ECylSrc> src;
    std::vector<double> vals;
    long long kurk_q = -1;
    int kurk_len = 0;
    DevBuf d_src, d_vals, d_kurk;
    // receivers
    std::vector<ECylRec> rec;
    SamplePlan plan;
    DevBuf d_rec, d_table, d_traces;
    KernelTimer timer;
};

namespace {

int ecyl_check(sm_ecyl_t h) {
    if (!h) return sm_fail(SM_EINVAL, "null e_cyl_iso handle");
    return SM_OK;
}

template <typename C>
ECylArgs<C> ecyl_args(sm_ecyl *h) {
    ECylArgs<C> a{};
    a.nx = h->nx;
    a.nz = h->nz;
    a.np = h->np;
    a.nx2 = h->nx2;
    a.nz2 = h->nz2;
    a.pitch = h->pitch;
    a.n = h->n;
    a.dx = static_cast<C>(h->dx);
    a.dz = static_cast<C>(h->dz);
    a.idx = static_cast<C>(1.0 / h->dx);
    a.idz = static_cast<C>(1.0 / h->dz);
    a.inv = h->inv.as<C>();
    C *f = h->fields.as<C>();
    for (int k = 0; k < 9; ++k) a.f[k] = f + (size_t)k * h->fstride;
    const C *m = h->mats.as<C>();
    for (int k = 0; k < 8; ++k) a.m[k] = m + (size_t)k * h->fstride;
    a.k = h->coef.as<C>();
    a.zm = h->zm.as<C>();
    a.rm = h->rm.as<C>();
    return a;
}

int ecyl_comp_ok(int c) {
    return c == SM_VR || c == SM_VT || c == SM_VZ || c == SM_TRR || c == SM_TTT || c == SM_TZZ ||
           c == SM_TRZ || c == SM_TRT || c == SM_TTZ || c == SM_DIV || c == SM_CURL;
}

int ecyl_field_of(int comp) {
    switch (comp) {
    case SM_VR: return C_VR;
    case SM_VT: return C_VT;
    case SM_VZ: return C_VZ;
    case SM_TRR: return C_TRR;
    case SM_TTT: return C_TTT;
    case SM_TZZ: return C_TZZ;
    case SM_TRZ: return C_TRZ;
    case SM_TRT: return C_TRT;
    case SM_TTZ: return C_TTZ;
    default: return -1;
    }
}

template <typename C>
int ecyl_step(sm_ecyl *h) {
    const ECylArgs<C> a = ecyl_args<C>(h);
    const dim3 grd((h->nz2 + 127) / 128, h->nx2);
    cudaEvent_t t0 = h->timer.begin(h->stream);
    if (h->n > 0)
        ecyl_velocity_kernel<C, true><<<grd, 128, 0, h->stream>>>(a);
    else
        ecyl_velocity_kernel<C, false><<<grd, 128, 0, h->stream>>>(a);
    const long long it = (long long)h->it;
    const int ns = (int)h->src.size();
    if (ns)
        ecyl_force_kernel<C><<<1, 32, 0, h->stream>>>(
            a, h->d_src.as<ECylSrc>(), ns, h->d_vals.as<double>(), it);
    if (h->n > 0)
        ecyl_stress_kernel<C, true><<<grd, 128, 0, h->stream>>>(a);
    else
        ecyl_stress_kernel<C, false><<<grd, 128, 0, h->stream>>>(a);
    h->timer.end(t0, h->stream);
    h->timer.launches += 2 + (ns ? 1 : 0);
    if (h->kurk_q >= 0) {
        ecyl_kurkjian_kernel<C><<<1, 32, 0, h->stream>>>(a, h->kurk_q, h->d_kurk.as<double>(),
                                                          h->kurk_len, it);
        h->timer.launches += 1;
    }
    const int nr = (int)h->rec.size();
    if (nr) {
        ecyl_gather_kernel<C><<<(nr + 127) / 128, 128, 0, h->stream>>>(
            a, h->d_rec.as<ECylRec>(), nr, h->d_table.as<int32_t>(), (long long)h->plan.nsteps_max,
            h->d_traces.as<double>(), it);
        h->timer.launches += 1;
    }
    h->it++;
    return SM_OK;
}

template <typename C>
int upload_pitched(DevBuf &dst, size_t k, size_t stride, const double *src, int nx2, int nz2,
                   int pitch, cudaStream_t s) {
    std::vector<C> tmp((size_t)nx2 * pitch, C(0));
    for (int i = 0; i < nx2; ++i)
        for (int j = 0; j < nz2; ++j) tmp[(size_t)i * pitch + j] = static_cast<C>(src[(size_t)i * nz2 + j]);
    SM_CUDA_TRY(cudaMemcpyAsync(dst.as<C>() + k * stride, tmp.data(), tmp.size() * sizeof(C),
                                cudaMemcpyHostToDevice, s));
    SM_CUDA_TRY(cudaStreamSynchronize(s));
    return SM_OK;
}

}  // namespace

extern "C" size_t sm_ecyl_device_bytes(size_t nx, size_t nz, size_t np, int precision) {
    const size_t e = precision == SM_FP64 ? 8 : 4;
    const size_t nx2 = nx + np, nz2 = nz + 2 * np, pitch = round_up(nz2, 32);
    return e * (17 * nx2 * pitch + NZV * nx2 * (2 * np + 1) + NRV * (np + 1) * nz2 + 15 * (np + 1));
}

extern "C" int sm_ecyl_create(int device, size_t nx, size_t nz, size_t np, int n, double dx,
                              double dz, double dt, const double *const *mat,
                              const double *const *coef, int precision, sm_ecyl_t *out) {
    if (!out) return sm_fail(SM_EINVAL, "sm_ecyl_create: out is NULL");
    *out = nullptr;
    if (precision != SM_FP32 && precision != SM_FP64)
        return sm_fail(SM_EINVAL, "sm_ecyl_create: e_cyl_iso runs in FP32 or FP64 storage");
    if (nx < 2 || nz < 2 || n < 0 || !(dx > 0) || !(dz > 0) || !(dt > 0) || !mat || !coef)
        return sm_fail(SM_EINVAL, "sm_ecyl_create: bad argument");
    if (nx + np > 65535 || nz + 2 * np > (1u << 24))
        return sm_fail(SM_EINVAL, "sm_ecyl_create: grid too large (at most 65535 radial columns)");
    for (int k = 0; k < 8; ++k)
        if (!mat[k]) return sm_fail(SM_EINVAL, "sm_ecyl_create: material %d is NULL", k);
    for (int k = 0; k < 15; ++k)
        if (!coef[k]) return sm_fail(SM_EINVAL, "sm_ecyl_create: coefficient array %d is NULL", k);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return sm_fail(SM_EINVAL, "sm_ecyl_create: no CUDA device %d", device);
    DeviceGuard g(device);
    std::unique_ptr<sm_ecyl> h(new (std::nothrow) sm_ecyl());
    if (!h) return sm_fail(SM_ENOMEM, "sm_ecyl_create: out of host memory");
    h->device = device;
    h->precision = precision;
    h->nx = (int)nx;
    h->nz = (int)nz;
    h->np = (int)np;
    h->nx2 = (int)(nx + np);
    h->nz2 = (int)(nz + 2 * np);
    h->pitch = (int)round_up((size_t)h->nz2, 32);
    h->n = n;
    h->dx = dx;
    h->dz = dz;
    h->dt = dt;
    h->elem = precision == SM_FP64 ? 8 : 4;
    SM_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->fstride = (size_t)h->nx2 * h->pitch;
    int rc;
    if ((rc = h->fields.alloc(9 * h->fstride * h->elem))) return rc;
    if ((rc = h->mats.alloc(8 * h->fstride * h->elem))) return rc;
    if ((rc = h->coef.alloc((9 * np + 6 * (np + 1)) * h->elem + h->elem))) return rc;
    if ((rc = h->zm.alloc(NZV * (size_t)h->nx2 * (2 * np + 1) * h->elem))) return rc;
    if ((rc = h->rm.alloc(NRV * (np + 1) * (size_t)h->nz2 * h->elem))) return rc;
    if ((rc = h->fields.zero(h->stream)) || (rc = h->mats.zero(h->stream)) ||
        (rc = h->zm.zero(h->stream)) || (rc = h->rm.zero(h->stream)))
        return rc;
    // materials times dt, in FP64, then to the storage type
    std::vector<double> tmp((size_t)h->nx2 * h->nz2);
    for (int k = 0; k < 8; ++k) {
        for (size_t q = 0; q < tmp.size(); ++q) tmp[q] = dt * mat[k][q];
        rc = precision == SM_FP64
                 ? upload_pitched<double>(h->mats, k, h->fstride, tmp.data(), h->nx2, h->nz2, h->pitch, h->stream)
                 : upload_pitched<float>(h->mats, k, h->fstride, tmp.data(), h->nx2, h->nz2, h->pitch, h->stream);
        if (rc) return rc;
    }
    {   // per-column reciprocals of the radial lengths (FP32 path)
        const size_t nx2 = (size_t)h->nx2;
        std::vector<double> r(4 * nx2, 0.0);
        for (size_t i = 0; i < nx2; ++i) {
            r[i] = i ? 1.0 / (2. * i * dx) : 0.0;
            r[nx2 + i] = i ? 1.0 / (i * dx) : 0.0;
            r[2 * nx2 + i] = 1.0 / ((i + 0.5) * dx);
            r[3 * nx2 + i] = 1.0 / (2. * (i + 0.5) * dx);
        }
        if ((rc = h->inv.alloc(r.size() * h->elem))) return rc;
        rc = precision == SM_FP64 ? upload_convert<double>(h->inv.p, r.data(), r.size(), h->stream)
                                  : upload_convert<float>(h->inv.p, r.data(), r.size(), h->stream);
        if (rc) return rc;
    }
    std::vector<double> kt;
    for (int k = 0; k < 15; ++k) kt.insert(kt.end(), coef[k], coef[k] + (k < 9 ? np : np + 1));
    kt.push_back(0.0);
    rc = precision == SM_FP64 ? upload_convert<double>(h->coef.p, kt.data(), kt.size(), h->stream)
                              : upload_convert<float>(h->coef.p, kt.data(), kt.size(), h->stream);
    if (rc) return rc;
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    *out = h.release();
    return SM_OK;
}

extern "C" int sm_ecyl_destroy(sm_ecyl_t h) {
    if (!h) return SM_OK;
    {
        DeviceGuard g(h->device);
        if (h->stream) cudaStreamSynchronize(h->stream);
        h->fields.release();
        h->mats.release();
        h->coef.release();
        h->zm.release();
        h->rm.release();
        h->inv.release();
        h->d_src.release();
        h->d_vals.release();
        h->d_kurk.release();
        h->d_rec.release();
        h->d_table.release();
        h->d_traces.release();
        if (h->stream) cudaStreamDestroy(h->stream);
    }
    delete h;
    return SM_OK;
}

// Sources: force types (SM_SRC_FR, SM_SRC_FT, SM_SRC_FZ, SM_SRC_BULK) add
// dt b[index] fct[it] after the velocity update; one SM_SRC_KURKJIAN source
// adds dt fct[it] to trr and tzz after the stress update (the reference
// handles a Kurkjian first source alone, e_cyl_iso.c:497-502,664-666).
extern "C" int sm_ecyl_set_sources(sm_ecyl_t h, size_t nsrc, const size_t *index,
                                   const int *type, const double *fct, const size_t *length,
                                   size_t stride) {
    if (int rc = ecyl_check(h)) return rc;
    if (nsrc && (!index || !type || !fct || !length))
        return sm_fail(SM_EINVAL, "sm_ecyl_set_sources: NULL array");
    DeviceGuard g(h->device);
    h->src.clear();
    h->vals.clear();
    h->kurk_q = -1;
    h->kurk_len = 0;
    const size_t N = (size_t)h->nx2 * h->nz2;
    std::vector<double> kurk;
    for (size_t s = 0; s < nsrc; ++s) {
        if (index[s] >= N) return sm_fail(SM_EINVAL, "sm_ecyl_set_sources: source %zu outside the grid", s);
        if (length[s] > stride) return sm_fail(SM_EINVAL, "sm_ecyl_set_sources: length > stride");
        const long long q = (long long)(index[s] / h->nz2) * h->pitch + (long long)(index[s] % h->nz2);
        if (type[s] == SM_SRC_KURKJIAN) {
            if (h->kurk_q >= 0)
                return sm_fail(SM_EINVAL, "sm_ecyl_set_sources: one Kurkjian source at most");
            h->kurk_q = q;
            h->kurk_len = (int)length[s];
            for (size_t t = 0; t < length[s]; ++t) kurk.push_back(h->dt * fct[s * stride + t]);
            continue;
        }
        if (type[s] != SM_SRC_FR && type[s] != SM_SRC_FT && type[s] != SM_SRC_FZ &&
            type[s] != SM_SRC_BULK)
            continue;   // the reference's cylindrical loop adds nothing for other types
        h->src.push_back(ECylSrc{q, type[s], (long long)h->vals.size(), (int)length[s]});
        h->vals.insert(h->vals.end(), fct + s * stride, fct + s * stride + length[s]);
    }
    int rc;
    if (!h->src.empty()) {
        if ((rc = h->d_src.alloc(h->src.size() * sizeof(ECylSrc)))) return rc;
        if ((rc = h->d_vals.alloc(std::max<size_t>(h->vals.size(), 1) * sizeof(double)))) return rc;
        SM_CUDA_TRY(cudaMemcpyAsync(h->d_src.p, h->src.data(), h->src.size() * sizeof(ECylSrc),
                                    cudaMemcpyHostToDevice, h->stream));
        if (!h->vals.empty())
            SM_CUDA_TRY(cudaMemcpyAsync(h->d_vals.p, h->vals.data(), h->vals.size() * sizeof(double),
                                        cudaMemcpyHostToDevice, h->stream));
    }
    if (h->kurk_q >= 0) {
        if ((rc = h->d_kurk.alloc(std::max<size_t>(kurk.size(), 1) * sizeof(double)))) return rc;
        if (!kurk.empty())
            SM_CUDA_TRY(cudaMemcpyAsync(h->d_kurk.p, kurk.data(), kurk.size() * sizeof(double),
                                        cudaMemcpyHostToDevice, h->stream));
    }
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SM_OK;
}

extern "C" int sm_ecyl_set_receivers(sm_ecyl_t h, size_t nrec, const size_t *index,
                                     const int *comp, const double *t0, const double *rdt,
                                     size_t nsteps_max) {
    if (int rc = ecyl_check(h)) return rc;
    if (nrec && (!index || !comp || !t0 || !rdt))
        return sm_fail(SM_EINVAL, "sm_ecyl_set_receivers: NULL array");
    DeviceGuard g(h->device);
    const size_t N = (size_t)h->nx2 * h->nz2;
    h->rec.clear();
    if (int rc = h->plan.build(nrec, t0, rdt, h->dt, nsteps_max)) return rc;
    long long out = 0;
    for (size_t r = 0; r < nrec; ++r) {
        if (index[r] >= N) return sm_fail(SM_EINVAL, "sm_ecyl_set_receivers: record %zu outside the grid", r);
        if (!ecyl_comp_ok(comp[r]))
            return sm_fail(SM_EINVAL, "sm_ecyl_set_receivers: component %d of record %zu is not "
                                      "an e_cyl_iso component", comp[r], r);
        const int grp = h->plan.group_of[r];
        h->rec.push_back(ECylRec{(int)(index[r] / h->nz2), (int)(index[r] % h->nz2), comp[r], grp, out});
        out += (long long)h->plan.count_total[grp];
    }
    int rc;
    if ((rc = h->d_traces.alloc(std::max<long long>(out, 1) * sizeof(double)))) return rc;
    if ((rc = h->d_traces.zero(h->stream))) return rc;
    if (nrec) {
        if ((rc = h->d_rec.alloc(nrec * sizeof(ECylRec)))) return rc;
        if ((rc = h->d_table.alloc(std::max<size_t>(h->plan.table.size(), 1) * sizeof(int32_t)))) return rc;
        SM_CUDA_TRY(cudaMemcpyAsync(h->d_rec.p, h->rec.data(), nrec * sizeof(ECylRec),
                                    cudaMemcpyHostToDevice, h->stream));
        if (!h->plan.table.empty())
            SM_CUDA_TRY(cudaMemcpyAsync(h->d_table.p, h->plan.table.data(),
                                        h->plan.table.size() * sizeof(int32_t),
                                        cudaMemcpyHostToDevice, h->stream));
    }
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SM_OK;
}

extern "C" int sm_ecyl_run(sm_ecyl_t h, size_t nsteps) {
    if (int rc = ecyl_check(h)) return rc;
    DeviceGuard g(h->device);
    for (size_t s = 0; s < nsteps; ++s) {
        const int rc = h->precision == SM_FP64 ? ecyl_step<double>(h) : ecyl_step<float>(h);
        if (rc) return rc;
    }
    SM_CUDA_TRY(cudaGetLastError());
    return SM_OK;
}

extern "C" int sm_ecyl_sync(sm_ecyl_t h) {
    if (int rc = ecyl_check(h)) return rc;
    DeviceGuard g(h->device);
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SM_OK;
}

extern "C" int sm_ecyl_reset(sm_ecyl_t h) {
    if (int rc = ecyl_check(h)) return rc;
    DeviceGuard g(h->device);
    int rc;
    if ((rc = h->fields.zero(h->stream)) || (rc = h->zm.zero(h->stream)) ||
        (rc = h->rm.zero(h->stream)) || (rc = h->d_traces.zero(h->stream)))
        return rc;
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->it = 0;
    return SM_OK;
}

extern "C" int sm_ecyl_read_traces(sm_ecyl_t h, size_t rec0, size_t nrec, double *out,
                                   size_t ld, size_t *counts) {
    if (int rc = ecyl_check(h)) return rc;
    if (rec0 + nrec > h->rec.size())
        return sm_fail(SM_EINVAL, "sm_ecyl_read_traces: records [%zu, %zu) of %zu", rec0,
                       rec0 + nrec, h->rec.size());
    DeviceGuard g(h->device);
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (size_t r = 0; r < nrec; ++r) {
        const ECylRec &e = h->rec[rec0 + r];
        size_t c = 0;
        const size_t lim = std::min(h->it, h->plan.nsteps_max);
        for (size_t it = 0; it < lim; ++it)
            if (h->plan.table[(size_t)e.group * h->plan.nsteps_max + it] >= 0) ++c;
        if (counts) counts[r] = c;
        if (out && c) {
            if (ld < c) return sm_fail(SM_EINVAL, "sm_ecyl_read_traces: ld %zu < %zu samples", ld, c);
            SM_CUDA_TRY(cudaMemcpy(out + r * ld, h->d_traces.as<double>() + e.out, c * sizeof(double),
                                   cudaMemcpyDeviceToHost));
        }
    }
    return SM_OK;
}

extern "C" int sm_ecyl_get_field(sm_ecyl_t h, int comp, double *out) {
    if (int rc = ecyl_check(h)) return rc;
    const int f = ecyl_field_of(comp);
    if (f < 0 || !out) return sm_fail(SM_EINVAL, "sm_ecyl_get_field: component %d", comp);
    DeviceGuard g(h->device);
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    const size_t n = h->fstride;
    if (h->precision == SM_FP64) {
        std::vector<double> tmp(n);
        SM_CUDA_TRY(cudaMemcpy(tmp.data(), h->fields.as<double>() + f * n, n * sizeof(double),
                               cudaMemcpyDeviceToHost));
        for (int i = 0; i < h->nx2; ++i)
            for (int j = 0; j < h->nz2; ++j) out[(size_t)i * h->nz2 + j] = tmp[(size_t)i * h->pitch + j];
    } else {
        std::vector<float> tmp(n);
        SM_CUDA_TRY(cudaMemcpy(tmp.data(), h->fields.as<float>() + f * n, n * sizeof(float),
                               cudaMemcpyDeviceToHost));
        for (int i = 0; i < h->nx2; ++i)
            for (int j = 0; j < h->nz2; ++j) out[(size_t)i * h->nz2 + j] = tmp[(size_t)i * h->pitch + j];
    }
    return SM_OK;
}

extern "C" int sm_ecyl_set_field(sm_ecyl_t h, int comp, const double *in) {
    if (int rc = ecyl_check(h)) return rc;
    const int f = ecyl_field_of(comp);
    if (f < 0 || !in) return sm_fail(SM_EINVAL, "sm_ecyl_set_field: component %d", comp);
    DeviceGuard g(h->device);
    return h->precision == SM_FP64
               ? upload_pitched<double>(h->fields, f, h->fstride, in, h->nx2, h->nz2, h->pitch, h->stream)
               : upload_pitched<float>(h->fields, f, h->fstride, in, h->nx2, h->nz2, h->pitch, h->stream);
}

extern "C" int sm_ecyl_stream(sm_ecyl_t h, void **stream) {
    if (int rc = ecyl_check(h)) return rc;
    if (!stream) return sm_fail(SM_EINVAL, "sm_ecyl_stream: NULL");
    *stream = (void *)h->stream;
    return SM_OK;
}

extern "C" int sm_ecyl_set_timing(sm_ecyl_t h, int on) {
    if (int rc = ecyl_check(h)) return rc;
    DeviceGuard g(h->device);
    h->timer.set(on != 0);
    return SM_OK;
}

extern "C" int sm_ecyl_kernel_stats(sm_ecyl_t h, int reset, double *ms, size_t *timed,
                                    size_t *launches) {
    if (int rc = ecyl_check(h)) return rc;
    DeviceGuard g(h->device);
    return h->timer.stats(reset, ms, timed, launches);
}
