// sm_a3d.cu -- a_iso_3d (3D acoustic, CPML) on sm_100a.
//
// Grid.  The reference's padded layout (i*ny2 + j)*nz2 + k with the z rows
// padded to a pitch of 32 elements.  Fields P, vx, vy, vz cover the whole
// grid.  The CPML memory variables (a_iso_3d.c:327-332 allocates six full
// volumes) are non-zero only where their coefficient a != 0, i.e. in the
// np-node frame of their own axis; outside it the reference's update
// mem = 1*mem + 0*g keeps them exactly 0 and g/1 + 0 == g.  So each is
// stored only on its two slabs:
//   psi_Px / psi_vx  2*np x-planes of ny2 x pitch
//   psi_Py / psi_vy  nx2 x 2*np y-rows of pitch
//   psi_Pz / psi_vz  nx2 x ny2 x 2*np
// Velocity slabs cover half nodes [0, np) and [n2-1-np, n2-2]; pressure
// slabs cover nodes [0, np) and [n2-np, n2-1].
//
// Materials.  rho (for the staggered buoyancy dt*2/(rho_a + rho_b),
// a_iso_3d.c:379-405, formed on the fly) and K = rho vp^2 dt (:407-409).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "sm_common.cuh"

namespace sm {

enum { A_VX = 0, A_VY = 1, A_VZ = 2, A_P = 3 };
enum { PS_PX = 0, PS_PY = 1, PS_PZ = 2, PS_VX = 3, PS_VY = 4, PS_VZ = 5 };

// coefficient table (compute type): per axis a, b, 1/k for nodes (n2) and
// half nodes (n2, last unused)
struct A3Coef {
    int n2[3];
    __host__ __device__ int base(int axis) const {
        int o = 0;
        for (int a = 0; a < axis; ++a) o += 6 * n2[a];
        return o;
    }
    // which: 0 a, 1 b, 2 1/k (nodes); 3 a_h, 4 b_h, 5 1/k_h (half nodes)
    __host__ __device__ int at(int axis, int which) const { return base(axis) + which * n2[axis]; }
    __host__ __device__ int size() const { return 6 * (n2[0] + n2[1] + n2[2]); }
};

struct A3Args {
    int nx2, ny2, nz2, pitch, np;
    long long sx, sy;          // strides of i and j in elements
    void *f[4];
    void *psi[6];
    const void *rho;           // compute type, padded layout
    const void *K;
    const void *coef;
    A3Coef cf;
    double two_dt;             // 2 dt
    double idx, idy, idz;      // 1/dx, 1/dy, 1/dz
    float sc[4], isc[4];
    float psc[6], pisc[6];
};

// slab plane of node/half-node index n along an axis of n2 nodes, or -1
__device__ __forceinline__ int half_slab(int n, int n2, int np) {
    if (n < np) return n;
    if (n >= n2 - 1 - np && n <= n2 - 2) return np + (n - (n2 - 1 - np));
    return -1;
}
__device__ __forceinline__ int node_slab(int n, int n2, int np) {
    if (n < np) return n;
    if (n >= n2 - np) return np + (n - (n2 - np));
    return -1;
}

template <typename S>
__global__ void __launch_bounds__(256) a3d_velocity_kernel(A3Args a) {
    using C = typename Store<S>::C;
    using St = Store<S>;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= a.nz2 || j >= a.ny2) return;
    const long long q = (long long)i * a.sx + (long long)j * a.sy + k;
    const S *P = static_cast<const S *>(a.f[A_P]);
    const C *rho = static_cast<const C *>(a.rho);
    const C *cf = static_cast<const C *>(a.coef);
    const C p = St::ld(P + q, a.isc[A_P]);
    const C r = rho[q];
    const C two_dt = static_cast<C>(a.two_dt);
    const int np = a.np;
    // vx, a_iso_3d.c:605-617 (i < nx2-1)
    if (i < a.nx2 - 1) {
        C g = (St::ld(P + q + a.sx, a.isc[A_P]) - p) * static_cast<C>(a.idx);
        const int s = half_slab(i, a.nx2, np);
        if (s >= 0) {
            S *m = static_cast<S *>(a.psi[PS_PX]);
            const long long c = ((long long)s * a.ny2 + j) * a.pitch + k;
            const C mm = cf[a.cf.at(0, 4) + i] * St::ld(m + c, a.pisc[PS_PX]) +
                         cf[a.cf.at(0, 3) + i] * g;
            St::st(m + c, mm, a.psc[PS_PX]);
            g = g * cf[a.cf.at(0, 5) + i] + mm;
        }
        S *v = static_cast<S *>(a.f[A_VX]);
        const C ir = two_dt / (r + rho[q + a.sx]);
        St::st(v + q, St::ld(v + q, a.isc[A_VX]) - ir * g, a.sc[A_VX]);
    }
    // vy, :620-634 (j < ny2-1)
    if (j < a.ny2 - 1) {
        C g = (St::ld(P + q + a.sy, a.isc[A_P]) - p) * static_cast<C>(a.idy);
        const int s = half_slab(j, a.ny2, np);
        if (s >= 0) {
            S *m = static_cast<S *>(a.psi[PS_PY]);
            const long long c = ((long long)i * 2 * np + s) * a.pitch + k;
            const C mm = cf[a.cf.at(1, 4) + j] * St::ld(m + c, a.pisc[PS_PY]) +
                         cf[a.cf.at(1, 3) + j] * g;
            St::st(m + c, mm, a.psc[PS_PY]);
            g = g * cf[a.cf.at(1, 5) + j] + mm;
        }
        S *v = static_cast<S *>(a.f[A_VY]);
        const C ir = two_dt / (r + rho[q + a.sy]);
        St::st(v + q, St::ld(v + q, a.isc[A_VY]) - ir * g, a.sc[A_VY]);
    }
    // vz, :637-651 (k < nz2-1)
    if (k < a.nz2 - 1) {
        C g = (St::ld(P + q + 1, a.isc[A_P]) - p) * static_cast<C>(a.idz);
        const int s = half_slab(k, a.nz2, np);
        if (s >= 0) {
            S *m = static_cast<S *>(a.psi[PS_PZ]);
            const long long c = ((long long)i * a.ny2 + j) * 2 * np + s;
            const C mm = cf[a.cf.at(2, 4) + k] * St::ld(m + c, a.pisc[PS_PZ]) +
                         cf[a.cf.at(2, 3) + k] * g;
            St::st(m + c, mm, a.psc[PS_PZ]);
            g = g * cf[a.cf.at(2, 5) + k] + mm;
        }
        S *v = static_cast<S *>(a.f[A_VZ]);
        const C ir = two_dt / (r + rho[q + 1]);
        St::st(v + q, St::ld(v + q, a.isc[A_VZ]) - ir * g, a.sc[A_VZ]);
    }
}

template <typename S>
__global__ void __launch_bounds__(256) a3d_pressure_kernel(A3Args a) {
    using C = typename Store<S>::C;
    using St = Store<S>;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    // a_iso_3d.c:659-683: i, j, k >= 1
    if (k >= a.nz2 || j >= a.ny2 || i < 1 || j < 1 || k < 1) return;
    const long long q = (long long)i * a.sx + (long long)j * a.sy + k;
    const S *vx = static_cast<const S *>(a.f[A_VX]);
    const S *vy = static_cast<const S *>(a.f[A_VY]);
    const S *vz = static_cast<const S *>(a.f[A_VZ]);
    const C *cf = static_cast<const C *>(a.coef);
    const int np = a.np;
    C dx = (St::ld(vx + q, a.isc[A_VX]) - St::ld(vx + q - a.sx, a.isc[A_VX])) * static_cast<C>(a.idx);
    C dy = (St::ld(vy + q, a.isc[A_VY]) - St::ld(vy + q - a.sy, a.isc[A_VY])) * static_cast<C>(a.idy);
    C dz = (St::ld(vz + q, a.isc[A_VZ]) - St::ld(vz + q - 1, a.isc[A_VZ])) * static_cast<C>(a.idz);
    int s = node_slab(i, a.nx2, np);
    if (s >= 0) {
        S *m = static_cast<S *>(a.psi[PS_VX]);
        const long long c = ((long long)s * a.ny2 + j) * a.pitch + k;
        const C mm = cf[a.cf.at(0, 1) + i] * St::ld(m + c, a.pisc[PS_VX]) + cf[a.cf.at(0, 0) + i] * dx;
        St::st(m + c, mm, a.psc[PS_VX]);
        dx = dx * cf[a.cf.at(0, 2) + i] + mm;
    }
    s = node_slab(j, a.ny2, np);
    if (s >= 0) {
        S *m = static_cast<S *>(a.psi[PS_VY]);
        const long long c = ((long long)i * 2 * np + s) * a.pitch + k;
        const C mm = cf[a.cf.at(1, 1) + j] * St::ld(m + c, a.pisc[PS_VY]) + cf[a.cf.at(1, 0) + j] * dy;
        St::st(m + c, mm, a.psc[PS_VY]);
        dy = dy * cf[a.cf.at(1, 2) + j] + mm;
    }
    s = node_slab(k, a.nz2, np);
    if (s >= 0) {
        S *m = static_cast<S *>(a.psi[PS_VZ]);
        const long long c = ((long long)i * a.ny2 + j) * 2 * np + s;
        const C mm = cf[a.cf.at(2, 1) + k] * St::ld(m + c, a.pisc[PS_VZ]) + cf[a.cf.at(2, 0) + k] * dz;
        St::st(m + c, mm, a.psc[PS_VZ]);
        dz = dz * cf[a.cf.at(2, 2) + k] + mm;
    }
    S *P = static_cast<S *>(a.f[A_P]);
    const C K = static_cast<const C *>(a.K)[q];
    St::st(P + q, St::ld(P + q, a.isc[A_P]) - K * (dx + dy + dz), a.sc[A_P]);
}

struct A3Src {
    long long q;
    long long voff;
    int len;
};

template <typename S>
__global__ void a3d_source_kernel(A3Args a, const A3Src *src, int nsrc, const double *vals,
                                  long long it) {
    using St = Store<S>;
    using C = typename Store<S>::C;
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    // one thread, in source order, as a_iso_3d.c:689-693
    S *P = static_cast<S *>(a.f[A_P]);
    for (int e = 0; e < nsrc; ++e) {
        const A3Src s = src[e];
        if (it >= s.len) continue;
        St::st(P + s.q, St::ld(P + s.q, a.isc[A_P]) + static_cast<C>(vals[s.voff + it]), a.sc[A_P]);
    }
}

struct A3Rec {
    long long q;
    int field;
    int group;
    long long out;
};

template <typename S>
__global__ void a3d_gather_kernel(A3Args a, const A3Rec *rec, int nrec, const int32_t *table,
                                  long long nsteps_max, long long it, double *traces) {
    using St = Store<S>;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec || it >= nsteps_max) return;
    const A3Rec e = rec[r];
    const int32_t slot = table[(long long)e.group * nsteps_max + it];
    if (slot < 0) return;
    const S *p = static_cast<const S *>(a.f[e.field]) + e.q;
    traces[e.out + slot] = static_cast<double>(St::ld(p, a.isc[e.field]));
}

}  // namespace sm

using namespace sm;

struct sm_a3d {
    int device = 0;
    int precision = SM_FP32;
    size_t nx2 = 0, ny2 = 0, nz2 = 0, np = 0;
    double dx = 0, dy = 0, dz = 0, dt = 0;
    int pitch = 0;
    size_t it = 0;
    cudaStream_t stream = nullptr;
    A3Args args{};
    DevBuf f[4], psi[6], rho, K, coef;
    std::vector<A3Src> src;
    std::vector<double> vals;
    DevBuf d_src, d_vals;
    int src_dirty = 1;
    std::vector<A3Rec> rec;
    SamplePlan plan;
    DevBuf d_rec, d_table, d_traces;
    int rec_dirty = 1;
    size_t elem = 4;
    size_t psi_cells[6] = {0, 0, 0, 0, 0, 0};
};

namespace {

int a3d_check(sm_a3d_t h) {
    if (!h) return sm_fail(SM_EINVAL, "null a_iso_3d handle");
    return SM_OK;
}

template <typename S>
void a3d_launch(sm_a3d *h) {
    dim3 blk(32, 8, 1);
    dim3 grd((unsigned)((h->nz2 + 31) / 32), (unsigned)((h->ny2 + 7) / 8), (unsigned)h->nx2);
    a3d_velocity_kernel<S><<<grd, blk, 0, h->stream>>>(h->args);
    a3d_pressure_kernel<S><<<grd, blk, 0, h->stream>>>(h->args);
    if (!h->src.empty())
        a3d_source_kernel<S><<<1, 32, 0, h->stream>>>(h->args, h->d_src.as<A3Src>(),
                                                      (int)h->src.size(), h->d_vals.as<double>(),
                                                      (long long)h->it);
    if (!h->rec.empty()) {
        int n = (int)h->rec.size();
        a3d_gather_kernel<S><<<(n + 127) / 128, 128, 0, h->stream>>>(
            h->args, h->d_rec.as<A3Rec>(), n, h->d_table.as<int32_t>(),
            (long long)h->plan.nsteps_max, (long long)h->it, h->d_traces.as<double>());
    }
}

int a3d_field_id(int comp) {
    switch (comp) {
    case SM_VX: return A_VX;
    case SM_VY: return A_VY;
    case SM_VZ: return A_VZ;
    case SM_P: return A_P;
    default: return -1;
    }
}

double a3_to_double(const void *p, size_t i, int prec, float isc) {
    switch (prec) {
    case SM_FP64: return static_cast<const double *>(p)[i];
    case SM_FP16: return (double)__half2float(static_cast<const __half *>(p)[i]) * isc;
    case SM_BF16: return (double)__bfloat162float(static_cast<const __nv_bfloat16 *>(p)[i]) * isc;
    default: return static_cast<const float *>(p)[i];
    }
}

void a3_from_double(void *p, size_t i, int prec, double v, float sc) {
    switch (prec) {
    case SM_FP64: static_cast<double *>(p)[i] = v; break;
    case SM_FP16: static_cast<__half *>(p)[i] = __float2half_rn((float)v * sc); break;
    case SM_BF16: static_cast<__nv_bfloat16 *>(p)[i] = __float2bfloat16_rn((float)v * sc); break;
    default: static_cast<float *>(p)[i] = (float)v; break;
    }
}

}  // namespace

extern "C" int sm_a3d_create(int device, size_t nx2, size_t ny2, size_t nz2, size_t np,
                             double dx, double dy, double dz, double dt, const double *vp,
                             const double *rho, const double *const *coef, int precision,
                             sm_a3d_t *out) {
    if (!out) return sm_fail(SM_EINVAL, "sm_a3d_create: out is NULL");
    *out = nullptr;
    if (nx2 < 2 * np + 2 || ny2 < 2 * np + 2 || nz2 < 2 * np + 2)
        return sm_fail(SM_EINVAL, "sm_a3d_create: grid smaller than the CPML frame");
    if (np < 1) return sm_fail(SM_EINVAL, "sm_a3d_create: np must be >= 1");
    if (!vp || !rho || !coef) return sm_fail(SM_EINVAL, "sm_a3d_create: NULL array");
    for (int c = 0; c < 18; ++c)
        if (!coef[c]) return sm_fail(SM_EINVAL, "sm_a3d_create: NULL coefficient array");
    if (!(dx > 0) || !(dy > 0) || !(dz > 0) || !(dt > 0))
        return sm_fail(SM_EINVAL, "sm_a3d_create: spacings and dt must be > 0");
    if (precision < SM_FP32 || precision > SM_BF16)
        return sm_fail(SM_EINVAL, "sm_a3d_create: unknown precision %d", precision);
    if (ny2 > 65535 * 8 || nx2 > 65535)
        return sm_fail(SM_EINVAL, "sm_a3d_create: grid too large");
    // outside the frame the coefficients must be the reference defaults
    const size_t n2[3] = {nx2, ny2, nz2};
    for (int ax = 0; ax < 3; ++ax) {
        const double *A = coef[3 * ax], *B = coef[3 * ax + 1], *Kk = coef[3 * ax + 2];
        const double *Ah = coef[9 + 3 * ax], *Bh = coef[9 + 3 * ax + 1], *Kh = coef[9 + 3 * ax + 2];
        for (size_t n = np; n + np < n2[ax]; ++n)
            if (A[n] != 0.0 || B[n] != 1.0 || Kk[n] != 1.0)
                return sm_fail(SM_EINVAL, "sm_a3d_create: node coefficients differ from "
                                          "(a,b,k)=(0,1,1) inside the frame, axis %d node %zu", ax, n);
        for (size_t n = np; n + 1 + np < n2[ax]; ++n)
            if (Ah[n] != 0.0 || Bh[n] != 1.0 || Kh[n] != 1.0)
                return sm_fail(SM_EINVAL, "sm_a3d_create: half-node coefficients differ from "
                                          "(a,b,k)=(0,1,1) inside the frame, axis %d node %zu", ax, n);
    }
    int ndev = 0;
    SM_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        return sm_fail(SM_EINVAL, "sm_a3d_create: no CUDA device %d", device);
    DeviceGuard g(device);
    std::unique_ptr<sm_a3d> h(new (std::nothrow) sm_a3d());
    if (!h) return sm_fail(SM_ENOMEM, "sm_a3d_create: out of host memory");
    h->device = device;
    h->precision = precision;
    h->nx2 = nx2; h->ny2 = ny2; h->nz2 = nz2; h->np = np;
    h->dx = dx; h->dy = dy; h->dz = dz; h->dt = dt;
    h->pitch = (int)round_up(nz2, 32);
    h->elem = storage_bytes(precision);
    SM_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    const size_t cb = precision == SM_FP64 ? 8 : 4;
    const size_t ncell = nx2 * ny2 * (size_t)h->pitch;
    int rc;
    for (int f = 0; f < 4; ++f)
        if ((rc = h->f[f].alloc(ncell * h->elem))) return rc;
    h->psi_cells[PS_PX] = h->psi_cells[PS_VX] = 2 * np * ny2 * (size_t)h->pitch;
    h->psi_cells[PS_PY] = h->psi_cells[PS_VY] = nx2 * 2 * np * (size_t)h->pitch;
    h->psi_cells[PS_PZ] = h->psi_cells[PS_VZ] = nx2 * ny2 * 2 * np;
    for (int p = 0; p < 6; ++p)
        if ((rc = h->psi[p].alloc(h->psi_cells[p] * h->elem))) return rc;
    if ((rc = h->rho.alloc(ncell * cb))) return rc;
    if ((rc = h->K.alloc(ncell * cb))) return rc;
    {
        // pitched copies of rho and K = rho vp^2 dt (a_iso_3d.c:407-409)
        std::vector<double> r(ncell, 0.0), kk(ncell, 0.0);
        for (size_t i = 0; i < nx2; ++i)
            for (size_t j = 0; j < ny2; ++j)
                for (size_t k = 0; k < nz2; ++k) {
                    size_t s = (i * ny2 + j) * nz2 + k;
                    size_t d = (i * ny2 + j) * h->pitch + k;
                    r[d] = rho[s];
                    kk[d] = rho[s] * vp[s] * vp[s] * dt;
                }
        // pitch padding: repeat the last real value so the on-the-fly
        // buoyancy never divides by zero there (those cells are not updated)
        for (size_t i = 0; i < nx2; ++i)
            for (size_t j = 0; j < ny2; ++j)
                for (size_t k = nz2; k < (size_t)h->pitch; ++k)
                    r[(i * ny2 + j) * h->pitch + k] = r[(i * ny2 + j) * h->pitch + nz2 - 1];
        rc = precision == SM_FP64 ? upload_convert<double>(h->rho.p, r.data(), ncell, h->stream)
                                  : upload_convert<float>(h->rho.p, r.data(), ncell, h->stream);
        if (rc) return rc;
        rc = precision == SM_FP64 ? upload_convert<double>(h->K.p, kk.data(), ncell, h->stream)
                                  : upload_convert<float>(h->K.p, kk.data(), ncell, h->stream);
        if (rc) return rc;
    }
    A3Coef cf{{(int)nx2, (int)ny2, (int)nz2}};
    {
        std::vector<double> t((size_t)cf.size(), 0.0);
        for (int ax = 0; ax < 3; ++ax) {
            for (size_t n = 0; n < n2[ax]; ++n) {
                t[cf.at(ax, 0) + n] = coef[3 * ax][n];
                t[cf.at(ax, 1) + n] = coef[3 * ax + 1][n];
                t[cf.at(ax, 2) + n] = 1.0 / coef[3 * ax + 2][n];
            }
            for (size_t n = 0; n + 1 < n2[ax]; ++n) {
                t[cf.at(ax, 3) + n] = coef[9 + 3 * ax][n];
                t[cf.at(ax, 4) + n] = coef[9 + 3 * ax + 1][n];
                t[cf.at(ax, 5) + n] = 1.0 / coef[9 + 3 * ax + 2][n];
            }
        }
        if ((rc = h->coef.alloc(t.size() * cb))) return rc;
        rc = precision == SM_FP64 ? upload_convert<double>(h->coef.p, t.data(), t.size(), h->stream)
                                  : upload_convert<float>(h->coef.p, t.data(), t.size(), h->stream);
        if (rc) return rc;
    }
    A3Args &a = h->args;
    a.nx2 = (int)nx2; a.ny2 = (int)ny2; a.nz2 = (int)nz2; a.pitch = h->pitch; a.np = (int)np;
    a.sy = h->pitch;
    a.sx = (long long)ny2 * h->pitch;
    for (int f = 0; f < 4; ++f) { a.f[f] = h->f[f].p; a.sc[f] = 1.f; a.isc[f] = 1.f; }
    for (int p = 0; p < 6; ++p) { a.psi[p] = h->psi[p].p; a.psc[p] = 1.f; a.pisc[p] = 1.f; }
    a.rho = h->rho.p;
    a.K = h->K.p;
    a.coef = h->coef.p;
    a.cf = cf;
    a.two_dt = dt * 2.;
    a.idx = 1.0 / dx; a.idy = 1.0 / dy; a.idz = 1.0 / dz;
    if ((rc = sm_a3d_reset(h.get()))) return rc;
    *out = h.release();
    return SM_OK;
}

extern "C" int sm_a3d_reset(sm_a3d_t h) {
    if (int rc = a3d_check(h)) return rc;
    DeviceGuard g(h->device);
    for (int f = 0; f < 4; ++f)
        if (int rc = h->f[f].zero(h->stream)) return rc;
    for (int p = 0; p < 6; ++p)
        if (int rc = h->psi[p].zero(h->stream)) return rc;
    if (int rc = h->d_traces.zero(h->stream)) return rc;
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->it = 0;
    return SM_OK;
}

extern "C" int sm_a3d_set_sources(sm_a3d_t h, size_t nsrc, const size_t *index, const double *fct,
                                  const size_t *length, size_t stride, double scale) {
    if (int rc = a3d_check(h)) return rc;
    if (nsrc && (!index || !fct || !length)) return sm_fail(SM_EINVAL, "sm_a3d_set_sources: NULL");
    const size_t N = h->nx2 * h->ny2 * h->nz2;
    h->src.clear();
    h->vals.clear();
    for (size_t s = 0; s < nsrc; ++s) {
        if (index[s] >= N) return sm_fail(SM_EINVAL, "sm_a3d_set_sources: source %zu outside", s);
        if (length[s] > stride) return sm_fail(SM_EINVAL, "sm_a3d_set_sources: length > stride");
        size_t k = index[s] % h->nz2, ij = index[s] / h->nz2;
        size_t j = ij % h->ny2, i = ij / h->ny2;
        A3Src e{};
        e.q = (long long)((i * h->ny2 + j) * h->pitch + k);
        e.voff = (long long)h->vals.size();
        e.len = (int)length[s];
        for (size_t t = 0; t < length[s]; ++t) h->vals.push_back(scale * fct[s * stride + t]);
        h->src.push_back(e);
    }
    h->src_dirty = 1;
    return SM_OK;
}

extern "C" int sm_a3d_set_receivers(sm_a3d_t h, size_t nrec, const size_t *index, const int *comp,
                                    const double *t0, const double *rdt, size_t nsteps_max) {
    if (int rc = a3d_check(h)) return rc;
    if (nrec && (!index || !comp || !t0 || !rdt))
        return sm_fail(SM_EINVAL, "sm_a3d_set_receivers: NULL");
    const size_t N = h->nx2 * h->ny2 * h->nz2;
    h->plan.build(nrec, t0, rdt, h->dt, nsteps_max);
    h->rec.clear();
    for (size_t r = 0; r < nrec; ++r) {
        if (index[r] >= N) return sm_fail(SM_EINVAL, "sm_a3d_set_receivers: receiver %zu outside", r);
        int f = a3d_field_id(comp[r]);
        if (f < 0) return sm_fail(SM_EINVAL, "sm_a3d_set_receivers: component %d unsupported", comp[r]);
        size_t k = index[r] % h->nz2, ij = index[r] / h->nz2;
        size_t j = ij % h->ny2, i = ij / h->ny2;
        A3Rec e{};
        e.q = (long long)((i * h->ny2 + j) * h->pitch + k);
        e.field = f;
        e.group = h->plan.group_of[r];
        e.out = (long long)r * (long long)h->plan.max_samples;
        h->rec.push_back(e);
    }
    h->rec_dirty = 1;
    return SM_OK;
}

namespace {
int a3d_upload(sm_a3d *h) {
    int rc;
    if (h->src_dirty) {
        if (!h->src.empty()) {
            if ((rc = h->d_src.alloc(h->src.size() * sizeof(A3Src)))) return rc;
            if ((rc = h->d_vals.alloc(std::max<size_t>(h->vals.size(), 1) * sizeof(double)))) return rc;
            SM_CUDA_TRY(cudaMemcpyAsync(h->d_src.p, h->src.data(), h->src.size() * sizeof(A3Src),
                                        cudaMemcpyHostToDevice, h->stream));
            if (!h->vals.empty())
                SM_CUDA_TRY(cudaMemcpyAsync(h->d_vals.p, h->vals.data(), h->vals.size() * sizeof(double),
                                            cudaMemcpyHostToDevice, h->stream));
        }
        h->src_dirty = 0;
    }
    if (h->rec_dirty) {
        if (!h->rec.empty()) {
            if ((rc = h->d_rec.alloc(h->rec.size() * sizeof(A3Rec)))) return rc;
            if ((rc = h->d_table.alloc(std::max<size_t>(h->plan.table.size(), 1) * sizeof(int32_t))))
                return rc;
            size_t nt = std::max<size_t>(h->rec.size() * h->plan.max_samples, 1);
            if ((rc = h->d_traces.alloc(nt * sizeof(double)))) return rc;
            SM_CUDA_TRY(cudaMemcpyAsync(h->d_rec.p, h->rec.data(), h->rec.size() * sizeof(A3Rec),
                                        cudaMemcpyHostToDevice, h->stream));
            if (!h->plan.table.empty())
                SM_CUDA_TRY(cudaMemcpyAsync(h->d_table.p, h->plan.table.data(),
                                            h->plan.table.size() * sizeof(int32_t),
                                            cudaMemcpyHostToDevice, h->stream));
            SM_CUDA_TRY(cudaMemsetAsync(h->d_traces.p, 0, h->d_traces.bytes, h->stream));
        }
        h->rec_dirty = 0;
    }
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SM_OK;
}
}  // namespace

extern "C" int sm_a3d_run(sm_a3d_t h, size_t nsteps) {
    if (int rc = a3d_check(h)) return rc;
    DeviceGuard g(h->device);
    if (h->src_dirty || h->rec_dirty)
        if (int rc = a3d_upload(h)) return rc;
    for (size_t s = 0; s < nsteps; ++s) {
        switch (h->precision) {
        case SM_FP64: a3d_launch<double>(h); break;
        case SM_FP16: a3d_launch<__half>(h); break;
        case SM_BF16: a3d_launch<__nv_bfloat16>(h); break;
        default: a3d_launch<float>(h); break;
        }
        h->it++;
    }
    SM_CUDA_TRY(cudaGetLastError());
    return SM_OK;
}

extern "C" int sm_a3d_sync(sm_a3d_t h) {
    if (int rc = a3d_check(h)) return rc;
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SM_OK;
}

extern "C" int sm_a3d_step_count(sm_a3d_t h, size_t *it) {
    if (int rc = a3d_check(h)) return rc;
    if (!it) return sm_fail(SM_EINVAL, "sm_a3d_step_count: NULL");
    *it = h->it;
    return SM_OK;
}

extern "C" int sm_a3d_read_traces(sm_a3d_t h, size_t rec0, size_t nrec, double *out, size_t ld,
                                  size_t *counts) {
    if (int rc = a3d_check(h)) return rc;
    if (rec0 + nrec > h->rec.size()) return sm_fail(SM_EINVAL, "sm_a3d_read_traces: range");
    DeviceGuard g(h->device);
    if (h->rec_dirty)
        if (int rc = a3d_upload(h)) return rc;
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    const size_t lim = std::min(h->it, h->plan.nsteps_max);
    std::vector<size_t> gcount(h->plan.count_total.size(), 0);
    for (size_t gi = 0; gi < gcount.size(); ++gi)
        for (size_t it = 0; it < lim; ++it)
            if (h->plan.table[gi * h->plan.nsteps_max + it] >= 0) ++gcount[gi];
    const size_t ms = h->plan.max_samples;
    if (out && nrec && ms) {
        // one bulk copy, then scatter into the caller's layout
        std::vector<double> buf(nrec * ms);
        SM_CUDA_TRY(cudaMemcpy(buf.data(), h->d_traces.as<double>() + rec0 * ms,
                               buf.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (size_t r = 0; r < nrec; ++r) {
            size_t c = gcount[h->rec[rec0 + r].group];
            if (ld < c) return sm_fail(SM_EINVAL, "sm_a3d_read_traces: ld too small");
            std::memcpy(out + r * ld, buf.data() + r * ms, c * sizeof(double));
        }
    }
    if (counts)
        for (size_t r = 0; r < nrec; ++r) counts[r] = gcount[h->rec[rec0 + r].group];
    return SM_OK;
}

extern "C" int sm_a3d_get_field(sm_a3d_t h, int comp, double *out) {
    if (int rc = a3d_check(h)) return rc;
    int f = a3d_field_id(comp);
    if (f < 0 || !out) return sm_fail(SM_EINVAL, "sm_a3d_get_field: bad argument");
    DeviceGuard g(h->device);
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    const size_t ncell = h->nx2 * h->ny2 * (size_t)h->pitch;
    std::vector<unsigned char> buf(ncell * h->elem);
    SM_CUDA_TRY(cudaMemcpy(buf.data(), h->f[f].p, buf.size(), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < h->nx2; ++i)
        for (size_t j = 0; j < h->ny2; ++j)
            for (size_t k = 0; k < h->nz2; ++k)
                out[(i * h->ny2 + j) * h->nz2 + k] =
                    a3_to_double(buf.data(), (i * h->ny2 + j) * h->pitch + k, h->precision,
                                 h->args.isc[f]);
    return SM_OK;
}

extern "C" int sm_a3d_set_field(sm_a3d_t h, int comp, const double *in) {
    if (int rc = a3d_check(h)) return rc;
    int f = a3d_field_id(comp);
    if (f < 0 || !in) return sm_fail(SM_EINVAL, "sm_a3d_set_field: bad argument");
    DeviceGuard g(h->device);
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    const size_t ncell = h->nx2 * h->ny2 * (size_t)h->pitch;
    std::vector<unsigned char> buf(ncell * h->elem, 0);
    for (size_t i = 0; i < h->nx2; ++i)
        for (size_t j = 0; j < h->ny2; ++j)
            for (size_t k = 0; k < h->nz2; ++k)
                a3_from_double(buf.data(), (i * h->ny2 + j) * h->pitch + k, h->precision,
                               in[(i * h->ny2 + j) * h->nz2 + k], h->args.sc[f]);
    SM_CUDA_TRY(cudaMemcpy(h->f[f].p, buf.data(), buf.size(), cudaMemcpyHostToDevice));
    return SM_OK;
}

extern "C" int sm_a3d_destroy(sm_a3d_t h) {
    if (!h) return SM_OK;
    DeviceGuard g(h->device);
    if (h->stream) {
        cudaStreamSynchronize(h->stream);
        cudaStreamDestroy(h->stream);
    }
    delete h;
    return SM_OK;
}

extern "C" int sm_device_info(int device, int *sm_count, size_t *hbm_bytes, size_t *hbm_free) {
    int ndev = 0;
    SM_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return sm_fail(SM_EINVAL, "no CUDA device %d", device);
    DeviceGuard g(device);
    cudaDeviceProp p;
    SM_CUDA_TRY(cudaGetDeviceProperties(&p, device));
    if (sm_count) *sm_count = p.multiProcessorCount;
    size_t fr = 0, tot = 0;
    SM_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    if (hbm_bytes) *hbm_bytes = tot;
    if (hbm_free) *hbm_free = fr;
    return SM_OK;
}
