// sm_eiso.cu -- e_iso (2D P-SV elastic, split-field PML) on sm_100a.
//
// Grid.  The reference keeps the interior (nx x nz, e_iso.c:384-393) and
// the PML frame (8 separate regions, pml.c:54-325) apart.  Here both live on
// one padded grid of NX = nx + 2*np columns by NZ = nz + 2*np rows (z fast,
// row pitch `pitch`), so a neighbour read is one address whatever region it
// lands in:
//   * field arrays (vx, vz, txx, tzz, txz) hold the total value everywhere;
//     in the frame the total is x part + z part, rewritten each update;
//   * split arrays hold the x and z parts of the frame cells only, in a
//     compact layout (left columns, then 2*np cells per middle column, then
//     right columns): 4 np^2 + 2 np (nx + nz) cells, the reference's count.
// Materials are edge-replicated onto the padded grid on the host (the frame
// uses the interior's edge values, pml.c), pre-scaled by dt/h, and shared by
// all shots of a batch.
//
// Update.  Interior cells (propagate.c:2511-2670):
//   v   += (dt/h * m) * (dx + dz)
// frame cells, one split part per direction (pml.c:39-1403):
//   q_x = A(x) q_x + B(x) (dt/h * m) dx,   A = (2 - dt d)/(2 + dt d),
//   B = 2/(2 + dt d); d = 0 along a strip gives A = B = 1.
// The reference's c1/c2 form (q*c2 + m*delta/h)*c1 is the same expression.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "sm_common.cuh"

namespace sm {

enum { F_VX = 0, F_VZ = 1, F_TXX = 2, F_TZZ = 3, F_TXZ = 4 };
enum { M_B = 0, M_BM = 1, M_LA = 2, M_L2M = 3, M_MU = 4 };

// profile table layout (8 arrays, compute type): A/B for x nodes, x half
// nodes (length NX each), z nodes, z half nodes (length NZ each)
struct EisoProf {
    int NX, NZ;
    __host__ __device__ int axn() const { return 0; }
    __host__ __device__ int bxn() const { return NX; }
    __host__ __device__ int axh() const { return 2 * NX; }
    __host__ __device__ int bxh() const { return 3 * NX; }
    __host__ __device__ int azn() const { return 4 * NX; }
    __host__ __device__ int bzn() const { return 4 * NX + NZ; }
    __host__ __device__ int azh() const { return 4 * NX + 2 * NZ; }
    __host__ __device__ int bzh() const { return 4 * NX + 3 * NZ; }
    __host__ __device__ int size() const { return 4 * NX + 4 * NZ; }
};

struct EisoArgs {
    int NX, NZ, pitch, np, nx, nz;
    long long fstride;   // elements between shots, field arrays
    long long sstride;   // elements between shots, split arrays
    int mid_off, right_off;
    void *f[5];
    void *fx[5];
    void *fz[5];
    const void *mat[5];
    const void *prof;
    float sc[5], isc[5];
};

__device__ __forceinline__ bool e_inside(const EisoArgs &a, int X, int Z) {
    return X >= a.np && X < a.np + a.nx && Z >= a.np && Z < a.np + a.nz;
}

__device__ __forceinline__ int e_pml_index(const EisoArgs &a, int X, int Z) {
    if (X < a.np) return X * a.NZ + Z;
    if (X >= a.np + a.nx) return a.right_off + (X - a.np - a.nx) * a.NZ + Z;
    return a.mid_off + (X - a.np) * 2 * a.np + (Z < a.np ? Z : Z - a.nz);
}

template <typename S>
__global__ void __launch_bounds__(256) eiso_velocity_kernel(EisoArgs a) {
    using C = typename Store<S>::C;
    using St = Store<S>;
    const int Z = blockIdx.x * blockDim.x + threadIdx.x;
    const int X = blockIdx.y * blockDim.y + threadIdx.y;
    if (X >= a.NX || Z >= a.NZ) return;
    const long long fb = (long long)blockIdx.z * a.fstride;
    const long long q = (long long)X * a.pitch + Z;
    const S *txx = static_cast<const S *>(a.f[F_TXX]) + fb;
    const S *tzz = static_cast<const S *>(a.f[F_TZZ]) + fb;
    const S *txz = static_cast<const S *>(a.f[F_TXZ]) + fb;
    S *vx = static_cast<S *>(a.f[F_VX]) + fb;
    S *vz = static_cast<S *>(a.f[F_VZ]) + fb;
    const C zero = C(0);
    // vx at (X, Z): backward x of txx, backward z of txz
    const C txx_c = St::ld(txx + q, a.isc[F_TXX]);
    const C txx_m = X > 0 ? St::ld(txx + q - a.pitch, a.isc[F_TXX]) : zero;
    const C txz_c = St::ld(txz + q, a.isc[F_TXZ]);
    const C txz_zm = Z > 0 ? St::ld(txz + q - 1, a.isc[F_TXZ]) : zero;
    // vz at (X+1/2, Z+1/2): forward x of txz, forward z of tzz
    const C txz_xp = X + 1 < a.NX ? St::ld(txz + q + a.pitch, a.isc[F_TXZ]) : zero;
    const C tzz_c = St::ld(tzz + q, a.isc[F_TZZ]);
    const C tzz_zp = Z + 1 < a.NZ ? St::ld(tzz + q + 1, a.isc[F_TZZ]) : zero;
    const C ax = txx_c - txx_m, az = txz_c - txz_zm;
    const C bx = txz_xp - txz_c, bz = tzz_zp - tzz_c;
    const C mb = static_cast<const C *>(a.mat[M_B])[q];
    const C mbm = static_cast<const C *>(a.mat[M_BM])[q];
    if (e_inside(a, X, Z)) {
        St::st(vx + q, St::ld(vx + q, a.isc[F_VX]) + mb * (ax + az), a.sc[F_VX]);
        St::st(vz + q, St::ld(vz + q, a.isc[F_VZ]) + mbm * (bx + bz), a.sc[F_VZ]);
        return;
    }
    const C *pr = static_cast<const C *>(a.prof);
    const EisoProf P{a.NX, a.NZ};
    const long long sb = (long long)blockIdx.z * a.sstride;
    const long long c = sb + e_pml_index(a, X, Z);
    S *vxx = static_cast<S *>(a.fx[F_VX]), *vxz = static_cast<S *>(a.fz[F_VX]);
    S *vzx = static_cast<S *>(a.fx[F_VZ]), *vzz = static_cast<S *>(a.fz[F_VZ]);
    const C px = pr[P.axn() + X] * St::ld(vxx + c, a.isc[F_VX]) + pr[P.bxn() + X] * (mb * ax);
    const C pz = pr[P.azn() + Z] * St::ld(vxz + c, a.isc[F_VX]) + pr[P.bzn() + Z] * (mb * az);
    const C qx = pr[P.axh() + X] * St::ld(vzx + c, a.isc[F_VZ]) + pr[P.bxh() + X] * (mbm * bx);
    const C qz = pr[P.azh() + Z] * St::ld(vzz + c, a.isc[F_VZ]) + pr[P.bzh() + Z] * (mbm * bz);
    St::st(vxx + c, px, a.sc[F_VX]);
    St::st(vxz + c, pz, a.sc[F_VX]);
    St::st(vzx + c, qx, a.sc[F_VZ]);
    St::st(vzz + c, qz, a.sc[F_VZ]);
    St::st(vx + q, px + pz, a.sc[F_VX]);
    St::st(vz + q, qx + qz, a.sc[F_VZ]);
}

template <typename S>
__global__ void __launch_bounds__(256) eiso_stress_kernel(EisoArgs a) {
    using C = typename Store<S>::C;
    using St = Store<S>;
    const int Z = blockIdx.x * blockDim.x + threadIdx.x;
    const int X = blockIdx.y * blockDim.y + threadIdx.y;
    if (X >= a.NX || Z >= a.NZ) return;
    const long long fb = (long long)blockIdx.z * a.fstride;
    const long long q = (long long)X * a.pitch + Z;
    const S *vx = static_cast<const S *>(a.f[F_VX]) + fb;
    const S *vz = static_cast<const S *>(a.f[F_VZ]) + fb;
    S *txx = static_cast<S *>(a.f[F_TXX]) + fb;
    S *tzz = static_cast<S *>(a.f[F_TZZ]) + fb;
    S *txz = static_cast<S *>(a.f[F_TXZ]) + fb;
    const C zero = C(0);
    const C vx_c = St::ld(vx + q, a.isc[F_VX]);
    const C vx_xp = X + 1 < a.NX ? St::ld(vx + q + a.pitch, a.isc[F_VX]) : zero;
    const C vx_zp = Z + 1 < a.NZ ? St::ld(vx + q + 1, a.isc[F_VX]) : zero;
    const C vz_c = St::ld(vz + q, a.isc[F_VZ]);
    const C vz_zm = Z > 0 ? St::ld(vz + q - 1, a.isc[F_VZ]) : zero;
    const C vz_xm = X > 0 ? St::ld(vz + q - a.pitch, a.isc[F_VZ]) : zero;
    // txx, tzz at (X+1/2, Z): forward x of vx, backward z of vz
    const C ax = vx_xp - vx_c, az = vz_c - vz_zm;
    // txz at (X, Z+1/2): forward z of vx, backward x of vz
    const C bz = vx_zp - vx_c, bx = vz_c - vz_xm;
    const C la = static_cast<const C *>(a.mat[M_LA])[q];
    const C l2m = static_cast<const C *>(a.mat[M_L2M])[q];
    const C mu = static_cast<const C *>(a.mat[M_MU])[q];
    if (e_inside(a, X, Z)) {
        St::st(txx + q, St::ld(txx + q, a.isc[F_TXX]) + (l2m * ax + la * az), a.sc[F_TXX]);
        St::st(tzz + q, St::ld(tzz + q, a.isc[F_TZZ]) + (l2m * az + la * ax), a.sc[F_TZZ]);
        St::st(txz + q, St::ld(txz + q, a.isc[F_TXZ]) + mu * (bz + bx), a.sc[F_TXZ]);
        return;
    }
    const C *pr = static_cast<const C *>(a.prof);
    const EisoProf P{a.NX, a.NZ};
    const long long sb = (long long)blockIdx.z * a.sstride;
    const long long c = sb + e_pml_index(a, X, Z);
    S *xxx = static_cast<S *>(a.fx[F_TXX]), *xxz = static_cast<S *>(a.fz[F_TXX]);
    S *zzx = static_cast<S *>(a.fx[F_TZZ]), *zzz = static_cast<S *>(a.fz[F_TZZ]);
    S *xzx = static_cast<S *>(a.fx[F_TXZ]), *xzz = static_cast<S *>(a.fz[F_TXZ]);
    const C Axh = pr[P.axh() + X], Bxh = pr[P.bxh() + X];
    const C Azn = pr[P.azn() + Z], Bzn = pr[P.bzn() + Z];
    const C s1 = Axh * St::ld(xxx + c, a.isc[F_TXX]) + Bxh * (l2m * ax);
    const C s2 = Azn * St::ld(xxz + c, a.isc[F_TXX]) + Bzn * (la * az);
    const C s3 = Axh * St::ld(zzx + c, a.isc[F_TZZ]) + Bxh * (la * ax);
    const C s4 = Azn * St::ld(zzz + c, a.isc[F_TZZ]) + Bzn * (l2m * az);
    const C s5 = pr[P.axn() + X] * St::ld(xzx + c, a.isc[F_TXZ]) + pr[P.bxn() + X] * (mu * bx);
    const C s6 = pr[P.azh() + Z] * St::ld(xzz + c, a.isc[F_TXZ]) + pr[P.bzh() + Z] * (mu * bz);
    St::st(xxx + c, s1, a.sc[F_TXX]);
    St::st(xxz + c, s2, a.sc[F_TXX]);
    St::st(zzx + c, s3, a.sc[F_TZZ]);
    St::st(zzz + c, s4, a.sc[F_TZZ]);
    St::st(xzx + c, s5, a.sc[F_TXZ]);
    St::st(xzz + c, s6, a.sc[F_TXZ]);
    St::st(txx + q, s1 + s2, a.sc[F_TXX]);
    St::st(tzz + q, s3 + s4, a.sc[F_TZZ]);
    St::st(txz + q, s5 + s6, a.sc[F_TXZ]);
}

// one entry per source, sorted by shot; one thread per shot adds its
// sources in order, as add_src does (src.c:170-184)
struct SrcEntry {
    long long q;      // padded cell index
    int shot;
    int type;         // SM_SRC_*
    long long voff;   // offset of its scaled samples in vals
    int len;
};

template <typename S>
__global__ void eiso_source_kernel(EisoArgs a, const SrcEntry *src, const int *shot_first,
                                   const double *vals, int nshots, long long it) {
    using St = Store<S>;
    using C = typename Store<S>::C;
    const int shot = blockIdx.x * blockDim.x + threadIdx.x;
    if (shot >= nshots) return;
    for (int e = shot_first[shot]; e < shot_first[shot + 1]; ++e) {
        const SrcEntry s = src[e];
        if (it >= s.len) continue;
        const C v = static_cast<C>(vals[s.voff + it]);
        const long long base = (long long)shot * a.fstride + s.q;
        if (s.type == SM_SRC_SX || s.type == SM_SRC_BULK) {
            S *p = static_cast<S *>(a.f[F_TXX]) + base;
            St::st(p, St::ld(p, a.isc[F_TXX]) + v, a.sc[F_TXX]);
        }
        if (s.type == SM_SRC_SZ || s.type == SM_SRC_BULK) {
            S *p = static_cast<S *>(a.f[F_TZZ]) + base;
            St::st(p, St::ld(p, a.isc[F_TZZ]) + v, a.sc[F_TZZ]);
        }
        if (s.type == SM_SRC_SXZ) {
            S *p = static_cast<S *>(a.f[F_TXZ]) + base;
            St::st(p, St::ld(p, a.isc[F_TXZ]) + v, a.sc[F_TXZ]);
        }
    }
}

struct RecEntry {
    long long q;       // padded cell index
    int shot;
    int field;         // F_*
    int group;         // sampling group
    long long out;     // offset of its first sample in the trace buffer
};

template <typename S>
__global__ void eiso_gather_kernel(EisoArgs a, const RecEntry *rec, int nrec,
                                   const int32_t *table, long long nsteps_max, long long it,
                                   double *traces) {
    using St = Store<S>;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec || it >= nsteps_max) return;
    const RecEntry e = rec[r];
    const int32_t slot = table[(long long)e.group * nsteps_max + it];
    if (slot < 0) return;
    const S *p = static_cast<const S *>(a.f[e.field]) + (long long)e.shot * a.fstride + e.q;
    traces[e.out + slot] = static_cast<double>(St::ld(p, a.isc[e.field]));
}

}  // namespace sm

using namespace sm;

struct ShotRecs {
    std::vector<RecEntry> entries;   // this shot's receivers (out offsets local)
    SamplePlan plan;
};

struct sm_eiso {
    int device = 0;
    int precision = SM_FP32;
    size_t nx = 0, nz = 0, np = 0, nshots = 1;
    double h = 0, dt = 0;
    int NX = 0, NZ = 0, pitch = 0;
    size_t npml_cells = 0;
    size_t it = 0;
    cudaStream_t stream = nullptr;
    EisoArgs args{};
    DevBuf fields[5], xpart[5], zpart[5], mat[5], prof;
    // sources
    std::vector<std::vector<SrcEntry>> shot_src;     // per shot (voff local)
    std::vector<std::vector<double>> shot_vals;      // per shot scaled samples
    DevBuf d_src, d_src_first, d_vals;
    int src_dirty = 1;
    // receivers
    std::vector<ShotRecs> shot_rec;
    DevBuf d_rec, d_table, d_traces;
    std::vector<size_t> rec_base;                    // per shot offset into flat list
    std::vector<long long> rec_out_base;             // per shot offset into traces
    int n_rec_total = 0;
    long long table_steps = 0;
    int rec_dirty = 1;
    size_t elem = 4;
    KernelTimer timer;
    // 16-bit storage: one exponent per field (total and split parts share it)
    Scaler16 scaler;
    std::vector<int> expo0;
    double mat_min[2] = {0, 0};   // min rho, min vp implied by the materials
    static constexpr int kScalePeriod = 16;
};

namespace {

int eiso_check(sm_eiso_t h) {
    if (!h) return sm_fail(SM_EINVAL, "null e_iso handle");
    return SM_OK;
}

template <typename S>
void launch_step(sm_eiso *h) {
    dim3 blk(32, 8, 1);
    dim3 grd((h->NZ + 31) / 32, (h->NX + 7) / 8, (unsigned)h->nshots);
    cudaEvent_t t0 = h->timer.begin(h->stream);
    eiso_velocity_kernel<S><<<grd, blk, 0, h->stream>>>(h->args);
    eiso_stress_kernel<S><<<grd, blk, 0, h->stream>>>(h->args);
    h->timer.end(t0, h->stream);
    h->timer.launches += 2;
}

template <typename S>
void launch_src(sm_eiso *h) {
    if (h->d_src.bytes == 0) return;
    int n = (int)h->nshots;
    h->timer.launches += 1;
    eiso_source_kernel<S><<<(n + 127) / 128, 128, 0, h->stream>>>(
        h->args, h->d_src.as<SrcEntry>(), h->d_src_first.as<int>(), h->d_vals.as<double>(), n,
        (long long)h->it);
}

template <typename S>
void launch_gather(sm_eiso *h) {
    if (h->n_rec_total == 0) return;
    int n = h->n_rec_total;
    h->timer.launches += 1;
    eiso_gather_kernel<S><<<(n + 127) / 128, 128, 0, h->stream>>>(
        h->args, h->d_rec.as<RecEntry>(), n, h->d_table.as<int32_t>(), h->table_steps,
        (long long)h->it, h->d_traces.as<double>());
}

bool eiso_is16(const sm_eiso *h) { return h->precision == SM_FP16 || h->precision == SM_BF16; }

void eiso_apply_scales(sm_eiso *h) {
    for (int f = 0; f < 5; ++f) {
        h->args.sc[f] = std::ldexp(1.0f, h->scaler.expo[f]);
        h->args.isc[f] = std::ldexp(1.0f, -h->scaler.expo[f]);
    }
}

int eiso_rescale(sm_eiso *h) {
    void *ptrs[15];
    size_t ns[15];
    int groups[15];
    static const char *names[5] = {"vx", "vz", "txx", "tzz", "txz"};
    const size_t fcells = (size_t)h->NX * h->pitch * h->nshots;
    for (int f = 0; f < 5; ++f) {
        ptrs[3 * f] = h->fields[f].p; ns[3 * f] = fcells; groups[3 * f] = f;
        ptrs[3 * f + 1] = h->xpart[f].p; ns[3 * f + 1] = h->npml_cells * h->nshots; groups[3 * f + 1] = f;
        ptrs[3 * f + 2] = h->zpart[f].p; ns[3 * f + 2] = h->npml_cells * h->nshots; groups[3 * f + 2] = f;
    }
    int rc = h->precision == SM_FP16
                 ? h->scaler.check<__half>(h->stream, 15, ptrs, ns, groups, names)
                 : h->scaler.check<__nv_bfloat16>(h->stream, 15, ptrs, ns, groups, names);
    eiso_apply_scales(h);
    return rc;
}

int upload_sources(sm_eiso *h) {
    std::vector<SrcEntry> all;
    std::vector<int> first(h->nshots + 1, 0);
    std::vector<double> vals;
    for (size_t s = 0; s < h->nshots; ++s) {
        first[s] = (int)all.size();
        long long base = (long long)vals.size();
        for (SrcEntry e : h->shot_src[s]) {
            e.voff += base;
            all.push_back(e);
        }
        vals.insert(vals.end(), h->shot_vals[s].begin(), h->shot_vals[s].end());
    }
    first[h->nshots] = (int)all.size();
    int rc;
    if (all.empty()) {
        h->d_src.release();
        h->src_dirty = 0;
        return SM_OK;
    }
    if ((rc = h->d_src.alloc(all.size() * sizeof(SrcEntry)))) return rc;
    if ((rc = h->d_src_first.alloc(first.size() * sizeof(int)))) return rc;
    if ((rc = h->d_vals.alloc(std::max<size_t>(vals.size(), 1) * sizeof(double)))) return rc;
    SM_CUDA_TRY(cudaMemcpyAsync(h->d_src.p, all.data(), all.size() * sizeof(SrcEntry),
                                cudaMemcpyHostToDevice, h->stream));
    SM_CUDA_TRY(cudaMemcpyAsync(h->d_src_first.p, first.data(), first.size() * sizeof(int),
                                cudaMemcpyHostToDevice, h->stream));
    if (!vals.empty())
        SM_CUDA_TRY(cudaMemcpyAsync(h->d_vals.p, vals.data(), vals.size() * sizeof(double),
                                    cudaMemcpyHostToDevice, h->stream));
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->src_dirty = 0;
    return SM_OK;
}

int upload_receivers(sm_eiso *h) {
    // flatten every shot's receivers; each shot's sampling groups get a
    // distinct group id range in one combined table with a common step count
    long long steps = 0;
    for (auto &sr : h->shot_rec) steps = std::max<long long>(steps, (long long)sr.plan.nsteps_max);
    std::vector<RecEntry> all;
    std::vector<int32_t> table;
    h->rec_base.assign(h->nshots, 0);
    h->rec_out_base.assign(h->nshots, 0);
    long long out = 0;
    int gbase = 0;
    for (size_t s = 0; s < h->nshots; ++s) {
        ShotRecs &sr = h->shot_rec[s];
        h->rec_base[s] = all.size();
        h->rec_out_base[s] = out;
        size_t ng = sr.plan.count_total.size();
        for (size_t g = 0; g < ng; ++g) {
            for (long long it = 0; it < steps; ++it)
                table.push_back(it < (long long)sr.plan.nsteps_max
                                    ? sr.plan.table[g * sr.plan.nsteps_max + it]
                                    : -1);
        }
        for (size_t r = 0; r < sr.entries.size(); ++r) {
            RecEntry e = sr.entries[r];
            e.group += gbase;
            e.out = out + (long long)r * (long long)sr.plan.max_samples;
            all.push_back(e);
        }
        out += (long long)sr.entries.size() * (long long)sr.plan.max_samples;
        gbase += (int)ng;
    }
    h->n_rec_total = (int)all.size();
    h->table_steps = steps;
    h->rec_dirty = 0;
    if (all.empty()) return SM_OK;
    int rc;
    if ((rc = h->d_rec.alloc(all.size() * sizeof(RecEntry)))) return rc;
    if ((rc = h->d_table.alloc(std::max<size_t>(table.size(), 1) * sizeof(int32_t)))) return rc;
    if ((rc = h->d_traces.alloc(std::max<long long>(out, 1) * sizeof(double)))) return rc;
    SM_CUDA_TRY(cudaMemcpyAsync(h->d_rec.p, all.data(), all.size() * sizeof(RecEntry),
                                cudaMemcpyHostToDevice, h->stream));
    if (!table.empty())
        SM_CUDA_TRY(cudaMemcpyAsync(h->d_table.p, table.data(), table.size() * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, h->stream));
    SM_CUDA_TRY(cudaMemsetAsync(h->d_traces.p, 0, h->d_traces.bytes, h->stream));
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SM_OK;
}

// host-side conversion between the device storage type and double
double to_double(const void *p, size_t i, int prec, float isc) {
    switch (prec) {
    case SM_FP64: return static_cast<const double *>(p)[i];
    case SM_FP16: return (double)__half2float(static_cast<const __half *>(p)[i]) * isc;
    case SM_BF16: return (double)__bfloat162float(static_cast<const __nv_bfloat16 *>(p)[i]) * isc;
    default: return static_cast<const float *>(p)[i];
    }
}

void from_double(void *p, size_t i, int prec, double v, float sc) {
    switch (prec) {
    case SM_FP64: static_cast<double *>(p)[i] = v; break;
    case SM_FP16: static_cast<__half *>(p)[i] = __float2half_rn((float)v * sc); break;
    case SM_BF16: static_cast<__nv_bfloat16 *>(p)[i] = __float2bfloat16_rn((float)v * sc); break;
    default: static_cast<float *>(p)[i] = (float)v; break;
    }
}

int field_id(int comp) {
    switch (comp) {
    case SM_VX: return F_VX;
    case SM_VZ: return F_VZ;
    case SM_TXX: return F_TXX;
    case SM_TZZ: return F_TZZ;
    case SM_TXZ: return F_TXZ;
    default: return -1;
    }
}

bool in_frame(const sm_eiso *h, size_t X, size_t Z) {
    return X < h->np || X >= h->np + h->nx || Z < h->np || Z >= h->np + h->nz;
}

size_t pml_index_host(const sm_eiso *h, size_t X, size_t Z) {
    size_t np = h->np;
    if (X < np) return X * h->NZ + Z;
    if (X >= np + h->nx) return (size_t)h->args.right_off + (X - np - h->nx) * h->NZ + Z;
    return (size_t)h->args.mid_off + (X - np) * 2 * np + (Z < np ? Z : Z - h->nz);
}

}  // namespace

extern "C" int sm_eiso_create(int device, size_t nx, size_t nz, size_t npml, double hh,
                              double dt, const double *la, const double *mu, const double *l2m,
                              const double *b, const double *bm, const double *d,
                              const double *dh, const double *dH, int precision, size_t nshots,
                              sm_eiso_t *out) {
    if (!out) return sm_fail(SM_EINVAL, "sm_eiso_create: out is NULL");
    *out = nullptr;
    if (nx < 2 || nz < 2) return sm_fail(SM_EINVAL, "sm_eiso_create: nx, nz must be >= 2");
    if (npml < 1)
        return sm_fail(SM_EINVAL,
                       "sm_eiso_create: npml must be >= 1 (the reference indexes [npml-1])");
    if (!la || !mu || !l2m || !b || !bm || !d || !dh || !dH)
        return sm_fail(SM_EINVAL, "sm_eiso_create: NULL array");
    if (!(hh > 0.0) || !(dt > 0.0)) return sm_fail(SM_EINVAL, "sm_eiso_create: h, dt must be > 0");
    if (nshots < 1 || nshots > 65535)
        return sm_fail(SM_EINVAL, "sm_eiso_create: nshots must be in [1, 65535]");
    if (precision < SM_FP32 || precision > SM_BF16)
        return sm_fail(SM_EINVAL, "sm_eiso_create: unknown precision %d", precision);
    const size_t NX = nx + 2 * npml, NZ = nz + 2 * npml;
    if (NX > (1u << 30) / 4 || NZ > (1u << 30) / 4 || NX * NZ > (size_t)1 << 31)
        return sm_fail(SM_EINVAL, "sm_eiso_create: grid too large");
    int ndev = 0;
    SM_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        return sm_fail(SM_EINVAL, "sm_eiso_create: no CUDA device %d", device);
    DeviceGuard g(device);

    std::unique_ptr<sm_eiso> h(new (std::nothrow) sm_eiso());
    if (!h) return sm_fail(SM_ENOMEM, "sm_eiso_create: out of host memory");
    h->device = device;
    h->precision = precision;
    h->nx = nx; h->nz = nz; h->np = npml; h->nshots = nshots;
    h->h = hh; h->dt = dt;
    h->NX = (int)NX; h->NZ = (int)NZ;
    h->pitch = (int)round_up(NZ, 32);
    h->npml_cells = 4 * npml * npml + 2 * npml * (nx + nz);
    h->elem = storage_bytes(precision);
    SM_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));

    const size_t cplx = precision == SM_FP64 ? 8 : 4;    // compute type bytes
    const size_t fcells = NX * (size_t)h->pitch;
    int rc;
    for (int f = 0; f < 5; ++f) {
        if ((rc = h->fields[f].alloc(fcells * nshots * h->elem))) return rc;
        if ((rc = h->xpart[f].alloc(h->npml_cells * nshots * h->elem))) return rc;
        if ((rc = h->zpart[f].alloc(h->npml_cells * nshots * h->elem))) return rc;
        if ((rc = h->mat[f].alloc(fcells * cplx))) return rc;
    }
    EisoProf P{(int)NX, (int)NZ};
    if ((rc = h->prof.alloc((size_t)P.size() * cplx))) return rc;

    // ---- materials on the padded grid: edge replicated, scaled by dt/h ----
    // pml.c reads the interior's edge values in the frame; for lambda and
    // lambda+2mu in the lower-right corner it reads [nx*nx-1]
    // (pml.c:1044-1084).  That index is kept while it lies inside the array
    // (nx <= nz) and replaced by the intended [nx*nz-1] otherwise.
    {
        const double *src[5] = {b, bm, la, l2m, mu};
        std::vector<double> m(fcells, 0.0);
        const double s = dt / hh;
        size_t lr = nx * nx - 1;
        if (lr >= nx * nz) lr = nx * nz - 1;
        for (int k = 0; k < 5; ++k) {
            std::fill(m.begin(), m.end(), 0.0);
            for (size_t X = 0; X < NX; ++X) {
                size_t i = X < npml ? 0 : (X - npml >= nx ? nx - 1 : X - npml);
                for (size_t Z = 0; Z < NZ; ++Z) {
                    size_t j = Z < npml ? 0 : (Z - npml >= nz ? nz - 1 : Z - npml);
                    size_t idx = i * nz + j;
                    if ((k == M_LA || k == M_L2M) && X >= npml + nx && Z >= npml + nz) idx = lr;
                    m[X * h->pitch + Z] = s * src[k][idx];
                }
            }
            rc = precision == SM_FP64 ? upload_convert<double>(h->mat[k].p, m.data(), fcells, h->stream)
                                      : upload_convert<float>(h->mat[k].p, m.data(), fcells, h->stream);
            if (rc) return rc;
        }
    }
    // ---- damping tables: A = (2 - dt d)/(2 + dt d), B = 2/(2 + dt d) ----
    {
        std::vector<double> t((size_t)P.size(), 1.0);
        auto fill = [&](int aoff, int boff, size_t n, size_t ncell, bool half) {
            for (size_t X = 0; X < n; ++X) {
                double dd = -1.0;
                if (X < npml) dd = half ? dh[X] : d[X];
                else if (X >= npml + ncell) {
                    size_t i = X - npml - ncell;
                    dd = half ? dH[npml - 1 - i] : d[npml - 1 - i];
                }
                if (dd >= 0.0) {
                    t[aoff + X] = (2. - dt * dd) / (2. + dt * dd);
                    t[boff + X] = 2. / (2. + dt * dd);
                }
            }
        };
        fill(P.axn(), P.bxn(), NX, nx, false);
        fill(P.axh(), P.bxh(), NX, nx, true);
        fill(P.azn(), P.bzn(), NZ, nz, false);
        fill(P.azh(), P.bzh(), NZ, nz, true);
        rc = precision == SM_FP64 ? upload_convert<double>(h->prof.p, t.data(), t.size(), h->stream)
                                  : upload_convert<float>(h->prof.p, t.data(), t.size(), h->stream);
        if (rc) return rc;
    }
    EisoArgs &a = h->args;
    a.NX = (int)NX; a.NZ = (int)NZ; a.pitch = h->pitch;
    a.np = (int)npml; a.nx = (int)nx; a.nz = (int)nz;
    a.fstride = (long long)fcells;
    a.sstride = (long long)h->npml_cells;
    a.mid_off = (int)(npml * NZ);
    a.right_off = (int)(npml * NZ + nx * 2 * npml);
    for (int f = 0; f < 5; ++f) {
        a.f[f] = h->fields[f].p;
        a.fx[f] = h->xpart[f].p;
        a.fz[f] = h->zpart[f].p;
        a.mat[f] = h->mat[f].p;
        a.sc[f] = 1.0f;
        a.isc[f] = 1.0f;
    }
    a.prof = h->prof.p;
    if (precision == SM_FP16 || precision == SM_BF16) {
        if ((rc = h->scaler.init(5, 15))) return rc;
        h->expo0.assign(5, 0);
        // smallest impedance rho * vp over the model: rho = 1/b and
        // vp^2 = (lambda + 2 mu) / rho at the nodes
        double zmin = -1.0;
        for (size_t q = 0; q < nx * nz; ++q) {
            const double rho = 1.0 / b[q];
            const double z = std::sqrt(std::max(l2m[q], 0.0) * rho);
            if (zmin < 0 || z < zmin) zmin = z;
        }
        h->mat_min[0] = zmin > 0 ? zmin : 1.0;
        eiso_apply_scales(h.get());
    }
    h->shot_src.assign(nshots, {});
    h->shot_vals.assign(nshots, {});
    h->shot_rec.assign(nshots, {});
    if ((rc = sm_eiso_reset(h.get()))) return rc;
    *out = h.release();
    return SM_OK;
}

extern "C" int sm_eiso_reset(sm_eiso_t h) {
    if (int rc = eiso_check(h)) return rc;
    DeviceGuard g(h->device);
    for (int f = 0; f < 5; ++f) {
        if (int rc = h->fields[f].zero(h->stream)) return rc;
        if (int rc = h->xpart[f].zero(h->stream)) return rc;
        if (int rc = h->zpart[f].zero(h->stream)) return rc;
    }
    if (int rc = h->d_traces.zero(h->stream)) return rc;
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->it = 0;
    if (eiso_is16(h)) {
        h->scaler.expo = h->expo0;
        eiso_apply_scales(h);
    }
    return SM_OK;
}

extern "C" int sm_eiso_set_sources(sm_eiso_t h, size_t shot, size_t nsrc, const size_t *index,
                                   const int *type, const double *fct, const size_t *length,
                                   size_t stride, double scale) {
    if (int rc = eiso_check(h)) return rc;
    if (shot != SM_ALL_SHOTS && shot >= h->nshots)
        return sm_fail(SM_EINVAL, "sm_eiso_set_sources: shot %zu out of range", shot);
    if (nsrc && (!index || !type || !fct || !length))
        return sm_fail(SM_EINVAL, "sm_eiso_set_sources: NULL array");
    std::vector<SrcEntry> e;
    std::vector<double> vals;
    for (size_t s = 0; s < nsrc; ++s) {
        if (index[s] >= h->nx * h->nz)
            return sm_fail(SM_EINVAL, "sm_eiso_set_sources: source %zu outside the grid", s);
        int t = type[s];
        if (t != SM_SRC_SX && t != SM_SRC_SZ && t != SM_SRC_SXZ && t != SM_SRC_BULK)
            return sm_fail(SM_EINVAL, "sm_eiso_set_sources: source type %d not supported", t);
        if (length[s] > stride)
            return sm_fail(SM_EINVAL, "sm_eiso_set_sources: length exceeds stride");
        size_t i = index[s] / h->nz, j = index[s] % h->nz;
        SrcEntry se{};
        se.q = (long long)(i + h->np) * h->pitch + (long long)(j + h->np);
        se.type = t;
        se.voff = (long long)vals.size();
        se.len = (int)length[s];
        for (size_t k = 0; k < length[s]; ++k) vals.push_back(scale * fct[s * stride + k]);
        e.push_back(se);
    }
    for (size_t s = 0; s < h->nshots; ++s) {
        if (shot != SM_ALL_SHOTS && s != shot) continue;
        h->shot_src[s] = e;
        for (auto &x : h->shot_src[s]) x.shot = (int)s;
        h->shot_vals[s] = vals;
    }
    h->src_dirty = 1;
    if (eiso_is16(h)) {
        // starting ranges: the stress a source cell accumulates (running sum
        // of the injected values) and the particle velocity it drives
        // (stress / (rho vp)); the range checks refine them during the run
        double tmax = 0.0;
        for (size_t s = 0; s < h->nshots; ++s)
            for (const SrcEntry &se : h->shot_src[s]) {
                double acc = 0.0;
                for (int t = 0; t < se.len; ++t) {
                    acc += h->shot_vals[s][se.voff + t];
                    tmax = std::max(tmax, std::fabs(acc));
                }
            }
        const int et = Scaler16::expo_for(tmax), ev = Scaler16::expo_for(tmax / h->mat_min[0]);
        h->expo0 = {ev, ev, et, et, et};
        for (int g = 0; g < 5; ++g) h->scaler.ceil[g] = h->expo0[g] + 2;
        if (h->it == 0) {
            h->scaler.expo = h->expo0;
            eiso_apply_scales(h);
        }
    }
    return SM_OK;
}

extern "C" int sm_eiso_set_receivers(sm_eiso_t h, size_t shot, size_t nrec, const size_t *index,
                                     const int *comp, const double *t0, const double *rdt,
                                     size_t nsteps_max) {
    if (int rc = eiso_check(h)) return rc;
    if (shot != SM_ALL_SHOTS && shot >= h->nshots)
        return sm_fail(SM_EINVAL, "sm_eiso_set_receivers: shot %zu out of range", shot);
    if (nrec && (!index || !comp || !t0 || !rdt))
        return sm_fail(SM_EINVAL, "sm_eiso_set_receivers: NULL array");
    ShotRecs sr;
    sr.plan.build(nrec, t0, rdt, h->dt, nsteps_max);
    for (size_t r = 0; r < nrec; ++r) {
        if (index[r] >= h->nx * h->nz)
            return sm_fail(SM_EINVAL, "sm_eiso_set_receivers: receiver %zu outside the grid", r);
        int f = field_id(comp[r]);
        if (f < 0)
            return sm_fail(SM_EINVAL, "sm_eiso_set_receivers: component %d not recorded by e_iso",
                           comp[r]);
        size_t i = index[r] / h->nz, j = index[r] % h->nz;
        RecEntry e{};
        e.q = (long long)(i + h->np) * h->pitch + (long long)(j + h->np);
        e.field = f;
        e.group = sr.plan.group_of[r];
        sr.entries.push_back(e);
    }
    for (size_t s = 0; s < h->nshots; ++s) {
        if (shot != SM_ALL_SHOTS && s != shot) continue;
        h->shot_rec[s] = sr;
        for (auto &x : h->shot_rec[s].entries) x.shot = (int)s;
    }
    h->rec_dirty = 1;
    return SM_OK;
}

extern "C" int sm_eiso_run(sm_eiso_t h, size_t nsteps) {
    if (int rc = eiso_check(h)) return rc;
    DeviceGuard g(h->device);
    if (h->src_dirty)
        if (int rc = upload_sources(h)) return rc;
    if (h->rec_dirty)
        if (int rc = upload_receivers(h)) return rc;
    for (size_t k = 0; k < nsteps; ++k) {
        switch (h->precision) {
        case SM_FP64: launch_step<double>(h); launch_src<double>(h); launch_gather<double>(h); break;
        case SM_FP16: launch_step<__half>(h); launch_src<__half>(h); launch_gather<__half>(h); break;
        case SM_BF16:
            launch_step<__nv_bfloat16>(h); launch_src<__nv_bfloat16>(h);
            launch_gather<__nv_bfloat16>(h);
            break;
        default: launch_step<float>(h); launch_src<float>(h); launch_gather<float>(h); break;
        }
        h->it++;
        if (eiso_is16(h) && h->it % sm_eiso::kScalePeriod == 0)
            if (int rc = eiso_rescale(h)) return rc;
    }
    SM_CUDA_TRY(cudaGetLastError());
    return SM_OK;
}

extern "C" int sm_eiso_sync(sm_eiso_t h) {
    if (int rc = eiso_check(h)) return rc;
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SM_OK;
}

extern "C" int sm_eiso_step_count(sm_eiso_t h, size_t *it) {
    if (int rc = eiso_check(h)) return rc;
    if (!it) return sm_fail(SM_EINVAL, "sm_eiso_step_count: NULL");
    *it = h->it;
    return SM_OK;
}

extern "C" int sm_eiso_read_traces(sm_eiso_t h, size_t shot, size_t rec0, size_t nrec,
                                   double *out, size_t ld, size_t *counts) {
    if (int rc = eiso_check(h)) return rc;
    if (shot >= h->nshots) return sm_fail(SM_EINVAL, "sm_eiso_read_traces: bad shot");
    DeviceGuard g(h->device);
    if (h->rec_dirty)
        if (int rc = upload_receivers(h)) return rc;
    const ShotRecs &sr = h->shot_rec[shot];
    if (rec0 + nrec > sr.entries.size())
        return sm_fail(SM_EINVAL, "sm_eiso_read_traces: receiver range out of bounds");
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    const size_t ms = sr.plan.max_samples;
    std::vector<double> buf(ms);
    for (size_t r = 0; r < nrec; ++r) {
        const RecEntry &e = sr.entries[rec0 + r];
        // samples taken so far by this receiver's group
        size_t c = 0;
        const size_t lim = std::min(h->it, sr.plan.nsteps_max);
        for (size_t it = 0; it < lim; ++it)
            if (sr.plan.table[(size_t)e.group * sr.plan.nsteps_max + it] >= 0) ++c;
        if (counts) counts[r] = c;
        if (!out || c == 0) continue;
        if (ld < c) return sm_fail(SM_EINVAL, "sm_eiso_read_traces: ld smaller than sample count");
        const long long off = h->rec_out_base[shot] + (long long)(rec0 + r) * (long long)ms;
        SM_CUDA_TRY(cudaMemcpy(out + r * ld, h->d_traces.as<double>() + off, c * sizeof(double),
                               cudaMemcpyDeviceToHost));
    }
    return SM_OK;
}

extern "C" int sm_eiso_get_field(sm_eiso_t h, size_t shot, int comp, int part, double *out) {
    if (int rc = eiso_check(h)) return rc;
    int f = field_id(comp);
    if (f < 0 || shot >= h->nshots || !out || part < SM_PART_TOTAL || part > SM_PART_Z)
        return sm_fail(SM_EINVAL, "sm_eiso_get_field: bad argument");
    DeviceGuard g(h->device);
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    const size_t NX = h->NX, NZ = h->NZ, e = h->elem;
    if (part == SM_PART_TOTAL) {
        std::vector<unsigned char> buf(NX * (size_t)h->pitch * e);
        SM_CUDA_TRY(cudaMemcpy(buf.data(),
                               static_cast<char *>(h->fields[f].p) + shot * h->args.fstride * e,
                               buf.size(), cudaMemcpyDeviceToHost));
        for (size_t X = 0; X < NX; ++X)
            for (size_t Z = 0; Z < NZ; ++Z)
                out[X * NZ + Z] = to_double(buf.data(), X * h->pitch + Z, h->precision,
                                            h->args.isc[f]);
        return SM_OK;
    }
    const DevBuf &src = part == SM_PART_X ? h->xpart[f] : h->zpart[f];
    std::vector<unsigned char> buf(h->npml_cells * e);
    SM_CUDA_TRY(cudaMemcpy(buf.data(), static_cast<char *>(src.p) + shot * h->npml_cells * e,
                           buf.size(), cudaMemcpyDeviceToHost));
    for (size_t X = 0; X < NX; ++X)
        for (size_t Z = 0; Z < NZ; ++Z)
            out[X * NZ + Z] = in_frame(h, X, Z) ? to_double(buf.data(), pml_index_host(h, X, Z),
                                                            h->precision, h->args.isc[f])
                                                : 0.0;
    return SM_OK;
}

extern "C" int sm_eiso_set_field(sm_eiso_t h, size_t shot, int comp, int part, const double *in) {
    if (int rc = eiso_check(h)) return rc;
    int f = field_id(comp);
    if (f < 0 || shot >= h->nshots || !in || part < SM_PART_TOTAL || part > SM_PART_Z)
        return sm_fail(SM_EINVAL, "sm_eiso_set_field: bad argument");
    DeviceGuard g(h->device);
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    const size_t NX = h->NX, NZ = h->NZ, e = h->elem;
    std::vector<unsigned char> tot(NX * (size_t)h->pitch * e), px(h->npml_cells * e),
        pz(h->npml_cells * e);
    char *dtot = static_cast<char *>(h->fields[f].p) + shot * h->args.fstride * e;
    char *dpx = static_cast<char *>(h->xpart[f].p) + shot * h->npml_cells * e;
    char *dpz = static_cast<char *>(h->zpart[f].p) + shot * h->npml_cells * e;
    SM_CUDA_TRY(cudaMemcpy(tot.data(), dtot, tot.size(), cudaMemcpyDeviceToHost));
    SM_CUDA_TRY(cudaMemcpy(px.data(), dpx, px.size(), cudaMemcpyDeviceToHost));
    SM_CUDA_TRY(cudaMemcpy(pz.data(), dpz, pz.size(), cudaMemcpyDeviceToHost));
    const float sc = h->args.sc[f], isc = h->args.isc[f];
    for (size_t X = 0; X < NX; ++X)
        for (size_t Z = 0; Z < NZ; ++Z) {
            const double v = in[X * NZ + Z];
            if (!in_frame(h, X, Z)) {
                if (part == SM_PART_TOTAL) from_double(tot.data(), X * h->pitch + Z, h->precision, v, sc);
                continue;
            }
            size_t c = pml_index_host(h, X, Z);
            if (part == SM_PART_X) from_double(px.data(), c, h->precision, v, sc);
            if (part == SM_PART_Z) from_double(pz.data(), c, h->precision, v, sc);
            double t = to_double(px.data(), c, h->precision, isc) +
                       to_double(pz.data(), c, h->precision, isc);
            from_double(tot.data(), X * h->pitch + Z, h->precision, t, sc);
        }
    SM_CUDA_TRY(cudaMemcpy(dtot, tot.data(), tot.size(), cudaMemcpyHostToDevice));
    SM_CUDA_TRY(cudaMemcpy(dpx, px.data(), px.size(), cudaMemcpyHostToDevice));
    SM_CUDA_TRY(cudaMemcpy(dpz, pz.data(), pz.size(), cudaMemcpyHostToDevice));
    return SM_OK;
}

extern "C" int sm_eiso_destroy(sm_eiso_t h) {
    if (!h) return SM_OK;
    {
        DeviceGuard g(h->device);
        if (h->stream) {
            cudaStreamSynchronize(h->stream);
            cudaStreamDestroy(h->stream);
        }
        delete h;
    }
    return SM_OK;
}

extern "C" int sm_eiso_stream(sm_eiso_t h, void **stream) {
    if (int rc = eiso_check(h)) return rc;
    if (!stream) return sm_fail(SM_EINVAL, "sm_eiso_stream: NULL");
    *stream = (void *)h->stream;
    return SM_OK;
}

extern "C" int sm_eiso_set_timing(sm_eiso_t h, int on) {
    if (int rc = eiso_check(h)) return rc;
    h->timer.on = on != 0;
    return SM_OK;
}

extern "C" int sm_eiso_kernel_stats(sm_eiso_t h, int reset, double *update_ms,
                                    size_t *update_launches, size_t *all_launches) {
    if (int rc = eiso_check(h)) return rc;
    DeviceGuard g(h->device);
    return h->timer.stats(reset, update_ms, update_launches, all_launches);
}
