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
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <set>
#include <tuple>
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
    void *f[5];          // wavefields read this step (totals)
    void *fx[5];         // ... and their x / z split parts in the frame
    void *fz[5];
    void *fo[5];         // written this step (the other buffer set)
    void *fxo[5];
    void *fzo[5];
    int *err;            // set by a bounded wait that gave up
    long long *step;     // steps begun; the step kernel counts, source and
                         // receiver kernels of step it read it + 1
    int nshots;          // shots in the buffers
    const void *mat[5];
    const void *prof;
    float sc[5], isc[5];
    // block-floating-point storage: exponent bytes of the set read and the
    // set written, [field][shot][nxb][pitch]; estride bytes per field
    void *fe;
    void *feo;
    long long estride;
    int nxb;
    // ... and its source patches: per shot the first patch (pfirst[nshots]
    // = total), per patch its first row and column, and their FP32 values
    // [patch][field][EISO_PR][EISO_PC] in the set read and the set written
    const int *pfirst;
    const int *pxz;
    float *pv;
    float *pvo;
};

__device__ __forceinline__ bool e_inside(const EisoArgs &a, int X, int Z) {
    return X >= a.np && X < a.np + a.nx && Z >= a.np && Z < a.np + a.nz;
}

__device__ __forceinline__ int e_pml_index(const EisoArgs &a, int X, int Z) {
    if (X < a.np) return X * a.NZ + Z;
    if (X >= a.np + a.nx) return a.right_off + (X - a.np - a.nx) * a.NZ + Z;
    return a.mid_off + (X - a.np) * 2 * a.np + (Z < a.np ? Z : Z - a.nz);
}

// split-part update in the frame: q' = A q + B (m * delta)  (pml.c, see above)
template <typename C>
__device__ __forceinline__ C e_split(C A, C B, C q, C m, C delta) {
    return r_fma(A, q, r_mul(B, r_mul(m, delta)));
}

// The old x / z split parts one march iteration at row X needs: vx at
// (X+1, Z), vz and the three stresses at (X, Z); zero where the cell is not
// in the frame.  Loaded one iteration ahead, like the rows.
template <typename C>
struct ESplit {
    C vx[2], vz[2], t[6];   // t: txx x, txx z, tzz x, tzz z, txz x, txz z
};

template <typename S, typename C>
__device__ __forceinline__ void e_load_split(const EisoArgs &a, long long sb, int X, int Z,
                                             bool zin, ESplit<C> &s) {
    using St = Store<S>;
    s.vx[0] = s.vx[1] = s.vz[0] = s.vz[1] = C(0);
#pragma unroll
    for (int k = 0; k < 6; ++k) s.t[k] = C(0);
    if (!zin) return;
    if (X + 1 >= 0 && X + 1 < a.NX && !e_inside(a, X + 1, Z)) {
        const long long c = sb + e_pml_index(a, X + 1, Z);
        s.vx[0] = St::ld(static_cast<const S *>(a.fx[F_VX]) + c, a.isc[F_VX]);
        s.vx[1] = St::ld(static_cast<const S *>(a.fz[F_VX]) + c, a.isc[F_VX]);
    }
    if (X >= 0 && X < a.NX && !e_inside(a, X, Z)) {
        const long long c = sb + e_pml_index(a, X, Z);
        s.vz[0] = St::ld(static_cast<const S *>(a.fx[F_VZ]) + c, a.isc[F_VZ]);
        s.vz[1] = St::ld(static_cast<const S *>(a.fz[F_VZ]) + c, a.isc[F_VZ]);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int f = F_TXX + k;
            s.t[2 * k] = St::ld(static_cast<const S *>(a.fx[f]) + c, a.isc[f]);
            s.t[2 * k + 1] = St::ld(static_cast<const S *>(a.fz[f]) + c, a.isc[f]);
        }
    }
}

// a frame cell's two split parts, updated, optionally stored to the new set;
// returns their sum, the total
template <typename S, typename C>
__device__ __forceinline__ C e_frame(const EisoArgs &a, int f, long long c, C Ax, C Bx, C Az,
                                     C Bz, C qx, C qz, C mx, C mz, C dx, C dz, bool store) {
    using St = Store<S>;
    const C px = e_split<C>(Ax, Bx, qx, mx, dx);
    const C pz = e_split<C>(Az, Bz, qz, mz, dz);
    if (store) {
        St::st(static_cast<S *>(a.fxo[f]) + c, px, a.sc[f]);
        St::st(static_cast<S *>(a.fzo[f]) + c, pz, a.sc[f]);
    }
    return r_add(px, pz);
}

// z profiles of one lane's cell: A / B at the node and at the half node
template <typename C>
struct EZProf {
    C An, Bn, Ah, Bh;
};

// vx at (X, Z) from its x / z differences of txx / txz (propagate.c:2511-2550,
// pml.c:39-360); q = the old split parts
template <typename S, typename C>
__device__ __forceinline__ C e_vx(const EisoArgs &a, long long sb, int X, int Z, C vold, C mb,
                                  C ax, C az, const C *q, const EZProf<C> &zp, bool store) {
    if (e_inside(a, X, Z)) return r_fma(mb, r_add(ax, az), vold);
    const C *pr = static_cast<const C *>(a.prof);
    const EisoProf P{a.NX, a.NZ};
    return e_frame<S, C>(a, F_VX, sb + e_pml_index(a, X, Z), pr[P.axn() + X], pr[P.bxn() + X],
                         zp.An, zp.Bn, q[0], q[1], mb, mb, ax, az, store);
}

// vz at (X+1/2, Z+1/2) (propagate.c:2552-2588, pml.c:371-680)
template <typename S, typename C>
__device__ __forceinline__ C e_vz(const EisoArgs &a, long long sb, int X, int Z, C vold, C mbm,
                                  C bx, C bz, const C *q, const EZProf<C> &zp, bool store) {
    if (e_inside(a, X, Z)) return r_fma(mbm, r_add(bx, bz), vold);
    const C *pr = static_cast<const C *>(a.prof);
    const EisoProf P{a.NX, a.NZ};
    return e_frame<S, C>(a, F_VZ, sb + e_pml_index(a, X, Z), pr[P.axh() + X], pr[P.bxh() + X],
                         zp.Ah, zp.Bh, q[0], q[1], mbm, mbm, bx, bz, store);
}

// ---------------------------------------------------------------------------
// Slab step kernel: one time step (e_iso.c:595-636) over a slab of TX rows and
// W warp columns of 30 z cells.  One TMA box brings the five old wavefields
// of rows X0-1 .. X0+TX and z cells Z0-1 .. Z0+30W (start rounded down to 16
// bytes; out-of-grid cells read as zero, the reference's boundary), one more
// the five materials; then each warp marches its column down the slab out of
// shared memory, as the band kernel does (z neighbours by shuffles, vx of
// row X and vz of row X-1 carried in registers), with no further waits.
// ---------------------------------------------------------------------------
struct EisoSlabMaps {
    CUtensorMap f;   // the old set's wavefields: (z, x, shot, field), box (BW, TX+2, 1, 5)
    CUtensorMap m;   // materials: (z, x, material), box (BWC, TX+2, 5)
};

template <typename S, int W, int TX>
struct ESlab {
    using C = typename Store<S>::C;
    static constexpr int HS = 16 / (int)sizeof(S), HC = 16 / (int)sizeof(C);
    static constexpr int RX = TX + 2;
    static constexpr int BW = (30 * W + 2 + HS - 1 + HS - 1) / HS * HS;
    static constexpr int BWC = (30 * W + 2 + HC - 1 + HC - 1) / HC * HC;
    static constexpr size_t al(size_t x) { return (x + 127) / 128 * 128; }
    static constexpr size_t oM = al(5 * (size_t)RX * BW * sizeof(S));
    static constexpr size_t oBar = al(oM + 5 * (size_t)RX * BWC * sizeof(C));
    static constexpr size_t bytes = oBar + 16;
    static constexpr unsigned tx =
        (unsigned)(5 * RX * BW * sizeof(S) + 5 * RX * BWC * sizeof(C));
};

template <typename S, int W, int TX, int MINB>
__global__ void __launch_bounds__(32 * W, MINB) eiso_slab_kernel(const EisoArgs a,
                                                                 const __grid_constant__ EisoSlabMaps mp) {
    using C = typename Store<S>::C;
    using St = Store<S>;
    using L = ESlab<S, W, TX>;
    extern __shared__ __align__(128) unsigned char smem[];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if ((blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x) == 0) ++*a.step;
    const S *fbox = reinterpret_cast<const S *>(smem);
    const C *mbox = reinterpret_cast<const C *>(smem + L::oM);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::oBar);
    const int Zc = blockIdx.x * W * 30;              // the slab's first column
    const int X0 = blockIdx.y * TX;
    const int X1 = min(X0 + TX, a.NX);
    const int shot = blockIdx.z;
    // box starts: Zc - 1 rounded down to 16 bytes (Zc - 1 >= -1)
    const int zs = (Zc - 1 + L::HS) / L::HS * L::HS - L::HS;
    const int zc = (Zc - 1 + L::HC) / L::HC * L::HC - L::HC;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_proxy_async();
        mbar_expect_tx(bar, L::tx);
        tma_load_4d(smem, &mp.f, zs, X0 - 1, shot, 0, bar);
        tma_load_3d(smem + L::oM, &mp.m, zc, X0 - 1, 0, bar);
    }
    __syncthreads();   // the barrier is initialised before anyone polls it
    const int Z0 = Zc + warp * 30;
    // warp 0 always has cells (the grid holds no empty slab) and keeps the
    // CTA alive until the copy has landed; later warps past the grid leave
    if (Z0 >= a.NZ) return;
    const int Z = Z0 - 1 + lane;
    const bool zin = Z >= 0 && Z < a.NZ;
    const bool own = lane >= 1 && lane <= 30 && Z < a.NZ;
    const long long fb = (long long)shot * a.fstride;
    const long long sb = (long long)shot * a.sstride;
    const C zero = C(0);
    const int of = Z - zs, om = Z - zc;              // this lane's cell in a box row
    // row X0-1+rho of field f / material m at this lane's cell
    auto F = [&](int rho, int f) -> C {
        return St::ld(fbox + (f * L::RX + rho) * L::BW + of, a.isc[f]);
    };
    auto M = [&](int rho, int m) -> C { return mbox[(m * L::RX + rho) * L::BWC + om]; };
    const bool zint = (Z0 - 1 >= a.np) && (Z0 + 30 <= a.np + a.nz - 1);
    EZProf<C> zp{C(1), C(1), C(1), C(1)};
    if (zin) {
        const C *pr = static_cast<const C *>(a.prof);
        const EisoProf P{a.NX, a.NZ};
        zp = EZProf<C>{pr[P.azn() + Z], pr[P.bzn() + Z], pr[P.azh() + Z], pr[P.bzh() + Z]};
    }
    S *vxo = static_cast<S *>(a.fo[F_VX]) + fb;
    S *vzo = static_cast<S *>(a.fo[F_VZ]) + fb;
    S *txxo = static_cast<S *>(a.fo[F_TXX]) + fb;
    S *tzzo = static_cast<S *>(a.fo[F_TZZ]) + fb;
    S *txzo = static_cast<S *>(a.fo[F_TXZ]) + fb;

    ESplit<C> sp;
    e_load_split<S, C>(a, sb, X0 - 1, Z, zin, sp);
    if (!__all_sync(full, mbar_wait(bar, 0, a.err, 4))) {
        mbar_wait(bar, 0, a.err, 4);   // a last bounded chance for the copy in flight
        return;
    }

    // ---- prologue: vx of row X0 and vz of row X0-1 (recomputed; stored
    // only for X0 == 0, the row no other slab reaches) ----
    C vxc, vzp;
    {
        const C c_txz = F(1, F_TXZ), p_tzz = F(0, F_TZZ);
        const C txz_zm = __shfl_up_sync(full, c_txz, 1);
        const C tzz_zp = __shfl_down_sync(full, p_tzz, 1);
        vxc = zin ? e_vx<S, C>(a, sb, X0, Z, F(1, F_VX), M(1, M_B), r_sub(F(1, F_TXX), F(0, F_TXX)),
                               r_sub(c_txz, txz_zm), sp.vx, zp, X0 == 0 && own)
                  : zero;
        if (X0 == 0 && own) St::st(vxo + (long long)X0 * a.pitch + Z, vxc, a.sc[F_VX]);
        vzp = zero;
        if (X0 >= 1 && zin)
            vzp = e_vz<S, C>(a, sb, X0 - 1, Z, F(0, F_VZ), M(0, M_BM), r_sub(c_txz, F(0, F_TXZ)),
                             r_sub(tzz_zp, p_tzz), sp.vz, zp, false);
    }

    // Lean loop: every row of this slab and the one after lie in the interior
    // update region: no frame tests, no split parts; the arithmetic is the
    // general loop's interior branch, operation for operation.
    if (zint && X0 >= a.np && X1 <= a.np + a.nx - 1) {
        long long q = fb + (long long)X0 * a.pitch + Z;
        S *const fo0 = static_cast<S *>(a.fo[0]);   // the five arrays of the new set
        const long long fso = static_cast<S *>(a.fo[1]) - fo0;
#pragma unroll 2
        for (int rc = 1; rc <= X1 - X0; ++rc, q += a.pitch) {
            const C n_txz = F(rc + 1, F_TXZ), c_txz = F(rc, F_TXZ), c_tzz = F(rc, F_TZZ);
            const C c_txx = F(rc, F_TXX), n_txx = F(rc + 1, F_TXX);
            const C n_vx = F(rc + 1, F_VX), c_vz = F(rc, F_VZ);
            const C n_b = M(rc + 1, M_B), c_bm = M(rc, M_BM);
            const C la = M(rc, M_LA), l2m = M(rc, M_L2M), mu = M(rc, M_MU);
            const C txz_zm = __shfl_up_sync(full, n_txz, 1);
            const C tzz_zp = __shfl_down_sync(full, c_tzz, 1);
            const C ax = r_sub(n_txx, c_txx), az = r_sub(n_txz, txz_zm);
            const C bx = r_sub(n_txz, c_txz), bz = r_sub(tzz_zp, c_tzz);
            const C vxn = r_fma(n_b, r_add(ax, az), n_vx);
            const C vzn = r_fma(c_bm, r_add(bx, bz), c_vz);
            const C vz_zm = __shfl_up_sync(full, vzn, 1);
            const C vx_zp = __shfl_down_sync(full, vxc, 1);
            const C sax = r_sub(vxn, vxc), saz = r_sub(vzn, vz_zm);
            const C sbz = r_sub(vx_zp, vxc), sbx = r_sub(vzn, vzp);
            const C txx = r_add(c_txx, r_fma(l2m, sax, r_mul(la, saz)));
            const C tzz = r_add(c_tzz, r_fma(l2m, saz, r_mul(la, sax)));
            const C txz = r_fma(mu, r_add(sbz, sbx), c_txz);
            if (own) {
                S *o = fo0 + q;
                St::st(o + F_VX * fso + a.pitch, vxn, a.sc[F_VX]);
                St::st(o + F_VZ * fso, vzn, a.sc[F_VZ]);
                St::st(o + F_TXX * fso, txx, a.sc[F_TXX]);
                St::st(o + F_TZZ * fso, tzz, a.sc[F_TZZ]);
                St::st(o + F_TXZ * fso, txz, a.sc[F_TXZ]);
            }
            vxc = vxn;
            vzp = vzn;
        }
        return;
    }

    e_load_split<S, C>(a, sb, X0, Z, zin, sp);
    for (int X = X0; X < X1; ++X) {
        const int rc = X - X0 + 1;                   // row X; row X+1 is rc + 1
        ESplit<C> sn;
        e_load_split<S, C>(a, sb, X + 1, Z, zin && X + 1 < X1, sn);
        const bool fast = zint && X >= a.np && X + 1 <= a.np + a.nx - 1;
        const long long q = (long long)X * a.pitch + Z;
        // ---- velocities: vx(X+1), vz(X) (propagate.c:2511-2588, pml.c:39-680) ----
        const C n_txz = F(rc + 1, F_TXZ), c_txz = F(rc, F_TXZ), c_tzz = F(rc, F_TZZ);
        const C c_txx = F(rc, F_TXX);
        const C txz_zm = __shfl_up_sync(full, n_txz, 1);
        const C tzz_zp = __shfl_down_sync(full, c_tzz, 1);
        const C ax = r_sub(F(rc + 1, F_TXX), c_txx), az = r_sub(n_txz, txz_zm);
        const C bx = r_sub(n_txz, c_txz), bz = r_sub(tzz_zp, c_tzz);
        C vxn, vzn;
        if (fast) {
            vxn = r_fma(M(rc + 1, M_B), r_add(ax, az), F(rc + 1, F_VX));
            vzn = r_fma(M(rc, M_BM), r_add(bx, bz), F(rc, F_VZ));
        } else {
            vxn = (X + 1 < a.NX && zin)
                      ? e_vx<S, C>(a, sb, X + 1, Z, F(rc + 1, F_VX), M(rc + 1, M_B), ax, az, sp.vx,
                                   zp, own)
                      : zero;
            vzn = zin ? e_vz<S, C>(a, sb, X, Z, F(rc, F_VZ), M(rc, M_BM), bx, bz, sp.vz, zp, own)
                      : zero;
        }
        // ---- stresses of row X (propagate.c:2590-2670, pml.c:684-1403) ----
        const C vz_zm = __shfl_up_sync(full, vzn, 1);
        const C vx_zp = __shfl_down_sync(full, vxc, 1);
        const C sax = r_sub(vxn, vxc), saz = r_sub(vzn, vz_zm);   // txx, tzz
        const C sbz = r_sub(vx_zp, vxc), sbx = r_sub(vzn, vzp);   // txz
        const C la = M(rc, M_LA), l2m = M(rc, M_L2M), mu = M(rc, M_MU);
        C txx, tzz, txz;
        if (fast || (zin && e_inside(a, X, Z))) {
            txx = r_add(c_txx, r_fma(l2m, sax, r_mul(la, saz)));
            tzz = r_add(c_tzz, r_fma(l2m, saz, r_mul(la, sax)));
            txz = r_fma(mu, r_add(sbz, sbx), c_txz);
        } else if (zin) {
            const C *pr = static_cast<const C *>(a.prof);
            const EisoProf P{a.NX, a.NZ};
            const long long cc = sb + e_pml_index(a, X, Z);
            const C Axh = pr[P.axh() + X], Bxh = pr[P.bxh() + X];
            txx = e_frame<S, C>(a, F_TXX, cc, Axh, Bxh, zp.An, zp.Bn, sp.t[0], sp.t[1], l2m, la,
                                sax, saz, own);
            tzz = e_frame<S, C>(a, F_TZZ, cc, Axh, Bxh, zp.An, zp.Bn, sp.t[2], sp.t[3], la, l2m,
                                sax, saz, own);
            txz = e_frame<S, C>(a, F_TXZ, cc, pr[P.axn() + X], pr[P.bxn() + X], zp.Ah, zp.Bh,
                                sp.t[4], sp.t[5], mu, mu, sbx, sbz, own);
        } else {
            txx = tzz = txz = zero;
        }
        if (own) {
            if (X + 1 < a.NX) St::st(vxo + q + a.pitch, vxn, a.sc[F_VX]);
            St::st(vzo + q, vzn, a.sc[F_VZ]);
            St::st(txxo + q, txx, a.sc[F_TXX]);
            St::st(tzzo + q, tzz, a.sc[F_TZZ]);
            St::st(txzo + q, txz, a.sc[F_TXZ]);
        }
        vxc = vxn;
        vzp = vzn;
        sp = sn;
    }
}

// ---------------------------------------------------------------------------
// Slab step kernel with materials from global memory: the slab kernel with
// only the wavefields in the TMA box (half the shared memory per cell, so
// twice the slabs in flight per SM).  The materials of a slab's rows are read
// from L2 (they are shared by every shot) into registers before the TMA wait,
// so their latency hides behind it.
// ---------------------------------------------------------------------------
template <typename S, int W, int TX>
struct ESlabG {
    static constexpr int HS = 16 / (int)sizeof(S);
    static constexpr int RX = TX + 2;
    static constexpr int BW = (30 * W + 2 + HS - 1 + HS - 1) / HS * HS;
    static constexpr int BWC = 4;   // unused: no materials box
    static constexpr size_t al(size_t x) { return (x + 127) / 128 * 128; }
    static constexpr size_t oBar = al(5 * (size_t)RX * BW * sizeof(S));
    static constexpr size_t bytes = oBar + 16;
    static constexpr unsigned tx = (unsigned)(5 * RX * BW * sizeof(S));
};

// the TMA load of slab (bx, by, shot) into a stage of ESlabG's layout,
// completing on the stage's barrier (thread 0 only)
template <typename S, int W, int TX>
__device__ __forceinline__ void eiso_slabg_issue(const CUtensorMap *fmap, int bx, int by, int shot,
                                                 unsigned char *smem) {
    using L = ESlabG<S, W, TX>;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::oBar);
    const int Zc = bx * W * 30;
    const int zs = (Zc - 1 + L::HS) / L::HS * L::HS - L::HS;
    fence_proxy_async();
    mbar_expect_tx(bar, L::tx);
    tma_load_4d(smem, fmap, zs, by * TX - 1, shot, 0, bar);
}

// the slab step of block (bx, by, shot) of one problem; fmap is the TMA map
// of its old set (box (BW, TX+2, 1, 5)); smem holds ESlabG's layout.
// parity < 0: the slab's own launch (thread 0 initialises the barrier and
// issues the load); parity >= 0: a persistent CTA that issued this stage's
// load earlier and waits for that phase of its barrier
template <typename S, int W, int TX>
__device__ __forceinline__ void eiso_slabg_body(const EisoArgs &a, const CUtensorMap *fmap,
                                                int bx, int by, int shot, unsigned char *smem,
                                                int parity = -1) {
    using C = typename Store<S>::C;
    using St = Store<S>;
    using L = ESlabG<S, W, TX>;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if ((bx | by | shot | threadIdx.x) == 0) ++*a.step;
    const S *fbox = reinterpret_cast<const S *>(smem);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::oBar);
    const int Zc = bx * W * 30;
    const int X0 = by * TX;
    const int X1 = min(X0 + TX, a.NX);
    const int zs = (Zc - 1 + L::HS) / L::HS * L::HS - L::HS;
    const unsigned ph = parity < 0 ? 0u : (unsigned)parity;
    if (parity < 0) {
        if (threadIdx.x == 0) {
            mbar_init(bar, 1);
            fence_proxy_async();
            eiso_slabg_issue<S, W, TX>(fmap, bx, by, shot, smem);
        }
        __syncthreads();   // the barrier is initialised before anyone polls it
    }
    const int Z0 = Zc + warp * 30;
    // warp 0 always has cells and keeps the CTA alive until the copy has
    // landed; later warps past the grid leave
    if (Z0 >= a.NZ) return;
    const int Z = Z0 - 1 + lane;
    const bool zin = Z >= 0 && Z < a.NZ;
    const bool own = lane >= 1 && lane <= 30 && Z < a.NZ;
    const long long fb = (long long)shot * a.fstride;
    const long long sb = (long long)shot * a.sstride;
    const C zero = C(0);
    const int of = Z - zs;
    auto F = [&](int rho, int f) -> C {
        return St::ld(fbox + (f * L::RX + rho) * L::BW + of, a.isc[f]);
    };
    // material m of row X0-1+rho at this lane's cell, zero off the grid (as
    // the TMA box would read it)
    auto M = [&](int rho, int m) -> C {
        const int x = X0 - 1 + rho;
        if (!zin || x < 0 || x >= a.NX) return zero;
        return __ldg(static_cast<const C *>(a.mat[m]) + (long long)x * a.pitch + Z);
    };
    const bool zint = (Z0 - 1 >= a.np) && (Z0 + 30 <= a.np + a.nz - 1);
    const bool lean = zint && X0 >= a.np && X1 <= a.np + a.nx - 1;
    S *const fo0 = static_cast<S *>(a.fo[0]);
    const long long fso = static_cast<S *>(a.fo[1]) - fo0;
    S *vxo = fo0 + F_VX * fso + fb, *vzo = fo0 + F_VZ * fso + fb;
    S *txxo = fo0 + F_TXX * fso + fb, *tzzo = fo0 + F_TZZ * fso + fb, *txzo = fo0 + F_TXZ * fso + fb;

    if (lean) {
        // materials of every row of the slab, read while the box is in flight
        C nb[TX], cbm[TX], cla[TX], cl2m[TX], cmu[TX];
        const C b1 = M(1, M_B), bm0 = M(0, M_BM);
#pragma unroll
        for (int r = 0; r < TX; ++r) {
            nb[r] = M(r + 2, M_B);
            cbm[r] = M(r + 1, M_BM);
            cla[r] = M(r + 1, M_LA);
            cl2m[r] = M(r + 1, M_L2M);
            cmu[r] = M(r + 1, M_MU);
        }
        if (!__all_sync(full, mbar_wait(bar, ph, a.err, 9))) {
            mbar_wait(bar, ph, a.err, 9);
            return;
        }
        C vxc, vzp;
        {
            const C c_txz = F(1, F_TXZ), p_tzz = F(0, F_TZZ);
            const C txz_zm = __shfl_up_sync(full, c_txz, 1);
            const C tzz_zp = __shfl_down_sync(full, p_tzz, 1);
            // interior cells (lean): e_vx / e_vz reduce to their interior branch
            vxc = r_fma(b1, r_add(r_sub(F(1, F_TXX), F(0, F_TXX)), r_sub(c_txz, txz_zm)), F(1, F_VX));
            vzp = zero;
            if (X0 - 1 >= a.np)
                vzp = r_fma(bm0, r_add(r_sub(c_txz, F(0, F_TXZ)), r_sub(tzz_zp, p_tzz)), F(0, F_VZ));
        }
        if (X0 - 1 < a.np) {
            // vz of row X0-1 lies in the frame: the general helper with its split parts
            ESplit<C> sp;
            const EisoProf P{a.NX, a.NZ};
            const C *pr = static_cast<const C *>(a.prof);
            e_load_split<S, C>(a, sb, X0 - 1, Z, zin, sp);
            const EZProf<C> zp{pr[P.azn() + Z], pr[P.bzn() + Z], pr[P.azh() + Z], pr[P.bzh() + Z]};
            const C c_txz = F(1, F_TXZ), p_tzz = F(0, F_TZZ);
            const C tzz_zp = __shfl_down_sync(full, p_tzz, 1);
            vzp = e_vz<S, C>(a, sb, X0 - 1, Z, F(0, F_VZ), bm0, r_sub(c_txz, F(0, F_TXZ)),
                             r_sub(tzz_zp, p_tzz), sp.vz, zp, false);
        }
        long long q = (long long)X0 * a.pitch + Z;
#pragma unroll
        for (int r = 0; r < TX; ++r, q += a.pitch) {
            if (r >= X1 - X0) break;
            const int rc = r + 1;
            const C n_txz = F(rc + 1, F_TXZ), c_txz = F(rc, F_TXZ), c_tzz = F(rc, F_TZZ);
            const C c_txx = F(rc, F_TXX), n_txx = F(rc + 1, F_TXX);
            const C n_vx = F(rc + 1, F_VX), c_vz = F(rc, F_VZ);
            const C txz_zm = __shfl_up_sync(full, n_txz, 1);
            const C tzz_zp = __shfl_down_sync(full, c_tzz, 1);
            const C ax = r_sub(n_txx, c_txx), az = r_sub(n_txz, txz_zm);
            const C bx = r_sub(n_txz, c_txz), bz = r_sub(tzz_zp, c_tzz);
            const C vxn = r_fma(nb[r], r_add(ax, az), n_vx);
            const C vzn = r_fma(cbm[r], r_add(bx, bz), c_vz);
            const C vz_zm = __shfl_up_sync(full, vzn, 1);
            const C vx_zp = __shfl_down_sync(full, vxc, 1);
            const C sax = r_sub(vxn, vxc), saz = r_sub(vzn, vz_zm);
            const C sbz = r_sub(vx_zp, vxc), sbx = r_sub(vzn, vzp);
            const C txx = r_add(c_txx, r_fma(cl2m[r], sax, r_mul(cla[r], saz)));
            const C tzz = r_add(c_tzz, r_fma(cl2m[r], saz, r_mul(cla[r], sax)));
            const C txz = r_fma(cmu[r], r_add(sbz, sbx), c_txz);
            if (own) {
                St::st(vxo + q + a.pitch, vxn, a.sc[F_VX]);
                St::st(vzo + q, vzn, a.sc[F_VZ]);
                St::st(txxo + q, txx, a.sc[F_TXX]);
                St::st(tzzo + q, tzz, a.sc[F_TZZ]);
                St::st(txzo + q, txz, a.sc[F_TXZ]);
            }
            vxc = vxn;
            vzp = vzn;
        }
        return;
    }

    // general march (frame): materials straight from L2
    const C *pr = static_cast<const C *>(a.prof);
    const EisoProf P{a.NX, a.NZ};
    EZProf<C> zp{C(1), C(1), C(1), C(1)};
    if (zin) zp = EZProf<C>{pr[P.azn() + Z], pr[P.bzn() + Z], pr[P.azh() + Z], pr[P.bzh() + Z]};
    ESplit<C> sp;
    e_load_split<S, C>(a, sb, X0 - 1, Z, zin, sp);
    if (!__all_sync(full, mbar_wait(bar, ph, a.err, 9))) {
        mbar_wait(bar, ph, a.err, 9);
        return;
    }
    C vxc, vzp;
    {
        const C c_txz = F(1, F_TXZ), p_tzz = F(0, F_TZZ);
        const C txz_zm = __shfl_up_sync(full, c_txz, 1);
        const C tzz_zp = __shfl_down_sync(full, p_tzz, 1);
        vxc = zin ? e_vx<S, C>(a, sb, X0, Z, F(1, F_VX), M(1, M_B), r_sub(F(1, F_TXX), F(0, F_TXX)),
                               r_sub(c_txz, txz_zm), sp.vx, zp, X0 == 0 && own)
                  : zero;
        if (X0 == 0 && own) St::st(vxo + (long long)X0 * a.pitch + Z, vxc, a.sc[F_VX]);
        vzp = zero;
        if (X0 >= 1 && zin)
            vzp = e_vz<S, C>(a, sb, X0 - 1, Z, F(0, F_VZ), M(0, M_BM), r_sub(c_txz, F(0, F_TXZ)),
                             r_sub(tzz_zp, p_tzz), sp.vz, zp, false);
    }
    e_load_split<S, C>(a, sb, X0, Z, zin, sp);
    for (int X = X0; X < X1; ++X) {
        const int rc = X - X0 + 1;
        ESplit<C> sn;
        e_load_split<S, C>(a, sb, X + 1, Z, zin && X + 1 < X1, sn);
        const bool fast = zint && X >= a.np && X + 1 <= a.np + a.nx - 1;
        const long long q = (long long)X * a.pitch + Z;
        const C n_b = M(rc + 1, M_B), c_bm = M(rc, M_BM);
        const C la = M(rc, M_LA), l2m = M(rc, M_L2M), mu = M(rc, M_MU);
        const C n_txz = F(rc + 1, F_TXZ), c_txz = F(rc, F_TXZ), c_tzz = F(rc, F_TZZ);
        const C c_txx = F(rc, F_TXX);
        const C txz_zm = __shfl_up_sync(full, n_txz, 1);
        const C tzz_zp = __shfl_down_sync(full, c_tzz, 1);
        const C ax = r_sub(F(rc + 1, F_TXX), c_txx), az = r_sub(n_txz, txz_zm);
        const C bx = r_sub(n_txz, c_txz), bz = r_sub(tzz_zp, c_tzz);
        C vxn, vzn;
        if (fast) {
            vxn = r_fma(n_b, r_add(ax, az), F(rc + 1, F_VX));
            vzn = r_fma(c_bm, r_add(bx, bz), F(rc, F_VZ));
        } else {
            vxn = (X + 1 < a.NX && zin)
                      ? e_vx<S, C>(a, sb, X + 1, Z, F(rc + 1, F_VX), n_b, ax, az, sp.vx, zp, own)
                      : zero;
            vzn = zin ? e_vz<S, C>(a, sb, X, Z, F(rc, F_VZ), c_bm, bx, bz, sp.vz, zp, own) : zero;
        }
        const C vz_zm = __shfl_up_sync(full, vzn, 1);
        const C vx_zp = __shfl_down_sync(full, vxc, 1);
        const C sax = r_sub(vxn, vxc), saz = r_sub(vzn, vz_zm);
        const C sbz = r_sub(vx_zp, vxc), sbx = r_sub(vzn, vzp);
        C txx, tzz, txz;
        if (fast || (zin && e_inside(a, X, Z))) {
            txx = r_add(c_txx, r_fma(l2m, sax, r_mul(la, saz)));
            tzz = r_add(c_tzz, r_fma(l2m, saz, r_mul(la, sax)));
            txz = r_fma(mu, r_add(sbz, sbx), c_txz);
        } else if (zin) {
            const long long cc = sb + e_pml_index(a, X, Z);
            const C Axh = pr[P.axh() + X], Bxh = pr[P.bxh() + X];
            txx = e_frame<S, C>(a, F_TXX, cc, Axh, Bxh, zp.An, zp.Bn, sp.t[0], sp.t[1], l2m, la,
                                sax, saz, own);
            tzz = e_frame<S, C>(a, F_TZZ, cc, Axh, Bxh, zp.An, zp.Bn, sp.t[2], sp.t[3], la, l2m,
                                sax, saz, own);
            txz = e_frame<S, C>(a, F_TXZ, cc, pr[P.axn() + X], pr[P.bxn() + X], zp.Ah, zp.Bh,
                                sp.t[4], sp.t[5], mu, mu, sbx, sbz, own);
        } else {
            txx = tzz = txz = zero;
        }
        if (own) {
            if (X + 1 < a.NX) St::st(vxo + q + a.pitch, vxn, a.sc[F_VX]);
            St::st(vzo + q, vzn, a.sc[F_VZ]);
            St::st(txxo + q, txx, a.sc[F_TXX]);
            St::st(tzzo + q, tzz, a.sc[F_TZZ]);
            St::st(txzo + q, txz, a.sc[F_TXZ]);
        }
        vxc = vxn;
        vzp = vzn;
        sp = sn;
    }
}

// Launch order of the slabs: the slab grid is gx (z) x gy (x) per shot, and
// the rectangle [bx0, bx1) x [by0, by1) holds the slabs whose every warp is
// clear of the PML frame (the lean path).  CTA b of the 1-D grid takes the
// rectangle's slabs of every shot first, then the frame's, so the lean
// loop and the frame's general path mostly run on the device at different
// times (one loop's code in the instruction caches at a time).  The order
// changes nothing else: each slab writes only its own cells.
struct SlabOrder {
    int gx, gy, bx0, bx1, by0, by1;
};

__device__ __forceinline__ void slab_of(const SlabOrder &o, int nshots, int b, int &bx, int &by,
                                        int &shot) {
    const int nix = o.bx1 - o.bx0, nin = nix * (o.by1 - o.by0);
    if (b < nin * nshots) {
        shot = b / nin;
        const int r = b - shot * nin;
        bx = o.bx0 + r % nix;
        by = o.by0 + r / nix;
        return;
    }
    b -= nin * nshots;
    const int nring = o.gx * o.gy - nin;
    shot = b / nring;
    int e = b - shot * nring;
    const int top = o.by0 * o.gx;   // rows of slabs before the rectangle
    if (e < top) {
        bx = e % o.gx;
        by = e / o.gx;
        return;
    }
    e -= top;
    const int bot = (o.gy - o.by1) * o.gx;   // ... and after it
    if (e < bot) {
        bx = e % o.gx;
        by = o.by1 + e / o.gx;
        return;
    }
    e -= bot;
    const int nox = o.gx - nix;   // the rectangle's rows: slabs left and right of it
    by = o.by0 + e / nox;
    const int c = e % nox;
    bx = c < o.bx0 ? c : o.bx1 + (c - o.bx0);
}

template <typename S, int W, int TX, int MINB>
__global__ void __launch_bounds__(32 * W, MINB) eiso_slabg_kernel(const EisoArgs a,
                                                                  const __grid_constant__ EisoSlabMaps mp) {
    extern __shared__ __align__(128) unsigned char smem[];
    eiso_slabg_body<S, W, TX>(a, &mp.f, blockIdx.x, blockIdx.y, blockIdx.z, smem);
}

// Persistent form of the slab step: a CTA per SM slot walks the slabs
// s = blockIdx.x, + gridDim.x, ... (s -> bx fastest, then by, then shot)
// through two shared-memory stages, the next slab's box in flight while the
// current one computes.
template <typename S, int W, int TX, int MINB>
__global__ void __launch_bounds__(32 * W, MINB)
    eiso_slabg_pkernel(const EisoArgs a, const __grid_constant__ EisoSlabMaps mp, int gx, int gy,
                       int nslab) {
    using L = ESlabG<S, W, TX>;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *stage[2] = {smem, smem + L::al(L::bytes)};
    if (threadIdx.x == 0) {
        mbar_init(reinterpret_cast<uint64_t *>(stage[0] + L::oBar), 1);
        mbar_init(reinterpret_cast<uint64_t *>(stage[1] + L::oBar), 1);
        fence_proxy_async();
    }
    __syncthreads();
    auto coords = [&](int s, int &bx, int &by, int &shot) {
        bx = s % gx;
        const int r = s / gx;
        by = r % gy;
        shot = r / gy;
    };
    int bx, by, shot;
    if (threadIdx.x == 0 && (int)blockIdx.x < nslab) {
        coords(blockIdx.x, bx, by, shot);
        eiso_slabg_issue<S, W, TX>(&mp.f, bx, by, shot, stage[0]);
    }
    int k = 0;
    for (int s = blockIdx.x; s < nslab; s += gridDim.x, ++k) {
        const int sn = s + gridDim.x;
        if (threadIdx.x == 0 && sn < nslab) {   // its stage was released at the last sync
            coords(sn, bx, by, shot);
            eiso_slabg_issue<S, W, TX>(&mp.f, bx, by, shot, stage[(k + 1) & 1]);
        }
        coords(s, bx, by, shot);
        eiso_slabg_body<S, W, TX>(a, &mp.f, bx, by, shot, stage[k & 1], (k >> 1) & 1);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Block-floating-point slab step (SM_BFP16).  The slab step above with the
// five wavefields stored as 16-bit mantissas sharing one exponent byte per
// block of EB consecutive x rows of one z column ([field][shot][nxb][pitch]
// bytes, nxb = ceil(NX / EB)); the frame's split parts and the materials
// stay FP32 and the arithmetic is the FP32 path's.  A warp's lane marches
// one z column down the slab, so each block is held by one thread: its
// exponent is the maximum over that thread's registers, no exchange across
// lanes.  The slab owns the rows [X0, X0 + TX) of every field, vx included
// (the FP32 slab step stores vx one row down, X0+1 .. X0+TX: a vx block
// would then straddle two CTAs); vx(X0) is the value the neighbouring slab
// computes too, bit for bit.  The stress update reads the unrounded
// velocities of the step; only the state the step stores is rounded.
// ---------------------------------------------------------------------------
#define EISO_EB 4
// Source patches: near a source the wavefield is many times larger than
// anywhere else and changes by orders of magnitude within a few cells, so the
// rounding of 16-bit block storage there (2^-16 of the block's largest value
// per step) radiates noise that dominates the traces of nearby receivers.
// Block storage therefore keeps the cells around each source in FP32: a
// patch of EISO_PR x rows (whole blocks, EISO_PB blocks on each side of the
// source's block) by EISO_PC z columns centred on the source, one per source
// (patches of a shot are disjoint; a source inside or next to another's patch
// gets none).  The patch's values live in a side array of the buffer set;
// the mantissas of those cells are written too (a state without its patches
// is still a valid rounded state).
#define EISO_PB 2
#define EISO_PR (EISO_EB * (2 * EISO_PB + 1))
#define EISO_PZ 4
#define EISO_PC (2 * EISO_PZ + 1)
#define EISO_PF (EISO_PR * EISO_PC)   // values per field of a patch

struct EisoBMaps {
    CUtensorMap f;   // mantissas of the old set: (z, x, shot, field), box (BW, TX+2, 1, 5)
    CUtensorMap e;   // exponents of the old set: (z, xblock, shot, field), box (BWE, TX/EB+2, 1, 5)
};

template <int W, int TX>
struct ESlabB {
    static_assert(TX % EISO_EB == 0, "slab rows must be whole blocks");
    static constexpr int HS = 8;                 // 16 bytes of int16
    static constexpr int RX = TX + 2;
    static constexpr int NB = TX / EISO_EB + 2;  // blocks in the box: above, own, below
    static constexpr int BW = (30 * W + 2 + HS - 1 + HS - 1) / HS * HS;
    static constexpr int BWE = (30 * W + 17 + 15) / 16 * 16;   // bytes, start rounded to 16
    static_assert(BW <= 256 && BWE <= 256, "TMA box dimension");
    static constexpr size_t al(size_t x) { return (x + 127) / 128 * 128; }
    static constexpr size_t oE = al(5 * (size_t)RX * BW * 2);
    static constexpr size_t oStg = oE + al(5 * (size_t)NB * BWE);   // [5][EB][threads] floats
    static constexpr size_t oBar = oStg + al(5 * (size_t)EISO_EB * 32 * W * 4);
    static constexpr size_t bytes = oBar + 16;
    static constexpr unsigned tx = (unsigned)(5 * RX * BW * 2 + 5 * NB * BWE);
};

// the two TMA loads of slab (bx, by, shot) into a stage of ESlabB's layout,
// completing on the stage's barrier (thread 0 only)
template <int W, int TX>
__device__ __forceinline__ void eiso_bslab_issue(const CUtensorMap *fmap, const CUtensorMap *emap,
                                                 int bx, int by, int shot, unsigned char *smem) {
    using L = ESlabB<W, TX>;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::oBar);
    const int Zc = bx * W * 30, X0 = by * TX;
    const int zs = (Zc - 1 + L::HS) / L::HS * L::HS - L::HS;
    const int zse = (Zc - 1 + 16) / 16 * 16 - 16;
    fence_proxy_async();
    mbar_expect_tx(bar, L::tx);
    tma_load_4d(smem, fmap, zs, X0 - 1, shot, 0, bar);
    tma_load_4d(smem + L::oE, emap, zse, X0 / EISO_EB - 1, shot, 0, bar);
}

// One slab.  parity < 0: the slab's own launch (thread 0 initialises the
// barrier and issues the loads); parity >= 0: a persistent CTA that issued
// this stage's loads earlier and waits for that phase of its barrier.
template <int W, int TX>
__device__ __forceinline__ void eiso_bslab_body(const EisoArgs &a, const CUtensorMap *fmap,
                                                const CUtensorMap *emap, int bx, int by, int shot,
                                                unsigned char *smem, int parity = -1) {
    using C = float;
    using L = ESlabB<W, TX>;
    constexpr int EB = EISO_EB;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if ((bx | by | shot | threadIdx.x) == 0) ++*a.step;
    const int16_t *fbox = reinterpret_cast<const int16_t *>(smem);
    const uint8_t *ebox = smem + L::oE;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::oBar);
    const int Zc = bx * W * 30;
    const int X0 = by * TX;
    const int X1 = min(X0 + TX, a.NX);
    const int zs = (Zc - 1 + L::HS) / L::HS * L::HS - L::HS;
    const int zse = (Zc - 1 + 16) / 16 * 16 - 16;
    const int xb0 = X0 / EB;
    const unsigned ph = parity < 0 ? 0u : (unsigned)parity;
    if (parity < 0) {
        if (threadIdx.x == 0) {
            mbar_init(bar, 1);
            fence_proxy_async();
            eiso_bslab_issue<W, TX>(fmap, emap, bx, by, shot, smem);
        }
        __syncthreads();
    }
    const int Z0 = Zc + warp * 30;
    if (Z0 >= a.NZ) return;
    const int Z = Z0 - 1 + lane;
    const bool zin = Z >= 0 && Z < a.NZ;
    const bool own = lane >= 1 && lane <= 30 && Z < a.NZ;
    const long long fb = (long long)shot * a.fstride;
    const long long sb = (long long)shot * a.sstride;
    const C zero = C(0);
    const int of = Z - zs, oe = Z - zse;
    // this lane's source patch (the one whose columns hold Z and whose rows
    // meet the box), -1 if none; cta_patch: the box meets any patch of the shot
    int lp = -1, lpx = 0, lpz = 0;
    bool cta_patch = false;
    if (a.pfirst) {
        for (int q = a.pfirst[shot]; q < a.pfirst[shot + 1]; ++q) {
            const int px = a.pxz[2 * q], pz = a.pxz[2 * q + 1];
            const bool rows = px <= X0 + TX && px + EISO_PR > X0 - 1;
            cta_patch = cta_patch || (rows && pz <= Zc + 30 * W && pz + EISO_PC > Zc - 1);
            if (rows && Z >= pz && Z < pz + EISO_PC) { lp = q; lpx = px; lpz = pz; }
        }
    }
    auto in_patch = [&](int X) { return lp >= 0 && X >= lpx && X < lpx + EISO_PR; };
    auto pidx = [&](int f, int X) {
        return ((long long)lp * 5 + f) * EISO_PF + (X - lpx) * EISO_PC + (Z - lpz);
    };
    // decoder of field f's block b of the box (0: the block holding row
    // X0-1; 1 .. TX/EB: the slab's own; TX/EB+1: the block holding X0+TX)
    auto DE = [&](int f, int b) -> BDec { return bfp_dec(ebox[(f * L::NB + b) * L::BWE + oe]); };
    auto blk = [&](int rho) { return rho == 0 ? 0 : (rho > TX ? L::NB - 1 : (rho - 1) / EB + 1); };
    auto F = [&](int rho, int f) -> C {
        return bfp_val(fbox[(f * L::RX + rho) * L::BW + of], DE(f, blk(rho)));
    };
    auto M = [&](int rho, int m) -> C {
        const int x = X0 - 1 + rho;
        if (!zin || x < 0 || x >= a.NX) return zero;
        return __ldg(static_cast<const C *>(a.mat[m]) + (long long)x * a.pitch + Z);
    };
    const bool zint = (Z0 - 1 >= a.np) && (Z0 + 30 <= a.np + a.nz - 1);
    const bool lean = zint && X0 >= a.np && X1 <= a.np + a.nx - 1 && !cta_patch;
    int16_t *const fo0 = static_cast<int16_t *>(a.fo[0]);
    const long long fso = static_cast<int16_t *>(a.fo[1]) - fo0;
    uint8_t *const eo0 = static_cast<uint8_t *>(a.feo) + (long long)shot * a.nxb * a.pitch + Z;
    // store block q (rows X0 + EB q ..) of field f from v[EB]; rows past the
    // grid's end (vmask false) are left out of the exponent and not stored
    bool overflow = false;   // a block beyond the format's range (reported once)
    auto store_block = [&](int f, int q, const C *v, const bool *vm) {
        unsigned mx = 0;
#pragma unroll
        for (int t = 0; t < EB; ++t) mx = vm[t] ? max(mx, bfp_absbits(v[t])) : mx;
        bool over;
        const unsigned e8 = bfp_e8(mx, &over);
        const float esc = bfp_escale(e8);
        int16_t *o = fo0 + f * fso + fb + (long long)(X0 + EB * q) * a.pitch + Z;
#pragma unroll
        for (int t = 0; t < EB; ++t)
            if (vm[t]) o[(long long)t * a.pitch] = bfp_man(v[t], esc);
        if (vm[0])   // a lane that owns the column and a block inside the grid
            eo0[(long long)f * a.estride + (long long)(xb0 + q) * a.pitch] = (uint8_t)e8;
        overflow = overflow || (vm[0] && over);
    };

    if (lean) {
        // the lean slab lies inside the grid (rows X0-1 .. X0+TX, every lane's
        // column): materials by unchecked loads from row pointers
        const long long mrow = (long long)(X0 - 1) * a.pitch + Z;
        const C *mB = static_cast<const C *>(a.mat[M_B]) + mrow;
        const C *mBM = static_cast<const C *>(a.mat[M_BM]) + mrow;
        const C *mLA = static_cast<const C *>(a.mat[M_LA]) + mrow;
        const C *mL2M = static_cast<const C *>(a.mat[M_L2M]) + mrow;
        const C *mMU = static_cast<const C *>(a.mat[M_MU]) + mrow;
        C nb[TX], cbm[TX], cla[TX], cl2m[TX], cmu[TX];
        const C b1 = __ldg(mB + a.pitch), bm0 = __ldg(mBM);
#pragma unroll
        for (int r = 0; r < TX; ++r) {
            nb[r] = __ldg(mB + (long long)(r + 2) * a.pitch);
            cbm[r] = __ldg(mBM + (long long)(r + 1) * a.pitch);
            cla[r] = __ldg(mLA + (long long)(r + 1) * a.pitch);
            cl2m[r] = __ldg(mL2M + (long long)(r + 1) * a.pitch);
            cmu[r] = __ldg(mMU + (long long)(r + 1) * a.pitch);
        }
        if (!__all_sync(full, mbar_wait(bar, ph, a.err, 9))) {
            mbar_wait(bar, ph, a.err, 9);
            return;
        }
        // each value decoded once; a field's decoder is taken when the march
        // enters the block (TXZ, TXX, VX are read one row ahead of TZZ, VZ)
        auto FVd = [&](int rho, int f, const BDec &d) -> C {
            return bfp_val(fbox[(f * L::RX + rho) * L::BW + of], d);
        };
        auto FV = [&](int rho, int f) -> C { return FVd(rho, f, DE(f, blk(rho))); };
        C vxc, vzp;
        C c_txz = FV(1, F_TXZ), c_txx = FV(1, F_TXX);
        {
            const C p_tzz = FV(0, F_TZZ);
            const C txz_zm = __shfl_up_sync(full, c_txz, 1);
            const C tzz_zp = __shfl_down_sync(full, p_tzz, 1);
            vxc = r_fma(b1, r_add(r_sub(c_txx, FV(0, F_TXX)), r_sub(c_txz, txz_zm)), FV(1, F_VX));
            vzp = zero;
            if (X0 - 1 >= a.np)
                vzp = r_fma(bm0, r_add(r_sub(c_txz, FV(0, F_TXZ)), r_sub(tzz_zp, p_tzz)), FV(0, F_VZ));
            if (X0 - 1 < a.np) {
                ESplit<C> sp;
                const EisoProf P{a.NX, a.NZ};
                const C *pr = static_cast<const C *>(a.prof);
                e_load_split<float, C>(a, sb, X0 - 1, Z, zin, sp);
                const EZProf<C> zp{pr[P.azn() + Z], pr[P.bzn() + Z], pr[P.azh() + Z], pr[P.bzh() + Z]};
                vzp = e_vz<float, C>(a, sb, X0 - 1, Z, FV(0, F_VZ), bm0, r_sub(c_txz, FV(0, F_TXZ)),
                                     r_sub(tzz_zp, p_tzz), sp.vz, zp, false);
            }
        }
        const bool vm[EB] = {own, own, own, own};
        C bvx[EB], bvz[EB], btxx[EB], btzz[EB], btxz[EB];
        bvx[0] = vxc;
        BDec dn[3], dc[2];   // decoders of TXZ, TXX, VX at row rc + 1; TZZ, VZ at row rc
#pragma unroll
        for (int r = 0; r < TX; ++r) {
            const int rc = r + 1;
            if (r == 0 || blk(rc + 1) != blk(rc)) {
                dn[0] = DE(F_TXZ, blk(rc + 1));
                dn[1] = DE(F_TXX, blk(rc + 1));
                dn[2] = DE(F_VX, blk(rc + 1));
            }
            if (r == 0 || blk(rc) != blk(rc - 1)) {
                dc[0] = DE(F_TZZ, blk(rc));
                dc[1] = DE(F_VZ, blk(rc));
            }
            const C n_txz = FVd(rc + 1, F_TXZ, dn[0]), n_txx = FVd(rc + 1, F_TXX, dn[1]);
            const C n_vx = FVd(rc + 1, F_VX, dn[2]);
            const C c_tzz = FVd(rc, F_TZZ, dc[0]), c_vz = FVd(rc, F_VZ, dc[1]);
            const C txz_zm = __shfl_up_sync(full, n_txz, 1);
            const C tzz_zp = __shfl_down_sync(full, c_tzz, 1);
            const C ax = r_sub(n_txx, c_txx), az = r_sub(n_txz, txz_zm);
            const C bx_ = r_sub(n_txz, c_txz), bz = r_sub(tzz_zp, c_tzz);
            const C vxn = r_fma(nb[r], r_add(ax, az), n_vx);
            const C vzn = r_fma(cbm[r], r_add(bx_, bz), c_vz);
            const C vz_zm = __shfl_up_sync(full, vzn, 1);
            const C vx_zp = __shfl_down_sync(full, vxc, 1);
            const C sax = r_sub(vxn, vxc), saz = r_sub(vzn, vz_zm);
            const C sbz = r_sub(vx_zp, vxc), sbx = r_sub(vzn, vzp);
            const int t = r % EB;
            bvz[t] = vzn;
            btxx[t] = r_add(c_txx, r_fma(cl2m[r], sax, r_mul(cla[r], saz)));
            btzz[t] = r_add(c_tzz, r_fma(cl2m[r], saz, r_mul(cla[r], sax)));
            btxz[t] = r_fma(cmu[r], r_add(sbz, sbx), c_txz);
            if (t == EB - 1) {
                const int q = r / EB;
                store_block(F_VX, q, bvx, vm);
                store_block(F_VZ, q, bvz, vm);
                store_block(F_TXX, q, btxx, vm);
                store_block(F_TZZ, q, btzz, vm);
                store_block(F_TXZ, q, btxz, vm);
                bvx[0] = vxn;
            } else {
                bvx[t + 1] = vxn;
            }
            vxc = vxn;
            vzp = vzn;
            c_txz = n_txz;
            c_txx = n_txx;
        }
        if (overflow) atomicExch(a.err, 4);
        return;
    }

    // general march (the frame, the grid's ends and source patches): one
    // row per iteration, not unrolled (the frame's code is long), the
    // values of a block staged per thread in shared memory until the
    // block's last row; split parts FP32 as in the other precisions; cells
    // of a source patch read and write their FP32 values
    float *stg = reinterpret_cast<float *>(smem + L::oStg) + threadIdx.x;
    auto S_ = [&](int f, int t) -> float & { return stg[(f * EB + t) * 32 * W]; };
    auto Fg = [&](int rho, int f) -> C {   // rho known at run time
        const int X = X0 - 1 + rho;
        if (in_patch(X)) return a.pv[pidx(f, X)];
        return bfp_val(fbox[(f * L::RX + rho) * L::BW + of], DE(f, blk(rho)));
    };
    // the block of rows X0 + EB q .. (the first n of them in the grid) of
    // every field, from the staged values
    auto store_staged = [&](int q, int n) {
        const int Xb = X0 + EB * q;
        const bool pb = in_patch(Xb);
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            C v[EB];
            bool vm[EB];
#pragma unroll
            for (int t = 0; t < EB; ++t) {
                v[t] = S_(f, t);
                vm[t] = own && t < n;
            }
            store_block(f, q, v, vm);
            if (pb && own)
                for (int t = 0; t < n; ++t) a.pvo[pidx(f, Xb + t)] = v[t];
        }
    };
    const C *pr = static_cast<const C *>(a.prof);
    const EisoProf P{a.NX, a.NZ};
    EZProf<C> zp{C(1), C(1), C(1), C(1)};
    if (zin) zp = EZProf<C>{pr[P.azn() + Z], pr[P.bzn() + Z], pr[P.azh() + Z], pr[P.bzh() + Z]};
    ESplit<C> sp;
    e_load_split<float, C>(a, sb, X0 - 1, Z, zin, sp);
    if (!__all_sync(full, mbar_wait(bar, ph, a.err, 9))) {
        mbar_wait(bar, ph, a.err, 9);
        return;
    }
    C vxc, vzp;
    {
        const C c_txz = Fg(1, F_TXZ), p_tzz = Fg(0, F_TZZ);
        const C txz_zm = __shfl_up_sync(full, c_txz, 1);
        const C tzz_zp = __shfl_down_sync(full, p_tzz, 1);
        // vx(X0) is this slab's row: its split parts are stored here
        vxc = zin ? e_vx<float, C>(a, sb, X0, Z, Fg(1, F_VX), M(1, M_B),
                                   r_sub(Fg(1, F_TXX), Fg(0, F_TXX)), r_sub(c_txz, txz_zm), sp.vx,
                                   zp, own)
                  : zero;
        vzp = zero;
        if (X0 >= 1 && zin)
            vzp = e_vz<float, C>(a, sb, X0 - 1, Z, Fg(0, F_VZ), M(0, M_BM),
                                 r_sub(c_txz, Fg(0, F_TXZ)), r_sub(tzz_zp, p_tzz), sp.vz, zp,
                                 false);
    }
    S_(F_VX, 0) = vxc;
    e_load_split<float, C>(a, sb, X0, Z, zin, sp);
#pragma unroll 1
    for (int X = X0; X < X1; ++X) {
        const int r = X - X0, rc = r + 1, t = r % EB;
        ESplit<C> sn;
        e_load_split<float, C>(a, sb, X + 1, Z, zin && X + 1 < X1, sn);
        const bool fast = zint && X >= a.np && X + 1 <= a.np + a.nx - 1;
        const C n_b = M(rc + 1, M_B), c_bm = M(rc, M_BM);
        const C la = M(rc, M_LA), l2m = M(rc, M_L2M), mu = M(rc, M_MU);
        const C n_txz = Fg(rc + 1, F_TXZ), c_txz = Fg(rc, F_TXZ), c_tzz = Fg(rc, F_TZZ);
        const C c_txx = Fg(rc, F_TXX);
        const C txz_zm = __shfl_up_sync(full, n_txz, 1);
        const C tzz_zp = __shfl_down_sync(full, c_tzz, 1);
        const C ax = r_sub(Fg(rc + 1, F_TXX), c_txx), az = r_sub(n_txz, txz_zm);
        const C bx_ = r_sub(n_txz, c_txz), bz = r_sub(tzz_zp, c_tzz);
        C vxn, vzn;
        if (fast) {
            vxn = r_fma(n_b, r_add(ax, az), Fg(rc + 1, F_VX));
            vzn = r_fma(c_bm, r_add(bx_, bz), Fg(rc, F_VZ));
        } else {
            // vx(X+1) belongs to this slab when X+1 < X1 (its split parts
            // are stored then); the last row's is the next slab's
            vxn = (X + 1 < a.NX && zin)
                      ? e_vx<float, C>(a, sb, X + 1, Z, Fg(rc + 1, F_VX), n_b, ax, az, sp.vx, zp,
                                       own && X + 1 < X1)
                      : zero;
            vzn = zin ? e_vz<float, C>(a, sb, X, Z, Fg(rc, F_VZ), c_bm, bx_, bz, sp.vz, zp, own)
                      : zero;
        }
        const C vz_zm = __shfl_up_sync(full, vzn, 1);
        const C vx_zp = __shfl_down_sync(full, vxc, 1);
        const C sax = r_sub(vxn, vxc), saz = r_sub(vzn, vz_zm);
        const C sbz = r_sub(vx_zp, vxc), sbx = r_sub(vzn, vzp);
        C txx = zero, tzz = zero, txz = zero;
        if (fast || (zin && e_inside(a, X, Z))) {
            txx = r_add(c_txx, r_fma(l2m, sax, r_mul(la, saz)));
            tzz = r_add(c_tzz, r_fma(l2m, saz, r_mul(la, sax)));
            txz = r_fma(mu, r_add(sbz, sbx), c_txz);
        } else if (zin) {
            const long long cc = sb + e_pml_index(a, X, Z);
            const C Axh = pr[P.axh() + X], Bxh = pr[P.bxh() + X];
            txx = e_frame<float, C>(a, F_TXX, cc, Axh, Bxh, zp.An, zp.Bn, sp.t[0], sp.t[1], l2m, la,
                                    sax, saz, own);
            tzz = e_frame<float, C>(a, F_TZZ, cc, Axh, Bxh, zp.An, zp.Bn, sp.t[2], sp.t[3], la, l2m,
                                    sax, saz, own);
            txz = e_frame<float, C>(a, F_TXZ, cc, pr[P.axn() + X], pr[P.bxn() + X], zp.Ah, zp.Bh,
                                    sp.t[4], sp.t[5], mu, mu, sbx, sbz, own);
        }
        S_(F_VZ, t) = vzn;
        S_(F_TXX, t) = txx;
        S_(F_TZZ, t) = tzz;
        S_(F_TXZ, t) = txz;
        if (t == EB - 1 || X + 1 == X1) {   // uniform across the CTA
            store_staged(r / EB, t + 1);
            S_(F_VX, 0) = vxn;   // the next block's first row
        } else {
            S_(F_VX, t + 1) = vxn;
        }
        vxc = vxn;
        vzp = vzn;
        sp = sn;
    }
    if (overflow) atomicExch(a.err, 4);
}

template <int W, int TX, int MINB>
__global__ void __launch_bounds__(32 * W, MINB) eiso_bslab_kernel(const EisoArgs a,
                                                                  const __grid_constant__ EisoBMaps mp,
                                                                  const SlabOrder o) {
    extern __shared__ __align__(128) unsigned char smem[];
    int bx, by, shot;
    slab_of(o, a.nshots, blockIdx.x, bx, by, shot);
    eiso_bslab_body<W, TX>(a, &mp.f, &mp.e, bx, by, shot, smem);
}

// Persistent form: a CTA per SM slot walks the slabs s = blockIdx.x,
// + gridDim.x, ... (s -> bx fastest, then by, then shot) through two shared-
// memory stages: the next slab's boxes are in flight while the current slab
// computes, so the load latency no longer stands between slabs.
template <int W, int TX, int MINB>
__global__ void __launch_bounds__(32 * W, MINB)
    eiso_bslab_pkernel(const EisoArgs a, const __grid_constant__ EisoBMaps mp, int gx, int gy,
                       int nslab) {
    using L = ESlabB<W, TX>;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *stage[2] = {smem, smem + L::al(L::bytes)};
    if (threadIdx.x == 0) {
        mbar_init(reinterpret_cast<uint64_t *>(stage[0] + L::oBar), 1);
        mbar_init(reinterpret_cast<uint64_t *>(stage[1] + L::oBar), 1);
        fence_proxy_async();
    }
    __syncthreads();
    auto coords = [&](int s, int &bx, int &by, int &shot) {
        bx = s % gx;
        const int r = s / gx;
        by = r % gy;
        shot = r / gy;
    };
    int bx, by, shot;
    if (threadIdx.x == 0 && (int)blockIdx.x < nslab) {
        coords(blockIdx.x, bx, by, shot);
        eiso_bslab_issue<W, TX>(&mp.f, &mp.e, bx, by, shot, stage[0]);
    }
    int k = 0;
    for (int s = blockIdx.x; s < nslab; s += gridDim.x, ++k) {
        const int sn = s + gridDim.x;
        if (threadIdx.x == 0 && sn < nslab) {   // its stage was released at the last sync
            coords(sn, bx, by, shot);
            eiso_bslab_issue<W, TX>(&mp.f, &mp.e, bx, by, shot, stage[(k + 1) & 1]);
        }
        coords(s, bx, by, shot);
        eiso_bslab_body<W, TX>(a, &mp.f, &mp.e, bx, by, shot, stage[k & 1], (k >> 1) & 1);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Tiled step kernel: one CTA updates a TX x TZ tile of one shot for a whole
// time step (e_iso.c:595-636).  The five old wavefields of rows X0-1 ..
// X0+TX and z cells Z0-HS .. Z0+TZ+HS-1 arrive by TMA (out-of-grid cells read
// as zero, which is the reference's boundary).  Phase 1 computes vx on
// [X0, X0+TX] x [Z0, Z0+TZ] and vz on [X0-1, X0+TX-1] x [Z0-1, Z0+TZ-1]
// into shared memory (the halo is recomputed by the neighbouring CTA
// bitwise, since the arithmetic is the same); phase 2 computes the stresses
// of the tile from them.  Only cells of the tile are written (ping-pong
// sets), and split parts of frame cells likewise.  Materials are read with
// plain loads, issued before the TMA wait: they are shared by every shot
// and stay in L2.
// ---------------------------------------------------------------------------
struct EisoMaps {
    CUtensorMap f[5];   // the old set's wavefields: (z, x, shot), box (BZ, TX+2, 1)
};

template <typename S, int TX, int TZ>
struct ETile {
    using C = typename Store<S>::C;
    static constexpr int HS = 16 / (int)sizeof(S);   // cells per 16 bytes
    static constexpr int BZ = TZ + 2 * HS;            // box width (z cells)
    static constexpr int RX = TX + 2;                 // box height (rows)
    static constexpr int VP = TZ + 1;                 // velocity tile pitch
    static constexpr int NVP = (TX + 1) * (TZ + 1);   // velocity points
    static constexpr size_t al(size_t x) { return (x + 127) / 128 * 128; }
    static constexpr size_t FB = (size_t)RX * BZ * sizeof(S);   // one field's box
    static constexpr size_t FS = al(FB);                          // its slot (128-aligned)
    static constexpr size_t oV = 5 * FS;
    static constexpr size_t oBar = al(oV + 2 * (size_t)NVP * sizeof(C));
    static constexpr size_t bytes = oBar + 16;
    static constexpr unsigned tx = (unsigned)(5 * FB);
};

template <typename S, int TX, int TZ, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) eiso_tile_kernel(const EisoArgs a,
                                                             const __grid_constant__ EisoMaps mp) {
    using C = typename Store<S>::C;
    using St = Store<S>;
    using L = ETile<S, TX, TZ>;
    constexpr int NV = (L::NVP + NT - 1) / NT;
    constexpr int NS = (TX * TZ + NT - 1) / NT;
    extern __shared__ __align__(128) unsigned char smem[];
    C *vxs = reinterpret_cast<C *>(smem + L::oV);
    C *vzs = vxs + L::NVP;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::oBar);
    const int tid = threadIdx.x;
    if ((blockIdx.x | blockIdx.y | blockIdx.z | tid) == 0) ++*a.step;
    const int Z0 = blockIdx.x * TZ, X0 = blockIdx.y * TX, shot = blockIdx.z;
    const long long fb = (long long)shot * a.fstride;
    const long long sb = (long long)shot * a.sstride;

    if (tid == 0) {
        mbar_init(bar, 1);
        fence_proxy_async();
        mbar_expect_tx(bar, L::tx);
#pragma unroll
        for (int f = 0; f < 5; ++f)
            tma_load_3d(smem + f * L::FS, &mp.f[f], Z0 - L::HS, X0 - 1, shot, bar);
    }
    // materials of this thread's points while the tile is in flight
    const C *mat_b = static_cast<const C *>(a.mat[M_B]);
    const C *mat_bm = static_cast<const C *>(a.mat[M_BM]);
    C mb[NV], mbm[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const int i = tid + j * NT;
        mb[j] = mbm[j] = C(0);
        if (i < L::NVP) {
            const int r = i / (TZ + 1), k = i % (TZ + 1);
            const int X = X0 + r, Z = Z0 + k;          // vx point
            if (X < a.NX && Z < a.NZ) mb[j] = mat_b[(long long)X * a.pitch + Z];
            const int Xz = X - 1, Zz = Z - 1;          // vz point
            if (Xz >= 0 && Xz < a.NX && Zz >= 0 && Zz < a.NZ)
                mbm[j] = mat_bm[(long long)Xz * a.pitch + Zz];
        }
    }
    C la[NS], l2m[NS], mu[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        const int i = tid + j * NT;
        la[j] = l2m[j] = mu[j] = C(0);
        const int X = X0 + i / TZ, Z = Z0 + i % TZ;
        if (i < TX * TZ && X < a.NX && Z < a.NZ) {
            const long long q = (long long)X * a.pitch + Z;
            la[j] = static_cast<const C *>(a.mat[M_LA])[q];
            l2m[j] = static_cast<const C *>(a.mat[M_L2M])[q];
            mu[j] = static_cast<const C *>(a.mat[M_MU])[q];
        }
    }
    __syncthreads();   // barrier initialised before anyone polls it
    if (!mbar_wait(bar, 0, a.err, 2)) {
        mbar_wait(bar, 0, a.err, 2);   // give copies in flight a last bounded chance
        return;
    }
    // field f at (X, Z), X in [X0-1, X0+TX], Z in [Z0-HS, Z0+TZ+HS)
    auto F = [&](int f, int X, int Z) -> C {
        return St::ld(reinterpret_cast<const S *>(smem + f * L::FS) + (X - X0 + 1) * L::BZ +
                          (Z - Z0 + L::HS),
                      a.isc[f]);
    };
    // the tile and its halo lie inside the interior update region
    const bool tint = X0 - 1 >= a.np && X0 + TX <= a.np + a.nx - 1 && Z0 - 1 >= a.np &&
                      Z0 + TZ <= a.np + a.nz - 1;
    const EisoProf P{a.NX, a.NZ};
    const C *pr = static_cast<const C *>(a.prof);
    S *vxo = static_cast<S *>(a.fo[F_VX]) + fb;
    S *vzo = static_cast<S *>(a.fo[F_VZ]) + fb;

    // ---- phase 1: velocities (propagate.c:2511-2588, pml.c:39-680) ----
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const int i = tid + j * NT;
        if (i >= L::NVP) break;
        const int r = i / (TZ + 1), k = i % (TZ + 1);
        {   // vx at (X, Z)
            const int X = X0 + r, Z = Z0 + k;
            C v = C(0);
            if (X < a.NX && Z < a.NZ) {
                const C ax = r_sub(F(F_TXX, X, Z), F(F_TXX, X - 1, Z));
                const C az = r_sub(F(F_TXZ, X, Z), F(F_TXZ, X, Z - 1));
                const C vold = F(F_VX, X, Z);
                if (tint || e_inside(a, X, Z)) {
                    v = r_fma(mb[j], r_add(ax, az), vold);
                } else {
                    const long long c = sb + e_pml_index(a, X, Z);
                    const bool own = X < X0 + TX && Z < Z0 + TZ;
                    v = e_frame<S, C>(a, F_VX, c, pr[P.axn() + X], pr[P.bxn() + X],
                                      pr[P.azn() + Z], pr[P.bzn() + Z],
                                      St::ld(static_cast<const S *>(a.fx[F_VX]) + c, a.isc[F_VX]),
                                      St::ld(static_cast<const S *>(a.fz[F_VX]) + c, a.isc[F_VX]),
                                      mb[j], mb[j], ax, az, own);
                }
                if (X < X0 + TX && Z < Z0 + TZ)
                    St::st(vxo + (long long)X * a.pitch + Z, v, a.sc[F_VX]);
            }
            vxs[r * L::VP + k] = v;
        }
        {   // vz at (X + 1/2, Z + 1/2), X = X0 - 1 + r, Z = Z0 - 1 + k
            const int X = X0 - 1 + r, Z = Z0 - 1 + k;
            C v = C(0);
            if (X >= 0 && X < a.NX && Z >= 0 && Z < a.NZ) {
                const C bx = r_sub(F(F_TXZ, X + 1, Z), F(F_TXZ, X, Z));
                const C bz = r_sub(F(F_TZZ, X, Z + 1), F(F_TZZ, X, Z));
                const C vold = F(F_VZ, X, Z);
                if (tint || e_inside(a, X, Z)) {
                    v = r_fma(mbm[j], r_add(bx, bz), vold);
                } else {
                    const long long c = sb + e_pml_index(a, X, Z);
                    const bool own = X >= X0 && Z >= Z0;
                    v = e_frame<S, C>(a, F_VZ, c, pr[P.axh() + X], pr[P.bxh() + X],
                                      pr[P.azh() + Z], pr[P.bzh() + Z],
                                      St::ld(static_cast<const S *>(a.fx[F_VZ]) + c, a.isc[F_VZ]),
                                      St::ld(static_cast<const S *>(a.fz[F_VZ]) + c, a.isc[F_VZ]),
                                      mbm[j], mbm[j], bx, bz, own);
                }
                if (X >= X0 && Z >= Z0) St::st(vzo + (long long)X * a.pitch + Z, v, a.sc[F_VZ]);
            }
            vzs[r * L::VP + k] = v;
        }
    }
    __syncthreads();

    // ---- phase 2: stresses of the tile (propagate.c:2590-2670, pml.c:684-1403) ----
    S *txxo = static_cast<S *>(a.fo[F_TXX]) + fb;
    S *tzzo = static_cast<S *>(a.fo[F_TZZ]) + fb;
    S *txzo = static_cast<S *>(a.fo[F_TXZ]) + fb;
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        const int i = tid + j * NT;
        if (i >= TX * TZ) break;
        const int r = i / TZ, k = i % TZ;
        const int X = X0 + r, Z = Z0 + k;
        if (X >= a.NX || Z >= a.NZ) continue;
        // vx(X, Z) at vxs[r][k]; vz(X, Z) at vzs[r+1][k+1]
        const C vxc = vxs[r * L::VP + k];
        const C vxn = vxs[(r + 1) * L::VP + k];
        const C vx_zp = vxs[r * L::VP + k + 1];
        const C vzc = vzs[(r + 1) * L::VP + k + 1];
        const C vz_zm = vzs[(r + 1) * L::VP + k];
        const C vzp = vzs[r * L::VP + k + 1];
        const C sax = r_sub(vxn, vxc), saz = r_sub(vzc, vz_zm);
        const C sbz = r_sub(vx_zp, vxc), sbx = r_sub(vzc, vzp);
        const C txx0 = F(F_TXX, X, Z), tzz0 = F(F_TZZ, X, Z), txz0 = F(F_TXZ, X, Z);
        C txx, tzz, txz;
        if (tint || e_inside(a, X, Z)) {
            txx = r_add(txx0, r_fma(l2m[j], sax, r_mul(la[j], saz)));
            tzz = r_add(tzz0, r_fma(l2m[j], saz, r_mul(la[j], sax)));
            txz = r_fma(mu[j], r_add(sbz, sbx), txz0);
        } else {
            const long long c = sb + e_pml_index(a, X, Z);
            const C Axh = pr[P.axh() + X], Bxh = pr[P.bxh() + X];
            const C Azn = pr[P.azn() + Z], Bzn = pr[P.bzn() + Z];
            auto old = [&](const void *base, int f) {
                return St::ld(static_cast<const S *>(base) + c, a.isc[f]);
            };
            txx = e_frame<S, C>(a, F_TXX, c, Axh, Bxh, Azn, Bzn, old(a.fx[F_TXX], F_TXX),
                                old(a.fz[F_TXX], F_TXX), l2m[j], la[j], sax, saz, true);
            tzz = e_frame<S, C>(a, F_TZZ, c, Axh, Bxh, Azn, Bzn, old(a.fx[F_TZZ], F_TZZ),
                                old(a.fz[F_TZZ], F_TZZ), la[j], l2m[j], sax, saz, true);
            txz = e_frame<S, C>(a, F_TXZ, c, pr[P.axn() + X], pr[P.bxn() + X], pr[P.azh() + Z],
                                pr[P.bzh() + Z], old(a.fx[F_TXZ], F_TXZ), old(a.fz[F_TXZ], F_TXZ),
                                mu[j], mu[j], sbx, sbz, true);
        }
        const long long q = (long long)X * a.pitch + Z;
        St::st(txxo + q, txx, a.sc[F_TXX]);
        St::st(tzzo + q, tzz, a.sc[F_TZZ]);
        St::st(txzo + q, txz, a.sc[F_TXZ]);
    }
}

// one entry per source, sorted by shot; one thread per shot adds its
// sources in order, as add_src does (src.c:170-184)
struct SrcEntry {
    long long q;      // padded cell index
    int shot;
    int type;         // SM_SRC_*
    long long voff;   // offset of its scaled samples in vals
    int len;
    // block storage: the cell's block (first cell qb, nb rows inside the
    // grid, the source's row rs in it) and its exponent index qe, per shot
    long long qb, qe;
    int nb, rs;
    long long pq;     // its cell's value (field 0) in the source patches, or -1
};

// add_src (src.c:170-184) for one shot, into the wavefields f just written
template <typename S>
__device__ __forceinline__ void eiso_inject(void *const *f, long long fstride, const float *sc,
                                            const float *isc, long long it, const SrcEntry *src,
                                            const int *shot_first, const double *vals, int shot) {
    using St = Store<S>;
    using C = typename Store<S>::C;
    for (int e = shot_first[shot]; e < shot_first[shot + 1]; ++e) {
        const SrcEntry s = src[e];
        if (it >= s.len) continue;
        const C v = static_cast<C>(vals[s.voff + it]);
        const long long base = (long long)shot * fstride + s.q;
        if (s.type == SM_SRC_SX || s.type == SM_SRC_BULK) {
            S *p = static_cast<S *>(f[F_TXX]) + base;
            St::st(p, St::ld(p, isc[F_TXX]) + v, sc[F_TXX]);
        }
        if (s.type == SM_SRC_SZ || s.type == SM_SRC_BULK) {
            S *p = static_cast<S *>(f[F_TZZ]) + base;
            St::st(p, St::ld(p, isc[F_TZZ]) + v, sc[F_TZZ]);
        }
        if (s.type == SM_SRC_SXZ) {
            S *p = static_cast<S *>(f[F_TXZ]) + base;
            St::st(p, St::ld(p, isc[F_TXZ]) + v, sc[F_TXZ]);
        }
    }
}

template <typename S>
__global__ void eiso_source_kernel(EisoArgs a, const SrcEntry *src, const int *shot_first,
                                   const double *vals, int nshots) {
    const long long it = *a.step - 1;
    const int shot = blockIdx.x * blockDim.x + threadIdx.x;
    if (shot >= nshots) return;
    eiso_inject<S>(a.f, a.fstride, a.sc, a.isc, it, src, shot_first, vals, shot);
}

struct RecEntry {
    long long q;       // padded cell index
    int shot;
    int field;         // F_*
    int group;         // sampling group
    long long out;     // offset of its first sample in the trace buffer
    long long qe;      // block storage: the exponent index of its block, per shot
    long long pq;      // its cell's value (field 0) in the source patches, or -1
};

// one receiver's sample of step it, if the record's predicate takes it
// (e_iso.c:641-669, resolved into the slot table on the host)
template <typename S>
__device__ __forceinline__ void eiso_sample(void *const *f, long long fstride, const float *isc,
                                            long long it, const RecEntry &e, const int32_t *table,
                                            long long nsteps_max, double *traces) {
    using St = Store<S>;
    if (it >= nsteps_max) return;
    const int32_t slot = table[(long long)e.group * nsteps_max + it];
    if (slot < 0) return;
    const S *p = static_cast<const S *>(f[e.field]) + (long long)e.shot * fstride + e.q;
    traces[e.out + slot] = static_cast<double>(St::ld(p, isc[e.field]));
}

template <typename S>
__global__ void eiso_gather_kernel(EisoArgs a, const RecEntry *rec, int nrec,
                                   const int32_t *table, long long nsteps_max,
                                   double *traces) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    eiso_sample<S>(a.f, a.fstride, a.isc, *a.step - 1, rec[r], table, nsteps_max, traces);
}

// block storage: add_src (src.c:170-184) for one shot; each addition decodes
// the block of the source cell, adds, and stores the block again with the
// exponent its new maximum takes
__device__ __forceinline__ void eiso_badd(int16_t *m, uint8_t *e, const SrcEntry &s,
                                          long long pitch, float add, int *err) {
    const BDec d = bfp_dec(e[s.qe]);
    float v[EISO_EB];
    unsigned mx = 0;
    for (int r = 0; r < s.nb; ++r) {
        v[r] = bfp_val(m[s.qb + r * pitch], d);
        if (r == s.rs) v[r] = v[r] + add;
        mx = max(mx, bfp_absbits(v[r]));
    }
    bool over;
    const unsigned e8 = bfp_e8(mx, &over);
    const float esc = bfp_escale(e8);
    for (int r = 0; r < s.nb; ++r) m[s.qb + r * pitch] = bfp_man(v[r], esc);
    e[s.qe] = (uint8_t)e8;
    if (over) atomicExch(err, 4);
}

__device__ __forceinline__ void eiso_binject(void *const *f, long long fstride, void *fe,
                                             long long estride, long long eshot, int pitch,
                                             long long it, const SrcEntry *src,
                                             const int *shot_first, const double *vals, int shot,
                                             int *err, float *pv) {
    for (int e = shot_first[shot]; e < shot_first[shot + 1]; ++e) {
        const SrcEntry s = src[e];
        if (it >= s.len) continue;
        const float v = static_cast<float>(vals[s.voff + it]);
        int fs[2] = {-1, -1};
        if (s.type == SM_SRC_SX || s.type == SM_SRC_BULK) fs[0] = F_TXX;
        if (s.type == SM_SRC_SZ || s.type == SM_SRC_BULK) fs[1] = F_TZZ;
        if (s.type == SM_SRC_SXZ) fs[0] = F_TXZ;
        for (int k = 0; k < 2; ++k) {
            if (fs[k] < 0) continue;
            eiso_badd(static_cast<int16_t *>(f[fs[k]]) + (long long)shot * fstride,
                      static_cast<uint8_t *>(fe) + fs[k] * estride + shot * eshot, s, pitch, v, err);
            // the source's patch holds the cell in FP32: add there exactly
            if (s.pq >= 0 && pv) pv[s.pq + fs[k] * EISO_PF] += v;
        }
    }
}

__global__ void eiso_bsource_kernel(EisoArgs a, const SrcEntry *src, const int *shot_first,
                                    const double *vals, int nshots) {
    const long long it = *a.step - 1;
    const int shot = blockIdx.x * blockDim.x + threadIdx.x;
    if (shot >= nshots) return;
    eiso_binject(a.f, a.fstride, a.fe, a.estride, (long long)a.nxb * a.pitch, a.pitch, it, src,
                 shot_first, vals, shot, a.err, a.pfirst ? a.pv : nullptr);
}

__device__ __forceinline__ void eiso_bsample(void *const *f, long long fstride, const void *fe,
                                             long long estride, long long eshot, long long it,
                                             const RecEntry &e, const int32_t *table,
                                             long long nsteps_max, double *traces,
                                             const float *pv) {
    if (it >= nsteps_max) return;
    const int32_t slot = table[(long long)e.group * nsteps_max + it];
    if (slot < 0) return;
    if (e.pq >= 0 && pv) {   // a cell of a source patch: its FP32 value
        traces[e.out + slot] = static_cast<double>(pv[e.pq + e.field * EISO_PF]);
        return;
    }
    const int16_t m = static_cast<const int16_t *>(f[e.field])[(long long)e.shot * fstride + e.q];
    const unsigned e8 =
        static_cast<const uint8_t *>(fe)[e.field * estride + e.shot * eshot + e.qe];
    traces[e.out + slot] = static_cast<double>(bfp_val(m, bfp_dec(e8)));
}

__global__ void eiso_bgather_kernel(EisoArgs a, const RecEntry *rec, int nrec,
                                    const int32_t *table, long long nsteps_max, double *traces) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    eiso_bsample(a.f, a.fstride, a.fe, a.estride, (long long)a.nxb * a.pitch, *a.step - 1, rec[r],
                 table, nsteps_max, traces, a.pfirst ? a.pv : nullptr);
}

// ---------------------------------------------------------------------------
// Grouped step: one launch advances up to kGroupMax e_iso problems of
// different grid sizes and shot counts by one time step.  Linear CTA b
// belongs to the problem p with first[p] <= b < first[p+1]; inside it the
// block is (bx, by, shot) of that problem's own slab grid and the update is
// the slab step above, so each problem gets the bits its own launch gives.
// Each problem's TMA map is a kernel parameter (read from parameter space
// like the single-problem launch's); its other arguments are copied into
// shared memory once per CTA.  Sources and receivers of all problems follow
// in one launch each.
// ---------------------------------------------------------------------------
constexpr int kGroupMax = 32;

struct EisoGroupStepParams {
    CUtensorMap f[kGroupMax];     // each problem's old-set slab map
    CUtensorMap e[kGroupMax];     // ... and exponent map (block storage)
    EisoArgs a[kGroupMax];        // its arguments for this step
    int first[kGroupMax + 1];     // first linear CTA of each problem
    int gx[kGroupMax], gy[kGroupMax];
    int n;
};
static_assert(sizeof(EisoGroupStepParams) <= 32000, "kernel parameters are limited to 32 KB");
static_assert(sizeof(EisoArgs) % 4 == 0, "EisoArgs is copied as 32-bit words");

template <typename S, int W, int TX, int MINB>
__global__ void __launch_bounds__(32 * W, MINB) eiso_group_step_kernel(
    const __grid_constant__ EisoGroupStepParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ EisoArgs sa;
    const int b = blockIdx.x;
    int p = 0;
    while (p + 1 < P.n && P.first[p + 1] <= b) ++p;
    const int local = b - P.first[p];
    const int bx = local % P.gx[p], rest = local / P.gx[p];
    const int by = rest % P.gy[p], shot = rest / P.gy[p];
    {
        const int *src = reinterpret_cast<const int *>(&P.a[p]);
        int *dst = reinterpret_cast<int *>(&sa);
        for (int i = threadIdx.x; i < (int)(sizeof(EisoArgs) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    eiso_slabg_body<S, W, TX>(sa, &P.f[p], bx, by, shot, smem);
}

template <int W, int TX, int MINB>
__global__ void __launch_bounds__(32 * W, MINB) eiso_bgroup_step_kernel(
    const __grid_constant__ EisoGroupStepParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ EisoArgs sa;
    const int b = blockIdx.x;
    int p = 0;
    while (p + 1 < P.n && P.first[p + 1] <= b) ++p;
    const int local = b - P.first[p];
    const int bx = local % P.gx[p], rest = local / P.gx[p];
    const int by = rest % P.gy[p], shot = rest / P.gy[p];
    {
        const int *src = reinterpret_cast<const int *>(&P.a[p]);
        int *dst = reinterpret_cast<int *>(&sa);
        for (int i = threadIdx.x; i < (int)(sizeof(EisoArgs) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    eiso_bslab_body<W, TX>(sa, &P.f[p], &P.e[p], bx, by, shot, smem);
}

// what the source and receiver kernels of one problem need after its step
struct EisoPost {
    void *f[5];                  // the wavefields just written
    long long fstride;
    const long long *step;
    float sc[5], isc[5];
    const SrcEntry *src;
    const int *src_first;
    const double *vals;
    const RecEntry *rec;
    const int32_t *table;
    long long nsteps_max;
    double *traces;
    // block storage
    void *fe;
    long long estride, eshot;
    int pitch;
    int *err;
    float *pv;   // source patches of the set just written (null: none)
};

struct EisoGroupPostParams {
    EisoPost q[kGroupMax];
    int first_src[kGroupMax + 1];   // prefix sums of the problems' source threads (shots)
    int first_rec[kGroupMax + 1];   // ... and receiver threads
    int n;
};
static_assert(sizeof(EisoGroupPostParams) <= 32000, "kernel parameters are limited to 32 KB");

template <typename S>
__global__ void eiso_group_source_kernel(const __grid_constant__ EisoGroupPostParams P) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.first_src[P.n]) return;
    int p = 0;
    while (p + 1 < P.n && P.first_src[p + 1] <= t) ++p;
    const EisoPost &q = P.q[p];
    if constexpr (std::is_same<S, Bfp16>::value)
        eiso_binject(q.f, q.fstride, q.fe, q.estride, q.eshot, q.pitch, *q.step - 1, q.src,
                     q.src_first, q.vals, t - P.first_src[p], q.err, q.pv);
    else
        eiso_inject<S>(q.f, q.fstride, q.sc, q.isc, *q.step - 1, q.src, q.src_first, q.vals,
                       t - P.first_src[p]);
}

template <typename S>
__global__ void eiso_group_gather_kernel(const __grid_constant__ EisoGroupPostParams P) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.first_rec[P.n]) return;
    int p = 0;
    while (p + 1 < P.n && P.first_rec[p + 1] <= t) ++p;
    const EisoPost &q = P.q[p];
    if constexpr (std::is_same<S, Bfp16>::value)
        eiso_bsample(q.f, q.fstride, q.fe, q.estride, q.eshot, *q.step - 1,
                     q.rec[t - P.first_rec[p]], q.table, q.nsteps_max, q.traces, q.pv);
    else
        eiso_sample<S>(q.f, q.fstride, q.isc, *q.step - 1, q.rec[t - P.first_rec[p]], q.table,
                       q.nsteps_max, q.traces);
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
    // two buffer sets of wavefields and split parts: a step reads set `cur`
    // and writes the other one
    // the five wavefields of a set are one allocation ([field][shot][x][z],
    // so one TMA box can span all five), likewise the five materials
    DevBuf fset[2], xpart[2][5], zpart[2][5], matbuf, prof;
    void *field(int set, int f) const {
        return static_cast<char *>(fset[set].p) + (size_t)f * fset_stride;
    }
    void *mat(int k) const { return static_cast<char *>(matbuf.p) + (size_t)k * mat_stride; }
    size_t fset_stride = 0, mat_stride = 0;   // bytes between consecutive arrays
    int cur = 0;
    int config = 0;  // index into kEisoConfigs (slab 2 x 8 with materials from L2;
                     // FP32 storage starts at 16, slab 2 x 4 at 64 registers)
    DevBuf err;      // bounded-wait failure flag of the step kernels
    EisoMaps maps[2];            // TMA maps of each buffer set (tile kernel)
    int maps_key = -1;           // (TX, TZ) the maps were built for
    EisoSlabMaps slab_maps[2];   // TMA maps of each buffer set (slab kernels)
    int slab_key = -1;           // box shape the slab maps were built for
    // block storage (SM_BFP16): exponent bytes of each set,
    // [field][shot][nxb][pitch], and the slab kernel's maps
    DevBuf fexp[2];
    size_t nxb = 0;
    EisoBMaps bmaps[2];
    int bmap_key = -1;
    // ... and its source patches (EISO_PR x EISO_PC cells in FP32 around
    // each source): first row and column per patch, first patch per shot
    std::vector<int> p_xz, p_first;
    DevBuf d_pxz, d_pfirst, pside[2];
    DevBuf d_step;               // device step counter (EisoArgs::step)
    // CUDA graphs of graph_steps steps, one per parity of the starting
    // buffer set; captured again when graph_epoch moved since (new sources,
    // receivers, launch configuration or 16-bit scales)
    int graph_steps = 0;
    unsigned graph_epoch = 1;
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        unsigned epoch = 0;
        int steps = 0;
        bool timed = false;      // captured with per-kernel timing on
        EventPairs tev;          // the timed launches' event nodes
    } graphs[2];
    ~sm_eiso() {
        for (Graph &g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            for (auto &p : g.tev) {
                cudaEventDestroy(p.first);
                cudaEventDestroy(p.second);
            }
        }
    }
    int sms = 148;
    uint64_t serial = 0;   // unique per handle in the process (grouped graphs' keys)
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

// point the kernel arguments at the current (read) and other (write) sets
void eiso_bind(sm_eiso *h) {
    const int c = h->cur, o = 1 - h->cur;
    h->args.fe = h->fexp[c].p;
    h->args.feo = h->fexp[o].p;
    h->args.pv = h->pside[c].as<float>();
    h->args.pvo = h->pside[o].as<float>();
    for (int f = 0; f < 5; ++f) {
        h->args.f[f] = h->field(c, f);
        h->args.fx[f] = h->xpart[c][f].p;
        h->args.fz[f] = h->zpart[c][f].p;
        h->args.fo[f] = h->field(o, f);
        h->args.fxo[f] = h->xpart[o][f].p;
        h->args.fzo[f] = h->zpart[o][f].p;
    }
}

// launch configurations of the step kernel (an index into this table):
//   slab, materials from global (kind 0): p = {warps per CTA, rows TX, min CTAs per SM}
//   tile (kind 1): p = {TX, TZ, threads, min CTAs per SM}
//   slab, materials by TMA (kind 2): p = {warps per CTA, rows TX, min CTAs per SM}
//   persistent slab, materials from global (kind 3): p = {warps per CTA, rows TX, min CTAs per SM}
// The minimum resident CTAs per SM caps the registers a thread may use.
struct EisoConfig {
    int kind;
    int p[4];
};
static const EisoConfig kEisoConfigs[] = {
    {0, {2, 8, 8, 0}},  {0, {2, 4, 12, 0}},   {0, {4, 4, 6, 0}},    {0, {1, 8, 16, 0}},
    {0, {4, 8, 4, 0}},  {0, {2, 16, 4, 0}},   {1, {8, 32, 128, 6}}, {1, {16, 64, 256, 2}},
    {1, {8, 64, 256, 3}}, {2, {2, 8, 8, 0}},  {2, {4, 8, 4, 0}},    {2, {1, 16, 12, 0}},
    {3, {2, 8, 8, 0}},  {3, {2, 8, 12, 0}},   {3, {4, 8, 6, 0}},    {3, {2, 4, 12, 0}},
    // 16: slabs of 4 rows by 2 warps bounded to 64 registers, 16 CTAs (32
    // warps) per SM: 0.393 ms per step on 64 shots of 1040 x 540 against
    // 0.412 for configuration 0 (80 registers, 12 CTAs); 4 rows by 4 warps
    // at 64 registers measured 0.464, 6 rows by 2 warps 0.430
    {0, {2, 4, 16, 0}}};
static const int kEisoNumConfigs = sizeof(kEisoConfigs) / sizeof(kEisoConfigs[0]);
// block storage: the slab step only, {warps per CTA, rows TX (whole blocks),
// min CTAs per SM}
struct EisoBConfig {
    int w, tx, minb, persistent;
};
static const EisoBConfig kEisoBConfigs[] = {
    {2, 8, 8, 0},  {4, 8, 4, 0},   {2, 4, 12, 0}, {4, 4, 6, 0}, {1, 8, 16, 0},
    {2, 8, 12, 0}, {2, 4, 16, 0},  {4, 8, 6, 0},
    {2, 8, 8, 1},  {2, 8, 12, 1},  {4, 8, 6, 1},  {2, 4, 16, 1}};
static const int kEisoBNumConfigs = sizeof(kEisoBConfigs) / sizeof(kEisoBConfigs[0]);

bool eiso_isb(const sm_eiso *h) { return h->precision == SM_BFP16; }
int eiso_ncfg(const sm_eiso *h) { return eiso_isb(h) ? kEisoBNumConfigs : kEisoNumConfigs; }

// TMA maps of the block-storage slab step: mantissas as the other slab
// maps (z, x, shot, field), exponents (z, x block, shot, field)
template <int W, int TX>
int eiso_make_bmaps(sm_eiso *h) {
    using L = ESlabB<W, TX>;
    const int key = W * 4096 + TX;
    if (h->bmap_key == key) return SM_OK;
    const size_t row = (size_t)h->pitch;
    const size_t fdims[4] = {(size_t)h->NZ, (size_t)h->NX, h->nshots, 5};
    const size_t fstr[3] = {row * 2, h->NX * row * 2, h->fset_stride};
    const unsigned fbox[4] = {(unsigned)L::BW, (unsigned)L::RX, 1, 5};
    const size_t edims[4] = {(size_t)h->NZ, h->nxb, h->nshots, 5};
    const size_t estr[3] = {row, h->nxb * row, (size_t)h->args.estride};
    const unsigned ebox[4] = {(unsigned)L::BWE, (unsigned)L::NB, 1, 5};
    for (int b = 0; b < 2; ++b) {
        if (int rc = make_map_nd(&h->bmaps[b].f, h->fset[b].p, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2,
                                 4, fdims, fstr, fbox))
            return rc;
        if (int rc = make_map_nd(&h->bmaps[b].e, h->fexp[b].p, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, 4,
                                 edims, estr, ebox))
            return rc;
    }
    h->bmap_key = key;
    return SM_OK;
}

template <typename S, int TX, int TZ>
int eiso_make_tile_maps(sm_eiso *h) {
    using L = ETile<S, TX, TZ>;
    const int key = TX * 4096 + TZ;
    if (h->maps_key == key) return SM_OK;
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < 5; ++f)
            if (int rc = make_map_3d(&h->maps[b].f[f], h->field(b, f), MapType<S>::v, sizeof(S),
                                     h->NZ, h->NX, h->nshots, h->pitch, L::BZ, L::RX))
                return rc;
    h->maps_key = key;
    return SM_OK;
}

// TMA maps of the slab kernels: the five wavefields of a set as one 4-D
// tensor (z, x, shot, field) and the materials as one 3-D tensor (z, x,
// material), boxes of L's shape
template <typename S, typename L, int KEY>
int eiso_make_slab_maps(sm_eiso *h) {
    using C = typename Store<S>::C;
    if (h->slab_key == KEY) return SM_OK;
    const size_t e = sizeof(S), c = sizeof(C), row = (size_t)h->pitch;
    const size_t fdims[4] = {(size_t)h->NZ, (size_t)h->NX, h->nshots, 5};
    const size_t fstr[3] = {row * e, h->NX * row * e, h->fset_stride};
    const unsigned fbox[4] = {(unsigned)L::BW, (unsigned)L::RX, 1, 5};
    const size_t mdims[3] = {(size_t)h->NZ, (size_t)h->NX, 5};
    const size_t mstr[2] = {row * c, h->mat_stride};
    const unsigned mbox[3] = {(unsigned)L::BWC, (unsigned)L::RX, 5};
    for (int b = 0; b < 2; ++b) {
        if (int rc = make_map_nd(&h->slab_maps[b].f, h->fset[b].p, MapType<S>::v, e, 4, fdims,
                                 fstr, fbox))
            return rc;
        if (int rc = make_map_nd(&h->slab_maps[b].m, h->matbuf.p, MapType<C>::v, c, 3, mdims, mstr,
                                 mbox))
            return rc;
    }
    h->slab_key = KEY;
    return SM_OK;
}

// dynamic shared memory above 48 KB must be allowed per kernel and device
template <typename K>
int allow_smem(K kernel, size_t bytes, int device) {
    static std::mutex mu;
    static std::set<std::pair<const void *, int>> done;   // (kernel, device)
    const std::pair<const void *, int> key(reinterpret_cast<const void *>(kernel), device);
    std::lock_guard<std::mutex> lk(mu);
    if (!done.count(key)) {
        SM_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bytes));
        done.insert(key);
    }
    return SM_OK;
}

template <typename S, int TX, int TZ, int NT, int MINB>
int ready_tile_cfg(sm_eiso *h) {
    if (int rc = eiso_make_tile_maps<S, TX, TZ>(h)) return rc;
    return allow_smem(eiso_tile_kernel<S, TX, TZ, NT, MINB>, ETile<S, TX, TZ>::bytes, h->device);
}

template <typename S, int TX, int TZ, int NT, int MINB>
int launch_tile_cfg(sm_eiso *h) {
    using L = ETile<S, TX, TZ>;
    dim3 grd((h->NZ + TZ - 1) / TZ, (h->NX + TX - 1) / TX, (unsigned)h->nshots);
    eiso_tile_kernel<S, TX, TZ, NT, MINB><<<grd, NT, L::bytes, h->stream>>>(h->args,
                                                                           h->maps[h->cur]);
    return SM_OK;
}

template <typename S, int W, int TX, int MINB>
int ready_slab_cfg(sm_eiso *h) {
    if (int rc = eiso_make_slab_maps<S, ESlab<S, W, TX>, W * 4096 + TX>(h)) return rc;
    return allow_smem(eiso_slab_kernel<S, W, TX, MINB>, ESlab<S, W, TX>::bytes, h->device);
}

template <typename S, int W, int TX, int MINB>
int launch_slab_cfg(sm_eiso *h) {
    using L = ESlab<S, W, TX>;
    const int wz = (h->NZ + 29) / 30;
    dim3 grd((wz + W - 1) / W, (h->NX + TX - 1) / TX, (unsigned)h->nshots);
    eiso_slab_kernel<S, W, TX, MINB><<<grd, 32 * W, L::bytes, h->stream>>>(h->args,
                                                                          h->slab_maps[h->cur]);
    return SM_OK;
}

template <typename S, int W, int TX, int MINB>
int ready_slabg_cfg(sm_eiso *h) {
    if (int rc = eiso_make_slab_maps<S, ESlabG<S, W, TX>, (1 << 20) + W * 4096 + TX>(h)) return rc;
    return allow_smem(eiso_slabg_kernel<S, W, TX, MINB>, ESlabG<S, W, TX>::bytes, h->device);
}

// the launch order of the slabs of W warps x TX rows (SlabOrder): the lean
// rectangle first, or (lean_first false) every shot's slabs in grid order.
// Measured on the 64-shot 1040 x 540 batch: block storage 0.514 against
// 0.553 ms per step with the rectangle first; FP32 0.440 against 0.415, so
// the FP32 slab step keeps its 3-D grid in grid order.
SlabOrder slab_order(const sm_eiso *h, int W, int TX, bool lean_first) {
    const int wz = (int)((h->NZ + 29) / 30);
    SlabOrder o{(wz + W - 1) / W, (int)((h->NX + TX - 1) / TX), 0, 0, 0, 0};
    o.by0 = o.by1 = o.gy;   // no rectangle: grid order
    if (!lean_first) return o;
    const long long np = (long long)h->np, nx = (long long)h->nx, nz = (long long)h->nz;
    // slab bx is lean in z when its first warp starts at Z0 - 1 >= np and its
    // last warp ends at Z0 + 30 <= np + nz - 1; slab by when its rows lie in
    // [np, np + nx - 1]
    o.bx0 = (int)std::min<long long>(o.gx, (np + 1 + 30LL * W - 1) / (30LL * W));
    o.bx1 = o.bx0;
    while (o.bx1 < o.gx && 30LL * W * o.bx1 + 30LL * W <= np + nz - 1) ++o.bx1;
    o.by0 = (int)std::min<long long>(o.gy, (np + TX - 1) / TX);
    o.by1 = o.by0;
    while (o.by1 < o.gy && (long long)TX * o.by1 + TX <= np + nx - 1) ++o.by1;
    if (o.bx1 <= o.bx0 || o.by1 <= o.by0) {   // no rectangle: every slab in the ring
        o.bx0 = o.bx1 = 0;
        o.by0 = o.by1 = o.gy;
    }
    return o;
}

template <typename S, int W, int TX, int MINB>
int launch_slabg_cfg(sm_eiso *h) {
    const int wz = (h->NZ + 29) / 30;
    dim3 grd((wz + W - 1) / W, (h->NX + TX - 1) / TX, (unsigned)h->nshots);
    eiso_slabg_kernel<S, W, TX, MINB><<<grd, 32 * W, ESlabG<S, W, TX>::bytes, h->stream>>>(
        h->args, h->slab_maps[h->cur]);
    return SM_OK;
}

template <typename S, int W, int TX>
constexpr size_t slabg_p_smem() {
    return 2 * ESlabG<S, W, TX>::al(ESlabG<S, W, TX>::bytes);
}

template <typename S, int W, int TX, int MINB>
int ready_slabg_p_cfg(sm_eiso *h) {
    if (int rc = eiso_make_slab_maps<S, ESlabG<S, W, TX>, (1 << 20) + W * 4096 + TX>(h)) return rc;
    return allow_smem(eiso_slabg_pkernel<S, W, TX, MINB>, slabg_p_smem<S, W, TX>(), h->device);
}

// as many CTAs as fit on the device at once, each walking its share of slabs
template <typename S, int W, int TX, int MINB>
int launch_slabg_p_cfg(sm_eiso *h) {
    const int gx = ((h->NZ + 29) / 30 + W - 1) / W, gy = (h->NX + TX - 1) / TX;
    const int nslab = gx * gy * (int)h->nshots;
    static int occ[64] = {};
    if (h->device >= 0 && h->device < 64 && occ[h->device] == 0) {
        int n = 0;
        SM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, eiso_slabg_pkernel<S, W, TX, MINB>, 32 * W, slabg_p_smem<S, W, TX>()));
        occ[h->device] = n > 0 ? n : 1;
    }
    const int per = (h->device >= 0 && h->device < 64) ? occ[h->device] : 1;
    const int grid = std::min(nslab, h->sms * per);
    eiso_slabg_pkernel<S, W, TX, MINB><<<grid, 32 * W, slabg_p_smem<S, W, TX>(), h->stream>>>(
        h->args, h->slab_maps[h->cur], gx, gy, nslab);
    return SM_OK;
}

template <int W, int TX, int MINB>
int ready_bslab_cfg(sm_eiso *h) {
    if (int rc = eiso_make_bmaps<W, TX>(h)) return rc;
    return allow_smem(eiso_bslab_kernel<W, TX, MINB>, ESlabB<W, TX>::bytes, h->device);
}

template <int W, int TX, int MINB>
int launch_bslab_cfg(sm_eiso *h) {
    const SlabOrder o = slab_order(h, W, TX, true);
    const unsigned n = (unsigned)(o.gx * o.gy) * (unsigned)h->nshots;
    eiso_bslab_kernel<W, TX, MINB><<<n, 32 * W, ESlabB<W, TX>::bytes, h->stream>>>(
        h->args, h->bmaps[h->cur], o);
    return SM_OK;
}

template <int W, int TX>
constexpr size_t bslab_p_smem() {
    return 2 * ESlabB<W, TX>::al(ESlabB<W, TX>::bytes);
}

template <int W, int TX, int MINB>
int ready_bslab_p_cfg(sm_eiso *h) {
    if (int rc = eiso_make_bmaps<W, TX>(h)) return rc;
    return allow_smem(eiso_bslab_pkernel<W, TX, MINB>, bslab_p_smem<W, TX>(), h->device);
}

// as many CTAs as fit on the device at once (each walks its share of slabs)
template <int W, int TX, int MINB>
int launch_bslab_p_cfg(sm_eiso *h) {
    const int gx = ((h->NZ + 29) / 30 + W - 1) / W, gy = (h->NX + TX - 1) / TX;
    const int nslab = gx * gy * (int)h->nshots;
    static int occ[64] = {};
    if (h->device >= 0 && h->device < 64 && occ[h->device] == 0) {
        int n = 0;
        SM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, eiso_bslab_pkernel<W, TX, MINB>, 32 * W, bslab_p_smem<W, TX>()));
        occ[h->device] = n > 0 ? n : 1;
    }
    const int per = (h->device >= 0 && h->device < 64) ? occ[h->device] : 1;
    const int grid = std::min(nslab, h->sms * per);
    eiso_bslab_pkernel<W, TX, MINB><<<grid, 32 * W, bslab_p_smem<W, TX>(), h->stream>>>(
        h->args, h->bmaps[h->cur], gx, gy, nslab);
    return SM_OK;
}

size_t eiso_bconfig_smem(int config) {
    switch (config) {
    case 0: case 5: return ESlabB<2, 8>::bytes;
    case 1: case 7: return ESlabB<4, 8>::bytes;
    case 2: case 6: return ESlabB<2, 4>::bytes;
    case 3: return ESlabB<4, 4>::bytes;
    case 8: case 9: return bslab_p_smem<2, 8>();
    case 10: return bslab_p_smem<4, 8>();
    case 11: return bslab_p_smem<2, 4>();
    default: return ESlabB<1, 8>::bytes;
    }
}

int eiso_bready(sm_eiso *h) {
    switch (h->config) {
    case 0: return ready_bslab_cfg<2, 8, 8>(h);
    case 1: return ready_bslab_cfg<4, 8, 4>(h);
    case 2: return ready_bslab_cfg<2, 4, 12>(h);
    case 3: return ready_bslab_cfg<4, 4, 6>(h);
    case 5: return ready_bslab_cfg<2, 8, 12>(h);
    case 6: return ready_bslab_cfg<2, 4, 16>(h);
    case 7: return ready_bslab_cfg<4, 8, 6>(h);
    case 8: return ready_bslab_p_cfg<2, 8, 8>(h);
    case 9: return ready_bslab_p_cfg<2, 8, 12>(h);
    case 10: return ready_bslab_p_cfg<4, 8, 6>(h);
    case 11: return ready_bslab_p_cfg<2, 4, 16>(h);
    default: return ready_bslab_cfg<1, 8, 16>(h);
    }
}

int eiso_blaunch(sm_eiso *h) {
    switch (h->config) {
    case 0: return launch_bslab_cfg<2, 8, 8>(h);
    case 1: return launch_bslab_cfg<4, 8, 4>(h);
    case 2: return launch_bslab_cfg<2, 4, 12>(h);
    case 3: return launch_bslab_cfg<4, 4, 6>(h);
    case 5: return launch_bslab_cfg<2, 8, 12>(h);
    case 6: return launch_bslab_cfg<2, 4, 16>(h);
    case 7: return launch_bslab_cfg<4, 8, 6>(h);
    case 8: return launch_bslab_p_cfg<2, 8, 8>(h);
    case 9: return launch_bslab_p_cfg<2, 8, 12>(h);
    case 10: return launch_bslab_p_cfg<4, 8, 6>(h);
    case 11: return launch_bslab_p_cfg<2, 4, 16>(h);
    default: return launch_bslab_cfg<1, 8, 16>(h);
    }
}

template <typename S>
size_t eiso_config_smem(int config) {
    switch (config) {
    case 0: return ESlabG<S, 2, 8>::bytes;
    case 1: return ESlabG<S, 2, 4>::bytes;
    case 2: return ESlabG<S, 4, 4>::bytes;
    case 3: return ESlabG<S, 1, 8>::bytes;
    case 4: return ESlabG<S, 4, 8>::bytes;
    case 5: return ESlabG<S, 2, 16>::bytes;
    case 6: return ETile<S, 8, 32>::bytes;
    case 7: return ETile<S, 16, 64>::bytes;
    case 8: return ETile<S, 8, 64>::bytes;
    case 9: return ESlab<S, 2, 8>::bytes;
    case 10: return ESlab<S, 4, 8>::bytes;
    case 12: case 13: return slabg_p_smem<S, 2, 8>();
    case 14: return slabg_p_smem<S, 4, 8>();
    case 15: return slabg_p_smem<S, 2, 4>();
    case 16: return ESlabG<S, 2, 4>::bytes;
    default: return ESlab<S, 1, 16>::bytes;
    }
}

size_t eiso_config_smem_prec(int precision, int config) {
    switch (precision) {
    case SM_BFP16: return eiso_bconfig_smem(config);
    case SM_FP64: return eiso_config_smem<double>(config);
    case SM_FP16: return eiso_config_smem<__half>(config);
    case SM_BF16: return eiso_config_smem<__nv_bfloat16>(config);
    default: return eiso_config_smem<float>(config);
    }
}

// TMA maps and shared-memory limits of the current configuration (kept out
// of stream capture)
template <typename S>
int eiso_ready(sm_eiso *h) {
    if constexpr (std::is_same<S, Bfp16>::value) return eiso_bready(h);
    else switch (h->config) {
    case 0: return ready_slabg_cfg<S, 2, 8, 8>(h);
    case 1: return ready_slabg_cfg<S, 2, 4, 12>(h);
    case 2: return ready_slabg_cfg<S, 4, 4, 6>(h);
    case 3: return ready_slabg_cfg<S, 1, 8, 16>(h);
    case 4: return ready_slabg_cfg<S, 4, 8, 4>(h);
    case 5: return ready_slabg_cfg<S, 2, 16, 4>(h);
    case 6: return ready_tile_cfg<S, 8, 32, 128, 6>(h);
    case 7: return ready_tile_cfg<S, 16, 64, 256, 2>(h);
    case 8: return ready_tile_cfg<S, 8, 64, 256, 3>(h);
    case 9: return ready_slab_cfg<S, 2, 8, 8>(h);
    case 10: return ready_slab_cfg<S, 4, 8, 4>(h);
    case 12: return ready_slabg_p_cfg<S, 2, 8, 8>(h);
    case 13: return ready_slabg_p_cfg<S, 2, 8, 12>(h);
    case 14: return ready_slabg_p_cfg<S, 4, 8, 6>(h);
    case 15: return ready_slabg_p_cfg<S, 2, 4, 12>(h);
    case 16: return ready_slabg_cfg<S, 2, 4, 16>(h);
    default: return ready_slab_cfg<S, 1, 16, 12>(h);
    }
}

template <typename S>
int launch_step(sm_eiso *h) {
    cudaEvent_t t0 = h->timer.begin(h->stream);
    int rc = SM_OK;
    if constexpr (std::is_same<S, Bfp16>::value) rc = eiso_blaunch(h);
    else switch (h->config) {
    case 0: rc = launch_slabg_cfg<S, 2, 8, 8>(h); break;
    case 1: rc = launch_slabg_cfg<S, 2, 4, 12>(h); break;
    case 2: rc = launch_slabg_cfg<S, 4, 4, 6>(h); break;
    case 3: rc = launch_slabg_cfg<S, 1, 8, 16>(h); break;
    case 4: rc = launch_slabg_cfg<S, 4, 8, 4>(h); break;
    case 5: rc = launch_slabg_cfg<S, 2, 16, 4>(h); break;
    case 6: rc = launch_tile_cfg<S, 8, 32, 128, 6>(h); break;
    case 7: rc = launch_tile_cfg<S, 16, 64, 256, 2>(h); break;
    case 8: rc = launch_tile_cfg<S, 8, 64, 256, 3>(h); break;
    case 9: rc = launch_slab_cfg<S, 2, 8, 8>(h); break;
    case 10: rc = launch_slab_cfg<S, 4, 8, 4>(h); break;
    case 12: rc = launch_slabg_p_cfg<S, 2, 8, 8>(h); break;
    case 13: rc = launch_slabg_p_cfg<S, 2, 8, 12>(h); break;
    case 14: rc = launch_slabg_p_cfg<S, 4, 8, 6>(h); break;
    case 15: rc = launch_slabg_p_cfg<S, 2, 4, 12>(h); break;
    case 16: rc = launch_slabg_cfg<S, 2, 4, 16>(h); break;
    default: rc = launch_slab_cfg<S, 1, 16, 12>(h); break;
    }
    if (rc) return rc;
    h->timer.end(t0, h->stream);
    h->timer.launches += 1;
    h->cur = 1 - h->cur;
    eiso_bind(h);
    return SM_OK;
}

template <typename S>
void launch_src(sm_eiso *h) {
    if (h->d_src.bytes == 0) return;
    int n = (int)h->nshots;
    h->timer.launches += 1;
    if constexpr (std::is_same<S, Bfp16>::value)
        eiso_bsource_kernel<<<(n + 127) / 128, 128, 0, h->stream>>>(
            h->args, h->d_src.as<SrcEntry>(), h->d_src_first.as<int>(), h->d_vals.as<double>(), n);
    else
        eiso_source_kernel<S><<<(n + 127) / 128, 128, 0, h->stream>>>(
            h->args, h->d_src.as<SrcEntry>(), h->d_src_first.as<int>(), h->d_vals.as<double>(), n);
}

template <typename S>
void launch_gather(sm_eiso *h) {
    if (h->n_rec_total == 0) return;
    int n = h->n_rec_total;
    h->timer.launches += 1;
    if constexpr (std::is_same<S, Bfp16>::value)
        eiso_bgather_kernel<<<(n + 127) / 128, 128, 0, h->stream>>>(
            h->args, h->d_rec.as<RecEntry>(), n, h->d_table.as<int32_t>(), h->table_steps,
            h->d_traces.as<double>());
    else
        eiso_gather_kernel<S><<<(n + 127) / 128, 128, 0, h->stream>>>(
            h->args, h->d_rec.as<RecEntry>(), n, h->d_table.as<int32_t>(), h->table_steps,
            h->d_traces.as<double>());
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
        ptrs[3 * f] = h->field(h->cur, f); ns[3 * f] = fcells; groups[3 * f] = f;
        ptrs[3 * f + 1] = h->xpart[h->cur][f].p; ns[3 * f + 1] = h->npml_cells * h->nshots; groups[3 * f + 1] = f;
        ptrs[3 * f + 2] = h->zpart[h->cur][f].p; ns[3 * f + 2] = h->npml_cells * h->nshots; groups[3 * f + 2] = f;
    }
    const std::vector<int> before = h->scaler.expo;
    int rc = h->precision == SM_FP16
                 ? h->scaler.check<__half>(h->stream, 15, ptrs, ns, groups, names)
                 : h->scaler.check<__nv_bfloat16>(h->stream, 15, ptrs, ns, groups, names);
    eiso_apply_scales(h);
    if (h->scaler.expo != before) h->graph_epoch++;   // scales are baked into graphs
    return rc;
}

// the patch holding padded cell (X, Z) of a shot, or -1
int eiso_patch_of(const sm_eiso *h, size_t shot, long X, long Z) {
    if (h->p_first.empty()) return -1;
    for (int q = h->p_first[shot]; q < h->p_first[shot + 1]; ++q) {
        const long px = h->p_xz[2 * q], pz = h->p_xz[2 * q + 1];
        if (X >= px && X < px + EISO_PR && Z >= pz && Z < pz + EISO_PC) return q;
    }
    return -1;
}

long long eiso_patch_index(const sm_eiso *h, int q, long X, long Z) {
    return (long long)q * 5 * EISO_PF + (X - h->p_xz[2 * q]) * EISO_PC + (Z - h->p_xz[2 * q + 1]);
}

// Source patches of block storage, from the shots' sources: one per source
// whose rectangle keeps clear of the shot's earlier patches (rows apart by a
// slab's reach, so a slab meets at most one patch per column); built only
// for a handle at step 0 (the patches start from a zero state), dropped
// otherwise.  Marks the receivers for upload (they look up their patch).
int eiso_build_patches(sm_eiso *h) {
    h->p_xz.clear();
    h->p_first.assign(h->nshots + 1, 0);
    h->args.pfirst = nullptr;
    h->args.pxz = nullptr;
    h->rec_dirty = 1;
    if (h->it != 0) {
        h->p_first.clear();
        return SM_OK;
    }
    constexpr long kReach = 18;   // rows of the widest slab box
    for (size_t s = 0; s < h->nshots; ++s) {
        h->p_first[s] = (int)(h->p_xz.size() / 2);
        for (SrcEntry &e : h->shot_src[s]) {
            const long X = (long)(e.q / h->pitch), Z = (long)(e.q % h->pitch);
            const long px = EISO_EB * (X / EISO_EB - EISO_PB), pz = Z - EISO_PZ;
            bool clear = true;
            for (int q = h->p_first[s]; q < (int)(h->p_xz.size() / 2); ++q) {
                const long qx = h->p_xz[2 * q], qz = h->p_xz[2 * q + 1];
                const bool zo = pz < qz + EISO_PC && qz < pz + EISO_PC;
                const bool xo = px - kReach < qx + EISO_PR && qx - kReach < px + EISO_PR;
                if (zo && xo) clear = false;
            }
            if (!clear) continue;
            h->p_xz.push_back((int)px);
            h->p_xz.push_back((int)pz);
        }
    }
    const int np = (int)(h->p_xz.size() / 2);
    h->p_first[h->nshots] = np;
    if (np == 0) {
        h->p_first.clear();
        return SM_OK;
    }
    int rc;
    if ((rc = h->d_pxz.alloc(h->p_xz.size() * sizeof(int)))) return rc;
    if ((rc = h->d_pfirst.alloc(h->p_first.size() * sizeof(int)))) return rc;
    for (int k = 0; k < 2; ++k) {
        if ((rc = h->pside[k].alloc((size_t)np * 5 * EISO_PF * sizeof(float)))) return rc;
        if ((rc = h->pside[k].zero(h->stream))) return rc;
    }
    SM_CUDA_TRY(cudaMemcpyAsync(h->d_pxz.p, h->p_xz.data(), h->p_xz.size() * sizeof(int),
                                cudaMemcpyHostToDevice, h->stream));
    SM_CUDA_TRY(cudaMemcpyAsync(h->d_pfirst.p, h->p_first.data(), h->p_first.size() * sizeof(int),
                                cudaMemcpyHostToDevice, h->stream));
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->args.pfirst = h->d_pfirst.as<int>();
    h->args.pxz = h->d_pxz.as<int>();
    eiso_bind(h);
    return SM_OK;
}

int upload_sources(sm_eiso *h) {
    h->graph_epoch++;
    if (eiso_isb(h))
        if (int rc = eiso_build_patches(h)) return rc;
    std::vector<SrcEntry> all;
    std::vector<int> first(h->nshots + 1, 0);
    std::vector<double> vals;
    for (size_t s = 0; s < h->nshots; ++s) {
        first[s] = (int)all.size();
        long long base = (long long)vals.size();
        for (SrcEntry e : h->shot_src[s]) {
            e.voff += base;
            e.pq = -1;
            const long X = (long)(e.q / h->pitch), Z = (long)(e.q % h->pitch);
            const int q = eiso_patch_of(h, s, X, Z);
            if (q >= 0) e.pq = eiso_patch_index(h, q, X, Z);
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
    h->graph_epoch++;
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
            e.pq = -1;
            const long X = (long)(e.q / h->pitch), Z = (long)(e.q % h->pitch);
            const int q = eiso_patch_of(h, s, X, Z);
            if (q >= 0) e.pq = eiso_patch_index(h, q, X, Z);
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
    // the trace buffer comes from the device cache: no step of this handle
    // may still write the old one when it goes back
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if ((rc = h->d_traces.alloc_pooled(std::max<long long>(out, 1) * sizeof(double), h->device)))
        return rc;
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

int eiso_check_err(sm_eiso *h) {
    int e = 0;
    SM_CUDA_TRY(cudaMemcpy(&e, h->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e == 4)
        return sm_fail(SM_ESTATE, "e_iso: a block of the 16-bit block storage exceeded its range "
                                  "(|value| >= 2^114)");
    if (e) return sm_fail(SM_ETIMEOUT, "e_iso step kernel: a bounded wait for a TMA load gave up");
    return SM_OK;
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

// ---- host set-up shared by sm_eiso_create and sm_eiso_run_noalloc ----

// Material k (M_B, M_BM, M_LA, M_L2M, M_MU; src is the reference's [nx][nz]
// array of it) on the padded grid of (nx + 2 np) rows of `pitch` values,
// edge replicated and multiplied by `scale` (dt/h); the pitch padding is 0.
// pml.c reads the interior's edge values in the frame; for lambda and
// lambda+2mu in the lower-right corner it reads [nx*nx-1]
// (pml.c:1044-1084).  That index is kept while it lies inside the array
// (nx <= nz) and replaced by the intended [nx*nz-1] otherwise.
void eiso_pad_material(size_t nx, size_t nz, size_t np, size_t pitch, double scale,
                       const double *src, int k, double *m) {
    const size_t NX = nx + 2 * np, NZ = nz + 2 * np;
    size_t lr = nx * nx - 1;
    if (lr >= nx * nz) lr = nx * nz - 1;
    for (size_t X = 0; X < NX; ++X) {
        const size_t i = X < np ? 0 : (X - np >= nx ? nx - 1 : X - np);
        double *row = m + X * pitch;
        for (size_t Z = 0; Z < NZ; ++Z) {
            const size_t j = Z < np ? 0 : (Z - np >= nz ? nz - 1 : Z - np);
            size_t idx = i * nz + j;
            if ((k == M_LA || k == M_L2M) && X >= np + nx && Z >= np + nz) idx = lr;
            row[Z] = scale * src[idx];
        }
        for (size_t Z = NZ; Z < pitch; ++Z) row[Z] = 0.0;
    }
}

// The damping tables of the split-field PML in the EisoProf layout:
// A = (2 - dt d)/(2 + dt d), B = 2/(2 + dt d) per node and half node of each
// axis, from the reference's profiles d (nodes), dh (half nodes, start side)
// and dH (half nodes, end side) read reversed on the far side; A = B = 1
// outside the frame (e_iso.c:482-500, pml.c:39-1403).
std::vector<double> eiso_damping_tables(size_t nx, size_t nz, size_t np, double dt,
                                        const double *d, const double *dh, const double *dH) {
    const size_t NX = nx + 2 * np, NZ = nz + 2 * np;
    const EisoProf P{(int)NX, (int)NZ};
    std::vector<double> t((size_t)P.size(), 1.0);
    auto fill = [&](int aoff, int boff, size_t n, size_t ncell, bool half) {
        for (size_t X = 0; X < n; ++X) {
            double dd = -1.0;
            if (X < np) dd = half ? dh[X] : d[X];
            else if (X >= np + ncell) {
                const size_t i = X - np - ncell;
                dd = half ? dH[np - 1 - i] : d[np - 1 - i];
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
    return t;
}

// One source at the reference's cell index (i*nz + j) as a padded-grid entry
// with its samples (scale * fct) appended to vals; `who` names the caller in
// the error message.
int eiso_source_entry(size_t nx, size_t nz, size_t np, size_t pitch, size_t index, int type,
                      const double *fct, size_t length, size_t stride, double scale,
                      const char *who, SrcEntry *e, std::vector<double> &vals) {
    if (index >= nx * nz) return sm_fail(SM_EINVAL, "%s: source outside the grid", who);
    if (type != SM_SRC_SX && type != SM_SRC_SZ && type != SM_SRC_SXZ && type != SM_SRC_BULK)
        return sm_fail(SM_EINVAL, "%s: source type %d not supported", who, type);
    if (length > stride) return sm_fail(SM_EINVAL, "%s: source length exceeds stride", who);
    *e = SrcEntry{};
    e->q = (long long)(index / nz + np) * (long long)pitch + (long long)(index % nz + np);
    {   // its block of EISO_EB rows along x (block storage)
        const size_t X = index / nz + np, Z = index % nz + np, NX = nx + 2 * np;
        const size_t xb = X / EISO_EB;
        e->qb = (long long)(xb * EISO_EB) * (long long)pitch + (long long)Z;
        e->qe = (long long)xb * (long long)pitch + (long long)Z;
        e->nb = (int)std::min<size_t>(EISO_EB, NX - xb * EISO_EB);
        e->rs = (int)(X - xb * EISO_EB);
    }
    e->pq = -1;
    e->type = type;
    e->voff = (long long)vals.size();
    e->len = (int)length;
    for (size_t k = 0; k < length; ++k) vals.push_back(scale * fct[k]);
    return SM_OK;
}

// One receiver at the reference's cell index as a padded-grid entry.
int eiso_receiver_entry(size_t nx, size_t nz, size_t np, size_t pitch, size_t index, int comp,
                        int group, const char *who, RecEntry *e) {
    if (index >= nx * nz) return sm_fail(SM_EINVAL, "%s: receiver outside the grid", who);
    const int f = field_id(comp);
    if (f < 0) return sm_fail(SM_EINVAL, "%s: component %d not recorded by e_iso", who, comp);
    *e = RecEntry{};
    e->q = (long long)(index / nz + np) * (long long)pitch + (long long)(index % nz + np);
    e->qe = (long long)((index / nz + np) / EISO_EB) * (long long)pitch + (long long)(index % nz + np);
    e->pq = -1;
    e->field = f;
    e->group = group;
    return SM_OK;
}

}  // namespace

// 2 MB rounding of each large array (the allocation granularity)
static size_t mb2(size_t b) { return (b + (2u << 20) - 1) / (2u << 20) * (2u << 20); }

extern "C" int sm_eiso_device_bytes(size_t nx, size_t nz, size_t npml, int precision,
                                    size_t nshots, size_t nrec, size_t nsteps_max,
                                    size_t *bytes) {
    if (!bytes) return sm_fail(SM_EINVAL, "sm_eiso_device_bytes: NULL");
    if (precision < SM_FP32 || precision > SM_BFP16)
        return sm_fail(SM_EINVAL, "sm_eiso_device_bytes: unknown precision %d", precision);
    const size_t NX = nx + 2 * npml, NZ = nz + 2 * npml, pitch = round_up(NZ, 32);
    const size_t fcells = NX * pitch, e = storage_bytes(precision);
    const size_t c = precision == SM_FP64 ? 8 : 4;
    const size_t pe = precision == SM_BFP16 ? 4 : e;          // split parts
    const size_t pml = 4 * npml * npml + 2 * npml * (nx + nz);
    size_t b = 2 * mb2(5 * fcells * nshots * e);              // two buffer sets
    if (precision == SM_BFP16)                                // their exponents
        b += 2 * mb2(5 * nshots * ((NX + EISO_EB - 1) / EISO_EB) * pitch);
    b += 20 * mb2(pml * nshots * pe);                         // split parts, both sets
    b += mb2(5 * fcells * c) + mb2((4 * NX + 4 * NZ) * c);    // materials, profiles
    b += mb2(nrec * nshots * nsteps_max * (sizeof(double) + sizeof(int32_t)));   // traces, table
    b += 16u << 20;                                           // small buffers, 16-bit scaler
    *bytes = b;
    return SM_OK;
}

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
    if (precision < SM_FP32 || precision > SM_BFP16)
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
    static std::atomic<uint64_t> serials{1};
    if (h) h->serial = serials.fetch_add(1);
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
    SM_CUDA_TRY(cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device));

    const size_t cplx = precision == SM_FP64 ? 8 : 4;    // compute type bytes
    const size_t fcells = NX * (size_t)h->pitch;
    int rc;
    h->fset_stride = fcells * nshots * h->elem;
    h->mat_stride = fcells * cplx;
    // block storage keeps the split parts in FP32
    const size_t pelem = precision == SM_BFP16 ? 4 : h->elem;
    // FP32 storage: slabs of 4 rows at 64 registers, the fastest measured
    // (the other storage types keep configuration 0)
    if (precision == SM_FP32) h->config = 16;
    if (precision == SM_BFP16) {
        h->config = 5;   // block-storage slab 2 x 8, 12 CTAs per SM: the fastest measured
        h->nxb = (NX + EISO_EB - 1) / EISO_EB;
        h->args.nxb = (int)h->nxb;
        h->args.estride = (long long)(nshots * h->nxb * (size_t)h->pitch);
    }
    for (int k = 0; k < 2; ++k) {
        if ((rc = h->fset[k].alloc_pooled(5 * h->fset_stride, device))) return rc;
        for (int f = 0; f < 5; ++f) {
            if ((rc = h->xpart[k][f].alloc_pooled(h->npml_cells * nshots * pelem, device))) return rc;
            if ((rc = h->zpart[k][f].alloc_pooled(h->npml_cells * nshots * pelem, device))) return rc;
        }
        if (precision == SM_BFP16 &&
            (rc = h->fexp[k].alloc_pooled(5 * (size_t)h->args.estride, device)))
            return rc;
    }
    if ((rc = h->matbuf.alloc_pooled(5 * h->mat_stride, device))) return rc;
    EisoProf P{(int)NX, (int)NZ};
    if ((rc = h->prof.alloc((size_t)P.size() * cplx))) return rc;
    if ((rc = h->err.alloc(sizeof(int)))) return rc;
    if ((rc = h->err.zero(h->stream))) return rc;
    if ((rc = h->d_step.alloc(sizeof(long long)))) return rc;
    if ((rc = h->d_step.zero(h->stream))) return rc;

    // ---- materials on the padded grid: edge replicated, scaled by dt/h ----
    {
        const double *src[5] = {b, bm, la, l2m, mu};
        std::vector<double> m(fcells, 0.0);
        for (int k = 0; k < 5; ++k) {
            eiso_pad_material(nx, nz, npml, (size_t)h->pitch, dt / hh, src[k], k, m.data());
            rc = precision == SM_FP64 ? upload_convert<double>(h->mat(k), m.data(), fcells, h->stream)
                                      : upload_convert<float>(h->mat(k), m.data(), fcells, h->stream);
            if (rc) return rc;
        }
    }
    // ---- damping tables: A = (2 - dt d)/(2 + dt d), B = 2/(2 + dt d) ----
    {
        const std::vector<double> t = eiso_damping_tables(nx, nz, npml, dt, d, dh, dH);
        rc = precision == SM_FP64 ? upload_convert<double>(h->prof.p, t.data(), t.size(), h->stream)
                                  : upload_convert<float>(h->prof.p, t.data(), t.size(), h->stream);
        if (rc) return rc;
    }
    EisoArgs &a = h->args;
    a.NX = (int)NX; a.NZ = (int)NZ; a.pitch = h->pitch;
    a.np = (int)npml; a.nx = (int)nx; a.nz = (int)nz;
    a.nshots = (int)nshots;
    a.fstride = (long long)fcells;
    a.sstride = (long long)h->npml_cells;
    a.mid_off = (int)(npml * NZ);
    a.right_off = (int)(npml * NZ + nx * 2 * npml);
    eiso_bind(h.get());
    for (int f = 0; f < 5; ++f) {
        a.mat[f] = h->mat(f);
        a.sc[f] = 1.0f;
        a.isc[f] = 1.0f;
    }
    a.prof = h->prof.p;
    a.err = h->err.as<int>();
    a.step = h->d_step.as<long long>();
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
    for (int k = 0; k < 2; ++k) {
        if (int rc = h->fset[k].zero(h->stream)) return rc;
        if (int rc = h->fexp[k].zero(h->stream)) return rc;
        if (int rc = h->pside[k].zero(h->stream)) return rc;
        for (int f = 0; f < 5; ++f) {
            if (int rc = h->xpart[k][f].zero(h->stream)) return rc;
            if (int rc = h->zpart[k][f].zero(h->stream)) return rc;
        }
    }
    h->cur = 0;
    eiso_bind(h);
    if (int rc = h->d_traces.zero(h->stream)) return rc;
    if (int rc = h->err.zero(h->stream)) return rc;
    if (int rc = h->d_step.zero(h->stream)) return rc;
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->it = 0;
    if (eiso_is16(h)) {
        if (h->scaler.expo != h->expo0) h->graph_epoch++;
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
        SrcEntry se;
        if (int rc = eiso_source_entry(h->nx, h->nz, h->np, (size_t)h->pitch, index[s], type[s],
                                       fct + s * stride, length[s], stride, scale,
                                       "sm_eiso_set_sources", &se, vals))
            return rc;
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
        RecEntry e;
        if (int rc = eiso_receiver_entry(h->nx, h->nz, h->np, (size_t)h->pitch, index[r], comp[r],
                                         sr.plan.group_of[r], "sm_eiso_set_receivers", &e))
            return rc;
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

namespace {

// one time step: update, sources, receivers
template <typename S>
int eiso_step_once(sm_eiso *h) {
    if (int rc = launch_step<S>(h)) return rc;
    launch_src<S>(h);
    launch_gather<S>(h);
    return SM_OK;
}

// the graph of h->graph_steps steps starting from buffer set h->cur
template <typename S>
int eiso_graph(sm_eiso *h, cudaGraphExec_t *out) {
    sm_eiso::Graph &gr = h->graphs[h->cur];
    if (gr.exec && gr.epoch == h->graph_epoch && gr.steps == h->graph_steps &&
        gr.timed == h->timer.on) {
        *out = gr.exec;
        return SM_OK;
    }
    if (gr.exec) {
        cudaGraphExecDestroy(gr.exec);
        gr.exec = nullptr;
    }
    h->timer.release(gr.tev);
    const size_t launches = h->timer.launches;
    const int cur = h->cur;
    SM_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    gr.timed = h->timer.on;
    h->timer.capture = gr.timed ? &gr.tev : nullptr;
    int rc = SM_OK;
    for (int k = 0; k < h->graph_steps && rc == SM_OK; ++k) rc = eiso_step_once<S>(h);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    h->timer.capture = nullptr;
    h->timer.launches = launches;
    h->cur = cur;   // an even number of steps: back to the starting set
    eiso_bind(h);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return sm_fail(SM_ECUDA, "stream capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&gr.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        gr.exec = nullptr;
        return sm_fail(SM_ECUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    }
    gr.epoch = h->graph_epoch;
    gr.steps = h->graph_steps;
    *out = gr.exec;
    return SM_OK;
}

template <typename S>
int eiso_run_t(sm_eiso *h, size_t nsteps) {
    if (int rc = eiso_ready<S>(h)) return rc;
    const size_t G = (size_t)h->graph_steps;
    const size_t per_step = 1 + (h->d_src.bytes ? 1 : 0) + (h->n_rec_total ? 1 : 0);
    while (nsteps > 0) {
        // graphs start anywhere, except in 16-bit storage, whose range
        // checks fall on multiples of the scale period between graphs
        if (G && nsteps >= G && (!eiso_is16(h) || h->it % G == 0)) {
            cudaGraphExec_t ex = nullptr;
            if (int rc = eiso_graph<S>(h, &ex)) return rc;
            SM_CUDA_TRY(cudaGraphLaunch(ex, h->stream));
            if (h->timer.on) h->timer.replayed(h->graphs[h->cur].tev);
            h->timer.launches += per_step * G;
            h->it += G;
            nsteps -= G;
        } else {
            if (int rc = eiso_step_once<S>(h)) return rc;
            h->it++;
            nsteps--;
        }
        if (eiso_is16(h) && h->it % sm_eiso::kScalePeriod == 0)
            if (int rc = eiso_rescale(h)) return rc;
    }
    return SM_OK;
}

}  // namespace

extern "C" int sm_eiso_run(sm_eiso_t h, size_t nsteps) {
    if (int rc = eiso_check(h)) return rc;
    DeviceGuard g(h->device);
    if (h->src_dirty)
        if (int rc = upload_sources(h)) return rc;
    if (h->rec_dirty)
        if (int rc = upload_receivers(h)) return rc;
    int rc;
    switch (h->precision) {
    case SM_FP64: rc = eiso_run_t<double>(h, nsteps); break;
    case SM_FP16: rc = eiso_run_t<__half>(h, nsteps); break;
    case SM_BF16: rc = eiso_run_t<__nv_bfloat16>(h, nsteps); break;
    case SM_BFP16: rc = eiso_run_t<Bfp16>(h, nsteps); break;
    default: rc = eiso_run_t<float>(h, nsteps); break;
    }
    if (rc) return rc;
    SM_CUDA_TRY(cudaGetLastError());
    return SM_OK;
}

namespace {

// one grouped step of the problems hs[0..n) (n <= kGroupMax), all on stream st
template <typename S>
int eiso_group_step(sm_eiso *const *hs, int n, cudaStream_t st) {
    constexpr bool B = std::is_same<S, Bfp16>::value;
    using T = std::conditional_t<B, int16_t, S>;
    using L = ESlabG<T, 2, 8>;
    static EisoGroupStepParams P;   // large: built in place, one caller at a time
    static EisoGroupPostParams Q;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    int total = 0;
    for (int k = 0; k < n; ++k) {
        sm_eiso *h = hs[k];
        if constexpr (B) {
            P.f[k] = h->bmaps[h->cur].f;
            P.e[k] = h->bmaps[h->cur].e;
        } else {
            P.f[k] = h->slab_maps[h->cur].f;
        }
        P.a[k] = h->args;
        P.gx[k] = ((h->NZ + 29) / 30 + 1) / 2;
        P.gy[k] = (h->NX + 7) / 8;
        P.first[k] = total;
        total += P.gx[k] * P.gy[k] * (int)h->nshots;
    }
    P.first[n] = total;
    P.n = n;
    if constexpr (B)
        eiso_bgroup_step_kernel<2, 8, 8><<<total, 64, ESlabB<2, 8>::bytes, st>>>(P);
    else
        eiso_group_step_kernel<S, 2, 8, 8><<<total, 64, L::bytes, st>>>(P);
    int nsrc = 0, nrec = 0;
    for (int k = 0; k < n; ++k) {
        sm_eiso *h = hs[k];
        h->cur = 1 - h->cur;
        eiso_bind(h);
        EisoPost &q = Q.q[k];
        for (int f = 0; f < 5; ++f) {
            q.f[f] = h->args.f[f];
            q.sc[f] = h->args.sc[f];
            q.isc[f] = h->args.isc[f];
        }
        q.fstride = h->args.fstride;
        q.step = h->args.step;
        q.src = h->d_src.as<SrcEntry>();
        q.src_first = h->d_src_first.as<int>();
        q.vals = h->d_vals.as<double>();
        q.rec = h->d_rec.as<RecEntry>();
        q.table = h->d_table.as<int32_t>();
        q.nsteps_max = h->table_steps;
        q.traces = h->d_traces.as<double>();
        q.fe = h->args.fe;
        q.estride = h->args.estride;
        q.eshot = (long long)h->nxb * h->pitch;
        q.pitch = h->pitch;
        q.err = h->args.err;
        q.pv = h->args.pfirst ? h->args.pv : nullptr;
        Q.first_src[k] = nsrc;
        Q.first_rec[k] = nrec;
        nsrc += h->d_src.bytes ? (int)h->nshots : 0;
        nrec += h->n_rec_total;
    }
    Q.first_src[n] = nsrc;
    Q.first_rec[n] = nrec;
    Q.n = n;
    if (nsrc) eiso_group_source_kernel<S><<<(nsrc + 127) / 128, 128, 0, st>>>(Q);
    if (nrec) eiso_group_gather_kernel<S><<<(nrec + 127) / 128, 128, 0, st>>>(Q);
    hs[0]->timer.launches += 1 + (nsrc ? 1 : 0) + (nrec ? 1 : 0);
    SM_CUDA_TRY(cudaGetLastError());
    return SM_OK;
}

// CUDA graphs of kGroupGraphSteps grouped steps, cached per group: the key
// holds each handle's serial, starting buffer set and graph epoch (sources,
// receivers, scales), so a graph is only replayed on the state it was
// captured for.  A few are kept, the least recently used dropped.
constexpr int kGroupGraphSteps = 16;
constexpr size_t kGroupGraphCache = 8;

struct GroupGraphKey {
    int device;
    std::vector<std::tuple<uint64_t, int, unsigned>> members;
    bool operator<(const GroupGraphKey &o) const {
        return std::tie(device, members) < std::tie(o.device, o.members);
    }
};
struct GroupGraph {
    cudaGraphExec_t exec = nullptr;
    uint64_t used = 0;
};
std::mutex g_group_mu;
std::map<GroupGraphKey, GroupGraph> g_group_graphs;
uint64_t g_group_clock = 0;

template <typename S>
int eiso_group_steps(sm_eiso *const *hs, int n, int steps) {
    for (int s = 0; s < steps; ++s)
        for (int k0 = 0; k0 < n; k0 += kGroupMax)
            if (int rc = eiso_group_step<S>(hs + k0, std::min(kGroupMax, n - k0), hs[0]->stream))
                return rc;
    return SM_OK;
}

template <typename S>
int eiso_group_graph(sm_eiso *const *hs, int n, cudaGraphExec_t *out) {
    GroupGraphKey key{hs[0]->device, {}};
    for (int k = 0; k < n; ++k) key.members.emplace_back(hs[k]->serial, hs[k]->cur, hs[k]->graph_epoch);
    std::lock_guard<std::mutex> lk(g_group_mu);
    auto it = g_group_graphs.find(key);
    if (it != g_group_graphs.end()) {
        it->second.used = ++g_group_clock;
        *out = it->second.exec;
        return SM_OK;
    }
    const size_t launches = hs[0]->timer.launches;
    SM_CUDA_TRY(cudaStreamBeginCapture(hs[0]->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = eiso_group_steps<S>(hs, n, kGroupGraphSteps);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(hs[0]->stream, &graph);
    hs[0]->timer.launches = launches;
    for (int k = 0; k < n; ++k) eiso_bind(hs[k]);   // an even number of steps: sets as before
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return sm_fail(SM_ECUDA, "stream capture: %s", cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return sm_fail(SM_ECUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    if (g_group_graphs.size() >= kGroupGraphCache) {
        auto old = g_group_graphs.begin();
        for (auto i = g_group_graphs.begin(); i != g_group_graphs.end(); ++i)
            if (i->second.used < old->second.used) old = i;
        // some stream may still run it: wait before the executable goes
        cudaDeviceSynchronize();
        cudaGraphExecDestroy(old->second.exec);
        g_group_graphs.erase(old);
    }
    g_group_graphs[key] = GroupGraph{exec, ++g_group_clock};
    *out = exec;
    return SM_OK;
}

template <typename S>
int eiso_group_run_t(sm_eiso *const *hs, int n, size_t nsteps) {
    if constexpr (std::is_same<S, Bfp16>::value) {
        for (int k = 0; k < n; ++k)
            if (int rc = eiso_make_bmaps<2, 8>(hs[k])) return rc;
        if (int rc = allow_smem(eiso_bgroup_step_kernel<2, 8, 8>, ESlabB<2, 8>::bytes,
                                hs[0]->device))
            return rc;
    } else {
        using L = ESlabG<S, 2, 8>;
        for (int k = 0; k < n; ++k)
            if (int rc = eiso_make_slab_maps<S, L, (1 << 20) + 2 * 4096 + 8>(hs[k])) return rc;
        if (int rc = allow_smem(eiso_group_step_kernel<S, 2, 8, 8>, L::bytes, hs[0]->device))
            return rc;
    }
    const bool is16 = eiso_is16(hs[0]);
    const size_t G = kGroupGraphSteps;
    int per_step = 1;
    for (int k0 = 0; k0 < n; k0 += kGroupMax) {
        bool src = false, rec = false;
        for (int k = k0; k < std::min(n, k0 + kGroupMax); ++k) {
            src = src || hs[k]->d_src.bytes;
            rec = rec || hs[k]->n_rec_total;
        }
        per_step += (k0 ? 1 : 0) + (src ? 1 : 0) + (rec ? 1 : 0);
    }
    while (nsteps > 0) {
        // a graph of G steps when no handle rescales inside it
        bool aligned = true;
        for (int k = 0; k < n && is16; ++k) aligned = aligned && hs[k]->it % G == 0;
        size_t done;
        if (nsteps >= G && aligned) {
            cudaGraphExec_t ex = nullptr;
            if (int rc = eiso_group_graph<S>(hs, n, &ex)) return rc;
            SM_CUDA_TRY(cudaGraphLaunch(ex, hs[0]->stream));
            hs[0]->timer.launches += per_step * G;
            done = G;
        } else {
            if (int rc = eiso_group_steps<S>(hs, n, 1)) return rc;
            done = 1;
        }
        nsteps -= done;
        for (int k = 0; k < n; ++k) {
            sm_eiso *h = hs[k];
            const size_t before = h->it;
            h->it += done;
            if (is16 && h->it / sm_eiso::kScalePeriod != before / sm_eiso::kScalePeriod)
                if (int rc = eiso_rescale(h)) return rc;
        }
    }
    return SM_OK;
}

}  // namespace

// Several e_iso handles of different grid sizes advanced together: every step
// is one launch over all their slabs (up to 32 handles per launch), one for
// all their sources and one for all their receivers.  Each handle ends where
// sm_eiso_run(h, nsteps) would have left it, bit for bit.  The work runs on
// the first handle's stream, ordered after the work already queued on every
// handle's stream; every handle's stream waits for it to finish.
extern "C" int sm_eiso_group_run(sm_eiso_t const *handles, int n, size_t nsteps) {
    if (!handles || n <= 0) return sm_fail(SM_EINVAL, "sm_eiso_group_run: no handles");
    for (int k = 0; k < n; ++k) {
        if (int rc = eiso_check(handles[k])) return rc;
        if (handles[k]->device != handles[0]->device ||
            handles[k]->precision != handles[0]->precision)
            return sm_fail(SM_EINVAL,
                           "sm_eiso_group_run: handle %d differs in device or precision from "
                           "handle 0", k);
        for (int j = 0; j < k; ++j)
            if (handles[j] == handles[k])
                return sm_fail(SM_EINVAL, "sm_eiso_group_run: handle %d appears twice", k);
    }
    if (nsteps == 0) return SM_OK;
    sm_eiso *const *hs = handles;
    DeviceGuard g(hs[0]->device);
    for (int k = 0; k < n; ++k) {
        if (hs[k]->src_dirty)
            if (int rc = upload_sources(hs[k])) return rc;
        if (hs[k]->rec_dirty)
            if (int rc = upload_receivers(hs[k])) return rc;
    }
    // run every handle on the first handle's stream for the duration
    const cudaStream_t st = hs[0]->stream;
    std::vector<cudaStream_t> own(n);
    cudaEvent_t ev = nullptr;
    SM_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    for (int k = 1; k < n; ++k) {
        cudaEventRecord(ev, hs[k]->stream);
        cudaStreamWaitEvent(st, ev, 0);
    }
    for (int k = 0; k < n; ++k) {
        own[k] = hs[k]->stream;
        hs[k]->stream = st;
    }
    int rc;
    switch (hs[0]->precision) {
    case SM_FP64: rc = eiso_group_run_t<double>(hs, n, nsteps); break;
    case SM_FP16: rc = eiso_group_run_t<__half>(hs, n, nsteps); break;
    case SM_BF16: rc = eiso_group_run_t<__nv_bfloat16>(hs, n, nsteps); break;
    case SM_BFP16: rc = eiso_group_run_t<Bfp16>(hs, n, nsteps); break;
    default: rc = eiso_group_run_t<float>(hs, n, nsteps); break;
    }
    for (int k = 0; k < n; ++k) hs[k]->stream = own[k];
    cudaEventRecord(ev, st);
    for (int k = 1; k < n; ++k) cudaStreamWaitEvent(hs[k]->stream, ev, 0);
    cudaEventDestroy(ev);
    if (rc) return rc;
    SM_CUDA_TRY(cudaGetLastError());
    return SM_OK;
}

// Launch-configuration search: every configuration that fits the device
// runs trial_steps steps from
// a zero state, timed with CUDA events; the fastest is kept.  Results are
// cached per (precision, grid, shots) for the life of the process.
extern "C" int sm_eiso_autotune(sm_eiso_t h, int trial_steps, int *config,
                                double *ms_per_step) {
    if (int rc = eiso_check(h)) return rc;
    if (h->it != 0)
        return sm_fail(SM_ESTATE, "sm_eiso_autotune: call before the first step (or after reset)");
    if (trial_steps <= 0) trial_steps = 32;
    DeviceGuard g(h->device);
    struct Key {
        int prec, NX, NZ, np;
        size_t shots;
        int dev;
        bool operator<(const Key &o) const {
            return std::tie(prec, NX, NZ, np, shots, dev) <
                   std::tie(o.prec, o.NX, o.NZ, o.np, o.shots, o.dev);
        }
    };
    struct Val {
        int config;
        double ms;
    };
    static std::map<Key, Val> cache;
    static std::mutex mu;
    const Key key{h->precision, h->NX, h->NZ, (int)h->np, h->nshots, h->device};
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            h->config = it->second.config;
            h->graph_epoch++;
            if (config) *config = h->config;
            if (ms_per_step) *ms_per_step = it->second.ms;
            return SM_OK;
        }
    }
    int lim = 0;
    SM_CUDA_TRY(cudaDeviceGetAttribute(&lim, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    cudaEvent_t e0, e1;
    SM_CUDA_TRY(cudaEventCreate(&e0));
    SM_CUDA_TRY(cudaEventCreate(&e1));
    const bool timing = h->timer.on;
    h->timer.on = false;
    Val best{-1, 0.0};
    int rc = SM_OK;
    for (int c = 0; c < eiso_ncfg(h) && rc == SM_OK; ++c) {
        if (eiso_config_smem_prec(h->precision, c) > (size_t)lim) continue;
        h->config = c;
        h->graph_epoch++;
        if ((rc = sm_eiso_reset(h))) break;
        // warm-up, and the time loop's graph (if the handle uses graphs)
        // captured outside the timed trial
        if ((rc = sm_eiso_run(h, 2 + (size_t)h->graph_steps))) break;
        cudaEventRecord(e0, h->stream);
        if ((rc = sm_eiso_run(h, (size_t)trial_steps))) break;
        cudaEventRecord(e1, h->stream);
        if ((rc = sm_eiso_sync(h))) break;
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        const double ms = t / trial_steps;
        if (best.config < 0 || ms < best.ms) best = Val{c, ms};
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->timer.on = timing;
    if (rc) return rc;
    if (best.config < 0) return sm_fail(SM_EINVAL, "sm_eiso_autotune: no configuration fits");
    h->config = best.config;
    h->graph_epoch++;
    if ((rc = sm_eiso_reset(h))) return rc;
    {
        std::lock_guard<std::mutex> lk(mu);
        cache[key] = best;
    }
    if (config) *config = best.config;
    if (ms_per_step) *ms_per_step = best.ms;
    return SM_OK;
}

extern "C" int sm_eiso_set_graph(sm_eiso_t h, int steps) {
    if (int rc = eiso_check(h)) return rc;
    if (steps != 0 && steps != 2 && steps != 4 && steps != 8 && steps != 16)
        return sm_fail(SM_EINVAL, "sm_eiso_set_graph: steps must be 0, 2, 4, 8 or 16 (got %d)",
                       steps);
    h->graph_steps = steps;
    h->graph_epoch++;
    return SM_OK;
}

extern "C" int sm_eiso_sync(sm_eiso_t h) {
    if (int rc = eiso_check(h)) return rc;
    DeviceGuard g(h->device);
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return eiso_check_err(h);
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
    if (int rc = eiso_check_err(h)) return rc;
    const size_t ms = sr.plan.max_samples;
    // samples taken so far, per sampling group of the shot
    const size_t lim = std::min(h->it, sr.plan.nsteps_max);
    std::vector<size_t> gcount(sr.plan.count_total.size(), 0);
    for (size_t gi = 0; gi < gcount.size(); ++gi)
        for (size_t it = 0; it < lim; ++it)
            if (sr.plan.table[gi * sr.plan.nsteps_max + it] >= 0) ++gcount[gi];
    size_t cmax = 0;
    bool same = true;
    for (size_t r = 0; r < nrec; ++r) {
        const size_t c = gcount[sr.entries[rec0 + r].group];
        if (counts) counts[r] = c;
        if (out && ld < c) return sm_fail(SM_EINVAL, "sm_eiso_read_traces: ld smaller than sample count");
        same = same && (r == 0 || c == cmax);
        cmax = std::max(cmax, c);
    }
    if (!out || !nrec || !cmax) return SM_OK;
    // the shot's receivers are consecutive rows of ms samples on the device
    const double *src = h->d_traces.as<double>() + h->rec_out_base[shot] + (long long)rec0 * (long long)ms;
    if (same) {
        SM_CUDA_TRY(cudaMemcpy2D(out, ld * sizeof(double), src, ms * sizeof(double),
                                 cmax * sizeof(double), nrec, cudaMemcpyDeviceToHost));
    } else {
        for (size_t r = 0; r < nrec; ++r) {
            const size_t c = gcount[sr.entries[rec0 + r].group];
            if (c)
                SM_CUDA_TRY(cudaMemcpy(out + r * ld, src + r * ms, c * sizeof(double),
                                       cudaMemcpyDeviceToHost));
        }
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
    if (eiso_isb(h)) {   // totals: mantissa times 2^(e8 - 126); split parts FP32
        if (part == SM_PART_TOTAL) {
            std::vector<int16_t> m(NX * (size_t)h->pitch);
            std::vector<uint8_t> ex(h->nxb * (size_t)h->pitch);
            SM_CUDA_TRY(cudaMemcpy(m.data(), static_cast<char *>(h->field(h->cur, f)) +
                                                 shot * h->args.fstride * 2,
                                   m.size() * 2, cudaMemcpyDeviceToHost));
            SM_CUDA_TRY(cudaMemcpy(ex.data(), static_cast<char *>(h->fexp[h->cur].p) +
                                                  f * h->args.estride + shot * ex.size(),
                                   ex.size(), cudaMemcpyDeviceToHost));
            for (size_t X = 0; X < NX; ++X)
                for (size_t Z = 0; Z < NZ; ++Z)
                    out[X * NZ + Z] = bfp_value_host(m[X * h->pitch + Z],
                                                     ex[(X / EISO_EB) * h->pitch + Z]);
            if (h->args.pfirst) {   // cells of source patches: their FP32 values
                std::vector<float> pv(h->pside[h->cur].bytes / sizeof(float));
                SM_CUDA_TRY(cudaMemcpy(pv.data(), h->pside[h->cur].p, h->pside[h->cur].bytes,
                                       cudaMemcpyDeviceToHost));
                for (int q = h->p_first[shot]; q < h->p_first[shot + 1]; ++q)
                    for (long X = h->p_xz[2 * q]; X < h->p_xz[2 * q] + EISO_PR; ++X)
                        for (long Z = h->p_xz[2 * q + 1]; Z < h->p_xz[2 * q + 1] + EISO_PC; ++Z)
                            if (X >= 0 && X < (long)NX && Z >= 0 && Z < (long)NZ)
                                out[X * NZ + Z] = pv[eiso_patch_index(h, q, X, Z) + f * EISO_PF];
            }
            return SM_OK;
        }
        const DevBuf &src = part == SM_PART_X ? h->xpart[h->cur][f] : h->zpart[h->cur][f];
        std::vector<float> buf(h->npml_cells);
        SM_CUDA_TRY(cudaMemcpy(buf.data(), static_cast<char *>(src.p) + shot * h->npml_cells * 4,
                               buf.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t X = 0; X < NX; ++X)
            for (size_t Z = 0; Z < NZ; ++Z)
                out[X * NZ + Z] = in_frame(h, X, Z) ? (double)buf[pml_index_host(h, X, Z)] : 0.0;
        return SM_OK;
    }
    if (part == SM_PART_TOTAL) {
        std::vector<unsigned char> buf(NX * (size_t)h->pitch * e);
        SM_CUDA_TRY(cudaMemcpy(buf.data(),
                               static_cast<char *>(h->field(h->cur, f)) + shot * h->args.fstride * e,
                               buf.size(), cudaMemcpyDeviceToHost));
        for (size_t X = 0; X < NX; ++X)
            for (size_t Z = 0; Z < NZ; ++Z)
                out[X * NZ + Z] = to_double(buf.data(), X * h->pitch + Z, h->precision,
                                            h->args.isc[f]);
        return SM_OK;
    }
    const DevBuf &src = part == SM_PART_X ? h->xpart[h->cur][f] : h->zpart[h->cur][f];
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
    if (eiso_isb(h)) {
        // split parts FP32; the totals (the interior value, or the sum of
        // the parts in the frame) encoded block by block as the step does
        std::vector<double> cur(NX * NZ);
        if (part != SM_PART_TOTAL)
            if (int rc = sm_eiso_get_field(h, shot, comp, SM_PART_TOTAL, cur.data())) return rc;
        std::vector<float> px(h->npml_cells), pz(h->npml_cells);
        char *dpx = static_cast<char *>(h->xpart[h->cur][f].p) + shot * h->npml_cells * 4;
        char *dpz = static_cast<char *>(h->zpart[h->cur][f].p) + shot * h->npml_cells * 4;
        SM_CUDA_TRY(cudaMemcpy(px.data(), dpx, px.size() * 4, cudaMemcpyDeviceToHost));
        SM_CUDA_TRY(cudaMemcpy(pz.data(), dpz, pz.size() * 4, cudaMemcpyDeviceToHost));
        std::vector<float> tot(NX * NZ);
        for (size_t X = 0; X < NX; ++X)
            for (size_t Z = 0; Z < NZ; ++Z) {
                const double v = in[X * NZ + Z];
                if (!in_frame(h, X, Z)) {
                    tot[X * NZ + Z] = (float)(part == SM_PART_TOTAL ? v : cur[X * NZ + Z]);
                    continue;
                }
                const size_t c = pml_index_host(h, X, Z);
                if (part == SM_PART_X) px[c] = (float)v;
                if (part == SM_PART_Z) pz[c] = (float)v;
                tot[X * NZ + Z] = px[c] + pz[c];
            }
        std::vector<int16_t> m(NX * (size_t)h->pitch, 0);
        std::vector<uint8_t> ex(h->nxb * (size_t)h->pitch, 0);
        for (size_t xb = 0; xb < h->nxb; ++xb)
            for (size_t Z = 0; Z < NZ; ++Z) {
                const size_t xa = xb * EISO_EB, xe = std::min(xa + EISO_EB, NX);
                float mx = 0.f;
                for (size_t X = xa; X < xe; ++X) mx = std::max(mx, std::fabs(tot[X * NZ + Z]));
                const unsigned e8 = bfp_e8_host(mx);
                ex[xb * h->pitch + Z] = (uint8_t)e8;
                for (size_t X = xa; X < xe; ++X) m[X * h->pitch + Z] = bfp_man_host(tot[X * NZ + Z], e8);
            }
        SM_CUDA_TRY(cudaMemcpy(static_cast<char *>(h->field(h->cur, f)) + shot * h->args.fstride * 2,
                               m.data(), m.size() * 2, cudaMemcpyHostToDevice));
        SM_CUDA_TRY(cudaMemcpy(static_cast<char *>(h->fexp[h->cur].p) + f * h->args.estride +
                                   shot * ex.size(),
                               ex.data(), ex.size(), cudaMemcpyHostToDevice));
        SM_CUDA_TRY(cudaMemcpy(dpx, px.data(), px.size() * 4, cudaMemcpyHostToDevice));
        SM_CUDA_TRY(cudaMemcpy(dpz, pz.data(), pz.size() * 4, cudaMemcpyHostToDevice));
        if (h->args.pfirst) {   // cells of source patches keep the FP32 totals
            std::vector<float> pv(h->pside[h->cur].bytes / sizeof(float));
            SM_CUDA_TRY(cudaMemcpy(pv.data(), h->pside[h->cur].p, h->pside[h->cur].bytes,
                                   cudaMemcpyDeviceToHost));
            for (int q = h->p_first[shot]; q < h->p_first[shot + 1]; ++q)
                for (long X = h->p_xz[2 * q]; X < h->p_xz[2 * q] + EISO_PR; ++X)
                    for (long Z = h->p_xz[2 * q + 1]; Z < h->p_xz[2 * q + 1] + EISO_PC; ++Z)
                        if (X >= 0 && X < (long)NX && Z >= 0 && Z < (long)NZ)
                            pv[eiso_patch_index(h, q, X, Z) + f * EISO_PF] = tot[X * NZ + Z];
            SM_CUDA_TRY(cudaMemcpy(h->pside[h->cur].p, pv.data(), h->pside[h->cur].bytes,
                                   cudaMemcpyHostToDevice));
        }
        return SM_OK;
    }
    std::vector<unsigned char> tot(NX * (size_t)h->pitch * e), px(h->npml_cells * e),
        pz(h->npml_cells * e);
    char *dtot = static_cast<char *>(h->field(h->cur, f)) + shot * h->args.fstride * e;
    char *dpx = static_cast<char *>(h->xpart[h->cur][f].p) + shot * h->npml_cells * e;
    char *dpz = static_cast<char *>(h->zpart[h->cur][f].p) + shot * h->npml_cells * e;
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

extern "C" int sm_eiso_set_config(sm_eiso_t h, int config) {
    if (int rc = eiso_check(h)) return rc;
    if (config < 0 || config >= eiso_ncfg(h))
        return sm_fail(SM_EINVAL, "sm_eiso_set_config: config %d not in [0, %d)", config,
                       eiso_ncfg(h));
    DeviceGuard g(h->device);
    int lim = 0;
    SM_CUDA_TRY(cudaDeviceGetAttribute(&lim, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    const size_t need = eiso_config_smem_prec(h->precision, config);
    if (need > (size_t)lim)
        return sm_fail(SM_EINVAL,
                       "sm_eiso_set_config: config %d needs %zu bytes of shared memory per block "
                       "(device limit %d)",
                       config, need, lim);
    h->config = config;
    h->graph_epoch++;
    return SM_OK;
}

extern "C" int sm_eiso_get_config(sm_eiso_t h, int *config, int *nconfigs) {
    if (int rc = eiso_check(h)) return rc;
    if (config) *config = h->config;
    if (nconfigs) *nconfigs = eiso_ncfg(h);
    return SM_OK;
}

extern "C" int sm_eiso_set_timing(sm_eiso_t h, int on) {
    if (int rc = eiso_check(h)) return rc;
    DeviceGuard g(h->device);
    h->timer.set(on != 0);
    return SM_OK;
}

extern "C" int sm_eiso_kernel_stats(sm_eiso_t h, int reset, double *update_ms,
                                    size_t *update_launches, size_t *all_launches) {
    if (int rc = eiso_check(h)) return rc;
    DeviceGuard g(h->device);
    return h->timer.stats(reset, update_ms, update_launches, all_launches);
}

// ===========================================================================
// Allocation-free single-shot run (no counterpart in the reference).
//
// Some callers of this library cannot call cudaMalloc: a host program whose
// device memory is all owned by its own allocator (a solver or a serving
// framework that hands out every byte itself), or code that runs where a
// device allocation is not allowed or would stall other work (allocation
// synchronises the device).  sm_eiso_run_noalloc gives them one e_iso shot
// without any device allocation: every device-side array of the run (two
// buffer sets of wavefields, split parts, materials, damping tables, source
// and receiver tables, traces, the step counter and the wait flag) lives in
// the file-scope array below, of fixed size, which every GPU that loads this
// library holds until the process exits.  The kernels are the tiled step
// kernel and the source / receiver kernels of the handle path, unchanged.
// ===========================================================================
namespace {

constexpr size_t kNoallocBytes = (size_t)24 << 20;   // 24 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// device address of g_noalloc_scratch on each device, looked up once per
// device with that device current (the host-side name is only a stand-in)
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[64] = {};

int noalloc_scratch(int device, unsigned char **out) {
    if (device < 0 || device >= 64) return sm_fail(SM_EINVAL, "sm_eiso_run_noalloc: device %d", device);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return sm_fail(SM_ECUDA, "sm_eiso_run_noalloc: cudaGetSymbolAddress: %s",
                           cudaGetErrorString(e));
        g_noalloc_ptr[device] = p;
    }
    *out = static_cast<unsigned char *>(g_noalloc_ptr[device]);
    return SM_OK;
}

// bump allocator over the scratch array (offsets only; nothing is allocated)
struct NoallocLayout {
    size_t off = 0;
    size_t take(size_t bytes) {
        const size_t o = off;
        off = round_up(off + bytes, 256);
        return o;
    }
};

}  // namespace

extern "C" int sm_eiso_run_noalloc(int device, void *stream, const sm_eiso_request *r,
                                   double *traces, size_t ld, size_t *counts) {
    using S = float;
    using L = ETile<S, 8, 32>;
    // launched without raising the kernel's dynamic shared-memory limit, so
    // its tile must stay within the default 48 KB
    static_assert(L::bytes <= 48 * 1024, "noalloc tile needs an opt-in shared-memory size");
    if (!r) return sm_fail(SM_EINVAL, "sm_eiso_run_noalloc: request is NULL");
    const sm_eiso_request &q = *r;
    if (q.precision != SM_FP32)
        return sm_fail(SM_EINVAL, "sm_eiso_run_noalloc: FP32 storage only (precision %d)",
                       q.precision);
    if (q.nx < 2 || q.nz < 2 || q.npml < 1)
        return sm_fail(SM_EINVAL, "sm_eiso_run_noalloc: nx, nz >= 2 and npml >= 1 required");
    if (!(q.h > 0.0) || !(q.dt > 0.0)) return sm_fail(SM_EINVAL, "sm_eiso_run_noalloc: h, dt > 0");
    if (!q.la || !q.mu || !q.l2m || !q.b || !q.bm || !q.d || !q.dh || !q.dH ||
        (q.nsrc && (!q.src_index || !q.src_type || !q.src_fct || !q.src_length)) ||
        (q.nrec && (!q.rec_index || !q.rec_comp || !q.rec_t0 || !q.rec_dt)))
        return sm_fail(SM_EINVAL, "sm_eiso_run_noalloc: NULL array in the request");
    if (q.nrec && !counts) return sm_fail(SM_EINVAL, "sm_eiso_run_noalloc: counts is NULL");
    const size_t nx = q.nx, nz = q.nz, np = q.npml;
    const size_t NX = nx + 2 * np, NZ = nz + 2 * np, pitch = round_up(NZ, 32);
    if (NX > (1u << 20) || NZ > (1u << 20)) return sm_fail(SM_EINVAL, "sm_eiso_run_noalloc: grid too large");
    const size_t fcells = NX * pitch;
    const size_t pml = 4 * np * np + 2 * np * (nx + nz);
    const EisoProf P{(int)NX, (int)NZ};

    // ---- host-side tables (sources, receiver sampling), as the handle path ----
    std::vector<SrcEntry> src;
    std::vector<double> vals;
    for (size_t s = 0; s < q.nsrc; ++s) {
        SrcEntry e;
        if (int rc = eiso_source_entry(nx, nz, np, pitch, q.src_index[s], q.src_type[s],
                                       q.src_fct + s * q.src_stride, q.src_length[s],
                                       q.src_stride, q.src_scale, "sm_eiso_run_noalloc", &e, vals))
            return rc;
        e.shot = 0;
        src.push_back(e);
    }
    SamplePlan plan;
    plan.build(q.nrec, q.rec_t0, q.rec_dt, q.dt, q.nsteps);
    std::vector<RecEntry> rec;
    for (size_t k = 0; k < q.nrec; ++k) {
        RecEntry e;
        if (int rc = eiso_receiver_entry(nx, nz, np, pitch, q.rec_index[k], q.rec_comp[k],
                                         plan.group_of[k], "sm_eiso_run_noalloc", &e))
            return rc;
        e.shot = 0;
        e.out = (long long)k * (long long)plan.max_samples;
        rec.push_back(e);
    }
    if (q.nrec && ld < plan.max_samples && traces)
        return sm_fail(SM_EINVAL, "sm_eiso_run_noalloc: ld %zu < %zu samples per receiver", ld,
                       plan.max_samples);

    // ---- layout in the scratch array, and the size check ----
    NoallocLayout lay;
    const size_t o_set[2] = {lay.take(5 * fcells * sizeof(S)), lay.take(5 * fcells * sizeof(S))};
    size_t o_split[2][10];
    for (int k = 0; k < 2; ++k)
        for (int a = 0; a < 10; ++a) o_split[k][a] = lay.take(pml * sizeof(S));
    const size_t o_mat = lay.take(5 * fcells * sizeof(S));
    const size_t o_prof = lay.take((size_t)P.size() * sizeof(S));
    const size_t o_err = lay.take(sizeof(int));
    const size_t o_step = lay.take(sizeof(long long));
    const size_t o_src = lay.take(std::max<size_t>(src.size(), 1) * sizeof(SrcEntry));
    const size_t o_first = lay.take(2 * sizeof(int));
    const size_t o_vals = lay.take(std::max<size_t>(vals.size(), 1) * sizeof(double));
    const size_t o_rec = lay.take(std::max<size_t>(rec.size(), 1) * sizeof(RecEntry));
    const size_t o_table = lay.take(std::max<size_t>(plan.table.size(), 1) * sizeof(int32_t));
    const size_t o_tr = lay.take(std::max<size_t>(q.nrec * plan.max_samples, 1) * sizeof(double));
    if (lay.off > kNoallocBytes)
        return sm_fail(SM_EINVAL,
                       "sm_eiso_run_noalloc: this shot needs %zu bytes of device scratch, the "
                       "library's fixed scratch holds %zu (use sm_eiso_create for larger shots)",
                       lay.off, kNoallocBytes);

    int ndev = 0;
    SM_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        return sm_fail(SM_EINVAL, "sm_eiso_run_noalloc: no CUDA device %d", device);
    DeviceGuard g(device);
    unsigned char *base = nullptr;
    if (int rc = noalloc_scratch(device, &base)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // ---- inputs into the scratch; what must start at zero is cleared ----
    SM_CUDA_TRY(cudaMemsetAsync(base, 0, o_mat, st));   // both sets and all split parts
    SM_CUDA_TRY(cudaMemsetAsync(base + o_err, 0, o_src - o_err, st));
    SM_CUDA_TRY(cudaMemsetAsync(base + o_tr, 0, lay.off - o_tr, st));
    {
        const double *m5[5] = {q.b, q.bm, q.la, q.l2m, q.mu};
        std::vector<double> m(fcells, 0.0);
        for (int k = 0; k < 5; ++k) {
            eiso_pad_material(nx, nz, np, pitch, q.dt / q.h, m5[k], k, m.data());
            if (int rc = upload_convert<S>(base + o_mat + k * fcells * sizeof(S), m.data(), fcells, st))
                return rc;
        }
        const std::vector<double> t = eiso_damping_tables(nx, nz, np, q.dt, q.d, q.dh, q.dH);
        if (int rc = upload_convert<S>(base + o_prof, t.data(), t.size(), st)) return rc;
    }
    const int first[2] = {0, (int)src.size()};
    if (!src.empty()) {
        SM_CUDA_TRY(cudaMemcpyAsync(base + o_src, src.data(), src.size() * sizeof(SrcEntry),
                                    cudaMemcpyHostToDevice, st));
        SM_CUDA_TRY(cudaMemcpyAsync(base + o_first, first, sizeof(first), cudaMemcpyHostToDevice, st));
        SM_CUDA_TRY(cudaMemcpyAsync(base + o_vals, vals.data(), vals.size() * sizeof(double),
                                    cudaMemcpyHostToDevice, st));
    }
    if (!rec.empty()) {
        SM_CUDA_TRY(cudaMemcpyAsync(base + o_rec, rec.data(), rec.size() * sizeof(RecEntry),
                                    cudaMemcpyHostToDevice, st));
        if (!plan.table.empty())
            SM_CUDA_TRY(cudaMemcpyAsync(base + o_table, plan.table.data(),
                                        plan.table.size() * sizeof(int32_t),
                                        cudaMemcpyHostToDevice, st));
    }
    SM_CUDA_TRY(cudaStreamSynchronize(st));   // host staging goes out of scope below

    // ---- kernel arguments and TMA maps over the scratch ----
    EisoArgs a{};
    a.NX = (int)NX; a.NZ = (int)NZ; a.pitch = (int)pitch;
    a.np = (int)np; a.nx = (int)nx; a.nz = (int)nz;
    a.fstride = (long long)fcells;
    a.sstride = (long long)pml;
    a.mid_off = (int)(np * NZ);
    a.right_off = (int)(np * NZ + nx * 2 * np);
    for (int f = 0; f < 5; ++f) {
        a.mat[f] = base + o_mat + f * fcells * sizeof(S);
        a.sc[f] = a.isc[f] = 1.0f;
    }
    a.prof = base + o_prof;
    a.err = reinterpret_cast<int *>(base + o_err);
    a.step = reinterpret_cast<long long *>(base + o_step);
    EisoMaps maps[2];
    auto field = [&](int set, int f) { return base + o_set[set] + f * fcells * sizeof(S); };
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < 5; ++f)
            if (int rc = make_map_3d(&maps[b].f[f], field(b, f), MapType<S>::v, sizeof(S), NZ, NX,
                                     1, pitch, L::BZ, L::RX))
                return rc;
    auto bind = [&](int cur) {
        for (int f = 0; f < 5; ++f) {
            a.f[f] = field(cur, f);
            a.fo[f] = field(1 - cur, f);
            a.fx[f] = base + o_split[cur][f];
            a.fz[f] = base + o_split[cur][5 + f];
            a.fxo[f] = base + o_split[1 - cur][f];
            a.fzo[f] = base + o_split[1 - cur][5 + f];
        }
    };

    // ---- the time loop: step, sources, receivers ----
    const dim3 grd((unsigned)((NZ + 31) / 32), (unsigned)((NX + 7) / 8), 1);
    int cur = 0;
    for (size_t it = 0; it < q.nsteps; ++it) {
        bind(cur);
        eiso_tile_kernel<S, 8, 32, 128, 6><<<grd, 128, L::bytes, st>>>(a, maps[cur]);
        cur = 1 - cur;
        bind(cur);
        if (!src.empty())
            eiso_source_kernel<S><<<1, 128, 0, st>>>(
                a, reinterpret_cast<const SrcEntry *>(base + o_src),
                reinterpret_cast<const int *>(base + o_first),
                reinterpret_cast<const double *>(base + o_vals), 1);
        if (!rec.empty())
            eiso_gather_kernel<S><<<(unsigned)((rec.size() + 127) / 128), 128, 0, st>>>(
                a, reinterpret_cast<const RecEntry *>(base + o_rec), (int)rec.size(),
                reinterpret_cast<const int32_t *>(base + o_table), (long long)plan.nsteps_max,
                reinterpret_cast<double *>(base + o_tr));
    }
    SM_CUDA_TRY(cudaGetLastError());

    // ---- traces back to the caller ----
    int err = 0;
    SM_CUDA_TRY(cudaMemcpyAsync(&err, base + o_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SM_CUDA_TRY(cudaStreamSynchronize(st));
    if (err) return sm_fail(SM_ETIMEOUT, "sm_eiso_run_noalloc: a bounded wait for a TMA load gave up");
    for (size_t k = 0; k < q.nrec; ++k) {
        size_t c = 0;
        const size_t lim = std::min(q.nsteps, plan.nsteps_max);
        for (size_t it = 0; it < lim; ++it)
            if (plan.table[(size_t)rec[k].group * plan.nsteps_max + it] >= 0) ++c;
        counts[k] = c;
        if (traces && c)
            SM_CUDA_TRY(cudaMemcpyAsync(traces + k * ld,
                                        base + o_tr + (size_t)rec[k].out * sizeof(double),
                                        c * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    SM_CUDA_TRY(cudaStreamSynchronize(st));
    return SM_OK;
}
