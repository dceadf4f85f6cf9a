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
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <tuple>
#include <type_traits>
#include <thread>
#include <vector>

#include "sm_common.cuh"

namespace sm {

// mbarriers reserved at the head of the step kernel's shared memory
#define D_HEAD_BARS 16
// most x planes one CTA marches through
#define A3_CHMAX 64

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
    int sx, sy;                // strides of i and j in elements (grids < 2^31 cells)
    int *err;                  // set by a kernel whose bounded wait gave up
    long long *step;           // steps begun; the step kernel counts, source and
                               // receiver kernels of step it read it + 1
    void *f[4];                // wavefields read this step
    void *psi[6];              // CPML memory variables read this step
    void *fo[4];               // ... and written this step (the other buffer)
    void *pso[6];
    int chunk;                 // x planes per CTA
    // tiles (32 k x TY j): nkt x njt in all; the interior class is the
    // rectangle [kt0, kt1) x [jt0, jt1) of tiles clear of the CPML frame and
    // the grid edge in y and z, the edge class every other tile
    int nkt, njt, kt0, kt1, jt0, jt1;
    int step_cls;              // the class whose first CTA counts the step
    const void *rho;           // compute type, padded layout
    const void *K;
    const void *coef;
    A3Coef cf;
    double two_dt;             // 2 dt
    double idx, idy, idz;      // 1/dx, 1/dy, 1/dz
    float sc[4], isc[4];
    float psc[6], pisc[6];
    // block-floating-point storage: exponent bytes of the fields read and
    // written this step, [nx2][nyb][pitch] (nyb blocks of A3_BJ y rows)
    void *fe[4];
    void *feo[4];
    int nyb;
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

// Shared-memory stage of the fused step: one x plane of every input the
// step reads, delivered by six TMA box loads.  P and rho carry a one-cell
// halo in j (rows j0-1 .. j0+TY) and the 16-byte chunks around the tile in
// k (elements k0-H .. k0+32+H, H = 16 bytes / element size); vy starts at
// row j0-1 and vz at column k0-H, which hold the recomputed halo cells.
template <typename S, int TY>
struct A3Lay {
    using C = typename Store<S>::C;
    static constexpr int HS = 16 / (int)sizeof(S), HC = 16 / (int)sizeof(C);
    static constexpr int WS = 32 + 2 * HS, WC = 32 + 2 * HC, WZ = 32 + HS;
    __host__ __device__ static constexpr size_t al(size_t x) { return (x + 127) / 128 * 128; }
    static constexpr size_t bP = (size_t)(TY + 2) * WS * sizeof(S);
    static constexpr size_t bR = (size_t)(TY + 2) * WC * sizeof(C);
    static constexpr size_t bX = (size_t)TY * 32 * sizeof(S);
    static constexpr size_t bY = (size_t)(TY + 1) * 32 * sizeof(S);
    static constexpr size_t bZ = (size_t)TY * WZ * sizeof(S);
    static constexpr size_t bK = (size_t)TY * 32 * sizeof(C);
    static constexpr size_t oP = 0, oR = al(bP), oX = oR + al(bR), oY = oX + al(bX);
    static constexpr size_t oZ = oY + al(bY), oK = oZ + al(bZ);
    static constexpr size_t stage = oK + al(bK);
    static constexpr unsigned tx = (unsigned)(bP + bR + bX + bY + bZ + bK);
    // head: the stage mbarriers, two vy row buffers [TY+1][32], the CPML
    // coefficient tables of the chunk's planes, the tile's rows and columns,
    // and two buffers [TY] of the halo column vz(k0-1)
    static constexpr size_t oVY = al(D_HEAD_BARS * 8);
    static constexpr size_t oCX = oVY + al((size_t)2 * (TY + 1) * 32 * sizeof(C));
    static constexpr size_t oCY = oCX + al((size_t)6 * (A3_CHMAX + 2) * sizeof(C));
    static constexpr size_t oCZ = oCY + al((size_t)6 * (TY + 1) * sizeof(C));
    static constexpr size_t oVZ = oCZ + al((size_t)6 * 33 * sizeof(C));
    static constexpr size_t head = oVZ + al((size_t)2 * TY * sizeof(C));
};

// one velocity component (a_iso_3d.c:605-651):
//   g = (P_hi - P_lo)/h;  psi = b psi + a g;  g = g/k + psi (frame only);
//   v -= 2 dt/(rho_lo + rho_hi) g
// The owner of a cell and a tile that recomputes it as halo call this same
// function, so both round identically.
template <typename C>
__device__ __forceinline__ C a3_vel(C vold, C p_lo, C p_hi, C r_lo, C r_hi, C ih, C two_dt,
                                    bool frame, C ca, C cb, C cik, C psi_old, C &psi_new) {
    C g = r_mul(r_sub(p_hi, p_lo), ih);
    if (frame) {
        psi_new = r_fma(cb, psi_old, r_mul(ca, g));
        g = r_fma(g, cik, psi_new);
    }
    return r_fma(-r_quot(two_dt, r_add(r_lo, r_hi)), g, vold);
}

// the same update outside the frame (psi = 0, k = 1): identical rounding to
// a3_vel with frame = false
template <typename C>
__device__ __forceinline__ C a3_vel0(C vold, C p_lo, C p_hi, C r_lo, C r_hi, C ih, C two_dt) {
    const C g = r_mul(r_sub(p_hi, p_lo), ih);
    return r_fma(-r_quot(two_dt, r_add(r_lo, r_hi)), g, vold);
}

// the frame correction of one pressure derivative (a_iso_3d.c:667-676)
template <typename C>
__device__ __forceinline__ C a3_dv(C g, C ca, C cb, C cik, C psi_old, C &psi_new) {
    psi_new = r_fma(cb, psi_old, r_mul(ca, g));
    return r_fma(g, cik, psi_new);
}

template <bool B>
using BoolT = std::integral_constant<bool, B>;

struct A3Maps {
    CUtensorMap P, vx, vy, vz, rho, K;
};

// One time step, fused (a_iso_3d.c:599-684).  A CTA of W warps owns a
// 32 (k) x TY (j) column tile, TY = W*R (each warp R consecutive rows), and
// marches along x over planes [i0, i1), i1 - i0 <= A3_CHMAX:
//   * thread 0 keeps a D-stage ring of shared-memory planes filled by TMA
//     (D-2 planes ahead); each stage completes on its own mbarrier;
//   * iteration i computes the velocities of plane i (vx needs P and rho of
//     plane i+1, already in the ring) and the pressure of plane i-1, whose
//     velocities were computed one iteration earlier: vx and vz stay in
//     registers, vy is kept in a shared row buffer (double-buffered by plane
//     parity), so one __syncthreads per plane suffices;
//   * vy on row j0-1 and vz on column k0-1 are recomputed from old values
//     (owned by the neighbouring tiles, which write them to the other
//     buffer, so nothing races): the row by warp 0, the column by lanes
//     0..R-1 of every warp, one row each;
//   * inside the CPML frame the memory variables of the next plane are
//     loaded one iteration ahead, and the coefficients of the tile's planes,
//     rows and columns sit in shared memory, so no global load waits in the
//     loop; each axis on which a tile (y, z) or a plane (x) is clear of the
//     frame and of the grid edge takes the plain update, so a tile on one
//     face of the frame pays the CPML only for that face's component.
// Old and new wavefields and CPML memory variables live in separate buffers
// (ping-pong): every stored value is read once and written once per step.
// Tile classes, one launch each: A3_INNER runs the interior rectangle with
// y and z fast at compile time (only the x frame planes take a general
// update, one component), A3_EDGE the ring of tiles around it with the flags
// read at run time; blockIdx.x numbers the ring's tiles.
enum { A3_INNER = 0, A3_EDGE = 1 };

// Tile (kt, jt) of ring index e, and its face: the ring is numbered by kind
// so that CTAs running side by side mostly take the same code -- first the
// tiles beside the interior rectangle in z (rows inside it: y is fast, face
// A3_FACE_Z), then those beside it in y (columns inside it: z is fast, face
// A3_FACE_Y), then the corners (both axes general, A3_FACE_GEN).
enum { A3_FACE_GEN = 0, A3_FACE_Z = 1, A3_FACE_Y = 2 };
// Whether the ring launch carries a body per face.  Measured on B200 at
// 288^3: no gain over the one general body (0.268 against 0.266 ms per FP32
// step; 0.327 against 0.326 in block storage), and three bodies triple the
// ring kernel's code (instruction-fetch stalls in the capture), so the ring
// takes the general body; the faces stay numbered for it.
#ifndef SM_A3D_FACE_BODIES
#define SM_A3D_FACE_BODIES 0
#endif
__device__ __forceinline__ int a3_edge_tile(const A3Args &a, int e, int &kt, int &jt) {
    const int nkin = a.kt1 - a.kt0, njin = a.jt1 - a.jt0;
    const int nkout = a.nkt - nkin, njout = a.njt - njin;
    auto kout = [&](int c) { return c < a.kt0 ? c : a.kt1 + (c - a.kt0); };
    auto jout = [&](int c) { return c < a.jt0 ? c : a.jt1 + (c - a.jt0); };
    if (e < nkout * njin) {
        kt = kout(e % nkout); jt = a.jt0 + e / nkout;
        return A3_FACE_Z;
    }
    e -= nkout * njin;
    if (e < nkin * njout) {
        kt = a.kt0 + e % nkin; jt = jout(e / nkin);
        return A3_FACE_Y;
    }
    e -= nkin * njout;
    kt = kout(e % nkout); jt = jout(e / nkout);
    return A3_FACE_GEN;
}

template <typename S, int W, int R, int D, int CLS, int FACE, bool FULL = false>
__device__ __forceinline__ void a3d_step_body(const A3Args &a, const A3Maps &m, int kt, int jt,
                                              int ch) {
    constexpr int TY = W * R;
    using C = typename Store<S>::C;
    using St = Store<S>;
    using L = A3Lay<S, TY>;
    static_assert(D >= 3 && D <= D_HEAD_BARS, "ring depth: planes l, l+1 and one in flight");
    static_assert(R <= 32, "rows per warp");
    constexpr int HS = L::HS, HC = L::HC, WS = L::WS, WC = L::WC, WZ = L::WZ;
    constexpr int NXT = A3_CHMAX + 2;   // coefficient table: planes i0-1 .. i1
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    C(*VYs)[TY + 1][32] = reinterpret_cast<C(*)[TY + 1][32]>(smem + L::oVY);
    C(*CX)[NXT] = reinterpret_cast<C(*)[NXT]>(smem + L::oCX);     // [6][NXT]
    C(*CY)[TY + 1] = reinterpret_cast<C(*)[TY + 1]>(smem + L::oCY);  // [6][TY+1]
    C(*CZ)[33] = reinterpret_cast<C(*)[33]>(smem + L::oCZ);          // [6][33]
    C(*VZH)[TY] = reinterpret_cast<C(*)[TY]>(smem + L::oVZ);         // [2][TY]
    unsigned char *ring = smem + L::head;

    const int lane = threadIdx.x, w = threadIdx.y;
    const int tid = w * 32 + lane;
    // the TMA loads are issued by the last warp's lane 0, the halo row is
    // computed by warp 0 and the halo column by warp HW (one lane per row),
    // so the three per-plane extras fall to different warps
    constexpr int HW = W > 2 ? 1 : 0;
    static_assert(TY <= 32, "one halo-column lane per tile row");
    const bool producer = tid == 32 * (W - 1);
    const int k0 = kt * 32, j0 = jt * TY;
    const int lo = a.np > 1 ? a.np : 1;
    const bool ytile = j0 >= lo && j0 + TY - 1 <= a.ny2 - 2 - a.np;
    const bool ztile = k0 >= lo && k0 + 31 <= a.nz2 - 2 - a.np;
    // checked before any barrier or copy: an interior tile that is not
    // clear means the host's rectangle is wrong
    if (CLS == A3_INNER && !(ytile && ztile)) {
        if (tid == 0) atomicExch(a.err, 3);
        return;
    }
    const int k = k0 + lane;
    const int i0 = ch * a.chunk;
    const int i1 = min(i0 + a.chunk, a.nx2);
    const int nx2 = a.nx2, ny2 = a.ny2, nz2 = a.nz2, np = a.np, pitch = a.pitch;
    const int sx = a.sx, sy = a.sy;   // element strides (all indices fit 31 bits)
    // an interior tile, and a FULL one, lies inside the grid in y and z
    constexpr bool INSIDE = CLS == A3_INNER || FULL;
    const bool kin = INSIDE || k < nz2;
    const S *Pin = static_cast<const S *>(a.f[A_P]);
    const S *Vxin = static_cast<const S *>(a.f[A_VX]);
    S *Pout = static_cast<S *>(a.fo[A_P]);
    S *Vxout = static_cast<S *>(a.fo[A_VX]);
    S *Vyout = static_cast<S *>(a.fo[A_VY]);
    S *Vzout = static_cast<S *>(a.fo[A_VZ]);
    const C *rho = static_cast<const C *>(a.rho);
    const C *cf = static_cast<const C *>(a.coef);
    const C two_dt = static_cast<C>(a.two_dt);
    const C idx = static_cast<C>(a.idx), idy = static_cast<C>(a.idy), idz = static_cast<C>(a.idz);
    const float isP = a.isc[A_P], isX = a.isc[A_VX], isY = a.isc[A_VY], isZ = a.isc[A_VZ];
    const S *psPx = static_cast<const S *>(a.psi[PS_PX]);
    const S *psPy = static_cast<const S *>(a.psi[PS_PY]);
    const S *psPz = static_cast<const S *>(a.psi[PS_PZ]);
    const S *psVx = static_cast<const S *>(a.psi[PS_VX]);
    const S *psVy = static_cast<const S *>(a.psi[PS_VY]);
    const S *psVz = static_cast<const S *>(a.psi[PS_VZ]);
    S *poPx = static_cast<S *>(a.pso[PS_PX]);
    S *poPy = static_cast<S *>(a.pso[PS_PY]);
    S *poPz = static_cast<S *>(a.pso[PS_PZ]);
    S *poVx = static_cast<S *>(a.pso[PS_VX]);
    S *poVy = static_cast<S *>(a.pso[PS_VY]);
    S *poVz = static_cast<S *>(a.pso[PS_VZ]);

    // coefficient tables: rows 0..2 half node (a, b, 1/k), 3..5 node
    for (int t = tid; t < 6 * NXT; t += 32 * W) {
        const int wch = t / NXT, e = t % NXT, p = i0 - 1 + e;
        const bool half = wch < 3;
        const bool ok = p >= 0 && p < (half ? nx2 - 1 : nx2);
        CX[wch][e] = ok ? cf[a.cf.at(0, half ? 3 + wch : wch - 3) + p] : C(wch % 3 == 0 ? 0 : 1);
    }
    for (int t = tid; t < 6 * (TY + 1); t += 32 * W) {
        const int wch = t / (TY + 1), e = t % (TY + 1), p = j0 - 1 + e;
        const bool half = wch < 3;
        const bool ok = p >= 0 && p < (half ? ny2 - 1 : ny2);
        CY[wch][e] = ok ? cf[a.cf.at(1, half ? 3 + wch : wch - 3) + p] : C(wch % 3 == 0 ? 0 : 1);
    }
    for (int t = tid; t < 6 * 33; t += 32 * W) {
        const int wch = t / 33, e = t % 33, p = k0 - 1 + e;
        const bool half = wch < 3;
        const bool ok = p >= 0 && p < (half ? nz2 - 1 : nz2);
        CZ[wch][e] = ok ? cf[a.cf.at(2, half ? 3 + wch : wch - 3) + p] : C(wch % 3 == 0 ? 0 : 1);
    }
    if (producer) {
        for (int d = 0; d < D; ++d) mbar_init(&bars[d], 1);
        fence_proxy_async();
    }

    // ring of planes i0 .. min(i1, nx2-1), local index l = plane - i0
    const int nload = min(i1 + 1, nx2) - i0;
    auto issue = [&](int l) {   // the producer thread only
        if (l >= nload) return;
        unsigned char *b = ring + (size_t)(l % D) * L::stage;
        uint64_t *bar = &bars[l % D];
        const int ip = i0 + l;
        fence_proxy_async();
        mbar_expect_tx(bar, L::tx);
        tma_load_3d(b + L::oP, &m.P, k0 - HS, j0 - 1, ip, bar);
        tma_load_3d(b + L::oR, &m.rho, k0 - HC, j0 - 1, ip, bar);
        tma_load_3d(b + L::oX, &m.vx, k0, j0, ip, bar);
        tma_load_3d(b + L::oY, &m.vy, k0, j0 - 1, ip, bar);
        tma_load_3d(b + L::oZ, &m.vz, k0 - HS, j0, ip, bar);
        tma_load_3d(b + L::oK, &m.K, k0, j0, ip, bar);
    };
    __syncthreads();   // barriers initialised, tables filled
    // the pressure of plane ip reads P and K of its plane from registers
    // (kept by the velocity pass of plane ip), so the stage of plane l-1 is
    // free in iteration l: the ring runs D-1 planes ahead
    if (producer)
        for (int l = 0; l < D - 1; ++l) issue(l);

    // per-row / per-column frame membership (fixed over the march)
    int jh[R], jn[R], joff[R];
    bool rin[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int j = j0 + w * R + r;
        rin[r] = INSIDE || (kin && j < ny2);
        jh[r] = j < ny2 ? half_slab(j, ny2, np) : -1;
        jn[r] = j < ny2 ? node_slab(j, ny2, np) : -1;
        joff[r] = j * sy + k;
    }
    const int kh = kin ? half_slab(k, nz2, np) : -1;
    const int kn = kin ? node_slab(k, nz2, np) : -1;
    const int jm = j0 - 1, km = k0 - 1;
    const int jmh = (jm >= 0) ? half_slab(jm, ny2, np) : -1;
    const int hrow = lane;                         // halo-column row of warp HW's lane
    const bool hwarp = w == HW && lane < TY;
    const bool hcol = hwarp && km >= 0 && (INSIDE || j0 + hrow < ny2);
    const int kmh = (km >= 0) ? half_slab(km, nz2, np) : -1;
    // Per-axis fast flags.  An axis is "fast" for a cell when neither its CPML
    // frame nor the grid edge touches it: the velocity component along the
    // axis is then the plain update (a3_vel0) and the pressure needs no
    // memory variable and no edge test for it.  y and z are decided per tile
    // (uniform over the CTA), x per plane.  Velocity: half nodes
    // np .. n2-2-np; pressure: nodes max(np,1) .. n2-1-np (the reference
    // updates the pressure from index 1).  The velocity and pressure bodies
    // are compiled twice: with every axis fast (interior tiles on planes
    // clear of the x frame: straight-line code) and with the flags read at
    // run time.  The halo row and column always take the general update.
    const bool yfast = CLS == A3_INNER || FACE == A3_FACE_Z || ytile;
    const bool zfast = CLS == A3_INNER || FACE == A3_FACE_Y || ztile;

    // memory variables prefetched one plane ahead (loaded only for the
    // axes and planes that use them)
    C fPx[R], fPy[R], fPz[R], fVx[R], fVy[R], fVz[R], fHy = C(0), fHz = C(0);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        fPx[r] = C(0); fPy[r] = C(0); fPz[r] = C(0);
        fVx[r] = C(0); fVy[r] = C(0); fVz[r] = C(0);
    }
    auto load_vpsi = [&](int ip) {   // for the velocities of plane ip
        const int s = (ip < nx2 - 1) ? half_slab(ip, nx2, np) : -1;
        if (s >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                fPx[r] = rin[r] ? St::ld(psPx + s * sx + joff[r], a.pisc[PS_PX]) : C(0);
        }
        if (!yfast) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                fPy[r] = (rin[r] && jh[r] >= 0) ? St::ld(psPy + (ip * 2 * np + jh[r]) * pitch + k, a.pisc[PS_PY]) : C(0);
        }
        if (!zfast) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int j = j0 + w * R + r;
                fPz[r] = (rin[r] && kh >= 0) ? St::ld(psPz + (ip * ny2 + j) * 2 * np + kh, a.pisc[PS_PZ]) : C(0);
            }
        }
        if (w == 0 && kin && jmh >= 0) fHy = St::ld(psPy + (ip * 2 * np + jmh) * pitch + k, a.pisc[PS_PY]);
        if (hcol && kmh >= 0) fHz = St::ld(psPz + (ip * ny2 + j0 + hrow) * 2 * np + kmh, a.pisc[PS_PZ]);
    };
    auto load_ppsi = [&](int ip) {   // for the pressure of plane ip
        const int s = node_slab(ip, nx2, np);
        if (s >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                fVx[r] = rin[r] ? St::ld(psVx + s * sx + joff[r], a.pisc[PS_VX]) : C(0);
        }
        if (!yfast) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                fVy[r] = (rin[r] && jn[r] >= 0) ? St::ld(psVy + (ip * 2 * np + jn[r]) * pitch + k, a.pisc[PS_VY]) : C(0);
        }
        if (!zfast) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int j = j0 + w * R + r;
                fVz[r] = (rin[r] && kn >= 0) ? St::ld(psVz + (ip * ny2 + j) * 2 * np + kn, a.pisc[PS_VZ]) : C(0);
            }
        }
    };

    // per-thread state carried between planes, one entry per row
    C vxa[R], vxb[R], vzp[R], pkp[R], kkp[R];   // ... and P, K of the previous plane
#pragma unroll
    for (int r = 0; r < R; ++r) {
        vxa[r] = C(0); vxb[r] = C(0); vzp[r] = C(0); pkp[r] = C(0); kkp[r] = C(0);
    }
    // vx(i0-1) (direct loads, once per CTA): the pressure of plane i0 needs it
    if (i0 >= 1) {
        const int s = half_slab(i0 - 1, nx2, np);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (!rin[r]) continue;
            const int qm = (i0 - 1) * sx + joff[r], q0 = qm + sx;
            C psi_old = C(0), psi_new;
            if (s >= 0) psi_old = St::ld(psPx + s * sx + joff[r], a.pisc[PS_PX]);
            vxa[r] = a3_vel<C>(St::ld(Vxin + qm, isX), St::ld(Pin + qm, isP), St::ld(Pin + q0, isP),
                               rho[qm], rho[q0], idx, two_dt, s >= 0, CX[0][0], CX[1][0], CX[2][0],
                               psi_old, psi_new);
        }
    }
    load_vpsi(i0);

    // ---- the lagged pressure half step of plane ip (a_iso_3d.c:659-683) ----
    auto pressure = [&](int ip, auto AFt) {
        constexpr bool AF = decltype(AFt)::value;
        const bool fx = AF || (ip >= lo && ip <= nx2 - 1 - np);
        const bool fy = AF || yfast, fz = AF || zfast;
        const C(*vy)[32] = VYs[ip & 1];
        const int sxn = fx ? -1 : node_slab(ip, nx2, np);
        const int e = ip - (i0 - 1);
        S *po = Pout + ip * sx;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int row = w * R + r, j = j0 + row;
            C vzm = __shfl_up_sync(0xffffffffu, vzp[r], 1);
            if (lane == 0) vzm = VZH[ip & 1][row];
            if (!rin[r]) continue;
            const C p_c = pkp[r];
            C pn = p_c;
            // the reference leaves index 0 of every axis untouched
            bool upd = true;
            if (!fx) upd = ip >= 1;
            if (!fy) upd = upd && j >= 1;
            if (!fz) upd = upd && k >= 1;
            if (upd) {
                C gx = r_mul(r_sub(vxa[r], vxb[r]), idx);
                C gy = r_mul(r_sub(vy[row + 1][lane], vy[row][lane]), idy);
                C gz = r_mul(r_sub(vzp[r], vzm), idz);
                C psi_new;
                if (sxn >= 0) {
                    gx = a3_dv<C>(gx, CX[3][e], CX[4][e], CX[5][e], fVx[r], psi_new);
                    St::st(poVx + sxn * sx + joff[r], psi_new, a.psc[PS_VX]);
                }
                if (!fy && jn[r] >= 0) {
                    gy = a3_dv<C>(gy, CY[3][row + 1], CY[4][row + 1], CY[5][row + 1], fVy[r], psi_new);
                    St::st(poVy + (ip * 2 * np + jn[r]) * pitch + k, psi_new, a.psc[PS_VY]);
                }
                if (!fz && kn >= 0) {
                    gz = a3_dv<C>(gz, CZ[3][lane + 1], CZ[4][lane + 1], CZ[5][lane + 1], fVz[r], psi_new);
                    St::st(poVz + (ip * ny2 + j) * 2 * np + kn, psi_new, a.psc[PS_VZ]);
                }
                pn = r_fma(-kkp[r], r_add(r_add(gx, gy), gz), p_c);
            }
            // written whether updated or not: both buffers always hold a
            // complete state
            St::st(po + joff[r], pn, a.sc[A_P]);
        }
    };

    for (int i = i0; i < i1; ++i) {
        const int l = i - i0;
        if (producer) issue(l + D - 1);
        // plane l was waited for as the next plane of iteration l-1
        if (l == 0 && !mbar_wait(&bars[0], 0, a.err, 1)) return;
        if (i + 1 < nx2 && !mbar_wait(&bars[(l + 1) % D], ((l + 1) / D) & 1, a.err, 1)) return;
        const unsigned char *cbuf = ring + (size_t)(l % D) * L::stage;
        const unsigned char *nbuf = ring + (size_t)((l + 1) % D) * L::stage;
        const S *cP = reinterpret_cast<const S *>(cbuf + L::oP);
        const C *cR = reinterpret_cast<const C *>(cbuf + L::oR);
        const S *cX = reinterpret_cast<const S *>(cbuf + L::oX);
        const S *cY = reinterpret_cast<const S *>(cbuf + L::oY);
        const S *cZ = reinterpret_cast<const S *>(cbuf + L::oZ);
        const S *nP = reinterpret_cast<const S *>(nbuf + L::oP);
        const C *nR = reinterpret_cast<const C *>(nbuf + L::oR);
        const C *cK = reinterpret_cast<const C *>(cbuf + L::oK);
        C(*vyw)[32] = VYs[i & 1];
        const bool xf = i >= np && i <= nx2 - 2 - np;
        const int sxh = (i < nx2 - 1) ? half_slab(i, nx2, np) : -1;
        const int e = i - (i0 - 1);
        S *ox = Vxout + i * sx, *oy = Vyout + i * sx, *oz = Vzout + i * sx;

        // ---- velocity half step at plane i (a_iso_3d.c:605-651) ----
        // A component on a fast axis is updated even in cells outside the
        // grid (from the zero fill): such values are neither stored nor
        // read by a cell inside the grid.
        C vxn[R], vzn[R], pkn[R], kkn[R];
        auto velocity = [&](auto AFt) {
        constexpr bool AF = decltype(AFt)::value;
        const bool fx = AF || xf, fy = AF || yfast, fz = AF || zfast;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int row = w * R + r, j = j0 + row;
            const int cc = (row + 1) * WS + HS + lane;
            const int rc = (row + 1) * WC + HC + lane;
            const C p_c = St::ld(cP + cc, isP);
            const C r_c = cR[rc];
            C vx = St::ld(cX + row * 32 + lane, isX);
            C vy = St::ld(cY + (row + 1) * 32 + lane, isY);
            C vz = St::ld(cZ + row * WZ + HS + lane, isZ);
            C psi_new;
            if (fx) {
                vx = a3_vel0<C>(vx, p_c, St::ld(nP + cc, isP), r_c, nR[rc], idx, two_dt);
            } else if (rin[r] && i < nx2 - 1) {
                vx = a3_vel<C>(vx, p_c, St::ld(nP + cc, isP), r_c, nR[rc], idx, two_dt, sxh >= 0,
                               CX[0][e], CX[1][e], CX[2][e], fPx[r], psi_new);
                if (sxh >= 0) St::st(poPx + sxh * sx + joff[r], psi_new, a.psc[PS_PX]);
            }
            if (fy) {
                vy = a3_vel0<C>(vy, p_c, St::ld(cP + cc + WS, isP), r_c, cR[rc + WC], idy, two_dt);
            } else if (rin[r] && j < ny2 - 1) {
                vy = a3_vel<C>(vy, p_c, St::ld(cP + cc + WS, isP), r_c, cR[rc + WC], idy, two_dt,
                               jh[r] >= 0, CY[0][row + 1], CY[1][row + 1], CY[2][row + 1], fPy[r],
                               psi_new);
                if (jh[r] >= 0)
                    St::st(poPy + (i * 2 * np + jh[r]) * pitch + k, psi_new, a.psc[PS_PY]);
            }
            if (fz) {
                vz = a3_vel0<C>(vz, p_c, St::ld(cP + cc + 1, isP), r_c, cR[rc + 1], idz, two_dt);
            } else if (rin[r] && k < nz2 - 1) {
                vz = a3_vel<C>(vz, p_c, St::ld(cP + cc + 1, isP), r_c, cR[rc + 1], idz, two_dt,
                               kh >= 0, CZ[0][lane + 1], CZ[1][lane + 1], CZ[2][lane + 1], fPz[r],
                               psi_new);
                if (kh >= 0) St::st(poPz + (i * ny2 + j) * 2 * np + kh, psi_new, a.psc[PS_PZ]);
            }
            vyw[row + 1][lane] = vy;
            vxn[r] = vx;
            vzn[r] = vz;
            pkn[r] = p_c;
            kkn[r] = cK[row * 32 + lane];
            if (rin[r]) {
                St::st(ox + joff[r], vx, a.sc[A_VX]);
                St::st(oy + joff[r], vy, a.sc[A_VY]);
                St::st(oz + joff[r], vz, a.sc[A_VZ]);
            }
        }
        };
        if (CLS == A3_INNER && xf) velocity(BoolT<true>{});
        else velocity(BoolT<false>{});
        // halo row: vy(i, j0-1, k), by warp 0
        if (w == 0) {
            C vyh = C(0);
            if (CLS == A3_INNER || (jm >= 0 && kin)) {
                C psi_new;
                vyh = a3_vel<C>(St::ld(cY + lane, isY), St::ld(cP + HS + lane, isP),
                                St::ld(cP + WS + HS + lane, isP), cR[HC + lane], cR[WC + HC + lane],
                                idy, two_dt, jmh >= 0, CY[0][0], CY[1][0], CY[2][0], fHy, psi_new);
            }
            vyw[0][lane] = vyh;
        }
        // halo column: vz(i, j, k0-1) of row `lane`, by warp HW; read by
        // the pressure of plane i (next iteration, after the barrier)
        if (hwarp) {
            C vzh = C(0);
            if (hcol) {
                const int cc = (hrow + 1) * WS + HS, rc = (hrow + 1) * WC + HC;
                C psi_new;
                vzh = a3_vel<C>(St::ld(cZ + hrow * WZ + HS - 1, isZ), St::ld(cP + cc - 1, isP),
                                St::ld(cP + cc, isP), cR[rc - 1], cR[rc], idz, two_dt, kmh >= 0,
                                CZ[0][0], CZ[1][0], CZ[2][0], fHz, psi_new);
            }
            VZH[i & 1][hrow] = vzh;
        }
        // memory variables for the next plane's velocities
        if (i + 1 < i1) load_vpsi(i + 1);
        // the pressure of the previous plane (its velocities are complete)
        if (i > i0) {
            const int ip = i - 1;
            if (CLS == A3_INNER && ip >= lo && ip <= nx2 - 1 - np) pressure(ip, BoolT<true>{});
            else pressure(ip, BoolT<false>{});
        }
        load_ppsi(i);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            vxb[r] = vxa[r];
            vxa[r] = vxn[r];
            vzp[r] = vzn[r];
            pkp[r] = pkn[r];
            kkp[r] = kkn[r];
        }
        __syncthreads();   // vy rows and halo column of plane i visible; the oldest stage may be refilled
    }
    // the last plane's pressure
    if (i1 > i0) {
        const int ip = i1 - 1;
        if (CLS == A3_INNER && ip >= lo && ip <= nx2 - 1 - np) pressure(ip, BoolT<true>{});
        else pressure(ip, BoolT<false>{});
    }
}

// One launch per tile class; the ring's CTAs take the body compiled for
// their face (one axis fast at compile time) or the general one.
template <typename S, int W, int R, int D, int MINB, int CLS>
__global__ void __launch_bounds__(32 * W, MINB)
    a3d_step_kernel(const A3Args a, const __grid_constant__ A3Maps m) {
    if (CLS == a.step_cls && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0)
        ++*a.step;
    if (CLS == A3_INNER) {
        a3d_step_body<S, W, R, D, CLS, A3_FACE_GEN>(a, m, a.kt0 + blockIdx.x, a.jt0 + blockIdx.y,
                                                    blockIdx.z);
        return;
    }
    int kt, jt;
    const int face = a3_edge_tile(a, blockIdx.x, kt, jt);
    const bool full = kt * 32 + 31 < a.nz2 && (jt + 1) * W * R <= a.ny2;
#if SM_A3D_FACE_BODIES
    if (full && face == A3_FACE_Z)
        a3d_step_body<S, W, R, D, CLS, A3_FACE_Z, true>(a, m, kt, jt, blockIdx.z);
    else if (full && face == A3_FACE_Y)
        a3d_step_body<S, W, R, D, CLS, A3_FACE_Y, true>(a, m, kt, jt, blockIdx.z);
    else
#endif
    if (full)
        a3d_step_body<S, W, R, D, CLS, A3_FACE_GEN, true>(a, m, kt, jt, blockIdx.z);
    else
        a3d_step_body<S, W, R, D, CLS, A3_FACE_GEN, false>(a, m, kt, jt, blockIdx.z);
    (void)face;
}

template <typename S, int TY, int D>
constexpr size_t a3d_step_smem() {
    return A3Lay<S, TY>::head + (size_t)D * A3Lay<S, TY>::stage;
}

// ===========================================================================
// Block-floating-point step (SM_BFP16).  The fused step of a3d_step_kernel
// with P, vx, vy, vz stored as 16-bit mantissas and one exponent byte per
// block of A3_BJ consecutive y rows of one z column ([nx2][nyb][pitch]
// bytes); the CPML memory variables, rho and K stay FP32, and the
// arithmetic is the FP32 path's, operation for operation.  Each thread owns
// exactly one block (its A3_BJ rows), so the exponent of a block it stores
// is the maximum over its own registers: no exchange between threads.  The
// velocities the lagged pressure reads are the unrounded values of this
// step (vx and vz in registers, vy in the shared row buffer): only the state
// a step leaves behind is rounded.  Decoded pressures are carried across
// planes in registers: P(i+1) is decoded once, for vx at plane i, and then
// serves as P(i) at plane i+1 and in the pressure update of plane i+1.
// ===========================================================================
#define A3_BJ 4

template <int TY>
struct A3BLay {
    static constexpr int NB = TY / A3_BJ;   // blocks (thread rows) of the tile
    // row widths (elements): P k0-8 .. k0+39, rho k0-4 .. k0+35, vz k0-8 .. k0+31;
    // exponent rows (bytes): P k0-16 .. k0+47, vz k0-16 .. k0+31
    static constexpr int WP = 48, WR = 40, WZ = 40, WEP = 64, WEZ = 48;
    __host__ __device__ static constexpr size_t al(size_t x) { return (x + 127) / 128 * 128; }
    static constexpr size_t bP = (size_t)(TY + 2) * WP * 2;
    static constexpr size_t bEP = (size_t)(NB + 2) * WEP;
    static constexpr size_t bR = (size_t)(TY + 2) * WR * 4;
    static constexpr size_t bX = (size_t)TY * 32 * 2;
    static constexpr size_t bEX = (size_t)NB * 32;
    static constexpr size_t bY = (size_t)(TY + 1) * 32 * 2;
    static constexpr size_t bEY = (size_t)(NB + 1) * 32;
    static constexpr size_t bZ = (size_t)TY * WZ * 2;
    static constexpr size_t bEZ = (size_t)NB * WEZ;
    static constexpr size_t bK = (size_t)TY * 32 * 4;
    static constexpr size_t oP = 0, oEP = al(bP), oR = oEP + al(bEP), oX = oR + al(bR);
    static constexpr size_t oEX = oX + al(bX), oY = oEX + al(bEX), oEY = oY + al(bY);
    static constexpr size_t oZ = oEY + al(bEY), oEZ = oZ + al(bZ), oK = oEZ + al(bEZ);
    static constexpr size_t stage = oK + al(bK);
    static constexpr unsigned tx =
        (unsigned)(bP + bEP + bR + bX + bEX + bY + bEY + bZ + bEZ + bK);
    // head as the FP32 step's: barriers, vy row buffers, coefficient tables
    static constexpr size_t head = A3Lay<float, TY>::head;
};

struct A3BMaps {
    CUtensorMap P, eP, vx, eX, vy, eY, vz, eZ, rho, K;
};

template <int W, int D, int CLS, int FACE, bool FULL = false>
__device__ __forceinline__ void a3d_bstep_body(const A3Args &a, const A3BMaps &m, int kt, int jt,
                                               int ch) {
    constexpr int R = A3_BJ, TY = W * R;
    using C = float;
    using PSt = Store<float>;
    using L = A3BLay<TY>;
    using HL = A3Lay<float, TY>;
    static_assert(D >= 4 && D <= D_HEAD_BARS, "ring depth");
    constexpr int NXT = A3_CHMAX + 2;
    constexpr int WP = L::WP, WR = L::WR, WZ = L::WZ, WEP = L::WEP, WEZ = L::WEZ;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    C(*VYs)[TY + 1][32] = reinterpret_cast<C(*)[TY + 1][32]>(smem + HL::oVY);
    C(*CX)[NXT] = reinterpret_cast<C(*)[NXT]>(smem + HL::oCX);
    C(*CY)[TY + 1] = reinterpret_cast<C(*)[TY + 1]>(smem + HL::oCY);
    C(*CZ)[33] = reinterpret_cast<C(*)[33]>(smem + HL::oCZ);
    C *VZH = reinterpret_cast<C *>(smem + HL::oVZ);   // [2][TY]: halo column by plane parity
    unsigned char *ring = smem + L::head;

    const int lane = threadIdx.x, w = threadIdx.y;
    const int tid = w * 32 + lane;
    // TMA loads issued by the last warp's lane 0, the halo row computed by
    // warp 0 and the halo column by warp HW (rows lane, lane + 32, ...)
    constexpr int HW = W > 2 ? 1 : 0;
    constexpr int NH = (TY + 31) / 32;
    const bool producer = tid == 32 * (W - 1);
    const int k0 = kt * 32, j0 = jt * TY, jb0 = jt * (TY / R);
    const int lo = a.np > 1 ? a.np : 1;
    const bool ytile = j0 >= lo && j0 + TY - 1 <= a.ny2 - 2 - a.np;
    const bool ztile = k0 >= lo && k0 + 31 <= a.nz2 - 2 - a.np;
    if (CLS == A3_INNER && !(ytile && ztile)) {
        if (tid == 0) atomicExch(a.err, 3);
        return;
    }
    const int k = k0 + lane;
    const int i0 = ch * a.chunk;
    const int i1 = min(i0 + a.chunk, a.nx2);
    const int nx2 = a.nx2, ny2 = a.ny2, nz2 = a.nz2, np = a.np, pitch = a.pitch;
    const int sx = a.sx, sy = a.sy;
    const int ex = a.nyb * pitch;   // exponent bytes per x plane
    // an interior tile, and a FULL one, lies inside the grid in y and z
    constexpr bool INSIDE = CLS == A3_INNER || FULL;
    const bool kin = INSIDE || k < nz2;
    const int16_t *Pin = static_cast<const int16_t *>(a.f[A_P]);
    const int16_t *Vxin = static_cast<const int16_t *>(a.f[A_VX]);
    const uint8_t *EPin = static_cast<const uint8_t *>(a.fe[A_P]);
    const uint8_t *EXin = static_cast<const uint8_t *>(a.fe[A_VX]);
    int16_t *Pout = static_cast<int16_t *>(a.fo[A_P]);
    int16_t *Vxout = static_cast<int16_t *>(a.fo[A_VX]);
    int16_t *Vyout = static_cast<int16_t *>(a.fo[A_VY]);
    int16_t *Vzout = static_cast<int16_t *>(a.fo[A_VZ]);
    uint8_t *EPout = static_cast<uint8_t *>(a.feo[A_P]);
    uint8_t *EXout = static_cast<uint8_t *>(a.feo[A_VX]);
    uint8_t *EYout = static_cast<uint8_t *>(a.feo[A_VY]);
    uint8_t *EZout = static_cast<uint8_t *>(a.feo[A_VZ]);
    const C *rho = static_cast<const C *>(a.rho);
    const C *cf = static_cast<const C *>(a.coef);
    const C two_dt = static_cast<C>(a.two_dt);
    const C idx = static_cast<C>(a.idx), idy = static_cast<C>(a.idy), idz = static_cast<C>(a.idz);
    const C *psPx = static_cast<const C *>(a.psi[PS_PX]);
    const C *psPy = static_cast<const C *>(a.psi[PS_PY]);
    const C *psPz = static_cast<const C *>(a.psi[PS_PZ]);
    const C *psVx = static_cast<const C *>(a.psi[PS_VX]);
    const C *psVy = static_cast<const C *>(a.psi[PS_VY]);
    const C *psVz = static_cast<const C *>(a.psi[PS_VZ]);
    C *poPx = static_cast<C *>(a.pso[PS_PX]);
    C *poPy = static_cast<C *>(a.pso[PS_PY]);
    C *poPz = static_cast<C *>(a.pso[PS_PZ]);
    C *poVx = static_cast<C *>(a.pso[PS_VX]);
    C *poVy = static_cast<C *>(a.pso[PS_VY]);
    C *poVz = static_cast<C *>(a.pso[PS_VZ]);

    // coefficient tables: rows 0..2 half node (a, b, 1/k), 3..5 node
    for (int t = tid; t < 6 * NXT; t += 32 * W) {
        const int wch = t / NXT, e = t % NXT, p = i0 - 1 + e;
        const bool half = wch < 3;
        const bool ok = p >= 0 && p < (half ? nx2 - 1 : nx2);
        CX[wch][e] = ok ? cf[a.cf.at(0, half ? 3 + wch : wch - 3) + p] : C(wch % 3 == 0 ? 0 : 1);
    }
    for (int t = tid; t < 6 * (TY + 1); t += 32 * W) {
        const int wch = t / (TY + 1), e = t % (TY + 1), p = j0 - 1 + e;
        const bool half = wch < 3;
        const bool ok = p >= 0 && p < (half ? ny2 - 1 : ny2);
        CY[wch][e] = ok ? cf[a.cf.at(1, half ? 3 + wch : wch - 3) + p] : C(wch % 3 == 0 ? 0 : 1);
    }
    for (int t = tid; t < 6 * 33; t += 32 * W) {
        const int wch = t / 33, e = t % 33, p = k0 - 1 + e;
        const bool half = wch < 3;
        const bool ok = p >= 0 && p < (half ? nz2 - 1 : nz2);
        CZ[wch][e] = ok ? cf[a.cf.at(2, half ? 3 + wch : wch - 3) + p] : C(wch % 3 == 0 ? 0 : 1);
    }
    if (producer) {
        for (int d = 0; d < D; ++d) mbar_init(&bars[d], 1);
        fence_proxy_async();
    }

    const int nload = min(i1 + 1, nx2) - i0;
    auto issue = [&](int l) {   // the producer thread only
        if (l >= nload) return;
        unsigned char *b = ring + (size_t)(l % D) * L::stage;
        uint64_t *bar = &bars[l % D];
        const int ip = i0 + l;
        fence_proxy_async();
        mbar_expect_tx(bar, L::tx);
        tma_load_3d(b + L::oP, &m.P, k0 - 8, j0 - 1, ip, bar);
        tma_load_3d(b + L::oEP, &m.eP, k0 - 16, jb0 - 1, ip, bar);
        tma_load_3d(b + L::oR, &m.rho, k0 - 4, j0 - 1, ip, bar);
        tma_load_3d(b + L::oX, &m.vx, k0, j0, ip, bar);
        tma_load_3d(b + L::oEX, &m.eX, k0, jb0, ip, bar);
        tma_load_3d(b + L::oY, &m.vy, k0, j0 - 1, ip, bar);
        tma_load_3d(b + L::oEY, &m.eY, k0, jb0 - 1, ip, bar);
        tma_load_3d(b + L::oZ, &m.vz, k0 - 8, j0, ip, bar);
        tma_load_3d(b + L::oEZ, &m.eZ, k0 - 16, jb0, ip, bar);
        tma_load_3d(b + L::oK, &m.K, k0, j0, ip, bar);
    };
    __syncthreads();   // barriers initialised, tables filled
    // the pressure of plane ip takes P and K of its plane from registers,
    // so the stage of plane l-1 is free in iteration l: D-1 planes ahead
    if (producer)
        for (int l = 0; l < D - 1; ++l) issue(l);

    // rows of this thread: one block, rows j0 + w*R + r
    int jh[R], jn[R], joff[R];
    bool rin[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int j = j0 + w * R + r;
        rin[r] = INSIDE || (kin && j < ny2);
        jh[r] = j < ny2 ? half_slab(j, ny2, np) : -1;
        jn[r] = j < ny2 ? node_slab(j, ny2, np) : -1;
        joff[r] = j * sy + k;
    }
    const bool bin = rin[0];                       // the block has a cell in the grid
    const int eoff = (jb0 + w) * pitch + k;         // this thread's exponent, plane 0
    const int kh = kin ? half_slab(k, nz2, np) : -1;
    const int kn = kin ? node_slab(k, nz2, np) : -1;
    const int jm = j0 - 1, km = k0 - 1;
    const int jmh = (jm >= 0) ? half_slab(jm, ny2, np) : -1;
    const bool hwarp = w == HW;
    const int kmh = (km >= 0) ? half_slab(km, nz2, np) : -1;
    const bool yfast = CLS == A3_INNER || FACE == A3_FACE_Z || ytile;
    const bool zfast = CLS == A3_INNER || FACE == A3_FACE_Y || ztile;

    // exponent byte of stage sb: P block b (0: rows above the tile), column
    // x = k - (k0 - 16); vx block w; vy block b (0: above); vz column x
    auto eP_ = [&](const unsigned char *sb, int b, int x) -> unsigned { return sb[L::oEP + b * WEP + x]; };
    auto eX_ = [&](const unsigned char *sb) -> unsigned { return sb[L::oEX + w * 32 + lane]; };
    auto eY_ = [&](const unsigned char *sb, int b) -> unsigned { return sb[L::oEY + b * 32 + lane]; };
    auto eZ_ = [&](const unsigned char *sb, int x) -> unsigned { return sb[L::oEZ + w * WEZ + x]; };
    auto mP = [&](const unsigned char *sb, int row, int x) -> int {   // row of the box, x = k - (k0-8)
        return reinterpret_cast<const int16_t *>(sb + L::oP)[row * WP + x];
    };

    C fPx[R], fPy[R], fPz[R], fVx[R], fVy[R], fVz[R], fHy = C(0), fHz[NH];
#pragma unroll
    for (int h = 0; h < NH; ++h) fHz[h] = C(0);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        fPx[r] = C(0); fPy[r] = C(0); fPz[r] = C(0);
        fVx[r] = C(0); fVy[r] = C(0); fVz[r] = C(0);
    }
    auto load_vpsi = [&](int ip) {
        const int s = (ip < nx2 - 1) ? half_slab(ip, nx2, np) : -1;
        if (s >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) fPx[r] = rin[r] ? psPx[s * sx + joff[r]] : C(0);
        }
        if (!yfast) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                fPy[r] = (rin[r] && jh[r] >= 0) ? psPy[(ip * 2 * np + jh[r]) * pitch + k] : C(0);
        }
        if (!zfast) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int j = j0 + w * R + r;
                fPz[r] = (rin[r] && kh >= 0) ? psPz[(ip * ny2 + j) * 2 * np + kh] : C(0);
            }
        }
        if (w == 0 && kin && jmh >= 0) fHy = psPy[(ip * 2 * np + jmh) * pitch + k];
        if (hwarp && km >= 0 && kmh >= 0) {
#pragma unroll
            for (int h = 0; h < NH; ++h) {
                const int hr = lane + 32 * h;
                if (hr < TY && j0 + hr < ny2) fHz[h] = psPz[(ip * ny2 + j0 + hr) * 2 * np + kmh];
            }
        }
    };
    auto load_ppsi = [&](int ip) {
        const int s = node_slab(ip, nx2, np);
        if (s >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) fVx[r] = rin[r] ? psVx[s * sx + joff[r]] : C(0);
        }
        if (!yfast) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                fVy[r] = (rin[r] && jn[r] >= 0) ? psVy[(ip * 2 * np + jn[r]) * pitch + k] : C(0);
        }
        if (!zfast) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int j = j0 + w * R + r;
                fVz[r] = (rin[r] && kn >= 0) ? psVz[(ip * ny2 + j) * 2 * np + kn] : C(0);
            }
        }
    };

    C vxa[R], vxb[R], vzp[R];
    C pc[R], pp[R];   // decoded P of plane i (own cells) and of plane i-1
    C kkp[R];         // K of plane i-1
#pragma unroll
    for (int r = 0; r < R; ++r) {
        vxa[r] = C(0); vxb[r] = C(0); vzp[r] = C(0); pc[r] = C(0); pp[r] = C(0); kkp[r] = C(0);
    }
    // vx(i0-1) (direct loads, once per CTA): the pressure of plane i0 needs it
    if (i0 >= 1 && bin) {
        const int s = half_slab(i0 - 1, nx2, np);
        const int eo = (i0 - 1) * ex + eoff;
        const BDec dX = bfp_dec(EXin[eo]), dP0 = bfp_dec(EPin[eo]), dP1 = bfp_dec(EPin[eo + ex]);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (!rin[r]) continue;
            const int qm = (i0 - 1) * sx + joff[r], q0 = qm + sx;
            C psi_old = C(0), psi_new;
            if (s >= 0) psi_old = psPx[s * sx + joff[r]];
            vxa[r] = a3_vel<C>(bfp_val(Vxin[qm], dX), bfp_val(Pin[qm], dP0), bfp_val(Pin[q0], dP1),
                               rho[qm], rho[q0], idx, two_dt, s >= 0, CX[0][0], CX[1][0], CX[2][0],
                               psi_old, psi_new);
        }
    }
    load_vpsi(i0);
    // P of the first plane, decoded once
    if (!mbar_wait(&bars[0], 0, a.err, 1)) return;
    {
        const BDec d = bfp_dec(eP_(ring, w + 1, lane + 16));
#pragma unroll
        for (int r = 0; r < R; ++r) pc[r] = bfp_val(mP(ring, w * R + r + 1, lane + 8), d);
    }

    // encode and store one block (rows of this thread) of a field at plane
    // ip: mantissas where the row is in the grid, the exponent once
    bool overflow = false;   // a block beyond the format's range (reported once, at the end)
    auto store_block = [&](int16_t *out, uint8_t *eout, int ip, const C *v) {
        unsigned mx = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) mx = rin[r] ? max(mx, bfp_absbits(v[r])) : mx;
        bool over;
        const unsigned e8 = bfp_e8(mx, &over);
        const float esc = bfp_escale(e8);
        int16_t *o = out + ip * sx;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (rin[r]) o[joff[r]] = bfp_man(v[r], esc);
        if (bin) eout[ip * ex + eoff] = (uint8_t)e8;
        overflow = overflow || (bin && over);
    };

    // ---- the lagged pressure half step of plane ip (a_iso_3d.c:659-683) ----
    auto pressure = [&](int ip, auto AFt) {
        constexpr bool AF = decltype(AFt)::value;
        const bool fx = AF || (ip >= lo && ip <= nx2 - 1 - np);
        const bool fy = AF || yfast, fz = AF || zfast;
        const C(*vy)[32] = VYs[ip & 1];
        const int sxn = fx ? -1 : node_slab(ip, nx2, np);
        const int e = ip - (i0 - 1);
        C pn[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int row = w * R + r, j = j0 + row;
            C vzm = __shfl_up_sync(0xffffffffu, vzp[r], 1);
            if (lane == 0) vzm = VZH[(ip & 1) * TY + row];
            const C p_c = pp[r];
            pn[r] = p_c;
            if (!rin[r]) continue;
            bool upd = true;
            if (!fx) upd = ip >= 1;
            if (!fy) upd = upd && j >= 1;
            if (!fz) upd = upd && k >= 1;
            if (upd) {
                C gx = r_mul(r_sub(vxa[r], vxb[r]), idx);
                C gy = r_mul(r_sub(vy[row + 1][lane], vy[row][lane]), idy);
                C gz = r_mul(r_sub(vzp[r], vzm), idz);
                C psi_new;
                if (sxn >= 0) {
                    gx = a3_dv<C>(gx, CX[3][e], CX[4][e], CX[5][e], fVx[r], psi_new);
                    poVx[sxn * sx + joff[r]] = psi_new;
                }
                if (!fy && jn[r] >= 0) {
                    gy = a3_dv<C>(gy, CY[3][row + 1], CY[4][row + 1], CY[5][row + 1], fVy[r], psi_new);
                    poVy[(ip * 2 * np + jn[r]) * pitch + k] = psi_new;
                }
                if (!fz && kn >= 0) {
                    gz = a3_dv<C>(gz, CZ[3][lane + 1], CZ[4][lane + 1], CZ[5][lane + 1], fVz[r], psi_new);
                    poVz[(ip * ny2 + j) * 2 * np + kn] = psi_new;
                }
                pn[r] = r_fma(-kkp[r], r_add(r_add(gx, gy), gz), p_c);
            }
        }
        // written whether updated or not: both buffers always hold a
        // complete state
        store_block(Pout, EPout, ip, pn);
    };

    for (int i = i0; i < i1; ++i) {
        const int l = i - i0;
        if (producer) issue(l + D - 1);
        // plane l was waited for as the next plane of iteration l-1
        if (l == 0 && !mbar_wait(&bars[0], 0, a.err, 1)) return;
        if (i + 1 < nx2 && !mbar_wait(&bars[(l + 1) % D], ((l + 1) / D) & 1, a.err, 1)) return;
        const unsigned char *cbuf = ring + (size_t)(l % D) * L::stage;
        const unsigned char *nbuf = ring + (size_t)((l + 1) % D) * L::stage;
        const C *cR = reinterpret_cast<const C *>(cbuf + L::oR);
        const C *nR = reinterpret_cast<const C *>(nbuf + L::oR);
        const C *cK = reinterpret_cast<const C *>(cbuf + L::oK);
        const int16_t *cX = reinterpret_cast<const int16_t *>(cbuf + L::oX);
        const int16_t *cY = reinterpret_cast<const int16_t *>(cbuf + L::oY);
        const int16_t *cZ = reinterpret_cast<const int16_t *>(cbuf + L::oZ);
        C(*vyw)[32] = VYs[i & 1];
        const bool xf = i >= np && i <= nx2 - 2 - np;
        const int sxh = (i < nx2 - 1) ? half_slab(i, nx2, np) : -1;
        const int e = i - (i0 - 1);
        // decoders of this plane's blocks (the next plane's P: its pressures
        // are decoded here once and carried)
        const BDec dPz = bfp_dec(eP_(cbuf, w + 1, lane + 17));
        const BDec dPy = bfp_dec(eP_(cbuf, w + 2, lane + 16));
        const BDec dX = bfp_dec(eX_(cbuf)), dY = bfp_dec(eY_(cbuf, w + 1));
        const BDec dZ = bfp_dec(eZ_(cbuf, lane + 16));
        C pnx[R];
        if (i + 1 < nx2) {
            const BDec dPn = bfp_dec(eP_(nbuf, w + 1, lane + 16));
#pragma unroll
            for (int r = 0; r < R; ++r) pnx[r] = bfp_val(mP(nbuf, w * R + r + 1, lane + 8), dPn);
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) pnx[r] = C(0);
        }

        // ---- velocity half step at plane i (a_iso_3d.c:605-651) ----
        C vxn[R], vyn[R], vzn[R];
        auto velocity = [&](auto AFt) {
        constexpr bool AF = decltype(AFt)::value;
        const bool fx = AF || xf, fy = AF || yfast, fz = AF || zfast;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int row = w * R + r, j = j0 + row;
            const int rc = (row + 1) * WR + 4 + lane;
            const C p_c = pc[r];
            const C p_n = pnx[r];
            const C p_y = r + 1 < R ? pc[r + 1] : bfp_val(mP(cbuf, row + 2, lane + 8), dPy);
            const C p_z = bfp_val(mP(cbuf, row + 1, lane + 9), dPz);
            const C r_c = cR[rc];
            C vx = bfp_val(cX[row * 32 + lane], dX);
            C vy = bfp_val(cY[(row + 1) * 32 + lane], dY);
            C vz = bfp_val(cZ[row * WZ + 8 + lane], dZ);
            C psi_new;
            if (fx) {
                vx = a3_vel0<C>(vx, p_c, p_n, r_c, nR[rc], idx, two_dt);
            } else if (rin[r] && i < nx2 - 1) {
                vx = a3_vel<C>(vx, p_c, p_n, r_c, nR[rc], idx, two_dt, sxh >= 0,
                               CX[0][e], CX[1][e], CX[2][e], fPx[r], psi_new);
                if (sxh >= 0) poPx[sxh * sx + joff[r]] = psi_new;
            }
            if (fy) {
                vy = a3_vel0<C>(vy, p_c, p_y, r_c, cR[rc + WR], idy, two_dt);
            } else if (rin[r] && j < ny2 - 1) {
                vy = a3_vel<C>(vy, p_c, p_y, r_c, cR[rc + WR], idy, two_dt, jh[r] >= 0,
                               CY[0][row + 1], CY[1][row + 1], CY[2][row + 1], fPy[r], psi_new);
                if (jh[r] >= 0) poPy[(i * 2 * np + jh[r]) * pitch + k] = psi_new;
            }
            if (fz) {
                vz = a3_vel0<C>(vz, p_c, p_z, r_c, cR[rc + 1], idz, two_dt);
            } else if (rin[r] && k < nz2 - 1) {
                vz = a3_vel<C>(vz, p_c, p_z, r_c, cR[rc + 1], idz, two_dt, kh >= 0,
                               CZ[0][lane + 1], CZ[1][lane + 1], CZ[2][lane + 1], fPz[r], psi_new);
                if (kh >= 0) poPz[(i * ny2 + j) * 2 * np + kh] = psi_new;
            }
            vyw[row + 1][lane] = vy;
            vxn[r] = vx;
            vyn[r] = vy;
            vzn[r] = vz;
        }
        };
        if (CLS == A3_INNER && xf) velocity(BoolT<true>{});
        else velocity(BoolT<false>{});
        store_block(Vxout, EXout, i, vxn);
        store_block(Vyout, EYout, i, vyn);
        store_block(Vzout, EZout, i, vzn);
        // halo row: vy(i, j0-1, k), by warp 0
        if (w == 0) {
            C vyh = C(0);
            if (CLS == A3_INNER || (jm >= 0 && kin)) {
                C psi_new;
                vyh = a3_vel<C>(bfp_val(cY[lane], bfp_dec(eY_(cbuf, 0))),
                                bfp_val(mP(cbuf, 0, lane + 8), bfp_dec(eP_(cbuf, 0, lane + 16))),
                                bfp_val(mP(cbuf, 1, lane + 8), bfp_dec(eP_(cbuf, 1, lane + 16))),
                                cR[4 + lane], cR[WR + 4 + lane], idy, two_dt, jmh >= 0, CY[0][0],
                                CY[1][0], CY[2][0], fHy, psi_new);
            }
            vyw[0][lane] = vyh;
        }
        // halo column: vz(i, j, k0-1) of rows lane, lane + 32, ..., by warp
        // HW; read by the pressure of plane i (next iteration, after the
        // barrier)
        if (hwarp) {
#pragma unroll
            for (int h = 0; h < NH; ++h) {
                const int hr = lane + 32 * h;
                if (hr >= TY) continue;
                C vzh = C(0);
                if (km >= 0 && (INSIDE || j0 + hr < ny2)) {
                    const int rc = (hr + 1) * WR + 4, hb = hr / R;
                    const BDec dP0 = bfp_dec(eP_(cbuf, hb + 1, 15));
                    const BDec dP1 = bfp_dec(eP_(cbuf, hb + 1, 16));
                    const BDec dZh = bfp_dec(cbuf[L::oEZ + hb * WEZ + 15]);
                    C psi_new;
                    vzh = a3_vel<C>(bfp_val(cZ[hr * WZ + 7], dZh), bfp_val(mP(cbuf, hr + 1, 7), dP0),
                                    bfp_val(mP(cbuf, hr + 1, 8), dP1), cR[rc - 1], cR[rc], idz,
                                    two_dt, kmh >= 0, CZ[0][0], CZ[1][0], CZ[2][0], fHz[h], psi_new);
                }
                VZH[(i & 1) * TY + hr] = vzh;
            }
        }
        if (i + 1 < i1) load_vpsi(i + 1);
        if (i > i0) {
            const int ip = i - 1;
            if (CLS == A3_INNER && ip >= lo && ip <= nx2 - 1 - np) pressure(ip, BoolT<true>{});
            else pressure(ip, BoolT<false>{});
        }
        load_ppsi(i);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            vxb[r] = vxa[r];
            vxa[r] = vxn[r];
            vzp[r] = vzn[r];
            pp[r] = pc[r];
            pc[r] = pnx[r];
            kkp[r] = cK[(w * R + r) * 32 + lane];
        }
        __syncthreads();
    }
    if (i1 > i0) {
        const int ip = i1 - 1;
        if (CLS == A3_INNER && ip >= lo && ip <= nx2 - 1 - np) pressure(ip, BoolT<true>{});
        else pressure(ip, BoolT<false>{});
    }
    if (overflow) atomicExch(a.err, 4);
}

template <int W, int D, int MINB, int CLS>
__global__ void __launch_bounds__(32 * W, MINB)
    a3d_bstep_kernel(const A3Args a, const __grid_constant__ A3BMaps m) {
    if (CLS == a.step_cls && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0)
        ++*a.step;
    if (CLS == A3_INNER) {
        a3d_bstep_body<W, D, CLS, A3_FACE_GEN>(a, m, a.kt0 + blockIdx.x, a.jt0 + blockIdx.y, blockIdx.z);
        return;
    }
    int kt, jt;
    const int face = a3_edge_tile(a, blockIdx.x, kt, jt);
    const bool full = kt * 32 + 31 < a.nz2 && (jt + 1) * W * A3_BJ <= a.ny2;
#if SM_A3D_FACE_BODIES
    if (full && face == A3_FACE_Z)
        a3d_bstep_body<W, D, CLS, A3_FACE_Z, true>(a, m, kt, jt, blockIdx.z);
    else if (full && face == A3_FACE_Y)
        a3d_bstep_body<W, D, CLS, A3_FACE_Y, true>(a, m, kt, jt, blockIdx.z);
    else
#endif
    if (full)
        a3d_bstep_body<W, D, CLS, A3_FACE_GEN, true>(a, m, kt, jt, blockIdx.z);
    else
        a3d_bstep_body<W, D, CLS, A3_FACE_GEN, false>(a, m, kt, jt, blockIdx.z);
    (void)face;
}

template <int TY, int D>
constexpr size_t a3d_bstep_smem() {
    return A3BLay<TY>::head + (size_t)D * A3BLay<TY>::stage;
}

struct A3Src {
    long long q;
    long long voff;
    int len;
    // block storage: the exponent index of the cell's block, the first
    // cell of the block (A3_BJ rows apart), its rows inside the grid and the
    // source's row in it
    long long qe, qb;
    int nb, rs;
};

// the sources of one problem at the step just taken: one thread, in source
// order, as a_iso_3d.c:689-693
template <typename S>
__device__ void a3d_inject(const A3Args &a, const A3Src *src, int nsrc, const double *vals) {
    using St = Store<S>;
    using C = typename Store<S>::C;
    const long long it = *a.step - 1;
    S *P = static_cast<S *>(a.f[A_P]);
    for (int e = 0; e < nsrc; ++e) {
        const A3Src s = src[e];
        if (it >= s.len) continue;
        St::st(P + s.q, St::ld(P + s.q, a.isc[A_P]) + static_cast<C>(vals[s.voff + it]), a.sc[A_P]);
    }
}

template <typename S>
__global__ void a3d_source_kernel(A3Args a, const A3Src *src, int nsrc, const double *vals) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    a3d_inject<S>(a, src, nsrc, vals);
}

struct A3Rec {
    long long q;
    int field;
    int group;
    long long out;
    long long qe;   // block storage: the exponent index of the cell's block
};

// block storage: one thread adds the sources in order; each addition
// decodes the source cell's block, adds, and stores the block again with
// the exponent its new maximum takes (a_iso_3d.c:689-693)
__device__ void a3d_binject(const A3Args &a, const A3Src *src, int nsrc, const double *vals) {
    const long long it = *a.step - 1;
    int16_t *P = static_cast<int16_t *>(a.f[A_P]);
    uint8_t *E = static_cast<uint8_t *>(a.fe[A_P]);
    for (int e = 0; e < nsrc; ++e) {
        const A3Src s = src[e];
        if (it >= s.len) continue;
        const BDec d = bfp_dec(E[s.qe]);
        float v[A3_BJ];
        unsigned mx = 0;
        for (int r = 0; r < s.nb; ++r) {
            v[r] = bfp_val(P[s.qb + (long long)r * a.sy], d);
            if (r == s.rs) v[r] = v[r] + static_cast<float>(vals[s.voff + it]);
            mx = max(mx, bfp_absbits(v[r]));
        }
        bool over;
        const unsigned e8 = bfp_e8(mx, &over);
        const float esc = bfp_escale(e8);
        for (int r = 0; r < s.nb; ++r) P[s.qb + (long long)r * a.sy] = bfp_man(v[r], esc);
        E[s.qe] = (uint8_t)e8;
        if (over) atomicExch(a.err, 4);
    }
}

__global__ void a3d_bsource_kernel(A3Args a, const A3Src *src, int nsrc, const double *vals) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    a3d_binject(a, src, nsrc, vals);
}

// receiver r of one problem at the step just taken (a_iso_3d.c:698-741)
template <typename S>
__device__ void a3d_sample(const A3Args &a, const A3Rec *rec, int r, const int32_t *table,
                           long long nsteps_max, double *traces) {
    const long long it = *a.step - 1;
    if (it >= nsteps_max) return;
    const A3Rec e = rec[r];
    const int32_t slot = table[(long long)e.group * nsteps_max + it];
    if (slot < 0) return;
    if constexpr (std::is_same<S, Bfp16>::value) {
        const int16_t m = static_cast<const int16_t *>(a.f[e.field])[e.q];
        const unsigned e8 = static_cast<const uint8_t *>(a.fe[e.field])[e.qe];
        traces[e.out + slot] = static_cast<double>(bfp_val(m, bfp_dec(e8)));
    } else {
        const S *p = static_cast<const S *>(a.f[e.field]) + e.q;
        traces[e.out + slot] = static_cast<double>(Store<S>::ld(p, a.isc[e.field]));
    }
}

__global__ void a3d_bgather_kernel(A3Args a, const A3Rec *rec, int nrec, const int32_t *table,
                                   long long nsteps_max, double *traces) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrec) a3d_sample<Bfp16>(a, rec, r, table, nsteps_max, traces);
}

template <typename S>
__global__ void a3d_gather_kernel(A3Args a, const A3Rec *rec, int nrec, const int32_t *table,
                                  long long nsteps_max, double *traces) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrec) a3d_sample<S>(a, rec, r, table, nsteps_max, traces);
}

// ---------------------------------------------------------------------------
// Several a_iso_3d problems (grids of different sizes) in one launch per
// step: linear CTA b finds its problem in a prefix table of CTA counts; a
// problem's CTAs are its ring tiles x chunks first, then its interior tiles
// x chunks, and each runs the body the problem's own launches run for that
// tile, so every problem gets the bits of its own step.  Each problem's TMA
// maps are kernel parameters (read from parameter space like the
// single-problem launches'); its other arguments are copied into shared
// memory once per CTA.  Sources and receivers of all problems follow in one
// launch each.
// ---------------------------------------------------------------------------
constexpr int kA3GroupMax = 16;

template <typename M>
struct A3GroupStepParams {
    M m[kA3GroupMax];              // each problem's maps, old set as input
    A3Args a[kA3GroupMax];         // its arguments for this step
    int first[kA3GroupMax + 1];    // first linear CTA of each problem
    int nedge[kA3GroupMax];        // its ring tiles
    int n;
};
static_assert(sizeof(A3GroupStepParams<A3BMaps>) <= 32000, "kernel parameters are limited to 32 KB");
static_assert(sizeof(A3Args) % 4 == 0, "A3Args is copied as 32-bit words");

// problem, tile and chunk of linear CTA b; returns the tile's class
template <typename M>
__device__ __forceinline__ int a3_group_tile(const A3GroupStepParams<M> &P, A3Args &sa, int &kt,
                                             int &jt, int &ch, int &p) {
    const int b = blockIdx.x;
    p = 0;
    while (p + 1 < P.n && P.first[p + 1] <= b) ++p;
    {
        const int *src = reinterpret_cast<const int *>(&P.a[p]);
        int *dst = reinterpret_cast<int *>(&sa);
        const int tid = threadIdx.y * blockDim.x + threadIdx.x;
        for (int i = tid; i < (int)(sizeof(A3Args) / 4); i += blockDim.x * blockDim.y) dst[i] = src[i];
    }
    __syncthreads();
    int local = b - P.first[p];
    if (local == 0 && threadIdx.x == 0 && threadIdx.y == 0) ++*sa.step;
    const int ne = P.nedge[p];
    const int nch = (sa.nx2 + sa.chunk - 1) / sa.chunk;
    if (local < ne * nch) {
        ch = local / ne;
        a3_edge_tile(sa, local % ne, kt, jt);
        return A3_EDGE;
    }
    local -= ne * nch;
    const int nk = sa.kt1 - sa.kt0, nin = nk * (sa.jt1 - sa.jt0);
    ch = local / nin;
    kt = sa.kt0 + (local % nin) % nk;
    jt = sa.jt0 + (local % nin) / nk;
    return A3_INNER;
}

template <typename S, int W, int R, int D, int MINB>
__global__ void __launch_bounds__(32 * W, MINB)
    a3d_group_step_kernel(const __grid_constant__ A3GroupStepParams<A3Maps> P) {
    __shared__ A3Args sa;
    int kt, jt, ch, p;
    if (a3_group_tile(P, sa, kt, jt, ch, p) == A3_EDGE)
        a3d_step_body<S, W, R, D, A3_EDGE, A3_FACE_GEN>(sa, P.m[p], kt, jt, ch);
    else
        a3d_step_body<S, W, R, D, A3_INNER, A3_FACE_GEN>(sa, P.m[p], kt, jt, ch);
}

template <int W, int D, int MINB>
__global__ void __launch_bounds__(32 * W, MINB)
    a3d_bgroup_step_kernel(const __grid_constant__ A3GroupStepParams<A3BMaps> P) {
    __shared__ A3Args sa;
    int kt, jt, ch, p;
    if (a3_group_tile(P, sa, kt, jt, ch, p) == A3_EDGE)
        a3d_bstep_body<W, D, A3_EDGE, A3_FACE_GEN>(sa, P.m[p], kt, jt, ch);
    else
        a3d_bstep_body<W, D, A3_INNER, A3_FACE_GEN>(sa, P.m[p], kt, jt, ch);
}

// what the source and receiver kernels of one problem need after its step
struct A3Post {
    A3Args a;                 // bound to the state just written
    const A3Src *src;
    const double *vals;
    const A3Rec *rec;
    const int32_t *table;
    long long nsteps_max;
    double *traces;
    int nsrc;
};

struct A3GroupPostParams {
    A3Post q[kA3GroupMax];
    int first_rec[kA3GroupMax + 1];   // prefix sums of the problems' receivers
    int n;
};
static_assert(sizeof(A3GroupPostParams) <= 32000, "kernel parameters are limited to 32 KB");

// block p adds problem p's sources (one thread, in source order)
template <typename S>
__global__ void a3d_group_source_kernel(const __grid_constant__ A3GroupPostParams P) {
    if (threadIdx.x != 0 || (int)blockIdx.x >= P.n) return;
    const A3Post &q = P.q[blockIdx.x];
    if (q.nsrc == 0) return;
    if constexpr (std::is_same<S, Bfp16>::value)
        a3d_binject(q.a, q.src, q.nsrc, q.vals);
    else
        a3d_inject<S>(q.a, q.src, q.nsrc, q.vals);
}

template <typename S>
__global__ void a3d_group_gather_kernel(const __grid_constant__ A3GroupPostParams P) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.first_rec[P.n]) return;
    int p = 0;
    while (p + 1 < P.n && P.first_rec[p + 1] <= t) ++p;
    const A3Post &q = P.q[p];
    a3d_sample<S>(q.a, q.rec, t - P.first_rec[p], q.table, q.nsteps_max, q.traces);
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
    // the edge-tile launch runs on `side`, forked from and joined back to
    // `stream` by the two events, so it overlaps the interior launch
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    A3Args args{};
    DevBuf f[2][4], psi[2][6], rho, K, coef;   // two buffer sets (ping-pong)
    int cur = 0;                               // set holding the current state
    int config = 8;                            // index into kA3Configs
    uint64_t serial = 0;                       // unique per handle (grouped graphs' keys)
    int sms = 148;
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
    KernelTimer timer;
    A3Maps maps[2];                            // TMA maps with set b as input
    A3BMaps bmaps[2];                          // ... for block storage (SM_BFP16)
    int maps_ty = -1;                          // tile rows the maps were made for
    // block storage: exponent bytes of the four fields per buffer set,
    // [nx2][nyb][pitch], nyb = ceil(ny2 / A3_BJ)
    DevBuf fe[2][4];
    size_t nyb = 0;
    DevBuf err;                                // kernel timeout flag
    DevBuf d_step;                             // device step counter (A3Args::step)
    // CUDA graphs of graph_steps steps, one per parity of the starting
    // buffer set; captured again when graph_epoch moved since
    int graph_steps = 0;
    unsigned graph_epoch = 1;
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        unsigned epoch = 0;
        int steps = 0;
        bool timed = false;      // captured with per-kernel timing on
        EventPairs tev;          // the timed launches' event nodes
    } graphs[2];
    ~sm_a3d() {
        for (Graph &g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            for (auto &p : g.tev) {
                cudaEventDestroy(p.first);
                cudaEventDestroy(p.second);
            }
        }
    }
    // 16-bit storage: exponents of the 4 fields (A_*) and 6 memory
    // variables (4 + PS_*), stored = value * 2^expo
    Scaler16 scaler;
    std::vector<int> expo0;                    // exponents restored by reset
    double rho_min = 0, vp_min = 0, hmin = 0;
    static constexpr int kScalePeriod = 16;    // steps between range checks
};

namespace {

int a3d_check(sm_a3d_t h) {
    if (!h) return sm_fail(SM_EINVAL, "null a_iso_3d handle");
    return SM_OK;
}

void a3d_bind(sm_a3d *h, int in) {
    for (int f = 0; f < 4; ++f) {
        h->args.f[f] = h->f[in][f].p;
        h->args.fo[f] = h->f[1 - in][f].p;
        h->args.fe[f] = h->fe[in][f].p;
        h->args.feo[f] = h->fe[1 - in][f].p;
    }
    for (int p = 0; p < 6; ++p) {
        h->args.psi[p] = h->psi[in][p].p;
        h->args.pso[p] = h->psi[1 - in][p].p;
    }
}

// launch configurations of the fused step: tile rows, ring stages and the
// minimum resident CTAs per SM the register budget is fitted to
struct A3Config {
    int warps, rows, stages, minb;
    int ty() const { return warps * rows; }
};
static const A3Config kA3Configs[] = {
    {8, 2, 5, 2}, {4, 4, 5, 3}, {8, 4, 4, 1}, {8, 1, 6, 3},
    {16, 2, 4, 1}, {4, 2, 6, 4}, {8, 2, 4, 3}, {4, 8, 4, 2},
    // 8: a 3-stage ring (one plane in flight), 64 registers: 4 CTAs of 8
    // warps per SM; the fastest measured at 288^3 and 544^3 (0.230 and 1.215
    // ms per step against 0.239 and 1.290 for configuration 6)
    {8, 2, 3, 4},
};
static const int kA3NumConfigs = sizeof(kA3Configs) / sizeof(kA3Configs[0]);
// block storage: every thread holds one block of A3_BJ rows
static const A3Config kA3BConfigs[] = {
    {8, A3_BJ, 4, 2}, {4, A3_BJ, 4, 3}, {8, A3_BJ, 5, 1}, {4, A3_BJ, 6, 3}, {16, A3_BJ, 4, 1},
    {8, A3_BJ, 4, 3}, {4, A3_BJ, 4, 5},
};
static const int kA3BNumConfigs = sizeof(kA3BConfigs) / sizeof(kA3BConfigs[0]);

bool a3d_isb(const sm_a3d *h) { return h->precision == SM_BFP16; }
const A3Config &a3d_cfg(const sm_a3d *h, int c) {
    return a3d_isb(h) ? kA3BConfigs[c] : kA3Configs[c];
}
int a3d_ncfg(const sm_a3d *h) { return a3d_isb(h) ? kA3BNumConfigs : kA3NumConfigs; }

// The interior rectangle of tiles for tile rows ty: tiles (32 k x ty j)
// whose every cell is clear in y and z of the CPML frame and of the grid
// edge (velocity half nodes np .. n2-2-np, pressure nodes max(np,1) ..
// n2-1-np), the same test the step kernel makes per tile.  Empty when no
// tile qualifies; the edge class is then every tile.
void a3d_tile_classes(sm_a3d *h, int ty) {
    A3Args &a = h->args;
    const long long np = (long long)h->np, lo = np > 1 ? np : 1;
    a.nkt = (int)((h->nz2 + 31) / 32);
    a.njt = (int)((h->ny2 + ty - 1) / ty);
    auto range = [&](long long n2, int w, int nt, int &t0, int &t1) {
        t0 = (int)((lo + w - 1) / w);                      // first t with t*w >= lo
        const long long last = (long long)n2 - 2 - np - (w - 1);
        t1 = last < 0 ? 0 : (int)(last / w) + 1;           // t*w + w-1 <= n2-2-np
        if (t1 > nt) t1 = nt;
        if (t1 < t0) t1 = t0;
    };
    range((long long)h->nz2, 32, a.nkt, a.kt0, a.kt1);
    range((long long)h->ny2, ty, a.njt, a.jt0, a.jt1);
    if (a.kt1 == a.kt0 || a.jt1 == a.jt0) {
        a.kt0 = a.kt1 = 0;
        a.jt0 = a.jt1 = a.njt;
    }
}

// step kernels one step launches: one per non-empty tile class
int a3d_step_kernels(sm_a3d *h) {
    a3d_tile_classes(h, a3d_cfg(h, h->config).ty());
    const A3Args &a = h->args;
    const int ninner = (a.kt1 - a.kt0) * (a.jt1 - a.jt0);
    return (ninner > 0) + (a.nkt * a.njt - ninner > 0);
}

// dynamic shared memory above 48 KB must be allowed per kernel and device;
// handles are created from several threads (the request loop's worker and
// its callers), so the per-device flags are read and set under a lock
template <typename S, int W, int R, int D, int MINB>
int a3d_ready_cfg(sm_a3d *h) {
    static std::mutex mu;
    static bool done[64] = {};   // per instantiation and device
    if (h->device < 0 || h->device >= 64) return sm_fail(SM_EINVAL, "device %d", h->device);
    std::lock_guard<std::mutex> lk(mu);
    if (!done[h->device]) {
        SM_CUDA_TRY(cudaFuncSetAttribute(a3d_step_kernel<S, W, R, D, MINB, A3_INNER>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)a3d_step_smem<S, W * R, D>()));
        SM_CUDA_TRY(cudaFuncSetAttribute(a3d_step_kernel<S, W, R, D, MINB, A3_EDGE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)a3d_step_smem<S, W * R, D>()));
        done[h->device] = true;
    }
    return SM_OK;
}

template <int W, int D, int MINB>
int a3d_bready_cfg(sm_a3d *h) {
    static std::mutex mu;
    static bool done[64] = {};
    if (h->device < 0 || h->device >= 64) return sm_fail(SM_EINVAL, "device %d", h->device);
    std::lock_guard<std::mutex> lk(mu);
    if (!done[h->device]) {
        SM_CUDA_TRY(cudaFuncSetAttribute(a3d_bstep_kernel<W, D, MINB, A3_INNER>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)a3d_bstep_smem<W * A3_BJ, D>()));
        SM_CUDA_TRY(cudaFuncSetAttribute(a3d_bstep_kernel<W, D, MINB, A3_EDGE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)a3d_bstep_smem<W * A3_BJ, D>()));
        done[h->device] = true;
    }
    return SM_OK;
}

// the block-storage step: the same two tile classes as the FP32 step
template <int W, int D, int MINB>
int a3d_blaunch_cfg(sm_a3d *h) {
    constexpr int TY = W * A3_BJ;
    constexpr size_t smem = a3d_bstep_smem<TY, D>();
    A3Args &a = h->args;
    a3d_tile_classes(h, TY);
    const unsigned nch = (unsigned)((h->nx2 + a.chunk - 1) / a.chunk);
    const int ninner = (a.kt1 - a.kt0) * (a.jt1 - a.jt0);
    const int nedge = a.nkt * a.njt - ninner;
    a.step_cls = ninner > 0 ? A3_INNER : A3_EDGE;
    dim3 blk(32, W, 1);
    if (nedge > 0 && ninner > 0) {
        cudaEventRecord(h->ev_fork, h->stream);
        cudaStreamWaitEvent(h->side, h->ev_fork, 0);
    }
    if (nedge > 0)
        a3d_bstep_kernel<W, D, MINB, A3_EDGE>
            <<<dim3((unsigned)nedge, 1, nch), blk, smem, ninner > 0 ? h->side : h->stream>>>(
                a, h->bmaps[h->cur]);
    if (ninner > 0)
        a3d_bstep_kernel<W, D, MINB, A3_INNER>
            <<<dim3((unsigned)(a.kt1 - a.kt0), (unsigned)(a.jt1 - a.jt0), nch), blk, smem,
               h->stream>>>(a, h->bmaps[h->cur]);
    if (nedge > 0 && ninner > 0) {
        cudaEventRecord(h->ev_join, h->side);
        cudaStreamWaitEvent(h->stream, h->ev_join, 0);
    }
    return (nedge > 0) + (ninner > 0);
}

template <typename S, int W, int R, int D, int MINB>
int a3d_launch_cfg(sm_a3d *h) {
    constexpr int TY = W * R;
    constexpr size_t smem = a3d_step_smem<S, TY, D>();
    A3Args &a = h->args;
    a3d_tile_classes(h, TY);
    const unsigned nch = (unsigned)((h->nx2 + a.chunk - 1) / a.chunk);
    const int ninner = (a.kt1 - a.kt0) * (a.jt1 - a.jt0);
    const int nedge = a.nkt * a.njt - ninner;
    a.step_cls = ninner > 0 ? A3_INNER : A3_EDGE;
    dim3 blk(32, W, 1);
    if (nedge > 0 && ninner > 0) {   // fork: the edge ring first, on the side stream
        cudaEventRecord(h->ev_fork, h->stream);
        cudaStreamWaitEvent(h->side, h->ev_fork, 0);
    }
    if (nedge > 0)
        a3d_step_kernel<S, W, R, D, MINB, A3_EDGE>
            <<<dim3((unsigned)nedge, 1, nch), blk, smem, ninner > 0 ? h->side : h->stream>>>(
                a, h->maps[h->cur]);
    if (ninner > 0)
        a3d_step_kernel<S, W, R, D, MINB, A3_INNER>
            <<<dim3((unsigned)(a.kt1 - a.kt0), (unsigned)(a.jt1 - a.jt0), nch), blk, smem,
               h->stream>>>(a, h->maps[h->cur]);
    if (nedge > 0 && ninner > 0) {   // join
        cudaEventRecord(h->ev_join, h->side);
        cudaStreamWaitEvent(h->stream, h->ev_join, 0);
    }
    return (nedge > 0) + (ninner > 0);
}

// TMA maps of one buffer set (as the step's input) for tile rows ty; box
// shapes follow A3Lay
template <typename S>
int a3d_make_maps(sm_a3d *h, int ty) {
    using C = typename Store<S>::C;
    const int HS = 16 / (int)sizeof(S), HC = 16 / (int)sizeof(C);
    const CUtensorMapDataType ds = MapType<S>::v, dc = MapType<C>::v;
    const size_t n0 = h->nz2, n1 = h->ny2, n2 = h->nx2, pt = h->pitch;
    int rc;
    for (int b = 0; b < 2; ++b) {
        A3Maps &m = h->maps[b];
        if ((rc = make_map_3d(&m.P, h->f[b][A_P].p, ds, sizeof(S), n0, n1, n2, pt, 32 + 2 * HS, ty + 2)))
            return rc;
        if ((rc = make_map_3d(&m.vx, h->f[b][A_VX].p, ds, sizeof(S), n0, n1, n2, pt, 32, ty))) return rc;
        if ((rc = make_map_3d(&m.vy, h->f[b][A_VY].p, ds, sizeof(S), n0, n1, n2, pt, 32, ty + 1)))
            return rc;
        if ((rc = make_map_3d(&m.vz, h->f[b][A_VZ].p, ds, sizeof(S), n0, n1, n2, pt, 32 + HS, ty)))
            return rc;
        if ((rc = make_map_3d(&m.rho, h->rho.p, dc, sizeof(C), n0, n1, n2, pt, 32 + 2 * HC, ty + 2)))
            return rc;
        if ((rc = make_map_3d(&m.K, h->K.p, dc, sizeof(C), n0, n1, n2, pt, 32, ty))) return rc;
    }
    h->maps_ty = ty;
    h->graph_epoch++;   // maps are baked into captured graphs
    return SM_OK;
}

// TMA maps of block storage: int16 mantissas and exponent bytes, boxes as
// A3BLay
int a3d_make_bmaps(sm_a3d *h, int ty) {
    const size_t n0 = h->nz2, n1 = h->ny2, n2 = h->nx2, pt = h->pitch, nb = h->nyb;
    const CUtensorMapDataType i16 = CU_TENSOR_MAP_DATA_TYPE_UINT16, u8 = CU_TENSOR_MAP_DATA_TYPE_UINT8;
    const CUtensorMapDataType f32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const unsigned nbt = (unsigned)(ty / A3_BJ);
    int rc;
    for (int b = 0; b < 2; ++b) {
        A3BMaps &m = h->bmaps[b];
        if ((rc = make_map_3d(&m.P, h->f[b][A_P].p, i16, 2, n0, n1, n2, pt, 48, ty + 2))) return rc;
        if ((rc = make_map_3d(&m.eP, h->fe[b][A_P].p, u8, 1, n0, nb, n2, pt, 64, nbt + 2))) return rc;
        if ((rc = make_map_3d(&m.vx, h->f[b][A_VX].p, i16, 2, n0, n1, n2, pt, 32, ty))) return rc;
        if ((rc = make_map_3d(&m.eX, h->fe[b][A_VX].p, u8, 1, n0, nb, n2, pt, 32, nbt))) return rc;
        if ((rc = make_map_3d(&m.vy, h->f[b][A_VY].p, i16, 2, n0, n1, n2, pt, 32, ty + 1))) return rc;
        if ((rc = make_map_3d(&m.eY, h->fe[b][A_VY].p, u8, 1, n0, nb, n2, pt, 32, nbt + 1))) return rc;
        if ((rc = make_map_3d(&m.vz, h->f[b][A_VZ].p, i16, 2, n0, n1, n2, pt, 40, ty))) return rc;
        if ((rc = make_map_3d(&m.eZ, h->fe[b][A_VZ].p, u8, 1, n0, nb, n2, pt, 48, nbt))) return rc;
        if ((rc = make_map_3d(&m.rho, h->rho.p, f32, 4, n0, n1, n2, pt, 40, ty + 2))) return rc;
        if ((rc = make_map_3d(&m.K, h->K.p, f32, 4, n0, n1, n2, pt, 32, ty))) return rc;
    }
    h->maps_ty = ty;
    h->graph_epoch++;   // maps are baked into captured graphs
    return SM_OK;
}

int a3d_ensure_maps(sm_a3d *h) {
    const int ty = a3d_cfg(h, h->config).ty();
    if (h->maps_ty == ty) return SM_OK;
    switch (h->precision) {
    case SM_BFP16: return a3d_make_bmaps(h, ty);
    case SM_FP64: return a3d_make_maps<double>(h, ty);
    case SM_FP16: return a3d_make_maps<__half>(h, ty);
    case SM_BF16: return a3d_make_maps<__nv_bfloat16>(h, ty);
    default: return a3d_make_maps<float>(h, ty);
    }
}

bool a3d_is16(const sm_a3d *h) { return h->precision == SM_FP16 || h->precision == SM_BF16; }

void a3d_apply_scales(sm_a3d *h) {
    for (int f = 0; f < 4; ++f) {
        h->args.sc[f] = std::ldexp(1.0f, h->scaler.expo[f]);
        h->args.isc[f] = std::ldexp(1.0f, -h->scaler.expo[f]);
    }
    for (int q = 0; q < 6; ++q) {
        h->args.psc[q] = std::ldexp(1.0f, h->scaler.expo[4 + q]);
        h->args.pisc[q] = std::ldexp(1.0f, -h->scaler.expo[4 + q]);
    }
}

int a3d_rescale(sm_a3d *h) {
    void *ptrs[10];
    size_t ns[10];
    const size_t ncell = h->nx2 * h->ny2 * (size_t)h->pitch;
    static const char *names[10] = {"vx", "vy", "vz", "P", "psi_Px", "psi_Py", "psi_Pz",
                                    "psi_vx", "psi_vy", "psi_vz"};
    static const int groups[10] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9};
    for (int f = 0; f < 4; ++f) { ptrs[f] = h->f[h->cur][f].p; ns[f] = ncell; }
    for (int q = 0; q < 6; ++q) { ptrs[4 + q] = h->psi[h->cur][q].p; ns[4 + q] = h->psi_cells[q]; }
    const std::vector<int> before = h->scaler.expo;
    int rc = h->precision == SM_FP16
                 ? h->scaler.check<__half>(h->stream, 10, ptrs, ns, groups, names)
                 : h->scaler.check<__nv_bfloat16>(h->stream, 10, ptrs, ns, groups, names);
    a3d_apply_scales(h);
    if (h->scaler.expo != before) h->graph_epoch++;   // scales are baked into graphs
    return rc;
}

int a3d_check_err(sm_a3d *h) {
    int e = 0;
    SM_CUDA_TRY(cudaMemcpy(&e, h->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e == 4)
        return sm_fail(SM_ESTATE, "a_iso_3d: a block of the 16-bit block storage exceeded its "
                                  "range (|value| >= 2^114)");
    if (e) return sm_fail(SM_ETIMEOUT, "a_iso_3d step kernel: a bounded wait for a TMA load gave up");
    return SM_OK;
}

template <typename S>
size_t a3d_config_smem(int config) {
    switch (config) {
    case 0: return a3d_step_smem<S, 16, 5>();
    case 1: return a3d_step_smem<S, 16, 5>();
    case 2: return a3d_step_smem<S, 32, 4>();
    case 3: return a3d_step_smem<S, 8, 6>();
    case 4: return a3d_step_smem<S, 32, 4>();
    case 5: return a3d_step_smem<S, 8, 6>();
    case 6: return a3d_step_smem<S, 16, 4>();
    case 8: return a3d_step_smem<S, 16, 3>();
    default: return a3d_step_smem<S, 32, 4>();
    }
}

// the block-storage configurations of kA3BConfigs as template arguments
size_t a3d_bconfig_smem(int config) {
    switch (config) {
    case 0: return a3d_bstep_smem<8 * A3_BJ, 4>();
    case 1: return a3d_bstep_smem<4 * A3_BJ, 4>();
    case 2: return a3d_bstep_smem<8 * A3_BJ, 5>();
    case 3: return a3d_bstep_smem<4 * A3_BJ, 6>();
    case 5: return a3d_bstep_smem<8 * A3_BJ, 4>();
    case 6: return a3d_bstep_smem<4 * A3_BJ, 4>();
    default: return a3d_bstep_smem<16 * A3_BJ, 4>();
    }
}

int a3d_bready(sm_a3d *h) {
    switch (h->config) {
    case 0: return a3d_bready_cfg<8, 4, 2>(h);
    case 1: return a3d_bready_cfg<4, 4, 3>(h);
    case 2: return a3d_bready_cfg<8, 5, 1>(h);
    case 3: return a3d_bready_cfg<4, 6, 3>(h);
    case 5: return a3d_bready_cfg<8, 4, 3>(h);
    case 6: return a3d_bready_cfg<4, 4, 5>(h);
    default: return a3d_bready_cfg<16, 4, 1>(h);
    }
}

int a3d_blaunch_step(sm_a3d *h) {
    switch (h->config) {
    case 0: return a3d_blaunch_cfg<8, 4, 2>(h);
    case 1: return a3d_blaunch_cfg<4, 4, 3>(h);
    case 2: return a3d_blaunch_cfg<8, 5, 1>(h);
    case 3: return a3d_blaunch_cfg<4, 6, 3>(h);
    case 5: return a3d_blaunch_cfg<8, 4, 3>(h);
    case 6: return a3d_blaunch_cfg<4, 4, 5>(h);
    default: return a3d_blaunch_cfg<16, 4, 1>(h);
    }
}

size_t a3d_config_smem_prec(int precision, int config) {
    switch (precision) {
    case SM_BFP16: return a3d_bconfig_smem(config);
    case SM_FP64: return a3d_config_smem<double>(config);
    case SM_FP16: return a3d_config_smem<__half>(config);
    case SM_BF16: return a3d_config_smem<__nv_bfloat16>(config);
    default: return a3d_config_smem<float>(config);
    }
}

template <typename S>
int a3d_ready(sm_a3d *h) {
    switch (h->config) {
    case 0: return a3d_ready_cfg<S, 8, 2, 5, 2>(h);
    case 1: return a3d_ready_cfg<S, 4, 4, 5, 3>(h);
    case 2: return a3d_ready_cfg<S, 8, 4, 4, 1>(h);
    case 3: return a3d_ready_cfg<S, 8, 1, 6, 3>(h);
    case 4: return a3d_ready_cfg<S, 16, 2, 4, 1>(h);
    case 5: return a3d_ready_cfg<S, 4, 2, 6, 4>(h);
    case 6: return a3d_ready_cfg<S, 8, 2, 4, 3>(h);
    case 8: return a3d_ready_cfg<S, 8, 2, 3, 4>(h);
    default: return a3d_ready_cfg<S, 4, 8, 4, 2>(h);
    }
}

// the step's kernels (one per non-empty tile class); returns how many
template <typename S>
int a3d_launch_step(sm_a3d *h) {
    switch (h->config) {
    case 0: return a3d_launch_cfg<S, 8, 2, 5, 2>(h);
    case 1: return a3d_launch_cfg<S, 4, 4, 5, 3>(h);
    case 2: return a3d_launch_cfg<S, 8, 4, 4, 1>(h);
    case 3: return a3d_launch_cfg<S, 8, 1, 6, 3>(h);
    case 4: return a3d_launch_cfg<S, 16, 2, 4, 1>(h);
    case 5: return a3d_launch_cfg<S, 4, 2, 6, 4>(h);
    case 6: return a3d_launch_cfg<S, 8, 2, 4, 3>(h);
    case 8: return a3d_launch_cfg<S, 8, 2, 3, 4>(h);
    default: return a3d_launch_cfg<S, 4, 8, 4, 2>(h);
    }
}

template <typename S>
void a3d_launch(sm_a3d *h) {
    constexpr bool B = std::is_same<S, Bfp16>::value;
    a3d_bind(h, h->cur);
    cudaEvent_t t0 = h->timer.begin(h->stream);
    int nstep;
    if constexpr (B) nstep = a3d_blaunch_step(h);
    else nstep = a3d_launch_step<S>(h);
    h->timer.end(t0, h->stream);
    h->cur = 1 - h->cur;
    // sources and receivers act on the state just written
    a3d_bind(h, h->cur);
    h->timer.launches += nstep + (h->src.empty() ? 0 : 1) + (h->rec.empty() ? 0 : 1);
    if (!h->src.empty()) {
        if constexpr (B)
            a3d_bsource_kernel<<<1, 32, 0, h->stream>>>(h->args, h->d_src.as<A3Src>(),
                                                        (int)h->src.size(), h->d_vals.as<double>());
        else
            a3d_source_kernel<S><<<1, 32, 0, h->stream>>>(h->args, h->d_src.as<A3Src>(),
                                                          (int)h->src.size(), h->d_vals.as<double>());
    }
    if (!h->rec.empty()) {
        int n = (int)h->rec.size();
        if constexpr (B)
            a3d_bgather_kernel<<<(n + 127) / 128, 128, 0, h->stream>>>(
                h->args, h->d_rec.as<A3Rec>(), n, h->d_table.as<int32_t>(),
                (long long)h->plan.nsteps_max, h->d_traces.as<double>());
        else
            a3d_gather_kernel<S><<<(n + 127) / 128, 128, 0, h->stream>>>(
                h->args, h->d_rec.as<A3Rec>(), n, h->d_table.as<int32_t>(),
                (long long)h->plan.nsteps_max, h->d_traces.as<double>());
    }
}

// x planes per CTA: enough CTAs for a few waves on the device, at least
// 16 planes per chunk so the recomputed plane i0-1 and the pipeline fill stay
// cheap.  Scalar storage (4 CTAs per SM) keeps chunks short, at most 20
// planes, so a launch runs many waves and its last, partial one is short
// (544^3 FP32: 1.22 ms per step with 16-20 planes, 1.38 with 64); block
// storage (2 CTAs per SM, a costlier fill per chunk) aims at half the CTAs
// and takes up to 64 planes (544^3: 1.23 ms with 48-64, 1.28 with 16).
int a3d_pick_chunk(size_t nx2, size_t ny2, size_t nz2, int sms, int ty, bool block) {
    const size_t tiles = ((nz2 + 31) / 32) * ((ny2 + ty - 1) / ty);
    const size_t want = (size_t)sms * (block ? 8 : 16);
    size_t nch = (want + tiles - 1) / tiles;
    if (nch < 1) nch = 1;
    size_t chunk = (nx2 + nch - 1) / nch;
    const size_t cap = block ? A3_CHMAX : 20;
    if (chunk > cap) chunk = (nx2 + (nx2 + cap - 1) / cap - 1) / ((nx2 + cap - 1) / cap);
    if (chunk < 16) chunk = 16;
    if (chunk > nx2) chunk = nx2;
    return (int)chunk;
}

int a3d_default_chunk(const sm_a3d *h, int config) {
    return a3d_pick_chunk(h->nx2, h->ny2, h->nz2, h->sms, a3d_cfg(h, config).ty(), a3d_isb(h));
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

static size_t a3d_mb2(size_t b) { return (b + (2u << 20) - 1) / (2u << 20) * (2u << 20); }

extern "C" int sm_a3d_device_bytes(size_t nx2, size_t ny2, size_t nz2, size_t np, int precision,
                                   size_t nrec, size_t nsteps_max, size_t *bytes) {
    if (!bytes) return sm_fail(SM_EINVAL, "sm_a3d_device_bytes: NULL");
    if (precision < SM_FP32 || precision > SM_BFP16)
        return sm_fail(SM_EINVAL, "sm_a3d_device_bytes: unknown precision %d", precision);
    const size_t pitch = round_up(nz2, 32), ncell = nx2 * ny2 * pitch;
    const size_t e = storage_bytes(precision), c = precision == SM_FP64 ? 8 : 4;
    const size_t pe = precision == SM_BFP16 ? 4 : e;          // CPML memory variables
    const size_t slabs = 2 * (2 * np * ny2 * pitch + nx2 * 2 * np * pitch + nx2 * ny2 * 2 * np);
    size_t b = 8 * a3d_mb2(ncell * e);                        // 4 fields, two sets
    if (precision == SM_BFP16)                                // their exponents
        b += 8 * a3d_mb2(nx2 * ((ny2 + A3_BJ - 1) / A3_BJ) * pitch);
    b += 2 * a3d_mb2(slabs * pe);                             // CPML memory variables
    b += 2 * a3d_mb2(ncell * c);                              // rho, K
    b += a3d_mb2(18 * (nx2 + ny2 + nz2) * c);                 // coefficients
    b += a3d_mb2(nrec * nsteps_max * (sizeof(double) + sizeof(int32_t)));
    b += 16u << 20;
    *bytes = b;
    return SM_OK;
}

// The model a handle is made from: the padded volume (pad = 0, extents
// nx2 x ny2 x nz2), or the unpadded one (extents nx x ny x nz) whose padded
// nodes take the value of the nearest interior node (io_utils.c:1096-1143),
// gathered as the materials are staged.
struct A3Model {
    const double *vp, *rho;
    size_t nx, ny, nz, pad;
    static size_t clamp(size_t n, size_t pad, size_t ext) {
        return n < pad ? 0 : (n - pad >= ext ? ext - 1 : n - pad);
    }
    // offset of the source row of padded row (i, j)
    size_t row(size_t i, size_t j) const { return (clamp(i, pad, nx) * ny + clamp(j, pad, ny)) * nz; }
    size_t col(size_t k) const { return clamp(k, pad, nz); }
};

// pitched rho and K = rho vp^2 dt (a_iso_3d.c:407-409) in the compute type,
// filled by a few host threads straight into the upload buffers (the model
// of a large grid is hundreds of MB).  Pitch padding: rho repeats the last
// real value so the on-the-fly buoyancy never divides by zero there (those
// cells are not updated), K is zero.
template <typename C>
int a3d_upload_materials(sm_a3d *h, const A3Model &m, double dt, size_t nx2, size_t ny2,
                         size_t nz2) {
    const size_t pitch = (size_t)h->pitch, ncell = nx2 * ny2 * pitch;
    // pinned staging (cached across handles): the copies run at full link speed
    PinnedBuf rb, kb;
    if (int rc = rb.get(ncell * sizeof(C))) return rc;
    if (int rc = kb.get(ncell * sizeof(C))) return rc;
    C *r = rb.as<C>(), *kk = kb.as<C>();
    const double *rho = m.rho, *vp = m.vp;
    auto fill = [&](size_t ib, size_t ie) {
        for (size_t i = ib; i < ie; ++i)
            for (size_t j = 0; j < ny2; ++j) {
                const size_t s0 = m.row(i, j), d0 = (i * ny2 + j) * pitch;
                for (size_t k = 0; k < nz2; ++k) {
                    const size_t sk = s0 + m.col(k);
                    r[d0 + k] = static_cast<C>(rho[sk]);
                    kk[d0 + k] = static_cast<C>(rho[sk] * vp[sk] * vp[sk] * dt);
                }
                for (size_t k = nz2; k < pitch; ++k) {
                    r[d0 + k] = r[d0 + nz2 - 1];
                    kk[d0 + k] = C(0);
                }
            }
    };
    // each thread fills its x planes in a few pieces and queues the copy of
    // a piece as soon as it is filled, so the link carries the first pieces
    // while the later ones are filled
    const size_t plane = ny2 * pitch;
    const int device = h->device;
    cudaStream_t st = h->stream;
    std::atomic<int> failed{0};
    auto part = [&](size_t ib, size_t ie) {
        cudaSetDevice(device);
        constexpr size_t kPieces = 4;
        for (size_t p = 0; p < kPieces; ++p) {
            const size_t pb = ib + (ie - ib) * p / kPieces, pe = ib + (ie - ib) * (p + 1) / kPieces;
            if (pb == pe) continue;
            fill(pb, pe);
            const size_t off = pb * plane, n = (pe - pb) * plane * sizeof(C);
            if (cudaMemcpyAsync(h->rho.as<C>() + off, r + off, n, cudaMemcpyHostToDevice, st) !=
                    cudaSuccess ||
                cudaMemcpyAsync(h->K.as<C>() + off, kk + off, n, cudaMemcpyHostToDevice, st) !=
                    cudaSuccess)
                failed = 1;
        }
    };
    const size_t nt = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 16);
    std::vector<std::thread> pool;
    for (size_t t = 0; t < nt; ++t) {
        const size_t ib = nx2 * t / nt, ie = nx2 * (t + 1) / nt;
        if (ib < ie) pool.emplace_back(part, ib, ie);
    }
    for (auto &th : pool) th.join();
    // the staging goes back to the cache only after every copy has run
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (failed) return sm_fail(SM_ECUDA, "sm_a3d_create: material upload failed");
    return SM_OK;
}

namespace {

int a3d_create(int device, size_t nx2, size_t ny2, size_t nz2, size_t np, double dx, double dy,
               double dz, double dt, const A3Model &m, const double *const *coef, int precision,
               sm_a3d_t *out) {
    if (!out) return sm_fail(SM_EINVAL, "sm_a3d_create: out is NULL");
    *out = nullptr;
    if (nx2 < 2 * np + 2 || ny2 < 2 * np + 2 || nz2 < 2 * np + 2)
        return sm_fail(SM_EINVAL, "sm_a3d_create: grid smaller than the CPML frame");
    if (!m.vp || !m.rho || !coef) return sm_fail(SM_EINVAL, "sm_a3d_create: NULL array");
    for (int c = 0; c < 18; ++c)
        if (!coef[c]) return sm_fail(SM_EINVAL, "sm_a3d_create: NULL coefficient array");
    if (!(dx > 0) || !(dy > 0) || !(dz > 0) || !(dt > 0))
        return sm_fail(SM_EINVAL, "sm_a3d_create: spacings and dt must be > 0");
    if (precision < SM_FP32 || precision > SM_BFP16)
        return sm_fail(SM_EINVAL, "sm_a3d_create: unknown precision %d", precision);
    if (ny2 > 65535 * 4 || nx2 > 65535 || (double)nx2 * ny2 * (nz2 + 31) >= 2147483647.0)
        return sm_fail(SM_EINVAL, "sm_a3d_create: grid too large (cells must stay below 2^31)");
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
    if (precision == SM_BFP16) h->config = 0;   // index into the block-storage table
    SM_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    SM_CUDA_TRY(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
    SM_CUDA_TRY(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    SM_CUDA_TRY(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    const size_t cb = precision == SM_FP64 ? 8 : 4;
    const size_t ncell = nx2 * ny2 * (size_t)h->pitch;
    int rc;
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < 4; ++f)
            if ((rc = h->f[b][f].alloc_pooled(ncell * h->elem, device))) return rc;
    h->psi_cells[PS_PX] = h->psi_cells[PS_VX] = 2 * np * ny2 * (size_t)h->pitch;
    h->psi_cells[PS_PY] = h->psi_cells[PS_VY] = nx2 * 2 * np * (size_t)h->pitch;
    h->psi_cells[PS_PZ] = h->psi_cells[PS_VZ] = nx2 * ny2 * 2 * np;
    // block storage keeps the CPML memory variables in FP32
    const size_t pelem = precision == SM_BFP16 ? 4 : h->elem;
    for (int b = 0; b < 2; ++b)
        for (int p = 0; p < 6; ++p)
            if ((rc = h->psi[b][p].alloc_pooled(h->psi_cells[p] * pelem, device))) return rc;
    if (precision == SM_BFP16) {
        h->nyb = (ny2 + A3_BJ - 1) / A3_BJ;
        for (int b = 0; b < 2; ++b)
            for (int f = 0; f < 4; ++f)
                if ((rc = h->fe[b][f].alloc_pooled(nx2 * h->nyb * (size_t)h->pitch, device))) return rc;
    }
    if ((rc = h->rho.alloc_pooled(ncell * cb, device))) return rc;
    if ((rc = h->K.alloc_pooled(ncell * cb, device))) return rc;
    rc = precision == SM_FP64 ? a3d_upload_materials<double>(h.get(), m, dt, nx2, ny2, nz2)
                              : a3d_upload_materials<float>(h.get(), m, dt, nx2, ny2, nz2);
    if (rc) return rc;
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
    a.sx = (int)(ny2 * h->pitch);
    a.nyb = (int)h->nyb;
    if (precision == SM_FP16 || precision == SM_BF16) {
        if ((rc = h->scaler.init(10, 10))) return rc;
        // the padded nodes repeat interior values: the source's minima
        const size_t N = m.nx * m.ny * m.nz;
        h->rho_min = m.rho[0];
        h->vp_min = m.vp[0];
        for (size_t q = 1; q < N; ++q) {
            if (m.rho[q] < h->rho_min) h->rho_min = m.rho[q];
            if (m.vp[q] < h->vp_min) h->vp_min = m.vp[q];
        }
        h->hmin = std::min(dx, std::min(dy, dz));
        h->expo0.assign(10, 0);
    }
    if ((rc = h->err.alloc(sizeof(int)))) return rc;
    if ((rc = h->err.zero(h->stream))) return rc;
    a.err = h->err.as<int>();
    if ((rc = h->d_step.alloc(sizeof(long long)))) return rc;
    a.step = h->d_step.as<long long>();
    for (int f = 0; f < 4; ++f) { a.sc[f] = 1.f; a.isc[f] = 1.f; }
    for (int p = 0; p < 6; ++p) { a.psc[p] = 1.f; a.pisc[p] = 1.f; }
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device);
    a.chunk = a3d_default_chunk(h.get(), h->config);
    static std::atomic<uint64_t> serials{1};
    h->serial = serials.fetch_add(1);
    a3d_bind(h.get(), 0);
    a.rho = h->rho.p;
    a.K = h->K.p;
    a.coef = h->coef.p;
    a.cf = cf;
    a.two_dt = dt * 2.;
    a.idx = 1.0 / dx; a.idy = 1.0 / dy; a.idz = 1.0 / dz;
    if (precision == SM_FP16 || precision == SM_BF16) a3d_apply_scales(h.get());
    if ((rc = sm_a3d_reset(h.get()))) return rc;
    *out = h.release();
    return SM_OK;
}

}  // namespace

extern "C" int sm_a3d_create(int device, size_t nx2, size_t ny2, size_t nz2, size_t np,
                             double dx, double dy, double dz, double dt, const double *vp,
                             const double *rho, const double *const *coef, int precision,
                             sm_a3d_t *out) {
    return a3d_create(device, nx2, ny2, nz2, np, dx, dy, dz, dt,
                      A3Model{vp, rho, nx2, ny2, nz2, 0}, coef, precision, out);
}

extern "C" int sm_a3d_create_unpadded(int device, size_t nx, size_t ny, size_t nz, size_t np,
                                      double dx, double dy, double dz, double dt,
                                      const double *vp, const double *rho,
                                      const double *const *coef, int precision, sm_a3d_t *out) {
    if (!out) return sm_fail(SM_EINVAL, "sm_a3d_create_unpadded: out is NULL");
    *out = nullptr;
    if (!nx || !ny || !nz) return sm_fail(SM_EINVAL, "sm_a3d_create_unpadded: empty model");
    return a3d_create(device, nx + 2 * np, ny + 2 * np, nz + 2 * np, np, dx, dy, dz, dt,
                      A3Model{vp, rho, nx, ny, nz, np}, coef, precision, out);
}

extern "C" int sm_a3d_reset(sm_a3d_t h) {
    if (int rc = a3d_check(h)) return rc;
    DeviceGuard g(h->device);
    for (int b = 0; b < 2; ++b) {
        for (int f = 0; f < 4; ++f) {
            if (int rc = h->f[b][f].zero(h->stream)) return rc;
            if (int rc = h->fe[b][f].zero(h->stream)) return rc;
        }
        for (int p = 0; p < 6; ++p)
            if (int rc = h->psi[b][p].zero(h->stream)) return rc;
    }
    h->cur = 0;
    if (a3d_is16(h)) {
        if (h->scaler.expo != h->expo0) h->graph_epoch++;
        h->scaler.expo = h->expo0;
        a3d_apply_scales(h);
    }
    if (int rc = h->d_traces.zero(h->stream)) return rc;
    if (int rc = h->d_step.zero(h->stream)) return rc;
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
        const size_t jb = j / A3_BJ;
        e.qe = (long long)((i * h->nyb + jb) * h->pitch + k);
        e.qb = (long long)((i * h->ny2 + jb * A3_BJ) * h->pitch + k);
        e.nb = (int)std::min<size_t>(A3_BJ, h->ny2 - jb * A3_BJ);
        e.rs = (int)(j - jb * A3_BJ);
        for (size_t t = 0; t < length[s]; ++t) h->vals.push_back(scale * fct[s * stride + t]);
        h->src.push_back(e);
    }
    h->src_dirty = 1;
    if (a3d_is16(h)) {
        // starting ranges from the source: the pressure a cell accumulates
        // (running sum of the injected values), the particle velocity that
        // pressure drives (p / (rho vp)), and their gradients for the memory
        // variables; the range checks refine them as the run proceeds
        double pmax = 0.0;
        for (const A3Src &e : h->src) {
            double acc = 0.0;
            for (int t = 0; t < e.len; ++t) {
                acc += h->vals[e.voff + t];
                pmax = std::max(pmax, std::fabs(acc));
            }
        }
        const double vmax = pmax / (h->rho_min * h->vp_min);
        const int ep = Scaler16::expo_for(pmax), ev = Scaler16::expo_for(vmax);
        const int egp = Scaler16::expo_for(pmax / h->hmin), egv = Scaler16::expo_for(vmax / h->hmin);
        std::vector<int> ex = {ev, ev, ev, ep, egp, egp, egp, egv, egv, egv};
        h->expo0 = ex;
        for (int g = 0; g < 10; ++g) h->scaler.ceil[g] = ex[g] + 2;
        if (h->it == 0) {
            h->scaler.expo = ex;
            a3d_apply_scales(h);
        }
    }
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
        e.qe = (long long)((i * h->nyb + j / A3_BJ) * h->pitch + k);
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
    h->graph_epoch++;
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
            // the trace buffer comes from the device cache: no step of this
            // handle may still write the old one when it goes back
            SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
            if ((rc = h->d_traces.alloc_pooled(nt * sizeof(double), h->device))) return rc;
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

namespace {

// the graph of h->graph_steps steps starting from buffer set h->cur
template <typename S>
int a3d_graph(sm_a3d *h, cudaGraphExec_t *out) {
    sm_a3d::Graph &gr = h->graphs[h->cur];
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
    for (int k = 0; k < h->graph_steps; ++k) a3d_launch<S>(h);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    h->timer.capture = nullptr;
    h->timer.launches = launches;
    h->cur = cur;   // an even number of steps: back to the starting set
    a3d_bind(h, h->cur);
    if (e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return sm_fail(SM_ECUDA, "stream capture: %s", cudaGetErrorString(e));
    }
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
int a3d_run_t(sm_a3d *h, size_t nsteps) {
    if constexpr (std::is_same<S, Bfp16>::value) {
        if (int rc = a3d_bready(h)) return rc;
    } else {
        if (int rc = a3d_ready<S>(h)) return rc;
    }
    const size_t G = (size_t)h->graph_steps;
    const size_t per_step =
        (size_t)a3d_step_kernels(h) + (h->src.empty() ? 0 : 1) + (h->rec.empty() ? 0 : 1);
    while (nsteps > 0) {
        // graphs start anywhere, except in 16-bit storage, whose range
        // checks fall on multiples of the scale period between graphs
        if (G && nsteps >= G && (!a3d_is16(h) || h->it % G == 0)) {
            cudaGraphExec_t ex = nullptr;
            if (int rc = a3d_graph<S>(h, &ex)) return rc;
            SM_CUDA_TRY(cudaGraphLaunch(ex, h->stream));
            if (h->timer.on) h->timer.replayed(h->graphs[h->cur].tev);
            h->timer.launches += per_step * G;
            h->it += G;
            nsteps -= G;
        } else {
            a3d_launch<S>(h);
            h->it++;
            nsteps--;
        }
        if (a3d_is16(h) && h->it % sm_a3d::kScalePeriod == 0)
            if (int rc = a3d_rescale(h)) return rc;
    }
    return SM_OK;
}

}  // namespace

extern "C" int sm_a3d_run(sm_a3d_t h, size_t nsteps) {
    if (int rc = a3d_check(h)) return rc;
    DeviceGuard g(h->device);
    if (int rc = a3d_ensure_maps(h)) return rc;
    if (h->src_dirty || h->rec_dirty)
        if (int rc = a3d_upload(h)) return rc;
    int rc;
    switch (h->precision) {
    case SM_FP64: rc = a3d_run_t<double>(h, nsteps); break;
    case SM_FP16: rc = a3d_run_t<__half>(h, nsteps); break;
    case SM_BF16: rc = a3d_run_t<__nv_bfloat16>(h, nsteps); break;
    case SM_BFP16: rc = a3d_run_t<Bfp16>(h, nsteps); break;
    default: rc = a3d_run_t<float>(h, nsteps); break;
    }
    if (rc) return rc;
    SM_CUDA_TRY(cudaGetLastError());
    return SM_OK;
}

namespace {

// The grouped step's launch configuration: the default one of the storage
// type (8 warps; FP32-like storage 2 rows per warp, block storage one block
// of A3_BJ rows per thread).  Results do not depend on it.
constexpr int kA3GW = 8, kA3GR = 2, kA3GD = 4;
// resident CTAs the grouped kernel's registers are fitted to (both tile
// bodies in one kernel: FP64 needs the larger budget to stay out of local memory)
template <typename S>
constexpr int a3d_group_minb() { return sizeof(S) == 8 ? 2 : 3; }
constexpr int kA3GBD = 4, kA3GBMinB = 2;

template <typename S>
constexpr int a3d_group_ty() {
    return std::is_same<S, Bfp16>::value ? kA3GW * A3_BJ : kA3GW * kA3GR;
}

template <typename S>
size_t a3d_group_smem() {
    if constexpr (std::is_same<S, Bfp16>::value)
        return a3d_bstep_smem<kA3GW * A3_BJ, kA3GBD>();
    else
        return a3d_step_smem<S, kA3GW * kA3GR, kA3GD>();
}

template <typename S>
int a3d_group_ready(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    if (device < 0 || device >= 64) return sm_fail(SM_EINVAL, "device %d", device);
    std::lock_guard<std::mutex> lk(mu);
    if (!done[device]) {
        if constexpr (std::is_same<S, Bfp16>::value)
            SM_CUDA_TRY(cudaFuncSetAttribute(a3d_bgroup_step_kernel<kA3GW, kA3GBD, kA3GBMinB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)a3d_group_smem<S>()));
        else
            SM_CUDA_TRY(cudaFuncSetAttribute(a3d_group_step_kernel<S, kA3GW, kA3GR, kA3GD, a3d_group_minb<S>()>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)a3d_group_smem<S>()));
        done[device] = true;
    }
    return SM_OK;
}

// one grouped step of the problems hs[0..n) (n <= kA3GroupMax), on stream st
template <typename S>
int a3d_group_step(sm_a3d *const *hs, int n, cudaStream_t st) {
    constexpr bool B = std::is_same<S, Bfp16>::value;
    using M = std::conditional_t<B, A3BMaps, A3Maps>;
    constexpr int TY = a3d_group_ty<S>();
    static A3GroupStepParams<M> P;   // large: built in place, one caller at a time
    static A3GroupPostParams Q;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    int total = 0;
    for (int k = 0; k < n; ++k) {
        sm_a3d *h = hs[k];
        a3d_bind(h, h->cur);
        a3d_tile_classes(h, TY);
        const A3Args &a = h->args;
        const int nch = (a.nx2 + a.chunk - 1) / a.chunk;
        const int ninner = (a.kt1 - a.kt0) * (a.jt1 - a.jt0);
        if constexpr (B) P.m[k] = h->bmaps[h->cur];
        else P.m[k] = h->maps[h->cur];
        P.a[k] = a;
        P.nedge[k] = a.nkt * a.njt - ninner;
        P.first[k] = total;
        total += a.nkt * a.njt * nch;
    }
    P.first[n] = total;
    P.n = n;
    const dim3 blk(32, kA3GW, 1);
    if constexpr (B)
        a3d_bgroup_step_kernel<kA3GW, kA3GBD, kA3GBMinB><<<total, blk, a3d_group_smem<S>(), st>>>(P);
    else
        a3d_group_step_kernel<S, kA3GW, kA3GR, kA3GD, a3d_group_minb<S>()><<<total, blk, a3d_group_smem<S>(), st>>>(P);
    int nrec = 0;
    bool src = false;
    for (int k = 0; k < n; ++k) {
        sm_a3d *h = hs[k];
        h->cur = 1 - h->cur;
        a3d_bind(h, h->cur);
        A3Post &q = Q.q[k];
        q.a = h->args;
        q.src = h->d_src.as<A3Src>();
        q.nsrc = (int)h->src.size();
        q.vals = h->d_vals.as<double>();
        q.rec = h->d_rec.as<A3Rec>();
        q.table = h->d_table.as<int32_t>();
        q.nsteps_max = (long long)h->plan.nsteps_max;
        q.traces = h->d_traces.as<double>();
        Q.first_rec[k] = nrec;
        nrec += (int)h->rec.size();
        src = src || !h->src.empty();
    }
    Q.first_rec[n] = nrec;
    Q.n = n;
    if (src) a3d_group_source_kernel<S><<<n, 32, 0, st>>>(Q);
    if (nrec) a3d_group_gather_kernel<S><<<(nrec + 127) / 128, 128, 0, st>>>(Q);
    hs[0]->timer.launches += 1 + (src ? 1 : 0) + (nrec ? 1 : 0);
    SM_CUDA_TRY(cudaGetLastError());
    return SM_OK;
}

template <typename S>
int a3d_group_steps(sm_a3d *const *hs, int n, int steps) {
    for (int s = 0; s < steps; ++s)
        for (int k0 = 0; k0 < n; k0 += kA3GroupMax)
            if (int rc = a3d_group_step<S>(hs + k0, std::min(kA3GroupMax, n - k0), hs[0]->stream))
                return rc;
    return SM_OK;
}

// CUDA graphs of kA3GroupGraphSteps grouped steps, cached per group: the key
// holds each handle's serial, starting buffer set and graph epoch (sources,
// receivers, scales, configuration), so a graph is only replayed on the
// state it was captured for.  A few are kept, the least recently used
// dropped.
constexpr int kA3GroupGraphSteps = 16;
constexpr size_t kA3GroupGraphCache = 8;

struct A3GroupKey {
    int device;
    std::vector<std::tuple<uint64_t, int, unsigned, int>> members;
    bool operator<(const A3GroupKey &o) const {
        return std::tie(device, members) < std::tie(o.device, o.members);
    }
};
struct A3GroupGraph {
    cudaGraphExec_t exec = nullptr;
    uint64_t used = 0;
};
std::mutex g_a3_group_mu;
std::map<A3GroupKey, A3GroupGraph> g_a3_group_graphs;
uint64_t g_a3_group_clock = 0;

template <typename S>
int a3d_group_graph(sm_a3d *const *hs, int n, cudaGraphExec_t *out) {
    A3GroupKey key{hs[0]->device, {}};
    for (int k = 0; k < n; ++k)
        key.members.emplace_back(hs[k]->serial, hs[k]->cur, hs[k]->graph_epoch, hs[k]->args.chunk);
    std::lock_guard<std::mutex> lk(g_a3_group_mu);
    auto it = g_a3_group_graphs.find(key);
    if (it != g_a3_group_graphs.end()) {
        it->second.used = ++g_a3_group_clock;
        *out = it->second.exec;
        return SM_OK;
    }
    const size_t launches = hs[0]->timer.launches;
    SM_CUDA_TRY(cudaStreamBeginCapture(hs[0]->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = a3d_group_steps<S>(hs, n, kA3GroupGraphSteps);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(hs[0]->stream, &graph);
    hs[0]->timer.launches = launches;
    for (int k = 0; k < n; ++k) a3d_bind(hs[k], hs[k]->cur);   // an even number of steps
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return sm_fail(SM_ECUDA, "stream capture: %s", cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return sm_fail(SM_ECUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    if (g_a3_group_graphs.size() >= kA3GroupGraphCache) {
        auto old = g_a3_group_graphs.begin();
        for (auto i = g_a3_group_graphs.begin(); i != g_a3_group_graphs.end(); ++i)
            if (i->second.used < old->second.used) old = i;
        // some stream may still run it: wait before the executable goes
        cudaDeviceSynchronize();
        cudaGraphExecDestroy(old->second.exec);
        g_a3_group_graphs.erase(old);
    }
    g_a3_group_graphs[key] = A3GroupGraph{exec, ++g_a3_group_clock};
    *out = exec;
    return SM_OK;
}

template <typename S>
int a3d_group_run_t(sm_a3d *const *hs, int n, size_t nsteps) {
    constexpr int TY = a3d_group_ty<S>();
    for (int k = 0; k < n; ++k) {
        sm_a3d *h = hs[k];
        if (h->maps_ty == TY) continue;
        int rc;
        if constexpr (std::is_same<S, Bfp16>::value) rc = a3d_make_bmaps(h, TY);
        else rc = a3d_make_maps<S>(h, TY);
        if (rc) return rc;
    }
    if (int rc = a3d_group_ready<S>(hs[0]->device)) return rc;
    const bool is16 = a3d_is16(hs[0]);
    const size_t G = kA3GroupGraphSteps;
    int per_step = 0;
    for (int k0 = 0; k0 < n; k0 += kA3GroupMax) {
        bool src = false, rec = false;
        for (int k = k0; k < std::min(n, k0 + kA3GroupMax); ++k) {
            src = src || !hs[k]->src.empty();
            rec = rec || !hs[k]->rec.empty();
        }
        per_step += 1 + (src ? 1 : 0) + (rec ? 1 : 0);
    }
    while (nsteps > 0) {
        // a graph of G steps when no handle rescales inside it
        bool aligned = true;
        for (int k = 0; k < n && is16; ++k) aligned = aligned && hs[k]->it % G == 0;
        size_t done;
        if (nsteps >= G && aligned) {
            cudaGraphExec_t ex = nullptr;
            if (int rc = a3d_group_graph<S>(hs, n, &ex)) return rc;
            SM_CUDA_TRY(cudaGraphLaunch(ex, hs[0]->stream));
            hs[0]->timer.launches += per_step * G;
            done = G;
        } else {
            if (int rc = a3d_group_steps<S>(hs, n, 1)) return rc;
            done = 1;
        }
        nsteps -= done;
        for (int k = 0; k < n; ++k) {
            sm_a3d *h = hs[k];
            const size_t before = h->it;
            h->it += done;
            if (is16 && h->it / sm_a3d::kScalePeriod != before / sm_a3d::kScalePeriod)
                if (int rc = a3d_rescale(h)) return rc;
        }
    }
    return SM_OK;
}

}  // namespace

// Several a_iso_3d handles of different grid sizes advanced together: every
// step is one launch over all their tiles (up to 16 handles per launch), one
// for all their sources and one for all their receivers.  Each handle ends
// where sm_a3d_run(h, nsteps) would have left it, bit for bit.  The work
// runs on the first handle's stream, ordered after the work already queued
// on every handle's stream; every handle's stream waits for it to finish.
extern "C" int sm_a3d_group_run(sm_a3d_t const *handles, int n, size_t nsteps) {
    if (!handles || n <= 0) return sm_fail(SM_EINVAL, "sm_a3d_group_run: no handles");
    for (int k = 0; k < n; ++k) {
        if (int rc = a3d_check(handles[k])) return rc;
        if (handles[k]->device != handles[0]->device ||
            handles[k]->precision != handles[0]->precision)
            return sm_fail(SM_EINVAL,
                           "sm_a3d_group_run: handle %d differs in device or precision from "
                           "handle 0", k);
        for (int j = 0; j < k; ++j)
            if (handles[j] == handles[k])
                return sm_fail(SM_EINVAL, "sm_a3d_group_run: handle %d appears twice", k);
    }
    if (nsteps == 0) return SM_OK;
    sm_a3d *const *hs = handles;
    DeviceGuard g(hs[0]->device);
    for (int k = 0; k < n; ++k) {
        sm_a3d *h = hs[k];
        if (!h->src_dirty && !h->rec_dirty) continue;
        if (int rc = a3d_upload(h)) return rc;
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
    case SM_FP64: rc = a3d_group_run_t<double>(hs, n, nsteps); break;
    case SM_FP16: rc = a3d_group_run_t<__half>(hs, n, nsteps); break;
    case SM_BF16: rc = a3d_group_run_t<__nv_bfloat16>(hs, n, nsteps); break;
    case SM_BFP16: rc = a3d_group_run_t<Bfp16>(hs, n, nsteps); break;
    default: rc = a3d_group_run_t<float>(hs, n, nsteps); break;
    }
    for (int k = 0; k < n; ++k) hs[k]->stream = own[k];
    cudaEventRecord(ev, st);
    for (int k = 1; k < n; ++k) cudaStreamWaitEvent(hs[k]->stream, ev, 0);
    cudaEventDestroy(ev);
    if (rc) return rc;
    SM_CUDA_TRY(cudaGetLastError());
    return SM_OK;
}

extern "C" int sm_a3d_set_graph(sm_a3d_t h, int steps) {
    if (int rc = a3d_check(h)) return rc;
    if (steps != 0 && steps != 2 && steps != 4 && steps != 8 && steps != 16)
        return sm_fail(SM_EINVAL, "sm_a3d_set_graph: steps must be 0, 2, 4, 8 or 16 (got %d)",
                       steps);
    h->graph_steps = steps;
    h->graph_epoch++;
    return SM_OK;
}

// Launch-configuration search, as sm_eiso_autotune: every configuration that
// fits, with a few x-chunk lengths, timed over trial_steps steps from a zero
// state; the fastest is kept and cached per (precision, grid, device).
extern "C" int sm_a3d_autotune(sm_a3d_t h, int trial_steps, int *config, int *chunk,
                               double *ms_per_step) {
    if (int rc = a3d_check(h)) return rc;
    if (h->it != 0)
        return sm_fail(SM_ESTATE, "sm_a3d_autotune: call before the first step (or after reset)");
    if (trial_steps <= 0) trial_steps = 32;
    DeviceGuard g(h->device);
    struct Key {
        int prec;
        size_t nx2, ny2, nz2, np;
        int dev;
        bool operator<(const Key &o) const {
            return std::tie(prec, nx2, ny2, nz2, np, dev) <
                   std::tie(o.prec, o.nx2, o.ny2, o.nz2, o.np, o.dev);
        }
    };
    struct Val {
        int config, chunk;
        double ms;
    };
    static std::map<Key, Val> cache;
    static std::mutex mu;
    const Key key{h->precision, h->nx2, h->ny2, h->nz2, h->np, h->device};
    Val best{-1, 0, 0.0};
    bool cached = false;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            best = it->second;
            cached = true;
        }
    }
    int rc = SM_OK;
    if (!cached) {
        int lim = 0;
        SM_CUDA_TRY(cudaDeviceGetAttribute(&lim, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
        cudaEvent_t e0, e1;
        SM_CUDA_TRY(cudaEventCreate(&e0));
        SM_CUDA_TRY(cudaEventCreate(&e1));
        const bool timing = h->timer.on;
        h->timer.on = false;
        for (int c = 0; c < a3d_ncfg(h) && rc == SM_OK; ++c) {
            if (a3d_config_smem_prec(h->precision, c) > (size_t)lim) continue;
            if ((rc = sm_a3d_set_config(h, c))) break;
            // the default chunk length, then other lengths it is not
            std::vector<int> chunks{0};
            for (int ch : {16, 20, 28, 32, 48, 64})
                if (ch != a3d_default_chunk(h, c) && (size_t)ch <= h->nx2) chunks.push_back(ch);
            for (int ch : chunks) {
                if ((rc = sm_a3d_set_config(h, c)) || (rc = sm_a3d_set_chunk(h, ch))) break;
                // warm-up, and the time loop's graph (if the handle uses
                // graphs) captured outside the timed trial
                if ((rc = sm_a3d_reset(h)) || (rc = sm_a3d_run(h, 2 + (size_t)h->graph_steps))) break;
                cudaEventRecord(e0, h->stream);
                if ((rc = sm_a3d_run(h, (size_t)trial_steps))) break;
                cudaEventRecord(e1, h->stream);
                if ((rc = sm_a3d_sync(h))) break;
                float t = 0.f;
                cudaEventElapsedTime(&t, e0, e1);
                const double ms = t / trial_steps;
                if (best.config < 0 || ms < best.ms) best = Val{c, ch, ms};
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        h->timer.on = timing;
        if (rc) return rc;
        if (best.config < 0) return sm_fail(SM_EINVAL, "sm_a3d_autotune: no configuration fits");
        std::lock_guard<std::mutex> lk(mu);
        cache[key] = best;
    }
    if ((rc = sm_a3d_set_config(h, best.config)) || (rc = sm_a3d_set_chunk(h, best.chunk)) ||
        (rc = sm_a3d_reset(h)))
        return rc;
    if (config) *config = best.config;
    if (chunk) *chunk = best.chunk;
    if (ms_per_step) *ms_per_step = best.ms;
    return SM_OK;
}

extern "C" int sm_a3d_sync(sm_a3d_t h) {
    if (int rc = a3d_check(h)) return rc;
    DeviceGuard g(h->device);
    SM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return a3d_check_err(h);
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
    if (int rc = a3d_check_err(h)) return rc;
    const size_t lim = std::min(h->it, h->plan.nsteps_max);
    std::vector<size_t> gcount(h->plan.count_total.size(), 0);
    for (size_t gi = 0; gi < gcount.size(); ++gi)
        for (size_t it = 0; it < lim; ++it)
            if (h->plan.table[gi * h->plan.nsteps_max + it] >= 0) ++gcount[gi];
    const size_t ms = h->plan.max_samples;
    if (out && nrec && ms) {
        size_t cmax = 0;
        bool same = true;
        for (size_t r = 0; r < nrec; ++r) {
            const size_t c = gcount[h->rec[rec0 + r].group];
            if (ld < c) return sm_fail(SM_EINVAL, "sm_a3d_read_traces: ld too small");
            same = same && (r == 0 || c == cmax);
            cmax = std::max(cmax, c);
        }
        const double *src = h->d_traces.as<double>() + rec0 * ms;
        if (same) {
            // every record has cmax samples: one strided copy into the caller's rows
            if (cmax)
                SM_CUDA_TRY(cudaMemcpy2D(out, ld * sizeof(double), src, ms * sizeof(double),
                                         cmax * sizeof(double), nrec, cudaMemcpyDeviceToHost));
        } else {
            // one bulk copy, then scatter into the caller's layout
            std::unique_ptr<double[]> buf(new (std::nothrow) double[nrec * ms]);
            if (!buf) return sm_fail(SM_ENOMEM, "sm_a3d_read_traces: out of host memory");
            SM_CUDA_TRY(cudaMemcpy(buf.get(), src, nrec * ms * sizeof(double),
                                   cudaMemcpyDeviceToHost));
            for (size_t r = 0; r < nrec; ++r)
                std::memcpy(out + r * ld, buf.get() + r * ms,
                            gcount[h->rec[rec0 + r].group] * sizeof(double));
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
    SM_CUDA_TRY(cudaMemcpy(buf.data(), h->f[h->cur][f].p, buf.size(), cudaMemcpyDeviceToHost));
    if (a3d_isb(h)) {   // mantissa times 2^(e8 - 126) of the cell's block
        std::vector<uint8_t> ex(h->fe[h->cur][f].bytes);
        SM_CUDA_TRY(cudaMemcpy(ex.data(), h->fe[h->cur][f].p, ex.size(), cudaMemcpyDeviceToHost));
        const int16_t *mm = reinterpret_cast<const int16_t *>(buf.data());
        for (size_t i = 0; i < h->nx2; ++i)
            for (size_t j = 0; j < h->ny2; ++j)
                for (size_t k = 0; k < h->nz2; ++k)
                    out[(i * h->ny2 + j) * h->nz2 + k] = bfp_value_host(
                        mm[(i * h->ny2 + j) * h->pitch + k],
                        ex[(i * h->nyb + j / A3_BJ) * h->pitch + k]);
        return SM_OK;
    }
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
    if (a3d_isb(h)) {   // each block of A3_BJ rows encoded as the kernels encode it
        std::vector<uint8_t> ex(h->fe[h->cur][f].bytes, 0);
        int16_t *mm = reinterpret_cast<int16_t *>(buf.data());
        for (size_t i = 0; i < h->nx2; ++i)
            for (size_t jb = 0; jb < h->nyb; ++jb)
                for (size_t k = 0; k < h->nz2; ++k) {
                    const size_t ja = jb * A3_BJ, je = std::min(ja + A3_BJ, h->ny2);
                    float mx = 0.f;
                    for (size_t j = ja; j < je; ++j)
                        mx = std::max(mx, std::fabs((float)in[(i * h->ny2 + j) * h->nz2 + k]));
                    const unsigned e8 = bfp_e8_host(mx);
                    ex[(i * h->nyb + jb) * h->pitch + k] = (uint8_t)e8;
                    for (size_t j = ja; j < je; ++j)
                        mm[(i * h->ny2 + j) * h->pitch + k] =
                            bfp_man_host((float)in[(i * h->ny2 + j) * h->nz2 + k], e8);
                }
        SM_CUDA_TRY(cudaMemcpy(h->fe[h->cur][f].p, ex.data(), ex.size(), cudaMemcpyHostToDevice));
        SM_CUDA_TRY(cudaMemcpy(h->f[h->cur][f].p, buf.data(), buf.size(), cudaMemcpyHostToDevice));
        return SM_OK;
    }
    for (size_t i = 0; i < h->nx2; ++i)
        for (size_t j = 0; j < h->ny2; ++j)
            for (size_t k = 0; k < h->nz2; ++k)
                a3_from_double(buf.data(), (i * h->ny2 + j) * h->pitch + k, h->precision,
                               in[(i * h->ny2 + j) * h->nz2 + k], h->args.sc[f]);
    SM_CUDA_TRY(cudaMemcpy(h->f[h->cur][f].p, buf.data(), buf.size(), cudaMemcpyHostToDevice));
    return SM_OK;
}

extern "C" int sm_a3d_destroy(sm_a3d_t h) {
    if (!h) return SM_OK;
    DeviceGuard g(h->device);
    if (h->stream) {
        cudaStreamSynchronize(h->stream);
        cudaStreamDestroy(h->stream);
    }
    if (h->side) {
        cudaStreamSynchronize(h->side);
        cudaStreamDestroy(h->side);
    }
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
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

extern "C" int sm_a3d_stream(sm_a3d_t h, void **stream) {
    if (int rc = a3d_check(h)) return rc;
    if (!stream) return sm_fail(SM_EINVAL, "sm_a3d_stream: NULL");
    *stream = (void *)h->stream;
    return SM_OK;
}

extern "C" int sm_a3d_set_timing(sm_a3d_t h, int on) {
    if (int rc = a3d_check(h)) return rc;
    DeviceGuard g(h->device);
    h->timer.set(on != 0);
    return SM_OK;
}

extern "C" int sm_a3d_kernel_stats(sm_a3d_t h, int reset, double *update_ms,
                                   size_t *update_launches, size_t *all_launches) {
    if (int rc = a3d_check(h)) return rc;
    DeviceGuard g(h->device);
    return h->timer.stats(reset, update_ms, update_launches, all_launches);
}

extern "C" int sm_a3d_set_config(sm_a3d_t h, int config) {
    if (int rc = a3d_check(h)) return rc;
    if (config < 0 || config >= a3d_ncfg(h))
        return sm_fail(SM_EINVAL, "sm_a3d_set_config: config %d not in [0, %d)", config,
                       a3d_ncfg(h));
    int maxsm = 0;
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
    if (a3d_config_smem_prec(h->precision, config) > (size_t)maxsm)
        return sm_fail(SM_EINVAL, "sm_a3d_set_config: config %d needs %zu bytes of shared memory "
                                  "in this precision (device limit %d)", config,
                       a3d_config_smem_prec(h->precision, config), maxsm);
    h->config = config;
    h->args.chunk = a3d_default_chunk(h, config);
    h->graph_epoch++;
    // maps are rebuilt for the new tile height at the next run
    return SM_OK;
}

extern "C" int sm_a3d_set_chunk(sm_a3d_t h, int chunk) {
    if (int rc = a3d_check(h)) return rc;
    if (chunk <= 0)
        h->args.chunk = a3d_default_chunk(h, h->config);
    else
        h->args.chunk = chunk > A3_CHMAX ? A3_CHMAX : (chunk > (int)h->nx2 ? (int)h->nx2 : chunk);
    h->graph_epoch++;
    return SM_OK;
}

extern "C" int sm_a3d_get_config(sm_a3d_t h, int *config, int *nconfigs) {
    if (int rc = a3d_check(h)) return rc;
    if (config) *config = h->config;
    if (nconfigs) *nconfigs = a3d_ncfg(h);
    return SM_OK;
}
