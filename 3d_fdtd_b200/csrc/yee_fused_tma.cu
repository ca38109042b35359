// yee_fused_tma.cu -- the FP32 single-pass Yee step with TMA staging.
//
// Same data flow and arithmetic as yee_fused.cu (see there): one launch per
// time step, ping-pong field sets, a block owns a 32 x TY tile of (x, y) columns
// and a z-chunk and streams along z computing E_new(k) (tile plus the +x column
// and +y row, the latter two only recomputed) and then H_new(k-1).
//
// Staging: per plane one thread issues, by TMA, three H boxes (tile plus a
// 1-cell halo on every side, hardware zero fill outside the grid), three E
// boxes and three (six if lossy) coefficient boxes onto one mbarrier.  A ring
// of three plane stages gives a prefetch distance of two planes.
//
// Work split: warp w owns rows [R w, R w + R) of the tile (R = TY / 8), lane =
// x.  A thread keeps its own cells' H_in(k-1) and E_new(k-1) in registers
// between planes, so shared memory is read only for neighbours in other rows or
// lanes; the +x column and +y row halo cells are spread over all warps.  One
// barrier per plane separates the E pass from the H pass: E_new planes live in a
// three-deep ring and the TMA for plane k+2 is issued after that barrier, so no
// second barrier is needed.
//
// TMA rules observed: every box starts at an x coordinate that is a multiple
// of 4 floats (16 bytes): the H box starts at X0-4 and is 40 floats wide;
// strides are multiples of 16 bytes, which needs nx % 4 == 0 (other widths use
// the cp.async kernel); shared-memory destinations are 128-byte aligned and the
// kernel checks that before issuing any copy.  Loads only, no multicast.
//
// Waits on the mbarriers are bounded in time (kWaitNs of %globaltimer).  A
// wait that gives up sets the grid's device error flag and a block-wide abort
// flag; the block then finishes its loop without waiting (results are
// garbage, the host reports FDTD_ERR_TIMEOUT) instead of hanging.
// k_wait_selftest runs the same bounded wait on a barrier nothing arrives on.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "kernels.h"

namespace fdtd {

constexpr int TX = 32;
constexpr int HW = TX + 8;   // H box width: x from X0-4 to X0+TX+3
constexpr int EW = TX + 4;   // E / coefficient box width: x from X0 to X0+TX+3
constexpr int HOFF = 4;      // box x index of tile column 0 in an H box
constexpr unsigned long long kWaitNs = 1000000000ull;   // 1 s: a plane's loads take microseconds

constexpr int pad128f(int nfloats) { return ((nfloats * 4 + 127) / 128) * 32; }

template <int TY, bool LOSSY>
struct alignas(128) TmaStage {
    static constexpr int NC = LOSSY ? 6 : 3;
    static constexpr int HBOX = (TY + 2) * HW, EBOX = (TY + 1) * EW;
    static constexpr int HBOXP = pad128f(HBOX), EBOXP = pad128f(EBOX);
    float h[3][HBOXP];     // H box c: [TY+2][HW], x fastest
    float e[3][EBOXP];     // E box c: [TY+1][EW]
    float c[NC][EBOXP];    // cb (and ca) boxes
    static constexpr unsigned kBytes = 3u * HBOX * 4 + (3u + NC) * EBOX * 4;
};

template <int TY, bool LOSSY>
struct TmaSmem {
    TmaStage<TY, LOSSY> st[3];
    float en[3][3][TY + 1][TX + 1];   // E_new ring (planes k-2 .. k), tile + the +1 column/row
    unsigned long long bar[3];
    int abort;
};
template <int TY, bool LOSSY> constexpr size_t tma_smem_bytes() { return sizeof(TmaSmem<TY, LOSSY>) + 128; }

__device__ __forceinline__ float Hat(const float *box, int lx, int ly) { return box[(ly + 1) * HW + lx + HOFF]; }
__device__ __forceinline__ float Eat(const float *box, int lx, int ly) { return box[ly * EW + lx]; }

// ---- PTX wrappers ----------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// true when the barrier's phase `parity` completed; false when *abort was set
// by another thread or limit_ns passed
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity,
                                                  unsigned long long limit_ns, volatile int *abort)
{
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (*abort) return false;   // checked first: after a refused start the barriers were never set up
        if (mbar_try_wait(bar, parity)) return true;
        // try_wait may suspend for a hardware-defined while: check the clock every time
        if (global_ns() - t0 > limit_ns) return false;
    }
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

template <int TY, bool LOSSY>
__device__ __forceinline__ void issue_plane(TmaSmem<TY, LOSSY> &sm, const FusedMaps &m, int k, int X0, int Y0)
{
    const int slot = (k + 3) % 3;
    TmaStage<TY, LOSSY> &s = sm.st[slot];
    unsigned long long *bar = &sm.bar[slot];
    fence_async_shared();
    mbar_expect_tx(bar, TmaStage<TY, LOSSY>::kBytes);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        tma_load_3d(&s.h[c][0], &m.h[c], X0 - HOFF, Y0 - 1, k, bar);
        tma_load_3d(&s.e[c][0], &m.e[c], X0, Y0, k, bar);
        tma_load_3d(&s.c[c][0], &m.cb[c], X0, Y0, k, bar);
        if (LOSSY) tma_load_3d(&s.c[3 + c][0], &m.ca[c], X0, Y0, k, bar);
    }
}

// true when every TMA destination is 128-byte aligned and every mbarrier 8-byte aligned
template <int TY, bool LOSSY>
__device__ __forceinline__ bool tma_layout_ok(const TmaSmem<TY, LOSSY> &sm)
{
    for (int s = 0; s < 3; s++) {
        for (int c = 0; c < 3; c++)
            if ((smem_u32(&sm.st[s].h[c][0]) & 127u) || (smem_u32(&sm.st[s].e[c][0]) & 127u)) return false;
        for (int c = 0; c < TmaStage<TY, LOSSY>::NC; c++)
            if (smem_u32(&sm.st[s].c[c][0]) & 127u) return false;
        if (smem_u32(&sm.bar[s]) & 7u) return false;
    }
    return true;
}

template <int TY, bool LOSSY>
__device__ __forceinline__ void wait_plane(TmaSmem<TY, LOSSY> &sm, int k, int z0, int *err)
{
    const int slot = (k + 3) % 3;
    const unsigned parity = (unsigned)(((k - z0 + 1) / 3) & 1);
    volatile int *abort = &sm.abort;
    if (mbar_wait_bounded(&sm.bar[slot], parity, kWaitNs, abort) || *abort) return;
    *abort = 1;
    atomicExch(err, 1);
}

// CPML data of one cell along x or y (loop invariant for a column)
struct Slab {
    int on;
    long long base;   // psi index without the k term
    float b, a, kinv;
};

__device__ __forceinline__ Slab slab_x(const FusedArgs &a, int gi, int gj, int w0)
{
    Slab r{0, 0, 1.f, 0.f, 1.f};
    const int si = slab_local(gi, a.nx, a.L);
    if (si >= 0) r = {1, si + 2LL * a.L * gj, __ldg(a.prof[w0][0] + gi), __ldg(a.prof[w0 + 1][0] + gi), __ldg(a.prof[w0 + 2][0] + gi)};
    return r;
}

__device__ __forceinline__ Slab slab_y(const FusedArgs &a, int gi, int gj, int w0)
{
    Slab r{0, 0, 1.f, 0.f, 1.f};
    const int sj = slab_local(gj, a.ny, a.L);
    if (sj >= 0) r = {1, gi + (long long)a.nx * sj, __ldg(a.prof[w0][1] + gj), __ldg(a.prof[w0 + 1][1] + gj), __ldg(a.prof[w0 + 2][1] + gj)};
    return r;
}

// per-plane constants (uniform over the block)
struct PlaneInfo {
    int k;
    bool interior;        // 1 <= k <= nz-2
    const float *src;     // source plane at k, or null
    int sk;               // CPML z-slab index, -1 outside
    float bz, az, kz;     // z profile values (E or H side)
};

// One E_new cell.  hN = H(k) at the cell, hxm/hym = H(k) at x-1 (Hy, Hz),
// hyy = H(k) at y-1 (Hx, Hz), hp = H(k-1) at the cell (Hx, Hy); e0 = E_in(k);
// c0 = cb (and ca).  Returns E_new in e0.
template <bool CPML, bool LOSSY>
__device__ __forceinline__ void e_update(const FusedArgs &a, const PlaneInfo &P, long long cij, bool store,
                                         const Slab &sx, const Slab &sy, float hx0, float hy0, float hz0,
                                         float hy_xm, float hz_xm, float hx_ym, float hz_ym, float hx_km,
                                         float hy_km, float &ex, float &ey, float &ez, const float *cb3,
                                         const float *ca3, float nxy_f_unused)
{
    const float dx = a.dx;
    const float dHz_dy = hz0 - hz_ym, dHy_dz = hy0 - hy_km, dHx_dz = hx0 - hx_km;
    const float dHz_dx = hz0 - hz_xm, dHy_dx = hy0 - hy_xm, dHx_dy = hx0 - hx_ym;
    float cx, cy, cz;
    if (!CPML) {
        cx = dHz_dy - dHy_dz;
        cy = dHx_dz - dHz_dx;
        cz = dHy_dx - dHx_dy;
    } else {
        const float div = 1.0f / dx;
        const long long nxy = (long long)a.nx * a.ny;
        float pxy = 0.f, pxz = 0.f, pyx = 0.f, pyz = 0.f, pzx = 0.f, pzy = 0.f;
        if (sx.on) {
            const long long s = sx.base + 2LL * a.L * a.ny * P.k;
            pyx = sx.b * __ldg(a.psi_in[0][0] + s) + sx.a * (dHz_dx * div);
            pzx = sx.b * __ldg(a.psi_in[0][1] + s) + sx.a * (dHy_dx * div);
            if (store) { a.psi_out[0][0][s] = pyx; a.psi_out[0][1][s] = pzx; }
        }
        if (sy.on) {
            const long long s = sy.base + (long long)a.nx * 2 * a.L * P.k;
            pxy = sy.b * __ldg(a.psi_in[1][0] + s) + sy.a * (dHz_dy * div);
            pzy = sy.b * __ldg(a.psi_in[1][1] + s) + sy.a * (dHx_dy * div);
            if (store) { a.psi_out[1][0][s] = pxy; a.psi_out[1][1][s] = pzy; }
        }
        if (P.sk >= 0) {
            const long long s = cij + nxy * P.sk;
            pxz = P.bz * __ldg(a.psi_in[2][0] + s) + P.az * (dHy_dz * div);
            pyz = P.bz * __ldg(a.psi_in[2][1] + s) + P.az * (dHx_dz * div);
            if (store) { a.psi_out[2][0][s] = pxz; a.psi_out[2][1][s] = pyz; }
        }
        cx = sy.kinv * dHz_dy - P.kz * dHy_dz + dx * (pxy - pxz);
        cy = P.kz * dHx_dz - sx.kinv * dHz_dx + dx * (pyz - pyx);
        cz = sx.kinv * dHy_dx - sy.kinv * dHx_dy + dx * (pzx - pzy);
    }
    if (P.src) {
        const long long nxy = (long long)a.nx * a.ny;
        cx -= dx * P.src[cij];
        cy -= dx * P.src[nxy + cij];
        cz -= dx * P.src[2 * nxy + cij];
    }
    if (LOSSY) {
        ex = ca3[0] * ex + cb3[0] * cx;
        ey = ca3[1] * ey + cb3[1] * cy;
        ez = ca3[2] * ez + cb3[2] * cz;
    } else {
        ex = ex + cb3[0] * cx;
        ey = ey + cb3[1] * cy;
        ez = ez + cb3[2] * cz;
    }
}

template <int TY, bool CPML, bool LOSSY>
__global__ void __launch_bounds__(TX * 8, 3)
k_fused_tma(FusedArgs a, const __grid_constant__ FusedMaps maps, int zc, int *err)
{
    constexpr int R = TY / 8;                // rows per thread
    using Stage = TmaStage<TY, LOSSY>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const unsigned pad = (128u - (smem_u32(smem_raw) & 127u)) & 127u;
    TmaSmem<TY, LOSSY> &sm = *reinterpret_cast<TmaSmem<TY, LOSSY> *>(smem_raw + pad);
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long long nxy = (long long)nx * ny;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, tid = threadIdx.x;
    const int X0 = blockIdx.x * TX, Y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, nz);
    if (z0 >= nz) return;
    const float dx = a.dx, hb = a.hb;

    if (tid == 0) {
        const bool layout_ok = tma_layout_ok<TY, LOSSY>(sm);
        if (layout_ok)
            for (int s = 0; s < 3; s++) mbar_init(&sm.bar[s], 1);
        sm.abort = layout_ok ? 0 : 1;
        if (!layout_ok) atomicExch(err, 2);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    const bool live = sm.abort == 0;
    if (tid == 0 && live) {
        issue_plane<TY, LOSSY>(sm, maps, z0 - 1, X0, Y0);
        issue_plane<TY, LOSSY>(sm, maps, z0, X0, Y0);
        if (z0 + 1 <= z1 && z0 + 1 < nz) issue_plane<TY, LOSSY>(sm, maps, z0 + 1, X0, Y0);
    }

    // this thread's cells: x = X0 + lane, rows y = Y0 + R*warp + r
    const int gi = X0 + lane;
    int gj[R];
    bool cell_ok[R];
    Slab sxE[R], syE[R], sxH[R], syH[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        gj[r] = Y0 + R * warp + r;
        cell_ok[r] = gi >= 1 && gi <= nx - 2 && gj[r] >= 1 && gj[r] <= ny - 2;
        sxE[r] = syE[r] = sxH[r] = syH[r] = Slab{0, 0, 1.f, 0.f, 1.f};
        if (CPML && cell_ok[r]) {
            sxE[r] = slab_x(a, gi, gj[r], 0);
            syE[r] = slab_y(a, gi, gj[r], 0);
            sxH[r] = slab_x(a, gi, gj[r], 3);
            syH[r] = slab_y(a, gi, gj[r], 3);
        }
    }
    // halo cells: the +x column (TY cells) and +y row (TX cells), spread over the warps
    constexpr int NHALO = TY + TX;
    constexpr int HALO_PER_WARP = (NHALO + 7) / 8;

    // carried registers: H_in(k-1) and E_new(k-1) of the thread's own cells
    float hpx[R], hpy[R], hpz[R], epx[R], epy[R], epz[R];

    // prologue: H_in(z0-1) at own cells
    if (z0 - 1 >= 0 || true) {
        wait_plane<TY, LOSSY>(sm, z0 - 1, z0, err);
        const Stage &S = sm.st[(z0 + 2) % 3];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int ly = R * warp + r;
            hpx[r] = Hat(S.h[0], lane, ly);
            hpy[r] = Hat(S.h[1], lane, ly);
            hpz[r] = Hat(S.h[2], lane, ly);
            epx[r] = epy[r] = epz[r] = 0.f;
        }
    }

    for (int k = z0; k <= z1; k++) {
        const int p3 = k % 3, pm3 = (k + 2) % 3;
        float enx[R], eny[R], enz[R];      // E_new(k) own
        float hnx[R], hny[R], hnz[R];      // H_in(k) own
        if (k < nz) {
            wait_plane<TY, LOSSY>(sm, k, z0, err);
            const Stage &S = sm.st[p3];
            PlaneInfo P;
            P.k = k;
            P.interior = k >= 1 && k <= nz - 2;
            P.src = nullptr;
            for (int t = 0; t < a.src.n; t++)
                if (a.src.k[t] == k) P.src = a.src.p[t];
            P.sk = CPML ? slab_local(k, nz, a.L) : -1;
            P.bz = 1.f; P.az = 0.f; P.kz = 1.f;
            if (CPML && P.sk >= 0) {
                P.bz = __ldg(a.prof[0][2] + k);
                P.az = __ldg(a.prof[1][2] + k);
                P.kz = __ldg(a.prof[2][2] + k);
            }
            const bool store = k < z1;
            // own cells
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int ly = R * warp + r;
                hnx[r] = Hat(S.h[0], lane, ly);
                hny[r] = Hat(S.h[1], lane, ly);
                hnz[r] = Hat(S.h[2], lane, ly);
                float ex = Eat(S.e[0], lane, ly), ey = Eat(S.e[1], lane, ly), ez = Eat(S.e[2], lane, ly);
                if (P.interior && cell_ok[r]) {
                    const float hx_ym = r > 0 ? hnx[r - 1] : Hat(S.h[0], lane, ly - 1);
                    const float hz_ym = r > 0 ? hnz[r - 1] : Hat(S.h[2], lane, ly - 1);
                    const float hy_xm = Hat(S.h[1], lane - 1, ly);
                    const float hz_xm = Hat(S.h[2], lane - 1, ly);
                    float cb3[3] = {Eat(S.c[0], lane, ly), Eat(S.c[1], lane, ly), Eat(S.c[2], lane, ly)};
                    float ca3[3] = {1.f, 1.f, 1.f};
                    if (LOSSY) { ca3[0] = Eat(S.c[3], lane, ly); ca3[1] = Eat(S.c[4], lane, ly); ca3[2] = Eat(S.c[5], lane, ly); }
                    const long long cij = gi + (long long)nx * gj[r];
                    e_update<CPML, LOSSY>(a, P, cij, store, sxE[r], syE[r], hnx[r], hny[r], hnz[r], hy_xm, hz_xm,
                                          hx_ym, hz_ym, hpx[r], hpy[r], ex, ey, ez, cb3, ca3, 0.f);
                    if (store) {
                        const long long q = cij + nxy * k;
                        a.f_out[0][q] = ex;
                        a.f_out[1][q] = ey;
                        a.f_out[2][q] = ez;
                    }
                }
                enx[r] = ex; eny[r] = ey; enz[r] = ez;
                sm.en[p3][0][ly][lane] = ex;
                sm.en[p3][1][ly][lane] = ey;
                sm.en[p3][2][ly][lane] = ez;
            }
            // halo cells of this warp (all neighbours from the boxes)
            if (lane < HALO_PER_WARP) {
                const int t = warp * HALO_PER_WARP + lane;
                if (t < NHALO) {
                    const int lx = t < TY ? TX : t - TY, ly = t < TY ? t : TY;
                    const int hgi = X0 + lx, hgj = Y0 + ly;
                    float ex = Eat(S.e[0], lx, ly), ey = Eat(S.e[1], lx, ly), ez = Eat(S.e[2], lx, ly);
                    if (P.interior && hgi >= 1 && hgi <= nx - 2 && hgj >= 1 && hgj <= ny - 2) {
                        const Stage &Sm = sm.st[pm3];
                        Slab hsx{0, 0, 1.f, 0.f, 1.f}, hsy{0, 0, 1.f, 0.f, 1.f};
                        if (CPML) {
                            hsx = slab_x(a, hgi, hgj, 0);
                            hsy = slab_y(a, hgi, hgj, 0);
                        }
                        float cb3[3] = {Eat(S.c[0], lx, ly), Eat(S.c[1], lx, ly), Eat(S.c[2], lx, ly)};
                        float ca3[3] = {1.f, 1.f, 1.f};
                        if (LOSSY) { ca3[0] = Eat(S.c[3], lx, ly); ca3[1] = Eat(S.c[4], lx, ly); ca3[2] = Eat(S.c[5], lx, ly); }
                        e_update<CPML, LOSSY>(a, P, hgi + (long long)nx * hgj, false, hsx, hsy, Hat(S.h[0], lx, ly),
                                              Hat(S.h[1], lx, ly), Hat(S.h[2], lx, ly), Hat(S.h[1], lx - 1, ly),
                                              Hat(S.h[2], lx - 1, ly), Hat(S.h[0], lx, ly - 1), Hat(S.h[2], lx, ly - 1),
                                              Hat(Sm.h[0], lx, ly), Hat(Sm.h[1], lx, ly), ex, ey, ez, cb3, ca3, 0.f);
                    }
                    sm.en[p3][0][ly][lx] = ex;
                    sm.en[p3][1][ly][lx] = ey;
                    sm.en[p3][2][ly][lx] = ez;
                }
            }
        }
        __syncthreads();
        // the stage of plane k-1 is no longer read: refill it with plane k+2
        if (tid == 0 && live && k + 2 <= z1 && k + 2 < nz) issue_plane<TY, LOSSY>(sm, maps, k + 2, X0, Y0);
        // H_new(k-1) at own cells: E_new(k-1) own in epx.., E_new(k) own in enx.., H_in(k-1) in hpx..
        const int km = k - 1;
        if (km >= z0 && km >= 1 && km <= nz - 2) {
            int skH = -1;
            float bzH = 1.f, azH = 0.f, kzH = 1.f;
            if (CPML) {
                skH = slab_local(km, nz, a.L);
                if (skH >= 0) {
                    bzH = __ldg(a.prof[3][2] + km);
                    azH = __ldg(a.prof[4][2] + km);
                    kzH = __ldg(a.prof[5][2] + km);
                }
            }
            const float *srcH = nullptr;
            for (int t = 0; t < a.src.n; t++)
                if (a.src.k[t] == km) srcH = a.src.p[t];
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int ly = R * warp + r;
                // E_new(k-1) at x+1 (Ey, Ez) and y+1 (Ex, Ez)
                float ey_xp = __shfl_down_sync(0xffffffffu, epy[r], 1);
                float ez_xp = __shfl_down_sync(0xffffffffu, epz[r], 1);
                if (lane == 31) {
                    ey_xp = sm.en[pm3][1][ly][TX];
                    ez_xp = sm.en[pm3][2][ly][TX];
                }
                const float ex_yp = r + 1 < R ? epx[r + 1 < R ? r + 1 : r] : sm.en[pm3][0][ly + 1][lane];
                const float ez_yp = r + 1 < R ? epz[r + 1 < R ? r + 1 : r] : sm.en[pm3][2][ly + 1][lane];
                if (!cell_ok[r]) continue;
                const float dEz_dy = ez_yp - epz[r];
                const float dEy_dz = eny[r] - epy[r];
                const float dEx_dz = enx[r] - epx[r];
                const float dEz_dx = ez_xp - epz[r];
                const float dEy_dx = ey_xp - epy[r];
                const float dEx_dy = ex_yp - epx[r];
                const long long cij = gi + (long long)nx * gj[r];
                float cx, cy, cz;
                if (!CPML) {
                    cx = dEz_dy - dEy_dz;
                    cy = dEx_dz - dEz_dx;
                    cz = dEy_dx - dEx_dy;
                } else {
                    const float div = 1.0f / dx;
                    float pxy = 0.f, pxz = 0.f, pyx = 0.f, pyz = 0.f, pzx = 0.f, pzy = 0.f;
                    const Slab &sx = sxH[r], &sy = syH[r];
                    if (sx.on) {
                        const long long s = sx.base + 2LL * a.L * ny * km;
                        pyx = sx.b * __ldg(a.psi_in[0][2] + s) + sx.a * (dEz_dx * div);
                        pzx = sx.b * __ldg(a.psi_in[0][3] + s) + sx.a * (dEy_dx * div);
                        a.psi_out[0][2][s] = pyx;
                        a.psi_out[0][3][s] = pzx;
                    }
                    if (sy.on) {
                        const long long s = sy.base + (long long)nx * 2 * a.L * km;
                        pxy = sy.b * __ldg(a.psi_in[1][2] + s) + sy.a * (dEz_dy * div);
                        pzy = sy.b * __ldg(a.psi_in[1][3] + s) + sy.a * (dEx_dy * div);
                        a.psi_out[1][2][s] = pxy;
                        a.psi_out[1][3][s] = pzy;
                    }
                    if (skH >= 0) {
                        const long long s = cij + nxy * skH;
                        pxz = bzH * __ldg(a.psi_in[2][2] + s) + azH * (dEy_dz * div);
                        pyz = bzH * __ldg(a.psi_in[2][3] + s) + azH * (dEx_dz * div);
                        a.psi_out[2][2][s] = pxz;
                        a.psi_out[2][3][s] = pyz;
                    }
                    cx = sy.kinv * dEz_dy - kzH * dEy_dz + dx * (pxy - pxz);
                    cy = kzH * dEx_dz - sx.kinv * dEz_dx + dx * (pyz - pyx);
                    cz = sx.kinv * dEy_dx - sy.kinv * dEx_dy + dx * (pzx - pzy);
                }
                if (srcH) {
                    cx += dx * srcH[3 * nxy + cij];
                    cy += dx * srcH[4 * nxy + cij];
                    cz += dx * srcH[5 * nxy + cij];
                }
                const long long q = cij + nxy * km;
                a.f_out[3][q] = hpx[r] - hb * cx;
                a.f_out[4][q] = hpy[r] - hb * cy;
                a.f_out[5][q] = hpz[r] - hb * cz;
            }
        }
        // carry: E_new(k), H_in(k) become the previous plane
        if (k < nz) {
#pragma unroll
            for (int r = 0; r < R; r++) {
                epx[r] = enx[r]; epy[r] = eny[r]; epz[r] = enz[r];
                hpx[r] = hnx[r]; hpy[r] = hny[r]; hpz[r] = hnz[r];
            }
        }
    }
    // every issued plane (z0-1 .. min(z1, nz-1)) was waited for in the loop
}

// ---- host side ---------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        cudaGetLastError();
    }
    return fn;
}

constexpr int kTY = 8;   // tile height (rows per thread = kTY / 8)

int fused_tma_supported(int nx, int ny, int nz) { return nx % 4 == 0 && nx >= 8 && ny >= 4 && nz >= 4 && encode_fn(); }

static bool encode(CUtensorMap *m, const float *base, int nx, int ny, int nz, int box_x, int box_y)
{
    cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    cuuint64_t strides[2] = {(cuuint64_t)nx * 4, (cuuint64_t)nx * ny * 4};
    cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1};
    cuuint32_t elem[3] = {1, 1, 1};
    CUresult r = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)base, dims, strides, box, elem,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool fused_make_maps(FusedMaps *m, const float *const f[6], const float *const cb[3], const float *const ca[3],
                     int nx, int ny, int nz)
{
    if (!encode_fn()) return false;
    for (int c = 0; c < 3; c++) {
        if (!encode(&m->h[c], f[3 + c], nx, ny, nz, HW, kTY + 2)) return false;
        if (!encode(&m->e[c], f[c], nx, ny, nz, EW, kTY + 1)) return false;
        if (!encode(&m->cb[c], cb[c], nx, ny, nz, EW, kTY + 1)) return false;
        if (ca && ca[c]) {
            if (!encode(&m->ca[c], ca[c], nx, ny, nz, EW, kTY + 1)) return false;
        } else {
            m->ca[c] = m->cb[c];
        }
    }
    return true;
}

template <bool CPML, bool LOSSY>
static void launch_tma(const FusedArgs &a, const FusedMaps &m, int *err, cudaStream_t st)
{
    auto kern = k_fused_tma<kTY, CPML, LOSSY>;
    const size_t smem = tma_smem_bytes<kTY, LOSSY>();
    static int slots = -1;
    if (slots < 0) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int per_sm = 0, dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TX * 8, smem);
        slots = per_sm * sms;
    }
    long long tiles = (long long)((a.nx + TX - 1) / TX) * ((a.ny + kTY - 1) / kTY);
    long long chunks = slots > 0 ? slots / tiles : 1;
    if (chunks < 1) chunks = 1;
    int zc = (int)((a.nz + chunks - 1) / chunks);
    if (zc < 8) zc = 8;
    dim3 grid((a.nx + TX - 1) / TX, (a.ny + kTY - 1) / kTY, (a.nz + zc - 1) / zc);
    kern<<<grid, TX * 8, smem, st>>>(a, m, zc, err);
}

void launch_fused_step_tma(const FusedArgs &a, const FusedMaps &m, int *err, cudaStream_t st)
{
    note_launch();
    const bool lossy = a.ca[0] != nullptr;
    if (a.L > 0) {
        if (lossy) launch_tma<true, true>(a, m, err, st);
        else launch_tma<true, false>(a, m, err, st);
    } else {
        if (lossy) launch_tma<false, true>(a, m, err, st);
        else launch_tma<false, false>(a, m, err, st);
    }
}

// Self-test of the bounded wait: one block waits on an mbarrier that expects
// one arrival which never comes.  The wait must give up after limit_ns, set
// *err like a pipeline wait does and leave the kernel (and the context) in
// good order; *elapsed_ns records how long it waited.
__global__ void k_wait_selftest(unsigned long long limit_ns, int *err, unsigned long long *elapsed_ns)
{
    __shared__ unsigned long long bar;
    __shared__ int abort;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        abort = 0;
    }
    __syncthreads();
    const unsigned long long t0 = global_ns();
    const bool done = mbar_wait_bounded(&bar, 0, limit_ns, &abort);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (!done) atomicExch(err, 1);
        *elapsed_ns = global_ns() - t0;
    }
}

void launch_wait_selftest(unsigned long long limit_ns, int *err, unsigned long long *elapsed_ns, cudaStream_t st)
{
    note_launch();
    k_wait_selftest<<<1, 32, 0, st>>>(limit_ns, err, elapsed_ns);
}

}  // namespace fdtd
