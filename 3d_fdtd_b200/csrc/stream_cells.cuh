// stream_cells.cuh -- the one-pass FP32 Yee tile of the streaming kernels
// (yee_stream.cu: one grid per launch; yee_sweep.cu: many grids and steps in
// one persistent launch).  See yee_stream.cu for the design.
#pragma once

#include "flat4_cells.cuh"

namespace fdtd {

constexpr int kStreamStages = 3;
// cell index within one array of a streaming grid: 32 bits (stream_supported
// refuses grids of 2^31 cells or more), so an index takes one register
using sidx_t = unsigned;
// 16 warps: up to 128 registers a thread at one block per SM (an SM's four
// sub-partitions hold 16K registers each, a quarter of the warps each)
constexpr int kStreamMaxThreads = 512;

__device__ __forceinline__ void cp_async16(float *smem, const float *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's most recent groups are still pending
template <int N> __device__ __forceinline__ void cp_async_wait_group()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ Vf<4> lds4(const float *p)
{
    const float4 t = *reinterpret_cast<const float4 *>(p);
    Vf<4> r;
    r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
    return r;
}
__device__ __forceinline__ void sts4(float *p, const Vf<4> &x)
{
    *reinterpret_cast<float4 *>(p) = make_float4(x.v[0], x.v[1], x.v[2], x.v[3]);
}
__device__ __forceinline__ Vf<2> lds2(const float *p)
{
    const float2 t = *reinterpret_cast<const float2 *>(p);
    Vf<2> r;
    r.v[0] = t.x; r.v[1] = t.y;
    return r;
}
__device__ __forceinline__ void sts2(float *p, const Vf<2> &x) { *reinterpret_cast<float2 *>(p) = make_float2(x.v[0], x.v[1]); }

// ---- CPML auxiliaries of one group of W consecutive x cells (an interior
//      quad, W = 4, or one x-slab cell, W = 1) for one field (E: A0 = 0, H:
//      A0 = 2).  x-slab: per element, staged in shared memory with the plane
//      (rows of 2L values); y- and z-slab: contiguous in x, read from global
//      memory.  The 1-D profiles of the slab cells sit in a shared table filled
//      at the start of the tile (stream_profile_table): read from global
//      memory at every use they missed L1 (the staged planes leave it a few
//      KB) and put an L2 round trip on every x-slab cell's update.
template <int W> struct XPsi {
    bool valid[W];
    float p0[W], p1[W];
    float b[W], c[W], k[W];     // the x profiles (b, a, 1/kappa) of a single x-slab cell (W = 1)
};
template <int W> struct YZPsi {
    int sj, sk;
    Vf<W> pxy, pzy, pxz, pyz;   // as YZSlab: (x,y) (z,y) (x,z) (y,z) for E, alike for H
    float py[3], pz[3];         // y and z profiles (b, a, 1/kappa) of a single x-slab cell (W = 1)
};

// x-slab auxiliaries of one x-slab cell from a staged row pair, with the
// cell's slab-local index and x profiles kept in registers for the tile
__device__ __forceinline__ void stream_xpsi_cell(XPsi<1> &xs, const float *row0, const float *row1, int si, bool valid,
                                                 const float (&prof)[3])
{
    xs.valid[0] = valid;
    xs.p0[0] = valid ? row0[si] : 0.f;
    xs.p1[0] = valid ? row1[si] : 0.f;
    xs.b[0] = prof[0];
    xs.c[0] = prof[1];
    xs.k[0] = prof[2];
}

// x-slab auxiliaries of the group at x = i0.. from a staged row pair (row0,
// row1: the two auxiliaries of this field for the cell row)
template <int W>
__device__ __forceinline__ void stream_xpsi(XPsi<W> &xs, const float *row0, const float *row1, int nx, int L, int i0)
{
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = i0 + e;
        const int si = slab_local(i, nx, L);
        xs.valid[e] = si >= 0 && i >= 1 && i <= nx - 2;
        xs.p0[e] = xs.valid[e] ? row0[si] : 0.f;
        xs.p1[e] = xs.valid[e] ? row1[si] : 0.f;
    }
}

// Shared profile table of a tile: [axis x, y, z][profile 0..5][2L slab-local
// cells] (profiles 0..2: b, a, 1/kappa of E; 3..5 of H; slab-local index as
// slab_local), filled by the whole block; the caller puts a block barrier
// between the fill and any read.
__device__ __forceinline__ void stream_profile_table(float *pt, const StreamArgs &a)
{
    const int L = a.L, PL = 2 * L;
    for (int s = (int)threadIdx.x; s < PL; s += (int)blockDim.x) {
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            const int N = ax == 0 ? a.nx : (ax == 1 ? a.ny : a.nz);
            const int g = s < L ? s : N - PL + s;
#pragma unroll
            for (int w = 0; w < 6; w++) pt[(ax * 6 + w) * PL + s] = __ldg(a.prof[w][ax] + g);
        }
    }
}

// COH: plain (coherent) loads, for launches in which other blocks wrote the
// auxiliaries (the multi-step sweep); else the read-only path
// (a single x-slab cell, W = 1, also takes its y and z profiles from the
// tile's table `pt` here, an iteration before they are used)
template <int W, int A0, bool COH>
__device__ __forceinline__ void stream_yzpsi_load(YZPsi<W> &s, const StreamArgs &a, int i0, int j, int k,
                                                  sidx_t ij0, sidx_t nxy, const float *pt = nullptr)
{
    const int nx = a.nx, L = a.L;
    s.sj = slab_local(j, a.ny, L);
    s.sk = slab_local(k, a.nz, L);
    s.pxy = fillv<W>(0.f); s.pzy = s.pxy; s.pxz = s.pxy; s.pyz = s.pxy;
    if (s.sj >= 0) {
        const sidx_t sy = (sidx_t)i0 + (sidx_t)nx * (sidx_t)(s.sj + 2 * L * k);
        s.pxy = ldf<W, COH>(a.psi_in[1][A0] + sy);
        s.pzy = ldf<W, COH>(a.psi_in[1][A0 + 1] + sy);
        if constexpr (W == 1) {
            const float *py = pt + (6 + 3 * (A0 / 2)) * 2 * L + s.sj;
#pragma unroll
            for (int w = 0; w < 3; w++) s.py[w] = py[w * 2 * L];
        }
    }
    if (s.sk >= 0) {
        const sidx_t sz = ij0 + nxy * (sidx_t)s.sk;
        s.pxz = ldf<W, COH>(a.psi_in[2][A0] + sz);
        s.pyz = ldf<W, COH>(a.psi_in[2][A0 + 1] + sz);
        if constexpr (W == 1) {
            const float *pz = pt + (12 + 3 * (A0 / 2)) * 2 * L + s.sk;
#pragma unroll
            for (int w = 0; w < 3; w++) s.pz[w] = pz[w * 2 * L];
        }
    }
}

// a quad wholly inside one x slab, with its auxiliaries 16-byte aligned (L
// even): copied as one vector; the elements x = 0 / nx-1 hold 0, which is
// their auxiliaries' value for good (they are never updated)
__device__ __forceinline__ bool xquad_whole(int i0, int nx, int L)
{
    return (L & 1) == 0 && (i0 + 3 < L || i0 >= nx - L);
}

// updated auxiliaries of the group: x slab (XS: the group may hold x-slab
// cells), then y and z slabs
template <int W, int A0, bool XS>
__device__ __forceinline__ void stream_psi_store(const XPsi<W> &xs, const YZPsi<W> &s, const StreamArgs &a, int i0,
                                                 int j, int k, sidx_t ij0, sidx_t nxy)
{
    const int nx = a.nx, L = a.L;
    if (XS) {
        const sidx_t s0 = (sidx_t)(2 * L) * ((sidx_t)j + (sidx_t)a.ny * (sidx_t)k);
#pragma unroll
        for (int e = 0; e < W; e++) {
            if (!xs.valid[e]) continue;
            const sidx_t sidx = s0 + (sidx_t)slab_local(i0 + e, nx, L);
            a.psi_out[0][A0][sidx] = xs.p0[e];
            a.psi_out[0][A0 + 1][sidx] = xs.p1[e];
        }
    }
    if (s.sj >= 0) {
        const sidx_t sy = (sidx_t)i0 + (sidx_t)nx * (sidx_t)(s.sj + 2 * L * k);
        stv<W>(a.psi_out[1][A0] + sy, s.pxy);
        stv<W>(a.psi_out[1][A0 + 1] + sy, s.pzy);
    }
    if (s.sk >= 0) {
        const sidx_t sz = ij0 + nxy * (sidx_t)s.sk;
        stv<W>(a.psi_out[2][A0] + sz, s.pxz);
        stv<W>(a.psi_out[2][A0 + 1] + sz, s.pyz);
    }
}

// One cell's curl with the CPML terms: the arithmetic of cpml_curl
// (flat4_cells.cuh) term for term, with the profiles from the tile's shared
// table `pt` (stream_profile_table).  pw = 0 for E (b, a, 1/kappa of E), 3 for
// H.  X: the cell may lie in an x slab (its x terms are compiled in); without
// X the x terms are the interior's (kappa 1, no auxiliary), exactly what the
// general expression gives there.
template <int W, bool X, int pw>
__device__ __forceinline__ Curl3 stream_cpml_curl(XPsi<W> &xs, YZPsi<W> &s, const float *pt, int nx, int L, int i, int e,
                                                  float d_zy, float d_yz, float d_xz, float d_zx, float d_yx,
                                                  float d_xy, float dx, float div)
{
    const int PL = 2 * L;
    float pyx = 0.f, pzx = 0.f, kx = 1.f;
    if (X && xs.valid[e]) {
        float b, c;
        if constexpr (W == 1) {
            b = xs.b[e]; c = xs.c[e]; kx = xs.k[e];
        } else {
            const float *px = pt + pw * PL + slab_local(i, nx, L);
            b = px[0]; c = px[PL]; kx = px[2 * PL];
        }
        pyx = b * xs.p0[e] + c * (d_zx * div);
        pzx = b * xs.p1[e] + c * (d_yx * div);
        xs.p0[e] = pyx;
        xs.p1[e] = pzx;
    }
    float vxy = 0.f, vzy = 0.f, vxz = 0.f, vyz = 0.f, ky = 1.f, kz = 1.f;
    if (s.sj >= 0) {
        float by, ay;
        if constexpr (W == 1) {
            by = s.py[0]; ay = s.py[1]; ky = s.py[2];
        } else {
            const float *py = pt + (6 + pw) * PL + s.sj;
            by = py[0]; ay = py[PL]; ky = py[2 * PL];
        }
        vxy = by * s.pxy.v[e] + ay * (d_zy * div);
        vzy = by * s.pzy.v[e] + ay * (d_xy * div);
        s.pxy.v[e] = vxy;
        s.pzy.v[e] = vzy;
    }
    if (s.sk >= 0) {
        float bz, az;
        if constexpr (W == 1) {
            bz = s.pz[0]; az = s.pz[1]; kz = s.pz[2];
        } else {
            const float *pz = pt + (12 + pw) * PL + s.sk;
            bz = pz[0]; az = pz[PL]; kz = pz[2 * PL];
        }
        vxz = bz * s.pxz.v[e] + az * (d_yz * div);
        vyz = bz * s.pyz.v[e] + az * (d_xz * div);
        s.pxz.v[e] = vxz;
        s.pyz.v[e] = vyz;
    }
    Curl3 c;
    c.x = ky * d_zy - kz * d_yz + dx * (vxy - vxz);
    c.y = kz * d_xz - kx * d_zx + dx * (vyz - pyx);
    c.z = kx * d_yx - ky * d_xy + dx * (pzx - vzy);
    return c;
}

// 4-byte asynchronous copy (x-slab auxiliaries, one per element)
__device__ __forceinline__ void cp_async4(float *smem, const float *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

// Work roles of the block's threads.  An interior thread owns 4 consecutive x
// cells (a quad) of one staged row.  On a CPML grid the quads that reach into
// an x slab (row ends) are not given to quad threads: every cell of them has
// a thread of its own (x-cell threads, 4 consecutive lanes per quad), in
// warps after the interior ones.  An x-slab cell's update carries the
// auxiliary recursion, its profiles and the row-end rules, several times the
// work of an interior cell, and the block waits for its slowest warp at each
// plane's barrier: a whole quad per thread (or a pair) made the x-slab
// threads the slowest of every plane.  Interior warps carry no x-slab code.
struct StreamRoles {
    int QL, QR;      // x-slab quads: q < QL or q >= QR (QL = QR = 0 when there is no x slab)
    int QI, NXQ;     // interior and x-slab quads per row
    int xbase;       // first thread of the x-cell warps
    int threads;     // block size
};

__host__ __device__ inline StreamRoles stream_roles(int nx, int L, int tp)
{
    StreamRoles r{};
    const int QX = nx / 4;
    if (L <= 0) {
        r.QL = 0; r.QR = QX; r.QI = QX; r.NXQ = 0;
        r.xbase = tp * QX;
        r.threads = (tp * QX + 31) / 32 * 32;
        return r;
    }
    r.QL = (L + 3) / 4;                                  // 4q < L
    r.QR = (nx - L - 3 + 3) / 4;                         // 4q + 3 >= nx - L
    if (r.QR < r.QL) r.QR = r.QL;
    if (r.QR > QX) r.QR = QX;
    r.QI = r.QR - r.QL;
    r.NXQ = QX - r.QI;
    r.xbase = (tp * r.QI + 31) / 32 * 32;
    r.threads = (r.xbase + tp * 4 * r.NXQ + 31) / 32 * 32;
    return r;
}

// E_new of one group of W cells at x = i0 (an interior quad, W = 4, or one
// x-slab cell, W = 1).  X: x-slab group (x terms, and the cells x = 0 / nx-1
// of the row ends stay); EDGE: the group may hold x = 0 / nx-1 (row ends of a
// grid without CPML).  hy_im0, hz_im0: Hy, Hz at x = i0 - 1.
template <int W, bool X, bool EDGE, bool CPML, bool LOSSY, bool COH>
__device__ __forceinline__ void stream_e_group(Vf<W> &ex, Vf<W> &ey, Vf<W> &ez, const Vf<W> &hx, const Vf<W> &hy,
                                               const Vf<W> &hz, const Vf<W> &hx_km, const Vf<W> &hy_km,
                                               const Vf<W> &hx_jm, const Vf<W> &hz_jm, float hy_im0, float hz_im0,
                                               const Vf<W> &b0, const Vf<W> &b1, const Vf<W> &b2, const Vf<W> &c0,
                                               const Vf<W> &c1, const Vf<W> &c2, XPsi<W> &xs, YZPsi<W> &yz,
                                               const float *pt, const StreamArgs &a, int i0, const float *sp,
                                               sidx_t ij0, sidx_t nxy, float dx, float div)
{
    const bool plain = !CPML || (!X && yz.sj < 0 && yz.sk < 0);
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = i0 + e;
        if ((X || EDGE) && (i < 1 || i > a.nx - 2)) continue;   // x = 0 and x = nx-1 stay
        const float hy_im = e == 0 ? hy_im0 : hy.v[e == 0 ? 0 : e - 1];
        const float hz_im = e == 0 ? hz_im0 : hz.v[e == 0 ? 0 : e - 1];
        const float dHz_dy = hz.v[e] - hz_jm.v[e];
        const float dHy_dz = hy.v[e] - hy_km.v[e];
        const float dHx_dz = hx.v[e] - hx_km.v[e];
        const float dHz_dx = hz.v[e] - hz_im;
        const float dHy_dx = hy.v[e] - hy_im;
        const float dHx_dy = hx.v[e] - hx_jm.v[e];
        float cx, cy, cz;
        if (plain) {
            cx = dHz_dy - dHy_dz;
            cy = dHx_dz - dHz_dx;
            cz = dHy_dx - dHx_dy;
        } else {
            const Curl3 c = stream_cpml_curl<W, X, 0>(xs, yz, pt, a.nx, a.L, i, e, dHz_dy, dHy_dz, dHx_dz, dHz_dx,
                                                      dHy_dx, dHx_dy, dx, div);
            cx = c.x; cy = c.y; cz = c.z;
        }
        if (sp) {
            cx -= dx * ldf1<COH>(sp + ij0 + e);
            cy -= dx * ldf1<COH>(sp + nxy + ij0 + e);
            cz -= dx * ldf1<COH>(sp + 2 * nxy + ij0 + e);
        }
        ex.v[e] = c0.v[e] * ex.v[e] + b0.v[e] * cx;
        ey.v[e] = c1.v[e] * ey.v[e] + b1.v[e] * cy;
        ez.v[e] = c2.v[e] * ez.v[e] + b2.v[e] * cz;
    }
}

// H_new of one group (same roles as stream_e_group); ey_ipw, ez_ipw: new Ey,
// Ez at x = i0 + W
template <int W, bool X, bool EDGE, bool CPML, bool COH>
__device__ __forceinline__ void stream_h_group(Vf<W> &nhx, Vf<W> &nhy, Vf<W> &nhz, const Vf<W> &ex, const Vf<W> &ey,
                                               const Vf<W> &exm, const Vf<W> &eym, const Vf<W> &ezm,
                                               const Vf<W> &ex_jp, const Vf<W> &ez_jp, float ey_ipw, float ez_ipw,
                                               XPsi<W> &xs, YZPsi<W> &yz, const float *pt, const StreamArgs &a,
                                               int i0, const float *sp, sidx_t ij0, sidx_t nxy, float dx,
                                               float div, float hb)
{
    const bool plain = !CPML || (!X && yz.sj < 0 && yz.sk < 0);
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = i0 + e;
        if ((X || EDGE) && (i < 1 || i > a.nx - 2)) continue;
        const float ey_ip = e == W - 1 ? ey_ipw : eym.v[e == W - 1 ? e : e + 1];
        const float ez_ip = e == W - 1 ? ez_ipw : ezm.v[e == W - 1 ? e : e + 1];
        const float dEz_dy = ez_jp.v[e] - ezm.v[e];
        const float dEy_dz = ey.v[e] - eym.v[e];
        const float dEx_dz = ex.v[e] - exm.v[e];
        const float dEz_dx = ez_ip - ezm.v[e];
        const float dEy_dx = ey_ip - eym.v[e];
        const float dEx_dy = ex_jp.v[e] - exm.v[e];
        float cx, cy, cz;
        if (plain) {
            cx = dEz_dy - dEy_dz;
            cy = dEx_dz - dEz_dx;
            cz = dEy_dx - dEx_dy;
        } else {
            const Curl3 c = stream_cpml_curl<W, X, 3>(xs, yz, pt, a.nx, a.L, i, e, dEz_dy, dEy_dz, dEx_dz, dEz_dx,
                                                      dEy_dx, dEx_dy, dx, div);
            cx = c.x; cy = c.y; cz = c.z;
        }
        if (sp) {
            cx += dx * ldf1<COH>(sp + 3 * nxy + ij0 + e);
            cy += dx * ldf1<COH>(sp + 4 * nxy + ij0 + e);
            cz += dx * ldf1<COH>(sp + 5 * nxy + ij0 + e);
        }
        nhx.v[e] = nhx.v[e] - hb * cx;
        nhy.v[e] = nhy.v[e] - hb * cy;
        nhz.v[e] = nhz.v[e] - hb * cz;
    }
}

// The tile's per-plane barrier.  The two thread roles run loops of their own
// (each with the registers of its own work only) and meet here once per
// iteration, the same number of times: every thread of the block takes part.
__device__ __forceinline__ void stream_plane_barrier() { asm volatile("bar.sync 1;\n" ::: "memory"); }

// One tile (band of rows x chunk of planes) of one grid's step, by the whole
// block, with `sm` the block's dynamic shared memory (stream_smem_floats of
// the grid's nx, a.ty, loss and L).  Ends with no copy in flight.
//
// Iteration it (plane k = k0 + it, it = 0..n) updates E of plane k (owned rows
// and the halo row j0 + rows) and H of plane k-1 (owned rows), with the
// staged planes of a 3-stage ring: stage it % 3 holds plane k, the previous
// stage plane k-1, and right after the barrier the previous stage takes the
// copies of plane k+2.  Each thread copies only slots that it reads itself in
// the iteration that refills them (old H of plane k-1, H's x-slab
// auxiliaries); the four x-cell lanes of a quad read their elements of slots
// that another of them copies, so they meet at a warp barrier in between.
//
// TPC > 0: the staged rows a.ty + 1 known at compile time (the per-step kernel
// is instantiated for 2..8; shared-memory offsets then fold into constants).
template <bool CPML, bool LOSSY, bool COH = false, int TPC = 0>
__device__ __forceinline__ void stream_tile(const StreamArgs &a, const StreamTile tl, float *sm)
{
    constexpr int S = kStreamStages;
    constexpr int NA = LOSSY ? 12 : 9;   // staged arrays: Hx Hy Hz, Ex Ey Ez, cb0..2 (, ca0..2)
    const int nx = a.nx, ny = a.ny, nz = a.nz, L = CPML ? a.L : 0;
    const int TP = TPC > 0 ? TPC : a.ty + 1;         // staged rows per array
    const int XW = stream_xpsi_stride(L);            // staged x-slab auxiliaries per row (2L, padded)
    const sidx_t nxy = (sidx_t)nx * (sidx_t)ny;
    const StreamRoles ro = stream_roles(nx, L, TP);
    const int tid = (int)threadIdx.x;
    const bool xw = CPML && tid >= ro.xbase;          // warp-uniform: xbase is a multiple of 32
    const int R = tl.rows;
    const int QX = nx >> 2;
    float *stage = sm;                               // [S][NA][TP][nx]
    float *xps = stage + (size_t)S * NA * TP * nx;   // [S][4][TP][XW]: x-slab auxiliaries E0 E1 H0 H1
    float *hlow = xps + (size_t)S * 4 * TP * XW;     // [S][2][nx]: Hx, Hz of row j0-1
    float *es = hlow + (size_t)S * 2 * nx;           // [2][3][TP][nx]: new E of the last two planes
    float *ptab = es + (size_t)2 * 3 * TP * nx;      // CPML profiles of the slab cells (stream_profile_table)
    if (CPML) {
        stream_profile_table(ptab, a);
        __syncthreads();   // x-slab cells read the table before the first plane's barrier
    }
    // shared-memory offsets fit 32 bits (the whole allocation is < 64K floats)
    auto stg = [&](int s, int arr, int row) -> float * { return stage + ((s * NA + arr) * TP + row) * nx; };
    auto xrow = [&](int s, int arr, int row) -> float * { return xps + ((s * 4 + arr) * TP + row) * XW; };
    auto esp = [&](int b, int c, int row) -> float * { return es + ((b * 3 + c) * TP + row) * nx; };
    auto hlw = [&](int s, int c) -> float * { return hlow + (s * 2 + c) * nx; };
    const int n = tl.k1 - tl.k0;                     // owned planes; iterations 0..n
    const float dx = a.dx, div = 1.0f / dx, hb = a.hb;
    // z-slab planes (block-uniform); with the y-slab rows (per thread, and
    // warp-uniform but for the warps that hold a band's last rows) they are
    // where a cell carries y or z auxiliaries: elsewhere interior quads run
    // the plain updates, with no auxiliary state; the general CPML expression
    // computes the same values there (kappa 1, no auxiliaries).
    auto z_plane = [&](int k) { return CPML && (k < L || k >= nz - L); };

    if (!xw) {
        // ---- interior quads (every quad of a grid without CPML); r = TP: idle
        const int r = tid < TP * ro.QI ? tid / ro.QI : TP;
        const int q = r < TP ? ro.QL + (tid - r * ro.QI) : 0;
        const bool act = r <= R;                     // owned row (r < R) or the halo row (r == R)
        const bool own = r < R;
        const int j = tl.j0 + r, i0 = 4 * q;
        const sidx_t ij0 = (sidx_t)i0 + (sidx_t)nx * (sidx_t)j;
        const bool row_upd = j >= 1 && j <= ny - 2;  // false only for a halo row on the shell
        const bool y_row = CPML && (j < L || j >= ny - L);
        auto yz_plane = [&](int k) { return y_row || z_plane(k); };
        // copies of iteration `it` (plane k0 + it) into stage (it + S) % S, one
        // group per call; `h_only`: just H (iteration -1, plane k0 - 1)
        auto issue = [&](int it, bool h_only) {
            if (it <= n && act) {
                const int s = (it + S) % S;
                const sidx_t g = ij0 + nxy * (sidx_t)(tl.k0 + it);
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    cp_async16(stg(s, c, r) + i0, a.f_in[3 + c] + g);
                    if (!h_only) {
                        cp_async16(stg(s, 3 + c, r) + i0, a.f_in[c] + g);
                        cp_async16(stg(s, 6 + c, r) + i0, a.cb[c] + g);
                        if (LOSSY) cp_async16(stg(s, 9 + c, r) + i0, a.ca[c] + g);
                    }
                }
                if (r == 0 && !h_only) {
                    cp_async16(hlw(s, 0) + i0, a.f_in[3] + g - nx);
                    cp_async16(hlw(s, 1) + i0, a.f_in[5] + g - nx);
                }
            }
            cp_async_commit_group();
        };
        issue(-1, true);
        issue(0, false);
        issue(1, false);
        // y- and z-slab auxiliaries of iteration `it`'s updates (E of plane k,
        // H of plane k-1), read from global memory one iteration ahead
        YZPsi<4> yze, yzh;
        auto load_yz = [&](int it) {
            yze.sj = yze.sk = yzh.sj = yzh.sk = -1;
            if (!CPML || it > n) return;
            const int k = tl.k0 + it;
            if (!yz_plane(k) && !yz_plane(k - 1)) return;
            if (act && row_upd && k <= nz - 2) stream_yzpsi_load<4, 0, COH>(yze, a, i0, j, k, ij0, nxy);
            if (own && it >= 1) stream_yzpsi_load<4, 2, COH>(yzh, a, i0, j, k - 1, ij0, nxy);
        };
        load_yz(0);
        XPsi<4> xnone;                               // interior quads hold no x-slab cell
#pragma unroll
        for (int e = 0; e < 4; e++) { xnone.valid[e] = false; xnone.p0[e] = xnone.p1[e] = 0.f; }

        for (int it = 0; it <= n; it++) {
            const int k = tl.k0 + it;
            const int s = it % S, sp_ = (it + S - 1) % S;      // this plane's stage, the previous plane's
            const bool e_upd = act && row_upd && k <= nz - 2;   // k >= 1 always
            const bool h_upd = own && it >= 1;
            cp_async_wait_group<1>();   // this thread's copies up to iteration it have landed
            stream_plane_barrier();     // ... and everyone's; new E of iteration it-1 visible
            // own slots of the previous plane's stage: old H (the E update's z
            // neighbours, the H update's base value); then that stage takes
            // plane it+2
            Vf<4> hxm = fillv<4>(0.f), hym = hxm, hzm = hxm;
            if (act) {
                hxm = lds4(stg(sp_, 0, r) + i0);
                hym = lds4(stg(sp_, 1, r) + i0);
                hzm = lds4(stg(sp_, 2, r) + i0);
            }
            issue(it + 2, false);

            // ---- E_new(k) of rows j0..j0+R
            Vf<4> ex = fillv<4>(0.f), ey = ex, ez = ex;
            if (act) {
                ex = lds4(stg(s, 3, r) + i0);
                ey = lds4(stg(s, 4, r) + i0);
                ez = lds4(stg(s, 5, r) + i0);
            }
            if (e_upd) {
                const Vf<4> hx = lds4(stg(s, 0, r) + i0), hy = lds4(stg(s, 1, r) + i0), hz = lds4(stg(s, 2, r) + i0);
                const Vf<4> hx_jm = lds4((r > 0 ? stg(s, 0, r - 1) : hlw(s, 0)) + i0);
                const Vf<4> hz_jm = lds4((r > 0 ? stg(s, 2, r - 1) : hlw(s, 1)) + i0);
                const float hy_im0 = q > 0 ? stg(s, 1, r)[i0 - 1] : 0.f;
                const float hz_im0 = q > 0 ? stg(s, 2, r)[i0 - 1] : 0.f;
                const Vf<4> b0 = lds4(stg(s, 6, r) + i0), b1 = lds4(stg(s, 7, r) + i0), b2 = lds4(stg(s, 8, r) + i0);
                Vf<4> c0 = fillv<4>(1.f), c1 = c0, c2 = c0;
                if (LOSSY) {
                    c0 = lds4(stg(s, 9, r) + i0);
                    c1 = lds4(stg(s, 10, r) + i0);
                    c2 = lds4(stg(s, 11, r) + i0);
                }
                const float *sp = a.src.n ? src_plane(a.src, k) : nullptr;
                if (!CPML)
                    stream_e_group<4, false, true, false, LOSSY, COH>(ex, ey, ez, hx, hy, hz, hxm, hym, hx_jm, hz_jm,
                                                                      hy_im0, hz_im0, b0, b1, b2, c0, c1, c2, xnone,
                                                                      yze, ptab, a, i0, sp, ij0, nxy, dx, div);
                else if (!yz_plane(k))
                    stream_e_group<4, false, false, false, LOSSY, COH>(ex, ey, ez, hx, hy, hz, hxm, hym, hx_jm,
                                                                       hz_jm, hy_im0, hz_im0, b0, b1, b2, c0, c1, c2,
                                                                       xnone, yze, ptab, a, i0, sp, ij0, nxy, dx,
                                                                       div);
                else
                    stream_e_group<4, false, false, true, LOSSY, COH>(ex, ey, ez, hx, hy, hz, hxm, hym, hx_jm, hz_jm,
                                                                      hy_im0, hz_im0, b0, b1, b2, c0, c1, c2, xnone,
                                                                      yze, ptab, a, i0, sp, ij0, nxy, dx, div);
            }
            if (act) {
                const int b = it & 1;
                sts4(esp(b, 0, r) + i0, ex);
                sts4(esp(b, 1, r) + i0, ey);
                sts4(esp(b, 2, r) + i0, ez);
            }
            if (own && it < n) {
                const sidx_t g = ij0 + nxy * (sidx_t)k;
                stv<4>(a.f_out[0] + g, ex);
                stv<4>(a.f_out[1] + g, ey);
                stv<4>(a.f_out[2] + g, ez);
                if (CPML && yz_plane(k)) stream_psi_store<4, 0, false>(xnone, yze, a, i0, j, k, ij0, nxy);
            }

            // ---- H_new(k-1) of rows j0..j0+R-1: own old H from the previous
            //      stage, the new E of plane k-1 from the shared array of
            //      iteration it-1 (own cells and neighbours), the new E of
            //      plane k from registers
            if (h_upd) {
                const int km = k - 1;
                const int b = (it - 1) & 1;
                const Vf<4> exm = lds4(esp(b, 0, r) + i0), eym = lds4(esp(b, 1, r) + i0), ezm = lds4(esp(b, 2, r) + i0);
                const Vf<4> ex_jp = lds4(esp(b, 0, r + 1) + i0), ez_jp = lds4(esp(b, 2, r + 1) + i0);
                const float ey_ipw = q < QX - 1 ? esp(b, 1, r)[i0 + 4] : 0.f;
                const float ez_ipw = q < QX - 1 ? esp(b, 2, r)[i0 + 4] : 0.f;
                Vf<4> nhx = hxm, nhy = hym, nhz = hzm;
                const float *sp = a.src.n ? src_plane(a.src, km) : nullptr;
                if (!CPML)
                    stream_h_group<4, false, true, false, COH>(nhx, nhy, nhz, ex, ey, exm, eym, ezm, ex_jp, ez_jp,
                                                               ey_ipw, ez_ipw, xnone, yzh, ptab, a, i0, sp, ij0, nxy,
                                                               dx, div, hb);
                else if (!yz_plane(km))
                    stream_h_group<4, false, false, false, COH>(nhx, nhy, nhz, ex, ey, exm, eym, ezm, ex_jp, ez_jp,
                                                                ey_ipw, ez_ipw, xnone, yzh, ptab, a, i0, sp, ij0, nxy,
                                                                dx, div, hb);
                else
                    stream_h_group<4, false, false, true, COH>(nhx, nhy, nhz, ex, ey, exm, eym, ezm, ex_jp, ez_jp,
                                                               ey_ipw, ez_ipw, xnone, yzh, ptab, a, i0, sp, ij0, nxy,
                                                               dx, div, hb);
                const sidx_t g = ij0 + nxy * (sidx_t)km;
                stv<4>(a.f_out[3] + g, nhx);
                stv<4>(a.f_out[4] + g, nhy);
                stv<4>(a.f_out[5] + g, nhz);
                if (CPML && yz_plane(km)) stream_psi_store<4, 2, false>(xnone, yzh, a, i0, j, km, ij0, nxy);
            }
            load_yz(it + 1);
        }
        cp_async_wait_group<0>();
        return;
    }
    if constexpr (CPML) {
        // ---- x-slab cells, one per thread; the 4 lanes of a quad are
        //      consecutive (NXC is a multiple of 4, xbase of 32) and share the
        //      quad's 16-byte copies: lane e moves staged arrays e, e+4, e+8
        //      (H0-2, E0-2, cb0-2, ca0-2 in that order), x-slab auxiliary e and,
        //      on the band's first row, Hx (lane 0) or Hz (lane 1) of row
        //      j0-1; r = TP: idle
        const int NXC = 4 * ro.NXQ;
        const int u = tid - ro.xbase;
        const int r = u < TP * NXC ? u / NXC : TP;
        const int cc = r < TP ? u - r * NXC : 0;
        const int v = cc >> 2, e4 = cc & 3;
        const int q = v < ro.QL ? v : ro.QR + (v - ro.QL);
        const int i0 = 4 * q, i = i0 + e4;
        const bool act = r <= R;
        const bool own = r < R;
        const int j = tl.j0 + r;
        const sidx_t ijq = (sidx_t)i0 + (sidx_t)nx * (sidx_t)j;   // the quad's first cell
        const sidx_t ij = ijq + (sidx_t)e4;                       // this thread's cell
        const bool row_upd = j >= 1 && j <= ny - 2;
        const bool y_row = j < L || j >= ny - L;
        auto yz_plane = [&](int k) { return y_row || z_plane(k); };
        const bool whole = xquad_whole(i0, nx, L);
        const int si = slab_local(i, nx, L);
        const bool xvalid = si >= 0 && i >= 1 && i <= nx - 2;   // x terms updated at this cell
        // the cell's x profiles (b, a, 1/kappa of E, then of H), for the tile
        float pxe[3] = {0.f, 0.f, 1.f}, pxh[3] = {0.f, 0.f, 1.f};
        if (xvalid) {
#pragma unroll
            for (int w = 0; w < 3; w++) {
                pxe[w] = __ldg(a.prof[w][0] + i);
                pxh[w] = __ldg(a.prof[3 + w][0] + i);
            }
        }
        // source array of staged array `arr` (selects, no branches: the lanes of
        // a warp take different arrays)
        auto src_of = [&](int arr) -> const float * {
            const int c = arr % 3;
            const float *p = arr < 3 ? a.f_in[3 + c] : a.f_in[c];
            if (arr >= 6) p = a.cb[c];
            if (LOSSY && arr >= 9) p = a.ca[c];
            return p;
        };
        auto issue = [&](int it, bool h_only) {
            if (it <= n && act) {
                const int s = (it + S) % S;
                const int k = tl.k0 + it;
                const sidx_t g = ijq + nxy * (sidx_t)k;
#pragma unroll
                for (int m = 0; m < 3; m++) {
                    const int arr = e4 + 4 * m;
                    if (arr < (h_only ? 3 : NA)) cp_async16(stg(s, arr, r) + i0, src_of(arr) + g);
                }
                if (!h_only) {
                    if (r == 0 && e4 < 2) cp_async16(hlw(s, e4) + i0, a.f_in[3 + 2 * e4] + g - nx);
                    const sidx_t xs0 = (sidx_t)(2 * L) * ((sidx_t)j + (sidx_t)ny * (sidx_t)k);
                    if (whole) {
                        // the quad lies in one slab and its 4 auxiliaries are 16-byte aligned
                        const int si0 = slab_local(i0, nx, L);
                        cp_async16(xrow(s, e4, r) + si0, a.psi_in[0][e4] + xs0 + si0);
                    } else if (si >= 0) {
#pragma unroll
                        for (int arr = 0; arr < 4; arr++) cp_async4(xrow(s, arr, r) + si, a.psi_in[0][arr] + xs0 + si);
                    }
                }
            }
            cp_async_commit_group();
        };
        issue(-1, true);
        issue(0, false);
        issue(1, false);
        YZPsi<1> yze, yzh;
        auto load_yz = [&](int it) {
            yze.sj = yze.sk = yzh.sj = yzh.sk = -1;
            if (it > n) return;
            const int k = tl.k0 + it;
            if (!yz_plane(k) && !yz_plane(k - 1)) return;
            if (act && row_upd && k <= nz - 2) stream_yzpsi_load<1, 0, COH>(yze, a, i, j, k, ij, nxy, ptab);
            if (own && it >= 1) stream_yzpsi_load<1, 2, COH>(yzh, a, i, j, k - 1, ij, nxy, ptab);
        };
        load_yz(0);

        for (int it = 0; it <= n; it++) {
            const int k = tl.k0 + it;
            const int s = it % S, sp_ = (it + S - 1) % S;
            const bool e_upd = act && row_upd && k <= nz - 2;
            const bool h_upd = own && it >= 1;
            cp_async_wait_group<1>();
            stream_plane_barrier();
            // own element of the previous stage: old H and H's x-slab
            // auxiliaries; every lane of the quad reads before any refills it
            Vf<1> hxm = fillv<1>(0.f), hym = hxm, hzm = hxm;
            if (act) {
                hxm.v[0] = stg(sp_, 0, r)[i];
                hym.v[0] = stg(sp_, 1, r)[i];
                hzm.v[0] = stg(sp_, 2, r)[i];
            }
            XPsi<1> xsh;
            stream_xpsi_cell(xsh, xrow(sp_, 2, r), xrow(sp_, 3, r), si, h_upd && xvalid, pxh);
            __syncwarp();
            issue(it + 2, false);

            // ---- E_new(k) of this cell
            Vf<1> ex = fillv<1>(0.f), ey = ex, ez = ex;
            if (act) {
                ex.v[0] = stg(s, 3, r)[i];
                ey.v[0] = stg(s, 4, r)[i];
                ez.v[0] = stg(s, 5, r)[i];
            }
            XPsi<1> xse;
            stream_xpsi_cell(xse, xrow(s, 0, r), xrow(s, 1, r), si, e_upd && xvalid, pxe);
            if (e_upd) {
                Vf<1> hx, hy, hz, hx_jm, hz_jm, b0, b1, b2, c0 = fillv<1>(1.f), c1 = c0, c2 = c0;
                hx.v[0] = stg(s, 0, r)[i];
                hy.v[0] = stg(s, 1, r)[i];
                hz.v[0] = stg(s, 2, r)[i];
                hx_jm.v[0] = (r > 0 ? stg(s, 0, r - 1) : hlw(s, 0))[i];
                hz_jm.v[0] = (r > 0 ? stg(s, 2, r - 1) : hlw(s, 1))[i];
                const float hy_im0 = i > 0 ? stg(s, 1, r)[i - 1] : 0.f;
                const float hz_im0 = i > 0 ? stg(s, 2, r)[i - 1] : 0.f;
                b0.v[0] = stg(s, 6, r)[i];
                b1.v[0] = stg(s, 7, r)[i];
                b2.v[0] = stg(s, 8, r)[i];
                if (LOSSY) {
                    c0.v[0] = stg(s, 9, r)[i];
                    c1.v[0] = stg(s, 10, r)[i];
                    c2.v[0] = stg(s, 11, r)[i];
                }
                const float *sp = a.src.n ? src_plane(a.src, k) : nullptr;
                stream_e_group<1, true, true, true, LOSSY, COH>(ex, ey, ez, hx, hy, hz, hxm, hym, hx_jm, hz_jm, hy_im0,
                                                                hz_im0, b0, b1, b2, c0, c1, c2, xse, yze, ptab, a, i,
                                                                sp, ij, nxy, dx, div);
            }
            if (act) {
                const int b = it & 1;
                esp(b, 0, r)[i] = ex.v[0];
                esp(b, 1, r)[i] = ey.v[0];
                esp(b, 2, r)[i] = ez.v[0];
            }
            if (own && it < n) {
                const sidx_t g = ij + nxy * (sidx_t)k;
                a.f_out[0][g] = ex.v[0];
                a.f_out[1][g] = ey.v[0];
                a.f_out[2][g] = ez.v[0];
                stream_psi_store<1, 0, true>(xse, yze, a, i, j, k, ij, nxy);
            }

            // ---- H_new(k-1) of this cell (owned rows)
            if (h_upd) {
                const int km = k - 1;
                const int b = (it - 1) & 1;
                Vf<1> exm, eym, ezm, ex_jp, ez_jp;
                exm.v[0] = esp(b, 0, r)[i];
                eym.v[0] = esp(b, 1, r)[i];
                ezm.v[0] = esp(b, 2, r)[i];
                ex_jp.v[0] = esp(b, 0, r + 1)[i];
                ez_jp.v[0] = esp(b, 2, r + 1)[i];
                const float ey_ipw = i < nx - 1 ? esp(b, 1, r)[i + 1] : 0.f;
                const float ez_ipw = i < nx - 1 ? esp(b, 2, r)[i + 1] : 0.f;
                Vf<1> nhx = hxm, nhy = hym, nhz = hzm;
                const float *sp = a.src.n ? src_plane(a.src, km) : nullptr;
                stream_h_group<1, true, true, true, COH>(nhx, nhy, nhz, ex, ey, exm, eym, ezm, ex_jp, ez_jp, ey_ipw,
                                                         ez_ipw, xsh, yzh, ptab, a, i, sp, ij, nxy, dx, div, hb);
                const sidx_t g = ij + nxy * (sidx_t)km;
                a.f_out[3][g] = nhx.v[0];
                a.f_out[4][g] = nhy.v[0];
                a.f_out[5][g] = nhz.v[0];
                stream_psi_store<1, 2, true>(xsh, yzh, a, i, j, km, ij, nxy);
            }
            load_yz(it + 1);
        }
        cp_async_wait_group<0>();
    }
}

}  // namespace fdtd
