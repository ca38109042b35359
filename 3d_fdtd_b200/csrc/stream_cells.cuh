// stream_cells.cuh -- the one-pass FP32 Yee tile of the streaming kernels
// (yee_stream.cu: one grid per launch; yee_sweep.cu: many grids and steps in
// one persistent launch).  See yee_stream.cu for the design.
#pragma once

#include "flat4_cells.cuh"

namespace fdtd {

constexpr int kStreamStages = 3;
// 12 warps: up to 168 registers a thread at one block per SM (warps take
// registers in groups of 4, so 13 warps would leave only 128)
constexpr int kStreamMaxThreads = 384;

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

// ---- CPML auxiliaries of one quad for one field (E: A0 = 0, H: A0 = 2).
//      x-slab: per element, staged in shared memory with the plane (rows of
//      2L values); y- and z-slab: contiguous in x, read from global memory.
//      The 1-D profiles of the slab cells sit in a shared table filled at the
//      start of the tile (stream_profile_table): read from global memory at
//      every use they missed L1 (the staged planes leave it a few KB) and put
//      an L2 round trip on every x-slab cell's update.
struct XPsi {
    bool valid[4];
    float p0[4], p1[4];
};
struct YZPsi {
    int sj, sk;
    Vf<4> pxy, pzy, pxz, pyz;   // as YZSlab: (x,y) (z,y) (x,z) (y,z) for E, alike for H
};

// x-slab auxiliaries of the quad from a staged row pair (row0, row1: the two
// auxiliaries of this field for the cell row)
__device__ __forceinline__ void stream_xpsi(XPsi &xs, const float *row0, const float *row1, int nx, int L, int q)
{
    const int i0 = 4 * q;
    const bool any = i0 < L || i0 + 3 >= nx - L;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int i = i0 + e;
        const int si = slab_local(i, nx, L);
        xs.valid[e] = any && si >= 0 && i >= 1 && i <= nx - 2;
        xs.p0[e] = xs.valid[e] ? row0[si] : 0.f;
        xs.p1[e] = xs.valid[e] ? row1[si] : 0.f;
    }
}

// Shared profile table of a tile: [axis x, y, z][profile 0..5][2L slab-local
// cells] (profiles 0..2: b, a, 1/kappa of E; 3..5 of H; slab-local index as
// slab_local), filled by the whole block.  The caller's first barrier orders
// the fill before any read.
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
template <int A0, bool COH>
__device__ __forceinline__ void stream_yzpsi_load(YZPsi &s, const StreamArgs &a, int q, int j, int k, long long ij0,
                                                  long long nxy)
{
    const int nx = a.nx, L = a.L, i0 = 4 * q;
    s.sj = slab_local(j, a.ny, L);
    s.sk = slab_local(k, a.nz, L);
    s.pxy = fillv<4>(0.f); s.pzy = s.pxy; s.pxz = s.pxy; s.pyz = s.pxy;
    if (s.sj >= 0) {
        const long long sy = (long long)i0 + (long long)nx * (s.sj + 2LL * L * k);
        s.pxy = ldf<4, COH>(a.psi_in[1][A0] + sy);
        s.pzy = ldf<4, COH>(a.psi_in[1][A0 + 1] + sy);
    }
    if (s.sk >= 0) {
        const long long sz = ij0 + nxy * s.sk;
        s.pxz = ldf<4, COH>(a.psi_in[2][A0] + sz);
        s.pyz = ldf<4, COH>(a.psi_in[2][A0 + 1] + sz);
    }
}

// a quad wholly inside one x slab, with its auxiliaries 16-byte aligned (L
// even): moved as one vector; the elements x = 0 / nx-1 hold 0, which is their
// auxiliaries' value for good (they are never updated)
__device__ __forceinline__ bool xquad_whole(int i0, int nx, int L)
{
    return (L & 1) == 0 && (i0 + 3 < L || i0 >= nx - L);
}

template <int A0>
__device__ __forceinline__ void stream_psi_store(const XPsi &xs, const YZPsi &s, const StreamArgs &a, int q, int j,
                                                 int k, long long ij0, long long nxy, bool xquad)
{
    const int nx = a.nx, L = a.L, i0 = 4 * q;
    const long long s0 = 2LL * L * (j + (long long)a.ny * k);
    if (xquad && xquad_whole(i0, nx, L)) {
        const long long si = s0 + slab_local(i0, nx, L);
        *reinterpret_cast<float4 *>(a.psi_out[0][A0] + si) = make_float4(xs.p0[0], xs.p0[1], xs.p0[2], xs.p0[3]);
        *reinterpret_cast<float4 *>(a.psi_out[0][A0 + 1] + si) = make_float4(xs.p1[0], xs.p1[1], xs.p1[2], xs.p1[3]);
    } else if (xquad) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
            if (!xs.valid[e]) continue;
            const long long sidx = s0 + slab_local(i0 + e, nx, L);
            a.psi_out[0][A0][sidx] = xs.p0[e];
            a.psi_out[0][A0 + 1][sidx] = xs.p1[e];
        }
    }
    if (s.sj >= 0) {
        const long long sy = (long long)i0 + (long long)nx * (s.sj + 2LL * L * k);
        stv<4>(a.psi_out[1][A0] + sy, s.pxy);
        stv<4>(a.psi_out[1][A0 + 1] + sy, s.pzy);
    }
    if (s.sk >= 0) {
        const long long sz = ij0 + nxy * s.sk;
        stv<4>(a.psi_out[2][A0] + sz, s.pxz);
        stv<4>(a.psi_out[2][A0 + 1] + sz, s.pyz);
    }
}

// One cell's curl with the CPML terms: the arithmetic of cpml_curl
// (flat4_cells.cuh) term for term, with the profiles from the tile's shared
// table `pt` (stream_profile_table).  pw = 0 for E (b, a, 1/kappa of E), 3 for
// H.  X: the cell may lie in an x slab (its x terms are compiled in); without
// X the x terms are the interior's (kappa 1, no auxiliary), exactly what the
// general expression gives there.
template <bool X, int pw>
__device__ __forceinline__ Curl3 stream_cpml_curl(XPsi &xs, YZPsi &s, const float *pt, int nx, int L, int i, int e,
                                                  float d_zy, float d_yz, float d_xz, float d_zx, float d_yx,
                                                  float d_xy, float dx, float div)
{
    const int PL = 2 * L;
    float pyx = 0.f, pzx = 0.f, kx = 1.f;
    if (X && xs.valid[e]) {
        const float *px = pt + pw * PL + slab_local(i, nx, L);
        const float b = px[0], c = px[PL];
        kx = px[2 * PL];
        pyx = b * xs.p0[e] + c * (d_zx * div);
        pzx = b * xs.p1[e] + c * (d_yx * div);
        xs.p0[e] = pyx;
        xs.p1[e] = pzx;
    }
    float vxy = 0.f, vzy = 0.f, vxz = 0.f, vyz = 0.f, ky = 1.f, kz = 1.f;
    if (s.sj >= 0) {
        const float *py = pt + (6 + pw) * PL + s.sj;
        const float by = py[0], ay = py[PL];
        ky = py[2 * PL];
        vxy = by * s.pxy.v[e] + ay * (d_zy * div);
        vzy = by * s.pzy.v[e] + ay * (d_xy * div);
        s.pxy.v[e] = vxy;
        s.pzy.v[e] = vzy;
    }
    if (s.sk >= 0) {
        const float *pz = pt + (12 + pw) * PL + s.sk;
        const float bz = pz[0], az = pz[PL];
        kz = pz[2 * PL];
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

// Work roles of the block's threads.  Each thread owns 4 consecutive x cells
// (a quad) of one staged row.  On a CPML grid the quads that reach into an x
// slab (row ends) sit in warps of their own, after the interior quads, so the
// x-slab work never diverges inside an interior warp and interior warps carry
// no x-slab code at all.
struct StreamRoles {
    int QL, QR;      // x-slab quads: q < QL or q >= QR (QL = QR = 0 when there is no x slab)
    int QI, NXQ;     // interior and x-slab quads per row
    int xbase;       // first thread of the x-slab warps
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
    r.threads = (r.xbase + tp * r.NXQ + 31) / 32 * 32;
    return r;
}

// E_new of one quad.  X: x-slab quad (x terms, and the cells x = 0 / nx-1 of
// the row ends stay); EDGE: the quad may hold x = 0 / nx-1 (row ends of a grid
// without CPML).
template <bool X, bool EDGE, bool CPML, bool LOSSY, bool COH>
__device__ __forceinline__ void stream_e_quad(Vf<4> &ex, Vf<4> &ey, Vf<4> &ez, const Vf<4> &hx, const Vf<4> &hy,
                                              const Vf<4> &hz, const Vf<4> &hx_km, const Vf<4> &hy_km,
                                              const Vf<4> &hx_jm, const Vf<4> &hz_jm, float hy_im0, float hz_im0,
                                              const Vf<4> &b0, const Vf<4> &b1, const Vf<4> &b2, const Vf<4> &c0,
                                              const Vf<4> &c1, const Vf<4> &c2, XPsi &xs, YZPsi &yz,
                                              const float *pt, const StreamArgs &a, int i0, const float *sp,
                                              long long ij0, long long nxy, float dx, float div)
{
    const bool plain = !CPML || (!X && yz.sj < 0 && yz.sk < 0);
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int i = i0 + e;
        if ((X || EDGE) && (i < 1 || i > a.nx - 2)) continue;   // x = 0 and x = nx-1 stay
        const float hy_im = e == 0 ? hy_im0 : hy.v[e - 1];
        const float hz_im = e == 0 ? hz_im0 : hz.v[e - 1];
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
            const Curl3 c = stream_cpml_curl<X, 0>(xs, yz, pt, a.nx, a.L, i, e, dHz_dy, dHy_dz, dHx_dz, dHz_dx,
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

// H_new of one quad (same roles as stream_e_quad)
template <bool X, bool EDGE, bool CPML, bool COH>
__device__ __forceinline__ void stream_h_quad(Vf<4> &nhx, Vf<4> &nhy, Vf<4> &nhz, const Vf<4> &ex, const Vf<4> &ey,
                                              const Vf<4> &exm, const Vf<4> &eym, const Vf<4> &ezm,
                                              const Vf<4> &ex_jp, const Vf<4> &ez_jp, float ey_ipw, float ez_ipw,
                                              XPsi &xs, YZPsi &yz, const float *pt, const StreamArgs &a, int i0,
                                              const float *sp, long long ij0, long long nxy, float dx, float div,
                                              float hb)
{
    const bool plain = !CPML || (!X && yz.sj < 0 && yz.sk < 0);
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int i = i0 + e;
        if ((X || EDGE) && (i < 1 || i > a.nx - 2)) continue;
        const float ey_ip = e == 3 ? ey_ipw : eym.v[e + 1];
        const float ez_ip = e == 3 ? ez_ipw : ezm.v[e + 1];
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
            const Curl3 c = stream_cpml_curl<X, 3>(xs, yz, pt, a.nx, a.L, i, e, dEz_dy, dEy_dz, dEx_dz, dEz_dx,
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

// One tile (band of rows x chunk of planes) of one grid's step, by the whole
// block, with `sm` the block's dynamic shared memory (stream_smem_floats of
// the grid's nx, a.ty, loss and L).  Ends with no copy in flight.
template <bool CPML, bool LOSSY, bool COH = false>
__device__ __forceinline__ void stream_tile(const StreamArgs &a, const StreamTile tl, float *sm)
{
    constexpr int S = kStreamStages;
    constexpr int NA = LOSSY ? 12 : 9;   // staged arrays: Hx Hy Hz, Ex Ey Ez, cb0..2 (, ca0..2)
    const int nx = a.nx, ny = a.ny, nz = a.nz, L = CPML ? a.L : 0;
    const int TP = a.ty + 1;                         // staged rows per array
    const int XW = stream_xpsi_stride(L);            // staged x-slab auxiliaries per row (2L, padded)
    const long long nxy = (long long)nx * ny;
    // thread -> (staged row r, quad q); r = TP marks an idle thread
    const StreamRoles ro = stream_roles(nx, L, TP);
    const int tid = (int)threadIdx.x;
    const bool xw = CPML && tid >= ro.xbase;          // warp-uniform: xbase is a multiple of 32
    int r, q;
    if (!xw) {
        r = tid < TP * ro.QI ? tid / ro.QI : TP;
        q = r < TP ? ro.QL + (tid - r * ro.QI) : 0;
    } else {
        const int u = tid - ro.xbase;
        r = u < TP * ro.NXQ ? u / ro.NXQ : TP;
        const int v = r < TP ? u - r * ro.NXQ : 0;
        q = v < ro.QL ? v : ro.QR + (v - ro.QL);
    }
    const int R = tl.rows;
    const bool act = r <= R;                         // owned row (r < R) or the halo row (r == R)
    const bool own = r < R;
    const int j = tl.j0 + r;
    const int i0 = 4 * q;
    const int QX = nx >> 2;
    const long long ij0 = (long long)i0 + (long long)nx * j;
    float *stage = sm;                               // [S][NA][TP][nx]
    float *xps = stage + (size_t)S * NA * TP * nx;   // [S][4][TP][XW]: x-slab auxiliaries E0 E1 H0 H1
    float *hlow = xps + (size_t)S * 4 * TP * XW;     // [S][2][nx]: Hx, Hz of row j0-1
    float *es = hlow + (size_t)S * 2 * nx;           // [2][3][TP][nx]: new E of the last two planes
    float *ptab = es + (size_t)2 * 3 * TP * nx;      // CPML profiles of the slab cells (stream_profile_table)
    if (CPML) stream_profile_table(ptab, a);
    auto stg = [&](int s, int arr, int row) -> float * { return stage + ((size_t)(s * NA + arr) * TP + row) * nx; };
    auto xrow = [&](int s, int arr, int row) -> float * { return xps + ((size_t)(s * 4 + arr) * TP + row) * XW; };
    auto esp = [&](int b, int c, int row) -> float * { return es + ((size_t)(b * 3 + c) * TP + row) * nx; };
    const int n = tl.k1 - tl.k0;                     // owned planes; iterations 0..n

    // Copies of iteration `it` (plane k0 + it) into stage (it + S) % S, one
    // group per call.  Every thread copies only its own slots (row r, quad q;
    // row 0 also the j0-1 slots; an x-slab quad its elements' auxiliaries),
    // and other threads read those slots only in the iteration that consumes
    // the stage, after the barrier that follows the copy.  `h_only`: just H
    // (iteration -1, plane k0 - 1: the previous plane of iteration 0).
    auto issue = [&](int it, bool h_only) {
        if (it <= n && act) {
            const int s = (it + S) % S;
            const int k = tl.k0 + it;
            const long long g = ij0 + nxy * k;
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
                cp_async16(hlow + (size_t)(s * 2 + 0) * nx + i0, a.f_in[3] + g - nx);
                cp_async16(hlow + (size_t)(s * 2 + 1) * nx + i0, a.f_in[5] + g - nx);
            }
            if (CPML && xw && !h_only) {
                const long long xs0 = 2LL * L * (j + (long long)ny * k);
                const int si0 = slab_local(i0, nx, L);
                if (xquad_whole(i0, nx, L)) {
                    // the quad lies in one slab and its 4 auxiliaries are 16-byte aligned
#pragma unroll
                    for (int arr = 0; arr < 4; arr++) cp_async16(xrow(s, arr, r) + si0, a.psi_in[0][arr] + xs0 + si0);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const int si = slab_local(i0 + e, nx, L);
                        if (si < 0) continue;
#pragma unroll
                        for (int arr = 0; arr < 4; arr++)
                            cp_async4(xrow(s, arr, r) + si, a.psi_in[0][arr] + xs0 + si);
                    }
                }
            }
        }
        cp_async_commit_group();
    };
    issue(-1, true);
    issue(0, false);
    issue(1, false);
    const float dx = a.dx, div = 1.0f / dx, hb = a.hb;
    const bool row_upd = j >= 1 && j <= ny - 2;      // false only for a halo row on the shell
    // y- and z-slab auxiliaries of iteration `it`'s updates (E of plane k, H of
    // plane k-1), read from global memory one iteration ahead
    YZPsi yze, yzh;
    // Iterations whose planes hold no y- or z-slab cell of the tile's rows
    // (block-uniform): interior quads run the plain updates there, with no
    // auxiliary state; the general CPML expression computes the same values
    // there (kappa 1, no auxiliaries).
    const bool y_rows = CPML && (tl.j0 < L || tl.j0 + R >= ny - L);
    auto yz_plane = [&](int k) { return y_rows || (CPML && (k < L || k >= nz - L)); };
    auto load_yz = [&](int it) {
        yze.sj = yze.sk = yzh.sj = yzh.sk = -1;
        if (!CPML || it > n) return;
        const int k = tl.k0 + it;
        if (!xw && !yz_plane(k) && !yz_plane(k - 1)) return;
        if (act && row_upd && k <= nz - 2) stream_yzpsi_load<0, COH>(yze, a, q, j, k, ij0, nxy);
        if (own && it >= 1) stream_yzpsi_load<2, COH>(yzh, a, q, j, k - 1, ij0, nxy);
    };
    load_yz(0);

    for (int it = 0; it <= n; it++) {
        const int k = tl.k0 + it;
        const int s = it % S, sp_ = (it + S - 1) % S;      // this plane's stage, the previous plane's
        const bool e_upd = act && row_upd && k <= nz - 2;   // k >= 1 always
        const bool h_upd = own && it >= 1;
        cp_async_wait_group<1>();   // this thread's copies up to iteration it have landed
        __syncthreads();            // ... and everyone's; new E of iteration it-1 visible
        // own slots of the previous plane's stage: old H (the E update's z
        // neighbours, the H update's base value) and the H update's x-slab
        // auxiliaries; then that stage takes plane it+2 (other threads read
        // these slots only in iteration it-1, which every thread has left)
        Vf<4> hxm = fillv<4>(0.f), hym = hxm, hzm = hxm;
        if (act) {
            hxm = lds4(stg(sp_, 0, r) + i0);
            hym = lds4(stg(sp_, 1, r) + i0);
            hzm = lds4(stg(sp_, 2, r) + i0);
        }
        XPsi xsh;
        if (CPML && xw && h_upd) stream_xpsi(xsh, xrow(sp_, 2, r), xrow(sp_, 3, r), nx, L, q);
        issue(it + 2, false);

        // ---- E_new(k) of rows j0..j0+R
        Vf<4> ex = fillv<4>(0.f), ey = ex, ez = ex;
        if (act) {
            ex = lds4(stg(s, 3, r) + i0);
            ey = lds4(stg(s, 4, r) + i0);
            ez = lds4(stg(s, 5, r) + i0);
        }
        XPsi xse;
        if (e_upd) {
            if (CPML && xw) stream_xpsi(xse, xrow(s, 0, r), xrow(s, 1, r), nx, L, q);
            const Vf<4> hx = lds4(stg(s, 0, r) + i0), hy = lds4(stg(s, 1, r) + i0), hz = lds4(stg(s, 2, r) + i0);
            const Vf<4> hx_jm = r > 0 ? lds4(stg(s, 0, r - 1) + i0) : lds4(hlow + (size_t)(s * 2 + 0) * nx + i0);
            const Vf<4> hz_jm = r > 0 ? lds4(stg(s, 2, r - 1) + i0) : lds4(hlow + (size_t)(s * 2 + 1) * nx + i0);
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
                stream_e_quad<false, true, false, LOSSY, COH>(ex, ey, ez, hx, hy, hz, hxm, hym, hx_jm, hz_jm, hy_im0,
                                                              hz_im0, b0, b1, b2, c0, c1, c2, xse, yze, ptab, a, i0,
                                                              sp, ij0, nxy, dx, div);
            else if (xw)
                stream_e_quad<true, true, true, LOSSY, COH>(ex, ey, ez, hx, hy, hz, hxm, hym, hx_jm, hz_jm, hy_im0,
                                                            hz_im0, b0, b1, b2, c0, c1, c2, xse, yze, ptab, a, i0, sp,
                                                            ij0, nxy, dx, div);
            else if (!yz_plane(k))
                stream_e_quad<false, false, false, LOSSY, COH>(ex, ey, ez, hx, hy, hz, hxm, hym, hx_jm, hz_jm, hy_im0,
                                                               hz_im0, b0, b1, b2, c0, c1, c2, xse, yze, ptab, a, i0,
                                                               sp, ij0, nxy, dx, div);
            else
                stream_e_quad<false, false, true, LOSSY, COH>(ex, ey, ez, hx, hy, hz, hxm, hym, hx_jm, hz_jm, hy_im0,
                                                              hz_im0, b0, b1, b2, c0, c1, c2, xse, yze, ptab, a, i0,
                                                              sp, ij0, nxy, dx, div);
        }
        if (act) {
            const int b = it & 1;
            sts4(esp(b, 0, r) + i0, ex);
            sts4(esp(b, 1, r) + i0, ey);
            sts4(esp(b, 2, r) + i0, ez);
        }
        if (own && it < n) {
            const long long g = ij0 + nxy * k;
            stv<4>(a.f_out[0] + g, ex);
            stv<4>(a.f_out[1] + g, ey);
            stv<4>(a.f_out[2] + g, ez);
            if (CPML && (xw || yz_plane(k))) stream_psi_store<0>(xse, yze, a, q, j, k, ij0, nxy, xw);
        }

        // ---- H_new(k-1) of rows j0..j0+R-1: own old H and x-slab auxiliaries
        //      from the previous stage, the new E of plane k-1 from the shared
        //      array of iteration it-1 (own cells and neighbours), the new E of
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
                stream_h_quad<false, true, false, COH>(nhx, nhy, nhz, ex, ey, exm, eym, ezm, ex_jp, ez_jp, ey_ipw,
                                                       ez_ipw, xsh, yzh, ptab, a, i0, sp, ij0, nxy, dx, div, hb);
            else if (xw)
                stream_h_quad<true, true, true, COH>(nhx, nhy, nhz, ex, ey, exm, eym, ezm, ex_jp, ez_jp, ey_ipw,
                                                     ez_ipw, xsh, yzh, ptab, a, i0, sp, ij0, nxy, dx, div, hb);
            else if (!yz_plane(km))
                stream_h_quad<false, false, false, COH>(nhx, nhy, nhz, ex, ey, exm, eym, ezm, ex_jp, ez_jp, ey_ipw,
                                                        ez_ipw, xsh, yzh, ptab, a, i0, sp, ij0, nxy, dx, div, hb);
            else
                stream_h_quad<false, false, true, COH>(nhx, nhy, nhz, ex, ey, exm, eym, ezm, ex_jp, ez_jp, ey_ipw,
                                                       ez_ipw, xsh, yzh, ptab, a, i0, sp, ij0, nxy, dx, div, hb);
            const long long g = ij0 + nxy * km;
            stv<4>(a.f_out[3] + g, nhx);
            stv<4>(a.f_out[4] + g, nhy);
            stv<4>(a.f_out[5] + g, nhz);
            if (CPML && (xw || yz_plane(km))) stream_psi_store<2>(xsh, yzh, a, q, j, km, ij0, nxy, xw);
        }
        load_yz(it + 1);
    }
    cp_async_wait_group<0>();
}

}  // namespace fdtd
