// flat4_cells.cuh -- per-cell E and H updates of the flat FP32 kernels
// (W consecutive x cells per thread, loads first, CPML slab state), shared by
// the per-field launches (yee_flat4.cu) and the multi-step wavefront kernel
// (yee_wave.cu).
//
// COH selects how the field arrays are read.  Within one per-field launch no
// block writes what another block reads, so the fields go through the
// read-only (non-coherent) path.  In the wavefront kernel other blocks of the
// same launch write the fields a block reads (after an acquire on their
// completion count), so every field load is a plain coherent load there; the
// coefficients, profiles and source planes stay read-only either way.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace fdtd {

constexpr int kBlock4 = 256;

template <int W> struct Vf { float v[W]; };

template <int W> __device__ __forceinline__ Vf<W> ldv(const float *p)
{
    Vf<W> r;
    if constexpr (W == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
        r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
    } else if constexpr (W == 2) {
        const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
        r.v[0] = t.x; r.v[1] = t.y;
    } else {
        r.v[0] = __ldg(p);
    }
    return r;
}

template <int W> __device__ __forceinline__ Vf<W> ldv_rw(const float *p)
{
    Vf<W> r;
    if constexpr (W == 4) {
        const float4 t = *reinterpret_cast<const float4 *>(p);
        r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
    } else if constexpr (W == 2) {
        const float2 t = *reinterpret_cast<const float2 *>(p);
        r.v[0] = t.x; r.v[1] = t.y;
    } else {
        r.v[0] = *p;
    }
    return r;
}

// field loads: read-only path (COH false) or plain coherent loads (COH true)
template <int W, bool COH> __device__ __forceinline__ Vf<W> ldf(const float *p)
{
    if constexpr (COH) return ldv_rw<W>(p);
    else return ldv<W>(p);
}

template <bool COH> __device__ __forceinline__ float ldf1(const float *p)
{
    if constexpr (COH) return *p;
    else return __ldg(p);
}

template <int W> __device__ __forceinline__ void stv(float *p, const Vf<W> &x)
{
    if constexpr (W == 4) *reinterpret_cast<float4 *>(p) = make_float4(x.v[0], x.v[1], x.v[2], x.v[3]);
    else if constexpr (W == 2) *reinterpret_cast<float2 *>(p) = make_float2(x.v[0], x.v[1]);
    else *p = x.v[0];
}

template <int W> __device__ __forceinline__ Vf<W> fillv(float s)
{
    Vf<W> r;
#pragma unroll
    for (int e = 0; e < W; e++) r.v[e] = s;
    return r;
}

__device__ __forceinline__ const float *src_plane(const SourcePlanes &s, int k)
{
    for (int t = 0; t < s.n; t++)
        if (s.k[t] == k) return s.p[t];
    return nullptr;
}

// source plane of plane k in step `ls` of a multi-step launch: the ring entry
// of that step for the scheduled plane, else the plane table
__device__ __forceinline__ const float *step_src_plane(const FlatArgs &a, int k, int ls)
{
    if (a.ring && k == a.ring_k) return a.ring + ls * a.ring_stride;
    return a.src.n ? src_plane(a.src, k) : nullptr;
}

// x-slab state of one group: per element the CPML profile (b, a, kappa) and the
// two auxiliaries of this field; valid[e] marks interior cells inside the slab.
template <int W> struct XSlab {
    bool any;
    bool valid[W];
    float b[W], c[W], k[W], p0[W], p1[W];
    long long s0;  // auxiliary row base: element i sits at s0 + slab_local(i)
};

// A0 = 0 for E (auxiliaries 0, 1; profiles 0..2), 2 for H (auxiliaries 2, 3; profiles 3..5)
template <int W, int A0, int SLABS>
__device__ __forceinline__ void xslab_load(XSlab<W> &x, const FlatArgs &a, int g, int j, int k)
{
    const int nx = a.nx, L = a.L;
    const int i0 = W * g;
    constexpr int pw = A0 == 0 ? 0 : 3;
    x.any = (SLABS & 1) && (i0 < L || i0 + W - 1 >= nx - L);
    x.s0 = 2LL * L * (j + (long long)a.ny * k);
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = i0 + e;
        const int si = slab_local(i, nx, L);
        x.valid[e] = x.any && si >= 0 && i >= 1 && i <= nx - 2;
        x.b[e] = 0.f; x.c[e] = 0.f; x.k[e] = 1.f; x.p0[e] = 0.f; x.p1[e] = 0.f;
        if (x.valid[e]) {
            const long long s = x.s0 + si;
            x.b[e] = __ldg(a.prof[pw + 0][0] + i);
            x.c[e] = __ldg(a.prof[pw + 1][0] + i);
            x.k[e] = __ldg(a.prof[pw + 2][0] + i);
            x.p0[e] = a.psi[0][A0][s];
            x.p1[e] = a.psi[0][A0 + 1][s];
        }
    }
}

template <int W, int A0, int SLABS>
__device__ __forceinline__ void xslab_store(const XSlab<W> &x, const FlatArgs &a, int g)
{
    if constexpr ((SLABS & 1) != 0) {
        if (!x.any) return;
#pragma unroll
        for (int e = 0; e < W; e++) {
            if (!x.valid[e]) continue;
            const long long s = x.s0 + slab_local(W * g + e, a.nx, a.L);
            a.psi[0][A0][s] = x.p0[e];
            a.psi[0][A0 + 1][s] = x.p1[e];
        }
    }
}

// y- and z-slab state of one group (auxiliaries contiguous in x)
template <int W> struct YZSlab {
    int sj, sk;
    float by, ay, ky, bz, az, kz;
    Vf<W> pxy, pzy, pxz, pyz;  // E: (x,y) (z,y) (x,z) (y,z); H alike with auxiliaries 2, 3
    long long sy, sz;
};

template <int W, int A0, int SLABS>
__device__ __forceinline__ void yzslab_load(YZSlab<W> &s, const FlatArgs &a, int g, int j, int k, long long ij0,
                                            long long nxy)
{
    const int L = a.L;
    constexpr int pw = A0 == 0 ? 0 : 3;
    s.sj = (SLABS & 2) ? slab_local(j, a.ny, L) : -1;
    s.sk = (SLABS & 4) ? slab_local(k, a.nz, L) : -1;
    s.by = 1.f; s.ay = 0.f; s.ky = 1.f; s.bz = 1.f; s.az = 0.f; s.kz = 1.f;
    s.pxy = fillv<W>(0.f); s.pzy = s.pxy; s.pxz = s.pxy; s.pyz = s.pxy;
    s.sy = 0; s.sz = 0;
    if (s.sj >= 0) {
        s.by = __ldg(a.prof[pw + 0][1] + j); s.ay = __ldg(a.prof[pw + 1][1] + j); s.ky = __ldg(a.prof[pw + 2][1] + j);
        s.sy = (long long)W * g + (long long)a.nx * (s.sj + 2LL * L * k);
        s.pxy = ldv_rw<W>(a.psi[1][A0] + s.sy);
        s.pzy = ldv_rw<W>(a.psi[1][A0 + 1] + s.sy);
    }
    if (s.sk >= 0) {
        s.bz = __ldg(a.prof[pw + 0][2] + k); s.az = __ldg(a.prof[pw + 1][2] + k); s.kz = __ldg(a.prof[pw + 2][2] + k);
        s.sz = ij0 + nxy * s.sk;
        s.pxz = ldv_rw<W>(a.psi[2][A0] + s.sz);
        s.pyz = ldv_rw<W>(a.psi[2][A0 + 1] + s.sz);
    }
}

template <int W, int A0, int SLABS>
__device__ __forceinline__ void yzslab_store(const YZSlab<W> &s, const FlatArgs &a)
{
    if ((SLABS & 2) && s.sj >= 0) {
        stv<W>(a.psi[1][A0] + s.sy, s.pxy);
        stv<W>(a.psi[1][A0 + 1] + s.sy, s.pzy);
    }
    if ((SLABS & 4) && s.sk >= 0) {
        stv<W>(a.psi[2][A0] + s.sz, s.pxz);
        stv<W>(a.psi[2][A0 + 1] + s.sz, s.pyz);
    }
}

// One cell's curl with the CPML terms.  d1, d2: the two differences of the
// component (e.g. dHz/dy, dHy/dz for x); the auxiliaries update in place.
struct Curl3 { float x, y, z; };

template <int W, int SLABS>
__device__ __forceinline__ Curl3 cpml_curl(XSlab<W> &xs, YZSlab<W> &s, int e, float d_zy, float d_yz, float d_xz,
                                           float d_zx, float d_yx, float d_xy, float dx, float div)
{
    // d_ab = difference of component a along axis b
    float pyx = 0.f, pzx = 0.f;
    if ((SLABS & 1) && xs.valid[e]) {
        pyx = xs.b[e] * xs.p0[e] + xs.c[e] * (d_zx * div);
        pzx = xs.b[e] * xs.p1[e] + xs.c[e] * (d_yx * div);
        xs.p0[e] = pyx;
        xs.p1[e] = pzx;
    }
    float vxy = 0.f, vzy = 0.f, vxz = 0.f, vyz = 0.f;
    if ((SLABS & 2) && s.sj >= 0) {
        vxy = s.by * s.pxy.v[e] + s.ay * (d_zy * div);
        vzy = s.by * s.pzy.v[e] + s.ay * (d_xy * div);
        s.pxy.v[e] = vxy;
        s.pzy.v[e] = vzy;
    }
    if ((SLABS & 4) && s.sk >= 0) {
        vxz = s.bz * s.pxz.v[e] + s.az * (d_yz * div);
        vyz = s.bz * s.pyz.v[e] + s.az * (d_xz * div);
        s.pxz.v[e] = vxz;
        s.pyz.v[e] = vyz;
    }
    const float kx = (SLABS & 1) ? xs.k[e] : 1.f;
    Curl3 c;
    c.x = s.ky * d_zy - s.kz * d_yz + dx * (vxy - vxz);
    c.y = s.kz * d_xz - kx * d_zx + dx * (vyz - pyx);
    c.z = kx * d_yx - s.ky * d_xy + dx * (pzx - vzy);
    return c;
}

// slot -> (group, row) of one region kind, and the plane of blockIdx.y
template <int KIND>
__device__ __forceinline__ void locate(const Region4 &r, int ngroups, int ny, int s, int by, int &g, int &j, int &k,
                                       bool &live)
{
    k = by < r.nA ? r.kA + by : r.kB + (by - r.nA);
    live = s < r.count;
    if (KIND == 0) {
        g = s % ngroups;
        j = s / ngroups;
        live = live && j >= 1 && j <= ny - 2;
    } else if (KIND == 1) {
        const int gw = r.gR - r.gL;
        g = r.gL + s % gw;
        j = r.L + s / gw;
    } else if (KIND == 3) {
        // rows 1..L-1 then ny-L..ny-2, columns [gL, gR)
        const int gw = r.gR - r.gL;
        const int row = s / gw;
        g = r.gL + (s - row * gw);
        j = row < r.L - 1 ? 1 + row : ny - r.L + (row - (r.L - 1));
    } else {
        // rows 1..ny-2, columns [0, gL) then [gR, ngroups)
        const int w = r.gL + ngroups - r.gR;
        const int row = s / w;
        const int rr = s - row * w;
        j = 1 + row;
        g = rr < r.gL ? rr : r.gR + (rr - r.gL);
    }
}

// E update of the W cells of group g, row j, plane k (all lanes of the warp
// call it); ls: step within a multi-step launch (selects the source ring entry)
template <int W, int SLABS, bool LOSSY, bool COH = false>
__device__ __forceinline__ void e_cells(const FlatArgs &a, int g, int j, int k, bool live, int ls = 0)
{
    constexpr bool CPML = SLABS != 0;
    const int nx = a.nx, ny = a.ny;
    const int ngroups = nx / W;
    const int lane = threadIdx.x & 31;
    const long long nxy = (long long)nx * ny;
    const long long ij0 = (long long)W * g + (long long)nx * j;
    const long long q0 = ij0 + nxy * k;
    // neighbour lanes hold the adjacent group of the same row when their keys are adjacent
    const int key = live ? j * ngroups + g : -2;
    // ---- phase 1: loads
    Vf<W> hy = fillv<W>(0.f), hz = hy;
    if (live) {
        hy = ldf<W, COH>(a.f[4] + q0);
        hz = ldf<W, COH>(a.f[5] + q0);
    }
    // the i-1 neighbour of element 0 is lane-1's last element when lane-1 holds group g-1
    float hy_im0 = __shfl_up_sync(0xffffffffu, hy.v[W - 1], 1);
    float hz_im0 = __shfl_up_sync(0xffffffffu, hz.v[W - 1], 1);
    const int key_prev = __shfl_up_sync(0xffffffffu, key, 1);
    if (!live) return;
    if (lane == 0 || g == 0 || key_prev != key - 1) {
        hy_im0 = g > 0 ? ldf1<COH>(a.f[4] + q0 - 1) : 0.f;
        hz_im0 = g > 0 ? ldf1<COH>(a.f[5] + q0 - 1) : 0.f;
    }
    const Vf<W> hx = ldf<W, COH>(a.f[3] + q0);
    const Vf<W> hx_jm = ldf<W, COH>(a.f[3] + q0 - nx), hz_jm = ldf<W, COH>(a.f[5] + q0 - nx);
    const Vf<W> hx_km = ldf<W, COH>(a.f[3] + q0 - nxy), hy_km = ldf<W, COH>(a.f[4] + q0 - nxy);
    const Vf<W> b0 = ldv<W>(a.cb[0] + q0), b1 = ldv<W>(a.cb[1] + q0), b2 = ldv<W>(a.cb[2] + q0);
    Vf<W> ex = ldv_rw<W>(a.f[0] + q0), ey = ldv_rw<W>(a.f[1] + q0), ez = ldv_rw<W>(a.f[2] + q0);
    Vf<W> c0 = fillv<W>(1.f), c1 = c0, c2 = c0;
    if (LOSSY) {
        c0 = ldv<W>(a.ca[0] + q0);
        c1 = ldv<W>(a.ca[1] + q0);
        c2 = ldv<W>(a.ca[2] + q0);
    }
    // source planes are a few of the nz planes: their values load in phase 2
    const float *sp = step_src_plane(a, k, ls);
    XSlab<W> xs;
    YZSlab<W> ys;
    if (CPML) {
        yzslab_load<W, 0, SLABS>(ys, a, g, j, k, ij0, nxy);
        xslab_load<W, 0, SLABS>(xs, a, g, j, k);
    }
    // ---- phase 2: arithmetic
    const float dx = a.dx, div = 1.0f / dx;
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = W * g + e;
        if (i < 1 || i > nx - 2) continue;  // x = 0 and x = nx-1 stay
        const float hy_im = e == 0 ? hy_im0 : hy.v[e - 1];
        const float hz_im = e == 0 ? hz_im0 : hz.v[e - 1];
        const float dHz_dy = hz.v[e] - hz_jm.v[e];
        const float dHy_dz = hy.v[e] - hy_km.v[e];
        const float dHx_dz = hx.v[e] - hx_km.v[e];
        const float dHz_dx = hz.v[e] - hz_im;
        const float dHy_dx = hy.v[e] - hy_im;
        const float dHx_dy = hx.v[e] - hx_jm.v[e];
        float cx, cy, cz;
        if (!CPML) {
            cx = dHz_dy - dHy_dz;
            cy = dHx_dz - dHz_dx;
            cz = dHy_dx - dHx_dy;
        } else {
            const Curl3 c = cpml_curl<W, SLABS>(xs, ys, e, dHz_dy, dHy_dz, dHx_dz, dHz_dx, dHy_dx, dHx_dy, dx, div);
            cx = c.x; cy = c.y; cz = c.z;
        }
        if (sp) {
            cx -= dx * __ldg(sp + ij0 + e);
            cy -= dx * __ldg(sp + nxy + ij0 + e);
            cz -= dx * __ldg(sp + 2 * nxy + ij0 + e);
        }
        ex.v[e] = c0.v[e] * ex.v[e] + b0.v[e] * cx;
        ey.v[e] = c1.v[e] * ey.v[e] + b1.v[e] * cy;
        ez.v[e] = c2.v[e] * ez.v[e] + b2.v[e] * cz;
    }
    // ---- phase 3: stores
    stv<W>(a.f[0] + q0, ex);
    stv<W>(a.f[1] + q0, ey);
    stv<W>(a.f[2] + q0, ez);
    if (CPML) {
        yzslab_store<W, 0, SLABS>(ys, a);
        xslab_store<W, 0, SLABS>(xs, a, g);
    }
}

// H update of the W cells of group g, row j, plane k (all lanes of the warp call it)
template <int W, int SLABS, bool COH = false>
__device__ __forceinline__ void h_cells(const FlatArgs &a, int g, int j, int k, bool live, int ls = 0)
{
    constexpr bool CPML = SLABS != 0;
    const int nx = a.nx, ny = a.ny;
    const int ngroups = nx / W;
    const int lane = threadIdx.x & 31;
    const long long nxy = (long long)nx * ny;
    const long long ij0 = (long long)W * g + (long long)nx * j;
    const long long q0 = ij0 + nxy * k;
    const int key = live ? j * ngroups + g : -2;
    // ---- phase 1: loads
    Vf<W> ey = fillv<W>(0.f), ez = ey;
    if (live) {
        ey = ldf<W, COH>(a.f[1] + q0);
        ez = ldf<W, COH>(a.f[2] + q0);
    }
    // the i+1 neighbour of the last element is lane+1's element 0 when lane+1 holds group g+1
    float ey_ipw = __shfl_down_sync(0xffffffffu, ey.v[0], 1);
    float ez_ipw = __shfl_down_sync(0xffffffffu, ez.v[0], 1);
    const int key_next = __shfl_down_sync(0xffffffffu, key, 1);
    if (!live) return;
    if (lane == 31 || g == ngroups - 1 || key_next != key + 1) {
        ey_ipw = g < ngroups - 1 ? ldf1<COH>(a.f[1] + q0 + W) : 0.f;
        ez_ipw = g < ngroups - 1 ? ldf1<COH>(a.f[2] + q0 + W) : 0.f;
    }
    const Vf<W> ex = ldf<W, COH>(a.f[0] + q0);
    const Vf<W> ex_jp = ldf<W, COH>(a.f[0] + q0 + nx), ez_jp = ldf<W, COH>(a.f[2] + q0 + nx);
    const Vf<W> ex_kp = ldf<W, COH>(a.f[0] + q0 + nxy), ey_kp = ldf<W, COH>(a.f[1] + q0 + nxy);
    Vf<W> hx = ldv_rw<W>(a.f[3] + q0), hy = ldv_rw<W>(a.f[4] + q0), hz = ldv_rw<W>(a.f[5] + q0);
    const float *sp = step_src_plane(a, k, ls);
    XSlab<W> xs;
    YZSlab<W> ys;
    if (CPML) {
        yzslab_load<W, 2, SLABS>(ys, a, g, j, k, ij0, nxy);
        xslab_load<W, 2, SLABS>(xs, a, g, j, k);
    }
    // ---- phase 2: arithmetic
    const float dx = a.dx, hb = a.hb, div = 1.0f / dx;
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = W * g + e;
        if (i < 1 || i > nx - 2) continue;
        const float ey_ip = e == W - 1 ? ey_ipw : ey.v[e + 1];
        const float ez_ip = e == W - 1 ? ez_ipw : ez.v[e + 1];
        const float dEz_dy = ez_jp.v[e] - ez.v[e];
        const float dEy_dz = ey_kp.v[e] - ey.v[e];
        const float dEx_dz = ex_kp.v[e] - ex.v[e];
        const float dEz_dx = ez_ip - ez.v[e];
        const float dEy_dx = ey_ip - ey.v[e];
        const float dEx_dy = ex_jp.v[e] - ex.v[e];
        float cx, cy, cz;
        if (!CPML) {
            cx = dEz_dy - dEy_dz;
            cy = dEx_dz - dEz_dx;
            cz = dEy_dx - dEx_dy;
        } else {
            const Curl3 c = cpml_curl<W, SLABS>(xs, ys, e, dEz_dy, dEy_dz, dEx_dz, dEz_dx, dEy_dx, dEx_dy, dx, div);
            cx = c.x; cy = c.y; cz = c.z;
        }
        if (sp) {
            cx += dx * __ldg(sp + 3 * nxy + ij0 + e);
            cy += dx * __ldg(sp + 4 * nxy + ij0 + e);
            cz += dx * __ldg(sp + 5 * nxy + ij0 + e);
        }
        hx.v[e] = hx.v[e] - hb * cx;
        hy.v[e] = hy.v[e] - hb * cy;
        hz.v[e] = hz.v[e] - hb * cz;
    }
    // ---- phase 3: stores
    stv<W>(a.f[3] + q0, hx);
    stv<W>(a.f[4] + q0, hy);
    stv<W>(a.f[5] + q0, hz);
    if (CPML) {
        yzslab_store<W, 2, SLABS>(ys, a);
        xslab_store<W, 2, SLABS>(xs, a, g);
    }
}


}  // namespace fdtd
