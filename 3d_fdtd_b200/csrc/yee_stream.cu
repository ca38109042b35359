// yee_stream.cu -- FP32 Yee step in one pass: E^{n+1} and H^{n+3/2} of every
// cell in a single launch, streaming z-planes through shared memory.
//
// Why one pass.  Updating E and H in two launches reads each field set twice
// per step (the E launch reads H, the H launch reads the new E), about 84 B per
// cell against the 60 B algorithmic minimum (6 components read and written
// once, 3 E coefficients read).  Here a block keeps the new E of the plane it
// just computed on chip and updates H of the plane below from it, so every
// value crosses HBM once per step.
//
// Tiles.  The interior rows 1..ny-2 are cut into bands of at most `ty` rows
// and the interior planes 1..nz-2 into chunks; one block owns one (band, chunk)
// tile, all tiles are resident at once (one block per SM) and advance through
// z in lockstep, so the rows a band reads from its neighbours were fetched
// from HBM by the neighbour a moment earlier and are still in L2.  Band rows
// and chunk lengths are balanced on the bytes they move (CPML slabs move more).
//
// Data flow.  Fields and CPML auxiliaries ping-pong between two sets (read
// `in`, write `out`), so no block reads a value another block has already
// replaced.  A band of R rows j0..j0+R-1 runs R+1 rows of threads: row R (the
// halo row j0+R, owned by the next band) only recomputes its new E, which the
// H update of row j0+R-1 needs.  Iteration it of a tile [k0, k1) handles plane
// k = k0 + it:
//   E_new(k)   for rows j0..j0+R (stored for owned rows and planes < k1)
//   H_new(k-1) for rows j0..j0+R-1 (it >= 1)
// so it runs k1 - k0 + 1 iterations, the last one computing E_new(k1) only for
// the H update of plane k1-1.  Cells on the outer shell (index 0 or N-1 on any
// axis) are never updated, as in the reference's interior-only update
// (timefield3d.c:1679-1837); both sets hold the same shell values, and a
// recomputed row or plane on the shell passes its E through unchanged.
//
// Pipeline.  Each thread owns 4 consecutive x cells of one row and moves them
// with 16-byte cp.async copies into a ring of 3 shared-memory stages: right
// after the plane's barrier each thread reads its own slots of plane k-1's
// stage (old H, the H update's x-slab auxiliaries) into registers and issues
// plane k+2 into that stage, so planes k+1 and k+2 are in flight while plane k
// computes.  Every thread copies into its own slots only.  One block barrier per plane:
// the new E of a plane goes to a double-buffered shared array read by the next
// iteration's H update (own cells, neighbour rows and columns).  Threads of row 0 also
// stage Hx, Hz of row j0-1 (the E update's j-1 neighbours); x neighbours come
// from the same shared rows.  CPML auxiliaries and source planes are read
// straight from global memory where a cell needs them (slab cells, source
// planes).
//
// Arithmetic: exactly the per-cell expressions of the flat kernels
// (flat4_cells.cuh: same curl differences, same CPML recursion in
// cpml_curl, same coefficient forms), so results match them to the bit as
// long as the compiler contracts the same products.
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
//      The 1-D profiles are read where they are used (a few hundred floats,
//      cached).
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

template <int A0>
__device__ __forceinline__ void stream_yzpsi_load(YZPsi &s, const StreamArgs &a, int q, int j, int k, long long ij0,
                                                  long long nxy)
{
    const int nx = a.nx, L = a.L, i0 = 4 * q;
    s.sj = slab_local(j, a.ny, L);
    s.sk = slab_local(k, a.nz, L);
    s.pxy = fillv<4>(0.f); s.pzy = s.pxy; s.pxz = s.pxy; s.pyz = s.pxy;
    if (s.sj >= 0) {
        const long long sy = (long long)i0 + (long long)nx * (s.sj + 2LL * L * k);
        s.pxy = ldv<4>(a.psi_in[1][A0] + sy);
        s.pzy = ldv<4>(a.psi_in[1][A0 + 1] + sy);
    }
    if (s.sk >= 0) {
        const long long sz = ij0 + nxy * s.sk;
        s.pxz = ldv<4>(a.psi_in[2][A0] + sz);
        s.pyz = ldv<4>(a.psi_in[2][A0 + 1] + sz);
    }
}

template <int A0>
__device__ __forceinline__ void stream_psi_store(const XPsi &xs, const YZPsi &s, const StreamArgs &a, int q, int j,
                                                 int k, long long ij0, long long nxy)
{
    const int nx = a.nx, L = a.L, i0 = 4 * q;
    const long long s0 = 2LL * L * (j + (long long)a.ny * k);
#pragma unroll
    for (int e = 0; e < 4; e++) {
        if (!xs.valid[e]) continue;
        const long long sidx = s0 + slab_local(i0 + e, nx, L);
        a.psi_out[0][A0][sidx] = xs.p0[e];
        a.psi_out[0][A0 + 1][sidx] = xs.p1[e];
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
// (flat4_cells.cuh) term for term, with the profiles read here.  pw = 0 for E
// (b, a, 1/kappa of E), 3 for H.
template <int pw>
__device__ __forceinline__ Curl3 stream_cpml_curl(XPsi &xs, YZPsi &s, const StreamArgs &a, int i, int j, int k, int e,
                                                  float d_zy, float d_yz, float d_xz, float d_zx, float d_yx,
                                                  float d_xy, float dx, float div)
{
    float pyx = 0.f, pzx = 0.f, kx = 1.f;
    if (xs.valid[e]) {
        const float b = __ldg(a.prof[pw + 0][0] + i), c = __ldg(a.prof[pw + 1][0] + i);
        kx = __ldg(a.prof[pw + 2][0] + i);
        pyx = b * xs.p0[e] + c * (d_zx * div);
        pzx = b * xs.p1[e] + c * (d_yx * div);
        xs.p0[e] = pyx;
        xs.p1[e] = pzx;
    }
    float vxy = 0.f, vzy = 0.f, vxz = 0.f, vyz = 0.f, ky = 1.f, kz = 1.f;
    if (s.sj >= 0) {
        const float by = __ldg(a.prof[pw + 0][1] + j), ay = __ldg(a.prof[pw + 1][1] + j);
        ky = __ldg(a.prof[pw + 2][1] + j);
        vxy = by * s.pxy.v[e] + ay * (d_zy * div);
        vzy = by * s.pzy.v[e] + ay * (d_xy * div);
        s.pxy.v[e] = vxy;
        s.pzy.v[e] = vzy;
    }
    if (s.sk >= 0) {
        const float bz = __ldg(a.prof[pw + 0][2] + k), az = __ldg(a.prof[pw + 1][2] + k);
        kz = __ldg(a.prof[pw + 2][2] + k);
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

// 4-byte asynchronous copy (x-slab auxiliary rows when 2L is not a multiple of 4)
__device__ __forceinline__ void cp_async4(float *smem, const float *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

template <bool CPML, bool LOSSY>
__global__ void __launch_bounds__(kStreamMaxThreads, 1) k_yee_stream(StreamArgs a)
{
    // programmatic dependent launch, as the flat kernels (see k_flat4_merged)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    constexpr int S = kStreamStages;
    constexpr int NA = LOSSY ? 12 : 9;   // staged arrays: Hx Hy Hz, Ex Ey Ez, cb0..2 (, ca0..2)
    extern __shared__ __align__(16) float sm[];
    const StreamTile tl = a.tiles[blockIdx.x];
    const int nx = a.nx, ny = a.ny, nz = a.nz, QX = nx >> 2, L = a.L;
    const int TP = a.ty + 1;                         // staged rows per array
    const int XW = stream_xpsi_stride(CPML ? L : 0); // staged x-slab auxiliaries per row (2L, padded)
    const long long nxy = (long long)nx * ny;
    const int r = (int)threadIdx.x / QX, q = (int)threadIdx.x - r * QX;
    const int R = tl.rows;
    const bool act = r <= R;                         // owned row (r < R) or the halo row (r == R)
    const bool own = r < R;
    const int j = tl.j0 + r;
    const int i0 = 4 * q;
    const long long ij0 = (long long)i0 + (long long)nx * j;
    float *stage = sm;                               // [S][NA][TP][nx]
    float *xps = stage + (size_t)S * NA * TP * nx;   // [S][4][TP][XW]: x-slab auxiliaries E0 E1 H0 H1
    float *hlow = xps + (size_t)S * 4 * TP * XW;     // [S][2][nx]: Hx, Hz of row j0-1
    float *es = hlow + (size_t)S * 2 * nx;           // [2][3][TP][nx]: new E of the last two planes
    auto stg = [&](int s, int arr, int row) -> float * { return stage + ((size_t)(s * NA + arr) * TP + row) * nx; };
    auto xrow = [&](int s, int arr, int row) -> float * { return xps + ((size_t)(s * 4 + arr) * TP + row) * XW; };
    auto esp = [&](int b, int c, int row) -> float * { return es + ((size_t)(b * 3 + c) * TP + row) * nx; };
    const int n = tl.k1 - tl.k0;                     // owned planes; iterations 0..n

    // Copies of iteration `it` (plane k0 + it) into stage (it + S) % S, one
    // group per call.  Every thread copies only its own slots (row r, quad q;
    // row 0 also the j0-1 slots; the row's x-slab auxiliaries in pieces spread
    // over the row's threads), and other threads read those slots only in the
    // iteration that consumes the stage, after the barrier that follows the
    // copy.  `h_only`: just H (iteration -1, plane k0 - 1: the previous plane
    // of iteration 0).
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
            if (CPML && !h_only && (i0 < L || i0 + 3 >= nx - L)) {
                // this quad's own x-slab auxiliaries (4 arrays, one slot per element)
                const long long xs0 = 2LL * L * (j + (long long)ny * k);
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int si = slab_local(i0 + e, nx, L);
                    if (si < 0) continue;
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
    const float dx = a.dx, div = 1.0f / dx, hb = a.hb;
    const bool row_upd = j >= 1 && j <= ny - 2;      // false only for a halo row on the shell

    for (int it = 0; it <= n; it++) {
        const int k = tl.k0 + it;
        const int s = it % S, sp_ = (it + S - 1) % S;      // this plane's stage, the previous plane's
        const bool e_upd = act && row_upd && k <= nz - 2;   // k >= 1 always
        const bool h_upd = own && it >= 1;
        // y- and z-slab auxiliaries of both updates, loaded before the wait so
        // their latency overlaps it
        YZPsi yze, yzh;
        if (CPML && e_upd) stream_yzpsi_load<0>(yze, a, q, j, k, ij0, nxy);
        if (CPML && h_upd) stream_yzpsi_load<2>(yzh, a, q, j, k - 1, ij0, nxy);
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
        if (CPML && h_upd) stream_xpsi(xsh, xrow(sp_, 2, r), xrow(sp_, 3, r), nx, L, q);
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
            if (CPML) stream_xpsi(xse, xrow(s, 0, r), xrow(s, 1, r), nx, L, q);
            const Vf<4> hx = lds4(stg(s, 0, r) + i0), hy = lds4(stg(s, 1, r) + i0), hz = lds4(stg(s, 2, r) + i0);
            const Vf<4> hx_km = hxm, hy_km = hym;
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
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int i = i0 + e;
                if (i < 1 || i > nx - 2) continue;
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
                    const Curl3 c = stream_cpml_curl<0>(xse, yze, a, i, j, k, e, dHz_dy, dHy_dz, dHx_dz, dHz_dx,
                                                        dHy_dx, dHx_dy, dx, div);
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
            if (CPML) stream_psi_store<0>(xse, yze, a, q, j, k, ij0, nxy);
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
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int i = i0 + e;
                if (i < 1 || i > nx - 2) continue;
                const float ey_ip = e == 3 ? ey_ipw : eym.v[e + 1];
                const float ez_ip = e == 3 ? ez_ipw : ezm.v[e + 1];
                const float dEz_dy = ez_jp.v[e] - ezm.v[e];
                const float dEy_dz = ey.v[e] - eym.v[e];
                const float dEx_dz = ex.v[e] - exm.v[e];
                const float dEz_dx = ez_ip - ezm.v[e];
                const float dEy_dx = ey_ip - eym.v[e];
                const float dEx_dy = ex_jp.v[e] - exm.v[e];
                float cx, cy, cz;
                if (!CPML) {
                    cx = dEz_dy - dEy_dz;
                    cy = dEx_dz - dEz_dx;
                    cz = dEy_dx - dEx_dy;
                } else {
                    const Curl3 c = stream_cpml_curl<3>(xsh, yzh, a, i, j, km, e, dEz_dy, dEy_dz, dEx_dz, dEz_dx,
                                                        dEy_dx, dEx_dy, dx, div);
                    cx = c.x; cy = c.y; cz = c.z;
                }
                if (sp) {
                    cx += dx * __ldg(sp + 3 * nxy + ij0 + e);
                    cy += dx * __ldg(sp + 4 * nxy + ij0 + e);
                    cz += dx * __ldg(sp + 5 * nxy + ij0 + e);
                }
                nhx.v[e] = nhx.v[e] - hb * cx;
                nhy.v[e] = nhy.v[e] - hb * cy;
                nhz.v[e] = nhz.v[e] - hb * cz;
            }
            const long long g = ij0 + nxy * km;
            stv<4>(a.f_out[3] + g, nhx);
            stv<4>(a.f_out[4] + g, nhy);
            stv<4>(a.f_out[5] + g, nhz);
            if (CPML) stream_psi_store<2>(xsh, yzh, a, q, j, km, ij0, nxy);
        }
    }
    cp_async_wait_group<0>();
}

// ---------------------------------------------------------------------------
// host side: the tile plan
// ---------------------------------------------------------------------------
static size_t stream_smem_floats(int nx, int ty, bool lossy, int L)
{
    const int NA = lossy ? 12 : 9;
    return ((size_t)kStreamStages * NA * (ty + 1) + 2 * kStreamStages + 6 * (size_t)(ty + 1)) * nx +
           (size_t)kStreamStages * 4 * (ty + 1) * stream_xpsi_stride(L);
}

// split items 0..n-1 of cost c[] into at most `parts` contiguous runs of at
// most `maxlen` items each, minimising the largest run cost (binary search on
// that cost); returns the run starts (size = runs actually used) or empty
static std::vector<int> split_runs(const std::vector<double> &c, int parts, int maxlen)
{
    const int n = (int)c.size();
    auto greedy = [&](double cap, std::vector<int> *starts) {
        int runs = 0, len = 0;
        double acc = 0;
        for (int t = 0; t < n; t++) {
            if (len == 0 || acc + c[t] > cap || len >= maxlen) {
                if (len > 0 || runs == 0) {
                    runs++;
                    if (starts) starts->push_back(t);
                }
                acc = 0;
                len = 0;
            }
            acc += c[t];
            len++;
        }
        return runs;
    };
    double lo = 0, hi = 0;
    for (double x : c) { lo = std::max(lo, x); hi += x; }
    if (greedy(hi, nullptr) > parts) return {};   // maxlen alone needs more runs
    for (int iter = 0; iter < 60; iter++) {
        const double mid = 0.5 * (lo + hi);
        if (greedy(mid, nullptr) <= parts) hi = mid; else lo = mid;
    }
    std::vector<int> starts;
    greedy(hi, &starts);
    return starts;
}

int stream_supported(int nx, int ny, int nz, bool lossy, int L)
{
    if (nx % 4 != 0 || nx < 8 || ny < 3 || nz < 3 || L < 0) return 0;
    const int QX = nx / 4;
    if (2 * QX > kStreamMaxThreads) return 0;                      // at least one row plus its halo row
    return stream_smem_floats(nx, 1, lossy, L) * sizeof(float) <= kStreamSmemBudget;
}

bool stream_plan(int nx, int ny, int nz, int L, bool lossy, int nsm, StreamPlan *out)
{
    if (!stream_supported(nx, ny, nz, lossy, L) || nsm <= 0) return false;
    const int QX = nx / 4, rows = ny - 2, planes = nz - 2;
    int ty_max = kStreamMaxThreads / QX - 1;
    while (ty_max > 1 && stream_smem_floats(nx, ty_max, lossy, L) * sizeof(float) > kStreamSmemBudget) ty_max--;
    ty_max = std::min(ty_max, rows);
    // bytes per cell of each row / plane (60 B, plus 32 B per CPML axis)
    std::vector<double> rc(rows), pc(planes);
    for (int t = 0; t < rows; t++) {
        const int jj = 1 + t;
        const bool ys = L > 0 && (jj < L || jj >= ny - L);
        rc[t] = (60.0 + (ys ? 32.0 : 0.0)) * nx + (L > 0 ? 64.0 * L : 0.0) + 44.0 * nx / std::max(1, ty_max);
    }
    for (int t = 0; t < planes; t++) {
        const int kk = 1 + t;
        const bool zs = L > 0 && (kk < L || kk >= nz - L);
        pc[t] = 60.0 + (zs ? 32.0 : 0.0);
    }
    // band count: the smallest that keeps >= 95 % of the SMs busy with chunks
    // of at least 8 planes (shorter chunks re-read their boundary planes too often)
    const int nb_min = (rows + ty_max - 1) / ty_max;
    const int nc_max = std::max(1, planes / 8);
    int best_nb = -1, best_nc = 0;
    double best_use = -1;
    for (int nb = nb_min; nb <= std::min(rows, 4 * nb_min); nb++) {
        const int nc = std::min(nsm / nb, nc_max);
        if (nc < 1) break;
        const double use = (double)nb * nc / nsm;
        if (use > best_use + 1e-9) { best_use = use; best_nb = nb; best_nc = nc; }
        if (use >= 0.95) break;
    }
    if (best_nb < 0) { best_nb = nb_min; best_nc = 1; }
    const std::vector<int> bs = split_runs(rc, best_nb, ty_max);
    const std::vector<int> cs = split_runs(pc, best_nc, planes);
    if (bs.empty() || cs.empty()) return false;
    out->tiles.clear();
    out->ty = 0;
    for (size_t b = 0; b < bs.size(); b++) {
        const int r0 = bs[b], r1 = b + 1 < bs.size() ? bs[b + 1] : rows;
        out->ty = std::max(out->ty, r1 - r0);
        for (size_t c = 0; c < cs.size(); c++) {
            const int p0 = cs[c], p1 = c + 1 < cs.size() ? cs[c + 1] : planes;
            out->tiles.push_back(StreamTile{1 + r0, r1 - r0, 1 + p0, 1 + p1});
        }
    }
    out->threads = ((out->ty + 1) * QX + 31) / 32 * 32;
    out->smem = stream_smem_floats(nx, out->ty, lossy, L) * sizeof(float);
    return true;
}

bool stream_configure(size_t smem, int threads)
{
    if (smem > kStreamSmemBudget) return false;
    const void *fns[4] = {(const void *)k_yee_stream<false, false>, (const void *)k_yee_stream<false, true>,
                          (const void *)k_yee_stream<true, false>, (const void *)k_yee_stream<true, true>};
    for (const void *f : fns) {
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return false;
        cudaFuncAttributes at{};
        if (cudaFuncGetAttributes(&at, f) != cudaSuccess || at.maxThreadsPerBlock < threads) return false;
    }
    return true;
}

void launch_yee_stream(const StreamArgs &a, const StreamPlan &p, cudaStream_t st)
{
    note_launch(1);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)p.tiles.size());
    cfg.blockDim = dim3((unsigned)p.threads);
    cfg.dynamicSmemBytes = p.smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const bool cpml = a.L > 0, lossy = a.ca[0] != nullptr;
    if (cpml && lossy) cudaLaunchKernelEx(&cfg, k_yee_stream<true, true>, a);
    else if (cpml) cudaLaunchKernelEx(&cfg, k_yee_stream<true, false>, a);
    else if (lossy) cudaLaunchKernelEx(&cfg, k_yee_stream<false, true>, a);
    else cudaLaunchKernelEx(&cfg, k_yee_stream<false, false>, a);
}

}  // namespace fdtd

// ---------------------------------------------------------------------------
// plan inspection (host only; no device work)
// ---------------------------------------------------------------------------
extern "C" int fdtd_stream_plan(int nx, int ny, int nz, int cpml_cells, int lossy, int nsm, int *tiles, int cap,
                                int *ty, int *threads, long long *smem_bytes)
{
    using namespace fdtd;
    if (cpml_cells < 0 || nsm <= 0 || !ty || !threads || !smem_bytes) return -1;
    StreamPlan p;
    if (!stream_plan(nx, ny, nz, cpml_cells, lossy != 0, nsm, &p)) return -1;
    *ty = p.ty;
    *threads = p.threads;
    *smem_bytes = (long long)p.smem;
    if (tiles) {
        if (cap < (int)p.tiles.size()) return -1;
        for (size_t t = 0; t < p.tiles.size(); t++) {
            tiles[4 * t + 0] = p.tiles[t].j0;
            tiles[4 * t + 1] = p.tiles[t].rows;
            tiles[4 * t + 2] = p.tiles[t].k0;
            tiles[4 * t + 3] = p.tiles[t].k1;
        }
    }
    return (int)p.tiles.size();
}
