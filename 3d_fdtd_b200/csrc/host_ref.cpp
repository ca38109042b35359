// host_ref.cpp -- host-side parts of the reference call surface: material
// rasterisers, taper geometry, vertex gradients and edge updates, the
// permittivity slice writer, and the reference's phase/twiddle arithmetic.
//
// These run once per design iteration on small data, so they stay on the
// host, written from the reference's documented behaviour (file:line cited per
// function).  Rasterisers write psi.ep/mu/sig exactly as the reference does and
// flag the grid's materials for upload before its next device step.  Writes
// that would fall outside the grid (undefined behaviour in the reference) are
// skipped.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "host_ref.h"

namespace fdtd {

static inline long long cidx(const timefield3d &p, int i, int j, int k)
{
    return i + (long long)p.i * (j + (long long)p.j * k);
}

static inline bool inside(const timefield3d &p, int i, int j, int k)
{
    return i >= 0 && i < p.i && j >= 0 && j < p.j && k >= 0 && k < p.k;
}

// timefield3d.c:1356-1366
void raster_background(timefield3d psi, float ep, float mu)
{
    long long n = 3LL * psi.i * psi.j * psi.k;
    for (long long q = 0; q < n; q++) { psi.ep[q] = ep; psi.mu[q] = mu; }
}

// timefield3d.c:1368-1392: ep, mu := values for every cell with j >= bottom
void raster_top_half_plane(timefield3d psi, float ep, float mu, int bottom)
{
    int j0 = bottom < 0 ? 0 : bottom;
    for (int k = 0; k < psi.k; k++)
        for (int j = j0; j < psi.j; j++)
            for (int i = 0; i < psi.i; i++) {
                long long q = 3 * cidx(psi, i, j, k);
                psi.ep[q] = ep; psi.mu[q] = mu;
                psi.ep[q + 1] = ep; psi.mu[q + 1] = mu;
                psi.ep[q + 2] = ep; psi.mu[q + 2] = mu;
            }
}

// timefield3d.c:1394-1414
void raster_background_permittivity(timefield3d psi, float ep)
{
    long long n = 3LL * psi.i * psi.j * psi.k;
    for (long long q = 0; q < n; q++) psi.ep[q] = ep;
}
void raster_background_permeability(timefield3d psi, float mu)
{
    long long n = 3LL * psi.i * psi.j * psi.k;
    for (long long q = 0; q < n; q++) psi.mu[q] = mu;
}

// timefield3d.c:1416-1446: components 0..2 (electric) or 3..5 (magnetic) of sig
void raster_background_conductivity(timefield3d psi, float sig, int magnetic)
{
    long long n = (long long)psi.i * psi.j * psi.k;
    int o = magnetic ? 3 : 0;
    for (long long q = 0; q < n; q++) { psi.sig[6 * q + o] = sig; psi.sig[6 * q + o + 1] = sig; psi.sig[6 * q + o + 2] = sig; }
}

// timefield3d.c:1457-1474 and 1476-1495: half-open box [start, end) per axis
void raster_prism(timefield3d psi, float v, int sx, int ex, int sy, int ey, int sz, int ez, int what)
{
    int i0 = sx < 0 ? 0 : sx, i1 = ex > psi.i ? psi.i : ex;
    int j0 = sy < 0 ? 0 : sy, j1 = ey > psi.j ? psi.j : ey;
    int k0 = sz < 0 ? 0 : sz, k1 = ez > psi.k ? psi.k : ez;
    for (int k = k0; k < k1; k++)
        for (int j = j0; j < j1; j++)
            for (int i = i0; i < i1; i++) {
                long long c = cidx(psi, i, j, k);
                if (what == 0) { psi.ep[3 * c] = v; psi.ep[3 * c + 1] = v; psi.ep[3 * c + 2] = v; }
                else { psi.sig[6 * c] = v; psi.sig[6 * c + 1] = v; psi.sig[6 * c + 2] = v; }
            }
}

// timefield3d.c:1511-1535: for z in [start_z, end_z), x from
// start_left + round(ls (z - start_z)) up to (excluding)
// start_right + round(rs (z - start_z)), y in [bottom, top).
void raster_taper(timefield3d psi, double ep, double mu, int start_left, int start_right, int end_left,
                  int end_right, int start_z, int end_z, int bottom, int top)
{
    double right_slope = (double)(end_right - start_right) / ((double)(end_z - start_z));
    double left_slope = (double)(end_left - start_left) / ((double)(end_z - start_z));
    for (int j = bottom; j < top; j++)
        for (int k = start_z; k < end_z; k++) {
            int i0 = (int)(start_left + std::round(left_slope * (k - start_z)));
            double i1 = start_right + std::round(right_slope * (k - start_z));
            for (int i = i0; i < i1; i++) {
                if (!inside(psi, i, j, k)) continue;
                long long q = 3 * cidx(psi, i, j, k);
                psi.ep[q] = (float)ep; psi.mu[q] = (float)mu;
                psi.ep[q + 1] = (float)ep; psi.mu[q + 1] = (float)mu;
                psi.ep[q + 2] = (float)ep; psi.mu[q + 2] = (float)mu;
            }
        }
}

// adjoint3d.c:243-257
void taper_insert(timefield3d psi, const adjoint3d_taper &t)
{
    int length = t.end - t.start;
    for (int n = 0; n < t.seg_num; n++) {
        int seg_start = t.start + (n * length) / t.seg_num;
        int seg_end = t.start + ((n + 1) * length) / t.seg_num;
        raster_taper(psi, t.ep, t.mu, t.left[n], t.right[n], t.left[n + 1], t.right[n + 1], seg_start, seg_end,
                     t.bottom, t.top);
    }
}

// adjoint3d.c:375-418: hat-weighted sum of the ep-gradient over the two
// segments adjacent to each interior vertex; right edge +, left edge -.
void taper_vertex_gradients(const adjoint3d_taper &t, double ep_diff)
{
    int length = t.end - t.start, height = t.top - t.bottom;
    t.left_grad[0] = 0;
    t.right_grad[0] = 0;
    for (int n = 1; n < t.seg_num; n++) {
        t.left_grad[n] = 0;
        t.right_grad[n] = 0;
        int seg_bck = ((n - 1) * length) / t.seg_num;
        int seg_mid = (n * length) / t.seg_num;
        int seg_fwd = ((n + 1) * length) / t.seg_num;
        for (int k = seg_bck; k < seg_mid; k++)
            for (int j = 0; j < height; j++) {
                double w = (double)(k - seg_bck) / (double)(seg_mid - seg_bck);
                t.right_grad[n] += w * t.ep_gradient[0 + 2 * (j + height * k)] * ep_diff;
                t.left_grad[n] -= w * t.ep_gradient[1 + 2 * (j + height * k)] * ep_diff;
            }
        for (int k = seg_mid; k < seg_fwd; k++)
            for (int j = 0; j < height; j++) {
                double w = (double)(seg_fwd - k) / (double)(seg_fwd - seg_mid);
                t.right_grad[n] += w * t.ep_gradient[0 + 2 * (j + height * k)] * ep_diff;
                t.left_grad[n] -= w * t.ep_gradient[1 + 2 * (j + height * k)] * ep_diff;
            }
    }
    t.left_grad[t.seg_num] = 0;
    t.right_grad[t.seg_num] = 0;
}

// adjoint3d.c:471-562.  Step along the normalised width gradient
// (right - left); if no interior vertex would move by >= half a pixel, zero
// the smallest component and renormalise, up to seg_num-1 times.  Returns the
// "no change" flag.
int taper_update_symmetric(const adjoint3d_taper &t, double goal, double disc, int min_width)
{
    const int S = t.seg_num;
    double *dir = (double *)malloc((S + 1) * sizeof(double));
    double mag = 0;
    auto recompute = [&]() {
        mag = 0;
        for (int i = 0; i < S + 1; i++) mag += (t.right_grad[i] - t.left_grad[i]) * (t.right_grad[i] - t.left_grad[i]);
        mag = std::sqrt(mag) * 0.5 * disc * disc;
        for (int i = 0; i < S + 1; i++) dir[i] = (t.right_grad[i] - t.left_grad[i]) * 0.5 * disc * disc / mag;
    };
    auto no_change = [&]() {
        int flag = 1;
        for (int i = 1; i < S; i++)
            if (std::fabs((goal / mag) * dir[i]) >= 0.5) flag = 0;
        return flag;
    };
    recompute();
    int flag = no_change();
    int zeroed = 0;
    while (flag == 1 && zeroed < S - 1) {
        double min_component = 1000;
        int min_index = 0;
        for (int i = 1; i < S; i++) {
            double m = std::fabs(dir[i]) * 2 * disc;
            if (m < min_component && m > 0) { min_component = m; min_index = i; }
        }
        t.right_grad[min_index] = 0;
        t.left_grad[min_index] = 0;
        recompute();
        flag = no_change();
        printf("zeroed out index %i\n", min_index);
        zeroed++;
    }
    for (int i = 1; i < S; i++) {
        t.left[i] -= (int)(std::round((goal / mag) * dir[i]));
        t.right[i] += (int)(std::round((goal / mag) * dir[i]));
        if (t.right[i] - t.left[i] < min_width) {
            t.right[i] = (t.right[i] + t.left[i] + min_width) / 2;
            t.left[i] = (t.right[i] + t.left[i] - min_width) / 2;
        }
    }
    free(dir);
    return flag;
}

// adjoint3d.c:564-664.  Independent left/right vertex steps; components are
// interleaved (right, left) per vertex and the "moves at least one pixel"
// test uses round(|step|) >= 1 over interior entries 2 .. 2*seg_num-1.
int taper_update_asymmetric(const adjoint3d_taper &t, double goal, double disc, int min_width)
{
    const int S = t.seg_num;
    double *dir = (double *)malloc(2 * (S + 1) * sizeof(double));
    double mag = 0;
    auto recompute = [&]() {
        mag = 0;
        for (int i = 0; i < S + 1; i++) {
            mag += t.right_grad[i] * t.right_grad[i];
            mag += t.left_grad[i] * t.left_grad[i];
        }
        mag = std::sqrt(mag) * 0.5 * disc * disc;
        for (int i = 0; i < S + 1; i++) {
            dir[2 * i] = t.right_grad[i] * 0.5 * disc * disc / mag;
            dir[2 * i + 1] = t.left_grad[i] * 0.5 * disc * disc / mag;
        }
    };
    auto no_change = [&]() {
        int flag = 1;
        for (int i = 2; i < 2 * S; i++)
            if (std::round(std::fabs((goal / mag) * dir[i])) >= 1) flag = 0;
        return flag;
    };
    recompute();
    int flag = no_change();
    int zeroed = 0;
    while (flag == 1 && zeroed < 2 * (S - 2)) {
        double min_component = 1e10;
        int min_index = 0;
        for (int i = 2; i < 2 * S; i++) {
            double m = std::fabs(dir[i]);
            if (m < min_component && m > 0) { min_component = m; min_index = i; }
        }
        if (min_index % 2 == 0) t.right_grad[min_index / 2] = 0;
        else t.left_grad[min_index / 2] = 0;
        recompute();
        flag = no_change();
        printf("zeroed out index %i\n", min_index);
        zeroed++;
    }
    for (int i = 1; i < S; i++) {
        t.right[i] += (int)(std::round((goal / mag) * dir[2 * i]));
        t.left[i] += (int)(std::round((goal / mag) * dir[2 * i + 1]));
        if (t.right[i] - t.left[i] < min_width) {
            t.right[i] = (t.right[i] + t.left[i] + min_width) / 2;
            t.left[i] = (t.right[i] + t.left[i] - min_width) / 2;
        }
    }
    free(dir);
    return flag;
}

// timefield3d.c:3241-3284: int width, int length, double disc, then
// width*length ints (1 where ep > (ep_min+ep_max)/2), x fastest.
int write_permittivity_y_slice(timefield3d psi, const char *filename, int left, int right, int start, int end,
                               int y_slice, double ep_min, double ep_max)
{
    int ysz = right - left, zsz = end - start;
    if (ysz < 0 || zsz < 0) return -1;
    int *map = (int *)malloc((size_t)(ysz > 0 ? ysz : 1) * (zsz > 0 ? zsz : 1) * sizeof(int));
    if (!map) return -1;
    for (int i = 0; i < ysz; i++)
        for (int j = 0; j < zsz; j++) {
            int x = i + left, z = j + start;
            int v = 0;
            if (inside(psi, x, y_slice, z)) v = psi.ep[3 * cidx(psi, x, y_slice, z)] > (ep_min + ep_max) / 2 ? 1 : 0;
            map[i + j * ysz] = v;
        }
    FILE *f = fopen(filename, "wb");
    if (!f) { free(map); return -1; }
    double d = psi.disc;
    fwrite(&ysz, sizeof(int), 1, f);
    fwrite(&zsz, sizeof(int), 1, f);
    fwrite(&d, sizeof(double), 1, f);
    fwrite(map, sizeof(int), (size_t)ysz * zsz, f);
    fclose(f);
    free(map);
    return 0;
}

// complex_exp(i x) by its power series to a 1e-30 term (complex.c:169-193)
void cexp_series(double x, double *re, double *im)
{
    double pr = 1, pi = 0, er = 0, ei = 0, fact = 1, dr = 1, di = 0;
    int n = 0;
    while (std::sqrt(dr * dr + di * di) >= 1e-30) {
        double scalar = 1.0 / fact;
        dr = scalar * pr;
        di = scalar * pi;
        er = er + scalar * pr;
        ei = ei + scalar * pi;
        n++;
        fact *= n;
        double nr = pr * 0 - pi * x, ni = pr * x + pi * 0;
        pr = nr;
        pi = ni;
    }
    *re = er;
    *im = ei;
}

// phase - (int)(phase / 2pi) 2pi with the 9-digit pi of timefield3d.c:3
double reduce_phase(double phase) { return phase - ((int)(phase / (2 * 3.141592652))) * 2 * 3.141592652; }

}  // namespace fdtd
