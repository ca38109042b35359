// capi.cu -- the exported C ABI (include/fdtd_b200.h).
//
// Reference entry points keep the reference's names, by-value structs and
// meaning (timefield3d.h, adjoint3d.h); the engine underneath keeps the state
// on the GPU.  Every entry point takes the API lock, records failures with
// set_error (never aborts) and returns.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "engine.h"
#include "host_ref.h"

using namespace fdtd;

#define LOCK std::lock_guard<std::mutex> lock_(api_mutex())

namespace {

Grid *dev_grid(const timefield3d &psi)
{
    Grid *g = grid_lookup(psi);
    if (!g) return nullptr;
    if (!grid_ensure_device(g)) return nullptr;
    return g;
}

void mark_materials(const timefield3d &psi, int mask)
{
    Grid *g = grid_lookup(psi, true);
    if (g) {
        g->mat_dirty |= mask;
        g->version++;
    }
}

template <typename T> bool launch_explicit_or_zsection(Grid *g, double dt, int efield, int k_lo, int k_hi, bool expl)
{
    GridView<T> v = view<T>(g, g->cur);
    CpmlView<T> c = cpml_view<T>(g, g->cur);
    SourcePlanes s = source_table(g);
    const bool cpml = !expl && g->boundary == FDTD_BOUNDARY_CPML;
    if (efield) launch_update_E<T>(v, c, s, (T)dt, (T)(1 / (g->dx)), k_lo, k_hi, expl || g->sig_e, cpml, expl, g->st);
    else launch_update_H<T>(v, c, s, (T)dt, (T)(1 / (g->dx)), k_lo, k_hi, expl || g->sig_m, true, cpml, expl, g->st);
    return cuda_ok(cudaGetLastError(), "interior update");
}

bool interior(Grid *g, double dt, int efield, int k_lo, int k_hi, bool expl)
{
    if (!grid_prepare_step(g, dt)) return false;
    if (g->cur != 0 && g->f[1][0] == nullptr) g->cur = 0;
    return g->prec == FDTD_F64 ? launch_explicit_or_zsection<double>(g, dt, efield, k_lo, k_hi, expl)
                               : launch_explicit_or_zsection<float>(g, dt, efield, k_lo, k_hi, expl);
}

bool ensure_old(Grid *g)
{
    size_t bytes = (size_t)g->n * (g->prec == FDTD_F64 ? 8 : 4);
    for (int m = 0; m < 6; m++)
        if (!g->old[m]) {
            if (!cuda_ok(cudaMalloc(&g->old[m], bytes), "cudaMalloc(old)")) return false;
            if (!cuda_ok(cudaMemsetAsync(g->old[m], 0, bytes, g->st), "cudaMemsetAsync(old)")) return false;
        }
    return true;
}

bool mur(Grid *g, double dt, int efield, int ks, int ke)
{
    if (ks < 0 || ke > g->nz || ks >= ke || (ks == 0 && ke < 2) || (ke == g->nz && ks > g->nz - 2)) {
        set_error(FDTD_ERR_ARG, "Mur boundary z-range [%d,%d) unsupported for nz=%d", ks, ke, g->nz);
        return false;
    }
    if (!ensure_old(g)) return false;
    if (g->prec == FDTD_F64) launch_mur<double>(view<double>(g, g->cur), dt, g->dx, efield, ks, ke, g->st);
    else launch_mur<float>(view<float>(g, g->cur), (float)dt, (float)g->dx, efield, ks, ke, g->st);
    return cuda_ok(cudaGetLastError(), "Mur boundary");
}

bool save_shell(Grid *g)
{
    if (!ensure_old(g)) return false;
    if (g->prec == FDTD_F64) launch_save_shell<double>(view<double>(g, g->cur), g->st);
    else launch_save_shell<float>(view<float>(g, g->cur), g->st);
    return cuda_ok(cudaGetLastError(), "shell snapshot");
}

bool upload_old(Grid *g, const double *old_field)
{
    if (!ensure_old(g)) return false;
    size_t bytes = (size_t)g->n * 6 * sizeof(double);
    if (!g->d_aos && !cuda_ok(cudaMalloc(&g->d_aos, bytes), "cudaMalloc(staging)")) return false;
    if (!cuda_ok(cudaMemcpyAsync(g->d_aos, old_field, bytes, cudaMemcpyHostToDevice, g->st), "upload old_field"))
        return false;
    if (g->prec == FDTD_F64) launch_aos_to_soa<double>(g->d_aos, (double *const *)g->old, g->n, g->st);
    else launch_aos_to_soa<float>(g->d_aos, (float *const *)g->old, g->n, g->st);
    return cuda_ok(cudaGetLastError(), "aos_to_soa(old)");
}

const void *const *fptr(Grid *g) { return (const void *const *)g->d_fptr[g->cur]; }

bool dft(Grid *g, double phase, int slice, int k_lo, int k_hi)
{
    if (slice >= g->ny || k_lo < 0 || k_hi > g->nz) {
        set_error(FDTD_ERR_ARG, "DFT slice %d / z-range [%d,%d) outside the grid", slice, k_lo, k_hi);
        return false;
    }
    double2 *acc;
    if (slice < 0) {
        size_t bytes = (size_t)g->n * 6 * sizeof(double2);
        if (!g->d_dft_full) {
            if (!cuda_ok(cudaMalloc(&g->d_dft_full, bytes), "cudaMalloc(dft)")) return false;
            cudaMemsetAsync(g->d_dft_full, 0, bytes, g->st);
        }
        acc = g->d_dft_full;
    } else {
        auto it = g->d_dft_slice.find(slice);
        if (it == g->d_dft_slice.end()) {
            size_t bytes = (size_t)g->nx * g->nz * 6 * sizeof(double2);
            double2 *p = nullptr;
            if (!cuda_ok(cudaMalloc(&p, bytes), "cudaMalloc(dft slice)")) return false;
            cudaMemsetAsync(p, 0, bytes, g->st);
            g->d_dft_slice[slice] = p;
            acc = p;
        } else {
            acc = it->second;
        }
    }
    double tr, ti;
    cexp_series(reduce_phase(phase), &tr, &ti);
    if (g->prec == FDTD_F64) launch_dft<double>((const double *const *)fptr(g), g->nx, g->ny, g->nz, slice, k_lo, k_hi, tr, ti, acc, g->st);
    else launch_dft<float>((const float *const *)fptr(g), g->nx, g->ny, g->nz, slice, k_lo, k_hi, tr, ti, acc, g->st);
    return cuda_ok(cudaGetLastError(), "dft");
}

// fourier_fields host mirror = whole-grid accumulator + every y-slice accumulator
bool sync_fourier_host(Grid *g)
{
    if (!g->dev || (!g->d_dft_full && g->d_dft_slice.empty())) return true;
    complex *h = g->h.fourier_fields;
    g->host_mirror_written = true;
    const long long n = g->n;
    if (!cuda_ok(cudaStreamSynchronize(g->st), "sync")) return false;
    if (g->d_dft_full) {
        std::vector<double2> tmp((size_t)n * 6);
        if (!cuda_ok(cudaMemcpy(tmp.data(), g->d_dft_full, tmp.size() * sizeof(double2), cudaMemcpyDeviceToHost), "dft D2H"))
            return false;
        for (long long q = 0; q < n; q++)
            for (int m = 0; m < 6; m++) { h[6 * q + m].re = tmp[m * n + q].x; h[6 * q + m].im = tmp[m * n + q].y; }
    }
    for (auto &kv : g->d_dft_slice) {
        const int j = kv.first;
        const long long ns = (long long)g->nx * g->nz;
        std::vector<double2> tmp((size_t)ns * 6);
        if (!cuda_ok(cudaMemcpy(tmp.data(), kv.second, tmp.size() * sizeof(double2), cudaMemcpyDeviceToHost), "dft D2H"))
            return false;
        for (int k = 0; k < g->nz; k++)
            for (int i = 0; i < g->nx; i++) {
                long long q = i + (long long)g->nx * (j + (long long)g->ny * k);
                for (int m = 0; m < 6; m++) {
                    double2 v = tmp[m * ns + i + (long long)g->nx * k];
                    if (g->d_dft_full) { h[6 * q + m].re += v.x; h[6 * q + m].im += v.y; }
                    else { h[6 * q + m].re = v.x; h[6 * q + m].im = v.y; }
                }
            }
    }
    return true;
}

// headless stand-in for the reference's gnuplot plots: raw float64 slice dumps
void plot_dump(const timefield3d &psi, const char *name, int axis, int index, int kind, int comp)
{
    const char *dir = getenv("FDTD_PLOT_DIR");
    if (!dir || !*dir) return;
    Grid *g = grid_lookup(psi);
    if (!g) return;
    int dims[3] = {psi.i, psi.j, psi.k};
    if (index < 0 || index >= dims[axis]) {
        set_error(FDTD_ERR_ARG, "%s: slice %d outside the grid", name, index);
        return;
    }
    if (kind == 0 && g->dev && !grid_download_fields(g)) return;
    if (kind == 1 && !sync_fourier_host(g)) return;
    int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
    int n1 = dims[a1], n2 = dims[a2];
    int width = kind == 1 ? 2 : 1;
    std::vector<double> out((size_t)n1 * n2 * width);
    for (int v = 0; v < n2; v++)
        for (int u = 0; u < n1; u++) {
            int c[3];
            c[axis] = index; c[a1] = u; c[a2] = v;
            long long q = c[0] + (long long)psi.i * (c[1] + (long long)psi.j * c[2]);
            size_t o = ((size_t)v * n1 + u) * width;
            if (kind == 0) out[o] = psi.fields[6 * q + comp];
            else if (kind == 1) { out[o] = psi.fourier_fields[6 * q + comp].re; out[o + 1] = psi.fourier_fields[6 * q + comp].im; }
            else out[o] = psi.ep[3 * q];
        }
    char path[4096];
    snprintf(path, sizeof path, "%s/%s_%d.bin", dir, name, index);
    FILE *f = fopen(path, "wb");
    if (!f) {
        set_error(FDTD_ERR_ARG, "cannot write %s", path);
        return;
    }
    fwrite(&n1, sizeof(int), 1, f);
    fwrite(&n2, sizeof(int), 1, f);
    fwrite(out.data(), sizeof(double), out.size(), f);
    fclose(f);
}

bool check_mode_plane(Grid *g, int cz)
{
    if (cz < 0 || cz >= g->nz) {
        set_error(FDTD_ERR_ARG, "plane z=%d outside the grid (nz=%d)", cz, g->nz);
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

// ============================================================================
// lifecycle
// ============================================================================
timefield3d timefield3d_new(int i, int j, int k, double disc)
{
    LOCK;
    timefield3d t{};
    if (i <= 0 || j <= 0 || k <= 0 || !(disc > 0)) {
        set_error(FDTD_ERR_ARG, "timefield3d_new(%d, %d, %d, %g): invalid size", i, j, k, disc);
        return t;
    }
    size_t n = (size_t)i * j * k;
    t.i = i; t.j = j; t.k = k; t.disc = disc;
    t.ep = (float *)malloc(3 * n * sizeof(float));
    t.mu = (float *)malloc(3 * n * sizeof(float));
    t.sig = (float *)calloc(6 * n, sizeof(float));
    t.fields = (double *)calloc(6 * n, sizeof(double));
    t.old_fields = (double *)calloc(6 * n, sizeof(double));
    t.fourier_fields = (complex *)calloc(6 * n, sizeof(complex));
    t.sources = (float *)calloc(6 * n, sizeof(float));
    if (!t.ep || !t.mu || !t.sig || !t.fields || !t.old_fields || !t.fourier_fields || !t.sources) {
        free(t.ep); free(t.mu); free(t.sig); free(t.fields); free(t.old_fields); free(t.fourier_fields); free(t.sources);
        set_error(FDTD_ERR_ALLOC, "timefield3d_new: host allocation of %zu cells failed", n);
        return timefield3d{};
    }
    // timefield3d_new sets ep = mu = 1 (timefield3d.c:25-29)
    for (size_t q = 0; q < 3 * n; q++) { t.ep[q] = 1.0f; t.mu[q] = 1.0f; }
    grid_register(t);
    return t;
}

void timefield3d_free(timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi, true);
    if (g && g->mirrors_pinned) {
        cudaHostUnregister(psi.ep);
        cudaHostUnregister(psi.mu);
        cudaHostUnregister(psi.sig);
        cudaGetLastError();
    }
    grid_unregister(psi);
    free(psi.ep); free(psi.mu); free(psi.sig); free(psi.fields); free(psi.old_fields);
    free(psi.fourier_fields); free(psi.sources);
}

timefield3d timefield3d_copy(timefield3d psi)
{
    Grid *g;
    {
        LOCK;
        g = grid_lookup(psi);
        if (!g) return timefield3d{};
        if (g->dev && g->f[g->cur][0] && !grid_download_fields(g)) return timefield3d{};
    }
    timefield3d c = timefield3d_new(psi.i, psi.j, psi.k, psi.disc);
    if (!c.fields) return c;
    LOCK;
    size_t n = (size_t)psi.i * psi.j * psi.k;
    memcpy(c.ep, psi.ep, 3 * n * sizeof(float));
    memcpy(c.mu, psi.mu, 3 * n * sizeof(float));
    memcpy(c.sig, psi.sig, 6 * n * sizeof(float));
    memcpy(c.fields, psi.fields, 6 * n * sizeof(double));
    Grid *gc = grid_lookup(c);
    gc->prec = g->prec;
    gc->boundary = g->boundary;
    gc->L = g->L; gc->order = g->order; gc->smax = g->smax; gc->kmax = g->kmax; gc->amax = g->amax;
    gc->fields_from_host = true;
    if (g->dev && !g->planes.empty()) {
        if (!grid_ensure_device(gc)) return c;
        size_t bytes = 6 * (size_t)psi.i * psi.j * sizeof(float);
        for (auto &p : g->planes) {
            Plane *np = grid_plane(gc, p.k, true);
            if (np) cudaMemcpyAsync(np->p, p.p, bytes, cudaMemcpyDeviceToDevice, g->st);
        }
        cudaStreamSynchronize(g->st);
    }
    return c;
}

void timefield3d_zero_fields(timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return;
    grid_zero(g);
    // host mirrors: the reference zeroes them (timefield3d.c:108-121); the
    // engine's mirrors are only meaningful after a sync, so clear only what a
    // sync may have written
    size_t n = (size_t)psi.i * psi.j * psi.k;
    if (!g->dev || g->host_mirror_written) {
        memset(psi.fields, 0, 6 * n * sizeof(double));
        memset(psi.old_fields, 0, 6 * n * sizeof(double));
        memset(psi.fourier_fields, 0, 6 * n * sizeof(complex));
    }
    if (!g->dev || g->host_sources_written) memset(psi.sources, 0, 6 * n * sizeof(float));
    g->host_mirror_written = false;
    g->host_sources_written = false;
    g->fields_from_host = false;
}

double *timefield3d_get_fields(timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return nullptr;
    if (g->dev && g->f[g->cur][0] && !grid_download_fields(g)) return nullptr;
    size_t bytes = 6 * (size_t)psi.i * psi.j * psi.k * sizeof(double);
    double *out = (double *)malloc(bytes);
    if (!out) {
        set_error(FDTD_ERR_ALLOC, "timefield3d_get_fields: %zu bytes", bytes);
        return nullptr;
    }
    memcpy(out, psi.fields, bytes);
    return out;
}

double *timefield3d_get_edge_fields(timefield3d psi) { return timefield3d_get_fields(psi); }

void timefield3d_update_old_edge_fields(timefield3d psi)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g) save_shell(g);
}

// ============================================================================
// plots (headless dumps)
// ============================================================================
#define FDTD_PLOT(fn, axis, kind, comp) \
    void fn(timefield3d psi, int slice_index) { LOCK; plot_dump(psi, #fn, axis, slice_index, kind, comp); }
FDTD_PLOT(timefield3d_plot_Ex_x_slice, 0, 0, 0)
FDTD_PLOT(timefield3d_plot_Ex_y_slice, 1, 0, 0)
FDTD_PLOT(timefield3d_plot_Ex_z_slice, 2, 0, 0)
FDTD_PLOT(timefield3d_plot_Ey_x_slice, 0, 0, 1)
FDTD_PLOT(timefield3d_plot_Ey_y_slice, 1, 0, 1)
FDTD_PLOT(timefield3d_plot_Ey_z_slice, 2, 0, 1)
FDTD_PLOT(timefield3d_plot_Ez_x_slice, 0, 0, 2)
FDTD_PLOT(timefield3d_plot_Ez_y_slice, 1, 0, 2)
FDTD_PLOT(timefield3d_plot_Ez_z_slice, 2, 0, 2)
FDTD_PLOT(timefield3d_plot_Ex_x_slice_fourier, 0, 1, 0)
FDTD_PLOT(timefield3d_plot_Ex_y_slice_fourier, 1, 1, 0)
FDTD_PLOT(timefield3d_plot_Ex_z_slice_fourier, 2, 1, 0)
FDTD_PLOT(timefield3d_plot_permittivity_x_slice, 0, 2, 0)
FDTD_PLOT(timefield3d_plot_permittivity_y_slice, 1, 2, 0)
FDTD_PLOT(timefield3d_plot_permittivity_z_slice, 2, 2, 0)
#undef FDTD_PLOT

// ============================================================================
// materials (host rasterisers)
// ============================================================================
void timefield3d_set_background(timefield3d psi, float ep, float mu) { LOCK; raster_background(psi, ep, mu); mark_materials(psi, kMatEp | kMatMu); }
void timefield3d_set_top_half_plane(timefield3d psi, float ep, float mu, int bottom) { LOCK; raster_top_half_plane(psi, ep, mu, bottom); mark_materials(psi, kMatEp | kMatMu); }
void timefield3d_set_background_permittivity(timefield3d psi, float ep) { LOCK; raster_background_permittivity(psi, ep); mark_materials(psi, kMatEp); }
void timefield3d_set_background_permeability(timefield3d psi, float mu) { LOCK; raster_background_permeability(psi, mu); mark_materials(psi, kMatMu); }
void timefield3d_set_background_electric_conductivity(timefield3d psi, float sig) { LOCK; raster_background_conductivity(psi, sig, 0); mark_materials(psi, kMatSig); }
void timefield3d_set_background_magnetic_conductivity(timefield3d psi, float sig) { LOCK; raster_background_conductivity(psi, sig, 1); mark_materials(psi, kMatSig); }
void timefield3d_set_background_complex_permittivity(timefield3d psi, double omega, float real_ep, float imag_ep)
{
    // timefield3d.c:1448-1455
    LOCK;
    raster_background_permittivity(psi, real_ep);
    raster_background_conductivity(psi, (float)(omega * imag_ep), 0);
    mark_materials(psi, kMatEp | kMatSig);
}
void timefield3d_set_prism_permittivity(timefield3d psi, float ep, int sx, int ex, int sy, int ey, int sz, int ez)
{
    LOCK;
    raster_prism(psi, ep, sx, ex, sy, ey, sz, ez, 0);
    mark_materials(psi, kMatEp);
}
void timefield3d_set_prism_electric_conductivity(timefield3d psi, float sig, int sx, int ex, int sy, int ey, int sz, int ez)
{
    LOCK;
    raster_prism(psi, sig, sx, ex, sy, ey, sz, ez, 1);
    mark_materials(psi, kMatSig);
}
void timefield3d_set_prism_complex_permittivity(timefield3d psi, double omega, float real_ep, float imag_ep, int sx,
                                                int ex, int sy, int ey, int sz, int ez)
{
    // timefield3d.c:1497-1504
    LOCK;
    raster_prism(psi, real_ep, sx, ex, sy, ey, sz, ez, 0);
    raster_prism(psi, (float)(omega * imag_ep), sx, ex, sy, ey, sz, ez, 1);
    mark_materials(psi, kMatEp | kMatSig);
}
void timefield3d_set_waveguide(timefield3d psi, float ep, int start_x, int end_x, int start_z, int end_z, int bottom, int top)
{
    // timefield3d.c:1506-1509
    LOCK;
    raster_prism(psi, ep, start_x, end_x, bottom, top, start_z, end_z, 0);
    mark_materials(psi, kMatEp);
}
void timefield3d_set_taper(timefield3d psi, double ep, double mu, int start_left, int start_right, int end_left,
                           int end_right, int start_z, int end_z, int bottom, int top)
{
    LOCK;
    raster_taper(psi, ep, mu, start_left, start_right, end_left, end_right, start_z, end_z, bottom, top);
    mark_materials(psi, kMatEp | kMatMu);
}

// ============================================================================
// stepping
// ============================================================================
void timefield3d_apply_H_timestep(timefield3d psi, double delta_t)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g) interior(g, delta_t, 0, 1, g->nz - 1, true);
}
void timefield3d_apply_E_timestep(timefield3d psi, double delta_t)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g) interior(g, delta_t, 1, 1, g->nz - 1, true);
}
void timefield3d_apply_H_timestep_zsection(timefield3d psi, double delta_t, int start_index, int stop_index)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g) interior(g, delta_t, 0, start_index + 1, stop_index - 1, false);
}
void timefield3d_apply_E_timestep_zsection(timefield3d psi, double delta_t, int start_index, int stop_index)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g) interior(g, delta_t, 1, start_index + 1, stop_index - 1, false);
}
void timefield3d_apply_H_first_order_abc(timefield3d psi, double *old_field, double delta_t)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g && upload_old(g, old_field)) mur(g, delta_t, 0, 0, g->nz);
}
void timefield3d_apply_E_first_order_abc(timefield3d psi, double *old_field, double delta_t)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g && upload_old(g, old_field)) mur(g, delta_t, 1, 0, g->nz);
}
void timefield3d_apply_H_first_order_abc_zsection(timefield3d psi, double delta_t, int start_index, int stop_index)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g) mur(g, delta_t, 0, start_index, stop_index);
}
void timefield3d_apply_E_first_order_abc_zsection(timefield3d psi, double delta_t, int start_index, int stop_index)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g) mur(g, delta_t, 1, start_index, stop_index);
}

void timefield3d_apply_timestep(timefield3d psi, double delta_t)
{
    // timefield3d.c:2723-2735: shell copy, explicit E, E-ABC, explicit H, H-ABC
    LOCK;
    Grid *g = dev_grid(psi);
    if (!g) return;
    if (g->boundary != FDTD_BOUNDARY_MUR) {
        set_error(FDTD_ERR_UNSUPPORTED, "timefield3d_apply_timestep (explicit update) needs the Mur boundary");
        return;
    }
    if (!grid_prepare_step(g, delta_t)) return;
    if (save_shell(g) && interior(g, delta_t, 1, 1, g->nz - 1, true) && mur(g, delta_t, 1, 0, g->nz) &&
        interior(g, delta_t, 0, 1, g->nz - 1, true) && mur(g, delta_t, 0, 0, g->nz) && enqueue_after_step(g, delta_t))
        g->host_steps++;
}

void timefield3d_apply_timestep_omp_full(timefield3d psi, double delta_t)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (!g || !grid_prepare_step(g, delta_t)) return;
    if (enqueue_step(g, delta_t, true)) g->host_steps++;
}

// timefield3d.c:2737-2785: same update and boundary values as the _full form
void timefield3d_apply_timestep_omp(timefield3d psi, double delta_t) { timefield3d_apply_timestep_omp_full(psi, delta_t); }

// ============================================================================
// running DFT
// ============================================================================
void timefield3d_update_fourier_fields(timefield3d psi, double phase)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g) dft(g, phase, -1, 0, g->nz);
}
void timefield3d_update_fourier_fields_y_slice(timefield3d psi, double phase, int slice_index)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g && slice_index >= 0) dft(g, phase, slice_index, 0, g->nz);
}
void timefield3d_update_fourier_fields_zsection(timefield3d psi, double phase, int start_index, int stop_index)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g) dft(g, phase, -1, start_index, stop_index);
}
void timefield3d_update_fourier_fields_y_slice_zsection(timefield3d psi, double phase, int slice_index, int start_index,
                                                        int stop_index)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (g && slice_index >= 0) dft(g, phase, slice_index, start_index, stop_index);
}
void timefield3d_update_fourier_fields_omp(timefield3d psi, double phase) { timefield3d_update_fourier_fields(psi, phase); }
void timefield3d_update_fourier_fields_y_slice_omp(timefield3d psi, double phase, int slice_index)
{
    timefield3d_update_fourier_fields_y_slice(psi, phase, slice_index);
}

// ============================================================================
// sources and overlap
// ============================================================================
static void mode_source_common(timefield3d psi, int cx, int cy, int cz, const mode &m, double phase, double amplitude,
                               int reverse, int adjoint)
{
    Grid *g = dev_grid(psi);
    if (!g || !check_mode_plane(g, cz)) return;
    DevMode *dm = mode_device(m);
    if (!dm) return;
    Plane *pl = grid_plane(g, cz, true);
    if (!pl) return;
    const long long off = (long long)g->nx * g->ny * cz;
    const float *epp[3] = {g->ep[0] + off, g->ep[1] + off, g->ep[2] + off};
    const float *mup[3] = {g->mu[0] + off, g->mu[1] + off, g->mu[2] + off};
    launch_mode_source(pl->p, epp, mup, g->nx, g->ny, cx, cy, dm->d, dm->mi, dm->mj, psi.disc / m.disc, amplitude,
                       cos(phase), sin(phase), nullptr, nullptr, 0, reverse, adjoint, g->st);
    cuda_ok(cudaGetLastError(), "mode source");
}

void timefield3d_mode_source(timefield3d psi, int center_x, int center_y, int center_z, mode source_mode, double phase,
                             double amplitude, int reverse)
{
    LOCK;
    mode_source_common(psi, center_x, center_y, center_z, source_mode, phase, amplitude, reverse, 0);
}

void timefield3d_mode_source_adjoint(timefield3d psi, int center_x, int center_y, int center_z, mode source_mode,
                                     double phase, int reverse)
{
    LOCK;
    mode_source_common(psi, center_x, center_y, center_z, source_mode, phase, 0.0, reverse, 1);
}

void timefield3d_TE_gaussian_source(timefield3d, int, int, int, double, double, double, double)
{
    set_error(FDTD_ERR_UNSUPPORTED, "timefield3d_TE_gaussian_source is not provided by this engine");
}
void timefield3d_TM_gaussian_source(timefield3d, int, int, int, double, double, double, double)
{
    set_error(FDTD_ERR_UNSUPPORTED, "timefield3d_TM_gaussian_source is not provided by this engine");
}

complex timefield3d_mode_overlap(timefield3d psi, int center_x, int center_y, int center_z, mode overlap_mode,
                                 double phase, int reverse, complex *cumulative_overlap)
{
    LOCK;
    complex inst{0, 0};
    Grid *g = dev_grid(psi);
    if (!g || !check_mode_plane(g, center_z)) return inst;
    DevMode *dm = mode_device(overlap_mode);
    if (!dm) return inst;
    OverlapJob j{};
    j.cx = center_x; j.cy = center_y; j.cz = center_z;
    j.mi = dm->mi; j.mj = dm->mj;
    j.reverse = reverse == 1;
    j.ratio = psi.disc / overlap_mode.disc;
    j.mode = dm->d;
    j.inst = g->d_inst;
    j.acc = nullptr;
    j.omega = nullptr;
    j.nfreq = 0;
    j.win = mode_window(g->nx, g->ny, j.cx, j.cy, j.mi, j.mj, j.ratio);
    if (!cuda_ok(cudaMemcpyAsync(g->d_job1, &j, sizeof j, cudaMemcpyHostToDevice, g->st), "overlap job")) return inst;
    const double scale = (-0.5 * psi.disc * psi.disc);
    const long long cells = (long long)j.win.wni * j.win.wnj;
    if (g->prec == FDTD_F64)
        launch_overlap<double>((const double *const *)fptr(g), g->nx, g->ny, g->d_job1, 1, cells, g->d_partials, scale,
                               0, g->d_step, 0, g->st);
    else
        launch_overlap<float>((const float *const *)fptr(g), g->nx, g->ny, g->d_job1, 1, cells, g->d_partials, scale,
                              0, g->d_step, 0, g->st);
    if (!cuda_ok(cudaMemcpyAsync(g->h_inst, g->d_inst, sizeof(double2), cudaMemcpyDeviceToHost, g->st), "overlap D2H") ||
        !cuda_ok(cudaStreamSynchronize(g->st), "overlap sync"))
        return inst;
    inst.re = g->h_inst->x;
    inst.im = g->h_inst->y;
    // cumulative += e^{i reduced phase} * inst, as timefield3d.c:3234-3236
    if (cumulative_overlap) {
        double tr, ti;
        cexp_series(reduce_phase(phase), &tr, &ti);
        cumulative_overlap->re = cumulative_overlap->re + (tr * inst.re - ti * inst.im);
        cumulative_overlap->im = cumulative_overlap->im + (tr * inst.im + ti * inst.re);
    }
    return inst;
}

void timefield3d_file_write_permittivity_y_slice(timefield3d psi, char *filename, int left, int right, int start,
                                                 int end, int y_slice, double ep_min, double ep_max)
{
    LOCK;
    if (write_permittivity_y_slice(psi, filename, left, right, start, end, y_slice, ep_min, ep_max) != 0)
        set_error(FDTD_ERR_ARG, "cannot write permittivity slice %s", filename ? filename : "(null)");
}

// ============================================================================
// tapers
// ============================================================================
adjoint3d_taper adjoint3d_taper_new(double ep, double mu, int seg_num, int start, int end, int *left, int *right,
                                    int bottom, int top, int duration)
{
    LOCK;
    adjoint3d_taper t{};
    t.ep = ep; t.mu = mu; t.seg_num = seg_num; t.start = start; t.end = end;
    t.bottom = bottom; t.top = top; t.duration = duration;
    if (seg_num <= 0 || end <= start || top <= bottom || duration <= 0 || !left || !right) {
        set_error(FDTD_ERR_ARG, "adjoint3d_taper_new: invalid taper");
        return t;
    }
    size_t height = top - bottom, length = end - start;
    t.left = (int *)malloc((seg_num + 1) * sizeof(int));
    t.right = (int *)malloc((seg_num + 1) * sizeof(int));
    // host edge storage in the reference layout; filled only by adjoint3d_taper_sync_host
    size_t n = 6 * 2 * height * length * (size_t)duration;
    t.forward_fields = (double *)calloc(n, sizeof(double));
    t.adjoint_fields = (double *)calloc(n, sizeof(double));
    t.ep_gradient = (double *)calloc(2 * height * length, sizeof(double));
    t.left_grad = (double *)calloc(seg_num + 1, sizeof(double));
    t.right_grad = (double *)calloc(seg_num + 1, sizeof(double));
    if (!t.left || !t.right || !t.forward_fields || !t.adjoint_fields || !t.ep_gradient || !t.left_grad || !t.right_grad) {
        set_error(FDTD_ERR_ALLOC, "adjoint3d_taper_new: host allocation failed");
        return t;
    }
    for (int i = 0; i < seg_num + 1; i++) { t.left[i] = left[i]; t.right[i] = right[i]; }
    return t;
}

void adjoint3d_taper_free(adjoint3d_taper taper)
{
    LOCK;
    if (taper.left) taper_unregister(taper);
    free(taper.left); free(taper.right); free(taper.forward_fields); free(taper.adjoint_fields);
    free(taper.ep_gradient); free(taper.left_grad); free(taper.right_grad);
}

void adjoint3d_taper_insert(timefield3d psi, adjoint3d_taper taper)
{
    LOCK;
    taper_insert(psi, taper);
    mark_materials(psi, kMatEp | kMatMu);
}

static void taper_store(adjoint3d_taper taper, timefield3d psi, int timestep, int which)
{
    Grid *g = dev_grid(psi);
    if (!g) return;
    if (timestep < 0 || timestep >= taper.duration) {
        set_error(FDTD_ERR_ARG, "taper store: timestep %d outside [0, %d)", timestep, taper.duration);
        return;
    }
    TaperDev *td = taper_lookup(taper, true);
    if (!taper_prepare(td, taper, g)) return;
    enqueue_taper_store(td, g, which, timestep, nullptr, 0, 0);
}

void adjoint3d_taper_store_forward_fields(adjoint3d_taper taper, timefield3d main_fields, int timestep)
{
    LOCK;
    taper_store(taper, main_fields, timestep, 0);
}

void adjoint3d_taper_store_adjoint_fields(adjoint3d_taper taper, timefield3d main_fields, int timestep)
{
    LOCK;
    taper_store(taper, main_fields, timestep, 1);
}

void adjoint3d_taper_calculate_ep_gradient(adjoint3d_taper taper)
{
    LOCK;
    TaperDev *td = taper_lookup(taper, false);
    if (!td || !td->d_fwd) {
        set_error(FDTD_ERR_ARG, "adjoint3d_taper_calculate_ep_gradient: no stored fields for this taper");
        return;
    }
    // the stores were queued on their grids' streams; wait for all of them
    if (!cuda_ok(cudaDeviceSynchronize(), "sync")) return;
    if (td->prec == FDTD_F64)
        launch_ep_gradient<double>((const double *)td->d_fwd, (const double *)td->d_adj, td->ncell, td->duration, td->d_grad, 0);
    else
        launch_ep_gradient<float>((const float *)td->d_fwd, (const float *)td->d_adj, td->ncell, td->duration, td->d_grad, 0);
    if (!cuda_ok(cudaGetLastError(), "ep gradient")) return;
    cuda_ok(cudaMemcpy(taper.ep_gradient, td->d_grad, td->ncell * sizeof(double), cudaMemcpyDeviceToHost), "gradient D2H");
}

void adjoint3d_taper_calculate_gradients_from_ep_gradient(adjoint3d_taper taper, double ep_diff)
{
    LOCK;
    taper_vertex_gradients(taper, ep_diff);
}

int adjoint3d_taper_update_symmetric(adjoint3d_taper taper, double improvement_goal, double disc, int min_width)
{
    LOCK;
    return taper_update_symmetric(taper, improvement_goal, disc, min_width);
}

int adjoint3d_taper_update_asymmetric(adjoint3d_taper taper, double improvement_goal, double disc, int min_width)
{
    LOCK;
    return taper_update_asymmetric(taper, improvement_goal, disc, min_width);
}

// ============================================================================
// extensions
// ============================================================================
const char *fdtd_error_string(int code)
{
    switch (code) {
    case FDTD_OK: return "ok";
    case FDTD_ERR_NO_DEVICE: return "no CUDA device";
    case FDTD_ERR_CUDA: return "CUDA error";
    case FDTD_ERR_ARG: return "invalid argument";
    case FDTD_ERR_ALLOC: return "allocation failed";
    case FDTD_ERR_UNSUPPORTED: return "unsupported";
    case FDTD_ERR_TIMEOUT: return "device wait timed out";
    case FDTD_ERR_NONFINITE: return "non-finite material value";
    default: return "unknown";
    }
}

int fdtd_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

const char *fdtd_version(void) { return "fdtd_b200 0.1 (sm_100a)"; }

int timefield3d_set_precision(timefield3d psi, int precision)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    return grid_set_precision(g, precision) ? FDTD_OK : fdtd_last_error();
}

int timefield3d_set_boundary(timefield3d psi, int boundary)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (boundary < FDTD_BOUNDARY_MUR || boundary > FDTD_BOUNDARY_PEC) {
        set_error(FDTD_ERR_ARG, "boundary %d", boundary);
        return FDTD_ERR_ARG;
    }
    g->boundary = boundary;
    g->version++;
    return FDTD_OK;
}

int timefield3d_set_yee_variant(timefield3d psi, int variant)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (variant < FDTD_YEE_AUTO || variant > FDTD_YEE_STREAM) {
        set_error(FDTD_ERR_ARG, "yee variant %d", variant);
        return FDTD_ERR_ARG;
    }
    g->yee_variant = variant;
    g->pp_synced = false;   // a ping-pong design starts again from two equal sets
    g->version++;
    return FDTD_OK;
}

int timefield3d_set_wave_steps(timefield3d psi, int steps_per_launch, int steps_per_sweep, int blocks_per_ticket)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (steps_per_launch < 1 || steps_per_launch > 4096 || steps_per_sweep < 1 ||
        steps_per_sweep > steps_per_launch || blocks_per_ticket < 1 || blocks_per_ticket > 64) {
        set_error(FDTD_ERR_ARG, "wave steps %d per launch, %d per sweep, %d blocks per ticket", steps_per_launch,
                  steps_per_sweep, blocks_per_ticket);
        return FDTD_ERR_ARG;
    }
    g->wave.steps = steps_per_launch;
    g->wave.sweep = steps_per_sweep;
    g->wave.group = blocks_per_ticket;
    return FDTD_OK;
}

int timefield3d_set_cpml(timefield3d psi, int thickness, int order, double sigma_max, double kappa_max, double alpha_max)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (thickness <= 0 || order < 0 || kappa_max < 1 || alpha_max < 0 || !std::isfinite(sigma_max)) {
        set_error(FDTD_ERR_ARG, "timefield3d_set_cpml: invalid parameters");
        return FDTD_ERR_ARG;
    }
    if (2 * thickness + 2 > psi.i || 2 * thickness + 2 > psi.j || 2 * thickness + 2 > psi.k) {
        set_error(FDTD_ERR_ARG, "CPML thickness %d too large for grid %dx%dx%d", thickness, psi.i, psi.j, psi.k);
        return FDTD_ERR_ARG;
    }
    if (g->dev && thickness != g->L) {
        cudaStreamSynchronize(g->st);
        for (int s = 0; s < 2; s++)
            for (int a = 0; a < 3; a++)
                for (int w = 0; w < 4; w++)
                    if (g->psi[s][a][w]) { cudaFree(g->psi[s][a][w]); g->psi[s][a][w] = nullptr; }
    }
    g->L = thickness;
    g->order = order;
    g->smax = sigma_max;
    g->kmax = kappa_max;
    g->amax = alpha_max;
    g->prof_dt = 0;
    g->boundary = FDTD_BOUNDARY_CPML;
    g->version++;
    return FDTD_OK;
}

int timefield3d_sync_host(timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (!g->dev || !g->f[g->cur][0]) return FDTD_OK;
    if (!grid_check_device_error(g) || !grid_download_fields(g) || !sync_fourier_host(g)) return fdtd_last_error();
    return FDTD_OK;
}

int timefield3d_sync_device(timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    g->mat_dirty = kMatAll;
    g->fields_from_host = true;
    if (!grid_ensure_device(g)) return fdtd_last_error();
    // sources: every z-plane holding a non-zero host source value
    const long long nxy = (long long)psi.i * psi.j;
    std::vector<float> plane(6 * nxy);
    for (int k = 0; k < psi.k; k++) {
        bool any = false;
        for (long long t = 0; t < nxy && !any; t++)
            for (int m = 0; m < 6; m++)
                if (psi.sources[6 * (t + nxy * k) + m] != 0.0f) { any = true; break; }
        Plane *pl = grid_plane(g, k, any);
        if (!pl) continue;
        for (long long t = 0; t < nxy; t++)
            for (int m = 0; m < 6; m++) plane[m * nxy + t] = psi.sources[6 * (t + nxy * k) + m];
        if (!cuda_ok(cudaMemcpyAsync(pl->p, plane.data(), plane.size() * sizeof(float), cudaMemcpyHostToDevice, g->st),
                     "upload sources"))
            return fdtd_last_error();
    }
    return cuda_ok(cudaStreamSynchronize(g->st), "sync") ? FDTD_OK : fdtd_last_error();
}

int timefield3d_synchronize(timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (!g->dev) return FDTD_OK;
    if (!cuda_ok(cudaStreamSynchronize(g->st), "cudaStreamSynchronize")) return fdtd_last_error();
    return grid_check_device_error(g) ? FDTD_OK : fdtd_last_error();
}

int timefield3d_set_source_value(timefield3d psi, int i, int j, int k, int m, float value)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (!g) return fdtd_last_error();
    if (i < 0 || i >= psi.i || j < 0 || j >= psi.j || k < 0 || k >= psi.k || m < 0 || m > 5) {
        set_error(FDTD_ERR_ARG, "source (%d,%d,%d,%d) outside the grid", i, j, k, m);
        return FDTD_ERR_ARG;
    }
    Plane *pl = grid_plane(g, k, true);
    if (!pl) return fdtd_last_error();
    const long long nxy = (long long)psi.i * psi.j;
    launch_set_value(pl->p, m * nxy + i + (long long)psi.i * j, value, g->st);
    psi.sources[6 * (i + (long long)psi.i * (j + (long long)psi.j * k)) + m] = value;
    g->host_sources_written = true;
    return cuda_ok(cudaGetLastError(), "set source") ? FDTD_OK : fdtd_last_error();
}

double timefield3d_get_field_value(timefield3d psi, int i, int j, int k, int m)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return NAN;
    if (i < 0 || i >= psi.i || j < 0 || j >= psi.j || k < 0 || k >= psi.k || m < 0 || m > 5) {
        set_error(FDTD_ERR_ARG, "field (%d,%d,%d,%d) outside the grid", i, j, k, m);
        return NAN;
    }
    long long q = i + (long long)psi.i * (j + (long long)psi.j * k);
    if (!g->dev || !g->f[g->cur][0]) return psi.fields[6 * q + m];
    double v = 0;
    if (g->prec == FDTD_F64) {
        if (!cuda_ok(cudaMemcpyAsync(&v, (double *)g->f[g->cur][m] + q, sizeof(double), cudaMemcpyDeviceToHost, g->st), "D2H")) return NAN;
    } else {
        float f = 0;
        if (!cuda_ok(cudaMemcpyAsync(&f, (float *)g->f[g->cur][m] + q, sizeof(float), cudaMemcpyDeviceToHost, g->st), "D2H")) return NAN;
        if (!cuda_ok(cudaStreamSynchronize(g->st), "sync")) return NAN;
        return f;
    }
    if (!cuda_ok(cudaStreamSynchronize(g->st), "sync")) return NAN;
    return v;
}

int timefield3d_add_probe(timefield3d psi, int i, int j, int k, int m, int capacity)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (!g) return -1;
    if (i < 0 || i >= psi.i || j < 0 || j >= psi.j || k < 0 || k >= psi.k || m < 0 || m > 5 || capacity <= 0) {
        set_error(FDTD_ERR_ARG, "probe (%d,%d,%d,%d) capacity %d", i, j, k, m, capacity);
        return -1;
    }
    // adding a probe re-creates the probe buffers (existing samples are dropped)
    if (!cuda_ok(cudaStreamSynchronize(g->st), "sync")) return -1;
    ProbeRec r;
    r.job.q = i + (long long)psi.i * (j + (long long)psi.j * k);
    r.job.m = m;
    r.cap = capacity;
    g->probes.push_back(r);
    int cap = 0;
    for (auto &p : g->probes) cap = std::max(cap, p.cap);
    cudaFree(g->d_probes); cudaFree(g->d_probe_buf); cudaFree(g->d_probe_count);
    g->d_probes = nullptr; g->d_probe_buf = nullptr; g->d_probe_count = nullptr;
    size_t np = g->probes.size();
    std::vector<ProbeJob> jobs;
    for (auto &p : g->probes) jobs.push_back(p.job);
    if (!cuda_ok(cudaMalloc(&g->d_probes, np * sizeof(ProbeJob)), "cudaMalloc(probes)") ||
        !cuda_ok(cudaMalloc(&g->d_probe_buf, np * cap * sizeof(double)), "cudaMalloc(probe buffer)") ||
        !cuda_ok(cudaMalloc(&g->d_probe_count, np * sizeof(int)), "cudaMalloc(probe count)"))
        return -1;
    cudaMemcpy(g->d_probes, jobs.data(), np * sizeof(ProbeJob), cudaMemcpyHostToDevice);
    cudaMemset(g->d_probe_count, 0, np * sizeof(int));
    cudaMemset(g->d_probe_buf, 0, np * cap * sizeof(double));
    g->probe_cap = cap;
    g->version++;
    return cuda_ok(cudaGetLastError(), "probes") ? (int)np - 1 : -1;
}

int timefield3d_read_probe(timefield3d psi, int id, double *out, int count)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (id < 0 || id >= (int)g->probes.size() || count < 0 || !out) {
        set_error(FDTD_ERR_ARG, "probe id %d", id);
        return FDTD_ERR_ARG;
    }
    int n = std::min(count, g->probe_cap);
    if (!grid_check_device_error(g) ||
        !cuda_ok(cudaMemcpy(out, g->d_probe_buf + (size_t)id * g->probe_cap, n * sizeof(double), cudaMemcpyDeviceToHost), "probe D2H"))
        return fdtd_last_error();
    return FDTD_OK;
}

int timefield3d_clear_probes(timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (g->dev) cudaStreamSynchronize(g->st);
    cudaFree(g->d_probes); cudaFree(g->d_probe_buf); cudaFree(g->d_probe_count);
    g->d_probes = nullptr; g->d_probe_buf = nullptr; g->d_probe_count = nullptr;
    g->probes.clear();
    g->probe_cap = 0;
    g->version++;
    return FDTD_OK;
}

int timefield3d_add_overlap_monitor(timefield3d psi, int center_x, int center_y, int center_z, mode overlap_mode,
                                    int reverse, int n_freq, const double *omega)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (!g) return -1;
    if (!check_mode_plane(g, center_z)) return -1;
    if (n_freq <= 0 || !omega) {
        set_error(FDTD_ERR_ARG, "monitor needs n_freq > 0 frequencies");
        return -1;
    }
    if (!cuda_ok(cudaStreamSynchronize(g->st), "sync")) return -1;
    Monitor mn{};
    mn.cx = center_x; mn.cy = center_y; mn.cz = center_z; mn.reverse = reverse == 1; mn.nfreq = n_freq;
    mn.mode_key = priv_mode_new(overlap_mode);
    if (!mn.mode_key) return -1;
    if (!cuda_ok(cudaMalloc(&mn.d_omega, n_freq * sizeof(double)), "cudaMalloc(omega)") ||
        !cuda_ok(cudaMalloc(&mn.d_acc, 2 * n_freq * sizeof(double2)), "cudaMalloc(monitor)"))
        return -1;
    cudaMemcpy(mn.d_omega, omega, n_freq * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemset(mn.d_acc, 0, 2 * n_freq * sizeof(double2));
    g->monitors.push_back(mn);
    // grow the job / partial buffers if needed, then rebuild the job list
    if ((int)g->monitors.size() > g->jobs_cap) {
        cudaFree(g->d_jobs); cudaFree(g->d_partials);
        g->d_jobs = nullptr; g->d_partials = nullptr;
        g->jobs_cap = (int)g->monitors.size() * 2;
        int parts = overlap_parts((long long)g->nx * g->ny);
        if (!cuda_ok(cudaMalloc(&g->d_jobs, g->jobs_cap * sizeof(OverlapJob)), "cudaMalloc(jobs)") ||
            !cuda_ok(cudaMalloc(&g->d_partials, (size_t)g->jobs_cap * parts * sizeof(double2)), "cudaMalloc(partials)"))
            return -1;
    }
    if (!g->d_jobs) {
        g->jobs_cap = std::max(g->jobs_cap, 8);
        int parts = overlap_parts((long long)g->nx * g->ny);
        if (!cuda_ok(cudaMalloc(&g->d_jobs, g->jobs_cap * sizeof(OverlapJob)), "cudaMalloc(jobs)") ||
            !cuda_ok(cudaMalloc(&g->d_partials, (size_t)g->jobs_cap * parts * sizeof(double2)), "cudaMalloc(partials)"))
            return -1;
    }
    if (!rebuild_jobs(g)) return -1;
    return (int)g->monitors.size() - 1;
}

int timefield3d_read_overlap_monitor(timefield3d psi, int id, complex *out)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (id < 0 || id >= (int)g->monitors.size() || !out) {
        set_error(FDTD_ERR_ARG, "monitor id %d", id);
        return FDTD_ERR_ARG;
    }
    Monitor &mn = g->monitors[id];
    std::vector<double2> acc(2 * mn.nfreq);
    if (!grid_check_device_error(g) ||
        !cuda_ok(cudaMemcpy(acc.data(), mn.d_acc, acc.size() * sizeof(double2), cudaMemcpyDeviceToHost), "monitor D2H"))
        return fdtd_last_error();
    for (int f = 0; f < mn.nfreq; f++) {
        out[f].re = acc[2 * f].x - acc[2 * f + 1].x;
        out[f].im = acc[2 * f].y - acc[2 * f + 1].y;
    }
    return FDTD_OK;
}

int timefield3d_clear_monitors(timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (g->dev) cudaStreamSynchronize(g->st);
    for (auto &mn : g->monitors) {
        cudaFree(mn.d_omega);
        cudaFree(mn.d_acc);
        priv_mode_free(mn.mode_key);
    }
    g->monitors.clear();
    g->njobs = 0;
    g->version++;
    return FDTD_OK;
}

long long timefield3d_step_count(timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    return g ? g->host_steps : -1;
}

int timefield3d_set_source_schedule(timefield3d psi, int center_x, int center_y, int center_z, mode source_mode,
                                    int reverse, int adjoint, int nsteps, const double *amplitude, const double *phase)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (!g) return fdtd_last_error();
    if (!check_mode_plane(g, center_z)) return FDTD_ERR_ARG;
    if (nsteps <= 0 || !phase || (!adjoint && !amplitude)) {
        set_error(FDTD_ERR_ARG, "source schedule needs nsteps > 0 and phase (and amplitude) arrays");
        return FDTD_ERR_ARG;
    }
    if (!cuda_ok(cudaStreamSynchronize(g->st), "sync")) return fdtd_last_error();
    if (g->sched.active) {
        cudaFree(g->sched.d_sched);
        priv_mode_free(g->sched.mode_key);
        g->sched = Schedule{};
    }
    std::vector<double> tab(3 * (size_t)nsteps);
    for (int n = 0; n < nsteps; n++) {
        tab[3 * n] = adjoint ? 0.0 : amplitude[n];
        tab[3 * n + 1] = cos(phase[n]);
        tab[3 * n + 2] = sin(phase[n]);
    }
    Schedule s{};
    s.cx = center_x; s.cy = center_y; s.cz = center_z; s.reverse = reverse; s.adjoint = adjoint; s.n = nsteps;
    s.mode_key = priv_mode_new(source_mode);
    if (!s.mode_key) return fdtd_last_error();
    if (!cuda_ok(cudaMalloc(&s.d_sched, tab.size() * sizeof(double)), "cudaMalloc(schedule)")) return fdtd_last_error();
    cudaMemcpy(s.d_sched, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice);
    s.active = true;
    g->sched = s;
    if (!grid_plane(g, center_z, true)) return fdtd_last_error();
    g->version++;
    return FDTD_OK;
}

int timefield3d_set_exact_adjoint_schedule(timefield3d psi, int center_x, int center_y, int center_z,
                                           mode monitor_mode, int reverse, int nsteps, double omega, double delta_t,
                                           double weight_re, double weight_im)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (!g) return fdtd_last_error();
    if (!check_mode_plane(g, center_z)) return FDTD_ERR_ARG;
    if (nsteps <= 0 || !(delta_t > 0) || !std::isfinite(omega) || !std::isfinite(weight_re) ||
        !std::isfinite(weight_im)) {
        set_error(FDTD_ERR_ARG, "exact adjoint schedule needs nsteps > 0, delta_t > 0 and finite omega and weight");
        return FDTD_ERR_ARG;
    }
    if (!cuda_ok(cudaStreamSynchronize(g->st), "sync")) return fdtd_last_error();
    if (g->sched.active) {
        cudaFree(g->sched.d_sched);
        priv_mode_free(g->sched.mode_key);
        g->sched = Schedule{};
    }
    // nsteps + 1 entries: entry u drives the E-update current of adjoint step u
    // (the monitor's weights of forward step nsteps - u, none for u = 0) and the
    // H-update current of step u - 1 (forward step nsteps - u)
    const int n = nsteps + 1;
    std::vector<double> tab(3 * (size_t)n);
    for (int u = 0; u < n; u++) {
        const double ph = omega * delta_t * (double)(nsteps - u);
        tab[3 * u] = u >= 1 ? 1.0 : 0.0;
        tab[3 * u + 1] = cos(ph);
        tab[3 * u + 2] = sin(ph);
    }
    Schedule sc{};
    sc.cx = center_x; sc.cy = center_y; sc.cz = center_z; sc.reverse = reverse; sc.adjoint = 2; sc.n = n;
    sc.kappa = 0.5 * g->dx * g->dx / delta_t;
    sc.wre = weight_re;
    sc.wim = weight_im;
    sc.mode_key = priv_mode_new(monitor_mode);
    if (!sc.mode_key) return fdtd_last_error();
    if (!cuda_ok(cudaMalloc(&sc.d_sched, tab.size() * sizeof(double)), "cudaMalloc(schedule)")) return fdtd_last_error();
    if (!cuda_ok(cudaMemcpy(sc.d_sched, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice), "schedule H2D"))
        return fdtd_last_error();
    sc.active = true;
    g->sched = sc;
    if (!grid_plane(g, center_z, true)) return fdtd_last_error();
    g->version++;
    return FDTD_OK;
}

int timefield3d_clear_source_schedule(timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (g->sched.active) {
        if (g->dev) cudaStreamSynchronize(g->st);
        cudaFree(g->sched.d_sched);
        priv_mode_free(g->sched.mode_key);
    }
    g->sched = Schedule{};
    g->version++;
    return FDTD_OK;
}

int adjoint3d_taper_bind_store(adjoint3d_taper taper, timefield3d psi, int which, int t0, int dir)
{
    LOCK;
    Grid *g = dev_grid(psi);
    if (!g) return fdtd_last_error();
    if ((which != 0 && which != 1) || (dir != 1 && dir != -1 && dir != 0)) {
        set_error(FDTD_ERR_ARG, "bind_store: which must be 0/1, dir -1/0/1");
        return FDTD_ERR_ARG;
    }
    TaperDev *td = taper_lookup(taper, true);
    if (!taper_prepare(td, taper, g)) return fdtd_last_error();
    for (auto &b : g->binds)
        if (b.taper_key == taper.left && b.which == which) {
            b.t0 = t0;
            b.dir = dir;
            g->version++;
            return FDTD_OK;
        }
    g->binds.push_back(TaperBind{taper.left, which, t0, dir});
    g->version++;
    return FDTD_OK;
}

int adjoint3d_taper_unbind_store(adjoint3d_taper taper, timefield3d psi)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    std::vector<TaperBind> keep;
    for (auto &b : g->binds)
        if (b.taper_key != taper.left) keep.push_back(b);
    g->binds.swap(keep);
    g->version++;
    return FDTD_OK;
}

int timefield3d_run(timefield3d psi, double delta_t, int nsteps)
{
    LOCK;
    TraceRange tr("timefield3d_run");
    Grid *g = dev_grid(psi);
    if (!g) return fdtd_last_error();
    if (nsteps < 0) {
        set_error(FDTD_ERR_ARG, "nsteps %d", nsteps);
        return FDTD_ERR_ARG;
    }
    return run_steps(g, delta_t, nsteps) ? FDTD_OK : fdtd_last_error();
}

int fdtd_set_device(int device)
{
    LOCK;
    if (!device_available()) return fdtd_last_error();
    return cuda_ok(cudaSetDevice(device), "cudaSetDevice") ? FDTD_OK : fdtd_last_error();
}

long long fdtd_launch_count(void) { return launch_count(); }

namespace {
bool mode_ok(const mode *m, const char *what)
{
    if (!m || m->i < 3 || m->j < 3 || !m->fields.m || !m->ep.m || !m->mu.m || !m->pml.m || !(m->disc > 0)) {
        set_error(FDTD_ERR_ARG, "%s: mode must be at least 3 x 3 with disc > 0 and all arrays allocated", what);
        return false;
    }
    return true;
}
int last_mode_restarts = 0;
}  // namespace

int fdtd_mode_apply_beta_squared(mode in, double omega, mode out)
{
    LOCK;
    if (!device_available()) return fdtd_last_error();
    if (!mode_ok(&in, "fdtd_mode_apply_beta_squared") || !mode_ok(&out, "fdtd_mode_apply_beta_squared"))
        return FDTD_ERR_ARG;
    if (out.i != in.i || out.j != in.j) {
        set_error(FDTD_ERR_ARG, "fdtd_mode_apply_beta_squared: output %dx%d, input %dx%d", out.i, out.j, in.i, in.j);
        return FDTD_ERR_ARG;
    }
    return mode_apply_beta2_device(in, omega, out) ? FDTD_OK : fdtd_last_error();
}

complex fdtd_mode_solve_beta_squared(mode *psi, double omega, double tol, mode *prev_modes, int prev_num, int size,
                                     int confinement, int lateral_symmetry)
{
    LOCK;
    complex zero{0.0, 0.0};
    last_mode_restarts = 0;
    if (!device_available()) return zero;
    if (!mode_ok(psi, "fdtd_mode_solve_beta_squared")) return zero;
    if (!(omega > 0) || !(tol > 0) || size < 2 || size > 512 || (confinement != 1 && confinement != 2) ||
        prev_num < 0 || (prev_num > 0 && !prev_modes)) {
        set_error(FDTD_ERR_ARG, "fdtd_mode_solve_beta_squared: omega %g tol %g size %d confinement %d prev_num %d",
                  omega, tol, size, confinement, prev_num);
        return zero;
    }
    for (int p = 0; p < prev_num; p++) {
        if (!mode_ok(&prev_modes[p], "fdtd_mode_solve_beta_squared (previous mode)")) return zero;
        if (prev_modes[p].i != psi->i || prev_modes[p].j != psi->j) {
            set_error(FDTD_ERR_ARG, "fdtd_mode_solve_beta_squared: previous mode %d is %dx%d, mode %dx%d", p,
                      prev_modes[p].i, prev_modes[p].j, psi->i, psi->j);
            return zero;
        }
    }
    std::complex<double> beta;
    int restarts = 0;
    if (!mode_solve_device(psi, omega, tol, prev_modes, prev_num, size, confinement, lateral_symmetry, 5000, &beta,
                           &restarts))
        return zero;
    last_mode_restarts = restarts;
    return complex{beta.real(), beta.imag()};
}

int fdtd_mode_solve_restarts(void) { return last_mode_restarts; }

int fdtd_sweep_run(const timefield3d *grids, int ngrids, double delta_t, const int *nsteps, int steps_per_launch,
                   int band_rows, double tiles_per_sm)
{
    LOCK;
    if (!grids || !nsteps || ngrids <= 0 || ngrids > kSweepMaxGrids || !(delta_t > 0) || !std::isfinite(delta_t)) {
        set_error(FDTD_ERR_ARG, "fdtd_sweep_run: grids, nsteps, ngrids in [1, %d] and a positive delta_t are required",
                  kSweepMaxGrids);
        return FDTD_ERR_ARG;
    }
    std::vector<Grid *> gs;
    std::vector<int> ns(nsteps, nsteps + ngrids);
    for (int i = 0; i < ngrids; i++) {
        Grid *g = dev_grid(grids[i]);
        if (!g) return fdtd_last_error() ? fdtd_last_error() : FDTD_ERR_ARG;
        gs.push_back(g);
    }
    TraceRange tr("fdtd_sweep_run");
    if (!run_sweep(gs, delta_t, ns, steps_per_launch, band_rows, tiles_per_sm)) return fdtd_last_error();
    return FDTD_OK;
}

int fdtd_sweep_barrier_selftest(double limit_seconds)
{
    LOCK;
    if (!device_available()) return fdtd_last_error();
    if (!(limit_seconds > 0.0) || limit_seconds > 10.0) {
        set_error(FDTD_ERR_ARG, "sweep barrier self-test limit %g s: must be in (0, 10]", limit_seconds);
        return FDTD_ERR_ARG;
    }
    int timed_out = 0;
    if (!sweep_barrier_selftest((unsigned long long)(limit_seconds * 1e9), &timed_out)) return fdtd_last_error();
    if (!timed_out) {
        set_error(FDTD_ERR_CUDA, "sweep barrier self-test: the wait completed although nothing could complete it");
        return FDTD_ERR_CUDA;
    }
    set_error(FDTD_ERR_TIMEOUT, "sweep barrier self-test: the bounded wait gave up as designed");
    return FDTD_ERR_TIMEOUT;
}

int fdtd_wait_selftest(double limit_seconds, double *elapsed_seconds)
{
    LOCK;
    if (!device_available()) return fdtd_last_error();
    if (!(limit_seconds > 0.0) || limit_seconds > 10.0) {
        set_error(FDTD_ERR_ARG, "wait self-test limit %g s: must be in (0, 10]", limit_seconds);
        return FDTD_ERR_ARG;
    }
    cudaStream_t st = nullptr;
    int *d_err = nullptr;
    unsigned long long *d_el = nullptr;
    int h_err = 0;
    unsigned long long h_el = 0;
    bool ok = cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate") &&
              cuda_ok(cudaMalloc(&d_err, sizeof(int)), "cudaMalloc") &&
              cuda_ok(cudaMalloc(&d_el, sizeof(unsigned long long)), "cudaMalloc") &&
              cuda_ok(cudaMemsetAsync(d_err, 0, sizeof(int), st), "cudaMemsetAsync");
    if (ok) {
        launch_wait_selftest((unsigned long long)(limit_seconds * 1e9), d_err, d_el, st);
        ok = cuda_ok(cudaGetLastError(), "wait self-test launch") &&
             cuda_ok(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync") &&
             cuda_ok(cudaMemcpyAsync(&h_el, d_el, sizeof(h_el), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync") &&
             cuda_ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    }
    if (d_err) cudaFree(d_err);
    if (d_el) cudaFree(d_el);
    if (st) cudaStreamDestroy(st);
    if (!ok) return fdtd_last_error();
    if (elapsed_seconds) *elapsed_seconds = (double)h_el * 1e-9;
    if (h_err) {
        set_error(FDTD_ERR_TIMEOUT, "wait self-test: the bounded wait gave up after %.3f s as designed",
                  (double)h_el * 1e-9);
        return FDTD_ERR_TIMEOUT;
    }
    set_error(FDTD_ERR_CUDA, "wait self-test: a wait on a barrier nothing arrives on completed");
    return FDTD_ERR_CUDA;
}

void *timefield3d_get_stream(timefield3d psi)
{
    LOCK;
    Grid *g = dev_grid(psi);
    return g ? (void *)g->st : nullptr;
}

int timefield3d_upload_materials(timefield3d psi)
{
    LOCK;
    TraceRange tr("timefield3d_upload_materials");
    Grid *g = dev_grid(psi);
    if (!g) return fdtd_last_error();
    return grid_upload_materials(g) ? FDTD_OK : fdtd_last_error();
}

int timefield3d_checkpoint_save(timefield3d psi, const char *path)
{
    LOCK;
    TraceRange tr("timefield3d_checkpoint_save");
    Grid *g = dev_grid(psi);
    if (!g) return fdtd_last_error();
    if (!path) return FDTD_ERR_ARG;
    return grid_checkpoint_save(g, path) ? FDTD_OK : fdtd_last_error();
}

int timefield3d_checkpoint_load(timefield3d psi, const char *path)
{
    LOCK;
    TraceRange tr("timefield3d_checkpoint_load");
    Grid *g = dev_grid(psi);
    if (!g) return fdtd_last_error();
    if (!path) return FDTD_ERR_ARG;
    return grid_checkpoint_load(g, path) ? FDTD_OK : fdtd_last_error();
}

void fdtd_inject_allocation_failures(int n)
{
    LOCK;
    inject_allocation_failures(n);
}

int timefield3d_set_kernel_timing(timefield3d psi, int on)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g || on < 0) return FDTD_ERR_ARG;
    if (g->dev && (!drain_kernel_timing(g, 0) || !drain_kernel_timing(g, 1))) return fdtd_last_error();
    g->ktime = on;
    g->kreplay = 0;
    g->ktime_ms = 0;
    g->ktime_n = 0;
    return FDTD_OK;
}

int timefield3d_read_kernel_timing(timefield3d psi, double *total_ms, long long *count)
{
    LOCK;
    Grid *g = grid_lookup(psi);
    if (!g || !total_ms || !count) return FDTD_ERR_ARG;
    if (g->dev && (!drain_kernel_timing(g, 0) || !drain_kernel_timing(g, 1))) return fdtd_last_error();
    *total_ms = g->ktime_ms;
    *count = g->ktime_n;
    g->ktime_ms = 0;
    g->ktime_n = 0;
    return FDTD_OK;
}

int timefield3d_release_mode(mode m)
{
    LOCK;
    mode_release(m.fields.m);
    return FDTD_OK;
}

int adjoint3d_taper_sync_host(adjoint3d_taper taper)
{
    LOCK;
    TaperDev *td = taper_lookup(taper, false);
    if (!td || !td->d_fwd) return FDTD_OK;
    if (!cuda_ok(cudaDeviceSynchronize(), "sync")) return fdtd_last_error();
    size_t cnt = (size_t)td->duration * td->ncell * 3;
    for (int w = 0; w < 2; w++) {
        double *host = w ? taper.adjoint_fields : taper.forward_fields;
        const void *dev = w ? td->d_adj : td->d_fwd;
        std::vector<double> tmp(cnt);
        if (td->prec == FDTD_F64) {
            if (!cuda_ok(cudaMemcpy(tmp.data(), dev, cnt * sizeof(double), cudaMemcpyDeviceToHost), "taper D2H")) return fdtd_last_error();
        } else {
            std::vector<float> f(cnt);
            if (!cuda_ok(cudaMemcpy(f.data(), dev, cnt * sizeof(float), cudaMemcpyDeviceToHost), "taper D2H")) return fdtd_last_error();
            for (size_t q = 0; q < cnt; q++) tmp[q] = f[q];
        }
        for (size_t c = 0; c < cnt / 3; c++)
            for (int m = 0; m < 3; m++) host[6 * c + m] = tmp[3 * c + m];
    }
    return FDTD_OK;
}

}  // extern "C"
