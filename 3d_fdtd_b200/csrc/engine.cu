// engine.cu -- device state of grids, modes and tapers; the step sequence;
// CUDA-graph capture of multi-step runs.
#include "engine.h"

#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <unordered_map>

namespace fdtd {

// ============================================================================
// status
// ============================================================================
static thread_local int t_err = FDTD_OK;
static thread_local char t_msg[512] = "";

void set_error(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_msg, sizeof t_msg, fmt, ap);
    va_end(ap);
    t_err = code;
    fprintf(stderr, "libfdtd_b200: error %d: %s\n", code, t_msg);
}
}  // namespace fdtd

extern "C" int fdtd_last_error(void) { return fdtd::t_err; }
extern "C" const char *fdtd_last_error_message(void) { return fdtd::t_msg; }
extern "C" void fdtd_clear_error(void)
{
    fdtd::t_err = FDTD_OK;
    fdtd::t_msg[0] = 0;
}

namespace fdtd {

static std::atomic<long long> g_launches{0};
void note_launch(int n) { g_launches += n; }
long long launch_count() { return g_launches.load(); }

bool cuda_ok(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return true;
    set_error(e == cudaErrorMemoryAllocation ? FDTD_ERR_ALLOC : FDTD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return false;
}

#define CK(call)                                   \
    do {                                           \
        if (!cuda_ok((call), #call)) return false; \
    } while (0)
#define CKL(what)                                        \
    do {                                                 \
        if (!cuda_ok(cudaGetLastError(), what)) return false; \
    } while (0)

bool device_available()
{
    static int state = -1;   // -1 unknown, 0 none, 1 ok
    static std::string why;
    if (state < 0) {
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0) {
            state = 0;
            why = e != cudaSuccess ? cudaGetErrorString(e) : "no CUDA device";
        } else {
            state = 1;
        }
    }
    if (state == 0) {
        set_error(FDTD_ERR_NO_DEVICE, "no usable CUDA device (%s); this library has no CPU fallback", why.c_str());
        return false;
    }
    return true;
}

std::mutex &api_mutex()
{
    static std::mutex m;
    return m;
}

TraceRange::TraceRange(const char *name) { nvtxRangePushA(name); }
TraceRange::~TraceRange() { nvtxRangePop(); }

// host-side fault injection: the next n engine allocations report failure
static std::atomic<int> g_fail_allocs{0};
void inject_allocation_failures(int n) { g_fail_allocs.store(n < 0 ? 0 : n); }

template <typename P> static bool dalloc(P **p, size_t bytes, cudaStream_t st, bool zero = true)
{
    if (*p) return true;
    if (g_fail_allocs.load() > 0) {
        g_fail_allocs--;
        set_error(FDTD_ERR_ALLOC, "device allocation of %zu bytes failed (injected)", bytes);
        return false;
    }
    void *v = nullptr;
    if (!cuda_ok(cudaMalloc(&v, bytes ? bytes : 16), "cudaMalloc")) return false;
    *p = (P *)v;
    if (zero) return cuda_ok(cudaMemsetAsync(v, 0, bytes ? bytes : 16, st), "cudaMemsetAsync");
    return true;
}

template <typename P> static void dfree(P *&p)
{
    if (p) cudaFree((void *)p);
    p = nullptr;
}

// ============================================================================
// modes
// ============================================================================
static std::unordered_map<const void *, DevMode *> &mode_table()
{
    static std::unordered_map<const void *, DevMode *> t;
    return t;
}

static uint64_t mode_fingerprint(const mode &m)
{
    // FNV-1a over the dimensions and up to 257 evenly spaced complex entries:
    // catches a mode rescaled in place (mode_smul) or replaced at the same
    // address, at O(1) cost per call.
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](const void *p, size_t n) {
        const unsigned char *c = (const unsigned char *)p;
        for (size_t i = 0; i < n; i++) { h ^= c[i]; h *= 1099511628211ull; }
    };
    mix(&m.i, sizeof m.i);
    mix(&m.j, sizeof m.j);
    mix(&m.disc, sizeof m.disc);
    long long n = 6LL * m.i * m.j;
    if (n <= 0 || !m.fields.m) return h;
    const int samples = 257;
    for (int s = 0; s < samples; s++) {
        long long q = (n - 1) * s / (samples - 1);
        mix(&m.fields.m[q], sizeof(complex));
    }
    return h;
}

double mode_power_norm_host(const mode &m)
{
    // mode_power_inner_product(psi, psi) (mode.c:1267-1310) and mode_power_norm (1330-1337)
    double sre = 0, sim = 0;
    for (int i = 0; i < m.i; i++)
        for (int j = 0; j < m.j; j++) {
            const complex *e = m.fields.m + 6 * (size_t)(i + j * m.i);
            double Exr = e[0].re, Exi = e[0].im, Eyr = e[1].re, Eyi = e[1].im;
            double Hxr = e[3].re, Hxi = e[3].im, Hyr = e[4].re, Hyi = e[4].im;
            double p1r = Hxr * Eyr - (-Hxi) * Eyi, p1i = Hxr * Eyi + (-Hxi) * Eyr;
            double q2r = Hyr * Exr - (-Hyi) * Exi, q2i = Hyr * Exi + (-Hyi) * Exr;
            double p3r = Hxr * Eyr - Hxi * (-Eyi), p3i = Hxr * (-Eyi) + Hxi * Eyr;
            double q4r = Hyr * Exr - Hyi * (-Exi), q4i = Hyr * (-Exi) + Hyi * Exr;
            sre = sre + ((p1r + (0 - q2r)) + (p3r + (0 - q4r)));
            sim = sim + ((p1i + (0 - q2i)) + (p3i + (0 - q4i)));
        }
    double s = (-0.5 * m.disc * m.disc);
    sre = s * sre;
    sim = s * sim;
    return std::sqrt(std::sqrt(sre * sre + sim * sim));
}

void mode_power_normalize_host(const mode &m)
{
    // mode_power_normalize (mode.c:1367-1379): fields *= 1/norm, in place
    double divisor = 1.0 / mode_power_norm_host(m);
    size_t n = 6 * (size_t)m.i * m.j;
    for (size_t q = 0; q < n; q++) {
        m.fields.m[q].re = divisor * m.fields.m[q].re;
        m.fields.m[q].im = divisor * m.fields.m[q].im;
    }
}

static uint64_t g_mode_version = 1;

DevMode *mode_device(const mode &m)
{
    if (m.i <= 0 || m.j <= 0 || !m.fields.m || !(m.disc > 0)) {
        set_error(FDTD_ERR_ARG, "invalid mode (i=%d j=%d disc=%g)", m.i, m.j, m.disc);
        return nullptr;
    }
    auto &tab = mode_table();
    const void *key = m.fields.m;
    uint64_t fp = mode_fingerprint(m);
    auto it = tab.find(key);
    if (it != tab.end() && it->second->fingerprint == fp && it->second->mi == m.i && it->second->mj == m.j &&
        it->second->disc == m.disc)
        return it->second;
    // first sight (or changed): power-normalise the caller's mode in place,
    // as the reference's source/overlap calls do, and upload it
    mode_power_normalize_host(m);
    DevMode *dm;
    if (it == tab.end()) {
        dm = new DevMode();
        dm->key = key;
        tab[key] = dm;
    } else {
        dm = it->second;
        // queued kernels may still read the old copy
        if (!cuda_ok(cudaDeviceSynchronize(), "cudaDeviceSynchronize")) return nullptr;
        if (dm->mi != m.i || dm->mj != m.j) dfree(dm->d);
    }
    dm->mi = m.i;
    dm->mj = m.j;
    dm->disc = m.disc;
    dm->fingerprint = mode_fingerprint(m);
    size_t bytes = 6 * (size_t)m.i * m.j * sizeof(double2);
    if (!dm->d && !cuda_ok(cudaMalloc(&dm->d, bytes), "cudaMalloc(mode)")) return nullptr;
    if (!cuda_ok(cudaMemcpy(dm->d, m.fields.m, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(mode)")) return nullptr;
    g_mode_version++;
    return dm;
}

void mode_release(const void *key)
{
    auto &tab = mode_table();
    auto it = tab.find(key);
    if (it == tab.end()) return;
    cudaDeviceSynchronize();
    dfree(it->second->d);
    delete it->second;
    tab.erase(it);
    g_mode_version++;
}

// private normalised device copy of a mode (monitors, schedules)
static double2 *mode_private_copy(const mode &m)
{
    if (m.i <= 0 || m.j <= 0 || !m.fields.m || !(m.disc > 0)) {
        set_error(FDTD_ERR_ARG, "invalid mode (i=%d j=%d disc=%g)", m.i, m.j, m.disc);
        return nullptr;
    }
    mode_power_normalize_host(m);
    size_t bytes = 6 * (size_t)m.i * m.j * sizeof(double2);
    double2 *d = nullptr;
    if (!cuda_ok(cudaMalloc(&d, bytes), "cudaMalloc(mode)")) return nullptr;
    if (!cuda_ok(cudaMemcpy(d, m.fields.m, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(mode)")) {
        cudaFree(d);
        return nullptr;
    }
    return d;
}

// monitors and schedules keep their own mode copies: key -> (device ptr, dims)
struct PrivMode {
    double2 *d;
    int mi, mj;
    double disc;
};
static std::unordered_map<const void *, PrivMode> &priv_modes()
{
    static std::unordered_map<const void *, PrivMode> t;
    return t;
}
static uint64_t g_priv_id = 1;

const void *priv_mode_new(const mode &m)
{
    double2 *d = mode_private_copy(m);
    if (!d) return nullptr;
    const void *key = (const void *)(uintptr_t)(g_priv_id++);
    priv_modes()[key] = PrivMode{d, m.i, m.j, m.disc};
    return key;
}

void priv_mode_free(const void *key)
{
    auto &t = priv_modes();
    auto it = t.find(key);
    if (it == t.end()) return;
    cudaFree(it->second.d);
    t.erase(it);
}

// ============================================================================
// grids
// ============================================================================
static std::unordered_map<const void *, Grid *> &grid_table()
{
    static std::unordered_map<const void *, Grid *> t;
    return t;
}

Grid *grid_lookup(const timefield3d &psi, bool quiet)
{
    auto &t = grid_table();
    auto it = t.find(psi.fields);
    if (it == t.end()) {
        if (!quiet) set_error(FDTD_ERR_ARG, "unknown grid (not created by timefield3d_new of this library)");
        return nullptr;
    }
    return it->second;
}

Grid *grid_register(const timefield3d &psi)
{
    Grid *g = new Grid();
    g->h = psi;
    g->nx = psi.i;
    g->ny = psi.j;
    g->nz = psi.k;
    g->n = (long long)psi.i * psi.j * psi.k;
    g->dx = psi.disc;
    grid_table()[psi.fields] = g;
    return g;
}

void grid_unregister(const timefield3d &psi)
{
    auto &t = grid_table();
    auto it = t.find(psi.fields);
    if (it == t.end()) return;
    delete it->second;
    t.erase(it);
}

static size_t esize(const Grid *g) { return g->prec == FDTD_F64 ? sizeof(double) : sizeof(float); }

static void free_fields(Grid *g)
{
    for (int s = 0; s < 2; s++) {
        for (int m = 0; m < 6; m++) dfree(g->f[s][m]);
        dfree(g->d_fptr[s]);
    }
    for (int m = 0; m < 6; m++) dfree(g->old[m]);
    for (int s = 0; s < 2; s++)
        for (int a = 0; a < 3; a++)
            for (int w = 0; w < 4; w++) dfree(g->psi[s][a][w]);
    for (int w = 0; w < 6; w++)
        for (int a = 0; a < 3; a++) dfree(g->prof[w][a]);
    g->prof_dt = 0;
    g->cur = 0;
}

Grid::~Grid()
{
    if (dev) {
        cudaStreamSynchronize(st);
        for (int s = 0; s < 3; s++)
            if (graph[s]) cudaGraphExecDestroy(graph[s]);
        for (int s = 0; s < 2; s++)
            for (int e = 0; e < 64; e++)
                if (kev[s][e]) cudaEventDestroy(kev[s][e]);
        free_fields(this);
        for (int c = 0; c < 3; c++) { dfree(ep[c]); dfree(mu[c]); dfree(cb[c]); dfree(ca[c]); }
        for (int m = 0; m < 6; m++) dfree(sig[m]);
        for (auto &p : planes) dfree(p.p);
        for (auto p : plane_pool) dfree(p);
        dfree(d_step); dfree(d_done); dfree(d_jobs); dfree(d_job1); dfree(d_partials); dfree(d_inst);
        dfree(wave.d_items); dfree(wave.d_cnt); dfree(wave.d_part); dfree(wave.d_ring);
        for (int s = 0; s < 2; s++)
            for (int e = 0; e < 2; e++)
                if (wave.ev[s][e]) cudaEventDestroy(wave.ev[s][e]);
        if (h_inst) cudaFreeHost(h_inst);
        if (h_flag) cudaFreeHost(h_flag);
        if (h_err) cudaFreeHost(h_err);
        dfree(d_err);
        delete fmaps[0];
        delete fmaps[1];
        dfree(d_tiles);
        dfree(d_flag);
        for (auto &mn : monitors) { dfree(mn.d_omega); dfree(mn.d_acc); priv_mode_free(mn.mode_key); }
        dfree(d_probes); dfree(d_probe_buf); dfree(d_probe_count);
        dfree(d_dft_full);
        for (auto &kv : d_dft_slice) dfree(kv.second);
        if (sched.active) { dfree(sched.d_sched); priv_mode_free(sched.mode_key); }
        dfree(d_aos);
        cudaStreamSynchronize(side);
        cudaEventDestroy(ev_fork);
        cudaEventDestroy(ev_join);
        cudaStreamDestroy(side);
        cudaStreamDestroy(st);
    }
}

template <typename T> GridView<T> view(Grid *g, int set)
{
    GridView<T> v;
    v.nx = g->nx; v.ny = g->ny; v.nz = g->nz; v.n = g->n;
    for (int m = 0; m < 6; m++) { v.f[m] = (T *)g->f[set][m]; v.old[m] = (T *)g->old[m]; v.sig[m] = g->sig[m]; }
    for (int c = 0; c < 3; c++) { v.ep[c] = g->ep[c]; v.mu[c] = g->mu[c]; }
    return v;
}
template GridView<float> view<float>(Grid *, int);
template GridView<double> view<double>(Grid *, int);

template <typename T> CpmlView<T> cpml_view(Grid *g, int in_set)
{
    CpmlView<T> c{};
    c.L = g->boundary == FDTD_BOUNDARY_CPML ? g->L : 0;
    for (int a = 0; a < 3; a++) {
        for (int w = 0; w < 4; w++) c.psi[a][w] = (T *)g->psi[in_set][a][w];
        for (int w = 0; w < 6; w++) c.prof[w][a] = (const T *)g->prof[w][a];
    }
    return c;
}
template CpmlView<float> cpml_view<float>(Grid *, int);
template CpmlView<double> cpml_view<double>(Grid *, int);

SourcePlanes source_table(Grid *g)
{
    SourcePlanes s{};
    s.n = (int)g->planes.size();
    for (int i = 0; i < s.n; i++) { s.k[i] = g->planes[i].k; s.p[i] = g->planes[i].p; }
    return s;
}

// deinterleave AoS float (stride s) into up to 6 SoA arrays; per component c
// flag[c] bit 1 = some value differs from `ref`, bit 2 = some value is not finite
__global__ void k_deinterleave(const float *aos, int stride, float *d0, float *d1, float *d2, float *d3, float *d4,
                               float *d5, long long n, float ref, int *flag)
{
    float *d[6] = {d0, d1, d2, d3, d4, d5};
    int local[6] = {0, 0, 0, 0, 0, 0};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 6; c++) {
            if (c >= stride) break;
            float v = aos[q * stride + c];
            d[c][q] = v;
            if (v != ref) local[c] |= 1;
            if (!isfinite(v)) local[c] |= 2;
        }
    }
    for (int c = 0; c < stride; c++)
        if (local[c]) atomicOr(flag + c, local[c]);
}

static bool upload_deinterleave(Grid *g, const float *host, int stride, float **dst, float ref, int *d_flags)
{
    size_t bytes = (size_t)g->n * stride * sizeof(float);
    if (!dalloc(&g->d_aos, (size_t)g->n * 6 * sizeof(double), g->st, false)) return false;
    CK(cudaMemcpyAsync(g->d_aos, host, bytes, cudaMemcpyHostToDevice, g->st));
    float *d[6] = {};
    for (int c = 0; c < stride; c++) d[c] = dst[c];
    int blocks = (int)std::min<long long>((g->n + 255) / 256, 4736);
    note_launch();
    k_deinterleave<<<blocks, 256, 0, g->st>>>((const float *)g->d_aos, stride, d[0], d[1], d[2], d[3], d[4], d[5],
                                                g->n, ref, d_flags);
    CKL("k_deinterleave");
    return true;
}

bool grid_upload_materials(Grid *g)
{
    // only the arrays the rasterisers touched (kMatEp / kMatMu / kMatSig bits);
    // flags: [0..2] ep != 1, [3..5] mu != 1, [6..11] sig != 0 (bit 2: not finite)
    const int dirty = g->mat_dirty;
    // Pin the host material mirrors once a grid uploads them a second time
    // (design loops re-rasterise and re-upload every evaluation); a grid
    // uploaded once does not pay for pinning (hundreds of ms per GB).
    if (++g->material_uploads == 2 && !g->mirrors_pinned) {
        cudaHostRegister(g->h.ep, (size_t)g->n * 3 * sizeof(float), cudaHostRegisterDefault);
        cudaHostRegister(g->h.mu, (size_t)g->n * 3 * sizeof(float), cudaHostRegisterDefault);
        cudaHostRegister(g->h.sig, (size_t)g->n * 6 * sizeof(float), cudaHostRegisterDefault);
        cudaGetLastError();
        g->mirrors_pinned = true;
    }
    if (dirty & kMatEp) {
        CK(cudaMemsetAsync(g->d_flag + 0, 0, 3 * sizeof(int), g->st));
        if (!upload_deinterleave(g, g->h.ep, 3, g->ep, 1.0f, g->d_flag + 0)) return false;
    }
    if (dirty & kMatMu) {
        CK(cudaMemsetAsync(g->d_flag + 3, 0, 3 * sizeof(int), g->st));
        if (!upload_deinterleave(g, g->h.mu, 3, g->mu, 1.0f, g->d_flag + 3)) return false;
    }
    if (dirty & kMatSig) {
        CK(cudaMemsetAsync(g->d_flag + 6, 0, 6 * sizeof(int), g->st));
        if (!upload_deinterleave(g, g->h.sig, 6, g->sig, 0.0f, g->d_flag + 6)) return false;
    }
    CK(cudaMemcpyAsync(g->h_flag, g->d_flag, 12 * sizeof(int), cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    int any = 0;
    for (int c = 0; c < 12; c++) any |= g->h_flag[c];
    if (any & 2) {
        set_error(FDTD_ERR_NONFINITE, "non-finite permittivity, permeability or conductivity");
        return false;
    }
    g->mu_nonunit = ((g->h_flag[3] | g->h_flag[4] | g->h_flag[5]) & 1) != 0;
    g->sig_e = ((g->h_flag[6] | g->h_flag[7] | g->h_flag[8]) & 1) != 0;
    g->sig_m = ((g->h_flag[9] | g->h_flag[10] | g->h_flag[11]) & 1) != 0;
    g->mat_dirty = 0;
    g->coef_valid = false;
    g->version++;
    return true;
}

// waits for the grid, then reports (and clears) a bounded device wait that gave up
bool grid_check_device_error(Grid *g)
{
    if (!g->dev || !g->d_err) return true;
    CK(cudaMemcpyAsync(g->h_err, g->d_err, sizeof(int), cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    if (*g->h_err) {
        CK(cudaMemsetAsync(g->d_err, 0, sizeof(int), g->st));
        set_error(FDTD_ERR_TIMEOUT, "a device-side wait gave up; results since the last check are invalid");
        return false;
    }
    return true;
}

bool grid_upload_fields(Grid *g)
{
    if (!dalloc(&g->d_aos, (size_t)g->n * 6 * sizeof(double), g->st, false)) return false;
    CK(cudaMemcpyAsync(g->d_aos, g->h.fields, (size_t)g->n * 6 * sizeof(double), cudaMemcpyHostToDevice, g->st));
    if (g->prec == FDTD_F64) launch_aos_to_soa<double>(g->d_aos, (double *const *)g->f[g->cur], g->n, g->st);
    else launch_aos_to_soa<float>(g->d_aos, (float *const *)g->f[g->cur], g->n, g->st);
    CKL("aos_to_soa");
    g->fields_from_host = false;
    g->pp_synced = false;
    return true;
}

bool grid_download_fields(Grid *g)
{
    if (!dalloc(&g->d_aos, (size_t)g->n * 6 * sizeof(double), g->st, false)) return false;
    if (g->prec == FDTD_F64) launch_soa_to_aos<double>(g->d_aos, (double *const *)g->f[g->cur], g->n, g->st);
    else launch_soa_to_aos<float>(g->d_aos, (float *const *)g->f[g->cur], g->n, g->st);
    CKL("soa_to_aos");
    g->host_mirror_written = true;
    CK(cudaMemcpyAsync(g->h.fields, g->d_aos, (size_t)g->n * 6 * sizeof(double), cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    return true;
}

static bool alloc_field_set(Grid *g, int s)
{
    size_t bytes = (size_t)g->n * esize(g);
    for (int m = 0; m < 6; m++)
        if (!dalloc(&g->f[s][m], bytes, g->st)) return false;
    if (!dalloc(&g->d_fptr[s], 6 * sizeof(void *), g->st, false)) return false;
    CK(cudaMemcpyAsync(g->d_fptr[s], g->f[s], 6 * sizeof(void *), cudaMemcpyHostToDevice, g->st));
    CK(cudaStreamSynchronize(g->st));
    return true;
}

bool grid_ensure_device(Grid *g)
{
    if (!device_available()) return false;
    if (!g->dev) {
        if (g->nx < 4 || g->ny < 4 || g->nz < 4) {
            set_error(FDTD_ERR_ARG, "grid %dx%dx%d: every dimension must be >= 4", g->nx, g->ny, g->nz);
            return false;
        }
        CK(cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&g->ev_join, cudaEventDisableTiming));
        g->dev = true;
        size_t fb = (size_t)g->n * sizeof(float);
        for (int c = 0; c < 3; c++) {
            if (!dalloc(&g->ep[c], fb, g->st, false) || !dalloc(&g->mu[c], fb, g->st, false)) return false;
        }
        for (int m = 0; m < 6; m++)
            if (!dalloc(&g->sig[m], fb, g->st, false)) return false;
        if (!dalloc(&g->d_step, sizeof(long long), g->st)) return false;
        if (!dalloc(&g->d_done, sizeof(unsigned), g->st)) return false;
        if (!dalloc(&g->d_flag, 12 * sizeof(int), g->st)) return false;
        CK(cudaMallocHost(&g->h_flag, 12 * sizeof(int)));
        CK(cudaMallocHost(&g->h_inst, sizeof(double2)));
        CK(cudaMallocHost(&g->h_err, sizeof(int)));
        if (!dalloc(&g->d_err, sizeof(int), g->st)) return false;
        if (!dalloc(&g->d_inst, sizeof(double2), g->st)) return false;
        if (!dalloc(&g->d_job1, sizeof(OverlapJob), g->st)) return false;
        g->jobs_cap = 8;
        if (!dalloc(&g->d_jobs, g->jobs_cap * sizeof(OverlapJob), g->st, false)) return false;
        const int parts = overlap_parts((long long)g->nx * g->ny);
        if (!dalloc(&g->d_partials, (size_t)g->jobs_cap * parts * sizeof(double2), g->st, false)) return false;
        g->mat_dirty = kMatAll;
    }
    if (!g->f[0][0]) {
        if (!alloc_field_set(g, 0)) return false;
        g->cur = 0;
    }
    if (g->mat_dirty && !grid_upload_materials(g)) return false;
    if (g->fields_from_host && !grid_upload_fields(g)) return false;
    return true;
}

bool grid_set_precision(Grid *g, int prec)
{
    if (prec != FDTD_F64 && prec != FDTD_F32) {
        set_error(FDTD_ERR_ARG, "precision %d", prec);
        return false;
    }
    if (prec == g->prec) return true;
    if (g->dev && g->f[0][0]) {
        if (!grid_download_fields(g)) return false;
        free_fields(g);
        g->fields_from_host = true;
    }
    g->prec = prec;
    g->coef_valid = false;
    g->version++;
    return true;
}

// CPML profiles along each axis, for step dt.  Depth fraction rho of an E node
// (p = i) or H node (p = i + 1/2): (L - 1/2 - p)/L on the low side,
// (p - (N - L - 1/2))/L on the high side; sigma = smax rho^m,
// kappa = 1 + (kmax - 1) rho^m, alpha = amax (1 - rho),
// b = exp(-(sigma/kappa + alpha) dt), a = sigma (b - 1)/(sigma kappa + kappa^2 alpha).
// Computed in double on the host (the CPU restatement uses the same code), so
// the FP64 path sees identical tables.
static void cpml_point(double rho, int order, double smax, double kmax, double amax, double dt, double *b, double *a,
                       double *kinv)
{
    if (rho <= 0) { *b = 1.0; *a = 0.0; *kinv = 1.0; return; }
    double r = std::pow(rho, order);
    double sigma = smax * r;
    double kappa = 1.0 + (kmax - 1.0) * r;
    double alpha = amax * (1.0 - rho);
    *b = std::exp(-(sigma / kappa + alpha) * dt);
    *a = sigma > 0 ? sigma * (*b - 1.0) / (sigma * kappa + kappa * kappa * alpha) : 0.0;
    *kinv = 1.0 / kappa;
}

static bool build_profiles(Grid *g, double dt)
{
    const int L = g->L;
    double smax = g->smax > 0 ? g->smax : 0.8 * (g->order + 1) / g->dx;
    int dims[3] = {g->nx, g->ny, g->nz};
    for (int a = 0; a < 3; a++) {
        int N = dims[a];
        std::vector<double> tab[6];
        for (int w = 0; w < 6; w++) tab[w].resize(N);
        for (int i = 0; i < N; i++)
            for (int h = 0; h < 2; h++) {
                double p = i + 0.5 * h;
                double rho = 0;
                if (p < L - 0.5) rho = (L - 0.5 - p) / L;
                else if (p > N - L - 0.5) rho = (p - (N - L - 0.5)) / L;
                cpml_point(rho, g->order, smax, g->kmax, g->amax, dt, &tab[3 * h][i], &tab[3 * h + 1][i],
                           &tab[3 * h + 2][i]);
            }
        for (int w = 0; w < 6; w++) {
            if (!dalloc(&g->prof[w][a], N * sizeof(double), g->st, false)) return false;
            // ordered on the grid's stream: queued steps still read the old tables
            // (pageable source: the copy is staged before the call returns)
            if (g->prec == FDTD_F64) {
                CK(cudaMemcpyAsync(g->prof[w][a], tab[w].data(), N * sizeof(double), cudaMemcpyHostToDevice, g->st));
            } else {
                std::vector<float> f(N);
                for (int i = 0; i < N; i++) f[i] = (float)tab[w][i];
                CK(cudaMemcpyAsync(g->prof[w][a], f.data(), N * sizeof(float), cudaMemcpyHostToDevice, g->st));
            }
        }
    }
    g->prof_dt = dt;
    return true;
}

// FP32 fast path: precomputed E coefficients, scalar H coefficient (mu = 1,
// no magnetic loss), CPML or PEC boundary
static bool fast32_path(const Grid *g)
{
    return g->prec == FDTD_F32 && g->boundary != FDTD_BOUNDARY_MUR && !g->sig_m && !g->mu_nonunit;
}

// which kernel design the fast path uses: the one-pass streaming kernel where
// the grid allows it (FDTD_YEE_STREAM, and FDTD_YEE_AUTO: it moves each array
// once a step and measured faster than the flat pair with and without CPML),
// the plane-streaming TMA / cp.async kernel on request, else the flat pair
static bool stream_path(const Grid *g)
{
    return fast32_path(g) && (g->yee_variant == FDTD_YEE_STREAM || g->yee_variant == FDTD_YEE_AUTO) &&
           stream_supported(g->nx, g->ny, g->nz, g->sig_e, g->boundary == FDTD_BOUNDARY_CPML ? g->L : 0);
}

static bool fused_path(const Grid *g)
{
    return fast32_path(g) && g->yee_variant == FDTD_YEE_FUSED && fused_supported(g->nx, g->ny, g->nz);
}

// designs that read one field set and write the other
static bool pingpong_path(const Grid *g) { return stream_path(g) || fused_path(g); }

// tile plan of the streaming kernel for the grid's shape (rebuilt when the
// shape, CPML thickness, loss or device changes)
static bool stream_prepare(Grid *g)
{
    int dev = 0, nsm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int L = g->boundary == FDTD_BOUNDARY_CPML ? g->L : 0;
    const int key[6] = {g->nx, g->ny, g->nz, L, g->sig_e ? 1 : 0, nsm};
    if (g->d_tiles && std::equal(key, key + 6, g->splan_key)) return true;
    StreamPlan p;
    if (!stream_plan(g->nx, g->ny, g->nz, L, g->sig_e, nsm, &p)) {
        set_error(FDTD_ERR_UNSUPPORTED, "streaming Yee kernel: no tile plan for grid %dx%dx%d", g->nx, g->ny, g->nz);
        return false;
    }
    if (!stream_configure(p.smem, p.threads)) {
        set_error(FDTD_ERR_CUDA, "streaming Yee kernel: blocks of %d threads with %zu bytes of shared memory cannot launch",
                  p.threads, p.smem);
        return false;
    }
    CK(cudaStreamSynchronize(g->st));
    dfree(g->d_tiles);
    if (!dalloc(&g->d_tiles, p.tiles.size() * sizeof(StreamTile), g->st, false)) return false;
    CK(cudaMemcpyAsync(g->d_tiles, p.tiles.data(), p.tiles.size() * sizeof(StreamTile), cudaMemcpyHostToDevice, g->st));
    g->splan = std::move(p);
    std::copy(key, key + 6, g->splan_key);
    g->version++;
    return true;
}

// FP32 E-update coefficients of the fused path: cb = main/dx, ca = main*coef,
// main = 1/(ep/dt + sig/2), coef = ep/dt - sig/2, computed in double.
__global__ void k_coef(const float *ep, const float *sig, float *cb, float *ca, long long n, double dt, double dx)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        double e = ep[q], s = sig ? sig[q] : 0.0;
        double main_coeff = 1.0 / (e / dt + 0.5 * s);
        cb[q] = (float)(main_coeff / dx);
        if (ca) ca[q] = (float)(main_coeff * (e / dt - 0.5 * s));
    }
}

bool grid_prepare_step(Grid *g, double dt)
{
    if (!grid_ensure_device(g)) return false;
    if (!(dt > 0) || !std::isfinite(dt)) {
        set_error(FDTD_ERR_ARG, "delta_t must be positive and finite (got %g)", dt);
        return false;
    }
    const bool fused = pingpong_path(g);
    if (g->boundary == FDTD_BOUNDARY_MUR) {
        size_t bytes = (size_t)g->n * esize(g);
        for (int m = 0; m < 6; m++)
            if (!dalloc(&g->old[m], bytes, g->st)) return false;
    }
    if (g->boundary == FDTD_BOUNDARY_CPML) {
        if (g->L <= 0) {
            set_error(FDTD_ERR_ARG, "CPML boundary selected without timefield3d_set_cpml");
            return false;
        }
        if (2 * g->L + 2 > g->nx || 2 * g->L + 2 > g->ny || 2 * g->L + 2 > g->nz) {
            set_error(FDTD_ERR_ARG, "CPML thickness %d too large for grid %dx%dx%d", g->L, g->nx, g->ny, g->nz);
            return false;
        }
        size_t L2 = 2 * (size_t)g->L, es = esize(g);
        size_t sz[3] = {L2 * g->ny * g->nz * es, (size_t)g->nx * L2 * g->nz * es, (size_t)g->nx * g->ny * L2 * es};
        for (int s = 0; s < (fused ? 2 : 1); s++)
            for (int a = 0; a < 3; a++)
                for (int w = 0; w < 4; w++)
                    if (!dalloc(&g->psi[s][a][w], sz[a], g->st)) return false;
        if (g->prof_dt != dt && !build_profiles(g, dt)) return false;
    }
    if (fused) {
        if (!g->f[1][0]) {
            if (!alloc_field_set(g, 1)) return false;
            g->pp_synced = false;
        }
        if (!g->pp_synced) {
            // the fused kernel writes only interior cells: start both sets equal
            const int a = g->cur, b = 1 - g->cur;
            const size_t fb = (size_t)g->n * sizeof(float);
            for (int m = 0; m < 6; m++) CK(cudaMemcpyAsync(g->f[b][m], g->f[a][m], fb, cudaMemcpyDeviceToDevice, g->st));
            if (g->boundary == FDTD_BOUNDARY_CPML) {
                size_t L2 = 2 * (size_t)g->L;
                size_t sz[3] = {L2 * g->ny * g->nz, (size_t)g->nx * L2 * g->nz, (size_t)g->nx * g->ny * L2};
                for (int ax = 0; ax < 3; ax++)
                    for (int w = 0; w < 4; w++)
                        CK(cudaMemcpyAsync(g->psi[b][ax][w], g->psi[a][ax][w], sz[ax] * sizeof(float),
                                           cudaMemcpyDeviceToDevice, g->st));
            }
            g->pp_synced = true;
        }
    }
    if (fast32_path(g)) {
        if (!g->coef_valid || g->coef_dt != dt) {
            size_t fb = (size_t)g->n * sizeof(float);
            for (int c = 0; c < 3; c++) {
                if (!dalloc(&g->cb[c], fb, g->st, false)) return false;
                if (g->sig_e && !dalloc(&g->ca[c], fb, g->st, false)) return false;
                int blocks = (int)std::min<long long>((g->n + 255) / 256, 4736);
                note_launch();
                k_coef<<<blocks, 256, 0, g->st>>>(g->ep[c], g->sig_e ? g->sig[c] : nullptr, g->cb[c],
                                                    g->sig_e ? g->ca[c] : nullptr, g->n, dt, g->dx);
                CKL("k_coef");
            }
            g->coef_valid = true;
            g->coef_dt = dt;
            delete g->fmaps[0];
            delete g->fmaps[1];
            g->fmaps[0] = g->fmaps[1] = nullptr;
            g->version++;
        }
        if (stream_path(g) && !stream_prepare(g)) return false;
        // TMA descriptors of the fused kernel (host-side encode; they only depend on the buffers)
        if (fused_path(g) && !g->fmaps[0] && fused_tma_supported(g->nx, g->ny, g->nz)) {
            {
                for (int s = 0; s < 2; s++) {
                    FusedMaps *m = new FusedMaps();
                    const float *ca3[3] = {g->sig_e ? g->ca[0] : nullptr, g->sig_e ? g->ca[1] : nullptr,
                                           g->sig_e ? g->ca[2] : nullptr};
                    if (!fused_make_maps(m, (const float *const *)g->f[s], g->cb, ca3, g->nx, g->ny, g->nz)) {
                        delete m;
                        m = nullptr;
                    }
                    g->fmaps[s] = m;
                }
                if (!g->fmaps[0] || !g->fmaps[1]) {
                    delete g->fmaps[0];
                    delete g->fmaps[1];
                    g->fmaps[0] = g->fmaps[1] = nullptr;
                }
            }
            g->version++;
        }
    }
    // overlap scratch for the monitors
    int parts = overlap_parts((long long)g->nx * g->ny);
    int need = std::max<int>(1, (int)g->monitors.size());
    if (g->jobs_cap < need) {
        dfree(g->d_jobs);
        dfree(g->d_partials);
        g->jobs_cap = std::max(need, 8);
    }
    if (!dalloc(&g->d_jobs, g->jobs_cap * sizeof(OverlapJob), g->st, false)) return false;
    if (!dalloc(&g->d_partials, (size_t)g->jobs_cap * parts * sizeof(double2), g->st, false)) return false;
    return true;
}

Plane *grid_plane(Grid *g, int k, bool create)
{
    for (auto &p : g->planes)
        if (p.k == k) return &p;
    if (!create) return nullptr;
    if ((int)g->planes.size() >= kMaxSourcePlanes) {
        set_error(FDTD_ERR_UNSUPPORTED, "more than %d z-planes hold sources (zero the grid to reset them)",
                  kMaxSourcePlanes);
        return nullptr;
    }
    size_t bytes = 6 * (size_t)g->nx * g->ny * sizeof(float);
    float *p = nullptr;
    if (!g->plane_pool.empty()) {
        p = g->plane_pool.back();
        g->plane_pool.pop_back();
    } else if (!cuda_ok(cudaMalloc(&p, bytes), "cudaMalloc(plane)")) {
        return nullptr;
    }
    if (!cuda_ok(cudaMemsetAsync(p, 0, bytes, g->st), "cudaMemsetAsync(plane)")) return nullptr;
    g->planes.push_back(Plane{k, p});
    g->version++;
    return &g->planes.back();
}

void grid_zero(Grid *g)
{
    // timefield3d_zero_fields (timefield3d.c:108-121): fields, old fields,
    // DFT accumulators and sources; plus the engine's CPML memory, monitors,
    // probes and step counter
    g->host_steps = 0;
    if (!g->dev) return;
    size_t es = esize(g);
    for (int s = 0; s < 2; s++)
        for (int m = 0; m < 6; m++) {
            if (g->f[s][m]) cudaMemsetAsync(g->f[s][m], 0, (size_t)g->n * es, g->st);
        }
    for (int m = 0; m < 6; m++)
        if (g->old[m]) cudaMemsetAsync(g->old[m], 0, (size_t)g->n * es, g->st);
    size_t L2 = 2 * (size_t)g->L;
    size_t sz[3] = {L2 * g->ny * g->nz * es, (size_t)g->nx * L2 * g->nz * es, (size_t)g->nx * g->ny * L2 * es};
    for (int s = 0; s < 2; s++)
        for (int a = 0; a < 3; a++)
            for (int w = 0; w < 4; w++)
                if (g->psi[s][a][w]) cudaMemsetAsync(g->psi[s][a][w], 0, sz[a], g->st);
    for (auto &p : g->planes) g->plane_pool.push_back(p.p);
    g->planes.clear();
    if (g->d_dft_full) cudaMemsetAsync(g->d_dft_full, 0, (size_t)g->n * 6 * sizeof(double2), g->st);
    for (auto &kv : g->d_dft_slice) cudaMemsetAsync(kv.second, 0, (size_t)g->nx * g->nz * 6 * sizeof(double2), g->st);
    for (auto &mn : g->monitors) cudaMemsetAsync(mn.d_acc, 0, 2 * mn.nfreq * sizeof(double2), g->st);
    if (g->d_probe_count) cudaMemsetAsync(g->d_probe_count, 0, g->probes.size() * sizeof(int), g->st);
    cudaMemsetAsync(g->d_step, 0, sizeof(long long), g->st);
    g->version++;
    cuda_ok(cudaGetLastError(), "timefield3d_zero_fields");
}

// ---------------------------------------------------------------------------
// the step
// ---------------------------------------------------------------------------
template <typename T> static bool step_split(Grid *g, double dt)
{
    GridView<T> v = view<T>(g, g->cur);
    CpmlView<T> c = cpml_view<T>(g, g->cur);
    SourcePlanes s = source_table(g);
    const T tdt = (T)dt, div = (T)(1 / (g->dx)), tdx = (T)g->dx;
    const bool cpml = g->boundary == FDTD_BOUNDARY_CPML;
    if (g->boundary == FDTD_BOUNDARY_MUR) launch_save_shell<T>(v, g->st);
    launch_update_E<T>(v, c, s, tdt, div, 1, g->nz - 1, g->sig_e, cpml, false, g->st);
    if (g->boundary == FDTD_BOUNDARY_MUR) launch_mur<T>(v, tdt, tdx, 1, 0, g->nz, g->st);
    launch_update_H<T>(v, c, s, tdt, div, 1, g->nz - 1, g->sig_m, g->mu_nonunit, cpml, false, g->st);
    if (g->boundary == FDTD_BOUNDARY_MUR) launch_mur<T>(v, tdt, tdx, 0, 0, g->nz, g->st);
    CKL("step");
    return true;
}

static FlatArgs flat_args(Grid *g, double dt)
{
    FlatArgs a{};
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    for (int m = 0; m < 6; m++) a.f[m] = (float *)g->f[g->cur][m];
    for (int c = 0; c < 3; c++) { a.cb[c] = g->cb[c]; a.ca[c] = g->sig_e ? g->ca[c] : nullptr; }
    a.hb = (float)(dt / g->dx);
    a.dx = (float)g->dx;
    a.L = g->boundary == FDTD_BOUNDARY_CPML ? g->L : 0;
    for (int ax = 0; ax < 3; ax++) {
        for (int w = 0; w < 4; w++) a.psi[ax][w] = (float *)g->psi[g->cur][ax][w];
        for (int w = 0; w < 6; w++) a.prof[w][ax] = (const float *)g->prof[w][ax];
    }
    a.src = source_table(g);
    a.ring = nullptr;
    a.ring_k = -1;
    return a;
}

static bool step_flat(Grid *g, double dt)
{
    const FlatArgs a = flat_args(g, dt);
    const bool four = g->yee_variant != FDTD_YEE_FLAT && flat4_supported(g->nx, g->nz);
    if (four) launch_flat4_step(a, g->st, g->side, g->ev_fork, g->ev_join);
    else launch_flat_step(a, g->st, nullptr);
    CKL("flat step");
    return true;
}

static bool step_fused(Grid *g, double dt)
{
    FusedArgs a{};
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    const int in = g->cur, out = 1 - g->cur;
    for (int m = 0; m < 6; m++) { a.f_in[m] = (const float *)g->f[in][m]; a.f_out[m] = (float *)g->f[out][m]; }
    for (int c = 0; c < 3; c++) { a.cb[c] = g->cb[c]; a.ca[c] = g->sig_e ? g->ca[c] : nullptr; }
    a.hb = (float)(dt / g->dx);
    a.dx = (float)g->dx;
    a.L = g->boundary == FDTD_BOUNDARY_CPML ? g->L : 0;
    for (int ax = 0; ax < 3; ax++) {
        for (int w = 0; w < 4; w++) {
            a.psi_in[ax][w] = (const float *)g->psi[in][ax][w];
            a.psi_out[ax][w] = (float *)g->psi[out][ax][w];
        }
        for (int w = 0; w < 6; w++) a.prof[w][ax] = (const float *)g->prof[w][ax];
    }
    a.src = source_table(g);
    if (g->fmaps[in]) launch_fused_step_tma(a, *g->fmaps[in], g->d_err, g->st);
    else launch_fused_step(a, g->st);
    CKL("fused step");
    g->cur = out;
    return true;
}

static bool step_stream(Grid *g, double dt)
{
    StreamArgs a{};
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    a.L = g->boundary == FDTD_BOUNDARY_CPML ? g->L : 0;
    a.ty = g->splan.ty;
    const int in = g->cur, out = 1 - g->cur;
    for (int m = 0; m < 6; m++) { a.f_in[m] = (const float *)g->f[in][m]; a.f_out[m] = (float *)g->f[out][m]; }
    for (int c = 0; c < 3; c++) { a.cb[c] = g->cb[c]; a.ca[c] = g->sig_e ? g->ca[c] : nullptr; }
    a.hb = (float)(dt / g->dx);
    a.dx = (float)g->dx;
    for (int ax = 0; ax < 3; ax++) {
        for (int w = 0; w < 4; w++) {
            a.psi_in[ax][w] = (const float *)g->psi[in][ax][w];
            a.psi_out[ax][w] = (float *)g->psi[out][ax][w];
        }
        for (int w = 0; w < 6; w++) a.prof[w][ax] = (const float *)g->prof[w][ax];
    }
    a.src = source_table(g);
    a.tiles = g->d_tiles;
    launch_yee_stream(a, g->splan, g->st);
    CKL("streaming step");
    g->cur = out;
    return true;
}

static bool schedule_job(Grid *g, SourceJob *sj);

bool enqueue_after_step(Grid *g, double dt)
{
    const void *const *fp = (const void *const *)g->d_fptr[g->cur];
    const bool f64 = g->prec == FDTD_F64;
    if (!g->probes.empty()) {
        if (f64) launch_probes<double>((const double *const *)fp, g->d_probes, (int)g->probes.size(), g->d_probe_buf, g->probe_cap, g->d_probe_count, g->st);
        else launch_probes<float>((const float *const *)fp, g->d_probes, (int)g->probes.size(), g->d_probe_buf, g->probe_cap, g->d_probe_count, g->st);
    }
    const double scale = (-0.5 * g->dx * g->dx);
    if (g->njobs > 0 && !g->in_run) {
        if (f64)
            launch_overlap<double>((const double *const *)fp, g->nx, g->ny, g->d_jobs, g->njobs, g->job_cells,
                                   g->d_partials, scale, dt, g->d_step, 0, g->st);
        else
            launch_overlap<float>((const float *const *)fp, g->nx, g->ny, g->d_jobs, g->njobs, g->job_cells,
                                  g->d_partials, scale, dt, g->d_step, 0, g->st);
    }
    for (auto &b : g->binds) {
        TaperDev *td = nullptr;
        adjoint3d_taper key{};
        key.left = (int *)b.taper_key;
        td = taper_lookup(key, false);
        if (!td) continue;
        if (!enqueue_taper_store(td, g, b.which, 0, g->d_step, b.t0, b.dir)) return false;
    }
    if (!g->in_run) {
        launch_step_advance(g->d_step, g->st);
    } else {
        // overlaps of this step, scheduled source of the next, counter: one launch
        TailArgs t{};
        t.f = fp;
        t.nx = g->nx; t.ny = g->ny;
        t.jobs = g->d_jobs; t.njobs = g->njobs;
        t.cells = g->job_cells;
        t.partials = g->d_partials;
        t.scale = scale; t.dt = dt;
        t.step = g->d_step;
        t.done = g->d_done;
        if (g->sched.active && !schedule_job(g, &t.src)) return false;
        if (f64) launch_step_tail<double>(t, g->st);
        else launch_step_tail<float>(t, g->st);
    }
    CKL("after step");
    return true;
}

bool rebuild_jobs(Grid *g)
{
    std::vector<OverlapJob> jobs;
    for (auto &mn : g->monitors) {
        auto it = priv_modes().find(mn.mode_key);
        if (it == priv_modes().end()) continue;
        OverlapJob j{};
        j.cx = mn.cx; j.cy = mn.cy; j.cz = mn.cz;
        j.mi = it->second.mi; j.mj = it->second.mj;
        j.reverse = mn.reverse;
        j.ratio = g->dx / it->second.disc;
        j.mode = it->second.d;
        j.inst = nullptr;
        j.acc = mn.d_acc;
        j.omega = mn.d_omega;
        j.nfreq = mn.nfreq;
        j.win = mode_window(g->nx, g->ny, j.cx, j.cy, j.mi, j.mj, j.ratio);
        jobs.push_back(j);
    }
    g->njobs = (int)jobs.size();
    g->job_z.clear();
    for (auto &j : jobs) g->job_z.push_back(j.cz);
    g->job_cells = 0;
    for (auto &j : jobs) g->job_cells = std::max(g->job_cells, (long long)j.win.wni * j.win.wnj);
    if (g->njobs)
        CK(cudaMemcpyAsync(g->d_jobs, jobs.data(), jobs.size() * sizeof(OverlapJob), cudaMemcpyHostToDevice, g->st));
    g->version++;
    return true;
}

// the scheduled source as a SourceJob (its plane must exist)
static bool schedule_job(Grid *g, SourceJob *sj)
{
    auto it = priv_modes().find(g->sched.mode_key);
    Plane *pl = grid_plane(g, g->sched.cz, false);
    if (it == priv_modes().end() || !pl) {
        set_error(FDTD_ERR_ARG, "scheduled source not prepared");
        return false;
    }
    const long long off = (long long)g->nx * g->ny * g->sched.cz;
    *sj = SourceJob{};
    sj->plane = pl->p;
    for (int c = 0; c < 3; c++) { sj->ep[c] = g->ep[c] + off; sj->mu[c] = g->mu[c] + off; }
    sj->nx = g->nx; sj->ny = g->ny; sj->cx = g->sched.cx; sj->cy = g->sched.cy;
    sj->mode = it->second.d; sj->mi = it->second.mi; sj->mj = it->second.mj;
    sj->ratio = g->dx / it->second.disc;
    sj->sched = g->sched.d_sched; sj->nsched = g->sched.n;
    sj->reverse = g->sched.reverse; sj->adjoint = g->sched.adjoint;
    sj->kappa = g->sched.kappa; sj->wre = g->sched.wre; sj->wim = g->sched.wim;
    return true;
}

// write the scheduled source of step (counter + offset)
static bool enqueue_schedule(Grid *g, int offset)
{
    SourceJob sj;
    if (!schedule_job(g, &sj)) return false;
    launch_mode_source_job(sj, 0, 0, 0, g->d_step, offset, g->st);
    return true;
}

bool enqueue_step(Grid *g, double dt, bool with_extras)
{
    // inside a run the previous step's tail kernel wrote this step's source
    if (g->sched.active && !g->in_run && !enqueue_schedule(g, 0)) return false;
    bool ok;
    // External: captured as an event-record node whose timestamp the host can
    // read after a replay (a plain record during capture is only a dependency)
    if (g->cap_ev) CK(cudaEventRecordWithFlags(g->cap_ev[2 * g->cap_step], g->st, cudaEventRecordExternal));
    if (g->prec == FDTD_F64) ok = step_split<double>(g, dt);
    else if (stream_path(g)) ok = step_stream(g, dt);
    else if (fused_path(g)) ok = step_fused(g, dt);
    else if (fast32_path(g)) ok = step_flat(g, dt);
    else ok = step_split<float>(g, dt);
    if (!ok) return false;
    if (g->cap_ev) CK(cudaEventRecordWithFlags(g->cap_ev[2 * g->cap_step + 1], g->st, cudaEventRecordExternal));
    return with_extras ? enqueue_after_step(g, dt) : true;
}

// ============================================================================
// multi-step wavefront launches (FDTD_YEE_WAVE)
// ============================================================================
// A run's full chunks go through one wavefront launch per chunk when the grid
// is on the FP32 flat4 path and the run carries nothing that needs per-step
// kernels (probes, taper stores); monitors and the scheduled source are
// handled inside (their planes must be updated planes, 1..nz-2).
static bool wave_path(Grid *g, double dt)
{
    if (!fast32_path(g) || g->yee_variant != FDTD_YEE_WAVE) return false;
    if (!flat4_supported(g->nx, g->nz) || !g->probes.empty() || !g->binds.empty()) return false;
    const FlatArgs a = flat_args(g, dt);
    if (a.L > 0 && !flat4_split_supported(a)) return false;
    for (int z : g->job_z)
        if (z < 1 || z > g->nz - 2) return false;
    if (g->sched.active && (g->sched.cz < 1 || g->sched.cz > g->nz - 2)) return false;
    return true;
}

// (re)build the wavefront tables for the grid's current configuration
static bool wave_tables(Grid *g, const Plan4 &p)
{
    auto &w = g->wave;
    const int sched_k = g->sched.active ? g->sched.cz : -1;
    if (w.version == g->version && w.built_steps == w.steps && w.built_sweep == w.sweep && w.built_group == w.group &&
        w.built_sched_k == sched_k && w.d_items)
        return true;
    CK(cudaStreamSynchronize(g->st));
    dfree(w.d_items); dfree(w.d_cnt); dfree(w.d_part); dfree(w.d_ring);
    w.nparts = g->njobs ? overlap_parts(g->job_cells) : 1;
    if (wave_items(p, g->nz, w.steps, w.sweep, w.group, g->job_z.data(), g->njobs, w.nparts, w.items, w.tickets) !=
        0) {
        set_error(FDTD_ERR_ARG, "wavefront run: sizes out of range");
        return false;
    }
    for (int l = 0; l < 2; l++) {
        if (!w.grid[l]) w.grid[l] = wave_grid(l == 1);
        if (w.grid[l] <= 0) {
            set_error(FDTD_ERR_CUDA, "wavefront run: kernel cannot be resident on this device");
            return false;
        }
    }
    const long long nxy = (long long)g->nx * g->ny;
    if (!dalloc(&w.d_items, w.items.size() * sizeof(WaveItem), g->st, false)) return false;
    if (!dalloc(&w.d_cnt, ((size_t)wave_counters(g->nz, w.steps) + 1) * sizeof(unsigned), g->st)) return false;
    if (!dalloc(&w.d_part, (size_t)w.steps * std::max(1, g->njobs) * w.nparts * sizeof(double2), g->st)) return false;
    if (sched_k >= 0 && !dalloc(&w.d_ring, (size_t)w.steps * 6 * nxy * sizeof(float), g->st, false)) return false;
    CK(cudaMemcpyAsync(w.d_items, w.items.data(), w.items.size() * sizeof(WaveItem), cudaMemcpyHostToDevice, g->st));
    w.version = g->version;
    w.built_steps = w.steps;
    w.built_sweep = w.sweep;
    w.built_group = w.group;
    w.built_sched_k = sched_k;
    return true;
}

// one wavefront launch of g->wave.steps steps; `timed`: event pair `set` around it
static bool enqueue_wave(Grid *g, double dt, bool timed, int set)
{
    FlatArgs a = flat_args(g, dt);
    const Plan4 p = flat4_plan(a);
    if (!wave_tables(g, p)) return false;
    auto &w = g->wave;
    WaveArgs wa{};
    wa.items = w.d_items;
    wa.nitems = (int)w.items.size();
    wa.tickets = w.tickets;
    wa.cnt = w.d_cnt;
    wa.next = w.d_cnt + wave_counters(g->nz, w.steps);
    wa.nz = g->nz;
    wa.steps = w.steps;
    wa.jobs = g->d_jobs;
    wa.njobs = g->njobs;
    wa.nparts = w.nparts;
    wa.partials = w.d_part;
    wa.group = w.group;
    wa.err = g->d_err;
    wa.wait_ns = 1000000000ull;
    WaveFinal fin{};
    fin.jobs = g->d_jobs;
    fin.njobs = g->njobs;
    fin.nparts = w.nparts;
    fin.steps = w.steps;
    fin.partials = w.d_part;
    fin.scale = (-0.5 * g->dx * g->dx);
    fin.dt = dt;
    fin.step = g->d_step;
    fin.done = g->d_done;
    SourceJob sj{};
    if (g->sched.active) {
        if (!schedule_job(g, &sj)) return false;
        fin.src = sj;
        a.ring_k = g->sched.cz;
    }
    if (timed) {
        for (int e = 0; e < 2; e++)
            if (!w.ev[set][e]) CK(cudaEventCreate(&w.ev[set][e]));
        CK(cudaEventRecord(w.ev[set][0], g->st));
    }
    CK(launch_wave(a, p, wa, w.grid[a.ca[0] ? 1 : 0], g->sched.active ? &sj : nullptr, w.d_ring, fin, g->st));
    if (timed) {
        CK(cudaEventRecord(w.ev[set][1], g->st));
        w.pending[set] = true;
        w.timed_steps[set] = w.steps;
    }
    return true;
}

static bool prepare_run(Grid *g, double dt)
{
    if (!grid_prepare_step(g, dt)) return false;
    if (!rebuild_jobs(g)) return false;
    if (g->sched.active && !grid_plane(g, g->sched.cz, true)) return false;
    for (auto &b : g->binds) {
        adjoint3d_taper key{};
        key.left = (int *)b.taper_key;
        TaperDev *td = taper_lookup(key, false);
        if (!td) {
            set_error(FDTD_ERR_ARG, "bound taper no longer exists");
            return false;
        }
        if (td->prec != g->prec || !td->d_cells) {
            set_error(FDTD_ERR_ARG, "bound taper not prepared for this grid");
            return false;
        }
    }
    return true;
}

static constexpr int kGraphSteps = 32;   // steps per captured graph (even: the fused path ping-pongs)

// capture kGraphSteps steps into g->graph[slot]; slots 1 and 2 also record an
// event pair around each step's Yee update (kernel timing)
static bool capture_graph(Grid *g, int slot, double dt)
{
    if (g->graph[slot] && g->graph_steps[slot] == kGraphSteps && g->graph_dt[slot] == dt &&
        g->graph_version[slot] == g->version && g->graph_cur[slot] == g->cur)
        return true;
    if (g->graph[slot]) {
        CK(cudaStreamSynchronize(g->st));
        cudaGraphExecDestroy(g->graph[slot]);
        g->graph[slot] = nullptr;
    }
    if (slot > 0) {
        for (int e = 0; e < 2 * kGraphSteps; e++)
            if (!g->kev[slot - 1][e]) CK(cudaEventCreate(&g->kev[slot - 1][e]));
        g->kpending[slot - 1] = false;
        g->cap_ev = g->kev[slot - 1];
    }
    const int cur0 = g->cur;
    const long long before = launch_count();
    cudaGraph_t gr;
    CK(cudaStreamBeginCapture(g->st, cudaStreamCaptureModeThreadLocal));
    bool ok = true;
    for (int s = 0; s < kGraphSteps && ok; s++) {
        g->cap_step = s;
        ok = enqueue_step(g, dt, true);
    }
    g->cap_ev = nullptr;
    cudaError_t ce = cudaStreamEndCapture(g->st, &gr);
    const long long nodes = launch_count() - before;
    note_launch((int)-nodes);   // captured, not executed
    if (!ok) {
        if (ce == cudaSuccess) cudaGraphDestroy(gr);
        g->cur = cur0;
        return false;
    }
    CK(ce);
    cudaError_t ie = cudaGraphInstantiate(&g->graph[slot], gr, 0);
    cudaGraphDestroy(gr);
    CK(ie);
    g->graph_steps[slot] = kGraphSteps;
    g->graph_dt[slot] = dt;
    g->graph_version[slot] = g->version;
    g->graph_cur[slot] = cur0;
    g->graph_nodes[slot] = nodes;
    if (g->cur != cur0) {
        set_error(FDTD_ERR_CUDA, "internal: odd graph length");
        return false;
    }
    return true;
}

// read the Yee-update times of timed graph (or wavefront launch) `set` once
// it has completed
bool drain_kernel_timing(Grid *g, int set)
{
    auto &w = g->wave;
    if (w.pending[set]) {
        CK(cudaEventSynchronize(w.ev[set][1]));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, w.ev[set][0], w.ev[set][1]));
        g->ktime_ms += ms;
        g->ktime_n += w.timed_steps[set];
        w.pending[set] = false;
    }
    if (!g->kpending[set]) return true;
    CK(cudaEventSynchronize(g->kev[set][2 * kGraphSteps - 1]));
    for (int s = 0; s < kGraphSteps; s++) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, g->kev[set][2 * s], g->kev[set][2 * s + 1]));
        g->ktime_ms += ms;
        g->ktime_n++;
    }
    g->kpending[set] = false;
    return true;
}

static bool run_steps_in(Grid *g, double dt, int nsteps);

// ============================================================================
// candidate sweeps: many grids in persistent launches (yee_sweep.cu)
// ============================================================================
bool run_sweep(const std::vector<Grid *> &gs, double dt, const std::vector<int> &nsteps, int steps_per_launch,
               int ty_cap, double tiles_per_sm)
{
    const int ng = (int)gs.size();
    if (ng <= 0 || ng > kSweepMaxGrids || (int)nsteps.size() != ng || steps_per_launch < 1 ||
        steps_per_launch > 4096 || ty_cap < 0 || !(tiles_per_sm > 0) || tiles_per_sm > 16) {
        set_error(FDTD_ERR_ARG, "sweep: grids not in [1, %d], or steps_per_launch not in [1, 4096], ty_cap < 0, or "
                                "tiles_per_sm not in (0, 16]",
                  kSweepMaxGrids);
        return false;
    }
    int nsm = 0;
    if (!sweep_setup(&nsm)) return false;
    const Grid *g0 = gs[0];
    const int L0 = g0->boundary == FDTD_BOUNDARY_CPML ? g0->L : 0;
    for (int i = 0; i < ng; i++) {
        Grid *g = gs[i];
        for (int k = 0; k < i; k++)
            if (gs[k] == g) {
                set_error(FDTD_ERR_ARG, "sweep: grid %d appears twice", i);
                return false;
            }
        const int L = g->boundary == FDTD_BOUNDARY_CPML ? g->L : 0;
        if (nsteps[i] < 0 || !fast32_path(g) || L != L0 || g->sig_e != g0->sig_e || !g->probes.empty() ||
            !g->binds.empty() || !stream_supported(g->nx, g->ny, g->nz, g->sig_e, L)) {
            set_error(FDTD_ERR_UNSUPPORTED,
                      "sweep: grid %d must be FP32 with a CPML (or PEC walls) like grid 0, the same loss, no probes or "
                      "bound tapers, nx a multiple of 4, and nsteps >= 0",
                      i);
            return false;
        }
    }
    // every grid on the one-pass path (two field and auxiliary sets), prepared
    // as for timefield3d_run; the first step's scheduled source written
    cudaStream_t sst = sweep_stream();
    for (Grid *g : gs) {
        if (g->yee_variant != FDTD_YEE_STREAM) {
            g->yee_variant = FDTD_YEE_STREAM;
            g->pp_synced = false;
            g->version++;
        }
        if (!prepare_run(g, dt)) return false;
        if (g->sched.active && !enqueue_schedule(g, 0)) return false;
        CK(cudaEventRecord(g->ev_fork, g->st));
        CK(cudaStreamWaitEvent(sst, g->ev_fork, 0));
    }
    // tile plans: each grid's share of nsm * tiles_per_sm tiles in proportion to its cells
    double total = 0;
    for (Grid *g : gs) total += (double)g->n;
    std::vector<StreamPlan> plans(ng);
    int threads = 0;
    size_t smem = 0, ntile = 0, npart = 0;
    std::vector<size_t> toff(ng), poff(ng);
    std::vector<int> nparts(ng);
    for (int i = 0; i < ng; i++) {
        Grid *g = gs[i];
        const int share = std::max(1, (int)std::lround(nsm * tiles_per_sm * (double)g->n / total));
        if (!stream_plan(g->nx, g->ny, g->nz, L0, g->sig_e, share, &plans[i], ty_cap)) {
            set_error(FDTD_ERR_UNSUPPORTED, "sweep: no tile plan for grid %d", i);
            return false;
        }
        threads = std::max(threads, plans[i].threads);
        smem = std::max(smem, plans[i].smem);
        toff[i] = ntile;
        ntile += plans[i].tiles.size();
        nparts[i] = g->njobs > 0 ? overlap_parts(g->job_cells) : 0;
        poff[i] = npart;
        npart += 2 * (size_t)g->njobs * nparts[i];
    }
    StreamTile **dt_tiles = sweep_tiles(ntile * sizeof(StreamTile));
    double2 **dt_parts = sweep_partials(std::max<size_t>(npart, 1) * sizeof(double2));
    if (!dt_tiles || !dt_parts) return false;
    std::vector<StreamTile> all;
    for (auto &p : plans) all.insert(all.end(), p.tiles.begin(), p.tiles.end());
    CK(cudaStreamSynchronize(sst));   // the previous sweep no longer reads the tables
    CK(cudaMemcpyAsync(*dt_tiles, all.data(), all.size() * sizeof(StreamTile), cudaMemcpyHostToDevice, sst));
    // per grid, the launch-independent part of its entry
    std::vector<SweepGrid> proto(ng);
    for (int i = 0; i < ng; i++) {
        Grid *g = gs[i];
        SweepGrid &e = proto[i];
        e = SweepGrid{};
        for (int p = 0; p < 2; p++) {
            StreamArgs &a = e.args[p];
            a.nx = g->nx; a.ny = g->ny; a.nz = g->nz; a.L = L0; a.ty = plans[i].ty;
            for (int m = 0; m < 6; m++) { a.f_in[m] = (const float *)g->f[p][m]; a.f_out[m] = (float *)g->f[1 - p][m]; }
            for (int c = 0; c < 3; c++) { a.cb[c] = g->cb[c]; a.ca[c] = g->sig_e ? g->ca[c] : nullptr; }
            a.hb = (float)(dt / g->dx);
            a.dx = (float)g->dx;
            for (int ax = 0; ax < 3; ax++) {
                for (int w = 0; w < 4; w++) {
                    a.psi_in[ax][w] = (const float *)g->psi[p][ax][w];
                    a.psi_out[ax][w] = (float *)g->psi[1 - p][ax][w];
                }
                for (int w = 0; w < 6; w++) a.prof[w][ax] = (const float *)g->prof[w][ax];
            }
            a.src = source_table(g);
            a.tiles = *dt_tiles + toff[i];
            e.fout[p] = (const float *const *)g->d_fptr[1 - p];
        }
        e.ntiles = (int)plans[i].tiles.size();
        e.nx = g->nx; e.ny = g->ny;
        e.jobs = g->d_jobs;
        e.njobs = g->njobs;
        e.nparts = nparts[i];
        e.partials = *dt_parts + poff[i];
        e.scale = -0.5 * g->dx * g->dx;
        e.dt = dt;
        e.step = g->d_step;
        if (g->sched.active) {
            if (!schedule_job(g, &e.src)) return false;
            e.src.win = mode_window(e.src.nx, e.src.ny, e.src.cx, e.src.cy, e.src.mi, e.src.mj, e.src.ratio);
            const long long cells = (long long)e.src.win.wni * e.src.win.wnj;
            e.src_warps = (int)std::max<long long>(1, std::min<long long>((cells + 31) / 32, 4 * 384));
        }
    }
    // launches of steps_per_launch steps until every grid has run its own count
    const int most = *std::max_element(nsteps.begin(), nsteps.end());
    std::vector<std::vector<SweepGrid>> launches;
    std::vector<int> lsteps;
    for (int l0 = 0; l0 < most; l0 += steps_per_launch) {
        std::vector<SweepGrid> row(proto);
        int lmax = 0;
        for (int i = 0; i < ng; i++) {
            row[i].steps = std::max(0, std::min(steps_per_launch, nsteps[i] - l0));
            row[i].base = gs[i]->host_steps + std::min(l0, nsteps[i]);
            row[i].p0 = (gs[i]->cur + std::min(l0, nsteps[i])) & 1;
            lmax = std::max(lmax, row[i].steps);
        }
        launches.push_back(std::move(row));
        lsteps.push_back(lmax);
    }
    // every grid's tiles, most expensive first (the blocks take them in this order)
    std::vector<std::pair<double, int2>> order;
    for (int i = 0; i < ng; i++)
        for (int t = 0; t < (int)plans[i].tiles.size(); t++)
            order.push_back({stream_tile_cost(gs[i]->nx, gs[i]->ny, gs[i]->nz, L0, plans[i].tiles[t]), make_int2(i, t)});
    std::stable_sort(order.begin(), order.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
    std::vector<int2> items;
    for (auto &o : order) items.push_back(o.second);
    // staged rows of the tiles, when every grid's plan has the same
    int tpc = plans[0].ty + 1;
    for (int i = 1; i < ng; i++)
        if (plans[i].ty + 1 != tpc) tpc = 0;
    if (!launches.empty() &&
        !sweep_launch(launches, lsteps, items, L0 > 0, g0->sig_e, tpc, threads, smem, 1000000000ull))
        return false;
    // the grids' own streams continue after the sweep
    CK(cudaEventRecord(sweep_event(), sst));
    for (int i = 0; i < ng; i++) {
        Grid *g = gs[i];
        CK(cudaStreamWaitEvent(g->st, sweep_event(), 0));
        launch_sweep_err_to_grid(sweep_err(), g->d_err, g->st);
        g->cur = (g->cur + nsteps[i]) & 1;
        g->host_steps += nsteps[i];
        // as after timefield3d_run, the plane holds the last step's source
        if (g->sched.active && nsteps[i] > 0 && !enqueue_schedule(g, -1)) return false;
    }
    CKL("sweep");
    return true;
}

bool run_steps(Grid *g, double dt, int nsteps)
{
    if (nsteps <= 0) return true;
    if (!prepare_run(g, dt)) return false;
    // Each step of a run ends with the step-tail kernel, which also writes the
    // next step's scheduled source: prime the first one here, and afterwards
    // leave the plane holding the last step's source, as a stepwise loop would.
    if (g->sched.active && !enqueue_schedule(g, 0)) return false;
    g->in_run = true;
    const bool ok = run_steps_in(g, dt, nsteps);
    g->in_run = false;
    if (!ok) return false;
    if (g->sched.active && !enqueue_schedule(g, -1)) return false;
    return true;
}

static bool run_steps_in(Grid *g, double dt, int nsteps)
{
    if (nsteps >= g->wave.steps && wave_path(g, dt)) {
        // wavefront launches of wave.steps steps; one in g->ktime timed
        const int full = nsteps / g->wave.steps, rest = nsteps % g->wave.steps;
        for (int r = 0; r < full; r++, g->kreplay++) {
            const bool timed = g->ktime > 0 && g->kreplay % g->ktime == 0;
            const int set = g->ktime > 0 ? (int)((g->kreplay / g->ktime) & 1) : 0;
            if (timed && !drain_kernel_timing(g, set)) return false;
            if (!enqueue_wave(g, dt, timed, set)) return false;
        }
        for (int s = 0; s < rest; s++)
            if (!enqueue_step(g, dt, true)) return false;
        g->host_steps += nsteps;
        return true;
    }
    int full = nsteps / kGraphSteps, rest = nsteps % kGraphSteps;
    if (full > 0 && !g->ktime) {
        if (!capture_graph(g, 0, dt)) return false;
        for (int r = 0; r < full; r++) {
            CK(cudaGraphLaunch(g->graph[0], g->st));
            note_launch((int)g->graph_nodes[0]);
        }
    } else if (full > 0) {
        // One replay in g->ktime runs a timed graph, the others the plain one
        // (the event records of a timed graph stand between the step's
        // kernels, which then cannot overlap their launches).  Two timed
        // graphs alternate: while one runs, the host reads the other's event
        // times, so the device never waits for the host.
        if (!capture_graph(g, 1, dt) || !capture_graph(g, 2, dt)) return false;
        if (g->ktime > 1 && !capture_graph(g, 0, dt)) return false;
        for (int r = 0; r < full; r++, g->kreplay++) {
            if (g->kreplay % g->ktime != 0) {
                CK(cudaGraphLaunch(g->graph[0], g->st));
                note_launch((int)g->graph_nodes[0]);
                continue;
            }
            const int set = (int)((g->kreplay / g->ktime) & 1);
            if (!drain_kernel_timing(g, set)) return false;
            CK(cudaGraphLaunch(g->graph[1 + set], g->st));
            note_launch((int)g->graph_nodes[1 + set]);
            g->kpending[set] = true;
        }
    }
    for (int s = 0; s < rest; s++)
        if (!enqueue_step(g, dt, true)) return false;
    g->host_steps += nsteps;
    return true;
}

// ============================================================================
// tapers
// ============================================================================
static std::unordered_map<const void *, TaperDev *> &taper_table()
{
    static std::unordered_map<const void *, TaperDev *> t;
    return t;
}

TaperDev::~TaperDev()
{
    dfree(d_fwd);
    dfree(d_adj);
    dfree(d_cells);
    dfree(d_grad);
}

TaperDev *taper_lookup(const adjoint3d_taper &t, bool create)
{
    auto &tab = taper_table();
    auto it = tab.find(t.left);
    if (it != tab.end()) return it->second;
    if (!create) return nullptr;
    TaperDev *td = new TaperDev();
    td->key = t.left;
    tab[t.left] = td;
    return td;
}

void taper_unregister(const adjoint3d_taper &t)
{
    auto &tab = taper_table();
    auto it = tab.find(t.left);
    if (it == tab.end()) return;
    cudaDeviceSynchronize();
    delete it->second;
    tab.erase(it);
}

bool taper_prepare(TaperDev *td, const adjoint3d_taper &t, Grid *g)
{
    if (!grid_ensure_device(g)) return false;
    const int height = t.top - t.bottom, length = t.end - t.start;
    if (height <= 0 || length <= 0 || t.duration <= 0 || t.seg_num <= 0) {
        set_error(FDTD_ERR_ARG, "taper: empty storage box (height %d length %d duration %d seg_num %d)", height, length,
                  t.duration, t.seg_num);
        return false;
    }
    const int ncell = 2 * height * length;
    const bool resize = td->ncell != ncell || td->duration != t.duration || td->prec != g->prec;
    td->seg_num = t.seg_num; td->start = t.start; td->end = t.end; td->bottom = t.bottom; td->top = t.top;
    td->height = height; td->length = length;
    size_t es = g->prec == FDTD_F64 ? 8 : 4;
    if (resize) {
        cudaDeviceSynchronize();
        dfree(td->d_fwd);
        dfree(td->d_adj);
        dfree(td->d_cells);
        dfree(td->d_grad);
        td->ncell = ncell;
        td->duration = t.duration;
        td->prec = g->prec;
        td->edges_seen.clear();
        size_t bytes = (size_t)t.duration * ncell * 3 * es;
        if (!dalloc(&td->d_fwd, bytes, g->st) || !dalloc(&td->d_adj, bytes, g->st)) return false;
        if (!dalloc(&td->d_cells, ncell * sizeof(long long), g->st, false)) return false;
        if (!dalloc(&td->d_grad, ncell * sizeof(double), g->st)) return false;
    }
    std::vector<int> edges(t.left, t.left + t.seg_num + 1);
    edges.insert(edges.end(), t.right, t.right + t.seg_num + 1);
    if (edges != td->edges_seen || td->nx_seen != g->nx || td->ny_seen != g->ny) {
        // edge pixel of (edge, j, k): adjoint3d.c:268-296, integer division
        // inside round(), i.e. edge[n] + trunc(d (k - k0) / (k1 - k0))
        std::vector<long long> cells(ncell);
        for (int n = 0; n < t.seg_num; n++) {
            int seg_mid = t.start + (n * length) / t.seg_num;
            int seg_fwd = t.start + ((n + 1) * length) / t.seg_num;
            for (int k = seg_mid; k < seg_fwd; k++)
                for (int j = t.bottom; j < t.top; j++)
                    for (int e = 0; e < 2; e++) {
                        const int *edge = e == 0 ? t.right : t.left;
                        int i = edge[n] + ((edge[n + 1] - edge[n]) * (k - seg_mid)) / (seg_fwd - seg_mid);
                        if (i < 0 || i >= g->nx || j < 0 || j >= g->ny || k < 0 || k >= g->nz) {
                            set_error(FDTD_ERR_ARG, "taper edge pixel (%d,%d,%d) outside the grid", i, j, k);
                            return false;
                        }
                        cells[e + 2 * ((j - t.bottom) + (size_t)height * (k - t.start))] =
                            i + (long long)g->nx * (j + (long long)g->ny * k);
                    }
        }
        CK(cudaStreamSynchronize(g->st));
        CK(cudaMemcpy(td->d_cells, cells.data(), ncell * sizeof(long long), cudaMemcpyHostToDevice));
        td->edges_seen = edges;
        td->nx_seen = g->nx;
        td->ny_seen = g->ny;
    }
    return true;
}

bool enqueue_taper_store(TaperDev *td, Grid *g, int which, int t_index, const long long *d_step, int t0, int dir)
{
    const void *const *fp = (const void *const *)g->d_fptr[g->cur];
    void *store = which ? td->d_adj : td->d_fwd;
    if (g->prec == FDTD_F64)
        launch_taper_store<double>((const double *const *)fp, td->d_cells, td->ncell, (double *)store, t_index, d_step, t0, dir, td->duration, g->st);
    else
        launch_taper_store<float>((const float *const *)fp, td->d_cells, td->ncell, (float *)store, t_index, d_step, t0, dir, td->duration, g->st);
    CKL("taper store");
    return true;
}

// ============================================================================
// checkpoint / resume
// ============================================================================
// File: "FDTDCKP1", int32 nx ny nz precision boundary L n_monitors n_planes
// has_psi, int64 host_steps device_step, per monitor int32 nfreq + 2 nfreq
// double2, per plane int32 k + 6 nx ny float, the 6 field components of the
// current set (n elements of the grid's precision), then (has_psi) the 12
// CPML auxiliary arrays of the current set.  Materials, modes, schedules and
// monitor definitions are the caller's set-up and are not stored.
namespace {
struct FileCloser {
    FILE *f;
    ~FileCloser() { if (f) fclose(f); }
};
bool wr(FILE *f, const void *p, size_t n) { return fwrite(p, 1, n, f) == n; }
bool rd(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n; }
}  // namespace

static void psi_sizes(const Grid *g, size_t sz[3])
{
    const size_t L2 = 2 * (size_t)g->L, es = esize(g);
    sz[0] = L2 * g->ny * g->nz * es;
    sz[1] = (size_t)g->nx * L2 * g->nz * es;
    sz[2] = (size_t)g->nx * g->ny * L2 * es;
}

bool grid_checkpoint_save(Grid *g, const char *path)
{
    if (!grid_ensure_device(g)) return false;
    CK(cudaStreamSynchronize(g->st));
    FileCloser fc{fopen(path, "wb")};
    if (!fc.f) {
        set_error(FDTD_ERR_ARG, "checkpoint: cannot open %s for writing", path);
        return false;
    }
    const bool has_psi = g->boundary == FDTD_BOUNDARY_CPML && g->psi[g->cur][0][0];
    int hdr[9] = {g->nx, g->ny, g->nz, g->prec, g->boundary, g->L, (int)g->monitors.size(), (int)g->planes.size(),
                  has_psi ? 1 : 0};
    long long dstep = 0;
    CK(cudaMemcpyAsync(&dstep, g->d_step, sizeof(long long), cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    long long steps[2] = {g->host_steps, dstep};
    bool ok = wr(fc.f, "FDTDCKP1", 8) && wr(fc.f, hdr, sizeof hdr) && wr(fc.f, steps, sizeof steps);
    std::vector<char> buf;
    for (auto &mn : g->monitors) {
        buf.resize(2 * (size_t)mn.nfreq * sizeof(double2));
        CK(cudaMemcpyAsync(buf.data(), mn.d_acc, buf.size(), cudaMemcpyDeviceToHost, g->st));
        CK(cudaStreamSynchronize(g->st));
        ok = ok && wr(fc.f, &mn.nfreq, sizeof(int)) && wr(fc.f, buf.data(), buf.size());
    }
    const size_t pb = 6 * (size_t)g->nx * g->ny * sizeof(float);
    for (auto &pl : g->planes) {
        buf.resize(pb);
        CK(cudaMemcpyAsync(buf.data(), pl.p, pb, cudaMemcpyDeviceToHost, g->st));
        CK(cudaStreamSynchronize(g->st));
        ok = ok && wr(fc.f, &pl.k, sizeof(int)) && wr(fc.f, buf.data(), pb);
    }
    const size_t fb = (size_t)g->n * esize(g);
    buf.resize(fb);
    for (int m = 0; m < 6 && ok; m++) {
        CK(cudaMemcpyAsync(buf.data(), g->f[g->cur][m], fb, cudaMemcpyDeviceToHost, g->st));
        CK(cudaStreamSynchronize(g->st));
        ok = wr(fc.f, buf.data(), fb);
    }
    if (has_psi) {
        size_t sz[3];
        psi_sizes(g, sz);
        for (int a = 0; a < 3; a++)
            for (int w = 0; w < 4 && ok; w++) {
                buf.resize(sz[a]);
                CK(cudaMemcpyAsync(buf.data(), g->psi[g->cur][a][w], sz[a], cudaMemcpyDeviceToHost, g->st));
                CK(cudaStreamSynchronize(g->st));
                ok = wr(fc.f, buf.data(), sz[a]);
            }
    }
    if (!ok) {
        set_error(FDTD_ERR_ALLOC, "checkpoint: short write to %s", path);
        return false;
    }
    return true;
}

bool grid_checkpoint_load(Grid *g, const char *path)
{
    // The whole file is read and checked into host memory first; device state
    // is written only once every part is known to be present and to fit this
    // grid, so a refused or truncated file leaves the grid as it was.  Every
    // write then goes on the grid's stream (after the allocations' zero fills
    // on that stream) and is waited for before returning.
    if (!grid_ensure_device(g)) return false;
    CK(cudaStreamSynchronize(g->st));
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f) {
        set_error(FDTD_ERR_ARG, "checkpoint: cannot open %s", path);
        return false;
    }
    char magic[8];
    int hdr[9];
    long long steps[2];
    if (!rd(fc.f, magic, 8) || memcmp(magic, "FDTDCKP1", 8) != 0 || !rd(fc.f, hdr, sizeof hdr) ||
        !rd(fc.f, steps, sizeof steps)) {
        set_error(FDTD_ERR_ARG, "checkpoint: %s is not a checkpoint of this library", path);
        return false;
    }
    if (hdr[0] != g->nx || hdr[1] != g->ny || hdr[2] != g->nz || hdr[3] != g->prec || hdr[4] != g->boundary ||
        (g->boundary == FDTD_BOUNDARY_CPML && hdr[5] != g->L) || hdr[6] != (int)g->monitors.size()) {
        set_error(FDTD_ERR_ARG,
                  "checkpoint: saved grid %dx%dx%d precision %d boundary %d L %d with %d monitors does not match this "
                  "grid (%dx%dx%d precision %d boundary %d L %d, %d monitors)",
                  hdr[0], hdr[1], hdr[2], hdr[3], hdr[4], hdr[5], hdr[6], g->nx, g->ny, g->nz, g->prec, g->boundary,
                  g->L, (int)g->monitors.size());
        return false;
    }
    if (hdr[7] < 0 || hdr[7] > kMaxSourcePlanes || (hdr[8] && g->boundary != FDTD_BOUNDARY_CPML)) {
        set_error(FDTD_ERR_ARG, "checkpoint: %s has %d source planes / CPML flag %d, not valid for this grid", path,
                  hdr[7], hdr[8]);
        return false;
    }
    // ---- read everything
    std::vector<std::vector<char>> acc(g->monitors.size());
    for (size_t q = 0; q < g->monitors.size(); q++) {
        int nf = 0;
        if (!rd(fc.f, &nf, sizeof nf)) goto short_read;
        if (nf != g->monitors[q].nfreq) {
            set_error(FDTD_ERR_ARG, "checkpoint: monitor frequency count %d does not match %d", nf,
                      g->monitors[q].nfreq);
            return false;
        }
        acc[q].resize(2 * (size_t)nf * sizeof(double2));
        if (!rd(fc.f, acc[q].data(), acc[q].size())) goto short_read;
    }
    {
        const size_t pb = 6 * (size_t)g->nx * g->ny * sizeof(float);
        std::vector<int> pk(hdr[7]);
        std::vector<std::vector<char>> pdata(hdr[7]);
        for (int q = 0; q < hdr[7]; q++) {
            pdata[q].resize(pb);
            if (!rd(fc.f, &pk[q], sizeof(int)) || !rd(fc.f, pdata[q].data(), pb)) goto short_read;
            if (pk[q] < 0 || pk[q] >= g->nz) {
                set_error(FDTD_ERR_ARG, "checkpoint: source plane z = %d outside the grid", pk[q]);
                return false;
            }
        }
        const size_t fb = (size_t)g->n * esize(g);
        std::vector<std::vector<char>> fields(6);
        for (int m = 0; m < 6; m++) {
            fields[m].resize(fb);
            if (!rd(fc.f, fields[m].data(), fb)) goto short_read;
        }
        size_t sz[3] = {0, 0, 0};
        std::vector<std::vector<char>> psi;
        if (hdr[8]) {
            psi_sizes(g, sz);
            psi.resize(12);
            for (int a = 0; a < 3; a++)
                for (int w = 0; w < 4; w++) {
                    psi[4 * a + w].resize(sz[a]);
                    if (!rd(fc.f, psi[4 * a + w].data(), sz[a])) goto short_read;
                }
        }
        // ---- allocate what the file needs (the only step that can still fail
        //      before device state changes; new planes and auxiliaries start zero)
        std::vector<Plane *> pl(hdr[7]);
        for (int q = 0; q < hdr[7]; q++)
            if (!(pl[q] = grid_plane(g, pk[q], true))) return false;
        if (g->boundary == FDTD_BOUNDARY_CPML) {
            psi_sizes(g, sz);
            for (int a = 0; a < 3; a++)
                for (int w = 0; w < 4; w++)
                    if (!dalloc(&g->psi[g->cur][a][w], sz[a], g->st)) return false;
        }
        // ---- write device state, in stream order
        for (size_t q = 0; q < g->monitors.size(); q++)
            CK(cudaMemcpyAsync(g->monitors[q].d_acc, acc[q].data(), acc[q].size(), cudaMemcpyHostToDevice, g->st));
        for (auto &p : g->planes) {
            int q = 0;
            while (q < hdr[7] && pl[q] != &p) q++;
            if (q < hdr[7]) CK(cudaMemcpyAsync(p.p, pdata[q].data(), pb, cudaMemcpyHostToDevice, g->st));
            else CK(cudaMemsetAsync(p.p, 0, pb, g->st));  // a plane of this grid the saved run did not hold
        }
        for (int m = 0; m < 6; m++)
            CK(cudaMemcpyAsync(g->f[g->cur][m], fields[m].data(), fb, cudaMemcpyHostToDevice, g->st));
        if (g->boundary == FDTD_BOUNDARY_CPML)
            for (int a = 0; a < 3; a++)
                for (int w = 0; w < 4; w++) {
                    if (hdr[8])
                        CK(cudaMemcpyAsync(g->psi[g->cur][a][w], psi[4 * a + w].data(), sz[a],
                                           cudaMemcpyHostToDevice, g->st));
                    else
                        CK(cudaMemsetAsync(g->psi[g->cur][a][w], 0, sz[a], g->st));
                }
        CK(cudaMemcpyAsync(g->d_step, &steps[1], sizeof(long long), cudaMemcpyHostToDevice, g->st));
        // host buffers are pageable: wait before they go out of scope
        CK(cudaStreamSynchronize(g->st));
    }
    g->host_steps = steps[0];
    g->fields_from_host = false;
    g->pp_synced = false;
    g->version++;
    return true;
short_read:
    set_error(FDTD_ERR_ARG, "checkpoint: %s is truncated", path);
    return false;
}

}  // namespace fdtd
