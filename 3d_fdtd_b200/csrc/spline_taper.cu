// spline_taper.cu -- a taper whose width is a natural cubic spline through
// control widths, rasterised with sub-pixel permittivity, and the adjoint
// gradient of an objective with respect to those widths.
//
// The reference shapes tapers from straight segments between integer vertices
// (timefield3d_set_taper, timefield3d.c:1511-1535; adjoint3d_taper_insert,
// adjoint3d.c:243-257) and fills whole cells.  Here width(k) on plane k is a
// natural cubic spline through `ncontrol` widths placed evenly on
// [start_z, end_z - 1]; the core spans x in [center_x - w/(2 disc),
// center_x + w/(2 disc)) in cell units, cell i covering [i, i+1).  A cell
// covered by a fraction f of the core gets ep_old + f (ep_core - ep_old) (the
// same for mu, all three components alike, as the reference fills them); a
// fully covered cell gets exactly ep_core and an uncovered one keeps its
// value, so integer edges reproduce the reference's whole-cell fill bit for
// bit.  Because eps moves continuously with the widths, finite differences of
// an objective with respect to a width are well defined.
//
// The gradient follows adjoint3d_taper_calculate_gradients_from_ep_gradient
// (adjoint3d.c:375-418) with the segment hat weights replaced by the spline
// weights: the cell holding each edge gets the field product
// g = sum_t sum_m E_fwd E_adj (adjoint3d.c:339-373), and
//   dF/dw_c = sum_k sum_j W[k][c] / (2 disc) (g_right + g_left) ep_diff,
// since the right edge moves by +dw/(2 disc) cells and the left one by -dw/(2 disc).
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace fdtd {

// W[(k - start_z) * K + c]: weight of control width c in width(k)
bool spline_basis(int K, int start_z, int end_z, std::vector<double> &W)
{
    const int L = end_z - start_z;
    if (K < 2 || L < 2) return false;
    const double h = (double)(L - 1) / (K - 1);
    W.assign((size_t)L * K, 0.0);
    std::vector<double> y(K), M(K), cp(K), dp(K);
    for (int c = 0; c < K; c++) {
        for (int i = 0; i < K; i++) y[i] = i == c ? 1.0 : 0.0;
        // natural spline: M_0 = M_{K-1} = 0;
        // M_{i-1} + 4 M_i + M_{i+1} = 6 (y_{i+1} - 2 y_i + y_{i-1}) / h^2, i = 1..K-2 (Thomas)
        std::fill(M.begin(), M.end(), 0.0);
        const int n = K - 2;
        if (n > 0) {
            for (int i = 0; i < n; i++) {
                const double rhs = 6.0 * (y[i + 2] - 2.0 * y[i + 1] + y[i]) / (h * h);
                const double b = 4.0 - (i > 0 ? cp[i - 1] : 0.0);
                cp[i] = 1.0 / b;
                dp[i] = (rhs - (i > 0 ? dp[i - 1] : 0.0)) / b;
            }
            M[n] = dp[n - 1];
            for (int i = n - 2; i >= 0; i--) M[i + 1] = dp[i] - cp[i] * M[i + 2];
        }
        for (int k = 0; k < L; k++) {
            const double z = (double)k;
            int s = (int)std::floor(z / h);
            if (s > K - 2) s = K - 2;
            if (s < 0) s = 0;
            const double a = z - s * h, b = (s + 1) * h - z;
            W[(size_t)k * K + c] = M[s] * b * b * b / (6.0 * h) + M[s + 1] * a * a * a / (6.0 * h) +
                                   (y[s] / h - M[s] * h / 6.0) * b + (y[s + 1] / h - M[s + 1] * h / 6.0) * a;
        }
    }
    return true;
}

namespace {

struct SplineGeom {
    int K = 0, start_z = 0, end_z = 0, bottom = 0, top = 0;
    double center_x = 0, disc = 0;
    std::vector<double> W, xl, xr;   // weights; core x-extent per plane
};

bool spline_geometry(const timefield3d &psi, int K, const double *widths, double center_x, int start_z, int end_z,
                     int bottom, int top, SplineGeom &sg)
{
    if (!widths || K < 2 || start_z < 0 || end_z > psi.k || end_z - start_z < 2 || bottom < 0 || top > psi.j ||
        bottom >= top || !(psi.disc > 0) || !std::isfinite(center_x)) {
        set_error(FDTD_ERR_ARG, "spline taper: %d widths, z [%d,%d), y [%d,%d) in a %dx%dx%d grid", K, start_z, end_z,
                  bottom, top, psi.i, psi.j, psi.k);
        return false;
    }
    if (!spline_basis(K, start_z, end_z, sg.W)) return false;
    sg.K = K; sg.start_z = start_z; sg.end_z = end_z; sg.bottom = bottom; sg.top = top;
    sg.center_x = center_x; sg.disc = psi.disc;
    const int L = end_z - start_z;
    sg.xl.resize(L);
    sg.xr.resize(L);
    for (int k = 0; k < L; k++) {
        double w = 0.0;
        for (int c = 0; c < K; c++) w += sg.W[(size_t)k * K + c] * widths[c];
        const double half = w / (2.0 * psi.disc);
        sg.xl[k] = center_x - half;
        sg.xr[k] = center_x + half;
        if (!std::isfinite(w) || w < 0 || sg.xl[k] < 0 || sg.xr[k] > psi.i) {
            set_error(FDTD_ERR_ARG, "spline taper: width %g um on plane %d puts the core at x [%g, %g) outside [0, %d)",
                      w, start_z + k, sg.xl[k], sg.xr[k], psi.i);
            return false;
        }
    }
    return true;
}

// host mirror, AoS ep/mu (index 3 q + c)
void raster_host(const timefield3d &psi, const SplineGeom &sg, double ep, double mu)
{
    const int nx = psi.i, ny = psi.j;
    for (int k = sg.start_z; k < sg.end_z; k++) {
        const double xl = sg.xl[k - sg.start_z], xr = sg.xr[k - sg.start_z];
        const int i0 = std::max(0, (int)std::floor(xl)), i1 = std::min(nx - 1, (int)std::ceil(xr) - 1);
        for (int j = sg.bottom; j < sg.top; j++)
            for (int i = i0; i <= i1; i++) {
                const double f = std::min((double)i + 1.0, xr) - std::max((double)i, xl);
                if (!(f > 0.0)) continue;
                const long long q = 3LL * (i + (long long)nx * (j + (long long)ny * k));
                for (int c = 0; c < 3; c++) {
                    if (f >= 1.0) {
                        psi.ep[q + c] = (float)ep;
                        psi.mu[q + c] = (float)mu;
                    } else {
                        const double oe = psi.ep[q + c], om = psi.mu[q + c];
                        const double de = ep - oe, dm = mu - om;
                        const double pe = f * de, pm = f * dm;
                        psi.ep[q + c] = (float)(oe + pe);
                        psi.mu[q + c] = (float)(om + pm);
                    }
                }
            }
    }
}

}  // namespace

// device copy, SoA float arrays; same arithmetic as raster_host
__global__ void k_spline_raster(float *ep0, float *ep1, float *ep2, float *mu0, float *mu1, float *mu2, int nx,
                                int ny, int start_z, int bottom, int rows, const double *xl, const double *xr,
                                double ep, double mu)
{
    const int k = start_z + blockIdx.y;
    const double l = xl[blockIdx.y], r = xr[blockIdx.y];
    const float fe = __double2float_rn(ep), fm = __double2float_rn(mu);
    float *e[3] = {ep0, ep1, ep2}, *m[3] = {mu0, mu1, mu2};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < rows * nx; t += gridDim.x * blockDim.x) {
        const int j = bottom + t / nx, i = t % nx;
        const double f = __dsub_rn(fmin((double)i + 1.0, r), fmax((double)i, l));
        if (!(f > 0.0)) continue;
        const long long q = i + (long long)nx * (j + (long long)ny * k);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (f >= 1.0) {
                e[c][q] = fe;
                m[c][q] = fm;
            } else {
                const double oe = e[c][q], om = m[c][q];
                e[c][q] = __double2float_rn(__dadd_rn(oe, __dmul_rn(f, __dsub_rn(ep, oe))));
                m[c][q] = __double2float_rn(__dadd_rn(om, __dmul_rn(f, __dsub_rn(mu, om))));
            }
        }
    }
}

namespace {

template <typename P> bool dalloc(P **p, size_t bytes, cudaStream_t st, bool zero = true)
{
    if (*p) return true;
    void *v = nullptr;
    if (!cuda_ok(cudaMalloc(&v, bytes ? bytes : 16), "cudaMalloc")) return false;
    *p = (P *)v;
    if (zero) return cuda_ok(cudaMemsetAsync(v, 0, bytes ? bytes : 16, st), "cudaMemsetAsync");
    return true;
}

template <typename P> void dfree(P *&p)
{
    if (p) cudaFree((void *)p);
    p = nullptr;
}

// store cell of plane k, row j, edge e (0 right, 1 left), offset d in -1..1
// from the cell holding the edge
inline size_t store_cell(int height, int k, int j, int e, int d)
{
    return ((size_t)(j + (size_t)height * k) * 2 + e) * 3 + (d + 1);
}

// the spline edge store: a TaperDev (same store / gradient kernels as the
// reference tapers) keyed by this object, cells [k][j][edge], edge 0 right
struct SplineStore {
    SplineGeom sg;
    int duration = 0;
    std::vector<long long> cells;   // built for (nx, ny)
    int nx = 0, ny = 0;
};

adjoint3d_taper store_key(const SplineStore *s)
{
    adjoint3d_taper key{};
    key.left = (int *)(const void *)s;
    return key;
}

bool store_prepare(SplineStore *s, Grid *g)
{
    if (!grid_ensure_device(g)) return false;
    TaperDev *td = taper_lookup(store_key(s), true);
    const int height = s->sg.top - s->sg.bottom, length = s->sg.end_z - s->sg.start_z;
    const int ncell = 6 * height * length;   // per (k, j, edge): the edge cell and its two x neighbours
    if (td->ncell != ncell || td->duration != s->duration || td->prec != g->prec) {
        cudaDeviceSynchronize();
        dfree(td->d_fwd); dfree(td->d_adj); dfree(td->d_cells); dfree(td->d_grad);
        td->ncell = ncell;
        td->duration = s->duration;
        td->prec = g->prec;
        td->height = height;
        td->length = length;
        s->nx = s->ny = 0;
        const size_t es = g->prec == FDTD_F64 ? 8 : 4;
        const size_t bytes = (size_t)s->duration * ncell * 3 * es;
        if (!dalloc(&td->d_fwd, bytes, g->st) || !dalloc(&td->d_adj, bytes, g->st)) return false;
        if (!dalloc(&td->d_cells, ncell * sizeof(long long), g->st, false)) return false;
        if (!dalloc(&td->d_grad, ncell * sizeof(double), g->st)) return false;
    }
    if (s->nx != g->nx || s->ny != g->ny) {
        s->cells.assign(ncell, 0);
        for (int k = 0; k < length; k++)
            for (int j = 0; j < height; j++)
                for (int e = 0; e < 2; e++) {
                    const double x = e == 0 ? s->sg.xr[k] : s->sg.xl[k];
                    for (int d = -1; d <= 1; d++) {
                        int i = (int)std::floor(x) + d;
                        i = std::max(0, std::min(g->nx - 1, i));
                        s->cells[store_cell(height, k, j, e, d)] =
                            i + (long long)g->nx * ((s->sg.bottom + j) + (long long)g->ny * (s->sg.start_z + k));
                    }
                }
        if (!cuda_ok(cudaStreamSynchronize(g->st), "sync") ||
            !cuda_ok(cudaMemcpy(td->d_cells, s->cells.data(), ncell * sizeof(long long), cudaMemcpyHostToDevice),
                     "spline cells H2D"))
            return false;
        s->nx = g->nx;
        s->ny = g->ny;
    }
    return true;
}

std::vector<SplineStore *> &stores()
{
    static std::vector<SplineStore *> v;
    return v;
}

bool store_known(const SplineStore *s)
{
    for (auto *p : stores())
        if (p == s) return true;
    return false;
}

}  // namespace

}  // namespace fdtd

using namespace fdtd;

extern "C" {

int fdtd_spline_basis(int ncontrol, int start_z, int end_z, double *weights)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    std::vector<double> W;
    if (!weights || !spline_basis(ncontrol, start_z, end_z, W)) {
        set_error(FDTD_ERR_ARG, "fdtd_spline_basis: %d control points over z [%d,%d)", ncontrol, start_z, end_z);
        return FDTD_ERR_ARG;
    }
    std::copy(W.begin(), W.end(), weights);
    return FDTD_OK;
}

int timefield3d_set_spline_taper(timefield3d psi, double ep, double mu, int ncontrol, const double *widths,
                                 double center_x, int start_z, int end_z, int bottom, int top)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    if (!std::isfinite(ep) || !std::isfinite(mu)) {
        set_error(FDTD_ERR_NONFINITE, "timefield3d_set_spline_taper: ep %g mu %g", ep, mu);
        return FDTD_ERR_NONFINITE;
    }
    SplineGeom sg;
    if (!spline_geometry(psi, ncontrol, widths, center_x, start_z, end_z, bottom, top, sg)) return fdtd_last_error();
    Grid *g = grid_lookup(psi, true);
    const bool device = g && g->dev && g->ep[0] && !(g->mat_dirty & (kMatEp | kMatMu));
    raster_host(psi, sg, ep, mu);   // the host arrays stay authoritative and complete
    if (!g) return FDTD_OK;
    if (!device) {
        g->mat_dirty |= kMatEp | kMatMu;
        g->version++;
        return FDTD_OK;
    }
    // device copy current: write the same values there instead of uploading 6 arrays
    const int L = end_z - start_z;
    std::vector<double> edges(2 * (size_t)L);
    std::copy(sg.xl.begin(), sg.xl.end(), edges.begin());
    std::copy(sg.xr.begin(), sg.xr.end(), edges.begin() + L);
    double *d_edges = nullptr;
    if (!cuda_ok(cudaMalloc(&d_edges, edges.size() * sizeof(double)), "cudaMalloc(spline edges)")) return fdtd_last_error();
    bool ok = cuda_ok(cudaMemcpyAsync(d_edges, edges.data(), edges.size() * sizeof(double), cudaMemcpyHostToDevice,
                                      g->st), "spline edges H2D");
    if (ok) {
        const int rows = top - bottom;
        const int bx = std::max(1, std::min(64, (rows * psi.i + 255) / 256));
        note_launch();
        k_spline_raster<<<dim3(bx, L), 256, 0, g->st>>>(g->ep[0], g->ep[1], g->ep[2], g->mu[0], g->mu[1], g->mu[2],
                                                        psi.i, psi.j, start_z, bottom, rows, d_edges, d_edges + L, ep,
                                                        mu);
        ok = cuda_ok(cudaGetLastError(), "spline raster") && cuda_ok(cudaStreamSynchronize(g->st), "spline raster");
    }
    cudaFree(d_edges);
    if (!ok) return fdtd_last_error();
    if (mu != 1.0) g->mu_nonunit = true;
    g->coef_valid = false;
    g->version++;
    return FDTD_OK;
}

fdtd_spline_store fdtd_spline_store_new(timefield3d psi, int ncontrol, const double *widths, double center_x,
                                        int start_z, int end_z, int bottom, int top, int duration)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    if (duration <= 0) {
        set_error(FDTD_ERR_ARG, "fdtd_spline_store_new: duration %d", duration);
        return nullptr;
    }
    auto *s = new SplineStore;
    if (!spline_geometry(psi, ncontrol, widths, center_x, start_z, end_z, bottom, top, s->sg)) {
        delete s;
        return nullptr;
    }
    s->duration = duration;
    stores().push_back(s);
    return (fdtd_spline_store)s;
}

int fdtd_spline_store_bind(fdtd_spline_store store, timefield3d psi, int which, int t0, int dir)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    auto *s = (SplineStore *)store;
    if (!store_known(s) || (which != 0 && which != 1) || (dir != 1 && dir != -1 && dir != 0)) {
        set_error(FDTD_ERR_ARG, "fdtd_spline_store_bind: unknown store, or which not 0/1, or dir not -1/0/1");
        return FDTD_ERR_ARG;
    }
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    if (!store_prepare(s, g)) return fdtd_last_error();
    for (auto &b : g->binds)
        if (b.taper_key == (const void *)s && b.which == which) {
            b.t0 = t0;
            b.dir = dir;
            g->version++;
            return FDTD_OK;
        }
    g->binds.push_back(TaperBind{(const void *)s, which, t0, dir});
    g->version++;
    return FDTD_OK;
}

int fdtd_spline_store_unbind(fdtd_spline_store store, timefield3d psi)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    Grid *g = grid_lookup(psi);
    if (!g) return FDTD_ERR_ARG;
    std::vector<TaperBind> keep;
    for (auto &b : g->binds)
        if (b.taper_key != (const void *)store) keep.push_back(b);
    g->binds.swap(keep);
    g->version++;
    return FDTD_OK;
}

// g of every stored cell (FP64 sums on the device): the reference's field
// product (exact = false) or the exact adjoint's (exact = true)
static bool cell_gradients(TaperDev *td, bool exact, std::vector<double> &gcell)
{
    if (!cuda_ok(cudaDeviceSynchronize(), "sync")) return false;
    if (exact && td->prec == FDTD_F64)
        launch_ep_gradient_exact<double>((const double *)td->d_fwd, (const double *)td->d_adj, td->ncell,
                                         td->duration, td->d_grad, 0);
    else if (exact)
        launch_ep_gradient_exact<float>((const float *)td->d_fwd, (const float *)td->d_adj, td->ncell, td->duration,
                                        td->d_grad, 0);
    else if (td->prec == FDTD_F64)
        launch_ep_gradient<double>((const double *)td->d_fwd, (const double *)td->d_adj, td->ncell, td->duration,
                                   td->d_grad, 0);
    else
        launch_ep_gradient<float>((const float *)td->d_fwd, (const float *)td->d_adj, td->ncell, td->duration,
                                  td->d_grad, 0);
    if (!cuda_ok(cudaGetLastError(), "ep gradient")) return false;
    gcell.assign(td->ncell, 0.0);
    return cuda_ok(cudaMemcpy(gcell.data(), td->d_grad, td->ncell * sizeof(double), cudaMemcpyDeviceToHost),
                   "gradient D2H");
}

static TaperDev *store_dev(SplineStore *s, const double *grad)
{
    TaperDev *td = store_known(s) ? taper_lookup(store_key(s), false) : nullptr;
    if (!td || !td->d_fwd || !grad) {
        set_error(FDTD_ERR_ARG, "spline store gradient: no stored fields for this store");
        return nullptr;
    }
    return td;
}

// d/dw_c of the core: the edge cell's fill fraction moves by 1/(2 disc) per um
// of width on both edges (timefield3d_set_spline_taper's fill rule)
static int spline_gradient(fdtd_spline_store store, double ep_diff, double *grad, double *cell_gradient, bool exact)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    auto *s = (SplineStore *)store;
    TaperDev *td = store_dev(s, grad);
    if (!td) return FDTD_ERR_ARG;
    std::vector<double> gcell;
    if (!cell_gradients(td, exact, gcell)) return fdtd_last_error();
    if (cell_gradient) std::copy(gcell.begin(), gcell.end(), cell_gradient);
    const SplineGeom &sg = s->sg;
    const int height = sg.top - sg.bottom, length = sg.end_z - sg.start_z;
    for (int c = 0; c < sg.K; c++) {
        double acc = 0.0;
        for (int k = 0; k < length; k++) {
            double row = 0.0;
            for (int j = 0; j < height; j++)
                row += gcell[store_cell(height, k, j, 0, 0)] + gcell[store_cell(height, k, j, 1, 0)];
            acc += sg.W[(size_t)k * sg.K + c] * row;
        }
        grad[c] = acc * ep_diff / (2.0 * sg.disc);
    }
    return FDTD_OK;
}

int fdtd_spline_store_gradient(fdtd_spline_store store, double ep_diff, double *grad, double *cell_gradient)
{
    return spline_gradient(store, ep_diff, grad, cell_gradient, false);
}

int fdtd_spline_store_gradient_exact(fdtd_spline_store store, double ep_diff, double *grad, double *cell_gradient)
{
    return spline_gradient(store, ep_diff, grad, cell_gradient, true);
}

// fill fraction of cell i for a core [xl, xr) (the raster's rule, clamped)
static double cover(int i, double xl, double xr)
{
    const double f = std::min((double)i + 1.0, xr) - std::max((double)i, xl);
    return f <= 0.0 ? 0.0 : (f >= 1.0 ? 1.0 : f);
}

int fdtd_spline_store_gradient_step(fdtd_spline_store store, double ep_diff, double delta, double *grad)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    auto *s = (SplineStore *)store;
    TaperDev *td = store_dev(s, grad);
    if (!td) return FDTD_ERR_ARG;
    const SplineGeom &sg = s->sg;
    if (!(delta > 0) || delta / (2.0 * sg.disc) > 1.0) {
        set_error(FDTD_ERR_ARG,
                  "spline store step gradient: delta %g um must be positive and move an edge by at most one cell",
                  delta);
        return FDTD_ERR_ARG;
    }
    std::vector<double> gcell;
    if (!cell_gradients(td, true, gcell)) return fdtd_last_error();
    const int height = sg.top - sg.bottom, length = sg.end_z - sg.start_z;
    for (int c = 0; c < sg.K; c++) {
        double acc = 0.0;
        for (int k = 0; k < length; k++) {
            const double sh = delta * std::fabs(sg.W[(size_t)k * sg.K + c]) / (2.0 * sg.disc);   // edge shift, cells
            const double sg_w = sg.W[(size_t)k * sg.K + c] >= 0 ? 1.0 : -1.0;
            const double xl = sg.xl[k], xr = sg.xr[k];
            const int base[2] = {(int)std::floor(xr), (int)std::floor(xl)};
            double row = 0.0;
            for (int e = 0; e < 2; e++)
                for (int d = -1; d <= 1; d++) {
                    const int i = base[e] + d;
                    if (e == 1 && i >= base[0] - 1) continue;   // already counted with the right edge's cells
                    // width + delta W (both edges out by sh when W >= 0) against width - delta W
                    const double df = sg_w * (cover(i, xl - sh, xr + sh) - cover(i, xl + sh, xr - sh));
                    if (df == 0.0) continue;
                    double gs = 0.0;
                    for (int j = 0; j < height; j++) gs += gcell[store_cell(height, k, j, e, d)];
                    row += gs * df;
                }
            acc += row;
        }
        grad[c] = acc * ep_diff / (2.0 * delta);
    }
    return FDTD_OK;
}

void fdtd_spline_store_free(fdtd_spline_store store)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    auto *s = (SplineStore *)store;
    auto &v = stores();
    for (size_t i = 0; i < v.size(); i++)
        if (v[i] == s) {
            taper_unregister(store_key(s));
            v.erase(v.begin() + i);
            delete s;
            return;
        }
}

}  // extern "C"
