/*
 * fdtd_oracle.c -- CPU restatement of the FDTD hot path (TEST INFRASTRUCTURE).
 *
 * This file is the checker, not the product: only the tests, the smoke check
 * and the CPU-baseline leg of bench.py load it.  See fdtd_oracle.h for the
 * list of reference functions it restates.  Parity of the restatement with the
 * reference itself is pinned by tests/test_oracle_vs_reference.py, which runs
 * the reference's own compiled sources (oracle/_ref/libref.so) side by side,
 * and by the golden vectors in tests/golden/.
 */
#include "fdtd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* the reference's two pi constants: timefield3d.c:3 (phase reduction) */
#define REF_PI 3.141592652
/* complex.c:4 */
#define SERIES_TOL 1e-30

struct orc_grid {
    int nx, ny, nz;
    double dx;
    int boundary;
    size_t n;
    double *f[6];
    double *old[6]; /* previous-step copy; only the 2-cell shell is maintained */
    float *ep[3], *mu[3], *sig[6], *src[6];
    /* CPML */
    int npml;
    double *prof[6][3]; /* b_E a_E kinv_E b_H a_H kinv_H, per axis, length n_axis */
    double *psi[3][4];  /* per slab axis: psiE(c1), psiE(c2), psiH(c1), psiH(c2) */
};

static int g_threads = 1;
void orc_step_threads(int nthreads) { g_threads = nthreads > 0 ? nthreads : 1; }

#define IDX(g, i, j, k) ((size_t)(i) + (size_t)(g)->nx * ((size_t)(j) + (size_t)(g)->ny * (size_t)(k)))

orc_grid *orc_new(int nx, int ny, int nz, double dx)
{
    orc_grid *g = calloc(1, sizeof(*g));
    g->nx = nx; g->ny = ny; g->nz = nz; g->dx = dx;
    g->n = (size_t)nx * ny * nz;
    g->boundary = ORC_BOUNDARY_MUR;
    for (int m = 0; m < 6; m++) {
        g->f[m] = calloc(g->n, sizeof(double));
        g->old[m] = calloc(g->n, sizeof(double));
        g->sig[m] = calloc(g->n, sizeof(float));
        g->src[m] = calloc(g->n, sizeof(float));
    }
    /* timefield3d_new sets ep = mu = 1 (timefield3d.c:25-29) */
    for (int c = 0; c < 3; c++) {
        g->ep[c] = malloc(g->n * sizeof(float));
        g->mu[c] = malloc(g->n * sizeof(float));
        for (size_t q = 0; q < g->n; q++) { g->ep[c][q] = 1.0f; g->mu[c][q] = 1.0f; }
    }
    return g;
}

static void free_cpml(orc_grid *g)
{
    for (int w = 0; w < 6; w++) for (int a = 0; a < 3; a++) { free(g->prof[w][a]); g->prof[w][a] = NULL; }
    for (int a = 0; a < 3; a++) for (int s = 0; s < 4; s++) { free(g->psi[a][s]); g->psi[a][s] = NULL; }
    g->npml = 0;
}

void orc_free(orc_grid *g)
{
    if (!g) return;
    for (int m = 0; m < 6; m++) { free(g->f[m]); free(g->old[m]); free(g->sig[m]); free(g->src[m]); }
    for (int c = 0; c < 3; c++) { free(g->ep[c]); free(g->mu[c]); }
    free_cpml(g);
    free(g);
}

static size_t slab_size(const orc_grid *g, int axis)
{
    size_t L2 = 2 * (size_t)g->npml;
    if (axis == 0) return L2 * g->ny * g->nz;
    if (axis == 1) return (size_t)g->nx * L2 * g->nz;
    return (size_t)g->nx * g->ny * L2;
}

/* timefield3d_zero_fields (timefield3d.c:108-121) plus the CPML memory */
void orc_zero(orc_grid *g)
{
    for (int m = 0; m < 6; m++) {
        memset(g->f[m], 0, g->n * sizeof(double));
        memset(g->old[m], 0, g->n * sizeof(double));
        memset(g->src[m], 0, g->n * sizeof(float));
    }
    if (g->npml)
        for (int a = 0; a < 3; a++)
            for (int s = 0; s < 4; s++) memset(g->psi[a][s], 0, slab_size(g, a) * sizeof(double));
}

double *orc_field(orc_grid *g, int m) { return g->f[m]; }
float *orc_ep(orc_grid *g, int c) { return g->ep[c]; }
float *orc_mu(orc_grid *g, int c) { return g->mu[c]; }
float *orc_sig(orc_grid *g, int m) { return g->sig[m]; }
float *orc_src(orc_grid *g, int m) { return g->src[m]; }
void orc_set_boundary(orc_grid *g, int b) { g->boundary = b; }

/* ---------------------------------------------------------------------------
 * CPML (no reference counterpart).  Convolutional PML after Roden & Gedney,
 * Microwave Opt. Tech. Lett. 27 (2000) 334, in the units of the reference
 * (c = eps0 = mu0 = 1, lengths in um).  On each axis of N cells the slabs are
 * cells [0, L) and [N-L, N).  Depth fraction rho of a position p (E nodes at
 * p = i, H nodes at p = i + 1/2):
 *     low side   rho = (L - 1/2 - p) / L   for p < L - 1/2
 *     high side  rho = (p - (N - L - 1/2)) / L   for p > N - L - 1/2
 * sigma = sigma_max rho^m, kappa = 1 + (kappa_max - 1) rho^m,
 * alpha = alpha_max (1 - rho) (zero where rho = 0);
 * b = exp(-(sigma/kappa + alpha) dt),  a = sigma (b - 1) / (sigma kappa + kappa^2 alpha).
 * The outer cells 0 and N-1 are never updated (PEC backing), as in the
 * reference's interior-only update.
 * ------------------------------------------------------------------------- */
static void cpml_point(double rho, int order, double smax, double kmax, double amax, double dt,
                       double *b, double *a, double *kinv)
{
    if (rho <= 0) { *b = 1.0; *a = 0.0; *kinv = 1.0; return; }
    double r = pow(rho, order);
    double sigma = smax * r;
    double kappa = 1.0 + (kmax - 1.0) * r;
    double alpha = amax * (1.0 - rho);
    *b = exp(-(sigma / kappa + alpha) * dt);
    *a = sigma > 0 ? sigma * (*b - 1.0) / (sigma * kappa + kappa * kappa * alpha) : 0.0;
    *kinv = 1.0 / kappa;
}

void orc_set_cpml(orc_grid *g, int npml, int order, double sigma_max, double kappa_max,
                  double alpha_max, double dt)
{
    free_cpml(g);
    if (npml <= 0) return;
    g->npml = npml;
    if (sigma_max <= 0) sigma_max = 0.8 * (order + 1) / g->dx;
    int dims[3] = {g->nx, g->ny, g->nz};
    for (int a = 0; a < 3; a++) {
        int N = dims[a];
        for (int w = 0; w < 6; w++) g->prof[w][a] = malloc(N * sizeof(double));
        for (int i = 0; i < N; i++) {
            for (int h = 0; h < 2; h++) {
                double p = i + 0.5 * h;
                double rho = 0;
                if (p < npml - 0.5) rho = (npml - 0.5 - p) / npml;
                else if (p > N - npml - 0.5) rho = (p - (N - npml - 0.5)) / npml;
                cpml_point(rho, order, sigma_max, kappa_max, alpha_max, dt,
                           &g->prof[3 * h + 0][a][i], &g->prof[3 * h + 1][a][i], &g->prof[3 * h + 2][a][i]);
            }
        }
        for (int s = 0; s < 4; s++) g->psi[a][s] = calloc(slab_size(g, a), sizeof(double));
    }
}

const double *orc_cpml_profile(orc_grid *g, int which, int axis)
{
    return g->npml ? g->prof[which][axis] : NULL;
}

/* slab-local index of cell (i,j,k) in the slab of `axis`, or -1 outside it */
static inline long slab_index(const orc_grid *g, int axis, int i, int j, int k)
{
    int L = g->npml;
    if (!L) return -1;
    if (axis == 0) {
        int s = i < L ? i : (i >= g->nx - L ? i - g->nx + 2 * L : -1);
        if (s < 0) return -1;
        return s + 2L * L * ((long)j + (long)g->ny * k);
    } else if (axis == 1) {
        int s = j < L ? j : (j >= g->ny - L ? j - g->ny + 2 * L : -1);
        if (s < 0) return -1;
        return i + (long)g->nx * (s + 2L * L * k);
    } else {
        int s = k < L ? k : (k >= g->nz - L ? k - g->nz + 2 * L : -1);
        if (s < 0) return -1;
        return i + (long)g->nx * (j + (long)g->ny * s);
    }
}

/* ---------------------------------------------------------------------------
 * Yee E update, timefield3d_apply_E_timestep_zsection (timefield3d.c:1759-1837)
 * over the interior i,j,k in [1, N-1).  Backward differences.  The source
 * current enters directly; the conductivity only through the semi-implicit
 * coefficients (the reference's zsection form drops the explicit sig*E term).
 * With CPML the curl is stretched: d/dq -> (1/kappa_q) d/dq + psi_q.
 * ------------------------------------------------------------------------- */
static void update_E(orc_grid *g, double dt)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double divisor = 1 / (g->dx);
    double *Ex = g->f[0], *Ey = g->f[1], *Ez = g->f[2];
    const double *Hx = g->f[3], *Hy = g->f[4], *Hz = g->f[5];
    const size_t sx = 1, sy = nx, sz = (size_t)nx * ny;
    const int cpml = g->boundary == ORC_BOUNDARY_CPML && g->npml > 0;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int k = 1; k < nz - 1; k++)
        for (int j = 1; j < ny - 1; j++)
            for (int i = 1; i < nx - 1; i++) {
                size_t q = IDX(g, i, j, k);
                double dHz_dy = (Hz[q] - Hz[q - sy]);
                double dHy_dz = (Hy[q] - Hy[q - sz]);
                double dHx_dz = (Hx[q] - Hx[q - sz]);
                double dHz_dx = (Hz[q] - Hz[q - sx]);
                double dHy_dx = (Hy[q] - Hy[q - sx]);
                double dHx_dy = (Hx[q] - Hx[q - sy]);
                double curl_x, curl_y, curl_z;
                if (!cpml) {
                    curl_x = divisor * (dHz_dy - dHy_dz);
                    curl_y = divisor * (dHx_dz - dHz_dx);
                    curl_z = divisor * (dHy_dx - dHx_dy);
                } else {
                    /* axis slabs: x -> (Ey, Ez), y -> (Ex, Ez), z -> (Ex, Ey) */
                    long sxi = slab_index(g, 0, i, j, k), syi = slab_index(g, 1, i, j, k), szi = slab_index(g, 2, i, j, k);
                    double kx = sxi >= 0 ? g->prof[2][0][i] : 1.0;
                    double ky = syi >= 0 ? g->prof[2][1][j] : 1.0;
                    double kz = szi >= 0 ? g->prof[2][2][k] : 1.0;
                    double pxy = 0, pxz = 0, pyx = 0, pyz = 0, pzx = 0, pzy = 0;
                    if (sxi >= 0) {
                        double b = g->prof[0][0][i], a = g->prof[1][0][i];
                        pyx = g->psi[0][0][sxi] = b * g->psi[0][0][sxi] + a * (dHz_dx * divisor);
                        pzx = g->psi[0][1][sxi] = b * g->psi[0][1][sxi] + a * (dHy_dx * divisor);
                    }
                    if (syi >= 0) {
                        double b = g->prof[0][1][j], a = g->prof[1][1][j];
                        pxy = g->psi[1][0][syi] = b * g->psi[1][0][syi] + a * (dHz_dy * divisor);
                        pzy = g->psi[1][1][syi] = b * g->psi[1][1][syi] + a * (dHx_dy * divisor);
                    }
                    if (szi >= 0) {
                        double b = g->prof[0][2][k], a = g->prof[1][2][k];
                        pxz = g->psi[2][0][szi] = b * g->psi[2][0][szi] + a * (dHy_dz * divisor);
                        pyz = g->psi[2][1][szi] = b * g->psi[2][1][szi] + a * (dHx_dz * divisor);
                    }
                    curl_x = divisor * (dHz_dy * ky - dHy_dz * kz) + (pxy - pxz);
                    curl_y = divisor * (dHx_dz * kz - dHz_dx * kx) + (pyz - pyx);
                    curl_z = divisor * (dHy_dx * kx - dHx_dy * ky) + (pzx - pzy);
                }
                double ep_x = g->ep[0][q], ep_y = g->ep[1][q], ep_z = g->ep[2][q];
                double sig_x = g->sig[0][q], sig_y = g->sig[1][q], sig_z = g->sig[2][q];
                double Jx = g->src[0][q], Jy = g->src[1][q], Jz = g->src[2][q];
                double main_coeff, E_coeff;
                main_coeff = 1.0 / (ep_x / dt + 0.5 * sig_x);
                E_coeff = ep_x / dt - 0.5 * sig_x;
                Ex[q] = main_coeff * (E_coeff * Ex[q] + curl_x - Jx);
                main_coeff = 1.0 / (ep_y / dt + 0.5 * sig_y);
                E_coeff = ep_y / dt - 0.5 * sig_y;
                Ey[q] = main_coeff * (E_coeff * Ey[q] + curl_y - Jy);
                main_coeff = 1.0 / (ep_z / dt + 0.5 * sig_z);
                E_coeff = ep_z / dt - 0.5 * sig_z;
                Ez[q] = main_coeff * (E_coeff * Ez[q] + curl_z - Jz);
            }
}

/* Yee H update, timefield3d_apply_H_timestep_zsection (timefield3d.c:1679-1757).
 * Forward differences.  The magnetic current is source + sig_m * H
 * (timefield3d.c:1705-1707) and sig_m also enters the coefficients. */
static void update_H(orc_grid *g, double dt)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double divisor = 1 / (g->dx);
    const double *Ex = g->f[0], *Ey = g->f[1], *Ez = g->f[2];
    double *Hx = g->f[3], *Hy = g->f[4], *Hz = g->f[5];
    const size_t sx = 1, sy = nx, sz = (size_t)nx * ny;
    const int cpml = g->boundary == ORC_BOUNDARY_CPML && g->npml > 0;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int k = 1; k < nz - 1; k++)
        for (int j = 1; j < ny - 1; j++)
            for (int i = 1; i < nx - 1; i++) {
                size_t q = IDX(g, i, j, k);
                double hx = Hx[q], hy = Hy[q], hz = Hz[q];
                double Mx = g->src[3][q] + hx * g->sig[3][q];
                double My = g->src[4][q] + hy * g->sig[4][q];
                double Mz = g->src[5][q] + hz * g->sig[5][q];
                double dEz_dy = (Ez[q + sy] - Ez[q]);
                double dEy_dz = (Ey[q + sz] - Ey[q]);
                double dEx_dz = (Ex[q + sz] - Ex[q]);
                double dEz_dx = (Ez[q + sx] - Ez[q]);
                double dEy_dx = (Ey[q + sx] - Ey[q]);
                double dEx_dy = (Ex[q + sy] - Ex[q]);
                double curl_x, curl_y, curl_z;
                if (!cpml) {
                    curl_x = divisor * (dEz_dy - dEy_dz);
                    curl_y = divisor * (dEx_dz - dEz_dx);
                    curl_z = divisor * (dEy_dx - dEx_dy);
                } else {
                    long sxi = slab_index(g, 0, i, j, k), syi = slab_index(g, 1, i, j, k), szi = slab_index(g, 2, i, j, k);
                    double kx = sxi >= 0 ? g->prof[5][0][i] : 1.0;
                    double ky = syi >= 0 ? g->prof[5][1][j] : 1.0;
                    double kz = szi >= 0 ? g->prof[5][2][k] : 1.0;
                    double pxy = 0, pxz = 0, pyx = 0, pyz = 0, pzx = 0, pzy = 0;
                    if (sxi >= 0) {
                        double b = g->prof[3][0][i], a = g->prof[4][0][i];
                        pyx = g->psi[0][2][sxi] = b * g->psi[0][2][sxi] + a * (dEz_dx * divisor);
                        pzx = g->psi[0][3][sxi] = b * g->psi[0][3][sxi] + a * (dEy_dx * divisor);
                    }
                    if (syi >= 0) {
                        double b = g->prof[3][1][j], a = g->prof[4][1][j];
                        pxy = g->psi[1][2][syi] = b * g->psi[1][2][syi] + a * (dEz_dy * divisor);
                        pzy = g->psi[1][3][syi] = b * g->psi[1][3][syi] + a * (dEx_dy * divisor);
                    }
                    if (szi >= 0) {
                        double b = g->prof[3][2][k], a = g->prof[4][2][k];
                        pxz = g->psi[2][2][szi] = b * g->psi[2][2][szi] + a * (dEy_dz * divisor);
                        pyz = g->psi[2][3][szi] = b * g->psi[2][3][szi] + a * (dEx_dz * divisor);
                    }
                    curl_x = divisor * (dEz_dy * ky - dEy_dz * kz) + (pxy - pxz);
                    curl_y = divisor * (dEx_dz * kz - dEz_dx * kx) + (pyz - pyx);
                    curl_z = divisor * (dEy_dx * kx - dEx_dy * ky) + (pzx - pzy);
                }
                double mu_x = g->mu[0][q], mu_y = g->mu[1][q], mu_z = g->mu[2][q];
                double sig_x = g->sig[3][q], sig_y = g->sig[4][q], sig_z = g->sig[5][q];
                double main_coeff, H_coeff;
                main_coeff = 1.0 / (mu_x / dt + 0.5 * sig_x);
                H_coeff = mu_x / dt - 0.5 * sig_x;
                Hx[q] = main_coeff * (H_coeff * hx - curl_x - Mx);
                main_coeff = 1.0 / (mu_y / dt + 0.5 * sig_y);
                H_coeff = mu_y / dt - 0.5 * sig_y;
                Hy[q] = main_coeff * (H_coeff * hy - curl_y - My);
                main_coeff = 1.0 / (mu_z / dt + 0.5 * sig_z);
                H_coeff = mu_z / dt - 0.5 * sig_z;
                Hz[q] = main_coeff * (H_coeff * hz - curl_z - Mz);
            }
}

/* ---------------------------------------------------------------------------
 * Mur first-order ABC.  Shell save: timefield3d_update_old_edge_fields
 * (timefield3d.c:246-346) copies the 2-cell shell of all six components.
 * Faces (timefield3d.c:2275-2721) run in the order x=0, y=0, z=0, x=end,
 * y=end, z=end; each sets the two tangential components
 *     F_b = F_in,old + s (F_in - F_b,old),  s = (v dt - dx)/(v dt + dx).
 * For E component c on a face normal to a, v = 1/sqrt(ep_c mu_t); for H
 * component c, v = 1/sqrt(ep_t mu_c), t being the third axis.  Later faces read
 * values earlier faces wrote (edges and corners), so the order is kept.
 * ------------------------------------------------------------------------- */
static void save_shell(orc_grid *g)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    for (int m = 0; m < 6; m++) {
        double *o = g->old[m];
        const double *f = g->f[m];
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    int shell = i <= 1 || i >= nx - 2 || j <= 1 || j >= ny - 2 || k <= 1 || k >= nz - 2;
                    if (shell) { size_t q = IDX(g, i, j, k); o[q] = f[q]; }
                }
    }
}

static void mur_face(orc_grid *g, double dt, int axis, int high, int efield)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    int dims[3] = {nx, ny, nz};
    /* tangential components and the third axis for each */
    int c1 = axis == 0 ? 1 : 0, c2 = axis == 2 ? 1 : 2;
    int t1 = 3 - axis - c1, t2 = 3 - axis - c2;
    int fix = high ? dims[axis] - 1 : 0, inner = high ? dims[axis] - 2 : 1;
    int ua = axis == 0 ? 1 : 0, va = axis == 2 ? 1 : 2; /* loop axes */
    for (int u = 0; u < dims[ua]; u++)
        for (int v = 0; v < dims[va]; v++) {
            int b3[3], n3[3];
            b3[axis] = fix; n3[axis] = inner;
            b3[ua] = n3[ua] = u; b3[va] = n3[va] = v;
            size_t qb = IDX(g, b3[0], b3[1], b3[2]), qi = IDX(g, n3[0], n3[1], n3[2]);
            for (int w = 0; w < 2; w++) {
                int c = w ? c2 : c1, t = w ? t2 : t1;
                double ep, mu;
                if (efield) { ep = g->ep[c][qb]; mu = g->mu[t][qb]; }
                else { ep = g->ep[t][qb]; mu = g->mu[c][qb]; }
                int m = efield ? c : 3 + c;
                double F_old = g->old[m][qb];
                double F_inner = g->f[m][qi];
                double F_inner_old = g->old[m][qi];
                double speed = 1 / sqrt(ep * mu);
                double scalar = (speed * dt - g->dx) / (speed * dt + g->dx);
                g->f[m][qb] = F_inner_old + scalar * (F_inner - F_old);
            }
        }
}

static void mur(orc_grid *g, double dt, int efield)
{
    for (int high = 0; high < 2; high++)
        for (int axis = 0; axis < 3; axis++) mur_face(g, dt, axis, high, efield);
}

/* one step: timefield3d_apply_timestep_omp_full (timefield3d.c:2787-2849) */
void orc_step(orc_grid *g, double dt)
{
    int murb = g->boundary == ORC_BOUNDARY_MUR;
    if (murb) save_shell(g);
    update_E(g, dt);
    if (murb) mur(g, dt, 1);
    update_H(g, dt);
    if (murb) mur(g, dt, 0);
}

/* ---------------------------------------------------------------------------
 * Modes.  mode_power_inner_product(psi, psi) (mode.c:1267-1310), norm
 * (mode.c:1330-1337), normalisation (mode.c:1367-1379).
 * ------------------------------------------------------------------------- */
double orc_mode_power_norm(const double *md, int mi, int mj, double mdisc)
{
    double sre = 0, sim = 0;
    for (int i = 0; i < mi; i++)
        for (int j = 0; j < mj; j++) {
            const double *e = md + 12 * (size_t)(i + j * mi);
            double Exr = e[0], Exi = e[1], Eyr = e[2], Eyi = e[3];
            double Hxr = e[6], Hxi = e[7], Hyr = e[8], Hyi = e[9];
            /* p1 = conj(Hx) Ey ; p2 = 0 - conj(Hy) Ex ; p3 = Hx conj(Ey) ; p4 = 0 - Hy conj(Ex) */
            double p1r = Hxr * Eyr - (-Hxi) * Eyi, p1i = Hxr * Eyi + (-Hxi) * Eyr;
            double q2r = Hyr * Exr - (-Hyi) * Exi, q2i = Hyr * Exi + (-Hyi) * Exr;
            double p2r = 0 - q2r, p2i = 0 - q2i;
            double p3r = Hxr * Eyr - Hxi * (-Eyi), p3i = Hxr * (-Eyi) + Hxi * Eyr;
            double q4r = Hyr * Exr - Hyi * (-Exi), q4i = Hyr * (-Exi) + Hyi * Exr;
            double p4r = 0 - q4r, p4i = 0 - q4i;
            sre = sre + ((p1r + p2r) + (p3r + p4r));
            sim = sim + ((p1i + p2i) + (p3i + p4i));
        }
    double s = (-0.5 * mdisc * mdisc);
    sre = s * sre; sim = s * sim;
    return sqrt(sqrt(sre * sre + sim * sim));
}

void orc_mode_power_normalize(double *md, int mi, int mj, double mdisc)
{
    double norm = orc_mode_power_norm(md, mi, mj, mdisc);
    double divisor = 1.0 / norm;
    for (size_t q = 0; q < 12 * (size_t)mi * mj; q++) md[q] = divisor * md[q];
}

/* timefield3d_mode_source (timefield3d.c:2977-3026) */
void orc_mode_source(orc_grid *g, int cx, int cy, int cz, double *md, int mi, int mj, double mdisc,
                     double phase, double amplitude, int reverse)
{
    int M_sign = -1 + 2 * reverse;
    orc_mode_power_normalize(md, mi, mj, mdisc);
    double c = cos(phase), s = sin(phase);
    for (int i = 0; i < g->nx; i++)
        for (int j = 0; j < g->ny; j++) {
            double xd = (i - cx) * (g->dx / mdisc);
            double yd = (j - cy) * (g->dx / mdisc);
            int mx = (int)xd + mi / 2, my = (int)yd + mj / 2;
            if (mx < 0 || mx >= mi || my < 0 || my >= mj) continue;
            size_t q = IDX(g, i, j, cz);
            for (int m = 0; m < 6; m++) {
                const double *e = md + 2 * (6 * (size_t)(mx + mi * my) + m);
                double permittivity = g->ep[m % 3][q];
                double permeability = g->mu[m % 3][q];
                if (m < 3)
                    g->src[m][q] = (float)(amplitude * permittivity * (e[0] * c + e[1] * s));
                else
                    g->src[m][q] = (float)(-M_sign * amplitude * permeability * (e[0] * c + e[1] * s));
            }
        }
}

/* timefield3d_mode_source_adjoint (timefield3d.c:3028-3068) */
void orc_mode_source_adjoint(orc_grid *g, int cx, int cy, int cz, double *md, int mi, int mj,
                             double mdisc, double phase, int reverse)
{
    int M_sign = -1 + 2 * reverse;
    orc_mode_power_normalize(md, mi, mj, mdisc);
    double c = cos(phase), s = sin(phase);
    for (int i = 0; i < g->nx; i++)
        for (int j = 0; j < g->ny; j++) {
            double xd = (i - cx) * (g->dx / mdisc);
            double yd = (j - cy) * (g->dx / mdisc);
            int mx = (int)xd + mi / 2, my = (int)yd + mj / 2;
            if (mx < 0 || mx >= mi || my < 0 || my >= mj) continue;
            size_t q = IDX(g, i, j, cz);
            const double *e = md + 12 * (size_t)(mx + mi * my);
            g->src[0][q] = (float)(1 * (e[8] * c + e[9] * s));
            g->src[1][q] = (float)(-1 * (e[6] * c + e[7] * s));
            g->src[2][q] = 0;
            g->src[3][q] = (float)(-1 * M_sign * (e[2] * c + e[3] * s));
            g->src[4][q] = (float)(1 * M_sign * (e[0] * c + e[1] * s));
            g->src[5][q] = 0;
        }
}

void orc_cexp_series(double x, double *re, double *im)
{
    /* complex_exp (complex.c:169-193) on the argument i*x */
    double pr = 1, pi = 0, er = 0, ei = 0, fact = 1;
    double dr = 1, di = 0;
    int n = 0;
    while (sqrt(dr * dr + di * di) >= SERIES_TOL) {
        double scalar = 1.0 / fact;
        dr = scalar * pr; di = scalar * pi;
        er = er + scalar * pr; ei = ei + scalar * pi;
        n++;
        fact *= n;
        /* power *= (0 + i x) */
        double nr = pr * 0 - pi * x, ni = pr * x + pi * 0;
        pr = nr; pi = ni;
    }
    *re = er; *im = ei;
}

double orc_reduce_phase(double phase)
{
    return phase - ((int)(phase / (2 * REF_PI))) * 2 * REF_PI;
}

void orc_overlap_instant(orc_grid *g, int cx, int cy, int cz, const double *md, int mi, int mj,
                         double mdisc, int reverse, double *inst)
{
    double sre = 0, sim = 0;
    const double *Ex = g->f[0], *Ey = g->f[1], *Hx = g->f[3], *Hy = g->f[4];
    for (int i = 0; i < g->nx; i++)
        for (int j = 0; j < g->ny; j++) {
            double xd = (i - cx) * (g->dx / mdisc);
            double yd = (j - cy) * (g->dx / mdisc);
            int mx = (int)xd + mi / 2, my = (int)yd + mj / 2;
            if (mx < 0 || mx >= mi || my < 0 || my >= mj) continue;
            const double *e = md + 12 * (size_t)(mx + mi * my);
            double mExr = e[0], mExi = e[1], mEyr = e[2], mEyi = e[3];
            double mHxr = e[6], mHxi = e[7], mHyr = e[8], mHyi = e[9];
            if (reverse == 1) {
                mHxr = 0 - mHxr; mHxi = 0 - (-mHxi);
                mHyr = 0 - mHyr; mHyi = 0 - (-mHyi);
            }
            size_t q = IDX(g, i, j, cz);
            double ex = Ex[q], ey = Ey[q], hx = Hx[q], hy = Hy[q];
            double p1r = hx * mEyr, p1i = hx * mEyi;
            double p2r = 0 - hy * mExr, p2i = 0 - hy * mExi;
            double p3r = ey * mHxr, p3i = ey * mHxi;
            double p4r = 0 - ex * mHyr, p4i = 0 - ex * mHyi;
            sre = sre + ((p1r + p2r) + (p3r + p4r));
            sim = sim + ((p1i + p2i) + (p3i + p4i));
        }
    double s = (-0.5 * g->dx * g->dx);
    inst[0] = s * sre;
    inst[1] = s * sim;
}

/* timefield3d_mode_overlap (timefield3d.c:3176-3239) */
void orc_mode_overlap(orc_grid *g, int cx, int cy, int cz, double *md, int mi, int mj, double mdisc,
                      double phase, int reverse, double *cum, double *inst)
{
    orc_mode_power_normalize(md, mi, mj, mdisc);
    orc_overlap_instant(g, cx, cy, cz, md, mi, mj, mdisc, reverse, inst);
    double tr, ti;
    orc_cexp_series(orc_reduce_phase(phase), &tr, &ti);
    cum[0] = cum[0] + (tr * inst[0] - ti * inst[1]);
    cum[1] = cum[1] + (tr * inst[1] + ti * inst[0]);
}

/* timefield3d_update_fourier_fields_y_slice (timefield3d.c:2922-2943) */
void orc_dft_y_slice(orc_grid *g, double phase, int slice, double *acc)
{
    double tr, ti;
    orc_cexp_series(orc_reduce_phase(phase), &tr, &ti);
    for (int k = 0; k < g->nz; k++)
        for (int i = 0; i < g->nx; i++) {
            size_t q = IDX(g, i, slice, k);
            for (int m = 0; m < 6; m++) {
                double f = g->f[m][q];
                double *a = acc + 2 * (m + 6 * ((size_t)i + (size_t)g->nx * k));
                a[0] = a[0] + f * tr;
                a[1] = a[1] + f * ti;
            }
        }
}

/* ---------------------------------------------------------------------------
 * Taper (adjoint3d.c:259-418).  The stored edge pixel uses integer division
 * inside round() (adjoint3d.c:276,285), so i = edge[n] + trunc(d*(k-k0)/(k1-k0)).
 * ------------------------------------------------------------------------- */
void orc_taper_store(orc_grid *g, int seg_num, int start, int end, int bottom, int top,
                     const int *left, const int *right, int t, double *store)
{
    int length = end - start, height = top - bottom;
    for (int n = 0; n < seg_num; n++) {
        int seg_mid = start + (n * length) / seg_num;
        int seg_fwd = start + ((n + 1) * length) / seg_num;
        for (int k = seg_mid; k < seg_fwd; k++)
            for (int j = bottom; j < top; j++)
                for (int e = 0; e < 2; e++) {
                    const int *edge = e == 0 ? right : left;
                    int i = edge[n] + ((edge[n + 1] - edge[n]) * (k - seg_mid)) / (seg_fwd - seg_mid);
                    size_t q = IDX(g, i, j, k);
                    double *s = store + 3 * (e + 2 * ((size_t)(j - bottom) + (size_t)height * ((k - start) + (size_t)length * t)));
                    s[0] = g->f[0][q]; s[1] = g->f[1][q]; s[2] = g->f[2][q];
                }
    }
}

/* adjoint3d_taper_calculate_ep_gradient (adjoint3d.c:339-373) */
void orc_taper_ep_gradient(int height, int length, int duration, const double *fwd, const double *adj,
                           double *ep_grad)
{
    for (int e = 0; e < 2; e++)
        for (int j = 0; j < height; j++)
            for (int k = 0; k < length; k++) {
                double sum = 0;
                for (int t = 0; t < duration; t++) {
                    size_t fi = 3 * (e + 2 * (j + (size_t)height * (k + (size_t)length * t)));
                    for (int m = 0; m < 3; m++) sum += fwd[fi + m] * adj[fi + m];
                }
                ep_grad[e + 2 * (j + height * k)] = sum;
            }
}

/* adjoint3d_taper_calculate_gradients_from_ep_gradient (adjoint3d.c:375-418) */
void orc_taper_vertex_gradient(int seg_num, int height, int length, const double *ep_grad,
                               double ep_diff, double *left_grad, double *right_grad)
{
    left_grad[0] = 0; right_grad[0] = 0;
    for (int n = 1; n < seg_num; n++) {
        left_grad[n] = 0; right_grad[n] = 0;
        int seg_bck = ((n - 1) * length) / seg_num;
        int seg_mid = (n * length) / seg_num;
        int seg_fwd = ((n + 1) * length) / seg_num;
        for (int k = seg_bck; k < seg_mid; k++)
            for (int j = 0; j < height; j++) {
                double w = (double)(k - seg_bck) / (double)(seg_mid - seg_bck);
                right_grad[n] += w * ep_grad[0 + 2 * (j + height * k)] * ep_diff;
                left_grad[n] -= w * ep_grad[1 + 2 * (j + height * k)] * ep_diff;
            }
        for (int k = seg_mid; k < seg_fwd; k++)
            for (int j = 0; j < height; j++) {
                double w = (double)(seg_fwd - k) / (double)(seg_fwd - seg_mid);
                right_grad[n] += w * ep_grad[0 + 2 * (j + height * k)] * ep_diff;
                left_grad[n] -= w * ep_grad[1 + 2 * (j + height * k)] * ep_diff;
            }
    }
    left_grad[seg_num] = 0; right_grad[seg_num] = 0;
}
