// kernels.h -- host-side launchers of the device kernels (internal header).
#pragma once

#include <cmath>
#include <vector>

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "common.cuh"

namespace fdtd {

// host-side count of kernel launches issued by this library (engine.cu)
void note_launch(int n = 1);
long long launch_count();

// Cells [wi, wi + wni) x [wj, wj + wnj) of an nx x ny plane outside which no
// cell maps to a sample of an mi x mj mode centred on (cx, cy) with ratio
// r = grid disc / mode disc: along x the sample index (int)((i - cx) r) + mi/2
// lies in [0, mi) only when -(mi/2) - 1 < (i - cx) r < mi - mi/2 (truncation
// toward zero), and likewise along y.  The window keeps two cells of margin
// beyond those bounds, so it is a superset under any rounding of the product;
// the kernels still test every cell, so the window only removes work.
struct ModeWindow {
    int wi, wj, wni, wnj;
};

inline void mode_window_axis(int n, int c, int m, double r, int &lo, int &cnt)
{
    if (!(r > 0) || !std::isfinite(r)) {   // no usable bound: the whole axis
        lo = 0;
        cnt = n;
        return;
    }
    double a = c + std::floor((double)(-(m / 2) - 1) / r) - 1;
    double b = c + std::ceil((double)(m - m / 2) / r) + 1;
    if (a < 0) a = 0;
    if (b > n - 1) b = n - 1;
    if (b < a) {
        lo = 0;
        cnt = 0;
        return;
    }
    lo = (int)a;
    cnt = (int)(b - a) + 1;
}

inline ModeWindow mode_window(int nx, int ny, int cx, int cy, int mi, int mj, double r)
{
    ModeWindow w{};
    mode_window_axis(nx, cx, mi, r, w.wi, w.wni);
    mode_window_axis(ny, cy, mj, r, w.wj, w.wnj);
    if (w.wni == 0 || w.wnj == 0) w.wni = w.wnj = 0;
    return w;
}

// one overlap reduction: plane cz of the grid against a device mode
struct OverlapJob {
    int cx, cy, cz;
    int mi, mj;
    int reverse;
    double ratio;           // grid disc / mode disc
    const double2 *mode;    // 6*mi*mj complex, entry 6*(i + mi*j) + m
    double2 *inst;          // instantaneous overlap out (or null)
    double2 *acc;           // per-frequency (sum, compensation) pairs (or null)
    const double *omega;    // n_freq angular frequencies
    int nfreq;
    ModeWindow win;         // mode_window of (cx, cy, mi, mj, ratio)
};

// plane source written from a complex mode (timefield3d_mode_source and
// its adjoint); sched != null: per-step (amplitude, cos, sin) triples
struct SourceJob {
    float *plane;               // 6 components of nx*ny
    const float *ep[3], *mu[3]; // material of the source plane
    int nx, ny, cx, cy;
    const double2 *mode;
    int mi, mj;
    double ratio;
    const double *sched;
    int nsched;
    int reverse, adjoint;       // adjoint 2: exact discrete adjoint of an overlap monitor (see plane_ops.cuh)
    double kappa, wre, wim;     // adjoint 2: disc^2 / (2 delta_t) and the complex weight of the objective
    ModeWindow win;             // set by launch_mode_source_job / the tail launcher
};

// one launch at the end of a run step: overlap monitors of the step, the
// scheduled source of the next step (src.plane != null) and the step counter
struct TailArgs {
    const void *const *f;       // device array of the 6 field pointers
    int nx, ny;
    const OverlapJob *jobs;
    int njobs, nparts;
    long long cells;            // largest overlap window of the jobs (cells)
    double2 *partials;
    double scale, dt;
    long long *step;
    SourceJob src;
    int src_blocks;
    unsigned *done;             // completion count, 0 between launches
};

struct ProbeJob {
    long long q;
    int m;
};

// yee_split.cu
template <typename T>
void launch_update_E(const GridView<T> &g, const CpmlView<T> &c, const SourcePlanes &s, T dt, T divisor, int k_lo,
                     int k_hi, bool sig, bool cpml, bool expl, cudaStream_t st);
template <typename T>
void launch_update_H(const GridView<T> &g, const CpmlView<T> &c, const SourcePlanes &s, T dt, T divisor, int k_lo,
                     int k_hi, bool sig, bool mu, bool cpml, bool expl, cudaStream_t st);
template <typename T> void launch_save_shell(const GridView<T> &g, cudaStream_t st);
template <typename T> void launch_mur(const GridView<T> &g, T dt, T dx, int efield, int ks, int ke, cudaStream_t st);
template <typename T> void launch_aos_to_soa(const double *aos, T *const d[6], long long n, cudaStream_t st);
template <typename T> void launch_soa_to_aos(double *aos, T *const s[6], long long n, cudaStream_t st);

// yee_fused.cu (FP32 single-pass E+H step)
struct FusedArgs {
    int nx, ny, nz;
    const float *f_in[6];
    float *f_out[6];
    const float *cb[3];      // E curl coefficients, per component (main_coeff / dx)
    const float *ca[3];      // E self coefficients (null: lossless, ca = 1)
    float hb;                // H curl coefficient (dt / (mu dx)), uniform mu = 1, no magnetic loss
    float dx;
    int L;                   // CPML thickness (0: none)
    const float *psi_in[3][4];
    float *psi_out[3][4];
    const float *prof[6][3];
    SourcePlanes src;
    // multi-step launches: per-step copies of the scheduled source plane
    // (plane ring_k), ring_stride floats apart; null otherwise
    const float *ring;
    int ring_k;
    long long ring_stride;
};
int fused_supported(int nx, int ny, int nz);
void launch_fused_step(const FusedArgs &a, cudaStream_t st);

// yee_flat.cu (FP32 step as two flat, one-thread-per-cell kernels, in place)
struct FlatArgs {
    int nx, ny, nz;
    float *f[6];
    const float *cb[3];
    const float *ca[3];      // null: lossless
    float hb, dx;
    int L;
    float *psi[3][4];
    const float *prof[6][3];
    SourcePlanes src;
    // multi-step launches: per-step copies of the scheduled source plane
    // (plane ring_k), ring_stride floats apart; null otherwise
    const float *ring;
    int ring_k;
    long long ring_stride;
};
void launch_flat_step(const FlatArgs &a, cudaStream_t st, cudaEvent_t mid);
int flat4_supported(int nx, int nz);
// cells of one flat4 launch: planes kA..kA+nA-1 then kB.., `count` (group, row)
// slots per plane laid out by region kind: 0 whole planes, 1 interior box
// [gL, gR) x [L, ny-L), 3 y-slab rows x [gL, gR), 4 all rows x the columns
// outside [gL, gR)
struct Region4 {
    int kA, nA, kB;
    int count;
    int gL, gR, L;
};
// block plan of the merged CPML launch: z-slab planes get nbz blocks each,
// middle planes nbm = nb_box + nb_y + nb_x
struct Plan4 {
    int L, nmid;
    int nbz, nbm, nb_box, nb_y;
    Region4 zs, box, yrows, xcols;
};
bool flat4_split_supported(const FlatArgs &a);
// block plan of one field update: a CPML grid that splits (flat4_split_supported)
// gets the regions above; a grid without CPML (L = 0) whole planes 1..nz-2 in zs
// with W = 4, nbz blocks per plane
Plan4 flat4_plan(const FlatArgs &a);
// E then H update.  With a CPML and a side stream the interior box runs on `st`
// and the shell on `side` (fork/join through the two events) for each field.
void launch_flat4_step(const FlatArgs &a, cudaStream_t st, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join);

// yee_stream.cu: the FP32 step in one pass (E and H of every cell), z-planes
// streamed through shared memory by (band of rows, chunk of planes) tiles
struct StreamTile {
    int j0, rows;            // owned rows [j0, j0 + rows), all in 1..ny-2
    int k0, k1;              // owned planes [k0, k1), all in 1..nz-2
};
struct StreamPlan {
    int ty = 0;              // rows of the largest band (shared memory holds ty + 1 rows)
    int threads = 0;         // block size: (ty + 1) rows of nx/4 threads, rounded up to a warp
    size_t smem = 0;         // dynamic shared memory per block (bytes)
    std::vector<StreamTile> tiles;   // one block each, all resident at once
};
struct StreamArgs {
    int nx, ny, nz, L, ty;
    const float *f_in[6];
    float *f_out[6];
    const float *cb[3];
    const float *ca[3];      // null: lossless
    float hb, dx;
    const float *psi_in[3][4];
    float *psi_out[3][4];
    const float *prof[6][3];
    SourcePlanes src;
    const StreamTile *tiles;
};
constexpr size_t kStreamSmemBudget = 231424;   // dynamic shared memory per block: the sm_100 maximum less 1 KB of static room
// staged x-slab auxiliaries per row: 2L, padded to 16 bytes
__host__ __device__ inline int stream_xpsi_stride(int L) { return (2 * L + 3) & ~3; }
int stream_supported(int nx, int ny, int nz, bool lossy, int L);
// tiles for a grid over nsm blocks (one per SM); ty_cap > 0 caps the rows of a
// band (the autotuner's tile-shape knob); false when the grid cannot use the kernel
bool stream_plan(int nx, int ny, int nz, int L, bool lossy, int nsm, StreamPlan *out, int ty_cap = 0);
// the plan's cost estimate of one tile (relative)
double stream_tile_cost(int nx, int ny, int nz, int L, const StreamTile &t);
// allow `smem` bytes of dynamic shared memory for every instantiation and check
// that blocks of `threads` threads can launch (host, not stream-ordered)
bool stream_configure(size_t smem, int threads);
void launch_yee_stream(const StreamArgs &a, const StreamPlan &p, cudaStream_t st);

// yee_sweep.cu: many grids advanced together by persistent launches of S
// steps (see the file's header); one entry per grid per launch
constexpr int kSweepMaxGrids = 48;   // grids of one sweep call (their tile arguments sit in constant memory)
struct SweepGrid {
    StreamArgs args[2];          // input set p (output 1 - p); args[p].tiles = this grid's sweep tiles
    int ntiles;
    const float *const *fout[2]; // field pointers of the output set when the input is set p
    int nx, ny;
    const OverlapJob *jobs;
    int njobs, nparts;
    double2 *partials;           // [2][njobs * nparts], by step parity
    double scale, dt;
    SourceJob src;               // plane null: no scheduled source
    int src_warps;
    long long base;              // steps taken when the launch starts
    long long *step;             // the grid's device step counter
    int p0;                      // input set of the grid's first step in the launch
    int steps;                   // steps of this grid in the launch (0: idle)
};

struct SweepArgs {
    const SweepGrid *grids;
    int ngrids, steps;           // steps: the most of any grid
    const int2 *items;           // every grid's tiles as (grid, tile), most expensive first
    int nitems;
    unsigned *next;              // per step of the launch: next item to hand out (zero at launch start)
    unsigned *bar;               // barrier arrivals, zero when the launch starts
    int *err;                    // set when a barrier wait gives up
    unsigned long long wait_ns;
    unsigned arrivals;           // arrivals per barrier (the grid size)
};
bool sweep_setup(int *nsm);
cudaStream_t sweep_stream();
cudaEvent_t sweep_event();
int *sweep_err();
StreamTile **sweep_tiles(size_t bytes);     // grown device buffers owned by the sweep
double2 **sweep_partials(size_t bytes);
bool sweep_launch(const std::vector<std::vector<SweepGrid>> &launches, const std::vector<int> &steps,
                  const std::vector<int2> &items, bool cpml, bool lossy, int tpc, int threads, size_t smem,
                  unsigned long long wait_ns);
void launch_sweep_err_to_grid(const int *sweep, int *grid, cudaStream_t st);
bool sweep_barrier_selftest(unsigned long long limit_ns, int *timed_out);

// yee_wave.cu: S steps of the flat4 update in one persistent, cooperative
// launch, wavefront-ordered in z (see the file's header)
struct WaveItem {
    int t0;          // first ticket
    int desc;        // kind (0 E, 1 H, 2 overlaps) | plane << 2 | step << 17
    int nblocks;     // blocks of work (a ticket takes up to `group` of them)
    int pad;
    int2 dep[3];     // {counter, finished tickets needed}; counter -1: none
};
struct WaveArgs {
    const WaveItem *items;
    int nitems, tickets;
    unsigned *cnt;                // finished tickets per item, wave_counters(nz, steps)
    unsigned *next;               // next ticket to hand out (cnt + wave_counters)
    int nz, steps;
    const OverlapJob *jobs;       // monitors (device)
    int njobs, nparts;
    double2 *partials;            // [step][job][part]
    int group;                    // blocks of work per ticket
    int *err;                     // set to 1 when a wait gives up
    unsigned long long wait_ns;   // bound of one wait
};
struct WaveFinal {
    const OverlapJob *jobs;
    int njobs, nparts, steps;
    const double2 *partials;
    double scale, dt;
    long long *step;
    unsigned *done;               // completion count, 0 between launches
    SourceJob src;                // scheduled source (plane null: none)
};
// item list in ticket order (a ticket: up to `group` blocks of work of one
// item); job_z: plane of each monitor (all in 1..nz-2); returns 0, or -1 when
// the sizes are out of range
int wave_items(const Plan4 &p, int nz, int steps, int sweep, int group, const int *job_z, int njobs, int nparts,
               std::vector<WaveItem> &out, int &tickets);
int wave_counters(int nz, int steps);
// co-resident blocks of the wavefront kernel on the current device (0: cannot run)
int wave_grid(bool lossy);
// counters reset, source ring (sched non-null; a.ring_k = its plane), the
// wavefront launch, then the finalize kernel
cudaError_t launch_wave(const FlatArgs &a, const Plan4 &p, const WaveArgs &w, int grid, const SourceJob *sched,
                        float *ring, const WaveFinal &fin, cudaStream_t st);

// yee_fused_tma.cu (the same step with TMA staging; needs nx % 4 == 0)
struct FusedMaps {
    CUtensorMap h[3];    // H components of the input set, box (TX+8) x (TY+2)
    CUtensorMap e[3];    // E components of the input set, box (TX+4) x (TY+1)
    CUtensorMap cb[3];
    CUtensorMap ca[3];
};
int fused_tma_supported(int nx, int ny, int nz);
bool fused_make_maps(FusedMaps *m, const float *const f[6], const float *const cb[3], const float *const ca[3],
                     int nx, int ny, int nz);
void launch_fused_step_tma(const FusedArgs &a, const FusedMaps &m, int *err, cudaStream_t st);
void launch_wait_selftest(unsigned long long limit_ns, int *err, unsigned long long *elapsed_ns, cudaStream_t st);

// aux_kernels.cu
void launch_mode_source(float *plane, const float *const ep_plane[3], const float *const mu_plane[3], int nx, int ny,
                        int cx, int cy, const double2 *mode, int mi, int mj, double ratio, double amplitude,
                        double cph, double sph, const double *sched, const long long *step, int nsched, int reverse,
                        int adjoint, cudaStream_t st);
void launch_mode_source_job(const SourceJob &sj, double amplitude, double cph, double sph, const long long *step,
                            int step_offset, cudaStream_t st);
template <typename T>
void launch_step_tail(TailArgs a, cudaStream_t st);
void launch_set_value(float *p, long long idx, float v, cudaStream_t st);
int overlap_parts(long long cells);
// cells: the largest overlap window (win.wni * win.wnj) of the jobs
template <typename T>
void launch_overlap(const T *const *f_dev, int nx, int ny, const OverlapJob *jobs_dev, int njobs, long long cells,
                    double2 *partials, double scale, double dt, const long long *step, int step_offset,
                    cudaStream_t st);
template <typename T>
void launch_dft(const T *const *f_dev, int nx, int ny, int nz, int slice, int k_lo, int k_hi, double tr, double ti,
                double2 *acc, cudaStream_t st);
template <typename T>
void launch_probes(const T *const *f_dev, const ProbeJob *probes, int np, double *buf, int cap, int *count,
                   cudaStream_t st);
void launch_step_advance(long long *step, cudaStream_t st);
template <typename T>
void launch_taper_store(const T *const *f_dev, const long long *cells, int ncell, T *store, int t_index,
                        const long long *step, int t0, int dir, int duration, cudaStream_t st);
template <typename T>
void launch_ep_gradient(const T *fwd, const T *adj, int ncell, int duration, double *grad, cudaStream_t st);
template <typename T>
void launch_ep_gradient_exact(const T *fwd, const T *adj, int ncell, int duration, double *grad, cudaStream_t st);
void launch_check_finite(const float *a, long long n, int *bad, cudaStream_t st);

// umma_gemm.cu: BF16 GEMM on tcgen05 (pre = alpha A B^T + beta C32 + bias;
// act 0 identity / 1 GELU; A [M][lda], B [N][ldb], K-major)
struct GemmArgs {
    const __nv_bfloat16 *A;
    const __nv_bfloat16 *B;
    int lda, ldb, M, N, K;
    const float *bias;
    int act;
    float alpha, beta;
    float *C32;
    int ldc32;
    __nv_bfloat16 *C16;
    int ldc16;
    float *Z32;
    int ldz;
    int *err;
};
bool gemm_bf16_launch(const GemmArgs &a, cudaStream_t st);

}  // namespace fdtd
