// engine.h -- device-side state of a grid and of a taper (internal header).
//
// A reference `timefield3d` is passed by value everywhere, so the engine keys
// its device state on the struct's `fields` pointer (unique per grid, shared by
// every by-value copy).  Tapers are keyed on their `left` pointer, modes on
// `fields.m`.
#pragma once

#include <complex>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fdtd_b200.h"
#include "kernels.h"

namespace fdtd {

// ---- mode solver (mode_solver.cu) --------------------------------------------
bool mode_apply_beta2_device(const mode &in, double omega, mode &out);
bool mode_solve_device(mode *psi, double omega, double tol, const mode *prev, int nprev, int size, int confinement,
                       int lateral_symmetry, int max_restarts, std::complex<double> *beta_out, int *restarts_out);

// ---- status ----------------------------------------------------------------
void set_error(int code, const char *fmt, ...);
bool cuda_ok(cudaError_t e, const char *what);
bool device_available();

// ---- device modes ------------------------------------------------------------
struct DevMode {
    const void *key = nullptr;
    uint64_t fingerprint = 0;
    int mi = 0, mj = 0;
    double disc = 0;
    double2 *d = nullptr;
};
// registers (power-normalising the host mode on first sight) and returns the
// device copy; null on failure
DevMode *mode_device(const mode &m);
void mode_release(const void *key);
// host power normalisation, mode.c:1267-1379
double mode_power_norm_host(const mode &m);
void mode_power_normalize_host(const mode &m);
// private power-normalised device copy of a mode (monitors, schedules), by handle
const void *priv_mode_new(const mode &m);
void priv_mode_free(const void *key);

// ---- grid ------------------------------------------------------------------
enum { kMatEp = 1, kMatMu = 2, kMatSig = 4, kMatAll = 7 };

struct Plane {
    int k;
    float *p;
};

struct Monitor {
    int cx, cy, cz, reverse, nfreq;
    const void *mode_key;
    double *d_omega = nullptr;
    double2 *d_acc = nullptr;   // 2*nfreq: (sum, compensation)
};

struct ProbeRec {
    ProbeJob job;
    int cap;
};

struct Schedule {
    bool active = false;
    int cx, cy, cz, reverse, adjoint, n;
    double kappa = 0, wre = 1, wim = 0;   // exact adjoint (adjoint 2)
    const void *mode_key = nullptr;
    double *d_sched = nullptr;   // 3*n: amplitude, cos, sin
};

struct TaperBind {
    const void *taper_key;
    int which, t0, dir;
};

struct Grid {
    timefield3d h{};          // host struct (pointers are the host mirrors)
    int nx = 0, ny = 0, nz = 0;
    long long n = 0;
    double dx = 0;
    int prec = FDTD_F64;
    int boundary = FDTD_BOUNDARY_MUR;
    int yee_variant = FDTD_YEE_AUTO;   // FP32 fast path: flat kernels or plane-streaming fused kernel

    // device state
    bool dev = false;
    cudaStream_t st = nullptr;
    cudaStream_t side = nullptr;      // second stream of the flat4 CPML shell kernels
    unsigned *d_done = nullptr;       // completion count of the step-tail kernel
    bool in_run = false;              // steps enqueued by run_steps end with the step-tail kernel
    int material_uploads = 0;         // the host mirrors are pinned at the second upload
    bool mirrors_pinned = false;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    void *f[2][6] = {};       // field sets; set 1 is the ping-pong buffer of the fused path
    int cur = 0;
    void *old[6] = {};        // Mur snapshot
    float *ep[3] = {}, *mu[3] = {}, *sig[6] = {};
    bool sig_e = false, sig_m = false, mu_nonunit = false;
    int mat_dirty = kMatAll;          // host material arrays newer than the device copies
    bool fields_from_host = false;   // host mirror must be uploaded before next use
    bool host_mirror_written = false; // a sync wrote psi.fields / fourier_fields
    bool host_sources_written = false; // timefield3d_set_source_value wrote psi.sources
    void **d_fptr[2] = {};           // device arrays of the 6 field pointers per set
    bool pp_synced = false;          // set 1-cur equals set cur on the shell (fused path)

    // CPML
    int L = 0, order = 3;
    double smax = -1, kmax = 1, amax = 0;
    double prof_dt = 0;
    void *psi[2][3][4] = {};
    void *prof[6][3] = {};

    // FP32 fused-path coefficients
    float *cb[3] = {}, *ca[3] = {};
    double coef_dt = 0;
    bool coef_valid = false;
    FusedMaps *fmaps[2] = {};        // TMA descriptors with set s as input (null: cp.async kernel)
    // one-pass streaming step (yee_stream.cu): tile plan of this grid's shape
    StreamPlan splan;
    StreamTile *d_tiles = nullptr;
    int splan_key[6] = {-1, -1, -1, -1, -1, -1};   // nx ny nz L lossy nsm the plan was built for
    int *d_err = nullptr;            // device error flag (a bounded wait gave up)
    int *h_err = nullptr;            // pinned

    // sources
    std::vector<Plane> planes;
    std::vector<float *> plane_pool;

    // step counter, overlap scratch
    long long *d_step = nullptr;
    long long host_steps = 0;
    OverlapJob *d_jobs = nullptr;       // monitors
    int jobs_cap = 0, njobs = 0;
    long long job_cells = 0;        // largest overlap window of the jobs
    OverlapJob *d_job1 = nullptr;       // single compat overlap
    double2 *d_partials = nullptr;
    double2 *d_inst = nullptr;
    double2 *h_inst = nullptr;          // pinned
    std::vector<Monitor> monitors;

    // probes
    std::vector<ProbeRec> probes;
    ProbeJob *d_probes = nullptr;
    double *d_probe_buf = nullptr;
    int *d_probe_count = nullptr;
    int probe_cap = 0;

    // running DFTs: whole grid, and y-slices by index
    double2 *d_dft_full = nullptr;
    std::map<int, double2 *> d_dft_slice;

    // scheduled source, taper binds
    Schedule sched;
    std::vector<TaperBind> binds;

    // staging
    double *d_aos = nullptr;            // 6n doubles, for host mirror transfers
    int *d_flag = nullptr;              // 12 material flags
    int *h_flag = nullptr;              // pinned

    // captured step graphs: [0] untimed; [1],[2] alternate when kernel timing is on
    cudaGraphExec_t graph[3] = {};
    int graph_steps[3] = {};
    double graph_dt[3] = {};
    uint64_t graph_version[3] = {};
    int graph_cur[3] = {};
    long long graph_nodes[3] = {};      // kernel launches per replay
    uint64_t version = 1;               // bumped on any configuration change

    // kernel timing: an event pair around the Yee update of every captured
    // step of one graph replay in `ktime` (0: off)
    int ktime = 0;
    long long kreplay = 0;              // graph replays since timing was set
    cudaEvent_t kev[2][64] = {};        // per timed graph, 2 per step
    bool kpending[2] = {false, false};
    cudaEvent_t *cap_ev = nullptr;      // events of the graph being captured
    int cap_step = 0;
    double ktime_ms = 0;
    long long ktime_n = 0;

    // multi-step wavefront launches (FDTD_YEE_WAVE, yee_wave.cu)
    struct Wave {
        int steps = 64, sweep = 16, group = 2;  // steps per launch, steps per sweep, blocks per ticket
        // configuration the device tables were built for
        uint64_t version = 0;
        int built_steps = 0, built_sweep = 0, built_group = 0, built_sched_k = -2;
        std::vector<WaveItem> items;        // kept: the source of the asynchronous upload
        WaveItem *d_items = nullptr;
        int tickets = 0, nparts = 1;
        unsigned *d_cnt = nullptr;
        double2 *d_part = nullptr;
        float *d_ring = nullptr;
        int grid[2] = {0, 0};               // co-resident blocks: lossless, lossy
        cudaEvent_t ev[2][2] = {};          // kernel timing: one pair per timed launch
        bool pending[2] = {false, false};
        int timed_steps[2] = {0, 0};
    } wave;
    std::vector<int> job_z;               // plane of each overlap job (d_jobs order)

    ~Grid();
};

Grid *grid_lookup(const timefield3d &psi, bool quiet = false);
Grid *grid_register(const timefield3d &psi);
void grid_unregister(const timefield3d &psi);

// device lifetime
bool grid_ensure_device(Grid *g);              // allocate device arrays, upload what is dirty
bool grid_upload_materials(Grid *g);
bool grid_upload_fields(Grid *g);              // host mirror -> device
bool grid_check_device_error(Grid *g);         // waits; FDTD_ERR_TIMEOUT if a device wait gave up
bool grid_download_fields(Grid *g);            // device -> host mirror (waits)
bool grid_set_precision(Grid *g, int prec);
bool grid_prepare_step(Grid *g, double dt);    // profiles / coefficients for dt
Plane *grid_plane(Grid *g, int k, bool create);
void grid_zero(Grid *g);
bool grid_checkpoint_save(Grid *g, const char *path);
bool grid_checkpoint_load(Grid *g, const char *path);
void inject_allocation_failures(int n);

// NVTX range for the duration of a scope (tracing with nsys / ncu; a no-op
// without a tool attached)
struct TraceRange {
    explicit TraceRange(const char *name);
    ~TraceRange();
};

// queued work
bool enqueue_step(Grid *g, double dt, bool with_extras);
bool enqueue_after_step(Grid *g, double dt);
bool run_steps(Grid *g, double dt, int nsteps);
bool run_sweep(const std::vector<Grid *> &gs, double dt, const std::vector<int> &nsteps, int steps_per_launch,
               int ty_cap, double tiles_per_sm);
bool drain_kernel_timing(Grid *g, int set);
bool rebuild_jobs(Grid *g);

// typed helpers
template <typename T> GridView<T> view(Grid *g, int set);
template <typename T> CpmlView<T> cpml_view(Grid *g, int in_set);
SourcePlanes source_table(Grid *g);

// taper
struct TaperDev {
    const void *key = nullptr;
    int seg_num = 0, start = 0, end = 0, bottom = 0, top = 0, duration = 0;
    int height = 0, length = 0, ncell = 0;
    int prec = -1;
    void *d_fwd = nullptr, *d_adj = nullptr;
    long long *d_cells = nullptr;
    std::vector<int> edges_seen;   // left/right copy the cell list was built for
    int nx_seen = 0, ny_seen = 0;
    double *d_grad = nullptr;
    ~TaperDev();
};
TaperDev *taper_lookup(const adjoint3d_taper &t, bool create);
void taper_unregister(const adjoint3d_taper &t);
bool taper_prepare(TaperDev *td, const adjoint3d_taper &t, Grid *g);
bool enqueue_taper_store(TaperDev *td, Grid *g, int which, int t_index, const long long *d_step, int t0, int dir);

std::mutex &api_mutex();

}  // namespace fdtd
