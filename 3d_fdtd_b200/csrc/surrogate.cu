// surrogate.cu -- the surrogate network of the taper optimiser: an MLP
// n_in -> H -> H -> H -> n_out with GELU (20 -> 256 -> 256 -> 256 -> 22 in the
// optimiser: 142,614 parameters), BF16 weights and activations, FP32
// accumulation on the tcgen05 tensor cores (umma_gemm.cu), FP32 master
// weights, Adam.  New work (the reference optimises by the adjoint gradient
// alone); its CPU FP64 restatement is oracle/surrogate.py.
//
// Layout: layer l maps in_l -> out_l; W_l is stored [out_l][in_pad_l] (FP32
// master and BF16 copy, K-major for the forward GEMM) and transposed
// [in_pad_l][out_pad_l] in BF16 for the backward GEMM; padded columns are zero
// and stay zero (the padded inputs are zero, so their gradients are).
// Forward: Z_l = H_{l-1} W_l^T + b_l (FP32, kept), H_l = bf16(GELU(Z_l)),
// Y = H_3 W_4^T + b_4 (FP32).  Loss: mean over batch and outputs of (Y-T)^2.
// Backward per layer: db = column sums of dZ (FP32), dW = dZ^T H_{l-1}
// (GEMM over the batch, both operands transposed to K-major BF16),
// dH_{l-1} = dZ W_l, dZ_{l-1} = dH_{l-1} GELU'(Z_{l-1}); dX = dZ_1 W_1 for the
// input gradient.  Rounding points (BF16 operands of every GEMM) are the ones
// the restatement reproduces.
#include <cmath>
#include <cuda_bf16.h>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace fdtd {

namespace {

constexpr int kLayers = 4;

int pad8(int x) { return (x + 7) / 8 * 8; }

__device__ __forceinline__ float gelu_grad(float x)
{
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// f32 [rows][cols] -> bf16 [rows][ldo] (columns cols..ldo-1 zero)
__global__ void k_pack_bf16(const float *in, int rows, int cols, int ldi, __nv_bfloat16 *out, int ldo)
{
    const long long n = (long long)rows * ldo;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t / ldo), c = (int)(t % ldo);
        out[t] = __float2bfloat16_rn(c < cols ? in[(long long)r * ldi + c] : 0.0f);
    }
}

// bf16 [rows][ld_in] (cols used) -> bf16 [cols_pad][ld_out] transposed (rows -> columns), zero padded
__global__ void k_transpose_bf16(const __nv_bfloat16 *in, int rows, int cols, int ldi, __nv_bfloat16 *out,
                                 int cols_pad, int ldo)
{
    const long long n = (long long)cols_pad * ldo;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / ldo), r = (int)(t % ldo);
        out[t] = (c < cols && r < rows) ? in[(long long)r * ldi + c] : __float2bfloat16_rn(0.0f);
    }
}

// f32 master W [out][inp] -> bf16 W [out][inp] and W^T [inp][outp]
__global__ void k_cast_weights(const float *W, int out, int inp, int outp, __nv_bfloat16 *Wb, __nv_bfloat16 *WbT)
{
    const long long n = (long long)inp * outp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / outp), o = (int)(t % outp);
        const __nv_bfloat16 v = __float2bfloat16_rn(o < out ? W[(long long)o * inp + i] : 0.0f);
        WbT[t] = v;
        if (o < out) Wb[(long long)o * inp + i] = v;
    }
}

// dZ = 2 (Y - T) / (B n) (f32 [B][n] and bf16 [B][np]); loss += sum (Y-T)^2 / (B n)
__global__ void k_mse(const float *Y, const float *T, int B, int n, int np, float *dZ, __nv_bfloat16 *dZb,
                      double *loss)
{
    const long long cnt = (long long)B * np;
    const float s = 2.0f / ((float)B * (float)n);
    double acc = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cnt; t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t / np), c = (int)(t % np);
        float g = 0.0f;
        if (c < n) {
            const float d = Y[(long long)r * n + c] - T[(long long)r * n + c];
            acc += (double)d * d;
            g = s * d;
            dZ[(long long)r * n + c] = g;
        }
        dZb[t] = __float2bfloat16_rn(g);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(loss, acc / ((double)B * n));
}

// given dY directly: dZ (f32 [B][n]) and bf16 [B][np]
__global__ void k_seed_grad(const float *dy, int B, int n, int np, float *dZ, __nv_bfloat16 *dZb)
{
    const long long cnt = (long long)B * np;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cnt; t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t / np), c = (int)(t % np);
        const float g = c < n ? dy[(long long)r * n + c] : 0.0f;
        if (c < n) dZ[(long long)r * n + c] = g;
        dZb[t] = __float2bfloat16_rn(g);
    }
}

// dZ = dH * GELU'(Z): f32 [B][n] and bf16 [B][n]
__global__ void k_gelu_back(const float *dH, const float *Z, long long cnt, float *dZ, __nv_bfloat16 *dZb)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cnt; t += (long long)gridDim.x * blockDim.x) {
        const float g = dH[t] * gelu_grad(Z[t]);
        dZ[t] = g;
        dZb[t] = __float2bfloat16_rn(g);
    }
}

// db[c] = sum_r dZ[r][c], one thread per column, rows in order
__global__ void k_col_sum(const float *dZ, int B, int n, float *db)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float s = 0.0f;
    for (int r = 0; r < B; r++) s += dZ[(long long)r * n + c];
    db[c] = s;
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2,
                       float eps, float c1, float c2)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const float gt = g[t];
        const float mt = b1 * m[t] + (1.0f - b1) * gt;
        const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
        m[t] = mt;
        v[t] = vt;
        p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
    }
}

int blocks_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 2368); }

struct Mlp {
    int nin = 0, hid = 0, nout = 0;
    int in[kLayers], inp[kLayers], out[kLayers], outp[kLayers];
    float *W[kLayers] = {}, *b[kLayers] = {}, *gW[kLayers] = {}, *gb[kLayers] = {};
    float *mW[kLayers] = {}, *vW[kLayers] = {}, *mb[kLayers] = {}, *vb[kLayers] = {};
    __nv_bfloat16 *Wb[kLayers] = {}, *WbT[kLayers] = {};
    int step = 0;
    int cap = 0;
    float *xs = nullptr, *ts = nullptr, *dys = nullptr;   // f32 staging [cap][nin], [cap][nout]
    __nv_bfloat16 *X = nullptr, *XT = nullptr;
    __nv_bfloat16 *H[kLayers] = {}, *HT[kLayers] = {};
    float *Z[kLayers] = {}, *Y = nullptr, *dZf = nullptr, *dH = nullptr, *dX = nullptr;
    __nv_bfloat16 *dZb = nullptr, *dZbT = nullptr;
    double *loss = nullptr;
    int *err = nullptr;
    cudaStream_t st = nullptr;
    std::vector<void *> allocs;

    template <typename T> bool alloc(T **p, size_t count)
    {
        void *v = nullptr;
        if (!cuda_ok(cudaMalloc(&v, count * sizeof(T) + 16), "cudaMalloc(mlp)")) return false;
        allocs.push_back(v);
        *p = (T *)v;
        return cuda_ok(cudaMemsetAsync(v, 0, count * sizeof(T) + 16, st), "cudaMemsetAsync(mlp)");
    }
    ~Mlp()
    {
        if (st) cudaStreamSynchronize(st);
        for (void *p : allocs) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    }
    long long wcount(int l) const { return (long long)out[l] * inp[l]; }
    long long params() const
    {
        long long n = 0;
        for (int l = 0; l < kLayers; l++) n += (long long)out[l] * in[l] + out[l];
        return n;
    }
};

bool mlp_setup(Mlp &m, int nin, int hid, int nout, unsigned long long seed)
{
    m.nin = nin; m.hid = hid; m.nout = nout;
    const int ins[kLayers] = {nin, hid, hid, hid}, outs[kLayers] = {hid, hid, hid, nout};
    for (int l = 0; l < kLayers; l++) {
        m.in[l] = ins[l]; m.inp[l] = pad8(ins[l]); m.out[l] = outs[l]; m.outp[l] = pad8(outs[l]);
    }
    if (!cuda_ok(cudaStreamCreateWithFlags(&m.st, cudaStreamNonBlocking), "stream")) return false;
    if (!m.alloc(&m.loss, 1) || !m.alloc(&m.err, 1)) return false;
    for (int l = 0; l < kLayers; l++) {
        const long long nw = m.wcount(l);
        if (!m.alloc(&m.W[l], nw) || !m.alloc(&m.gW[l], nw) || !m.alloc(&m.mW[l], nw) || !m.alloc(&m.vW[l], nw) ||
            !m.alloc(&m.b[l], m.out[l]) || !m.alloc(&m.gb[l], m.out[l]) || !m.alloc(&m.mb[l], m.out[l]) ||
            !m.alloc(&m.vb[l], m.out[l]) || !m.alloc(&m.Wb[l], nw) ||
            !m.alloc(&m.WbT[l], (size_t)m.inp[l] * m.outp[l]))
            return false;
    }
    // PyTorch-Linear-like init: U(-1/sqrt(in), 1/sqrt(in)), seeded splitmix64
    unsigned long long s = seed;
    auto uni = [&s]() {
        s += 0x9E3779B97F4A7C15ull;
        unsigned long long z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    std::vector<float> hw, hb;
    for (int l = 0; l < kLayers; l++) {
        const double bound = 1.0 / std::sqrt((double)m.in[l]);
        hw.assign(m.wcount(l), 0.0f);
        for (int o = 0; o < m.out[l]; o++)
            for (int i = 0; i < m.in[l]; i++) hw[(size_t)o * m.inp[l] + i] = (float)((2 * uni() - 1) * bound);
        hb.resize(m.out[l]);
        for (auto &v : hb) v = (float)((2 * uni() - 1) * bound);
        if (!cuda_ok(cudaMemcpyAsync(m.W[l], hw.data(), hw.size() * 4, cudaMemcpyHostToDevice, m.st), "init") ||
            !cuda_ok(cudaMemcpyAsync(m.b[l], hb.data(), hb.size() * 4, cudaMemcpyHostToDevice, m.st), "init") ||
            !cuda_ok(cudaStreamSynchronize(m.st), "init"))
            return false;
    }
    return true;
}

bool refresh_bf16(Mlp &m)
{
    for (int l = 0; l < kLayers; l++) {
        note_launch();
        k_cast_weights<<<blocks_for((long long)m.inp[l] * m.outp[l]), 256, 0, m.st>>>(m.W[l], m.out[l], m.inp[l],
                                                                                        m.outp[l], m.Wb[l], m.WbT[l]);
    }
    return cuda_ok(cudaGetLastError(), "cast weights");
}

bool ensure_cap(Mlp &m, int B)
{
    if (B <= m.cap) return true;
    // buffers sized for B (old ones stay allocated until the network is freed)
    const int h = m.hid, mx = std::max(m.hid, m.outp[kLayers - 1]);
    if (!m.alloc(&m.xs, (size_t)B * m.nin) || !m.alloc(&m.ts, (size_t)B * m.nout) ||
        !m.alloc(&m.dys, (size_t)B * m.nout) || !m.alloc(&m.X, (size_t)B * m.inp[0]) ||
        !m.alloc(&m.XT, (size_t)m.inp[0] * B) || !m.alloc(&m.Y, (size_t)B * m.nout) ||
        !m.alloc(&m.dZf, (size_t)B * mx) || !m.alloc(&m.dH, (size_t)B * h) || !m.alloc(&m.dX, (size_t)B * m.inp[0]) ||
        !m.alloc(&m.dZb, (size_t)B * mx) || !m.alloc(&m.dZbT, (size_t)mx * B))
        return false;
    for (int l = 1; l < kLayers; l++)
        if (!m.alloc(&m.H[l], (size_t)B * h) || !m.alloc(&m.HT[l], (size_t)h * B) || !m.alloc(&m.Z[l], (size_t)B * h))
            return false;
    m.cap = B;
    return true;
}

GemmArgs gemm(const Mlp &m, const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *Bm, int ldb, int M, int N, int K)
{
    GemmArgs g{};
    g.A = A; g.lda = lda; g.B = Bm; g.ldb = ldb; g.M = M; g.N = N; g.K = K;
    g.alpha = 1.0f; g.beta = 0.0f; g.err = m.err;
    return g;
}

bool forward(Mlp &m, int B)
{
    note_launch();
    k_pack_bf16<<<blocks_for((long long)B * m.inp[0]), 256, 0, m.st>>>(m.xs, B, m.nin, m.nin, m.X, m.inp[0]);
    const __nv_bfloat16 *hin = m.X;
    int ldin = m.inp[0];
    for (int l = 0; l < kLayers; l++) {
        GemmArgs g = gemm(m, hin, ldin, m.Wb[l], m.inp[l], B, m.out[l], m.inp[l]);
        g.bias = m.b[l];
        if (l < kLayers - 1) {
            g.act = 1;
            g.Z32 = m.Z[l + 1]; g.ldz = m.hid;
            g.C16 = m.H[l + 1]; g.ldc16 = m.hid;
            hin = m.H[l + 1];
            ldin = m.hid;
        } else {
            g.C32 = m.Y; g.ldc32 = m.nout;
        }
        if (!gemm_bf16_launch(g, m.st)) return false;
    }
    return true;
}

// backward from dZ of the last layer (already in dZf / dZb); weight grads
// when `weights`, dX when `input`
bool backward(Mlp &m, int B, bool weights, bool input)
{
    for (int l = kLayers - 1; l >= 0; l--) {
        const int o = m.out[l], op = m.outp[l], ld = (l == kLayers - 1) ? op : m.hid;
        if (weights) {
            note_launch();
            k_col_sum<<<(o + 127) / 128, 128, 0, m.st>>>(m.dZf, B, o, m.gb[l]);
            note_launch();
            k_transpose_bf16<<<blocks_for((long long)op * B), 256, 0, m.st>>>(m.dZb, B, o, ld, m.dZbT, op, B);
            const __nv_bfloat16 *hT;
            if (l == 0) {
                note_launch();
                k_transpose_bf16<<<blocks_for((long long)m.inp[0] * B), 256, 0, m.st>>>(m.X, B, m.inp[0], m.inp[0],
                                                                                          m.XT, m.inp[0], B);
                hT = m.XT;
            } else {
                note_launch();
                k_transpose_bf16<<<blocks_for((long long)m.hid * B), 256, 0, m.st>>>(m.H[l], B, m.hid, m.hid, m.HT[l],
                                                                                       m.hid, B);
                hT = m.HT[l];
            }
            GemmArgs g = gemm(m, m.dZbT, B, hT, B, o, m.inp[l], B);
            g.C32 = m.gW[l]; g.ldc32 = m.inp[l];
            if (!gemm_bf16_launch(g, m.st)) return false;
        }
        if (l > 0) {
            GemmArgs g = gemm(m, m.dZb, ld, m.WbT[l], op, B, m.hid, op);
            g.C32 = m.dH; g.ldc32 = m.hid;
            if (!gemm_bf16_launch(g, m.st)) return false;
            note_launch();
            k_gelu_back<<<blocks_for((long long)B * m.hid), 256, 0, m.st>>>(m.dH, m.Z[l], (long long)B * m.hid,
                                                                              m.dZf, m.dZb);
        } else if (input) {
            GemmArgs g = gemm(m, m.dZb, m.hid, m.WbT[0], m.hid, B, m.inp[0], m.hid);
            g.C32 = m.dX; g.ldc32 = m.inp[0];
            if (!gemm_bf16_launch(g, m.st)) return false;
        }
    }
    return cuda_ok(cudaGetLastError(), "mlp backward");
}

bool upload(Mlp &m, float *dst, const float *src, size_t count)
{
    return cuda_ok(cudaMemcpyAsync(dst, src, count * sizeof(float), cudaMemcpyHostToDevice, m.st), "mlp H2D");
}

bool check_err(Mlp &m)
{
    int e = 0;
    if (!cuda_ok(cudaMemcpyAsync(&e, m.err, sizeof(int), cudaMemcpyDeviceToHost, m.st), "err D2H") ||
        !cuda_ok(cudaStreamSynchronize(m.st), "mlp sync"))
        return false;
    if (e) {
        cudaMemsetAsync(m.err, 0, sizeof(int), m.st);
        set_error(FDTD_ERR_TIMEOUT, "surrogate: a tensor-core GEMM wait gave up");
        return false;
    }
    return true;
}

bool batch_ok(const Mlp *m, int B)
{
    if (!m || B <= 0 || B % 8) {
        set_error(FDTD_ERR_ARG, "surrogate: batch %d must be a positive multiple of 8", B);
        return false;
    }
    return true;
}

std::vector<Mlp *> &nets()
{
    static std::vector<Mlp *> v;
    return v;
}

Mlp *net(void *h)
{
    for (auto *p : nets())
        if (p == h) return p;
    set_error(FDTD_ERR_ARG, "surrogate: unknown network handle");
    return nullptr;
}

}  // namespace
}  // namespace fdtd

using namespace fdtd;

extern "C" {

void *fdtd_mlp_new(int n_in, int hidden, int n_out, unsigned long long seed)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    if (!device_available()) return nullptr;
    if (n_in <= 0 || hidden <= 0 || hidden % 8 || n_out <= 0) {
        set_error(FDTD_ERR_ARG, "fdtd_mlp_new: n_in %d hidden %d (multiple of 8) n_out %d", n_in, hidden, n_out);
        return nullptr;
    }
    auto *m = new Mlp;
    if (!mlp_setup(*m, n_in, hidden, n_out, seed) || !refresh_bf16(*m) || !check_err(*m)) {
        delete m;
        return nullptr;
    }
    nets().push_back(m);
    return m;
}

long long fdtd_mlp_param_count(void *h)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    Mlp *m = net(h);
    return m ? m->params() : -1;
}

// flat order: W_1 [out][in], b_1, ..., W_4, b_4 (unpadded)
int fdtd_mlp_get_params(void *h, float *out)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    Mlp *m = net(h);
    if (!m || !out) return FDTD_ERR_ARG;
    if (!cuda_ok(cudaStreamSynchronize(m->st), "sync")) return fdtd_last_error();
    size_t off = 0;
    std::vector<float> w;
    for (int l = 0; l < kLayers; l++) {
        w.resize(m->wcount(l));
        if (!cuda_ok(cudaMemcpy(w.data(), m->W[l], w.size() * 4, cudaMemcpyDeviceToHost), "D2H")) return fdtd_last_error();
        for (int o = 0; o < m->out[l]; o++)
            for (int i = 0; i < m->in[l]; i++) out[off++] = w[(size_t)o * m->inp[l] + i];
        if (!cuda_ok(cudaMemcpy(out + off, m->b[l], m->out[l] * 4, cudaMemcpyDeviceToHost), "D2H")) return fdtd_last_error();
        off += m->out[l];
    }
    return FDTD_OK;
}

int fdtd_mlp_set_params(void *h, const float *in)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    Mlp *m = net(h);
    if (!m || !in) return FDTD_ERR_ARG;
    if (!cuda_ok(cudaStreamSynchronize(m->st), "sync")) return fdtd_last_error();
    size_t off = 0;
    std::vector<float> w;
    for (int l = 0; l < kLayers; l++) {
        w.assign(m->wcount(l), 0.0f);
        for (int o = 0; o < m->out[l]; o++)
            for (int i = 0; i < m->in[l]; i++) w[(size_t)o * m->inp[l] + i] = in[off++];
        if (!cuda_ok(cudaMemcpy(m->W[l], w.data(), w.size() * 4, cudaMemcpyHostToDevice), "H2D") ||
            !cuda_ok(cudaMemcpy(m->b[l], in + off, m->out[l] * 4, cudaMemcpyHostToDevice), "H2D"))
            return fdtd_last_error();
        off += m->out[l];
        cudaMemset(m->mW[l], 0, m->wcount(l) * 4); cudaMemset(m->vW[l], 0, m->wcount(l) * 4);
        cudaMemset(m->mb[l], 0, m->out[l] * 4); cudaMemset(m->vb[l], 0, m->out[l] * 4);
    }
    m->step = 0;
    return refresh_bf16(*m) && check_err(*m) ? FDTD_OK : fdtd_last_error();
}

int fdtd_mlp_forward(void *h, const float *x, int batch, float *y)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    Mlp *m = net(h);
    if (!batch_ok(m, batch) || !x || !y) return FDTD_ERR_ARG;
    if (!ensure_cap(*m, batch) || !upload(*m, m->xs, x, (size_t)batch * m->nin) || !forward(*m, batch)) return fdtd_last_error();
    if (!cuda_ok(cudaMemcpyAsync(y, m->Y, (size_t)batch * m->nout * 4, cudaMemcpyDeviceToHost, m->st), "D2H"))
        return fdtd_last_error();
    return check_err(*m) ? FDTD_OK : fdtd_last_error();
}

static int grads_common(Mlp *m, const float *x, const float *t, int batch, double *loss)
{
    if (!ensure_cap(*m, batch) || !upload(*m, m->xs, x, (size_t)batch * m->nin) ||
        !upload(*m, m->ts, t, (size_t)batch * m->nout) || !forward(*m, batch))
        return fdtd_last_error();
    if (!cuda_ok(cudaMemsetAsync(m->loss, 0, sizeof(double), m->st), "memset")) return fdtd_last_error();
    const int L = kLayers - 1;
    note_launch();
    k_mse<<<blocks_for((long long)batch * m->outp[L]), 256, 0, m->st>>>(m->Y, m->ts, batch, m->nout, m->outp[L],
                                                                          m->dZf, m->dZb, m->loss);
    if (!backward(*m, batch, true, false)) return fdtd_last_error();
    if (loss && !cuda_ok(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->st), "D2H"))
        return fdtd_last_error();
    return FDTD_OK;
}

int fdtd_mlp_gradients(void *h, const float *x, const float *t, int batch, float *grad, double *loss)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    Mlp *m = net(h);
    if (!batch_ok(m, batch) || !x || !t) return FDTD_ERR_ARG;
    int r = grads_common(m, x, t, batch, loss);
    if (r != FDTD_OK || !check_err(*m)) return r != FDTD_OK ? r : fdtd_last_error();
    if (grad) {
        size_t off = 0;
        std::vector<float> w;
        for (int l = 0; l < kLayers; l++) {
            w.resize(m->wcount(l));
            if (!cuda_ok(cudaMemcpy(w.data(), m->gW[l], w.size() * 4, cudaMemcpyDeviceToHost), "D2H")) return fdtd_last_error();
            for (int o = 0; o < m->out[l]; o++)
                for (int i = 0; i < m->in[l]; i++) grad[off++] = w[(size_t)o * m->inp[l] + i];
            if (!cuda_ok(cudaMemcpy(grad + off, m->gb[l], m->out[l] * 4, cudaMemcpyDeviceToHost), "D2H")) return fdtd_last_error();
            off += m->out[l];
        }
    }
    return FDTD_OK;
}

int fdtd_mlp_train_step(void *h, const float *x, const float *t, int batch, float lr, double *loss)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    Mlp *m = net(h);
    if (!batch_ok(m, batch) || !x || !t || !(lr > 0)) return FDTD_ERR_ARG;
    int r = grads_common(m, x, t, batch, loss);
    if (r != FDTD_OK) return r;
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f - std::pow(b1, (float)m->step), c2 = 1.0f - std::pow(b2, (float)m->step);
    for (int l = 0; l < kLayers; l++) {
        note_launch(2);
        k_adam<<<blocks_for(m->wcount(l)), 256, 0, m->st>>>(m->W[l], m->gW[l], m->mW[l], m->vW[l], m->wcount(l), lr, b1,
                                                           b2, eps, c1, c2);
        k_adam<<<blocks_for(m->out[l]), 256, 0, m->st>>>(m->b[l], m->gb[l], m->mb[l], m->vb[l], m->out[l], lr, b1, b2,
                                                        eps, c1, c2);
    }
    if (!refresh_bf16(*m)) return fdtd_last_error();
    return check_err(*m) ? FDTD_OK : fdtd_last_error();
}

int fdtd_mlp_input_gradient(void *h, const float *x, const float *dy, int batch, float *dx)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    Mlp *m = net(h);
    if (!batch_ok(m, batch) || !x || !dy || !dx) return FDTD_ERR_ARG;
    if (!ensure_cap(*m, batch) || !upload(*m, m->xs, x, (size_t)batch * m->nin) ||
        !upload(*m, m->dys, dy, (size_t)batch * m->nout) || !forward(*m, batch))
        return fdtd_last_error();
    const int L = kLayers - 1;
    note_launch();
    k_seed_grad<<<blocks_for((long long)batch * m->outp[L]), 256, 0, m->st>>>(m->dys, batch, m->nout, m->outp[L],
                                                                                m->dZf, m->dZb);
    if (!backward(*m, batch, false, true)) return fdtd_last_error();
    std::vector<float> full((size_t)batch * m->inp[0]);
    if (!cuda_ok(cudaMemcpyAsync(full.data(), m->dX, full.size() * 4, cudaMemcpyDeviceToHost, m->st), "D2H") ||
        !check_err(*m))
        return fdtd_last_error();
    for (int r = 0; r < batch; r++)
        for (int c = 0; c < m->nin; c++) dx[(size_t)r * m->nin + c] = full[(size_t)r * m->inp[0] + c];
    return FDTD_OK;
}

void fdtd_mlp_free(void *h)
{
    std::lock_guard<std::mutex> lock(api_mutex());
    auto &v = nets();
    for (size_t i = 0; i < v.size(); i++)
        if (v[i] == h) {
            delete v[i];
            v.erase(v.begin() + i);
            return;
        }
}

}  // extern "C"
