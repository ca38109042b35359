// umma_gemm.cu -- BF16 GEMM on the 5th-generation tensor cores (tcgen05), FP32
// accumulation in tensor memory, fused bias / activation epilogue.  Used by
// the surrogate network (surrogate.cu); the FDTD stencil has no contraction.
//
//   pre[m][n] = alpha * sum_k A[m][k] B[n][k] + beta * C32[m][n] + bias[n]
//   Z32 = pre (optional), post = act(pre) (identity or GELU),
//   C32 = post (optional, FP32), C16 = post (optional, BF16)
// A is M x K and B is N x K, both K-major (row stride lda / ldb elements,
// multiples of 8; K a multiple of 8).  Ragged M, N and K are zero-filled.
//
// One CTA (4 warps) owns a 128 x BN tile of C, BN in {32, 64, 128, 256}:
//   warp 0 allocates BN TMEM columns (tcgen05.alloc) for the FP32
//   accumulator (TMEM lane = row of the tile);
//   per K tile of 32: all threads stage A (128 x 32) and B (BN x 32) in shared
//   memory in the canonical K-major layout without swizzle -- 8-row x 16-byte
//   core matrices, the two 8-element K halves of an MMA step 128 B apart
//   (LBO), successive 8-row groups 512 B apart (SBO) -- then, after a
//   generic-to-async proxy fence and a barrier, one thread issues two
//   tcgen05.mma.cta_group::1.kind::f16 (M 128, N BN, K 16 each) and
//   tcgen05.commit to an mbarrier that every thread waits on before the
//   tiles are overwritten;
//   epilogue: each warp reads its 32 TMEM lanes with tcgen05.ld 32x32b.x16.
// Waits are bounded in time; a wait that gives up sets *err, waits (bounded)
// for the MMAs in flight, frees the TMEM and returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "engine.h"

namespace fdtd {

constexpr int kGemmBM = 128, kGemmBK = 32, kGemmThreads = 128;
constexpr unsigned kGemmSBO = (kGemmBK / 8) * 128;   // bytes between 8-row groups
constexpr unsigned kGemmLBO = 128;                   // bytes between the two K halves of a step
constexpr unsigned long long kGemmWaitNs = 1000000000ull;

__device__ __forceinline__ unsigned su32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtime()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_test(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(su32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_for(unsigned long long *bar, unsigned parity, unsigned long long ns)
{
    const unsigned long long t0 = gtime();
    for (;;) {
        if (mbar_test(bar, parity)) return true;
        if (gtime() - t0 > ns) return false;
    }
}

// K-major, no swizzle, version 1 (Blackwell) shared-memory matrix descriptor
__device__ __forceinline__ unsigned long long umma_desc(unsigned saddr)
{
    return (unsigned long long)((saddr >> 4) & 0x3FFFu) | ((unsigned long long)((kGemmLBO >> 4) & 0x3FFFu) << 16) |
           ((unsigned long long)((kGemmSBO >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D F32, A and B BF16, both K-major, M 128, N bn
__host__ __device__ constexpr unsigned umma_idesc(int bn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(bn >> 3) << 17) | ((unsigned)(kGemmBM >> 4) << 24);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

template <int BN>
__global__ void __launch_bounds__(kGemmThreads) k_umma_gemm(GemmArgs g)
{
    __shared__ __align__(1024) unsigned char sA[kGemmBM * kGemmBK * 2];
    __shared__ __align__(1024) unsigned char sB[BN * kGemmBK * 2];
    __shared__ __align__(8) unsigned long long bar;
    __shared__ unsigned tmem_base;
    __shared__ int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * BN;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base)),
                     "r"((unsigned)BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&bar)));
        abort_flag = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const unsigned tmem = tmem_base;
    const int ktiles = (g.K + kGemmBK - 1) / kGemmBK;
    unsigned phase = 0;
    int issued = 0;   // commits not yet waited for
    for (int kt = 0; kt < ktiles; kt++) {
        const int k0 = kt * kGemmBK;
        // stage A: 128 rows x 4 chunks of 8 elements; B: BN rows x 4 chunks
        for (int q = tid; q < kGemmBM * (kGemmBK / 8); q += kGemmThreads) {
            const int r = q / (kGemmBK / 8), c = q % (kGemmBK / 8);
            const int gm = m0 + r, gk = k0 + 8 * c;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gm < g.M && gk < g.K) v = *reinterpret_cast<const uint4 *>(g.A + (long long)gm * g.lda + gk);
            *reinterpret_cast<uint4 *>(sA + (r >> 3) * kGemmSBO + c * 128 + (r & 7) * 16) = v;
        }
        for (int q = tid; q < BN * (kGemmBK / 8); q += kGemmThreads) {
            const int r = q / (kGemmBK / 8), c = q % (kGemmBK / 8);
            const int gn = n0 + r, gk = k0 + 8 * c;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gn < g.N && gk < g.K) v = *reinterpret_cast<const uint4 *>(g.B + (long long)gn * g.ldb + gk);
            *reinterpret_cast<uint4 *>(sB + (r >> 3) * kGemmSBO + c * 128 + (r & 7) * 16) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int s = 0; s < kGemmBK / 16; s++) {
                const unsigned long long da = umma_desc(su32(sA) + s * 256), db = umma_desc(su32(sB) + s * 256);
                const unsigned acc = (kt > 0 || s > 0) ? 1u : 0u;
                asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                             " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                             "l"(da), "l"(db), "r"(umma_idesc(BN)), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(&bar))
                         : "memory");
        }
        issued = 1;
        if (!mbar_wait_for(&bar, phase, kGemmWaitNs)) abort_flag = 1;
        __syncthreads();
        if (abort_flag) break;
        issued = 0;
        phase ^= 1u;
    }
    if (abort_flag) {
        if (tid == 0) atomicExch(g.err, 1);
        if (issued) mbar_wait_for(&bar, phase, kGemmWaitNs);   // MMAs still in flight
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;");
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int cc = 0; cc < BN / 16; cc++) {
            unsigned r[16];
            const unsigned taddr = tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(cc * 16);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                           "=r"(r[14]), "=r"(r[15])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row >= g.M) continue;
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int col = n0 + cc * 16 + i;
                if (col >= g.N) continue;
                float v = g.alpha * __uint_as_float(r[i]);
                if (g.beta != 0.0f) v += g.beta * g.C32[(long long)row * g.ldc32 + col];
                if (g.bias) v += g.bias[col];
                if (g.Z32) g.Z32[(long long)row * g.ldz + col] = v;
                if (g.act == 1) v = gelu(v);
                if (g.C32) g.C32[(long long)row * g.ldc32 + col] = v;
                if (g.C16) g.C16[(long long)row * g.ldc16 + col] = __float2bfloat16_rn(v);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((unsigned)BN));
}

bool gemm_bf16_launch(const GemmArgs &a, cudaStream_t st)
{
    if (a.M <= 0 || a.N <= 0 || a.K <= 0) return true;
    if (a.K % 8 || a.lda % 8 || a.ldb % 8 || a.lda < a.K || a.ldb < a.K ||
        ((uintptr_t)a.A & 15) || ((uintptr_t)a.B & 15) || !a.err) {
        set_error(FDTD_ERR_ARG, "gemm: K %d, lda %d, ldb %d must be multiples of 8 (>= K), operands 16-byte aligned",
                  a.K, a.lda, a.ldb);
        return false;
    }
    const int bn = a.N <= 32 ? 32 : a.N <= 64 ? 64 : a.N <= 128 ? 128 : 256;
    dim3 grid((a.M + kGemmBM - 1) / kGemmBM, (a.N + bn - 1) / bn);
    note_launch();
    switch (bn) {
    case 32: k_umma_gemm<32><<<grid, kGemmThreads, 0, st>>>(a); break;
    case 64: k_umma_gemm<64><<<grid, kGemmThreads, 0, st>>>(a); break;
    case 128: k_umma_gemm<128><<<grid, kGemmThreads, 0, st>>>(a); break;
    default: k_umma_gemm<256><<<grid, kGemmThreads, 0, st>>>(a); break;
    }
    return cuda_ok(cudaGetLastError(), "gemm launch");
}

}  // namespace fdtd

using namespace fdtd;

extern "C" int fdtd_gemm_bf16(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const float *bias,
                              int act, float alpha, float beta, float *C32, int ldc32, void *C16, int ldc16,
                              float *Z32, int ldz, int *err, void *stream)
{
    if (!device_available()) return fdtd_last_error();
    if ((beta != 0.0f && !C32) || act < 0 || act > 1) {
        set_error(FDTD_ERR_ARG, "fdtd_gemm_bf16: beta needs C32; act must be 0 or 1");
        return FDTD_ERR_ARG;
    }
    GemmArgs a{(const __nv_bfloat16 *)A, (const __nv_bfloat16 *)B, lda, ldb, M, N, K, bias, act, alpha, beta,
               C32, ldc32, (__nv_bfloat16 *)C16, ldc16, Z32, ldz, err};
    return gemm_bf16_launch(a, (cudaStream_t)stream) ? FDTD_OK : fdtd_last_error();
}
