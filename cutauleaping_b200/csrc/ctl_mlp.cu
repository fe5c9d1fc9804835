// Surrogate MLP kernels for sm_100a: a tcgen05 GEMM with fused epilogues,
// the Gaussian negative-log-likelihood gradient, bias gradients and Adam.
//
// The surrogate (fitness mode, aresio/cuTauLeaping kernel.cu:365-423 computes
// fitness by full simulation; this build screens candidates first) maps
// (8 log rate constants, t) to per-species mean and log-variance:
//   9 -> 256 -> 256 -> 256 -> 256 -> 2*S_out, SiLU, BF16 weights, FP32 accumulate.
//
// GEMM: C[M][N] = A[M][K] . B[N][K]^T, A and B BF16 row-major with K
// contiguous ("K-major").  One CTA of 128 threads computes a 128 x BN tile
// (BN = N <= 256): all threads stage 128x64 / BNx64 tiles of A and B in the
// canonical no-swizzle K-major shared-memory layout (8-row x 16-byte core
// matrices), one elected thread issues tcgen05.mma (M = 128, N = BN, K = 16)
// into a TMEM accumulator and tcgen05.commit signals a per-stage mbarrier;
// two stages overlap the next tile's loads with the current MMAs.  The
// epilogue reads TMEM with tcgen05.ld (warp w owns lanes 32w..32w+31 = rows).
// Split-K over grid.z serves the weight gradients (K = batch).
// Every mbarrier wait is bounded: on timeout the kernel raises an error flag
// instead of hanging.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "ctl_internal.h"

namespace ctl {
namespace mlp {

constexpr int BM = 128, BK = 64, THREADS = 128;
constexpr uint32_t WAIT_LIMIT = 1u << 24;

struct Gemm {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    int lda, ldb, M, N, K, kt_per_split, epi;
    const float* bias;          // [N]
    const float* z_in;          // [M][ldz] pre-activations (SiLU gradient)
    int ldz;
    float* out_f32;             // [M][ldo]
    int ldo;
    __nv_bfloat16* out_bf;      // [M][ldob]
    int ldob;
    __nv_bfloat16* out_bfT;     // [N][ldobT]
    int ldobT;
    unsigned* err;
};

// ---- PTX helpers ------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: returns false (and raises *err) after WAIT_LIMIT polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned* err) {
    for (uint32_t i = 0; i < WAIT_LIMIT; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i > 32) __nanosleep(64);
    }
    if (err) atomicOr(err, 1u);
    return false;
}

__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor, K-major, no swizzle: start address,
// leading byte offset (between the two 8-element K chunks of one MMA) and
// stride byte offset (between 8-row groups), all >> 4; version 1 (sm_100).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;  // descriptor version for tcgen05
    return d;                 // base offset 0, absolute-LBO off, swizzle none (bits 61-63 = 0)
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, K-major A and B.
__device__ __forceinline__ uint32_t make_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// ---- the GEMM -----------------------------------------------------------------

enum { EPI_ATOMIC_F32 = 0, EPI_BIAS_SILU = 1, EPI_BIAS = 2, EPI_SILU_GRAD = 3, EPI_F32 = 4 };

// Copy a ROWS x 64 BF16 tile (rows r0.., columns k0..k0+63) into the
// canonical layout: chunk (row, kb) of 8 elements at (kb*ROWS/8 + row/8)*128
// + (row%8)*16 bytes.  Consecutive threads take consecutive rows.
__device__ __forceinline__ void stage_tile(uint8_t* dst, const __nv_bfloat16* src, int ld, int r0,
                                           int k0, int rows) {
    const int chunks = rows * (BK / 8);
    for (int c = (int)threadIdx.x; c < chunks; c += THREADS) {
        const int row = c % rows, kb = c / rows;
        const uint4 v = *reinterpret_cast<const uint4*>(src + (size_t)(r0 + row) * ld + k0 + kb * 8);
        *reinterpret_cast<uint4*>(dst + (size_t)(kb * (rows / 8) + row / 8) * 128 + (row % 8) * 16) = v;
    }
}

__global__ void __launch_bounds__(THREADS, 1) gemm_kernel(Gemm p) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_slot;
    const int BN = p.N < 256 ? p.N : 256;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int ktiles = p.K / BK;
    const int kt0 = blockIdx.z * p.kt_per_split;
    const int kt1 = min(kt0 + p.kt_per_split, ktiles);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    uint8_t* sA[2] = {smem, smem + BM * BK * 2};
    uint8_t* sB[2] = {smem + 2 * BM * BK * 2, smem + 2 * BM * BK * 2 + BN * BK * 2};
    uint32_t ncols = 32;
    while ((int)ncols < BN) ncols <<= 1;

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_slot)), "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = make_idesc(BM, BN);
    uint32_t par[2] = {0u, 0u};
    bool ok = true;
    int last = -1;
    for (int kt = kt0; kt < kt1 && ok; kt++) {
        const int i = kt - kt0, s = i & 1;
        if (i >= 2) {  // the MMAs that read this stage two tiles ago are done
            ok = mbar_wait(&bars[s], par[s], p.err);
            par[s] ^= 1u;
            ok = __syncthreads_and(ok) != 0;  // uniform: the loop holds block barriers
            if (!ok) break;
        }
        stage_tile(sA[s], p.A, p.lda, m0, kt * BK, BM);
        stage_tile(sB[s], p.B, p.ldb, n0, kt * BK, BN);
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a = smem_u32(sA[s]), b = smem_u32(sB[s]);
#pragma unroll
            for (int kk = 0; kk < BK / 16; kk++) {
                // K chunk 2kk starts (2kk)*(rows/8)*128 bytes into the tile
                const uint64_t da = make_desc(a + kk * 2 * (BM / 8) * 128, (BM / 8) * 128, 128);
                const uint64_t db = make_desc(b + kk * 2 * (BN / 8) * 128, (BN / 8) * 128, 128);
                mma_bf16(tmem, da, db, idesc, (i > 0 || kk > 0) ? 1u : 0u);
            }
            mma_commit(&bars[s]);
        }
        last = s;
    }
    if (last >= 0 && ok) ok = mbar_wait(&bars[last], par[last], p.err);
    ok = __syncthreads_and(ok) != 0;  // tcgen05.ld below is warp-collective
    tc_fence_after();
    if (last >= 0 && ok) {
        const int row = m0 + warp * 32 + lane;
        for (int c = 0; c < BN; c += 8) {
            float v[8];
            tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
            const int n = n0 + c;
            if (p.epi == EPI_ATOMIC_F32) {
#pragma unroll
                for (int j = 0; j < 8; j++) atomicAdd(p.out_f32 + (size_t)row * p.ldo + n + j, v[j]);
            } else if (p.epi == EPI_F32) {
#pragma unroll
                for (int j = 0; j < 8; j++) p.out_f32[(size_t)row * p.ldo + n + j] = v[j];
            } else if (p.epi == EPI_BIAS) {
#pragma unroll
                for (int j = 0; j < 8; j++) p.out_f32[(size_t)row * p.ldo + n + j] = v[j] + p.bias[n + j];
            } else if (p.epi == EPI_BIAS_SILU) {
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const float z = v[j] + p.bias[n + j];
                    p.out_f32[(size_t)row * p.ldo + n + j] = z;
                    const __nv_bfloat16 h = __float2bfloat16(silu(z));
                    p.out_bf[(size_t)row * p.ldob + n + j] = h;
                    if (p.out_bfT) p.out_bfT[(size_t)(n + j) * p.ldobT + row] = h;
                }
            } else {  // EPI_SILU_GRAD
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const float z = p.z_in[(size_t)row * p.ldz + n + j];
                    const __nv_bfloat16 d = __float2bfloat16(v[j] * silu_grad(z));
                    p.out_bf[(size_t)row * p.ldob + n + j] = d;
                    if (p.out_bfT) p.out_bfT[(size_t)(n + j) * p.ldobT + row] = d;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// ---- small kernels ------------------------------------------------------------------

// Gaussian NLL per element: 0.5 (lv + (y - mu)^2 exp(-lv)), outputs
// y = [mu | lv | padding] (row stride ldy), targets tgt [B][S].  Writes dY
// (BF16, row stride ldd; padding columns untouched) and its transpose
// ([.][ldT], rows 0..2S-1), scaled by 1/(B*S), and accumulates the loss sum.
__global__ void nll_grad_kernel(const float* __restrict__ y, int ldy, const float* __restrict__ tgt, int B,
                                int S, __nv_bfloat16* __restrict__ dy, int ldd, __nv_bfloat16* __restrict__ dyT,
                                int ldT, float* __restrict__ loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < B * S) {
        const int b = i / S, s = i % S;
        const float mu = y[(size_t)b * ldy + s];
        float lv = y[(size_t)b * ldy + S + s];
        lv = fminf(fmaxf(lv, -12.0f), 12.0f);
        const float iv = __expf(-lv);
        const float d = tgt[(size_t)b * S + s] - mu;
        l = 0.5f * (lv + d * d * iv);
        const float sc = 1.0f / ((float)B * (float)S);
        const float gmu = -d * iv * sc;
        const float glv = 0.5f * (1.0f - d * d * iv) * sc;
        const __nv_bfloat16 a = __float2bfloat16(gmu), c = __float2bfloat16(glv);
        dy[(size_t)b * ldd + s] = a;
        dy[(size_t)b * ldd + S + s] = c;
        dyT[(size_t)s * ldT + b] = a;
        dyT[(size_t)(S + s) * ldT + b] = c;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l);
}

// Column sums of a BF16 [B][N] matrix into FP32 g[N] (bias gradients).
__global__ void colsum_kernel(const __nv_bfloat16* __restrict__ d, int B, int N, int ld, float* __restrict__ g) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int rows = (B + gridDim.y - 1) / gridDim.y;
    const int b0 = blockIdx.y * rows, b1 = min(B, b0 + rows);
    float acc = 0.0f;
    for (int b = b0; b < b1; b++) acc += __bfloat162float(d[(size_t)b * ld + n]);
    atomicAdd(g + n, acc);
}

// Adam on FP32 master weights; refreshes the BF16 copy W [rows][cols] and its
// transpose WT [cols][rows] used by the backward GEMMs.
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, int n, int rows, int cols, float lr, float b1, float b2,
                            float eps, float c1, float c2, float wd, __nv_bfloat16* __restrict__ wb,
                            __nv_bfloat16* __restrict__ wbT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] + wd * w[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float wi = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    w[i] = wi;
    if (wb) {
        const __nv_bfloat16 h = __float2bfloat16(wi);
        wb[i] = h;
        if (wbT) {
            const int r = i / cols, c = i % cols;
            wbT[(size_t)c * rows + r] = h;
        }
    }
}

}  // namespace mlp
}  // namespace ctl

using namespace ctl;

static ctl_status mlp_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CTL_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return CTL_ERR_CUDA;
}

extern "C" ctl_status ctl_mlp_gemm(const ctl_gemm_desc* d, void* stream) {
    if (!d || !d->A || !d->B) return CTL_ERR_ARG;
    if (d->M % 128 || d->K % 64 || d->N % 16 || d->N <= 0 || (d->N > 256 && d->N % 256)) {
        set_error("ctl_mlp_gemm: M % 128, K % 64, N % 16 (and N % 256 above 256) must be 0");
        return CTL_ERR_SHAPE;
    }
    if (d->lda % 8 || d->ldb % 8) {
        set_error("ctl_mlp_gemm: leading dimensions must be multiples of 8 elements");
        return CTL_ERR_SHAPE;
    }
    mlp::Gemm p;
    p.A = static_cast<const __nv_bfloat16*>(d->A);
    p.B = static_cast<const __nv_bfloat16*>(d->B);
    p.lda = d->lda; p.ldb = d->ldb; p.M = d->M; p.N = d->N; p.K = d->K;
    p.epi = d->epilogue;
    p.bias = d->bias; p.z_in = d->z_in; p.ldz = d->ldz;
    p.out_f32 = d->out_f32; p.ldo = d->ldo;
    p.out_bf = static_cast<__nv_bfloat16*>(d->out_bf); p.ldob = d->ldob;
    p.out_bfT = static_cast<__nv_bfloat16*>(d->out_bfT); p.ldobT = d->ldobT;
    p.err = d->err;
    const int ktiles = d->K / 64;
    const int splits = d->splits > 0 ? (d->splits < ktiles ? d->splits : ktiles) : 1;
    p.kt_per_split = (ktiles + splits - 1) / splits;
    const int BN = d->N < 256 ? d->N : 256;
    const size_t smem = (size_t)2 * mlp::BM * mlp::BK * 2 + (size_t)2 * BN * mlp::BK * 2;
    static bool attr_set = false;
    if (!attr_set) {
        ctl_status st = mlp_cuda(cudaFuncSetAttribute(mlp::gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      2 * mlp::BM * mlp::BK * 2 + 2 * 256 * mlp::BK * 2),
                                 "cudaFuncSetAttribute(gemm)");
        if (st != CTL_OK) return st;
        attr_set = true;
    }
    dim3 grid((unsigned)(d->M / 128), (unsigned)((d->N + BN - 1) / BN), (unsigned)splits);
    mlp::gemm_kernel<<<grid, mlp::THREADS, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return mlp_cuda(cudaGetLastError(), "gemm_kernel launch");
}

extern "C" ctl_status ctl_mlp_nll_grad(const float* y, int32_t ldy, const float* tgt, int32_t B, int32_t S,
                                       void* dy, int32_t ldd, void* dyT, int32_t ldT, float* loss, void* stream) {
    if (!y || !tgt || !dy || !dyT || !loss || B <= 0 || S <= 0 || 2 * S > 128 || ldT < B || ldy < 2 * S ||
        ldd < 2 * S)
        return CTL_ERR_ARG;
    const int n = B * S;
    mlp::nll_grad_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        y, ldy, tgt, B, S, static_cast<__nv_bfloat16*>(dy), ldd, static_cast<__nv_bfloat16*>(dyT), ldT, loss);
    return mlp_cuda(cudaGetLastError(), "nll_grad_kernel launch");
}

extern "C" ctl_status ctl_mlp_colsum(const void* d, int32_t B, int32_t N, int32_t ld, float* g, void* stream) {
    if (!d || !g || B <= 0 || N <= 0) return CTL_ERR_ARG;
    dim3 grid((unsigned)((N + 127) / 128), (unsigned)(B > 64 * 1024 ? 128 : (B + 511) / 512));
    mlp::colsum_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(d), B, N, ld, g);
    return mlp_cuda(cudaGetLastError(), "colsum_kernel launch");
}

extern "C" ctl_status ctl_mlp_adam(float* w, const float* g, float* m1, float* m2, int32_t rows, int32_t cols,
                                   float lr, float beta1, float beta2, float eps, int32_t step, float wd,
                                   void* wb, void* wbT, void* stream) {
    if (!w || !g || !m1 || !m2 || rows <= 0 || cols <= 0 || step <= 0) return CTL_ERR_ARG;
    const int n = rows * cols;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    mlp::adam_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w, g, m1, m2, n, rows, cols, lr, beta1, beta2, eps, c1, c2, wd, static_cast<__nv_bfloat16*>(wb),
        static_cast<__nv_bfloat16*>(wbT));
    return mlp_cuda(cudaGetLastError(), "adam_kernel launch");
}
