// Surrogate MLP: BF16 operands, FP32 accumulation on the 5th-generation tensor cores.
//
// Every layer product is one tile GEMM C[M, N] = A[M, K] . B[N, K]^T (both operands K-major):
// a CTA of four warps owns a 128-row tile, stages 64-wide K slices of A and B in shared memory in
// the canonical no-swizzle K-major layout (8x16-byte core matrices), one thread issues
// tcgen05.mma (kind::f16, BF16 in, FP32 accumulate) into a tensor-memory accumulator, and
// tcgen05.commit arrives on an mbarrier that frees the stage. The epilogue reads the accumulator
// with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31) and fuses bias, GELU or the GELU
// derivative, and writes FP32, BF16 and transposed BF16 copies (the transposed copies are the
// K-major operands of the weight-gradient products). Weight gradients use split-K with a
// fixed-order reduction, so every result is deterministic. Adam keeps FP32 master weights and
// refreshes the BF16 copies in the same pass.
//
// Every wait is bounded (about one second of global time): a CTA that gives up records an error
// flag, still waits (bounded) for its own tensor-core work, frees its tensor memory and returns.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <new>
#include <vector>

#include "../../include/vp_b200.h"
#include "vp_internal.h"

namespace vpb {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int BM = 128;        // rows per tile (the tcgen05 M)
constexpr int BK = 64;         // K per shared-memory stage
constexpr int NT = 128;        // threads per CTA
constexpr int MAX_LAYERS = 8;

struct GemmArgs {
    const bf16* A;
    long long lda;           // A[m, k] at A[m * lda + k]
    const bf16* B;
    long long ldb;           // B[n, k] at B[n * ldb + k]
    int M, N, K;             // K, lda, ldb multiples of 8; A and B 16-byte aligned
    int k_per_split;         // multiple of BK; CTA z covers [z * k_per_split, ...)
    const float* bias;       // [N] or null
    int act;                 // 0: y = z; 1: y = gelu(z); 2: y = z * gelu'(aux)
    const float* aux;
    long long ldaux;
    float* C32;              // y (FP32); with split-K the raw partial of split z at C32 + z * split_stride
    long long ldc32;
    long long split_stride;
    float* Zout;             // z (act 1)
    long long ldz;
    bf16* C16;               // y (BF16), columns [N, pad8(N)) written as zero
    long long ldc16;
    bf16* C16T;              // y^T (BF16), rows n, columns [M, pad8(M)) written as zero
    long long ldc16t;
    unsigned* err;
    unsigned long long wait_ns;   // limit of each bounded tensor-core wait (0: one poll)
};

__host__ __device__ constexpr int pad8(int x) { return (x + 7) & ~7; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle: start address, leading-dimension byte offset
// (between the two 8-element K groups of one MMA), stride byte offset (between 8-row groups),
// descriptor version 1 at bits 46-47, base offset 0, layout type 0.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B (bits 7-9
// and 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
template <int BN>
__device__ __forceinline__ uint32_t idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Non-blocking test of the phase (try_wait may suspend the thread for a hardware-defined time).
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the phase of the given parity: gives up after limit_ns nanoseconds (checked
// every 256 polls, and after at most 2^24 polls); limit_ns == 0 gives up at the first poll that
// does not find the phase complete (a non-blocking test).
__device__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned long long limit_ns) {
    if (limit_ns == 0) return mbar_test_wait(bar, parity);
    const uint64_t t0 = global_ns();
    for (unsigned it = 0; it < (1u << 24); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 255u && global_ns() - t0 > limit_ns) return false;
    }
    return false;
}

// Limit of the wait that drains a CTA's own tensor-core work before it frees its tensor memory
// (used whatever the host-set limit is, so that a CTA that gave up never frees columns that an
// MMA in flight still writes).
constexpr unsigned long long kDrainWaitNs = 1000000000ull;
// Default limit of the waits that detect a stalled tensor-core pipeline.
constexpr unsigned long long kDefaultWaitNs = 1000000000ull;

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 lanes x 16 consecutive FP32 columns: thread l of the warp gets lane (base lane + l).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// One K slice of `rows` rows into the canonical layout: element (r, k) at
// (r / 8) * 1024 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2 bytes. Eight consecutive threads
// fill the eight rows of one core matrix (conflict-free 128-byte shared stores).
template <int ROWS>
__device__ __forceinline__ void load_slice(unsigned char* dst, const bf16* src, long long ld, int r0, int rmax,
                                           int k0, int k_end) {
    for (int idx = threadIdx.x; idx < ROWS * 8; idx += NT) {
        const int r = (idx & 7) + ((idx >> 6) << 3);
        const int kg = (idx >> 3) & 7;
        const int gr = r0 + r, gk = k0 + kg * 8;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (gr < rmax && gk < k_end) v = __ldg(reinterpret_cast<const uint4*>(src + (long long)gr * ld + gk));
        *reinterpret_cast<uint4*>(dst + (r >> 3) * 1024 + kg * 128 + (r & 7) * 16) = v;
    }
}

template <int BN>
constexpr size_t gemm_smem_bytes() {
    return (size_t)2 * (BM + BN) * BK * 2 + 1024;   // two stages plus alignment slack
}

template <int BN>
__global__ void __launch_bounds__(NT) vp_mlp_gemm_kernel(const GemmArgs g) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_base_s;
    constexpr int A_BYTES = BM * BK * 2, STAGE = (BM + BN) * BK * 2;
    unsigned char* sm = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int k_begin = blockIdx.z * g.k_per_split;
    const int k_end = min(g.K, k_begin + g.k_per_split);
    const int nk = (k_end - k_begin + BK - 1) / BK;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        tmem_alloc(&tmem_base_s, BN);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    const uint32_t idesc = idesc_bf16<BN>();
    bool ok = true;
    int issued = -1;
    for (int kc = 0; kc < nk; ++kc) {
        const int s = kc & 1;
        if (kc >= 2) {
            const bool w = mbar_wait(&bars[s], ((kc - 2) >> 1) & 1, g.wait_ns);
            if (!__syncthreads_and(w)) {
                ok = false;
                break;
            }
        }
        unsigned char* sA = sm + s * STAGE;
        unsigned char* sB = sA + A_BYTES;
        const int k0 = k_begin + kc * BK;
        load_slice<BM>(sA, g.A, g.lda, m0, g.M, k0, k_end);
        load_slice<BN>(sB, g.B, g.ldb, n0, g.N, k0, k_end);
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
                umma_bf16(tmem, umma_desc(a0 + kk * 256, 128, 1024), umma_desc(b0 + kk * 256, 128, 1024), idesc,
                          (kc | kk) != 0 ? 1u : 0u);
            }
            umma_commit(&bars[s]);
        }
        issued = kc;
    }
    if (issued >= 0) {
        const bool w = mbar_wait(&bars[issued & 1], (issued >> 1) & 1, g.wait_ns);
        ok = __syncthreads_and(ok && w);
        if (!ok) {
            // the commit of the last issued slice completes after every MMA this CTA issued
            const bool d = mbar_wait(&bars[issued & 1], (issued >> 1) & 1, kDrainWaitNs);
            __syncthreads_and(d);
        }
    }
    if (ok && issued >= 0) {
        tc_fence_after();
        const int m = m0 + warp * 32 + lane;
        const int Mp = pad8(g.M), Np = pad8(g.N);
        const bool split = gridDim.z > 1;
        for (int c0 = 0; c0 < BN; c0 += 16) {
            if (n0 + c0 >= Np) break;   // warp-uniform
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int n = n0 + c0 + j;
                if (n >= Np) continue;
                const bool valid = (m < g.M) && (n < g.N);
                if (split) {
                    if (valid) g.C32[blockIdx.z * g.split_stride + (long long)m * g.ldc32 + n] = v[j];
                    continue;
                }
                float y = 0.f;
                if (valid) {
                    float z = v[j] + (g.bias ? __ldg(g.bias + n) : 0.f);
                    if (g.act == 1) {
                        if (g.Zout) g.Zout[(long long)m * g.ldz + n] = z;
                        y = gelu(z);
                    } else if (g.act == 2) {
                        y = z * gelu_grad(__ldg(g.aux + (long long)m * g.ldaux + n));
                    } else {
                        y = z;
                    }
                    if (g.C32) g.C32[(long long)m * g.ldc32 + n] = y;
                }
                if (g.C16 && m < g.M) g.C16[(long long)m * g.ldc16 + n] = __float2bfloat16_rn(y);
                if (g.C16T && m < Mp && n < g.N) g.C16T[(long long)n * g.ldc16t + m] = __float2bfloat16_rn(y);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, BN);
    }
    if (!ok && tid == 0 && g.err) atomicOr(g.err, 1u);
}

// ---------------------------------------------------------------------------------------------
// elementwise and reduction kernels
// ---------------------------------------------------------------------------------------------

// FP32 rows (optionally gathered through `rows`) to BF16 [M, pad8(K)] and BF16^T [K, pad8(M)]
// (pads zero); also an FP32 copy when requested.
__global__ void vp_mlp_pack_kernel(const float* __restrict__ src, long long ld, const int* __restrict__ rows,
                                   int M, int K, bf16* dst, long long ldd, bf16* dstT, long long ldt,
                                   float* dst32, long long ld32) {
    const int Mp = pad8(M), Kp = pad8(K);
    const long long total = (long long)Mp * Kp;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(i / Kp), k = (int)(i - (long long)m * Kp);
        float x = 0.f;
        if (m < M && k < K) {
            const long long r = rows ? rows[m] : m;
            x = src[r * ld + k];
            if (dst32) dst32[(long long)m * ld32 + k] = x;
        }
        const bf16 b = __float2bfloat16_rn(x);
        if (dst && m < M) dst[(long long)m * ldd + k] = b;
        if (dstT && k < K) dstT[(long long)k * ldt + m] = b;
    }
}

// d = 2 (y - t) / (M N) for the mean-squared error; writes FP32, BF16 and BF16^T copies and one
// partial sum of squared errors per block.
__global__ void vp_mlp_mse_kernel(const float* __restrict__ y, long long ldy, const float* __restrict__ t,
                                  long long ldt, const int* __restrict__ rows, int M, int N, float* d32,
                                  long long ld32, bf16* d16, long long ld16, bf16* d16T, long long ld16t,
                                  float* partial) {
    __shared__ float red[32];
    const int Mp = pad8(M), Np = pad8(N);
    const long long total = (long long)Mp * Np;
    const float scale = 2.0f / ((float)M * (float)N);
    float acc = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(i / Np), n = (int)(i - (long long)m * Np);
        float d = 0.f;
        if (m < M && n < N) {
            const long long r = rows ? rows[m] : m;
            const float e = y[(long long)m * ldy + n] - t[r * ldt + n];
            acc += e * e;
            d = scale * e;
            d32[(long long)m * ld32 + n] = d;
        }
        const bf16 b = __float2bfloat16_rn(d);
        if (m < M) d16[(long long)m * ld16 + n] = b;
        if (n < N) d16T[(long long)n * ld16t + m] = b;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        partial[blockIdx.x] = s;
    }
}

// loss = sum(partial[0..n)) / count, fixed order.
__global__ void vp_mlp_loss_kernel(const float* __restrict__ partial, int n, float inv_count, float* loss) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        float s = 0.f;
        for (int i = 0; i < n; ++i) s += partial[i];
        *loss = s * inv_count;
    }
}

// out[n] = sum_m src[m * ld + n], m < M, fixed order (blockDim 32 x 8).
__global__ void vp_mlp_colsum_kernel(const float* __restrict__ src, long long ld, int M, int N, float* out) {
    __shared__ float red[8][33];
    const int n = blockIdx.x * 32 + threadIdx.x;
    float s = 0.f;
    if (n < N)
        for (int m = threadIdx.y; m < M; m += 8) s += src[(long long)m * ld + n];
    red[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && n < N) {
        float t = 0.f;
        for (int k = 0; k < 8; ++k) t += red[k][threadIdx.x];
        out[n] = t;
    }
}

// out[m * ldo + n] = sum_z part[z * stride + m * ldp + n], fixed order.
__global__ void vp_mlp_splitk_reduce_kernel(const float* __restrict__ part, long long stride, long long ldp,
                                            int splits, int M, int N, float* out, long long ldo) {
    const long long total = (long long)M * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(i / N), n = (int)(i - (long long)m * N);
        float s = 0.f;
        for (int z = 0; z < splits; ++z) s += part[z * stride + (long long)m * ldp + n];
        out[(long long)m * ldo + n] = s;
    }
}

struct LayerRefs {
    long long off_W[MAX_LAYERS], off_b[MAX_LAYERS];
    int n_out[MAX_LAYERS], n_in[MAX_LAYERS];
    bf16* Wb[MAX_LAYERS];
    bf16* WbT[MAX_LAYERS];
    int L;
};

// BF16 copies of the weights: Wb[l][n * pad8(K) + k], WbT[l][k * pad8(N) + n].
__device__ __forceinline__ void refresh_copy(const LayerRefs& R, long long i, float w) {
    for (int l = 0; l < R.L; ++l) {
        const long long rel = i - R.off_W[l];
        if (rel >= 0 && rel < (long long)R.n_out[l] * R.n_in[l]) {
            const int n = (int)(rel / R.n_in[l]), k = (int)(rel - (long long)n * R.n_in[l]);
            const bf16 b = __float2bfloat16_rn(w);
            R.Wb[l][(long long)n * pad8(R.n_in[l]) + k] = b;
            R.WbT[l][(long long)k * pad8(R.n_out[l]) + n] = b;
            return;
        }
    }
}

__global__ void vp_mlp_refresh_kernel(const float* __restrict__ p, long long n, const LayerRefs R) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        refresh_copy(R, i, p[i]);
}

// Adam (Kingma & Ba): m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2;
// p -= lr * (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps), t = *step + 1.
__global__ void vp_mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                   float* __restrict__ v, long long n, const int* __restrict__ step, float lr,
                                   float b1, float b2, float eps, const LayerRefs R) {
    const int t = *step + 1;
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float w = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = w;
        refresh_copy(R, i, w);
    }
}

__global__ void vp_mlp_step_kernel(int* step) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *step += 1;
}

// ---------------------------------------------------------------------------------------------
// Surrogate search: Adam on one input vector c minimising J(c) = sum_n w_n exp(mu_n + sd_n y_n),
// y = net(c * x_scale), for `iters` steps in one single-CTA launch. The network's products are
// warp GEMVs on the same BF16 weights (Wb for the forward, WbT for the backward) with the
// activations and cotangents rounded to BF16 where the tensor-core path rounds them, FP32
// accumulation, the same GELU; the best iterate (smallest J evaluated) is returned.
// ---------------------------------------------------------------------------------------------
constexpr int kSearchMaxWidth = 512;

struct SearchArgs {
    LayerRefs R;
    const float* params;   // FP32 master parameters (biases)
    int w[MAX_LAYERS + 1];
    const float* c0;
    int iters;
    float lr, b1, b2, eps, x_scale;
    const float* y_mean;
    const float* y_std;
    const float* wt;
    float* best_c;
    float* best_J;
};

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// out[r] = sum_k M[r * ld + k] * in[k] for r < rows (warp per row, lanes over k, fixed order).
__device__ __forceinline__ void warp_gemv(const bf16* __restrict__ M, int ld, int rows, int cols,
                                          const float* __restrict__ in, float* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r = warp; r < rows; r += nw) {
        const bf16* row = M + (size_t)r * ld;
        float acc = 0.f;
        for (int k = lane; k < cols; k += 32) acc = fmaf(__bfloat162float(row[k]), in[k], acc);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) out[r] = acc;
    }
}

__global__ void __launch_bounds__(1024) vp_mlp_search_kernel(const SearchArgs A) {
    __shared__ float act[MAX_LAYERS + 1][kSearchMaxWidth];   // layer inputs (BF16-rounded)
    __shared__ float pre[MAX_LAYERS][kSearchMaxWidth];       // pre-activations z_l
    __shared__ float g[2][kSearchMaxWidth];                  // cotangents (ping-pong)
    __shared__ float c[kSearchMaxWidth], mo[kSearchMaxWidth], ve[kSearchMaxWidth];
    __shared__ float red[32];
    __shared__ float sJ, sBest;
    const int L = A.R.L, n_in = A.w[0], n_out = A.w[L];
    const int tid = threadIdx.x;
    for (int k = tid; k < n_in; k += blockDim.x) {
        c[k] = A.c0[k];
        mo[k] = 0.f;
        ve[k] = 0.f;
        A.best_c[k] = A.c0[k];
    }
    if (tid == 0) sBest = INFINITY;
    __syncthreads();
    for (int it = 1; it <= A.iters; ++it) {
        // forward
        for (int k = tid; k < n_in; k += blockDim.x) act[0][k] = bf16r(c[k] * A.x_scale);
        __syncthreads();
        for (int l = 0; l < L; ++l) {
            const int K = A.w[l], N = A.w[l + 1];
            warp_gemv(A.R.Wb[l], pad8(K), N, K, act[l], pre[l]);
            __syncthreads();
            const float* b = A.params + A.R.off_b[l];
            for (int r = tid; r < N; r += blockDim.x) {
                const float z = pre[l][r] + b[r];
                pre[l][r] = z;
                if (l < L - 1) act[l + 1][r] = bf16r(gelu(z));
            }
            __syncthreads();
        }
        // J and the output cotangent
        float part = 0.f;
        for (int r = tid; r < n_out; r += blockDim.x) {
            const float e = A.wt[r] * expf(A.y_mean[r] + A.y_std[r] * pre[L - 1][r]);
            part += e;
            g[0][r] = bf16r(e * A.y_std[r]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if ((tid & 31) == 0) red[tid >> 5] = part;
        __syncthreads();
        if (tid == 0) {
            float J = 0.f;
            for (int q = 0; q < (int)(blockDim.x >> 5); ++q) J += red[q];
            sJ = J;
        }
        __syncthreads();
        if (sJ < sBest) {   // uniform: every thread reads the same shared values
            for (int k = tid; k < n_in; k += blockDim.x) A.best_c[k] = c[k];
            __syncthreads();
            if (tid == 0) sBest = sJ;
        }
        // backward to the input
        int cur = 0;
        for (int l = L - 1; l >= 0; --l) {
            const int K = A.w[l], N = A.w[l + 1];
            warp_gemv(A.R.WbT[l], pad8(N), K, N, g[cur], g[cur ^ 1]);
            __syncthreads();
            if (l > 0)
                for (int k = tid; k < K; k += blockDim.x) g[cur ^ 1][k] = bf16r(g[cur ^ 1][k] * gelu_grad(pre[l - 1][k]));
            __syncthreads();
            cur ^= 1;
        }
        // Adam on c (gradient = x_scale * dJ/dx)
        const float c1 = 1.0f - powf(A.b1, (float)it), c2 = 1.0f - powf(A.b2, (float)it);
        for (int k = tid; k < n_in; k += blockDim.x) {
            const float gk = g[cur][k] * A.x_scale;
            const float m = A.b1 * mo[k] + (1.0f - A.b1) * gk;
            const float v = A.b2 * ve[k] + (1.0f - A.b2) * gk * gk;
            mo[k] = m;
            ve[k] = v;
            c[k] -= A.lr * (m / c1) / (sqrtf(v / c2) + A.eps);
        }
        __syncthreads();
    }
    if (tid == 0) *A.best_J = sBest;
}

}  // namespace mlp
}  // namespace vpb

// =============================================================================================
// host side
// =============================================================================================

using namespace vpb;
using namespace vpb::mlp;

struct vp_mlp {
    int L = 0;
    int w[MAX_LAYERS + 1] = {};
    int max_batch = 0;
    int device = 0;
    long long n_params = 0;
    LayerRefs R{};
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    int* step = nullptr;
    // activations, sized for max_batch rows
    bf16 *Xb = nullptr, *XbT = nullptr;
    float* Z[MAX_LAYERS] = {};
    bf16* Ab[MAX_LAYERS] = {};
    bf16* AbT[MAX_LAYERS] = {};
    float* Y = nullptr;
    float* D32[MAX_LAYERS] = {};   // cotangent on the pre-activation of layer l (FP32)
    bf16* Db[MAX_LAYERS] = {};
    bf16* DbT[MAX_LAYERS] = {};
    float* splitk = nullptr;
    size_t splitk_floats = 0;
    float* partial = nullptr;
    int n_partial = 0;
    unsigned* err = nullptr;
    unsigned long long wait_ns = kDefaultWaitNs;   // limit of the bounded tensor-core waits
    std::vector<void*> allocs;
    int last_M = 0;
};

namespace {

int mlp_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return VP_OK;
    return set_err(VP_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

#define MLP_CUDA(call, what)                       \
    do {                                           \
        int rc_ = mlp_cuda((call), what);          \
        if (rc_ != VP_OK) return rc_;              \
    } while (0)

template <typename T>
int mlp_alloc(vp_mlp* n, T** p, size_t count) {
    void* q = nullptr;
    MLP_CUDA(cudaMalloc(&q, std::max<size_t>(1, count) * sizeof(T)), "cudaMalloc(mlp)");
    MLP_CUDA(cudaMemset(q, 0, std::max<size_t>(1, count) * sizeof(T)), "cudaMemset(mlp)");
    n->allocs.push_back(q);
    *p = static_cast<T*>(q);
    return VP_OK;
}

void mlp_free(vp_mlp* n) {
    if (!n) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(n->device);
    for (void* p : n->allocs) cudaFree(p);
    cudaSetDevice(prev);
    delete n;
}

template <int BN>
int set_gemm_smem() {
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && done[dev]) return VP_OK;
    MLP_CUDA(cudaFuncSetAttribute(vp_mlp_gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)gemm_smem_bytes<BN>()),
             "cudaFuncSetAttribute(mlp gemm)");
    if (dev < 64) done[dev] = true;
    return VP_OK;
}

int gemm_bn(int N) { return N <= 64 ? 64 : 128; }

// C = epilogue(A . B^T). splits > 1 only with act 0, no bias, C32 given.
int launch_gemm(GemmArgs g, int splits, float* splitk_ws, size_t splitk_floats, cudaStream_t s) {
    const int BN = gemm_bn(g.N);
    const int mt = (g.M + BM - 1) / BM, ntile = (g.N + BN - 1) / BN;
    const int nk_total = (g.K + BK - 1) / BK;
    splits = std::max(1, std::min(splits, nk_total));
    float* final_out = g.C32;
    long long final_ld = g.ldc32;
    if (splits > 1) {
        const int chunks = (nk_total + splits - 1) / splits;
        splits = (nk_total + chunks - 1) / chunks;
        g.k_per_split = chunks * BK;
        g.split_stride = (long long)g.M * g.N;
        if ((size_t)splits * g.M * g.N > splitk_floats) {
            splits = 1;
        } else {
            g.C32 = splitk_ws;
            g.ldc32 = g.N;
        }
    }
    if (splits == 1) {
        g.k_per_split = nk_total * BK;
        g.split_stride = 0;
        g.C32 = final_out;
        g.ldc32 = final_ld;
    }
    dim3 grid(mt, ntile, splits);
    if (BN == 64) {
        int rc = set_gemm_smem<64>();
        if (rc != VP_OK) return rc;
        vp_mlp_gemm_kernel<64><<<grid, NT, gemm_smem_bytes<64>(), s>>>(g);
    } else {
        int rc = set_gemm_smem<128>();
        if (rc != VP_OK) return rc;
        vp_mlp_gemm_kernel<128><<<grid, NT, gemm_smem_bytes<128>(), s>>>(g);
    }
    count_launch();
    MLP_CUDA(cudaGetLastError(), "mlp gemm launch");
    if (splits > 1) {
        const long long total = (long long)g.M * g.N;
        const int blocks = (int)std::min<long long>(1024, (total + 255) / 256);
        vp_mlp_splitk_reduce_kernel<<<blocks, 256, 0, s>>>(splitk_ws, g.split_stride, g.N, splits, g.M, g.N,
                                                           final_out, final_ld);
        count_launch();
        MLP_CUDA(cudaGetLastError(), "mlp split-K reduce launch");
    }
    return VP_OK;
}

GemmArgs gemm_args(const bf16* A, long long lda, const bf16* B, long long ldb, int M, int N, int K,
                   unsigned* err) {
    GemmArgs g{};
    g.A = A;
    g.lda = lda;
    g.B = B;
    g.ldb = ldb;
    g.M = M;
    g.N = N;
    g.K = K;
    g.err = err;
    g.wait_ns = kDefaultWaitNs;
    return g;
}

int check_batch(const vp_mlp* n, int M) {
    if (M < 1 || M > n->max_batch) return set_err(VP_ERR_ARG, "batch %d outside [1, %d]", M, n->max_batch);
    return VP_OK;
}

int splits_for(int out_tiles, int K) {
    const int nk = (K + BK - 1) / BK;
    return std::max(1, std::min(nk, 148 / std::max(1, out_tiles)));
}

int mlp_forward_impl(vp_mlp* n, const float* X, long long ldx, const int* rows, int M, cudaStream_t s) {
    const int Mp = pad8(M);
    {
        const long long total = (long long)Mp * pad8(n->w[0]);
        const int blocks = (int)std::min<long long>(1024, (total + 255) / 256);
        vp_mlp_pack_kernel<<<blocks, 256, 0, s>>>(X, ldx, rows, M, n->w[0], n->Xb, pad8(n->w[0]), n->XbT,
                                                  pad8(n->max_batch), nullptr, 0);
        count_launch();
        MLP_CUDA(cudaGetLastError(), "mlp pack launch");
    }
    for (int l = 0; l < n->L; ++l) {
        const int K = n->w[l], N = n->w[l + 1];
        const bf16* Ain = l == 0 ? n->Xb : n->Ab[l - 1];
        GemmArgs g = gemm_args(Ain, pad8(K), n->R.Wb[l], pad8(K), M, N, pad8(K), n->err);
        g.wait_ns = n->wait_ns;
        g.bias = n->params + n->R.off_b[l];
        if (l == n->L - 1) {
            g.act = 0;
            g.C32 = n->Y;
            g.ldc32 = pad8(N);
        } else {
            g.act = 1;
            g.Zout = n->Z[l];
            g.ldz = N;
            g.C16 = n->Ab[l];
            g.ldc16 = pad8(N);
            g.C16T = n->AbT[l];
            g.ldc16t = pad8(n->max_batch);
        }
        int rc = launch_gemm(g, 1, nullptr, 0, s);
        if (rc != VP_OK) return rc;
    }
    n->last_M = M;
    (void)Mp;
    return VP_OK;
}

// Backward from the cotangent already in D32/Db/DbT[L-1].
int mlp_backward_impl(vp_mlp* n, int M, bool param_grads, float* g_X, long long ldgx, cudaStream_t s) {
    const int Mp = pad8(M);
    const long long ldT = pad8(n->max_batch);
    for (int l = n->L - 1; l >= 0; --l) {
        const int K = n->w[l], N = n->w[l + 1];
        if (param_grads) {
            // dW[N, K] = D^T[N, M] . Ain^T[K, M]^T
            const bf16* AinT = l == 0 ? n->XbT : n->AbT[l - 1];
            GemmArgs g = gemm_args(n->DbT[l], ldT, AinT, ldT, N, K, Mp, n->err);
            g.wait_ns = n->wait_ns;
            g.act = 0;
            g.C32 = n->grads + n->R.off_W[l];
            g.ldc32 = K;
            const int tiles = ((N + BM - 1) / BM) * ((K + gemm_bn(K) - 1) / gemm_bn(K));
            int rc = launch_gemm(g, splits_for(tiles, Mp), n->splitk, n->splitk_floats, s);
            if (rc != VP_OK) return rc;
            vp_mlp_colsum_kernel<<<(N + 31) / 32, dim3(32, 8), 0, s>>>(n->D32[l], N, M, N,
                                                                      n->grads + n->R.off_b[l]);
            count_launch();
            MLP_CUDA(cudaGetLastError(), "mlp colsum launch");
        }
        if (l == 0 && g_X == nullptr) break;
        // dA[M, K] = D[M, N] . W[N, K]  (B operand W^T[K, pad8(N)])
        GemmArgs g = gemm_args(n->Db[l], pad8(N), n->R.WbT[l], pad8(N), M, K, pad8(N), n->err);
        g.wait_ns = n->wait_ns;
        if (l > 0) {
            g.act = 2;
            g.aux = n->Z[l - 1];
            g.ldaux = K;
            g.C32 = n->D32[l - 1];
            g.ldc32 = K;
            g.C16 = n->Db[l - 1];
            g.ldc16 = pad8(K);
            g.C16T = n->DbT[l - 1];
            g.ldc16t = ldT;
        } else {
            g.act = 0;
            g.C32 = g_X;
            g.ldc32 = ldgx;
        }
        int rc = launch_gemm(g, 1, nullptr, 0, s);
        if (rc != VP_OK) return rc;
    }
    (void)Mp;
    return VP_OK;
}

}  // namespace

extern "C" {

int vp_mlp_create(int32_t n_layers, const int32_t* widths, int32_t max_batch, vp_mlp** out) {
    if (!out || !widths) return set_err(VP_ERR_ARG, "widths and out_mlp must not be NULL");
    *out = nullptr;
    if (n_layers < 1 || n_layers > MAX_LAYERS)
        return set_err(VP_ERR_ARG, "n_layers must be in [1, %d] (got %d)", MAX_LAYERS, n_layers);
    if (max_batch < 1) return set_err(VP_ERR_ARG, "max_batch must be >= 1");
    for (int l = 0; l <= n_layers; ++l)
        if (widths[l] < 1 || widths[l] > 4096) return set_err(VP_ERR_ARG, "layer widths must be in [1, 4096]");
    vp_mlp* n = new (std::nothrow) vp_mlp();
    if (!n) return set_err(VP_ERR_ARG, "out of host memory");
    cudaGetDevice(&n->device);
    n->L = n_layers;
    n->max_batch = max_batch;
    for (int l = 0; l <= n_layers; ++l) n->w[l] = widths[l];
    long long off = 0;
    n->R.L = n_layers;
    for (int l = 0; l < n_layers; ++l) {
        n->R.n_in[l] = widths[l];
        n->R.n_out[l] = widths[l + 1];
        n->R.off_W[l] = off;
        off += (long long)widths[l] * widths[l + 1];
        n->R.off_b[l] = off;
        off += widths[l + 1];
    }
    n->n_params = off;
    const size_t Bp = pad8(max_batch);
    int rc = VP_OK;
    auto A = [&](auto** p, size_t count) {
        if (rc == VP_OK) rc = mlp_alloc(n, p, count);
    };
    A(&n->params, off);
    A(&n->grads, off);
    A(&n->adam_m, off);
    A(&n->adam_v, off);
    A(&n->step, 1);
    A(&n->err, 1);
    for (int l = 0; l < n_layers; ++l) {
        A(&n->R.Wb[l], (size_t)widths[l + 1] * pad8(widths[l]));
        A(&n->R.WbT[l], (size_t)widths[l] * pad8(widths[l + 1]));
    }
    A(&n->Xb, Bp * pad8(widths[0]));
    A(&n->XbT, (size_t)widths[0] * Bp);
    size_t split_need = 0;
    for (int l = 0; l < n_layers; ++l) {
        const int Nl = widths[l + 1];
        if (l < n_layers - 1) {
            A(&n->Z[l], Bp * Nl);
            A(&n->Ab[l], Bp * pad8(Nl));
            A(&n->AbT[l], (size_t)Nl * Bp);
        }
        A(&n->D32[l], Bp * Nl);
        A(&n->Db[l], Bp * pad8(Nl));
        A(&n->DbT[l], (size_t)Nl * Bp);
        split_need = std::max(split_need, (size_t)148 * Nl * widths[l]);
    }
    A(&n->Y, Bp * pad8(widths[n_layers]));
    n->splitk_floats = split_need;
    A(&n->splitk, split_need);
    n->n_partial = 512;
    A(&n->partial, n->n_partial);
    if (rc != VP_OK) {
        mlp_free(n);
        return rc;
    }
    *out = n;
    return VP_OK;
}

int vp_mlp_destroy(vp_mlp* n) {
    mlp_free(n);
    return VP_OK;
}

int vp_mlp_param_count(const vp_mlp* n, int64_t* count) {
    if (!n || !count) return set_err(VP_ERR_ARG, "mlp and count must not be NULL");
    *count = n->n_params;
    return VP_OK;
}

int vp_mlp_set_params(vp_mlp* n, const float* params, void* stream) {
    if (!n || !params) return set_err(VP_ERR_ARG, "mlp and params must not be NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    MLP_CUDA(cudaMemcpyAsync(n->params, params, n->n_params * sizeof(float), cudaMemcpyDeviceToDevice, s),
             "copy params");
    MLP_CUDA(cudaMemsetAsync(n->adam_m, 0, n->n_params * sizeof(float), s), "zero adam m");
    MLP_CUDA(cudaMemsetAsync(n->adam_v, 0, n->n_params * sizeof(float), s), "zero adam v");
    MLP_CUDA(cudaMemsetAsync(n->step, 0, sizeof(int), s), "zero step");
    const int blocks = (int)std::min<long long>(1024, (n->n_params + 255) / 256);
    vp_mlp_refresh_kernel<<<blocks, 256, 0, s>>>(n->params, n->n_params, n->R);
    count_launch();
    MLP_CUDA(cudaGetLastError(), "mlp refresh launch");
    return VP_OK;
}

int vp_mlp_get_params(const vp_mlp* n, float* params, float* grads, void* stream) {
    if (!n) return set_err(VP_ERR_ARG, "mlp must not be NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (params)
        MLP_CUDA(cudaMemcpyAsync(params, n->params, n->n_params * sizeof(float), cudaMemcpyDeviceToDevice, s),
                 "copy params");
    if (grads)
        MLP_CUDA(cudaMemcpyAsync(grads, n->grads, n->n_params * sizeof(float), cudaMemcpyDeviceToDevice, s),
                 "copy grads");
    return VP_OK;
}

int vp_mlp_forward(vp_mlp* n, const float* X, int64_t ldx, const int32_t* rows, int32_t M, float* Y,
                   int64_t ldy, void* stream) {
    if (!n || !X) return set_err(VP_ERR_ARG, "mlp and X must not be NULL");
    int rc = check_batch(n, M);
    if (rc != VP_OK) return rc;
    if (ldx < n->w[0]) return set_err(VP_ERR_ARG, "ldx (%lld) < input width %d", (long long)ldx, n->w[0]);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    rc = mlp_forward_impl(n, X, ldx, rows, M, s);
    if (rc != VP_OK) return rc;
    if (Y) {
        const int Nout = n->w[n->L];
        if (ldy < Nout) return set_err(VP_ERR_ARG, "ldy (%lld) < output width %d", (long long)ldy, Nout);
        MLP_CUDA(cudaMemcpy2DAsync(Y, ldy * sizeof(float), n->Y, pad8(Nout) * sizeof(float), Nout * sizeof(float),
                                   M, cudaMemcpyDeviceToDevice, s),
                 "copy mlp output");
    }
    return VP_OK;
}

int vp_mlp_backward(vp_mlp* n, const float* g_Y, int64_t ldg, int32_t M, int32_t param_grads, float* g_X,
                    int64_t ldgx, void* stream) {
    if (!n || !g_Y) return set_err(VP_ERR_ARG, "mlp and g_Y must not be NULL");
    int rc = check_batch(n, M);
    if (rc != VP_OK) return rc;
    if (M != n->last_M) return set_err(VP_ERR_ARG, "backward batch %d differs from the last forward's %d", M, n->last_M);
    const int L = n->L, Nout = n->w[L];
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long total = (long long)pad8(M) * pad8(Nout);
    const int blocks = (int)std::min<long long>(1024, (total + 255) / 256);
    vp_mlp_pack_kernel<<<blocks, 256, 0, s>>>(g_Y, ldg, nullptr, M, Nout, n->Db[L - 1], pad8(Nout), n->DbT[L - 1],
                                              pad8(n->max_batch), n->D32[L - 1], Nout);
    count_launch();
    MLP_CUDA(cudaGetLastError(), "mlp pack launch");
    return mlp_backward_impl(n, M, param_grads != 0, g_X, ldgx, s);
}

int vp_mlp_mse_backward(vp_mlp* n, const float* target, int64_t ldt, const int32_t* rows, int32_t M,
                        float* loss, void* stream) {
    if (!n || !target) return set_err(VP_ERR_ARG, "mlp and target must not be NULL");
    int rc = check_batch(n, M);
    if (rc != VP_OK) return rc;
    if (M != n->last_M) return set_err(VP_ERR_ARG, "backward batch %d differs from the last forward's %d", M, n->last_M);
    const int L = n->L, Nout = n->w[L];
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long total = (long long)pad8(M) * pad8(Nout);
    const int blocks = (int)std::min<long long>(n->n_partial, (total + 255) / 256);
    vp_mlp_mse_kernel<<<blocks, 256, 0, s>>>(n->Y, pad8(Nout), target, ldt, rows, M, Nout, n->D32[L - 1], Nout,
                                             n->Db[L - 1], pad8(Nout), n->DbT[L - 1], pad8(n->max_batch),
                                             n->partial);
    count_launch();
    MLP_CUDA(cudaGetLastError(), "mlp mse launch");
    if (loss) {
        vp_mlp_loss_kernel<<<1, 32, 0, s>>>(n->partial, blocks, 1.0f / ((float)M * (float)Nout), loss);
        count_launch();
        MLP_CUDA(cudaGetLastError(), "mlp loss launch");
    }
    return mlp_backward_impl(n, M, true, nullptr, 0, s);
}

int vp_mlp_adam(vp_mlp* n, float lr, float beta1, float beta2, float eps, void* stream) {
    if (!n) return set_err(VP_ERR_ARG, "mlp must not be NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = (int)std::min<long long>(1024, (n->n_params + 255) / 256);
    vp_mlp_adam_kernel<<<blocks, 256, 0, s>>>(n->params, n->grads, n->adam_m, n->adam_v, n->n_params, n->step, lr,
                                              beta1, beta2, eps, n->R);
    count_launch();
    MLP_CUDA(cudaGetLastError(), "mlp adam launch");
    vp_mlp_step_kernel<<<1, 32, 0, s>>>(n->step);
    count_launch();
    MLP_CUDA(cudaGetLastError(), "mlp step launch");
    return VP_OK;
}

int vp_mlp_status(vp_mlp* n, uint32_t* flags) {
    if (!n || !flags) return set_err(VP_ERR_ARG, "mlp and flags must not be NULL");
    MLP_CUDA(cudaMemcpy(flags, n->err, sizeof(unsigned), cudaMemcpyDeviceToHost), "read mlp status");
    return VP_OK;
}

int vp_mlp_clear_status(vp_mlp* n) {
    if (!n) return set_err(VP_ERR_ARG, "mlp must not be NULL");
    MLP_CUDA(cudaMemset(n->err, 0, sizeof(unsigned)), "clear mlp status");
    MLP_CUDA(cudaDeviceSynchronize(), "clear mlp status");
    return VP_OK;
}

int vp_mlp_set_wait_limit(vp_mlp* n, uint64_t ns) {
    if (!n) return set_err(VP_ERR_ARG, "mlp must not be NULL");
    n->wait_ns = ns;
    return VP_OK;
}

int vp_mlp_search(vp_mlp* n, const float* c0, int32_t iters, float lr, float beta1, float beta2, float eps,
                  float x_scale, const float* y_mean, const float* y_std, const float* weights, float* best_c,
                  float* best_J, void* stream) {
    if (!n || !c0 || !y_mean || !y_std || !weights || !best_c || !best_J)
        return set_err(VP_ERR_ARG, "pointers must not be NULL");
    if (iters < 1) return set_err(VP_ERR_ARG, "iters must be >= 1");
    for (int l = 0; l <= n->L; ++l)
        if (n->w[l] > kSearchMaxWidth) return set_err(VP_ERR_ARG, "layer width %d exceeds %d", n->w[l], kSearchMaxWidth);
    SearchArgs A{};
    A.R = n->R;
    A.params = n->params;
    for (int l = 0; l <= n->L; ++l) A.w[l] = n->w[l];
    A.c0 = c0;
    A.iters = iters;
    A.lr = lr;
    A.b1 = beta1;
    A.b2 = beta2;
    A.eps = eps;
    A.x_scale = x_scale;
    A.y_mean = y_mean;
    A.y_std = y_std;
    A.wt = weights;
    A.best_c = best_c;
    A.best_J = best_J;
    vp_mlp_search_kernel<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(A);
    count_launch();
    MLP_CUDA(cudaGetLastError(), "mlp search launch");
    return VP_OK;
}

int vp_gemm_bf16(const void* A, int64_t lda, const void* B, int64_t ldb, int32_t M, int32_t N, int32_t K,
                 const float* bias, int32_t act, const float* aux, int64_t ldaux, float* C32, int64_t ldc32,
                 void* C16, int64_t ldc16, void* C16T, int64_t ldc16t, uint32_t* err, void* stream) {
    if (!A || !B) return set_err(VP_ERR_ARG, "A and B must not be NULL");
    if (M < 1 || N < 1 || K < 8) return set_err(VP_ERR_ARG, "need M, N >= 1 and K >= 8");
    if (K % 8 || lda % 8 || ldb % 8 || lda < K || ldb < K)
        return set_err(VP_ERR_ARG, "K, lda and ldb must be multiples of 8 with lda, ldb >= K");
    if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15)
        return set_err(VP_ERR_ARG, "A and B must be 16-byte aligned");
    if (act < 0 || act > 2 || (act == 2 && !aux)) return set_err(VP_ERR_ARG, "act must be 0, 1 or 2 (2 needs aux)");
    if (!C32 && !C16 && !C16T) return set_err(VP_ERR_ARG, "no output given");
    GemmArgs g = gemm_args(static_cast<const bf16*>(A), lda, static_cast<const bf16*>(B), ldb, M, N, K,
                           reinterpret_cast<unsigned*>(err));
    g.bias = bias;
    g.act = act;
    g.aux = aux;
    g.ldaux = ldaux;
    g.C32 = C32;
    g.ldc32 = ldc32;
    g.C16 = static_cast<bf16*>(C16);
    g.ldc16 = ldc16;
    g.C16T = static_cast<bf16*>(C16T);
    g.ldc16t = ldc16t;
    return launch_gemm(g, 1, nullptr, 0, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
