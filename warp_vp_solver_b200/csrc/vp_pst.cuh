// Device helpers shared by the persistent loops (vp_persist.cu) and the strip step kernels
// (vp_strip.cu): column-group constants, asynchronous copies, the circulant field products, the
// per-quad constants and the out-of-line rare forms of the v step, V^T and the slope.
#pragma once

#include "../../include/vp_b200.h"
#include "vp_device.cuh"

namespace vpb {
namespace {

constexpr int kPstGroup = 64;              // threads of a column group: one tile of 256 columns
constexpr int kPstGroups = 4;              // column groups per CTA (different chunks of a band)
constexpr int kPstThreads = kPstGroup * kPstGroups;
constexpr int kPstWarps = kPstThreads / 32;
constexpr int kPstC = 4 * kPstGroup;       // columns per tile
constexpr int kPstW = kPstC + 8;            // staged row: 4 halo columns on each side
constexpr int kPstMaxStages = 8;            // stage buffers: tiles in flight ahead of the compute

__device__ __forceinline__ uint32_t pst_smem(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long pst_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Asynchronous 16-byte (or 4-byte) copies from global to shared memory through L2 (.cg: no L1
// allocation, so data written earlier in this launch by other CTAs is read coherently), grouped
// per tile with commit/wait_group.
__device__ __forceinline__ void pst_cp16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(pst_smem(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void pst_cp4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(pst_smem(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void pst_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most n of this thread's copy groups are pending (n < 8).
__device__ __forceinline__ void pst_cp_wait(int n) {
    switch (n) {
        case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
        case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
        case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
        case 3: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
        case 4: asm volatile("cp.async.wait_group 4;" ::: "memory"); break;
        case 5: asm volatile("cp.async.wait_group 5;" ::: "memory"); break;
        case 6: asm volatile("cp.async.wait_group 6;" ::: "memory"); break;
        default: asm volatile("cp.async.wait_group 7;" ::: "memory"); break;
    }
}

__device__ __forceinline__ unsigned pst_ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned pst_add_release(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Grid-wide barrier number `index` (0, 1, ...) of a launch of G CTAs on a counter that was zero at
// the launch: returns false (in every thread of the CTA) when it did not complete within limit_ns
// (limit 0: only the last CTA to arrive passes), after raising VP_STATUS_WAIT_TIMEOUT.
__device__ bool pst_grid_barrier(unsigned* ctr, unsigned index, unsigned G, unsigned long long limit_ns,
                                 unsigned* status, int* s_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned target = (index + 1u) * G;
        const unsigned prev = pst_add_release(ctr, 1u);
        bool ok = true;
        if (prev + 1u != target) {
            if (limit_ns == 0) {
                ok = false;
            } else {
                const unsigned long long t0 = pst_now();
                unsigned it = 0;
                while (pst_ld_acquire(ctr) < target) {
                    if ((++it & 31u) == 0 && pst_now() - t0 > limit_ns) {
                        ok = false;
                        break;
                    }
                }
            }
        }
        __threadfence();
        if (!ok) atomicOr(status, VP_STATUS_WAIT_TIMEOUT);
        *s_flag = ok ? 1 : 0;
    }
    __syncthreads();
    return *s_flag != 0;
}

__device__ __forceinline__ int pst_wrap(int r, int n) {   // r in [-2n, 3n)
    r += r < 0 ? n : 0;
    r += r < 0 ? n : 0;
    r -= r >= n ? n : 0;
    return r >= n ? r - n : r;
}

__device__ __forceinline__ float pst_lerp(float a, float b, float t) { return a + t * (b - a); }

// V step of one cell for a shift (m reduced mod nv, t) outside the staged halo: h read from global
// memory through L2 (the state was written by this launch), the f_eq correction in float64.
__device__ float pst_v_cell(const float* h, const double* __restrict__ feq, int nv, int row, int j, int m,
                            float t) {
    int c0 = j + m;
    c0 -= c0 >= nv ? nv : 0;
    const int c1 = c0 + 1 == nv ? 0 : c0 + 1;
    const float* hr = h + (size_t)row * nv;
    const float a = __ldcg(hr + c0), b = __ldcg(hr + c1);
    float o = (1.f - t) * a + t * b;
    const double fj = __ldg(feq + j);
    const double tt = (double)t;
    o += (float)((1.0 - tt) * (__ldg(feq + c0) - fj) + tt * (__ldg(feq + c1) - fj));
    return o;
}

// Signed v shift of a row for the tiles: (m, t) with m in (-nv/2, nv/2].
__device__ __forceinline__ int2 pst_rinfo(const VShift<float> v, int nv) {
    int2 r;
    r.x = v.m > nv / 2 ? v.m - nv : v.m;
    r.y = __float_as_int(v.t);
    return r;
}

// Issues (one commit group) the copies of the inputs of the circulant product for n_rows rows
// starting at `first` (unreduced) into shared memory: rho (nx floats, 16-byte loads through L2:
// written by this launch) at fs and the coefficient slice cs[u] = ctab[f0 + 1 + u], u < nx + n_rows
// + 4 (f0 = first mod nx) after it, where ctab[j] = c[(j - nx) mod nx]; then coefficient (row r, k)
// = cs[nx - 1 + r - k]. Returns f0. The caller waits for the group (groups committed after it may
// stay in flight) and then needs a block barrier.
__device__ __forceinline__ int pst_field_issue(float* fs, const float* rho, const float* __restrict__ ctab,
                                               int nx, int first, int n_rows) {
    const int f0 = pst_wrap(first, nx);
    for (int k = (int)threadIdx.x; k < nx / 4; k += blockDim.x) pst_cp16(fs + 4 * k, rho + 4 * k);
    float* cs = fs + nx;
    const int len = nx + n_rows + 4;
    for (int u = threadIdx.x; u < len; u += blockDim.x) pst_cp4(cs + u, ctab + f0 + 1 + u);
    pst_cp_commit();
    return f0;
}

// pst_field_issue, then a wait for every copy group of the thread and a block barrier.
__device__ __forceinline__ int pst_field_inputs(float* fs, const float* rho, const float* __restrict__ ctab,
                                                int nx, int first, int n_rows) {
    const int f0 = pst_field_issue(fs, rho, ctab, nx, first, n_rows);
    pst_cp_wait(0);
    __syncthreads();
    return f0;
}

// E_r = sum_k c[(f0 + r - k) mod nx] rho_k for r < n_rows from the staged inputs; calls out(r, E_r)
// from one lane per row. A warp takes 4 consecutive rows; lane g sums k = g, g + 32, ... in order
// (consecutive lanes read consecutive words of both arrays), then a fixed-order butterfly combines
// the 32 partial sums.
template <typename F>
__device__ __forceinline__ void pst_circ_rows(const float* fs, int nx, int n_rows, F&& out) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int ngrp = (n_rows + 3) >> 2;
    const float* cs = fs + nx;
    for (int grp = (int)(threadIdx.x >> 5); grp < ngrp; grp += nw) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        const float* cp = cs + nx - 1 + 4 * grp - lane;
#pragma unroll 4
        for (int k = lane; k < nx; k += 32) {
            const float xk = fs[k];
            acc[0] += cp[0] * xk;
            acc[1] += cp[1] * xk;
            acc[2] += cp[2] * xk;
            acc[3] += cp[3] * xk;
            cp -= 32;
        }
#pragma unroll
        for (int st = 0; st < 2; ++st) {
            const int o = 16 >> st;
            const int n = 2 >> st;
            const bool upper = (lane & o) != 0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (q < n) {
                    const float send = upper ? acc[q] : acc[q + n];
                    const float keep = upper ? acc[q + n] : acc[q];
                    acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, o);
                }
            }
        }
        float sum = acc[0];
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        const int r = 4 * grp + (lane >> 3);
        if ((lane & 7) == 0 && r < n_rows) out(r, sum);
    }
}

// The transposed product: E_r = sum_k c[(k - f0 - r) mod nx] x_k (Poisson^T, the adjoint's field),
// staged as cs[u] = ctab[2 nx - f0 - n_rows - 2 + u], u < nx + n_rows + 6: coefficient (row r, k)
// = cs[n_rows + 2 - r + k]. Needs n_rows <= nx - 8. pst_field_issue_t only issues the copies (one
// commit group); pst_field_inputs_t also waits for them and ends with a block barrier.
__device__ __forceinline__ int pst_field_issue_t(float* fs, const float* x, const float* __restrict__ ctab,
                                                 int nx, int first, int n_rows) {
    const int f0 = pst_wrap(first, nx);
    for (int k = (int)threadIdx.x; k < nx / 4; k += blockDim.x) pst_cp16(fs + 4 * k, x + 4 * k);
    float* cs = fs + nx;
    const int len = nx + n_rows + 6;
    const float* src = ctab + (2 * nx - f0 - n_rows - 2);
    for (int u = threadIdx.x; u < len; u += blockDim.x) pst_cp4(cs + u, src + u);
    pst_cp_commit();
    return f0;
}

__device__ __forceinline__ int pst_field_inputs_t(float* fs, const float* x, const float* __restrict__ ctab,
                                                  int nx, int first, int n_rows) {
    const int f0 = pst_field_issue_t(fs, x, ctab, nx, first, n_rows);
    pst_cp_wait(0);
    __syncthreads();
    return f0;
}

template <typename F>
__device__ __forceinline__ void pst_circ_rows_t(const float* fs, int nx, int n_rows, F&& out) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int ngrp = (n_rows + 3) >> 2;
    const float* cs = fs + nx;
    for (int grp = (int)(threadIdx.x >> 5); grp < ngrp; grp += nw) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        const float* cp = cs + n_rows + 2 - 4 * grp + lane;
#pragma unroll 4
        for (int k = lane; k < nx; k += 32) {
            const float xk = fs[k];
            acc[0] += cp[0] * xk;
            acc[1] += cp[-1] * xk;
            acc[2] += cp[-2] * xk;
            acc[3] += cp[-3] * xk;
            cp += 32;
        }
#pragma unroll
        for (int st = 0; st < 2; ++st) {
            const int o = 16 >> st;
            const int n = 2 >> st;
            const bool upper = (lane & o) != 0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (q < n) {
                    const float send = upper ? acc[q] : acc[q + n];
                    const float keep = upper ? acc[q + n] : acc[q];
                    acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, o);
                }
            }
        }
        float sum = acc[0];
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        const int r = 4 * grp + (lane >> 3);
        if ((lane & 7) == 0 && r < n_rows) out(r, sum);
    }
}

// Per-quad constants of the tiles (x weights, f_eq differences, smallest shift and its delta bits,
// the f_eq difference left of the quad), kept in shared memory for the whole launch when the
// grid's nv/4 records fit in kPstQuadSmemBytes.
struct __align__(16) PstQuad {
    float4 t;
    float4 D;
    int bm, mask;
    float Dm1, pad;
};
constexpr size_t kPstQuadSmemBytes = 24 * 1024;

// Floats of the field's shared-memory inputs for up to n_rows rows (rho, coefficient slice).
inline size_t pst_field_floats(int nx, int n_rows) { return (size_t)2 * nx + n_rows + 8; }

// V step of one row of a quad for the shifts other than 0 and -1 (kept out of line so that the
// unrolled tile loop stays small): shifts in [-4, 4) from the staged row and the A_m, B_m tables,
// larger ones in the float64 form from global memory.
__device__ __noinline__ float4 pst_v_rare(const float* __restrict__ vtab, const double* __restrict__ feq, int nv,
                                          const float* sr, const float* src, int ms, float tv, int row, int j0) {
    float4 o;
    if (ms >= -kStageHalo && ms < kStageHalo) {
        const float* pp = sr + ms;
        const float v[5] = {pp[0], pp[1], pp[2], pp[3], pp[4]};
        const float4 A = __ldg(reinterpret_cast<const float4*>(vtab + (size_t)(ms + kStageHalo) * nv + j0));
        const float4 B = __ldg(reinterpret_cast<const float4*>(vtab + (size_t)(2 * kStageHalo + ms + kStageHalo) * nv + j0));
        o.x = v[0] + tv * (v[1] - v[0]) + (A.x + tv * B.x);
        o.y = v[1] + tv * (v[2] - v[1]) + (A.y + tv * B.y);
        o.z = v[2] + tv * (v[3] - v[2]) + (A.z + tv * B.z);
        o.w = v[3] + tv * (v[4] - v[3]) + (A.w + tv * B.w);
    } else {
        const int mr = ms < 0 ? ms + nv : ms;
        o.x = pst_v_cell(src, feq, nv, row, j0, mr, tv);
        o.y = pst_v_cell(src, feq, nv, row, j0 + 1, mr, tv);
        o.z = pst_v_cell(src, feq, nv, row, j0 + 2, mr, tv);
        o.w = pst_v_cell(src, feq, nv, row, j0 + 3, mr, tv);
    }
    return o;
}

// V^T of one quad row for shifts other than 0 and -1 (out of line): staged for |shift| <= 4,
// global memory beyond.
__device__ __noinline__ float4 pst_vt_rare(const float* sr, const float* w_src, int nv, int ms, float tv,
                                           int row, int j0) {
    float4 o;
    if (ms >= -kStageHalo + 1 && ms <= kStageHalo - 1) {
        const float* pp = sr - ms - 1;
        const float v[5] = {pp[0], pp[1], pp[2], pp[3], pp[4]};
        o.x = v[1] + tv * (v[0] - v[1]);
        o.y = v[2] + tv * (v[1] - v[2]);
        o.z = v[3] + tv * (v[2] - v[3]);
        o.w = v[4] + tv * (v[3] - v[4]);
    } else {
        const int mr = ms < 0 ? ms + nv : ms;
        const float* wr = w_src + (size_t)row * nv;
        float r[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            int c0 = j0 + e - mr;
            c0 += c0 < 0 ? nv : 0;
            const int c1 = c0 == 0 ? nv - 1 : c0 - 1;
            r[e] = (1.f - tv) * __ldcg(wr + c0) + tv * __ldcg(wr + c1);
        }
        o = make_float4(r[0], r[1], r[2], r[3]);
    }
    return o;
}

// Slope (h + f_eq)[j + m + 1] - (h + f_eq)[j + m] of one quad row of h_{n-1} for shifts other than
// 0 and -1 (out of line).
__device__ __noinline__ float4 pst_slope_rare(const float* hr_s, const float* h_src, const float* vtab,
                                              const double* feq, int nv, int ms, int row, int j0) {
    float4 o;
    if (ms >= -kStageHalo && ms < kStageHalo) {
        const float* pp = hr_s + ms;
        const float4 B = __ldg(reinterpret_cast<const float4*>(vtab + (size_t)(2 * kStageHalo + ms + kStageHalo) * nv + j0));
        o.x = (pp[1] - pp[0]) + B.x;
        o.y = (pp[2] - pp[1]) + B.y;
        o.z = (pp[3] - pp[2]) + B.z;
        o.w = (pp[4] - pp[3]) + B.w;
    } else {
        const int mr = ms < 0 ? ms + nv : ms;
        const float* hr = h_src + (size_t)row * nv;
        float r[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            int d0 = j0 + e + mr;
            d0 -= d0 >= nv ? nv : 0;
            const int d1 = d0 + 1 == nv ? 0 : d0 + 1;
            r[e] = (__ldcg(hr + d1) - __ldcg(hr + d0)) + (float)(__ldg(feq + d1) - __ldg(feq + d0));
        }
        o = make_float4(r[0], r[1], r[2], r[3]);
    }
    return o;
}

}  // namespace
}  // namespace vpb
