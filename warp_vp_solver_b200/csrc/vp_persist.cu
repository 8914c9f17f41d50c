// Persistent forward time loop for large grids (float32, x-invariant f_eq, Strang scheme).
//
// One cooperative launch runs a whole forward loop (warp_vp_solver/solver.py:470-612): the
// per-step launches, the one-CTA Poisson tail and the host round trips of the reference (and of
// the per-step kernels in vp_kernels.cu) become one kernel whose CTAs meet at a software grid
// barrier once per step (twice on grids whose field is solved in slices, below).
//
// Work split. CTA g owns `bands_per_cta` consecutive bands of R rows, full width; a band is
// processed as n_chunks tiles of R rows x C = 256 columns. Because a CTA owns whole rows, the row
// sums of h_{n+1} (rho_{n+1}) are complete inside it and need no cross-CTA partials.
//
// Tile. Thread t (64 per CTA) owns the 4 consecutive columns j0 = c0 + 4t .. j0 + 3. The x shifts
// m_j of 4 neighbouring columns differ by at most one cell (checked on the host), so the thread
// walks one window of R + 4 rows of the v-step output o, rows r0 + 2*bm + k (bm = the smallest
// shift of its quad); a column whose shift is bm + 1 reads the same window two rows lower (a
// register select). The window rows of a tile are staged into shared memory by bulk-async copies
// (cp.async.bulk, no multicast) completed on an mbarrier, double-buffered so that the next tile's
// rows arrive while this one computes. Per window row the v step reads its 5 source cells with one
// 16-byte and one 4-byte shared-memory load and forms V(f_eq) - f_eq for the usual shifts m = 0
// and m = -1 from the first differences D of f_eq held in registers:
//   m = 0:  o = h[j] + t*((h[j+1] - h[j]) + D[j])
//   m = -1: o = (h[j-1] - D[j-1]) + t*((h[j] - h[j-1]) + D[j-1])
// (the same value as lerp + correction of the per-step kernels, associated differently); shifts in
// [-4, 4) use the A_m, B_m tables, larger ones the float64 form from global memory.
//
// Field. After the barrier every CTA needs E + H on the rows its next tiles read. On grids where
// that window times nx is small (configuration 3: 28 rows x 512), each CTA evaluates
// E_i = sum_k c[(i-k) mod nx] rho_k for its window rows itself (c = real(ifft(m)), the circulant
// form of warp_vp_solver/poisson.py:34-69); otherwise CTA g solves a slice of nx/G rows, publishes
// their v shifts, and a second barrier precedes the tiles. The energies of the own rows go to
// per-CTA partials that CTA 0 sums in a fixed order one step later, so every result is
// deterministic.
//
// Every wait is bounded: a grid barrier that does not complete within the plan's wait limit
// raises VP_STATUS_WAIT_TIMEOUT in the plan's status word and the CTA returns (no bulk copy is in
// flight at a barrier); the bulk-copy waits give up after one second the same way.

#include "../../include/vp_b200.h"
#include "vp_device.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace vpb {

namespace {

constexpr int kPstThreads = 64;
constexpr int kPstC = 4 * kPstThreads;      // columns per tile
constexpr int kPstW = kPstC + 8;            // staged row: 4 halo columns on each side
constexpr unsigned long long kCopyWaitNs = 1000000000ull;

__device__ __forceinline__ uint32_t pst_smem(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long pst_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void pst_mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pst_smem(bar)) : "memory");
}

__device__ __forceinline__ void pst_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(pst_smem(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool pst_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(pst_smem(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bulk-async copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global to
// this CTA's shared memory, counted on `bar`.
__device__ __forceinline__ void pst_bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            pst_smem(dst)),
        "l"(src), "r"(bytes), "r"(pst_smem(bar))
        : "memory");
}

__device__ __forceinline__ void pst_fence_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
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
    pst_fence_async_global();   // this thread's state stores are visible to later bulk copies
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

}  // namespace

// E_i = sum_k c[(i-k) mod nx] rho_k for n_rows rows i = (first + r) mod nx, r < n_rows; calls
// out(r, E_i) from one lane per row. A warp takes 4 consecutive rows; lane g sums k = g, g + 32,
// ... in order (the table ctab[j] = c[(j - nx) mod nx] covers the unreduced row indices), then a
// fixed-order butterfly combines the 32 partial sums.
template <typename F>
__device__ __forceinline__ void pst_circ_rows(const float* __restrict__ ctab, const float* __restrict__ rho,
                                              int nx, int first, int n_rows, F&& out) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int ngrp = (n_rows + 3) >> 2;
    for (int grp = (int)(threadIdx.x >> 5); grp < ngrp; grp += nw) {
        const int i0 = pst_wrap(first + 4 * grp, nx);
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        const float* cp = ctab + nx + i0 - lane;
#pragma unroll 4
        for (int k = lane; k < nx; k += 32) {
            const float xk = __ldcg(rho + k);
            acc[0] += __ldg(cp) * xk;
            acc[1] += __ldg(cp + 1) * xk;
            acc[2] += __ldg(cp + 2) * xk;
            acc[3] += __ldg(cp + 3) * xk;
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

// Shared memory of a launch: two stage buffers, the row records of the union window, the row-sum
// scratch.
size_t persist_smem_bytes(int span_max, int win_rows, int R) {
    size_t b = (size_t)2 * span_max * kPstW * sizeof(float);
    b += ((size_t)win_rows * sizeof(int2) + 15) & ~(size_t)15;
    b += (size_t)(kPstThreads / 32) * R * sizeof(float) + 16;
    return b;
}

template <int R>
__global__ void __launch_bounds__(kPstThreads) vp_persist_fwd_kernel(const PersistArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[2];
    __shared__ int s_flag;
    __shared__ double s_ee[kPstThreads / 32];

    const int nx = a.nx, nv = a.nv, nch = a.n_chunks;
    const size_t nxnv = (size_t)nx * nv;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int g = blockIdx.x, G = gridDim.x;
    const int b0 = g * a.bands_per_cta;
    const int r_lo = b0 * R;                          // first own row
    const int own_rows = a.bands_per_cta * R;
    float* stage0 = reinterpret_cast<float*>(smem);
    float* stage1 = stage0 + (size_t)a.span_max * kPstW;
    int2* rinfo = reinterpret_cast<int2*>(stage1 + (size_t)a.span_max * kPstW);
    float* red = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(rinfo) +
                                          (((size_t)a.win_rows * sizeof(int2) + 15) & ~(size_t)15));
    const bool replay = a.mode == 1;
    const int n_first = replay ? a.first_step : 0;
    const int n_end = a.n_steps;                      // steps n_first .. n_end - 1
    const int ntile = a.bands_per_cta * nch;

    if (tid == 0) {
        pst_mbar_init(&full[0]);
        pst_mbar_init(&full[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    auto slot = [&](int n) -> float* {
        if (a.ckpt != nullptr && n % a.K == 0) return a.ckpt + (size_t)(n / a.K) * nxnv;
        if (replay) return a.seg + (size_t)(n % a.K - 1) * nxnv;
        return (n & 1) ? a.hbuf1 : a.hbuf0;
    };

    unsigned bar_index = 0;
    bool alive = true;
    auto barrier = [&]() -> bool {
        if (!pst_grid_barrier(a.bar, bar_index++, (unsigned)G, a.wait_ns, a.status, &s_flag)) alive = false;
        return alive;
    };

    // ---- staging: tile i of a step (band b0 + i / nch, chunk i % nch) into stage i & 1 ----
    unsigned long long tiles_issued = 0, tiles_used = 0;   // over the whole launch
    auto issue = [&](int i, const float* src) {
        const unsigned long long mine = tiles_issued++;
        if (wid != 0) return;
        const int bi = i / nch, c = i - bi * nch;
        const int r0 = (b0 + bi) * R, c0 = c * kPstC;
        const int2 cm = __ldg(a.chunk + c);           // (min bm, max bm) over the chunk
        const int span = 2 * (cm.y - cm.x) + R + 4;
        const int lo = r0 + 2 * cm.x;
        float* st = (mine & 1) ? stage1 : stage0;
        uint64_t* fb = &full[mine & 1];
        if (lane == 0) pst_expect_tx(fb, (unsigned)(span * kPstW * sizeof(float)));
        __syncwarp();
        pst_fence_async_global();
        for (int k = lane; k < span; k += 32) {
            const float* srow = src + (size_t)pst_wrap(lo + k, nx) * nv;
            float* drow = st + (size_t)k * kPstW;
            if (c0 > 0 && c0 + kPstC < nv) {
                pst_bulk_g2s(drow, srow + c0 - 4, kPstW * sizeof(float), fb);
            } else {
                const int lc = c0 == 0 ? nv - 4 : c0 - 4;
                const int rc = c0 + kPstC == nv ? 0 : c0 + kPstC;
                pst_bulk_g2s(drow, srow + lc, 16, fb);
                pst_bulk_g2s(drow + 4, srow + c0, kPstC * sizeof(float), fb);
                pst_bulk_g2s(drow + 4 + kPstC, srow + rc, 16, fb);
            }
        }
    };
    auto wait_stage = [&]() -> bool {
        uint64_t* fb = &full[tiles_used & 1];
        const unsigned parity = (unsigned)((tiles_used >> 1) & 1);
        bool ok = pst_try_wait(fb, parity);
        if (!ok) {
            const unsigned long long t0 = pst_now();
            while (!(ok = pst_try_wait(fb, parity)))
                if (pst_now() - t0 > kCopyWaitNs) break;
        }
        if (!ok && tid == 0) atomicOr(a.status, VP_STATUS_WAIT_TIMEOUT);
        return __syncthreads_and(ok) != 0;
    };

    // ---- field: v shifts of the union window rows into rinfo ----
    const int win_first = r_lo + a.win_lo;            // global row of rinfo[0] (unreduced)
    auto field_local = [&](int n) {
        // E of every union window row from rho_n; own rows also write E_hist, the tape and the
        // energy partial
        const float* rho = a.rho + (size_t)(n & 1) * nx;
        double e2 = 0.0;
        pst_circ_rows(a.ctab, rho, nx, win_first, a.win_rows, [&](int u, float E) {
            const int i = pst_wrap(win_first + u, nx);
            const float Et = E + __ldg(a.H + i);
            const VShift<float> vs = make_vshift<float>(Et, a.dtdv, nv);
            rinfo[u] = pst_rinfo(vs, nv);
            const int own = u + a.win_lo;             // row offset from r_lo
            if (own >= 0 && own < own_rows) {
                if (a.E_hist != nullptr) a.E_hist[(size_t)n * nx + i] = Et;
                if (a.E_tape != nullptr) a.E_tape[(size_t)n * nx + i] = E;
                if (a.vsh_tape != nullptr) a.vsh_tape[(size_t)n * nx + i] = vs;
                e2 += (double)(trap_w<float>(i, nx) * E * E);
            }
        });
        return e2;
    };
    auto field_slice = [&](int n) {
        const float* rho = a.rho + (size_t)(n & 1) * nx;
        const int S = (nx + G - 1) / G;
        const int first = g * S;
        const int cnt = max(0, min(S, nx - first));
        double e2 = 0.0;
        pst_circ_rows(a.ctab, rho, nx, first, cnt, [&](int u, float E) {
            const int i = first + u;
            const float Et = E + __ldg(a.H + i);
            const VShift<float> vs = make_vshift<float>(Et, a.dtdv, nv);
            a.vsh_g[i] = vs;
            if (a.E_hist != nullptr) a.E_hist[(size_t)n * nx + i] = Et;
            if (a.E_tape != nullptr) a.E_tape[(size_t)n * nx + i] = E;
            if (a.vsh_tape != nullptr) a.vsh_tape[(size_t)n * nx + i] = vs;
            e2 += (double)(trap_w<float>(i, nx) * E * E);
        });
        return e2;
    };
    auto rinfo_from = [&](const VShift<float>* vsh) {
        for (int u = tid; u < a.win_rows; u += blockDim.x) {
            const VShift<float>* p = vsh + pst_wrap(win_first + u, nx);
            VShift<float> v;
            v.m = __ldcg(&p->m);
            v.t = __ldcg(&p->t);
            rinfo[u] = pst_rinfo(v, nv);
        }
    };
    auto publish_energy = [&](int n, double e2) {
        e2 = warp_sum(e2);
        if (lane == 0) s_ee[wid] = e2;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < kPstThreads / 32; ++w) s += s_ee[w];
            a.eep[(size_t)(n & 3) * G + g] = s;
        }
    };
    auto sum_energy = [&](int n) {   // CTA 0, after the barrier that published step n's partials
        if (g != 0 || a.ee_hist == nullptr || wid != 0) return;
        double s = 0.0;
        for (int c = lane; c < G; c += 32) s += __ldcg(a.eep + (size_t)(n & 3) * G + c);
        // fixed order: lane partials, then a fixed butterfly
        s = warp_sum(s);
        if (lane == 0) a.ee_hist[n] = (float)(0.5 * s * (double)a.dx);
    };

    // ---- per-thread column constants ----
    // (reloaded per chunk: quad record, x weights, f_eq differences, trapezoid weights)

    // ---- row sums of a band: acc[R] over the CTA's threads in a fixed order -> rho ----
    auto band_rows = [&](float (&acc)[R], int r0, float* rho_out) {
        constexpr int LG = R >= 32 ? 5 : R >= 16 ? 4 : R >= 8 ? 3 : R >= 4 ? 2 : R >= 2 ? 1 : 0;
#pragma unroll
        for (int st = 0; st < LG; ++st) {
            const int o = 16 >> st;
            const int n = R >> (st + 1);
            const bool upper = (lane & o) != 0;
#pragma unroll
            for (int i = 0; i < (R >> 1); ++i) {
                if (i < n) {
                    const float send = upper ? acc[i] : acc[i + n];
                    const float keep = upper ? acc[i + n] : acc[i];
                    acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
                }
            }
        }
        float v = acc[0];
#pragma unroll
        for (int o = 16 >> LG; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((lane & ((32 >> LG) - 1)) == 0) red[wid * R + (lane >> (5 - LG))] = v;
        __syncthreads();
        if (tid < R) {
            float s = 0.f;
            for (int w = 0; w < kPstThreads / 32; ++w) s += red[w * R + tid];
            rho_out[r0 + tid] = -a.dv * s;
        }
        __syncthreads();
    };

    // ---- prologue (full mode): h_0 = X(f_iv - f_eq) on the own rows, rho_0 ----
    if (!replay) {
        float* h0 = slot(0);
        for (int bi = 0; bi < a.bands_per_cta; ++bi) {
            const int r0 = (b0 + bi) * R;
            float acc[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = 0.f;
            for (int c = 0; c < nch; ++c) {
                const int q = c * kPstThreads + tid;
                const int j0 = 4 * q;
                const int2 qi = __ldg(a.quad + q);
                const float4 tq = __ldg(a.tq + q);
                const double2 fa = __ldg(reinterpret_cast<const double2*>(a.feq + j0));
                const double2 fb = __ldg(reinterpret_cast<const double2*>(a.feq + j0 + 2));
                const double fe[4] = {fa.x, fa.y, fb.x, fb.y};
                const float tt[4] = {tq.x, tq.y, tq.z, tq.w};
                float d[R + 2][4];
#pragma unroll
                for (int k = 0; k < R + 2; ++k) {
                    const int row = pst_wrap(r0 + qi.x + k, nx);
                    const double2* fr = reinterpret_cast<const double2*>(a.f_iv + (size_t)row * nv + j0);
                    const double2 u = __ldg(fr), v = __ldg(fr + 1);
                    d[k][0] = (float)(u.x - fe[0]);
                    d[k][1] = (float)(u.y - fe[1]);
                    d[k][2] = (float)(v.x - fe[2]);
                    d[k][3] = (float)(v.y - fe[3]);
                }
                float hv[R][4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const bool dl = (qi.y >> e) & 1;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const float p0 = dl ? d[r + 1][e] : d[r][e];
                        const float p1 = dl ? d[r + 2][e] : d[r + 1][e];
                        hv[r][e] = pst_lerp(p0, p1, tt[e]);
                    }
                }
                const float w0 = j0 == 0 ? 0.5f : 1.f, w3 = j0 + 3 == nv - 1 ? 0.5f : 1.f;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    *reinterpret_cast<float4*>(h0 + (size_t)(r0 + r) * nv + j0) =
                        make_float4(hv[r][0], hv[r][1], hv[r][2], hv[r][3]);
                    acc[r] += w0 * hv[r][0] + hv[r][1] + hv[r][2] + w3 * hv[r][3];
                }
            }
            band_rows(acc, r0, a.rho);   // rho_0 in buffer 0
        }
        if (!barrier()) return;
    }

    for (int n = n_first; n < n_end && alive; ++n) {
        const bool last = !replay && n == a.n_steps - 1;
        const float* src = slot(n);
        float* dst = last ? nullptr : slot(n + 1);
        // the first two tiles of the step load while the field is solved
        issue(0, src);
        if (ntile > 1) issue(1, src);
        if (replay) {
            rinfo_from(a.vsh_tape_in + (size_t)n * nx);
        } else if (a.field_dist == 0) {
            const double e2 = field_local(n);
            publish_energy(n, e2);
            if (n >= 1) sum_energy(n - 1);
        } else {
            const double e2 = field_slice(n);
            publish_energy(n, e2);
            if (!barrier()) break;
            if (n >= 1) sum_energy(n - 1);
            rinfo_from(a.vsh_g);
        }
        __syncthreads();

        float* rho_next = a.rho + (size_t)((n + 1) & 1) * nx;
        float acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = 0.f;
        for (int i = 0; i < ntile; ++i) {
            const int bi = i / nch, c = i - bi * nch;
            const int r0 = (b0 + bi) * R, c0 = c * kPstC;
            const int q = c * kPstThreads + tid;
            const int j0 = c0 + 4 * tid;
            const int2 cm = __ldg(a.chunk + c);
            const int2 qi = __ldg(a.quad + q);
            const float4 tq = __ldg(a.tq + q);
            const float tt[4] = {tq.x, tq.y, tq.z, tq.w};
            const float4 D4 = __ldg(reinterpret_cast<const float4*>(a.dfeq + j0));
            const float Dm1 = __ldg(a.dfeq + (j0 == 0 ? nv - 1 : j0 - 1));
            if (!wait_stage()) {
                alive = false;
                break;
            }
            const float* st = (tiles_used & 1) ? stage1 : stage0;
            ++tiles_used;
            // window row k of this thread: stage row 2*(bm - cm.x) + k, global row r0 + 2*bm + k
            const float* sb = st + (size_t)(2 * (qi.x - cm.x)) * kPstW + 4 + 4 * tid;
            const int ib = (r0 - r_lo) + 2 * qi.x - a.win_lo;   // rinfo index of window row 0
            float O[R + 4][4];
#pragma unroll
            for (int k = 0; k < R + 4; ++k) {
                const int2 ri = rinfo[ib + k];
                const float tv = __int_as_float(ri.y);
                const float* sr = sb + (size_t)k * kPstW;
                if (ri.x == 0) {
                    const float4 h = *reinterpret_cast<const float4*>(sr);
                    const float h4 = sr[4];
                    O[k][0] = h.x + tv * ((h.y - h.x) + D4.x);
                    O[k][1] = h.y + tv * ((h.z - h.y) + D4.y);
                    O[k][2] = h.z + tv * ((h.w - h.z) + D4.z);
                    O[k][3] = h.w + tv * ((h4 - h.w) + D4.w);
                } else if (ri.x == -1) {
                    const float hm = sr[-1];
                    const float4 h = *reinterpret_cast<const float4*>(sr);
                    O[k][0] = (hm - Dm1) + tv * ((h.x - hm) + Dm1);
                    O[k][1] = (h.x - D4.x) + tv * ((h.y - h.x) + D4.x);
                    O[k][2] = (h.y - D4.y) + tv * ((h.z - h.y) + D4.y);
                    O[k][3] = (h.z - D4.z) + tv * ((h.w - h.z) + D4.z);
                } else if (ri.x >= -kStageHalo && ri.x < kStageHalo) {
                    const float* p = sr + ri.x;
                    const float v[5] = {p[0], p[1], p[2], p[3], p[4]};
                    const float4 A = __ldg(reinterpret_cast<const float4*>(a.vtab + (size_t)(ri.x + kStageHalo) * nv + j0));
                    const float4 B = __ldg(reinterpret_cast<const float4*>(
                        a.vtab + (size_t)(2 * kStageHalo + ri.x + kStageHalo) * nv + j0));
                    O[k][0] = v[0] + tv * (v[1] - v[0]) + (A.x + tv * B.x);
                    O[k][1] = v[1] + tv * (v[2] - v[1]) + (A.y + tv * B.y);
                    O[k][2] = v[2] + tv * (v[3] - v[2]) + (A.z + tv * B.z);
                    O[k][3] = v[3] + tv * (v[4] - v[3]) + (A.w + tv * B.w);
                } else {
                    // shift beyond the staged halo: the float64 form from global memory
                    const int row = pst_wrap(r0 + 2 * qi.x + k, nx);
                    VShift<float> vs;
                    vs.m = ri.x < 0 ? ri.x + nv : ri.x;
                    vs.t = tv;
#pragma unroll
                    for (int e = 0; e < 4; ++e) O[k][e] = pst_v_cell(src, a.feq, nv, row, j0 + e, vs.m, vs.t);
                }
            }
            // x steps per column: window offset 0 or 2 rows (delta bit), d = X(o), h' = X(d)
            float dd[R + 1][4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const bool dl = (qi.y >> e) & 1;
                float p0 = dl ? O[2][e] : O[0][e];
#pragma unroll
                for (int q2 = 0; q2 <= R; ++q2) {
                    const float p1 = dl ? O[q2 + 3][e] : O[q2 + 1][e];
                    dd[q2][e] = pst_lerp(p0, p1, tt[e]);
                    p0 = p1;
                }
            }
            if (a.f_hist != nullptr || (last && a.f_final != nullptr)) {
                float* fh = a.f_hist != nullptr ? a.f_hist + (size_t)(n - n_first) * nxnv : nullptr;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const double fe = __ldg(a.feq + j0 + e);
                    const int base = r0 + qi.x + ((qi.y >> e) & 1);
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int row = pst_wrap(base + r, nx);
                        const double f = fe + (double)dd[r][e];
                        if (fh != nullptr) fh[(size_t)row * nv + j0 + e] = (float)f;
                        if (last && a.f_final != nullptr) a.f_final[(size_t)row * nv + j0 + e] = f;
                    }
                }
            }
            if (dst != nullptr) {
                const float w0 = j0 == 0 ? 0.5f : 1.f, w3 = j0 + 3 == nv - 1 ? 0.5f : 1.f;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const float h0v = pst_lerp(dd[r][0], dd[r + 1][0], tt[0]);
                    const float h1v = pst_lerp(dd[r][1], dd[r + 1][1], tt[1]);
                    const float h2v = pst_lerp(dd[r][2], dd[r + 1][2], tt[2]);
                    const float h3v = pst_lerp(dd[r][3], dd[r + 1][3], tt[3]);
                    *reinterpret_cast<float4*>(dst + (size_t)(r0 + r) * nv + j0) = make_float4(h0v, h1v, h2v, h3v);
                    acc[r] += w0 * h0v + h1v + h2v + w3 * h3v;
                }
            }
            __syncthreads();   // the stage is free
            if (i + 2 < ntile) issue(i + 2, src);
            if (c == nch - 1) {
                if (!replay && !last) band_rows(acc, r0, rho_next);
#pragma unroll
                for (int r = 0; r < R; ++r) acc[r] = 0.f;
            }
        }
        if (!alive) break;
        if (!barrier()) break;
    }
    // a CTA that stopped early still owns the bulk copies it issued: wait for them (bounded)
    while (tiles_used < tiles_issued) {
        wait_stage();
        ++tiles_used;
    }
    if (alive && !replay) sum_energy(a.n_steps - 1);
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------

static const int kPstRows[] = {16, 8, 4};

template <int R>
static cudaError_t pst_set_smem(size_t smem) {
    return cudaFuncSetAttribute(vp_persist_fwd_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int R>
static int pst_max_blocks(size_t smem) {
    int n = 0;
    if (pst_set_smem<R>(smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, vp_persist_fwd_kernel<R>, kPstThreads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

static int pst_max_blocks_r(int R, size_t smem) {
    switch (R) {
        case 4: return pst_max_blocks<4>(smem);
        case 8: return pst_max_blocks<8>(smem);
        case 16: return pst_max_blocks<16>(smem);
        default: return 0;
    }
}

// Host tables and launch shape of the persistent path for one grid. Returns false when the grid
// is not eligible: nv a multiple of 256, the x shifts of every 4 neighbouring columns within one
// cell of each other, windows shorter than a period.
bool persist_prepare(PersistHost& ph, int nx, int nv, const std::vector<long long>& m_signed,
                     const std::vector<double>& tx, int n_sms, int force_rows) {
    ph = PersistHost{};
    if (nv % kPstC != 0 || nx < 8) return false;
    const int nq = nv / 4;
    ph.quad.resize(nq);
    ph.tq.resize((size_t)4 * nq);
    long long all_lo = 1LL << 40, all_hi = -(1LL << 40);
    for (int q = 0; q < nq; ++q) {
        long long lo = m_signed[4 * q], hi = lo;
        for (int e = 1; e < 4; ++e) {
            lo = std::min(lo, m_signed[4 * q + e]);
            hi = std::max(hi, m_signed[4 * q + e]);
        }
        if (hi - lo > 1 || 2 * std::llabs(lo) > nx || 2 * std::llabs(hi) > nx) return false;
        int mask = 0;
        for (int e = 0; e < 4; ++e) mask |= (m_signed[4 * q + e] - lo == 1 ? 1 : 0) << e;
        ph.quad[q] = make_int2((int)lo, mask);
        for (int e = 0; e < 4; ++e) ph.tq[(size_t)4 * q + e] = (float)tx[4 * q + e];
        all_lo = std::min(all_lo, lo);
        all_hi = std::max(all_hi, lo);
    }
    const int nch = nv / kPstC;
    ph.chunk.resize(nch);
    int dmax = 0;
    for (int c = 0; c < nch; ++c) {
        int lo = 1 << 30, hi = -(1 << 30);
        for (int q = c * kPstThreads; q < (c + 1) * kPstThreads; ++q) {
            lo = std::min(lo, ph.quad[q].x);
            hi = std::max(hi, ph.quad[q].x);
        }
        ph.chunk[c] = make_int2(lo, hi);
        dmax = std::max(dmax, hi - lo);
    }
    // rows per band: the largest R of 16, 8, 4 that gives at least 0.8 bands per SM (or forced)
    int R = 0;
    for (int r : kPstRows) {
        if (nx % r != 0) continue;
        if (force_rows > 0 && r != force_rows) continue;
        R = r;
        if (force_rows > 0 || nx / r >= (4 * n_sms) / 5) break;
    }
    if (R == 0) return false;
    const int span_max = 2 * dmax + R + 4;
    if (span_max > nx) return false;
    const int bands = nx / R;
    // CTAs: bands / bands_per_cta, the smallest bands_per_cta that fits on the device at once
    for (int bpc = 1; bpc <= bands; ++bpc) {
        if (bands % bpc != 0) continue;
        const int G = bands / bpc;
        // the union window of the CTA's tiles (offsets from its first row), widened to cover
        // its own rows
        const int win_lo = std::min(2 * (int)all_lo, 0);
        const int win_end = std::max(bpc * R + 2 * (int)all_hi + 4, bpc * R);
        const int win_rows = win_end - win_lo;
        const size_t smem = persist_smem_bytes(span_max, win_rows, R);
        if (smem > 200 * 1024) continue;
        const int per_sm = pst_max_blocks_r(R, smem);
        if (per_sm <= 0) return false;
        if ((long long)per_sm * n_sms < G) continue;
        ph.R = R;
        ph.G = G;
        ph.bands_per_cta = bpc;
        ph.span_max = span_max;
        ph.win_lo = win_lo;
        ph.win_rows = win_rows;
        ph.smem = smem;
        // the field on each CTA's own window when that costs little, else in slices + a barrier
        ph.field_dist = (long long)win_rows * nx > (1LL << 17) ? 1 : 0;
        return true;
    }
    return false;
}

cudaError_t launch_persist_fwd(const PersistArgs& args, const PersistHost& ph, cudaStream_t s) {
    PersistArgs a = args;
    a.bands_per_cta = ph.bands_per_cta;
    a.span_max = ph.span_max;
    a.win_lo = ph.win_lo;
    a.win_rows = ph.win_rows;
    a.field_dist = ph.field_dist;
    cudaError_t e = cudaMemsetAsync(a.bar, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ph.G, 1, 1);
    cfg.blockDim = dim3(kPstThreads, 1, 1);
    cfg.dynamicSmemBytes = ph.smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    switch (ph.R) {
        case 4: e = cudaLaunchKernelEx(&cfg, vp_persist_fwd_kernel<4>, a); break;
        case 8: e = cudaLaunchKernelEx(&cfg, vp_persist_fwd_kernel<8>, a); break;
        case 16: e = cudaLaunchKernelEx(&cfg, vp_persist_fwd_kernel<16>, a); break;
        default: return cudaErrorInvalidValue;
    }
    count_launch();
    return e;
}

}  // namespace vpb
