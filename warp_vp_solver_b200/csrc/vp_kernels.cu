// Fused Strang-step kernels (forward and discrete adjoint) for sm_100a.
//
// Scheme (warp_vp_solver/solver.py:17-28, one step):
//   f_half = X(f); rho = dv*trapz(f_eq - f_half); E = Poisson(rho); ee = 0.5*dx*trapz(E^2);
//   f_one = V_{E+H}(f_half); f = X(f_one)
// with X the periodic linear semi-Lagrangian half step along x (kernels.py:109-130) and V the
// full step along v (kernels.py:133-153, 367-393).
//
// Representation. The state is delta = f - f_eq (float32 or float64). Each x half-step shifts
// column j by a fixed s_j = 0.5*v_j*dt/dx cells (integer part m_j, weight t_j, precomputed on
// the host in float64); the v step shifts row i by s_i = (E_i + H_i)*dt/dv cells. The pipeline
// carries h_n = delta after the leading x half-step of step n (f_half - f_eq), so that one launch
// per step reads h_n once and writes h_{n+1} once:
//
//   o  = V(h_n) + [V(f_eq) - f_eq]        rows around the block, per-row shift from E_n + H
//   d  = X(o)   + [X(f_eq) - f_eq]        = f_{n+1} - f_eq      (history / final output)
//   h' = X(d)   + [X(f_eq) - f_eq]        = h_{n+1}, and its row sums -> rho_{n+1}
//
// The f_eq corrections are formed in float64 from differences of f_eq and are exactly zero for
// an x-invariant f_eq in the x direction.
//
// Thread mapping. A CTA owns R consecutive rows [r0, r0+R) and a chunk of columns; each thread
// owns one column j at a time. Because the x shift of column j is one number, the rows column j
// needs are a contiguous window offset by m_j: R+2 rows of o, R+1 rows of d, R rows of h'. The
// windows live in registers with compile-time indices, so the two x half-steps need no shared
// memory and no block barrier. The v step reads h_n straight from global memory (coalesced along
// the row, each value reused by the neighbouring thread through L1).
//
// Step-global dependency. rho needs whole rows and E needs all of rho. Each CTA writes its rows'
// partial sums; the last CTA to finish (threadfence + atomic counter, no spinning) reduces them
// in a fixed order and runs the in-block FFT Poisson solve for the next step, writing E, E+H,
// ee and the next v shifts. The next launch in the stream consumes them.
//
// The adjoint mirrors this with gathers instead of the reference's atomic scatters
// (kernels.py:215-273): X^T g at row k is (1-t) g[k-m] + t g[k-m-1], V^T likewise along v, so
// every output is written by exactly one thread and the result is bitwise reproducible.

#include "vp_device.cuh"

namespace vpb {

template <typename T, bool FEQ2D>
__device__ __forceinline__ double feq_at(const double* __restrict__ feq, int rs, int row, int col) {
    return FEQ2D ? __ldg(feq + (size_t)row * rs + col) : __ldg(feq + col);
}

// V step of one cell: o[row, j] for the delta state h (plus the f_eq correction).
template <typename T, bool FEQ2D>
__device__ __forceinline__ T v_cell(const T* __restrict__ h, const double* __restrict__ feq,
                                    int feq_rs, int nv, int row, int j, const VShift<T> s) {
    int c0 = wrap1(j + s.m, nv);
    int c1 = c0 + 1;
    c1 = c1 == nv ? 0 : c1;
    const T* hr = h + (size_t)row * nv;
    const T a = __ldg(hr + c0);
    const T b = __ldg(hr + c1);
    T o = lerp(a, b, s.t);
    const double fj = feq_at<T, FEQ2D>(feq, feq_rs, row, j);
    const double f0 = feq_at<T, FEQ2D>(feq, feq_rs, row, c0) - fj;
    const double f1 = feq_at<T, FEQ2D>(feq, feq_rs, row, c1) - fj;
    const double tt = (double)s.t;
    o += (T)((1.0 - tt) * f0 + tt * f1);
    return o;
}

// f_eq[d0 + 1] - f_eq[d0] with d0 = j + m (the adjoint's slope term): B_m[j] from the tables, or
// the float64 difference.
template <typename T, bool FEQ2D>
__device__ __forceinline__ T feq_slope(const double* __restrict__ feq, int feq_rs, const T* __restrict__ vtab,
                                       int nv, int row, int j, int m, int d0, int d1) {
    if (!FEQ2D && vtab != nullptr) {
        const int ms = m >= nv / 2 ? m - nv : m;
        if (ms >= -kStageHalo && ms < kStageHalo)
            return __ldg(vtab + (size_t)(3 * kStageHalo + ms) * nv + j);   // B_m row
    }
    return (T)(feq_at<T, FEQ2D>(feq, feq_rs, row, d1) - feq_at<T, FEQ2D>(feq, feq_rs, row, d0));
}

// X(f_eq) - f_eq at (row, j) for an x-dependent f_eq (zero otherwise).
template <typename T, bool FEQ2D>
__device__ __forceinline__ T x_corr(const double* __restrict__ feq, int feq_rs, int nx, int row,
                                    int m, double t64, int j) {
    if (!FEQ2D) return T(0);
    int q0 = wrap1(row + m, nx);
    int q1 = q0 + 1;
    q1 = q1 == nx ? 0 : q1;
    const double fj = __ldg(feq + (size_t)row * feq_rs + j);
    const double a0 = __ldg(feq + (size_t)q0 * feq_rs + j) - fj;
    const double a1 = __ldg(feq + (size_t)q1 * feq_rs + j) - fj;
    return (T)((1.0 - t64) * a0 + t64 * a1);
}

// Reduce the R per-thread row accumulators over the block and store them as this chunk's
// partial sums for rows [r0, r0+R).
template <typename T, int R>
__device__ __forceinline__ void store_row_partials(T (&acc)[R], T* red, T* part_row) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    // transposed butterfly: R sums over the warp in log2(R) halving exchanges plus an xor tree
    // (R - 1 + 5 - log2(R) shuffles instead of 5 R); lane l ends with row l >> (5 - log2 R)
    constexpr int LG = R >= 32 ? 5 : R >= 16 ? 4 : R >= 8 ? 3 : R >= 4 ? 2 : R >= 2 ? 1 : 0;
    static_assert((1 << LG) == R, "rows per CTA must be a power of two <= 32");
#pragma unroll
    for (int st = 0; st < LG; ++st) {
        const int o = 16 >> st;
        const int n = R >> (st + 1);
        const bool upper = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < (R >> 1); ++i) {
            if (i < n) {
                const T send = upper ? acc[i] : acc[i + n];
                const T keep = upper ? acc[i + n] : acc[i];
                acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
            }
        }
    }
    T v = acc[0];
#pragma unroll
    for (int o = 16 >> LG; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((lane & ((32 >> LG) - 1)) == 0) red[wid * R + (lane >> (5 - LG))] = v;
    __syncthreads();
    if (threadIdx.x < R) {
        T s = T(0);
        for (int w = 0; w < nw; ++w) s += red[w * R + threadIdx.x];
        part_row[threadIdx.x] = s;
    }
}

// Completion counter: returns true in every thread of the CTA that finished the last of
// `total` units of work counted on `counter`.
__device__ __forceinline__ bool last_unit_done(unsigned* counter, unsigned total, int* flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned prev = atomicAdd(counter, 1u);
        *flag = (prev == total - 1) ? 1 : 0;
    }
    __syncthreads();
    const bool last = *flag != 0;
    if (last) __threadfence();
    return last;
}

// Completion counter: returns true in every thread of the CTA that finished last.
__device__ __forceinline__ bool last_cta_done(unsigned* counter, int* flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned total = gridDim.x * gridDim.y;
        const unsigned prev = atomicAdd(counter, 1u);
        *flag = (prev == total - 1) ? 1 : 0;
    }
    __syncthreads();
    const bool last = *flag != 0;
    if (last) __threadfence();
    return last;
}

// Forward tail (one CTA): rho_{n+1} from the chunk partial sums, E_{n+1} = Poisson(rho), ee, and
// the next step's E + H and v shifts.
template <typename T>
__device__ void fwd_tail(const FwdArgs<T>& a, PoissonArea<T> w, T* red) {
    const int nx = a.nx;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        T s = T(0);
        for (int c = 0; c < a.n_chunks; ++c) s += __ldcg(a.part + (size_t)c * nx + i);
        poisson_put<T>(a.P, w.z, i, -a.dv * s);
    }
    poisson_core<T>(a.P, w.z, w.tw, false);
    T e2 = T(0);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const T E = poisson_get<T>(a.P, w.z, i);
        e2 += trap_w<T>(i, nx) * E * E;
        const T Et = E + __ldg(a.H + i);
        a.E_out[i] = E;
        if (a.E_hist_out != nullptr) a.E_hist_out[i] = Et;
        a.vsh_out[i] = make_vshift<T>(Et, a.dtdv, a.nv);
    }
    const T tot = block_sum<T>(e2, red);
    if (threadIdx.x == 0 && a.ee_out != nullptr) *a.ee_out = T(0.5) * tot * a.dx;
}

// Backward tail (one CTA), for step n-1: g_E_total = -dt/dv * sum_j slope*w + g_E_hist;
// g_H += g_E_total; g_E = g_E_total + ee^T; grho_{n-1} = Poisson^T g_E.
template <typename T>
__device__ void bwd_tail(const BwdArgs<T>& a, PoissonArea<T> w) {
    const int nx = a.nx;
    const T gee = a.gee != nullptr ? *a.gee : T(0);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        T s = T(0);
        for (int c = 0; c < a.n_chunks; ++c) s += __ldcg(a.part + (size_t)c * nx + i);
        T gEt = a.neg_dt_dv * s;
        if (a.gE_hist != nullptr) gEt += __ldg(a.gE_hist + i);
        a.gH[i] += gEt;
        // ee^T (kernels.py:302-322): dx * w_i * E_i * g_ee
        poisson_put<T>(a.P, w.z, i, gEt + a.dx * trap_w<T>(i, nx) * __ldg(a.E_prev + i) * gee);
    }
    poisson_core<T>(a.P, w.z, w.tw, true);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) a.grho_out[i] = poisson_get<T>(a.P, w.z, i);
}

// ----------------------------------------------------------------------------------------------
// Forward
// PHASE 0 (prologue): h_0 = X(f_iv - f_eq) + Xcorr, rho_0, tail -> E_0.
// PHASE 1 (step n):   h_n -> o -> d (= f_{n+1} - f_eq) -> [h_{n+1}, rho_{n+1}, tail -> E_{n+1}]
// PHASE 3 (merged-Strang inner step, warp_vp_solver/solver.py:618-736): h_n -> o -> h_{n+1} =
//                     X(dt)(o) with the full-step x tables, f_hist[n] = f_eq + h_{n+1}, rho_{n+1}.
//                     The bracket is skipped when h_out == null (last step). With part == null
//                     the launch only propagates the state (segment recomputation in the adjoint).
// ----------------------------------------------------------------------------------------------
// One tile of the fused forward: rows [r0, r0+R) x columns [c_begin, c_end), one column per
// thread at a time; accumulates the trapezoid-weighted row sums of h_{n+1} into acc.
template <typename T, int R, bool FEQ2D, int PHASE>
__device__ __forceinline__ void fwd_tile(const FwdArgs<T>& a, int r0, int c_begin, int c_end,
                                         T (&acc)[R]) {
    const int nx = a.nx, nv = a.nv;
    const bool next = a.h_out != nullptr;
    for (int j = c_begin + (int)threadIdx.x; j < c_end; j += blockDim.x) {
        const int m = __ldg(a.mx + j);
        const T t = __ldg(a.tx + j);
        const double t64 = FEQ2D ? __ldg(a.tx64 + j) : 0.0;
        const T wj = trap_w<T>(j, nv);
        if (PHASE == 3) {
            // merged inner step (full-step x tables in mx/tx): h' rows r0 + e from o rows r0 + m + k
            const int base = wrap1(r0 + m, nx);
            T o[R + 1];
#pragma unroll
            for (int k = 0; k < R + 1; ++k) {
                const int row = wrap1(base + k, nx);
                o[k] = v_cell<T, FEQ2D>(a.h_in, a.feq, a.feq_rs, nv, row, j, a.vsh[row]);
            }
#pragma unroll
            for (int e = 0; e < R; ++e) {
                T hv = lerp(o[e], o[e + 1], t);
                if (FEQ2D) hv += x_corr<T, FEQ2D>(a.feq, a.feq_rs, nx, r0 + e, m, t64, j);
                if (a.f_hist_n != nullptr)
                    a.f_hist_n[(size_t)(r0 + e) * nv + j] = (T)(feq_at<T, FEQ2D>(a.feq, a.feq_rs, r0 + e, j) + (double)hv);
                if (next) {
                    a.h_out[(size_t)(r0 + e) * nv + j] = hv;
                    acc[e] += wj * hv;
                }
            }
            continue;
        }
        T d[R + 1];
        if (PHASE == 0) {
            const int base = wrap1(r0 + m, nx);
#pragma unroll
            for (int k = 0; k < R + 1; ++k) {
                const int row = wrap1(base + k, nx);
                const double fv = __ldg(a.f_iv + (size_t)row * nv + j);
                d[k] = (T)(fv - feq_at<T, FEQ2D>(a.feq, a.feq_rs, row, j));
            }
        } else {
            const int base = wrap2(r0 + 2 * m, nx);
            T o[R + 2];
#pragma unroll
            for (int k = 0; k < R + 2; ++k) {
                const int row = wrap1(base + k, nx);
                const VShift<T> vs = a.vsh[row];
                o[k] = v_cell<T, FEQ2D>(a.h_in, a.feq, a.feq_rs, nv, row, j, vs);
            }
            const int dbase = wrap1(r0 + m, nx);
#pragma unroll
            for (int k = 0; k < R + 1; ++k) {
                d[k] = lerp(o[k], o[k + 1], t);
                if (FEQ2D) d[k] += x_corr<T, FEQ2D>(a.feq, a.feq_rs, nx, wrap1(dbase + k, nx), m, t64, j);
            }
            if (a.f_hist_n != nullptr || a.f_final != nullptr) {
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    const int row = wrap1(dbase + k, nx);
                    const double f = feq_at<T, FEQ2D>(a.feq, a.feq_rs, row, j) + (double)d[k];
                    if (a.f_hist_n != nullptr) a.f_hist_n[(size_t)row * nv + j] = (T)f;
                    if (a.f_final != nullptr) a.f_final[(size_t)row * nv + j] = f;
                }
            }
        }
        if (PHASE == 0 || next) {
#pragma unroll
            for (int e = 0; e < R; ++e) {
                T hv = lerp(d[e], d[e + 1], t);
                if (FEQ2D) hv += x_corr<T, FEQ2D>(a.feq, a.feq_rs, nx, r0 + e, m, t64, j);
                a.h_out[(size_t)(r0 + e) * nv + j] = hv;
                acc[e] += wj * hv;
            }
        }
    }

}

template <typename T, int R, bool FEQ2D, int PHASE>
__global__ void __launch_bounds__(256) vp_fwd_kernel(const FwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    T* red = reinterpret_cast<T*>(smem);
    __shared__ int s_last;

    const int nx = a.nx, nv = a.nv;
    const int r0 = blockIdx.x * R;
    const int c_begin = blockIdx.y * a.chunk_cols;
    const int c_end = min(nv, c_begin + a.chunk_cols);
    const bool next = a.h_out != nullptr;

    T acc[R];
#pragma unroll
    for (int e = 0; e < R; ++e) acc[e] = T(0);
    fwd_tile<T, R, FEQ2D, PHASE>(a, r0, c_begin, c_end, acc);

    if (a.part == nullptr || (PHASE != 0 && !next)) return;
    store_row_partials<T, R>(acc, red, a.part + (size_t)blockIdx.y * nx + r0);
    if (a.counter == nullptr) return;   // the tail runs as its own launch (large nx)
    if (!last_cta_done(a.counter, &s_last)) return;

    const size_t red_bytes = (size_t)32 * R * sizeof(T);
    fwd_tail<T>(a, poisson_area<T>(a.P, smem + ((red_bytes + 15) & ~(size_t)15)), red);
    if (threadIdx.x == 0) *a.counter = 0u;
}

// ----------------------------------------------------------------------------------------------
// Backward (discrete adjoint, warp_vp_solver/solver.py:814-929 per step)
// PHASE 0 (n = T):   c = g_f_final + g_f_hist[T-1]; w_{T-1} = X^T c; row sums for g_E_total.
// PHASE 1 (n >= 1):  gh = V^T w_n + rho^T grho_n; c = X^T gh (+ g_f_hist[n-1]); w_{n-1} = X^T c.
// PHASE 2 (n = 0):   g_f_iv = X^T (V^T w_0 + rho^T grho_0).
// PHASE 3 (merged inner step, solver.py:1111-1338): c = V^T w_n + rho^T grho_n + g_f_hist[n-1];
//                    w_{n-1} = X(dt)^T c with the full-step x tables.
// Tail (phases 0, 1), for step n-1: g_E_total = -dt/dv * sum_j slope*w + g_E_hist; g_H += g_E_total;
// g_E = g_E_total + ee^T; grho_{n-1} = Poisson^T g_E.
// ----------------------------------------------------------------------------------------------
// One tile of the fused adjoint: rows [r0, r0+R) x columns [c_begin, c_end); accumulates the
// slope-weighted row sums for g_E_total into acc (phases 0 and 1).
template <typename T, int R, bool FEQ2D, int PHASE>
__device__ __forceinline__ void bwd_tile(const BwdArgs<T>& a, int r0, int c_begin, int c_end,
                                         T (&acc)[R]) {
    const int nx = a.nx, nv = a.nv;
    for (int j = c_begin + (int)threadIdx.x; j < c_end; j += blockDim.x) {
        const int m = __ldg(a.mx + j);
        const T t = __ldg(a.tx + j);
        const T wr = -a.dv * trap_w<T>(j, nv);   // rho^T weight (kernels.py:292-299)
        if (PHASE == 2) {
            // gh rows r0 - m - 1 + k, k in [0, R+1); out rows r0 + e
            const int base = wrapneg(r0 - m - 1, nx);   // r0 - m - 1 >= -nx
            T gh[R + 1];
#pragma unroll
            for (int k = 0; k < R + 1; ++k) {
                const int row = wrap1(base + k, nx);
                const VShift<T> vs = a.vsh_n[row];
                int c0 = wrapneg(j - vs.m, nv);
                int c1 = wrapneg(c0 - 1, nv);
                const T* wrow = a.w_in + (size_t)row * nv;
                gh[k] = lerp(__ldg(wrow + c0), __ldg(wrow + c1), vs.t) + wr * __ldg(a.grho + row);
            }
#pragma unroll
            for (int e = 0; e < R; ++e) {
                a.gfiv_out[(size_t)(r0 + e) * nv + j] = lerp(gh[e + 1], gh[e], t);
            }
            continue;
        }
        // c rows r0 - m - 1 + k, k in [0, R+1)
        const int cbase = wrapneg(r0 - m - 1, nx);
        T c[R + 1];
        if (PHASE == 0) {
#pragma unroll
            for (int k = 0; k < R + 1; ++k) {
                const int row = wrap1(cbase + k, nx);
                T v = T(0);
                if (a.c_src != nullptr) v += __ldg(a.c_src + (size_t)row * nv + j);
                if (a.c_src2 != nullptr) v += __ldg(a.c_src2 + (size_t)row * nv + j);
                c[k] = v;
            }
        } else if (PHASE == 3) {
            // merged inner step (full-step x tables): c = V^T w + rho^T grho (+ g_f_hist) on the
            // rows of the single X^T window
#pragma unroll
            for (int k = 0; k < R + 1; ++k) {
                const int row = wrap1(cbase + k, nx);
                const VShift<T> vs = a.vsh_n[row];
                int c0 = wrapneg(j - vs.m, nv);
                int c1 = wrapneg(c0 - 1, nv);
                const T* wrow = a.w_in + (size_t)row * nv;
                c[k] = lerp(__ldg(wrow + c0), __ldg(wrow + c1), vs.t) + wr * __ldg(a.grho + row);
                if (a.gfh != nullptr) c[k] += __ldg(a.gfh + (size_t)row * nv + j);
            }
        } else {
            // gh rows r0 - 2m - 2 + k, k in [0, R+2)
            const int base = wrapneg2(r0 - 2 * m - 2, nx);   // r0 - 2m - 2 >= -2nx
            T gh[R + 2];
#pragma unroll
            for (int k = 0; k < R + 2; ++k) {
                const int row = wrap1(base + k, nx);
                const VShift<T> vs = a.vsh_n[row];
                int c0 = wrapneg(j - vs.m, nv);
                int c1 = wrapneg(c0 - 1, nv);
                const T* wrow = a.w_in + (size_t)row * nv;
                gh[k] = lerp(__ldg(wrow + c0), __ldg(wrow + c1), vs.t) + wr * __ldg(a.grho + row);
            }
#pragma unroll
            for (int k = 0; k < R + 1; ++k) {
                c[k] = lerp(gh[k + 1], gh[k], t);
                if (a.gfh != nullptr) c[k] += __ldg(a.gfh + (size_t)wrap1(cbase + k, nx) * nv + j);
            }
        }
        // w rows r0 + e, and the slope reduction for g_E_total of step n-1
#pragma unroll
        for (int e = 0; e < R; ++e) {
            const T wv = lerp(c[e + 1], c[e], t);
            const int row = r0 + e;
            a.w_out[(size_t)row * nv + j] = wv;
            const VShift<T> vp = a.vsh_prev[row];
            const int d0 = wrap1(j + vp.m, nv);
            int d1 = d0 + 1;
            d1 = d1 == nv ? 0 : d1;
            const T* hr = a.h_prev + (size_t)row * nv;
            const T sl = (__ldg(hr + d1) - __ldg(hr + d0)) +
                         feq_slope<T, FEQ2D>(a.feq, a.feq_rs, a.vtab, nv, row, j, vp.m, d0, d1);
            acc[e] += sl * wv;
        }
    }

}

template <typename T, int R, bool FEQ2D, int PHASE>
__global__ void __launch_bounds__(256) vp_bwd_kernel(const BwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    T* red = reinterpret_cast<T*>(smem);
    __shared__ int s_last;

    const int nx = a.nx, nv = a.nv;
    const int r0 = blockIdx.x * R;
    const int c_begin = blockIdx.y * a.chunk_cols;
    const int c_end = min(nv, c_begin + a.chunk_cols);

    T acc[R];
#pragma unroll
    for (int e = 0; e < R; ++e) acc[e] = T(0);
    bwd_tile<T, R, FEQ2D, PHASE>(a, r0, c_begin, c_end, acc);

    if (PHASE == 2) return;
    store_row_partials<T, R>(acc, red, a.part + (size_t)blockIdx.y * nx + r0);
    if (a.counter == nullptr) return;   // the tail runs as its own launch (large nx)
    if (!last_cta_done(a.counter, &s_last)) return;

    const size_t red_bytes = (size_t)32 * R * sizeof(T);
    bwd_tail<T>(a, poisson_area<T>(a.P, smem + ((red_bytes + 15) & ~(size_t)15)));
    if (threadIdx.x == 0) *a.counter = 0u;
}

// Tails as their own single-CTA launches (used when the Poisson work area does not fit in the
// fused kernels' shared-memory budget).
template <typename T>
__global__ void __launch_bounds__(1024) vp_fwd_tail_kernel(const FwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ T red[32];
    fwd_tail<T>(a, poisson_area<T>(a.P, smem), red);
}

template <typename T>
__global__ void __launch_bounds__(1024) vp_bwd_tail_kernel(const BwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    bwd_tail<T>(a, poisson_area<T>(a.P, smem));
}

// ----------------------------------------------------------------------------------------------
// Staged forward step (x-invariant f_eq). The arithmetic of fwd_tile PHASE 1, organised for
// throughput on large grids:
//  * a CTA owns rows [r0, r0+R) and C = blockDim.x columns [c0, c0+C) (one column per thread);
//  * the rows its columns' x windows touch, [r0 + 2 min m, r0 + 2 max m + R + 2), are staged in
//    shared memory with a halo of kStageHalo cells on each side along v, by coalesced 16-byte
//    loads (each staged value is read from global memory once per CTA);
//  * the v step reads its two source cells from shared memory at any offset and adds the f_eq
//    correction from per-shift tables A_m[j] = f_eq[j+m] - f_eq[j], B_m[j] = f_eq[j+m+1] -
//    f_eq[j+m] (float64 differences rounded once on the host): V(f_eq) - f_eq = A_m + t B_m;
//  * the x window is walked row by row with a rolling (o, d) pair.
// Rows whose v shift lies outside [-kStageHalo, kStageHalo) take the float64 scalar form.
// ----------------------------------------------------------------------------------------------
template <typename T>
struct Vec16 {
    using type = float4;
};
template <>
struct Vec16<double> {
    using type = double2;
};

// Shared memory of the staged kernel, after the row-partial scratch: the staged rows
// [span][C + 2 kStageHalo], the per-row shift records [span], and the correction tables of the
// CTA's columns [2][2 kStageHalo][C].
template <typename T>
__host__ __device__ constexpr size_t staged_bytes(int span, int C) {
    return (size_t)span * (C + 2 * kStageHalo) * sizeof(T) + (((size_t)span * 8 + 15) & ~(size_t)15) +
           (size_t)4 * kStageHalo * C * sizeof(T);
}

template <typename T, int R, int C>
__global__ void __launch_bounds__(C) vp_fwds_kernel(const FwdArgs<T> a) {
    using V = typename Vec16<T>::type;
    constexpr int VE = 16 / sizeof(T);
    constexpr int HV = kStageHalo;
    constexpr int W = C + 2 * HV;
    constexpr int PER_ROW = W / VE;
    constexpr int NM = 2 * HV;
    extern __shared__ __align__(16) unsigned char smem[];
    T* red = reinterpret_cast<T*>(smem);
    const size_t red_bytes = (((size_t)32 * R * sizeof(T)) + 15) & ~(size_t)15;
    const int span_max = a.stage_span;
    T* stage = reinterpret_cast<T*>(smem + red_bytes);
    int2* rinfo = reinterpret_cast<int2*>(smem + red_bytes + (size_t)span_max * W * sizeof(T));
    T* tabs = reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(rinfo) + (((size_t)span_max * 8 + 15) & ~(size_t)15));
    __shared__ int s_last, s_min, s_max;

    const int nx = a.nx, nv = a.nv;
    const int r0 = blockIdx.x * R;
    const int tid = threadIdx.x;
    const bool next = a.h_out != nullptr;
    const bool outf = a.f_hist_n != nullptr || a.f_final != nullptr;
    const int g_begin = blockIdx.y * a.chunk_cols;
    const int g_end = min(nv, g_begin + a.chunk_cols);

    T acc[R];
#pragma unroll
    for (int e = 0; e < R; ++e) acc[e] = T(0);

    for (int c0 = g_begin; c0 < g_end; c0 += C) {
        const int j = c0 + tid;   // C divides nv and the group width
        const int m = __ldg(a.mx + j);
        const int sm = m > nx / 2 ? m - nx : m;   // signed x offset
        int mn = sm, mxv = sm;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mxv = max(mxv, __shfl_xor_sync(0xffffffffu, mxv, o));
        }
        if (tid == 0) {
            s_min = mn;
            s_max = mxv;
        }
        __syncthreads();
        if ((tid & 31) == 0 && tid != 0) {
            atomicMin(&s_min, mn);
            atomicMax(&s_max, mxv);
        }
        __syncthreads();
        const int lo = r0 + 2 * s_min;
        const int span = 2 * (s_max - s_min) + R + 2;
        const bool staged = span <= span_max;
        const int lo_w = wrapboth(lo, nx);   // signed offsets in (-nx/2, nx/2]: lo in [-nx-2, 2nx)
        if (staged) {
            for (int idx = tid; idx < span * PER_ROW; idx += C) {
                const int q = idx / PER_ROW, v = idx - q * PER_ROW;
                int row = lo_w + q;
                row -= row >= nx ? nx : 0;
                int col = c0 - HV + v * VE;
                col += col < 0 ? nv : 0;
                col -= col >= nv ? nv : 0;
                reinterpret_cast<V*>(stage + q * W)[v] =
                    __ldg(reinterpret_cast<const V*>(a.h_in + (size_t)row * nv + col));
            }
            for (int q = tid; q < span; q += C) {
                int row = lo_w + q;
                row -= row >= nx ? nx : 0;
                const VShift<T> vs = a.vsh[row];
                const int ms = vs.m >= nv / 2 ? vs.m - nv : vs.m;
                int2 info;
                info.x = (ms >= -HV && ms < HV) ? ms + HV : -1;
                if constexpr (sizeof(T) == 4) {
                    info.y = __float_as_int((float)vs.t);
                } else {
                    info.y = row;   // float64: the weight is read back from the shift record
                }
                rinfo[q] = info;
            }
#pragma unroll
            for (int r = 0; r < 2 * NM; ++r) tabs[r * C + tid] = __ldg(a.vtab + (size_t)r * nv + j);
        }
        __syncthreads();
        {
            const T t = __ldg(a.tx + j);
            const T wj = trap_w<T>(j, nv);
            const int gbase = wrap2(r0 + 2 * m, nx);
            const int sbase = r0 + 2 * sm - lo;
            const int dbase = wrap1(r0 + m, nx);
            const double fe = outf ? __ldg(a.feq + j) : 0.0;
            const T* srow = stage + sbase * W + tid + HV;
            auto vstep = [&](int k) -> T {
                if (staged) {
                    const int2 info = rinfo[sbase + k];
                    if (info.x >= 0) {
                        T tv;
                        if constexpr (sizeof(T) == 4) tv = __int_as_float(info.y);
                        else tv = a.vsh[info.y].t;
                        const T* sr = srow + k * W + (info.x - HV);
                        const T corr = tabs[info.x * C + tid] + tv * tabs[(NM + info.x) * C + tid];
                        return lerp(sr[0], sr[1], tv) + corr;
                    }
                }
                const int grow = wrap1(gbase + k, nx);
                return v_cell<T, false>(a.h_in, a.feq, 0, nv, grow, j, a.vsh[grow]);
            };
            T o0 = vstep(0);
            const T o1 = vstep(1);
            T dp = lerp(o0, o1, t);
            o0 = o1;
            T* hout = next ? a.h_out + (size_t)r0 * nv + j : nullptr;
#pragma unroll
            for (int k = 2; k < R + 2; ++k) {
                const T on = vstep(k);
                const T dn = lerp(o0, on, t);
                if (outf) {
                    const int fr = wrap1(dbase + k - 2, nx);
                    const double f = fe + (double)dp;
                    if (a.f_hist_n != nullptr) a.f_hist_n[(size_t)fr * nv + j] = (T)f;
                    if (a.f_final != nullptr) a.f_final[(size_t)fr * nv + j] = f;
                }
                if (next) {
                    const T hv = lerp(dp, dn, t);
                    hout[(size_t)(k - 2) * nv] = hv;
                    acc[k - 2] += wj * hv;
                }
                o0 = on;
                dp = dn;
            }
        }
        __syncthreads();   // the next column block restages
    }

    if (a.part == nullptr || !next) return;
    store_row_partials<T, R>(acc, red, a.part + (size_t)blockIdx.y * nx + r0);
    if (a.counter == nullptr) return;
    if (!last_cta_done(a.counter, &s_last)) return;
    // the Poisson work area reuses the staging buffer (every thread of this CTA is past it)
    fwd_tail<T>(a, poisson_area<T>(a.P, smem + red_bytes), red);
    if (threadIdx.x == 0) *a.counter = 0u;
}

template <typename T, int R, int C>
static cudaError_t fwds_launch(const FwdArgs<T>& args, const LaunchCfg& c, cudaStream_t s) {
    // the column groups are the staged shape's (multiples of C), whatever the caller's args hold
    FwdArgs<T> a = args;
    a.chunk_cols = c.chunk_cols;
    a.n_chunks = c.n_chunks;
    if (a.chunk_cols < C || a.chunk_cols % C != 0 || a.nv % a.chunk_cols != 0) return cudaErrorInvalidValue;
    dim3 grid(a.nx / R, a.nv / a.chunk_cols);
    vp_fwds_kernel<T, R, C><<<grid, C, c.smem, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

#define VP_FWDS_C(RR)                                                             \
    if (c.R == RR) return c.threads == 256 ? fwds_launch<T, RR, 256>(a, c, s) :   \
                                             fwds_launch<T, RR, 128>(a, c, s);

template <typename T>
cudaError_t launch_fwd_staged(const FwdArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
    if (c.threads != 128 && c.threads != 256) return cudaErrorInvalidValue;
    VP_FWDS_C(4) VP_FWDS_C(8) VP_FWDS_C(16) VP_FWDS_C(32)
    return cudaErrorInvalidValue;
}
#undef VP_FWDS_C

size_t staged_smem_bytes(int span, int C, size_t real_size) {
    return real_size == 8 ? staged_bytes<double>(span, C) : staged_bytes<float>(span, C);
}

// ----------------------------------------------------------------------------------------------
// Staged adjoint step (PHASE 1 of vp_bwd_kernel, x-invariant f_eq). Per column block of C
// columns a CTA stages (a) the rows of w_n its columns' windows touch, [r0 - 2 max m - 2,
// r0 - 2 min m + R), with a 4-cell halo along v, each with its shift record (m, t) and rho
// cotangent; (b) its own R rows of h_{n-1} with the same halo and step n-1's shift records; (c) the
// f_eq slope tables B_m of its columns. Then each thread walks its column: gh = V^T w + rho^T,
// c = X^T gh (+ g_f_hist), w_{n-1} = X^T c, and the slope row sums for g_E_total of step n-1.
// Rows whose shift leaves the halo use the global-memory form of bwd_tile.
// ----------------------------------------------------------------------------------------------
template <typename T>
__host__ __device__ constexpr size_t staged_bwd_bytes(int span, int R, int C) {
    return (size_t)(span + R) * (C + 2 * kStageHalo) * sizeof(T) + (((size_t)(span + R) * 8 + 15) & ~(size_t)15) +
           (((size_t)span * sizeof(T) + 15) & ~(size_t)15) + (size_t)2 * kStageHalo * C * sizeof(T);
}

template <typename T, int R, int C>
__global__ void __launch_bounds__(C) vp_bwds_kernel(const BwdArgs<T> a) {
    using V = typename Vec16<T>::type;
    constexpr int VE = 16 / sizeof(T);
    constexpr int HV = kStageHalo;
    constexpr int W = C + 2 * HV;
    constexpr int PER_ROW = W / VE;
    constexpr int NM = 2 * HV;
    extern __shared__ __align__(16) unsigned char smem[];
    T* red = reinterpret_cast<T*>(smem);
    const size_t red_bytes = (((size_t)32 * R * sizeof(T)) + 15) & ~(size_t)15;
    const int span_max = a.stage_span;
    T* sw = reinterpret_cast<T*>(smem + red_bytes);               // [span_max][W]
    T* sh = sw + (size_t)span_max * W;                               // [R][W]
    int2* iw = reinterpret_cast<int2*>(sh + (size_t)R * W);          // [span_max]
    int2* ih = iw + span_max;                                        // [R]
    T* sg = reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(iw) +
                                 (((size_t)(span_max + R) * 8 + 15) & ~(size_t)15));   // [span_max]
    T* tabB = reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(sg) +
                                   (((size_t)span_max * sizeof(T) + 15) & ~(size_t)15));  // [NM][C]
    __shared__ int s_last, s_min, s_max;

    const int nx = a.nx, nv = a.nv;
    const int r0 = blockIdx.x * R;
    const int tid = threadIdx.x;
    const int g_begin = blockIdx.y * a.chunk_cols;
    const int g_end = min(nv, g_begin + a.chunk_cols);
    const T* vB = a.vtab + (size_t)NM * nv;

    T acc[R];
#pragma unroll
    for (int e = 0; e < R; ++e) acc[e] = T(0);

    for (int c0 = g_begin; c0 < g_end; c0 += C) {
        const int j = c0 + tid;
        const int m = __ldg(a.mx + j);
        const int sm = m > nx / 2 ? m - nx : m;
        int mn = sm, mxv = sm;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mxv = max(mxv, __shfl_xor_sync(0xffffffffu, mxv, o));
        }
        if (tid == 0) {
            s_min = mn;
            s_max = mxv;
        }
        __syncthreads();
        if ((tid & 31) == 0 && tid != 0) {
            atomicMin(&s_min, mn);
            atomicMax(&s_max, mxv);
        }
        __syncthreads();
        const int lo = r0 - 2 * s_max - 2;
        const int span = 2 * (s_max - s_min) + R + 2;
        const bool staged = span <= span_max;
        const int lo_w = wrapboth(lo, nx);   // signed offsets in (-nx/2, nx/2]: lo in [-nx-2, 2nx)
        if (staged) {
            for (int idx = tid; idx < (span + R) * PER_ROW; idx += C) {
                const int q = idx / PER_ROW, v = idx - q * PER_ROW;
                int col = c0 - HV + v * VE;
                col += col < 0 ? nv : 0;
                col -= col >= nv ? nv : 0;
                const T* src;
                if (q < span) {
                    int row = lo_w + q;
                    row -= row >= nx ? nx : 0;
                    src = a.w_in + (size_t)row * nv + col;
                } else {
                    src = a.h_prev + (size_t)(r0 + q - span) * nv + col;
                }
                const int dst_row = q < span ? q : span_max + (q - span);
                reinterpret_cast<V*>(sw + (size_t)dst_row * W)[v] = __ldg(reinterpret_cast<const V*>(src));
            }
            for (int q = tid; q < span + R; q += C) {
                int row;
                VShift<T> vs;
                if (q < span) {
                    row = lo_w + q;
                    row -= row >= nx ? nx : 0;
                    vs = a.vsh_n[row];
                    sg[q] = __ldg(a.grho + row);
                } else {
                    row = r0 + q - span;
                    vs = a.vsh_prev[row];
                }
                const int ms = vs.m >= nv / 2 ? vs.m - nv : vs.m;
                int2 info;
                info.x = (ms >= -HV && ms < HV) ? ms + HV : -1;
                if constexpr (sizeof(T) == 4) info.y = __float_as_int((float)vs.t);
                else info.y = row;
                if (q < span) iw[q] = info;
                else ih[q - span] = info;
            }
#pragma unroll
            for (int r = 0; r < NM; ++r) tabB[r * C + tid] = __ldg(vB + (size_t)r * nv + j);
        }
        __syncthreads();
        {
            const T t = __ldg(a.tx + j);
            const T wr = -a.dv * trap_w<T>(j, nv);
            const int sbase = 2 * (s_max - sm);            // staged row of gh[0]
            const int gbase = wrapneg2(r0 - 2 * m - 2, nx);
            const int cbase = wrapneg(r0 - m - 1, nx);
            auto ghstep = [&](int k) -> T {
                if (staged) {
                    const int2 info = iw[sbase + k];
                    if (info.x >= 0) {
                        T tv;
                        if constexpr (sizeof(T) == 4) tv = __int_as_float(info.y);
                        else tv = a.vsh_n[info.y].t;
                        const T* sr = sw + (size_t)(sbase + k) * W + tid + 2 * HV - info.x;
                        return lerp(sr[0], sr[-1], tv) + wr * sg[sbase + k];
                    }
                }
                const int row = wrap1(gbase + k, nx);
                const VShift<T> vs = a.vsh_n[row];
                const int cc0 = wrapneg(j - vs.m, nv);
                const int cc1 = wrapneg(cc0 - 1, nv);
                const T* wrow = a.w_in + (size_t)row * nv;
                return lerp(__ldg(wrow + cc0), __ldg(wrow + cc1), vs.t) + wr * __ldg(a.grho + row);
            };
            auto slope = [&](int e) -> T {
                if (staged) {
                    const int2 info = ih[e];
                    if (info.x >= 0) {
                        const T* hr = sh + (size_t)e * W + tid + info.x;   // column j + ms
                        return (hr[1] - hr[0]) + tabB[info.x * C + tid];
                    }
                }
                const int row = r0 + e;
                const VShift<T> vp = a.vsh_prev[row];
                const int d0 = wrap1(j + vp.m, nv);
                int d1 = d0 + 1;
                d1 = d1 == nv ? 0 : d1;
                const T* hr = a.h_prev + (size_t)row * nv;
                return (__ldg(hr + d1) - __ldg(hr + d0)) +
                       (T)(feq_at<T, false>(a.feq, 0, row, d1) - feq_at<T, false>(a.feq, 0, row, d0));
            };
            T g0 = ghstep(0);
            T g1 = ghstep(1);
            T cp = lerp(g1, g0, t);
            if (a.gfh != nullptr) cp += __ldg(a.gfh + (size_t)cbase * nv + j);
            g0 = g1;
            T* wout = a.w_out + (size_t)r0 * nv + j;
#pragma unroll
            for (int k = 2; k < R + 2; ++k) {
                const T gk = ghstep(k);
                T cn = lerp(gk, g0, t);
                if (a.gfh != nullptr) cn += __ldg(a.gfh + (size_t)wrap1(cbase + k - 1, nx) * nv + j);
                const T wv = lerp(cn, cp, t);
                wout[(size_t)(k - 2) * nv] = wv;
                acc[k - 2] += slope(k - 2) * wv;
                g0 = gk;
                cp = cn;
            }
        }
        __syncthreads();
    }

    store_row_partials<T, R>(acc, red, a.part + (size_t)blockIdx.y * nx + r0);
    if (a.counter == nullptr) return;
    if (!last_cta_done(a.counter, &s_last)) return;
    bwd_tail<T>(a, poisson_area<T>(a.P, smem + red_bytes));
    if (threadIdx.x == 0) *a.counter = 0u;
}

template <typename T, int R, int C>
static cudaError_t bwds_launch(const BwdArgs<T>& args, const LaunchCfg& c, cudaStream_t s) {
    BwdArgs<T> a = args;
    a.chunk_cols = c.chunk_cols;
    a.n_chunks = c.n_chunks;
    if (a.chunk_cols < C || a.chunk_cols % C != 0 || a.nv % a.chunk_cols != 0) return cudaErrorInvalidValue;
    dim3 grid(a.nx / R, a.nv / a.chunk_cols);
    vp_bwds_kernel<T, R, C><<<grid, C, c.smem, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

#define VP_BWDS_C(RR)                                                             \
    if (c.R == RR) return c.threads == 256 ? bwds_launch<T, RR, 256>(a, c, s) :   \
                                             bwds_launch<T, RR, 128>(a, c, s);

template <typename T>
cudaError_t launch_bwd_staged(const BwdArgs<T>& a, const LaunchCfg& c, cudaStream_t s) {
    if (c.threads != 128 && c.threads != 256) return cudaErrorInvalidValue;
    VP_BWDS_C(4) VP_BWDS_C(8) VP_BWDS_C(16) VP_BWDS_C(32)
    return cudaErrorInvalidValue;
}
#undef VP_BWDS_C

size_t staged_bwd_smem_bytes(int span, int R, int C, size_t real_size) {
    return real_size == 8 ? staged_bwd_bytes<double>(span, R, C) : staged_bwd_bytes<float>(span, R, C);
}

template <typename T>
cudaError_t set_staged_bwd_smem_limit(size_t bytes) {
#define VP_SET(R, C)                                                                                 \
    if (cudaError_t e = cudaFuncSetAttribute(vp_bwds_kernel<T, R, C>,                               \
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes); \
        e != cudaSuccess)                                                                           \
        return e;
    VP_SET(4, 128) VP_SET(8, 128) VP_SET(16, 128) VP_SET(32, 128)
    VP_SET(4, 256) VP_SET(8, 256) VP_SET(16, 256) VP_SET(32, 256)
#undef VP_SET
    return cudaSuccess;
}

template cudaError_t launch_bwd_staged<float>(const BwdArgs<float>&, const LaunchCfg&, cudaStream_t);
template cudaError_t launch_bwd_staged<double>(const BwdArgs<double>&, const LaunchCfg&, cudaStream_t);
template cudaError_t set_staged_bwd_smem_limit<float>(size_t);
template cudaError_t set_staged_bwd_smem_limit<double>(size_t);

template <typename T>
cudaError_t set_staged_smem_limit(size_t bytes) {
#define VP_SET(R, C)                                                                                 \
    if (cudaError_t e = cudaFuncSetAttribute(vp_fwds_kernel<T, R, C>,                               \
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes); \
        e != cudaSuccess)                                                                           \
        return e;
    VP_SET(4, 128) VP_SET(8, 128) VP_SET(16, 128) VP_SET(32, 128)
    VP_SET(4, 256) VP_SET(8, 256) VP_SET(16, 256) VP_SET(32, 256)
#undef VP_SET
    return cudaSuccess;
}

template cudaError_t launch_fwd_staged<float>(const FwdArgs<float>&, const LaunchCfg&, cudaStream_t);
template cudaError_t launch_fwd_staged<double>(const FwdArgs<double>&, const LaunchCfg&, cudaStream_t);
template cudaError_t set_staged_smem_limit<float>(size_t);
template cudaError_t set_staged_smem_limit<double>(size_t);

// ----------------------------------------------------------------------------------------------
// Launchers
// ----------------------------------------------------------------------------------------------

template <typename T, int R, bool F2>
static cudaError_t fwd_dispatch_phase(const FwdArgs<T>& a, const LaunchCfg& c, int phase,
                                      cudaStream_t s) {
    dim3 grid(a.nx / R, c.n_chunks);
    if (phase == 0)
        vp_fwd_kernel<T, R, F2, 0><<<grid, c.threads, c.smem, s>>>(a);
    else if (phase == 3)
        vp_fwd_kernel<T, R, F2, 3><<<grid, c.threads, c.smem, s>>>(a);
    else
        vp_fwd_kernel<T, R, F2, 1><<<grid, c.threads, c.smem, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

template <typename T, int R, bool F2>
static cudaError_t bwd_dispatch_phase(const BwdArgs<T>& a, const LaunchCfg& c, int phase,
                                      cudaStream_t s) {
    dim3 grid(a.nx / R, c.n_chunks);
    if (phase == 0)
        vp_bwd_kernel<T, R, F2, 0><<<grid, c.threads, c.smem, s>>>(a);
    else if (phase == 1)
        vp_bwd_kernel<T, R, F2, 1><<<grid, c.threads, c.smem, s>>>(a);
    else if (phase == 3)
        vp_bwd_kernel<T, R, F2, 3><<<grid, c.threads, c.smem, s>>>(a);
    else
        vp_bwd_kernel<T, R, F2, 2><<<grid, c.threads, c.smem, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

#define VP_R_SWITCH(FN, ...)                                              \
    switch (c.R) {                                                        \
        case 1: return FN<T, 1, F2>(__VA_ARGS__);                         \
        case 2: return FN<T, 2, F2>(__VA_ARGS__);                         \
        case 4: return FN<T, 4, F2>(__VA_ARGS__);                         \
        case 8: return FN<T, 8, F2>(__VA_ARGS__);                         \
        case 16: return FN<T, 16, F2>(__VA_ARGS__);                       \
        default: return cudaErrorInvalidValue;                            \
    }

template <typename T, bool F2>
static cudaError_t fwd_r(const FwdArgs<T>& a, const LaunchCfg& c, int phase, cudaStream_t s) {
    VP_R_SWITCH(fwd_dispatch_phase, a, c, phase, s)
}
template <typename T, bool F2>
static cudaError_t bwd_r(const BwdArgs<T>& a, const LaunchCfg& c, int phase, cudaStream_t s) {
    VP_R_SWITCH(bwd_dispatch_phase, a, c, phase, s)
}

template <typename T>
cudaError_t launch_fwd(const FwdArgs<T>& a, const LaunchCfg& c, int phase, bool feq2d,
                       cudaStream_t s) {
    return feq2d ? fwd_r<T, true>(a, c, phase, s) : fwd_r<T, false>(a, c, phase, s);
}

template <typename T>
cudaError_t launch_bwd(const BwdArgs<T>& a, const LaunchCfg& c, int phase, bool feq2d,
                       cudaStream_t s) {
    return feq2d ? bwd_r<T, true>(a, c, phase, s) : bwd_r<T, false>(a, c, phase, s);
}

// Sums the column-chunk partials of every row into chunk 0 (part[i] = sum over c of
// part[c*nx + i], c ascending: the order the tails use), so that the one-CTA tail reads nx values
// instead of n_chunks*nx. Used before a separate tail launch when there are many partials.
template <typename T>
__global__ void __launch_bounds__(256) vp_part_sum_kernel(T* part, int n_chunks, int nx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx) return;
    T s = __ldcg(part + i);
    int c = 1;
    for (; c + 8 <= n_chunks; c += 8) {
        T v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = __ldcg(part + (size_t)(c + u) * nx + i);
#pragma unroll
        for (int u = 0; u < 8; ++u) s += v[u];
    }
    for (; c < n_chunks; ++c) s += __ldcg(part + (size_t)c * nx + i);
    part[i] = s;
}

// Row partials above this count are pre-summed by vp_part_sum_kernel across many CTAs.
constexpr long long kTailPartialsDirect = 1 << 15;

template <typename T, typename Args>
static cudaError_t presum_partials(Args& a, cudaStream_t s) {
    if (a.part == nullptr || a.n_chunks <= 1 || (long long)a.n_chunks * a.nx <= kTailPartialsDirect)
        return cudaSuccess;
    vp_part_sum_kernel<T><<<(a.nx + 255) / 256, 256, 0, s>>>(a.part, a.n_chunks, a.nx);
    count_launch();
    a.n_chunks = 1;
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_fwd_tail(const FwdArgs<T>& args, int threads, size_t smem, bool tw_stage, cudaStream_t s) {
    FwdArgs<T> a = args;
    if (cudaError_t e = presum_partials<T>(a, s)) return e;
    a.P.tw_stage = tw_stage ? 1 : 0;
    vp_fwd_tail_kernel<T><<<1, threads, smem, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_bwd_tail(const BwdArgs<T>& args, int threads, size_t smem, bool tw_stage, cudaStream_t s) {
    BwdArgs<T> a = args;
    if (cudaError_t e = presum_partials<T>(a, s)) return e;
    a.P.tw_stage = tw_stage ? 1 : 0;
    vp_bwd_tail_kernel<T><<<1, threads, smem, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t set_tail_smem_limit(size_t bytes) {
    cudaError_t e = cudaFuncSetAttribute(vp_fwd_tail_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(vp_bwd_tail_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template cudaError_t launch_fwd_tail<float>(const FwdArgs<float>&, int, size_t, bool, cudaStream_t);
template cudaError_t launch_fwd_tail<double>(const FwdArgs<double>&, int, size_t, bool, cudaStream_t);
template cudaError_t launch_bwd_tail<float>(const BwdArgs<float>&, int, size_t, bool, cudaStream_t);
template cudaError_t launch_bwd_tail<double>(const BwdArgs<double>&, int, size_t, bool, cudaStream_t);
template cudaError_t set_tail_smem_limit<float>(size_t);
template cudaError_t set_tail_smem_limit<double>(size_t);

template cudaError_t launch_fwd<float>(const FwdArgs<float>&, const LaunchCfg&, int, bool, cudaStream_t);
template cudaError_t launch_fwd<double>(const FwdArgs<double>&, const LaunchCfg&, int, bool, cudaStream_t);
template cudaError_t launch_bwd<float>(const BwdArgs<float>&, const LaunchCfg&, int, bool, cudaStream_t);
template cudaError_t launch_bwd<double>(const BwdArgs<double>&, const LaunchCfg&, int, bool, cudaStream_t);

// ----------------------------------------------------------------------------------------------
// Ensembles: one persistent launch per time step advances every instance. CTAs stride over the
// instances' tiles (instances ordered longest first; a host-built map gives each tile's instance,
// first row and column chunk); the CTA that completes an instance's last tile runs that
// instance's Poisson tail. Per-tile arithmetic is fwd_tile / bwd_tile above.
// ----------------------------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ FwdArgs<T> batch_fwd_args(const BatchStep<T>& b, const BatchInst<T>& I) {
    FwdArgs<T> a{};
    const long long nn = (long long)I.nx * I.nv;
    a.nx = I.nx;
    a.nv = I.nv;
    a.n_chunks = I.n_chunks;
    a.chunk_cols = I.chunk_cols;
    a.mx = I.mx;
    a.tx = I.tx;
    a.tx64 = I.tx64;
    a.feq = I.feq;
    a.feq_rs = I.feq_rs;
    a.vtab = I.vtab;
    a.P = I.P;
    a.dv = I.dv;
    a.dx = I.dx;
    a.dtdv = I.dtdv;
    a.H = b.H + I.off_x;
    a.f_iv = b.f_iv ? b.f_iv + I.off_f : nullptr;
    a.h_in = b.c_in ? b.c_in + b.c_in_mul * I.off_f + (long long)b.c_in_step * nn : nullptr;
    a.h_out = b.c_out ? b.c_out + b.c_out_mul * I.off_f + (long long)b.c_out_step * nn : nullptr;
    a.vsh = b.vsh_in ? b.vsh_in + (long long)b.vsh_in_mul * I.off_x + (long long)b.vsh_in_step * I.nx : nullptr;
    a.vsh_out = b.vsh_out ? b.vsh_out + (long long)b.vsh_out_mul * I.off_x + (long long)b.vsh_out_step * I.nx : nullptr;
    a.E_out = b.E_out ? b.E_out + (long long)b.E_out_mul * I.off_x + (long long)b.E_out_step * I.nx : nullptr;
    a.f_final = b.f_final ? b.f_final + I.off_f : nullptr;
    a.f_hist_n = nullptr;
    a.E_hist_out = b.E_hist ? b.E_hist + (long long)b.n_steps * I.off_x + (long long)b.hist_step * I.nx : nullptr;
    a.ee_out = b.ee_hist ? b.ee_hist + (long long)I.index * b.n_steps + b.hist_step : nullptr;
    a.part = b.part + I.off_part;
    a.counter = b.counters + I.index;
    return a;
}

template <typename T>
__device__ __forceinline__ BwdArgs<T> batch_bwd_args(const BatchStep<T>& b, const BatchInst<T>& I) {
    BwdArgs<T> a{};
    const long long nn = (long long)I.nx * I.nv;
    a.nx = I.nx;
    a.nv = I.nv;
    a.n_chunks = I.n_chunks;
    a.chunk_cols = I.chunk_cols;
    a.mx = I.mx;
    a.tx = I.tx;
    a.feq = I.feq;
    a.feq_rs = I.feq_rs;
    a.vtab = I.vtab;
    a.P = I.P;
    a.dv = I.dv;
    a.dx = I.dx;
    a.neg_dt_dv = I.neg_dt_dv;
    a.w_in = b.c_in ? b.c_in + b.c_in_mul * I.off_f + (long long)b.c_in_step * nn : nullptr;
    a.w_out = b.c_out ? b.c_out + b.c_out_mul * I.off_f + (long long)b.c_out_step * nn : nullptr;
    a.grho = b.grho ? b.grho + I.off_x : nullptr;
    a.grho_out = b.grho_out ? b.grho_out + I.off_x : nullptr;
    a.vsh_n = b.vsh_in ? b.vsh_in + (long long)b.vsh_in_mul * I.off_x + (long long)b.vsh_in_step * I.nx : nullptr;
    a.h_prev = b.h_prev ? b.h_prev + (long long)b.n_steps * I.off_f + (long long)b.h_prev_step * nn : nullptr;
    a.vsh_prev = b.vsh_prev ? b.vsh_prev + (long long)b.n_steps * I.off_x + (long long)b.vsh_prev_step * I.nx : nullptr;
    a.E_prev = b.E_prev ? b.E_prev + (long long)b.n_steps * I.off_x + (long long)b.E_prev_step * I.nx : nullptr;
    a.gfh = nullptr;
    a.c_src = b.g_ff ? b.g_ff + I.off_f : nullptr;
    a.c_src2 = nullptr;
    a.gE_hist = b.g_Eh ? b.g_Eh + (long long)b.n_steps * I.off_x + (long long)b.g_step * I.nx : nullptr;
    a.gee = b.g_ee ? b.g_ee + (long long)I.index * b.n_steps + b.g_step : nullptr;
    a.gH = b.g_H + I.off_x;
    a.gfiv_out = b.g_fiv ? b.g_fiv + I.off_f : nullptr;
    a.part = b.part + I.off_part;
    a.counter = b.counters + I.index;
    return a;
}

template <typename T, int R, bool FEQ2D, int PHASE>
__global__ void __launch_bounds__(256) vp_batch_fwd_kernel(const BatchStep<T> b) {
    extern __shared__ __align__(16) unsigned char smem[];
    T* red = reinterpret_cast<T*>(smem);
    __shared__ int s_last;
    const size_t red_bytes = (((size_t)32 * R * sizeof(T)) + 15) & ~(size_t)15;
    for (int tile = blockIdx.x; tile < b.n_tiles; tile += gridDim.x) {
        const int4 tm = __ldg(b.tiles + tile);
        const BatchInst<T> I = b.inst[tm.x];
        const FwdArgs<T> a = batch_fwd_args<T>(b, I);
        const int r0 = tm.y, ch = tm.z, c_begin = ch * I.chunk_cols;
        const int c_end = min(I.nv, c_begin + I.chunk_cols);
        T acc[R];
#pragma unroll
        for (int e = 0; e < R; ++e) acc[e] = T(0);
        fwd_tile<T, R, FEQ2D, PHASE>(a, r0, c_begin, c_end, acc);
        if (PHASE == 0 || !b.last) {
            store_row_partials<T, R>(acc, red, a.part + (size_t)ch * I.nx + r0);
            if (last_unit_done(a.counter, (unsigned)I.n_tiles, &s_last)) {
                fwd_tail<T>(a, poisson_area<T>(a.P, smem + red_bytes), red);
                if (threadIdx.x == 0) *a.counter = 0u;
            }
        }
        __syncthreads();   // shared scratch is reused by the next tile
    }
}

template <typename T, int R, bool FEQ2D, int PHASE>
__global__ void __launch_bounds__(256) vp_batch_bwd_kernel(const BatchStep<T> b) {
    extern __shared__ __align__(16) unsigned char smem[];
    T* red = reinterpret_cast<T*>(smem);
    __shared__ int s_last;
    const size_t red_bytes = (((size_t)32 * R * sizeof(T)) + 15) & ~(size_t)15;
    for (int tile = blockIdx.x; tile < b.n_tiles; tile += gridDim.x) {
        const int4 tm = __ldg(b.tiles + tile);
        const BatchInst<T> I = b.inst[tm.x];
        const BwdArgs<T> a = batch_bwd_args<T>(b, I);
        const int r0 = tm.y, ch = tm.z, c_begin = ch * I.chunk_cols;
        const int c_end = min(I.nv, c_begin + I.chunk_cols);
        T acc[R];
#pragma unroll
        for (int e = 0; e < R; ++e) acc[e] = T(0);
        bwd_tile<T, R, FEQ2D, PHASE>(a, r0, c_begin, c_end, acc);
        if (PHASE != 2) {
            store_row_partials<T, R>(acc, red, a.part + (size_t)ch * I.nx + r0);
            if (last_unit_done(a.counter, (unsigned)I.n_tiles, &s_last)) {
                bwd_tail<T>(a, poisson_area<T>(a.P, smem + red_bytes));
                if (threadIdx.x == 0) *a.counter = 0u;
            }
        }
        __syncthreads();
    }
}

template <typename T, int R, bool F2>
static cudaError_t batch_fwd_phase(const BatchStep<T>& b, int phase, int grid, int threads, size_t smem,
                                   cudaStream_t s) {
    if (phase == 0)
        vp_batch_fwd_kernel<T, R, F2, 0><<<grid, threads, smem, s>>>(b);
    else
        vp_batch_fwd_kernel<T, R, F2, 1><<<grid, threads, smem, s>>>(b);
    count_launch();
    return cudaGetLastError();
}

template <typename T, int R, bool F2>
static cudaError_t batch_bwd_phase(const BatchStep<T>& b, int phase, int grid, int threads, size_t smem,
                                   cudaStream_t s) {
    if (phase == 0)
        vp_batch_bwd_kernel<T, R, F2, 0><<<grid, threads, smem, s>>>(b);
    else if (phase == 1)
        vp_batch_bwd_kernel<T, R, F2, 1><<<grid, threads, smem, s>>>(b);
    else
        vp_batch_bwd_kernel<T, R, F2, 2><<<grid, threads, smem, s>>>(b);
    count_launch();
    return cudaGetLastError();
}

#define VP_BATCH_R(FN, ...)                                                    \
    switch (R) {                                                               \
        case 1: return feq2d ? FN<T, 1, true>(__VA_ARGS__) : FN<T, 1, false>(__VA_ARGS__); \
        case 2: return feq2d ? FN<T, 2, true>(__VA_ARGS__) : FN<T, 2, false>(__VA_ARGS__); \
        case 4: return feq2d ? FN<T, 4, true>(__VA_ARGS__) : FN<T, 4, false>(__VA_ARGS__); \
        case 8: return feq2d ? FN<T, 8, true>(__VA_ARGS__) : FN<T, 8, false>(__VA_ARGS__); \
        default: return cudaErrorInvalidValue;                                 \
    }

template <typename T>
cudaError_t launch_batch_fwd(const BatchStep<T>& b, int R, int phase, bool feq2d, int grid,
                             int threads, size_t smem, cudaStream_t s) {
    VP_BATCH_R(batch_fwd_phase, b, phase, grid, threads, smem, s)
}

template <typename T>
cudaError_t launch_batch_bwd(const BatchStep<T>& b, int R, int phase, bool feq2d, int grid,
                             int threads, size_t smem, cudaStream_t s) {
    VP_BATCH_R(batch_bwd_phase, b, phase, grid, threads, smem, s)
}

template <typename K>
static int occ(K kernel, int threads, size_t smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// Resident CTAs per SM of the ensemble kernels (the persistent grid is this times the SM count).
template <typename T>
int batch_blocks_per_sm(int R, bool fwd, bool feq2d, int threads, size_t smem) {
#define VP_OCC(RR)                                                                                     \
    if (R == RR) {                                                                                     \
        if (fwd) return feq2d ? occ(vp_batch_fwd_kernel<T, RR, true, 1>, threads, smem)                 \
                              : occ(vp_batch_fwd_kernel<T, RR, false, 1>, threads, smem);               \
        return feq2d ? occ(vp_batch_bwd_kernel<T, RR, true, 1>, threads, smem)                          \
                     : occ(vp_batch_bwd_kernel<T, RR, false, 1>, threads, smem);                        \
    }
    VP_OCC(1) VP_OCC(2) VP_OCC(4) VP_OCC(8)
#undef VP_OCC
    return 0;
}

template cudaError_t launch_batch_fwd<float>(const BatchStep<float>&, int, int, bool, int, int, size_t, cudaStream_t);
template cudaError_t launch_batch_fwd<double>(const BatchStep<double>&, int, int, bool, int, int, size_t, cudaStream_t);
template cudaError_t launch_batch_bwd<float>(const BatchStep<float>&, int, int, bool, int, int, size_t, cudaStream_t);
template cudaError_t launch_batch_bwd<double>(const BatchStep<double>&, int, int, bool, int, int, size_t, cudaStream_t);
template int batch_blocks_per_sm<float>(int, bool, bool, int, size_t);
template int batch_blocks_per_sm<double>(int, bool, bool, int, size_t);

}  // namespace vpb
