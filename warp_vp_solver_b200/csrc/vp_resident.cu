// Cluster-resident forward and adjoint for grids whose state fits in the distributed shared
// memory of one thread-block cluster (up to 16 CTAs).
//
// One cluster runs the whole time loop of one instance in a single launch. CTA c of the cluster
// owns rows [c*RC, (c+1)*RC) of the (nx, nv) grid, full width, in shared memory. Thread t owns
// column j = t % NVP and the RPT consecutive rows g .. g+RPT-1 (g = c*RC + (t / NVP)*RPT) of that
// column. As in the per-step streaming kernels, a thread computes a whole Strang step for its
// rows from a window of the previous state: the x shift of column j is one number, so
//   o = V(h) + [V(f_eq) - f_eq]    on rows g+2m .. g+2m+RPT+1   (h read from the owning CTAs)
//   d = X(o) + [X(f_eq) - f_eq]    on rows g+m  .. g+m+RPT      (= f_{n+1} - f_eq)
//   h' = X(d) + [X(f_eq) - f_eq]   on rows g    .. g+RPT-1      (written to the own rows)
// and the row sums of h' give rho. One hardware cluster barrier per time step (barrier.cluster
// arrive/wait; no software spinning) publishes h' and rho; the state planes and the rho vector
// are double-buffered so that the next step never overwrites data another CTA may still read.
// The adjoint mirrors it with gathers (V^T + rho^T, X^T, X^T, dE/dE_total row sums).
//
// Poisson is evaluated in every CTA for all rows as the equivalent real circulant product
// E_i = sum_k c[(i-k) mod nx] rho_k with c = real(ifft(m)) built once per plan from the same
// spectral multiplier as the FFT path (warp_vp_solver/poisson.py:34-69): nx^2 multiply-adds
// spread over the CTA's threads with no block barrier inside, where an in-block FFT needs
// ~2*log2(nx) barriers. The per-step streaming kernels (vp_kernels.cu) and the standalone
// vp_poisson use the in-block radix-2 FFT.
//
// Every thread of every CTA executes the same sequence of cluster barriers: all loops and
// branches that contain a barrier depend only on kernel arguments.

#include <cooperative_groups.h>

#include "vp_device.cuh"

namespace cg = cooperative_groups;

namespace vpb {

// Shared-memory layout: three RC x nv planes, seven nx vectors, nx v shifts, the f_eq row and
// its first differences.
template <typename T> struct ResSmem {
    T* p0;
    T* p1;
    T* p2;
    T* vec0;         // nx: row sums from every CTA, even steps
    T* vec1;         // nx: row sums from every CTA, odd steps
    T* circ;         // nx: c = real(ifft(m))
    T* fld;          // nx: E (forward) or grho (adjoint), all rows
    T* aux;          // nx: H (forward) or g_E (adjoint)
    VShift<T>* vsh;  // nx: v shifts of the current step, all rows
    double* feq;     // nv: the f_eq row (x-invariant f_eq)
    T* dfeq;         // nv: f_eq[j+1] - f_eq[j] rounded from float64 (periodic)
    T* red;          // 32
    double* eep;     // 2 x 16 partial energies (read by CTA 0)
    T* own;          // RC: accumulated g_H of the own rows (adjoint)
};

__host__ __device__ inline size_t res_align(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline size_t res_smem_bytes(int nx, int nv, int RC, size_t rs) {
    size_t b = 0;
    b += res_align((size_t)RC * nv * rs) * 3;
    b += res_align((size_t)nx * rs) * 5;
    b += res_align((size_t)nx * (rs == 8 ? 16 : 8));
    b += res_align((size_t)nv * 8);
    b += res_align((size_t)nv * rs);
    b += res_align((size_t)32 * rs);
    b += res_align((size_t)32 * 8);
    b += res_align((size_t)RC * rs);
    return b;
}

template <typename T>
__device__ ResSmem<T> res_carve(unsigned char* smem, int nx, int nv, int RC) {
    ResSmem<T> s;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = smem + off;
        off += res_align(bytes);
        return p;
    };
    s.p0 = reinterpret_cast<T*>(take((size_t)RC * nv * sizeof(T)));
    s.p1 = reinterpret_cast<T*>(take((size_t)RC * nv * sizeof(T)));
    s.p2 = reinterpret_cast<T*>(take((size_t)RC * nv * sizeof(T)));
    s.vec0 = reinterpret_cast<T*>(take((size_t)nx * sizeof(T)));
    s.vec1 = reinterpret_cast<T*>(take((size_t)nx * sizeof(T)));
    s.circ = reinterpret_cast<T*>(take((size_t)nx * sizeof(T)));
    s.fld = reinterpret_cast<T*>(take((size_t)nx * sizeof(T)));
    s.aux = reinterpret_cast<T*>(take((size_t)nx * sizeof(T)));
    s.vsh = reinterpret_cast<VShift<T>*>(take((size_t)nx * sizeof(VShift<T>)));
    s.feq = reinterpret_cast<double*>(take((size_t)nv * sizeof(double)));
    s.dfeq = reinterpret_cast<T*>(take((size_t)nv * sizeof(T)));
    s.red = reinterpret_cast<T*>(take((size_t)32 * sizeof(T)));
    s.eep = reinterpret_cast<double*>(take((size_t)32 * sizeof(double)));
    s.own = reinterpret_cast<T*>(take((size_t)RC * sizeof(T)));
    return s;
}

// v shift from the total field, with a cheap path for the common |shift| < nv case.
template <typename T>
__device__ __forceinline__ VShift<T> res_vshift(T Et, T dtdv, int nv) {
    const T s = Et * dtdv;
    const T mf = vfloor(-s);
    VShift<T> v;
    v.t = -s - mf;
    if (mf >= T(-nv) && mf < T(nv)) {
        const int m = (int)mf;
        v.m = m < 0 ? m + nv : m;
        return v;
    }
    return make_vshift<T>(Et, dtdv, nv);
}

// V(f_eq) - f_eq at column j for a row with shift (m, t). For the usual sub-cell shifts
// (m = 0, or m = nv-1 i.e. -1) it is t*D[j] or -(1-t)*D[j-1] with D the first differences of
// f_eq rounded from float64; other shifts use the float64 values.
template <typename T, bool FEQ2D>
__device__ __forceinline__ T res_vcorr(const ResSmem<T>& S, const double* __restrict__ feq, int rs,
                                       int i, int j, int c0, int c1, const VShift<T> v, int nv) {
    if (!FEQ2D) {
        if (v.m == 0) return v.t * S.dfeq[j];
        if (v.m == nv - 1) return -(T(1) - v.t) * S.dfeq[c0];
        const double fj = S.feq[j];
        const double tt = (double)v.t;
        return (T)((1.0 - tt) * (S.feq[c0] - fj) + tt * (S.feq[c1] - fj));
    } else {
        const double fj = __ldg(feq + (size_t)i * rs + j);
        const double tt = (double)v.t;
        return (T)((1.0 - tt) * (__ldg(feq + (size_t)i * rs + c0) - fj) +
                   tt * (__ldg(feq + (size_t)i * rs + c1) - fj));
    }
}

// X(f_eq) - f_eq at (row i, column j) for an x-dependent f_eq.
__device__ __forceinline__ double res_xcorr(const double* __restrict__ feq, int rs, int nx, int i,
                                            int m, double t64, int j) {
    const int q0 = wrap1(i + m, nx), q1 = q0 + 1 == nx ? 0 : q0 + 1;
    const double fi = __ldg(feq + (size_t)i * rs + j);
    return (1.0 - t64) * (__ldg(feq + (size_t)q0 * rs + j) - fi) +
           t64 * (__ldg(feq + (size_t)q1 * rs + j) - fi);
}

// Row q (0 <= q < nx) of a plane distributed over the cluster with RC rows per CTA.
template <typename T, int RC>
__device__ __forceinline__ const T* res_row(cg::cluster_group& cl, const T* plane, int q, int nv,
                                            int me) {
    const int cta = q / RC;
    const int l = q - cta * RC;
    const T* base = (cta == me) ? plane : cl.map_shared_rank(plane, cta);
    return base + l * nv;
}

// Split cluster barrier: arrive (release: this thread's earlier shared/global writes become
// visible cluster-wide) ... wait (acquire). Work placed between the two overlaps the barrier;
// the global writes of the outputs go there so the release does not wait for them.
__device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Row sums of the plane `vals` (RC x nv, already weighted) for the CTA's own rows, written to
// vec[gr0 + r] of every CTA of the cluster. Starts with a block barrier; the caller's cluster
// barrier publishes the stores.
template <typename T, int RC>
__device__ __forceinline__ void res_rowsum_broadcast(cg::cluster_group& cluster, const T* vals,
                                                     T* vec, int nv, int gr0, int CN) {
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    for (int r = wid; r < RC; r += nw) {
        T s = T(0);
        for (int j = lane; j < nv; j += 32) s += vals[(size_t)r * nv + j];
        s = warp_sum(s);
        if (lane < CN) cluster.map_shared_rank(vec, lane)[gr0 + r] = s;
    }
}

// out[i] = sum_k c[(i-k) mod nx] x[k] (adjoint: c[(k-i) mod nx]) for the n_rows rows
// i = (first + r) mod nx, r < n_rows; a power-of-two group of tpr lanes per row. Starts and ends
// with a block barrier.
template <typename T>
__device__ __forceinline__ void res_circ_rows(const T* circ, const T* x, T* out, int nx, int first,
                                              int n_rows, bool adjoint) {
    __syncthreads();
    int tpr = 32;
    while (tpr > 1 && tpr * n_rows > (int)blockDim.x) tpr >>= 1;
    const int g = threadIdx.x % tpr;
    const int rows_per_pass = blockDim.x / tpr;
    const int passes = (n_rows + rows_per_pass - 1) / rows_per_pass;
    for (int p = 0; p < passes; ++p) {
        const int r = p * rows_per_pass + (int)threadIdx.x / tpr;
        const int i = wrap1(first + (r < n_rows ? r : 0), nx);
        T s = T(0);
        if (r < n_rows) {
            for (int k = g; k < nx; k += tpr) {
                int d = adjoint ? (k - i) : (i - k);
                d = wrapneg(d, nx);
                s += circ[d] * x[k];
            }
        }
        for (int o = tpr >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (r < n_rows && g == 0) out[i] = s;
    }
    __syncthreads();
}

template <typename T>
__device__ void res_init_tables(ResSmem<T>& S, const PoissonTables<T>& P, const double* feq,
                                bool feq2d, int nx, int nv) {
    for (int i = threadIdx.x; i < nx; i += blockDim.x) S.circ[i] = __ldg(P.circ + i);
    if (!feq2d) {
        for (int j = threadIdx.x; j < nv; j += blockDim.x) {
            const double f = __ldg(feq + j);
            S.feq[j] = f;
            S.dfeq[j] = (T)(__ldg(feq + (j + 1 == nv ? 0 : j + 1)) - f);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Forward
// ---------------------------------------------------------------------------------------------

// Poisson for step s on the rows this CTA's windows touch, their v shifts, the own rows'
// outputs and the partial energy of the own rows (summed by CTA 0 one barrier later).
// `rho_sum` holds the row sums of h_s from every CTA.
template <typename T>
__device__ void res_fwd_field(const ResFwdArgs<T>& a, ResSmem<T>& S, cg::cluster_group& cluster,
                              T* rho_sum, int s, int gr0, int RC, int me, int CN) {
    const int nx = a.nx, nv = a.nv;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) rho_sum[i] *= -a.dv;   // rho
    const int first = ((gr0 + a.win_lo) % nx + nx) % nx;
    res_circ_rows<T>(S.circ, rho_sum, S.fld, nx, first, a.win_n, false);
    for (int r = threadIdx.x; r < a.win_n; r += blockDim.x) {
        const int i = wrap1(first + r, nx);
        S.vsh[i] = res_vshift<T>(S.fld[i] + S.aux[i], a.dtdv, nv);
    }
    if (threadIdx.x < 32) {
        double e2 = 0.0;
        for (int r = threadIdx.x; r < RC; r += 32) {
            const int i = gr0 + r;
            const T E = S.fld[i];
            const T Et = E + S.aux[i];
            if (a.E_hist != nullptr) a.E_hist[(size_t)s * nx + i] = Et;
            if (a.E_tape != nullptr) a.E_tape[(size_t)s * nx + i] = E;
            if (a.vsh_tape != nullptr) a.vsh_tape[(size_t)s * nx + i] = res_vshift<T>(Et, a.dtdv, nv);
            e2 += (double)(trap_w<T>(i, nx) * E * E);
        }
        e2 = warp_sum(e2);
        if (threadIdx.x == 0) cluster.map_shared_rank(S.eep, 0)[(s & 1) * 16 + me] = e2;
    }
    // CTA 0: energy of step s-1, whose partials were published by the last cluster barrier
    if (me == 0 && threadIdx.x == 0 && s >= 1 && a.ee_hist != nullptr) {
        double tot = 0.0;
        for (int c = 0; c < CN; ++c) tot += S.eep[((s - 1) & 1) * 16 + c];
        a.ee_hist[s - 1] = (T)(0.5 * tot * (double)a.dx);
    }
    __syncthreads();
}

template <typename T, int RC, int RPT, bool FEQ2D>
__global__ void __launch_bounds__(1024) vp_res_fwd_kernel(const ResFwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int nx = a.nx, nv = a.nv;
    const int me = (int)cluster.block_rank();
    const int CN = (int)cluster.num_blocks();
    const int gr0 = me * RC;
    constexpr int G = RC / RPT;
    const int NVP = blockDim.x / G;
    const int j = threadIdx.x % NVP;
    const int rt = (threadIdx.x / NVP) * RPT;   // first own row of this thread (CTA-local)
    const int g = gr0 + rt;                      // first own row of this thread (global)
    const bool colv = j < nv;
    ResSmem<T> S = res_carve<T>(smem, nx, nv, RC);
    T* Hb[2] = {S.p0, S.p1};   // h of even / odd steps, own rows (read remotely)
    T* Wt = S.p2;              // weighted h' for the row sums
    res_init_tables<T>(S, a.P, a.feq, FEQ2D, nx, nv);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) S.aux[i] = __ldg(a.H + i);

    // per-column constants of the x half-step
    int m = 0;
    T t = T(0), wj = T(0);
    double t64 = 0.0, feq_j = 0.0;
    if (colv) {
        m = __ldg(a.mx + j);
        t = __ldg(a.tx + j);
        t64 = __ldg(a.tx64 + j);
        wj = trap_w<T>(j, nv);
        feq_j = FEQ2D ? 0.0 : __ldg(a.feq + j);
    }
    __syncthreads();

    // ---- prologue: h_0 = X(f_iv - f_eq) + corr for the own rows, straight from global memory ----
    if (colv) {
        T d[RPT + 1];
        const int base = wrap1(g + m, nx);
#pragma unroll
        for (int k = 0; k <= RPT; ++k) {
            const int q = wrap1(base + k, nx);
            const double fe = FEQ2D ? __ldg(a.feq + (size_t)q * a.feq_rs + j) : feq_j;
            d[k] = (T)(__ldg(a.f_iv + (size_t)q * nv + j) - fe);
        }
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            const int i = g + k;
            T h = lerp(d[k], d[k + 1], t);
            if (FEQ2D) h += (T)res_xcorr(a.feq, a.feq_rs, nx, i, m, t64, j);
            Hb[0][(size_t)(rt + k) * nv + j] = h;
            Wt[(size_t)(rt + k) * nv + j] = wj * h;
            if (a.h_tape != nullptr) a.h_tape[(size_t)i * nv + j] = h;
        }
    }
    res_rowsum_broadcast<T, RC>(cluster, Wt, S.vec0, nv, gr0, CN);
    cluster.sync();
    res_fwd_field<T>(a, S, cluster, S.vec0, 0, gr0, RC, me, CN);

    for (int n = 0; n < a.n_steps; ++n) {
        const T* cur = Hb[n & 1];
        T* nxt = Hb[(n + 1) & 1];
        const bool last = (n == a.n_steps - 1);
        T d[RPT + 1];
        T hv[RPT];
        int dq = 0;
        if (colv) {
            // o on rows g+2m .. g+2m+RPT+1 (h of those rows, from the owning CTAs)
            T o[RPT + 2];
            const int q0 = wrap2(g + 2 * m, nx);
            if (q0 >= gr0 && q0 + RPT + 1 < gr0 + RC) {
                // the whole window lies in this CTA: plain shared-memory loads
#pragma unroll
                for (int k = 0; k < RPT + 2; ++k) {
                    const int q = q0 + k;
                    const VShift<T> v = S.vsh[q];
                    const T* hr = cur + (q - gr0) * nv;
                    const int c0 = wrap1(j + v.m, nv);
                    const int c1 = c0 + 1 == nv ? 0 : c0 + 1;
                    o[k] = lerp(hr[c0], hr[c1], v.t) + res_vcorr<T, FEQ2D>(S, a.feq, a.feq_rs, q, j, c0, c1, v, nv);
                }
            } else {
#pragma unroll
                for (int k = 0; k < RPT + 2; ++k) {
                    const int q = wrap1(q0 + k, nx);
                    const VShift<T> v = S.vsh[q];
                    const T* hr = res_row<T, RC>(cluster, cur, q, nv, me);
                    const int c0 = wrap1(j + v.m, nv);
                    const int c1 = c0 + 1 == nv ? 0 : c0 + 1;
                    o[k] = lerp(hr[c0], hr[c1], v.t) + res_vcorr<T, FEQ2D>(S, a.feq, a.feq_rs, q, j, c0, c1, v, nv);
                }
            }
            // d on rows g+m .. g+m+RPT (= f_{n+1} - f_eq)
            dq = wrap1(g + m, nx);
#pragma unroll
            for (int k = 0; k <= RPT; ++k) {
                d[k] = lerp(o[k], o[k + 1], t);
                if (FEQ2D) d[k] += (T)res_xcorr(a.feq, a.feq_rs, nx, wrap1(dq + k, nx), m, t64, j);
            }
            if (!last) {
#pragma unroll
                for (int k = 0; k < RPT; ++k) {
                    T h = lerp(d[k], d[k + 1], t);
                    if (FEQ2D) h += (T)res_xcorr(a.feq, a.feq_rs, nx, g + k, m, t64, j);
                    hv[k] = h;
                    nxt[(rt + k) * nv + j] = h;
                    Wt[(rt + k) * nv + j] = wj * h;
                }
            }
        }
        T* rs = ((n + 1) & 1) ? S.vec1 : S.vec0;
        if (!last) res_rowsum_broadcast<T, RC>(cluster, Wt, rs, nv, gr0, CN);
        cluster_arrive();
        // outputs to global memory, overlapped with the barrier
        if (colv) {
            if (a.f_hist != nullptr || (a.f_final != nullptr && last)) {
#pragma unroll
                for (int k = 0; k < RPT; ++k) {
                    const int q = wrap1(dq + k, nx);
                    const double fe = FEQ2D ? __ldg(a.feq + (size_t)q * a.feq_rs + j) : feq_j;
                    const double f = fe + (double)d[k];
                    if (a.f_hist != nullptr) a.f_hist[((size_t)n * nx + q) * nv + j] = (T)f;
                    if (a.f_final != nullptr && last) a.f_final[(size_t)q * nv + j] = f;
                }
            }
            if (!last && a.h_tape != nullptr) {
#pragma unroll
                for (int k = 0; k < RPT; ++k) a.h_tape[((size_t)(n + 1) * nx + g + k) * nv + j] = hv[k];
            }
        }
        cluster_wait();
        if (!last) res_fwd_field<T>(a, S, cluster, rs, n + 1, gr0, RC, me, CN);
    }
    // energy of the last step (its partials were stored before the last barrier)
    if (me == 0 && threadIdx.x == 0 && a.ee_hist != nullptr) {
        const int s = a.n_steps - 1;
        double tot = 0.0;
        for (int c = 0; c < CN; ++c) tot += S.eep[(s & 1) * 16 + c];
        a.ee_hist[s] = (T)(0.5 * tot * (double)a.dx);
    }
}

// ---------------------------------------------------------------------------------------------
// Adjoint
// ---------------------------------------------------------------------------------------------

// Tail of the adjoint for step s (every CTA, all rows): g_E_total = -dt/dv * rowsum + g_E_hist[s];
// g_H += g_E_total (own rows); g_E = g_E_total + ee^T; grho = Poisson^T(g_E) (all rows); the v
// shifts of step s (all rows).
template <typename T>
__device__ void res_bwd_field(const ResBwdArgs<T>& a, ResSmem<T>& S, const T* sums, int s, int gr0,
                              int RC) {
    const int nx = a.nx;
    const T gee = a.g_ee != nullptr ? __ldg(a.g_ee + s) : T(0);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        T gEt = a.neg_dt_dv * sums[i];
        if (a.g_Eh != nullptr) gEt += __ldg(a.g_Eh + (size_t)s * nx + i);
        if (i >= gr0 && i < gr0 + RC) S.own[i - gr0] += gEt;
        S.aux[i] = gEt + a.dx * trap_w<T>(i, nx) * __ldg(a.E_tape + (size_t)s * nx + i) * gee;
    }
    const int first = ((gr0 + a.win_lo) % nx + nx) % nx;
    for (int r = threadIdx.x; r < a.win_n; r += blockDim.x) {
        const int i = wrap1(first + r, nx);
        S.vsh[i] = a.vsh_tape[(size_t)s * nx + i];
    }
    res_circ_rows<T>(S.circ, S.aux, S.fld, nx, first, a.win_n, true);
}

// w on the own rows g .. g+RPT-1 from c on rows g-m-1 .. g-m+RPT-1 (held in registers), the
// slope * w products for the dE row sums (needs h and the v shifts of step np).
template <typename T, int RPT, bool FEQ2D>
__device__ __forceinline__ void res_bwd_w(const ResBwdArgs<T>& a, const ResSmem<T>& S,
                                          const T (&c)[RPT + 1], T* nxt, T* Wt, int np, int g,
                                          int rt, int j, T t) {
    const int nx = a.nx, nv = a.nv;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        const int i = g + k;
        const T wv = lerp(c[k + 1], c[k], t);
        nxt[(size_t)(rt + k) * nv + j] = wv;
        const VShift<T> vp = a.vsh_tape[(size_t)np * nx + i];
        const int d0 = wrap1(j + vp.m, nv);
        const int d1 = d0 + 1 == nv ? 0 : d0 + 1;
        const T* hr = a.h_tape + ((size_t)np * nx + i) * nv;
        T sl = __ldg(hr + d1) - __ldg(hr + d0);
        if (FEQ2D)
            sl += (T)(__ldg(a.feq + (size_t)i * a.feq_rs + d1) - __ldg(a.feq + (size_t)i * a.feq_rs + d0));
        else
            sl += S.dfeq[d0];
        Wt[(size_t)(rt + k) * nv + j] = sl * wv;
    }
}

template <typename T, int RC, int RPT, bool FEQ2D>
__global__ void __launch_bounds__(1024) vp_res_bwd_kernel(const ResBwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int nx = a.nx, nv = a.nv, T_steps = a.n_steps;
    const int me = (int)cluster.block_rank();
    const int CN = (int)cluster.num_blocks();
    const int gr0 = me * RC;
    constexpr int G = RC / RPT;
    const int NVP = blockDim.x / G;
    const int j = threadIdx.x % NVP;
    const int rt = (threadIdx.x / NVP) * RPT;
    const int g = gr0 + rt;
    const bool colv = j < nv;
    ResSmem<T> S = res_carve<T>(smem, nx, nv, RC);
    T* Wb[2] = {S.p0, S.p1};   // cotangent on the v-step output of even / odd steps, own rows
    T* Wt = S.p2;              // slope * w for the row sums
    res_init_tables<T>(S, a.P, a.feq, FEQ2D, nx, nv);
    for (int r = threadIdx.x; r < RC; r += blockDim.x) S.own[r] = T(0);
    int m = 0;
    T t = T(0), wr = T(0);
    if (colv) {
        m = __ldg(a.mx + j);
        t = __ldg(a.tx + j);
        wr = -a.dv * trap_w<T>(j, nv);   // rho^T weight (warp_vp_solver/kernels.py:292-299)
    }
    __syncthreads();

    // ---- prologue (n = T): c = g_f_final + g_f_hist[T-1] on rows g-m-1 .. g-m+RPT-1 ----
    {
        T* nxt = Wb[(T_steps - 1) & 1];
        if (colv) {
            T c[RPT + 1];
            int base = (g - m - 1) % nx;
            base = wrapneg(base, nx);
#pragma unroll
            for (int k = 0; k <= RPT; ++k) {
                const int q = wrap1(base + k, nx);
                T v = T(0);
                if (a.g_ff != nullptr) v += __ldg(a.g_ff + (size_t)q * nv + j);
                if (a.g_fh != nullptr) v += __ldg(a.g_fh + ((size_t)(T_steps - 1) * nx + q) * nv + j);
                c[k] = v;
            }
            res_bwd_w<T, RPT, FEQ2D>(a, S, c, nxt, Wt, T_steps - 1, g, rt, j, t);
        }
        T* rs = ((T_steps - 1) & 1) ? S.vec1 : S.vec0;
        res_rowsum_broadcast<T, RC>(cluster, Wt, rs, nv, gr0, CN);
        cluster.sync();
        res_bwd_field<T>(a, S, rs, T_steps - 1, gr0, RC);
    }

    for (int n = T_steps - 1; n >= 0; --n) {
        const T* cur = Wb[n & 1];
        T* nxt = Wb[(n + 1) & 1];   // == Wb[(n-1) & 1]
        if (colv) {
            // gh = V^T(w_n) + rho^T(grho_n) on rows g-2m-2 .. g-2m+RPT-1 (w read from the owners)
            const int ng = n == 0 ? RPT + 1 : RPT + 2;   // rows of gh needed
            T gh[RPT + 2];
            int base = (g - (n == 0 ? 1 : 2) * m - (n == 0 ? 1 : 2)) % nx;
            base = wrapneg(base, nx);
#pragma unroll
            for (int k = 0; k < RPT + 2; ++k) {
                if (k < ng) {
                    const int q = wrap1(base + k, nx);
                    const VShift<T> v = S.vsh[q];
                    const T* wrow = res_row<T, RC>(cluster, cur, q, nv, me);
                    const int c0 = wrapneg(j - v.m, nv);
                    const int c1 = wrapneg(c0 - 1, nv);
                    gh[k] = lerp(wrow[c0], wrow[c1], v.t) + wr * S.fld[q];
                }
            }
            if (n == 0) {
                // gradient on f_iv: c on the own rows from gh on rows g-m-1 .. g-m+RPT-1
#pragma unroll
                for (int k = 0; k < RPT; ++k) a.g_fiv[(size_t)(g + k) * nv + j] = lerp(gh[k + 1], gh[k], t);
            } else {
                // c on rows g-m-1 .. g-m+RPT-1 (+ g_f_hist[n-1]), then w_{n-1} on the own rows
                T c[RPT + 1];
                int cb = (g - m - 1) % nx;
                cb = wrapneg(cb, nx);
#pragma unroll
                for (int k = 0; k <= RPT; ++k) {
                    c[k] = lerp(gh[k + 1], gh[k], t);
                    if (a.g_fh != nullptr)
                        c[k] += __ldg(a.g_fh + ((size_t)(n - 1) * nx + wrap1(cb + k, nx)) * nv + j);
                }
                res_bwd_w<T, RPT, FEQ2D>(a, S, c, nxt, Wt, n - 1, g, rt, j, t);
            }
        }
        T* rs = ((n - 1) & 1) ? S.vec1 : S.vec0;
        if (n > 0) res_rowsum_broadcast<T, RC>(cluster, Wt, rs, nv, gr0, CN);
        cluster_arrive();
        cluster_wait();
        if (n > 0) res_bwd_field<T>(a, S, rs, n - 1, gr0, RC);
    }
    for (int r = threadIdx.x; r < RC; r += blockDim.x) a.g_H[gr0 + r] = S.own[r];
}

// ---------------------------------------------------------------------------------------------
// Host-side launch helpers
// ---------------------------------------------------------------------------------------------

// Rows per thread for RC rows per CTA: the fewest (most threads) that keep the CTA at <= 1024
// threads, and at least RC/8 (at most 8 row groups).
int res_rows_per_thread(int RC, int nv) {
    const int nvp = ((nv + 31) / 32) * 32;
    int rpt = RC;
    while (rpt > 1 && rpt > RC / 8 && (RC / (rpt / 2)) * nvp <= 1024) rpt /= 2;
    return rpt;
}

int res_threads(int RC, int nv) {
    const int nvp = ((nv + 31) / 32) * 32;
    return (RC / res_rows_per_thread(RC, nv)) * nvp;
}

template <typename T, int RC, int RPT, bool F2>
static cudaError_t res_prepare_one(size_t smem) {
    cudaError_t e;
    e = cudaFuncSetAttribute(vp_res_fwd_kernel<T, RC, RPT, F2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(vp_res_bwd_kernel<T, RC, RPT, F2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(vp_res_fwd_kernel<T, RC, RPT, F2>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(vp_res_bwd_kernel<T, RC, RPT, F2>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

static cudaLaunchConfig_t res_cfg(int cn, int threads, size_t smem, cudaStream_t s, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cn, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cn;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

template <typename T, int RC, int RPT, bool F2>
static int res_max_clusters_rc(int cn, int threads, size_t smem) {
    if (res_prepare_one<T, RC, RPT, F2>(smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = res_cfg(cn, threads, smem, nullptr, attr);
    int n1 = 0, n2 = 0;
    if (cudaOccupancyMaxActiveClusters(&n1, vp_res_fwd_kernel<T, RC, RPT, F2>, &cfg) != cudaSuccess ||
        cudaOccupancyMaxActiveClusters(&n2, vp_res_bwd_kernel<T, RC, RPT, F2>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n1 < n2 ? n1 : n2;
}

template <typename T, int RC, int RPT, bool F2>
static cudaError_t res_launch_rc(bool fwd, const void* args, int cn, int threads, size_t smem, cudaStream_t s) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = res_cfg(cn, threads, smem, s, attr);
    cudaError_t e = fwd ? cudaLaunchKernelEx(&cfg, vp_res_fwd_kernel<T, RC, RPT, F2>, *static_cast<const ResFwdArgs<T>*>(args))
                        : cudaLaunchKernelEx(&cfg, vp_res_bwd_kernel<T, RC, RPT, F2>, *static_cast<const ResBwdArgs<T>*>(args));
    count_launch();
    return e;
}

bool res_rows_supported(int rc) { return rc == 1 || rc == 2 || rc == 4 || rc == 8 || rc == 16 || rc == 32; }

// (RC, RPT) instantiations reachable from res_rows_per_thread (RPT in [RC/8, RC]).
#define VP_RES_ONE(FN, R, P, F2V, ...) \
    if (RC == R && RPT == P) return F2V ? FN<T, R, P, true>(__VA_ARGS__) : FN<T, R, P, false>(__VA_ARGS__);
#define VP_RES_CASES(FN, F2V, ...)                                                            \
    VP_RES_ONE(FN, 1, 1, F2V, __VA_ARGS__) VP_RES_ONE(FN, 2, 1, F2V, __VA_ARGS__)             \
    VP_RES_ONE(FN, 2, 2, F2V, __VA_ARGS__) VP_RES_ONE(FN, 4, 1, F2V, __VA_ARGS__)             \
    VP_RES_ONE(FN, 4, 2, F2V, __VA_ARGS__) VP_RES_ONE(FN, 4, 4, F2V, __VA_ARGS__)             \
    VP_RES_ONE(FN, 8, 1, F2V, __VA_ARGS__) VP_RES_ONE(FN, 8, 2, F2V, __VA_ARGS__)             \
    VP_RES_ONE(FN, 8, 4, F2V, __VA_ARGS__) VP_RES_ONE(FN, 8, 8, F2V, __VA_ARGS__)             \
    VP_RES_ONE(FN, 16, 2, F2V, __VA_ARGS__) VP_RES_ONE(FN, 16, 4, F2V, __VA_ARGS__)           \
    VP_RES_ONE(FN, 16, 8, F2V, __VA_ARGS__) VP_RES_ONE(FN, 16, 16, F2V, __VA_ARGS__)          \
    VP_RES_ONE(FN, 32, 4, F2V, __VA_ARGS__) VP_RES_ONE(FN, 32, 8, F2V, __VA_ARGS__)           \
    VP_RES_ONE(FN, 32, 16, F2V, __VA_ARGS__) VP_RES_ONE(FN, 32, 32, F2V, __VA_ARGS__)

template <typename T>
int res_max_clusters(bool feq2d, int cn, int RC, int nv, size_t smem) {
    const int RPT = res_rows_per_thread(RC, nv);
    const int threads = res_threads(RC, nv);
    if (threads > 1024) return 0;
    VP_RES_CASES(res_max_clusters_rc, feq2d, cn, threads, smem)
    return 0;
}

template <typename T>
cudaError_t launch_res_fwd(const ResFwdArgs<T>& a, bool feq2d, int cn, int threads, size_t smem,
                           cudaStream_t s) {
    const int RC = a.Rc;
    const int RPT = res_rows_per_thread(RC, a.nv);
    VP_RES_CASES(res_launch_rc, feq2d, true, &a, cn, threads, smem, s)
    return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_res_bwd(const ResBwdArgs<T>& a, bool feq2d, int cn, int threads, size_t smem,
                           cudaStream_t s) {
    const int RC = a.Rc;
    const int RPT = res_rows_per_thread(RC, a.nv);
    VP_RES_CASES(res_launch_rc, feq2d, false, &a, cn, threads, smem, s)
    return cudaErrorInvalidValue;
}

size_t res_smem_size(int nx, int nv, int Rc, size_t real_size) {
    return res_smem_bytes(nx, nv, Rc, real_size);
}

template int res_max_clusters<float>(bool, int, int, int, size_t);
template int res_max_clusters<double>(bool, int, int, int, size_t);
template cudaError_t launch_res_fwd<float>(const ResFwdArgs<float>&, bool, int, int, size_t, cudaStream_t);
template cudaError_t launch_res_fwd<double>(const ResFwdArgs<double>&, bool, int, int, size_t, cudaStream_t);
template cudaError_t launch_res_bwd<float>(const ResBwdArgs<float>&, bool, int, int, size_t, cudaStream_t);
template cudaError_t launch_res_bwd<double>(const ResBwdArgs<double>&, bool, int, int, size_t, cudaStream_t);

}  // namespace vpb
