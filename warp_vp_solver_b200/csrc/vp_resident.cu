// Cluster-resident forward and adjoint for grids whose state fits in the distributed shared
// memory of one thread-block cluster (up to 16 CTAs).
//
// One cluster runs the whole time loop of one instance in a single launch. CTA c of the cluster
// owns rows [c*RC, (c+1)*RC) of the (nx, nv) grid, full width, in shared memory. Thread t owns
// column j = t % NVP and the RPT consecutive rows g .. g+RPT-1 (g = c*RC + (t / NVP)*RPT) of that
// column. As in the per-step streaming kernels, a thread computes a whole Strang step for its
// rows from a window of the previous state: the x shift of column j is one number, so
//   o = V(h) + [V(f_eq) - f_eq]    on rows g+2m .. g+2m+RPT+1   (own rows or the halo copy)
//   d = X(o) + [X(f_eq) - f_eq]    on rows g+m  .. g+m+RPT      (= f_{n+1} - f_eq)
//   h' = X(d) + [X(f_eq) - f_eq]   on rows g    .. g+RPT-1      (written to the own rows)
// and the row sums of h' give rho. One hardware cluster barrier per time step (barrier.cluster
// arrive/wait; no software spinning) publishes h' and rho; the state planes and the rho vector
// are double-buffered so that the next step never overwrites data another CTA may still read.
// The adjoint mirrors it with gathers (V^T + rho^T, X^T, X^T, dE/dE_total row sums).
//
// Poisson is evaluated in every CTA, for its own and halo rows, as the equivalent real circulant product
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

// Halo rows. CTA c keeps, besides its own rows, the rows [gr0 - h_lo, gr0) and
// [gr0 + RC, gr0 + RC + h_hi) (mod nx) of the state plane it reads in a step: the windows of the
// forward (rows g + 2m .. g + 2m + RPT + 1) and of the adjoint (rows g - 2m - 2 .. g - 2m + RPT - 1)
// for every column's x offset m in [mx_lo, mx_hi] lie inside. The halo is filled from the owning
// CTAs once per step, right after the cluster barrier that publishes the plane (coalesced 16-byte
// distributed-shared-memory loads), so that the step itself reads shared memory of its own CTA
// only. Plane row l holds global row gr0 - h_lo + l (mod nx); the own rows are l in
// [h_lo, h_lo + RC). The per-row field values and v shifts use the same local row index.

// Shared-memory layout: two state planes of W = h_lo + RC + h_hi rows, the row-partial plane,
// the nx vectors, the per-row field and v shifts of the W rows, the f_eq row and its first
// differences.
template <typename T> struct ResSmem {
    T* p0;
    T* p1;
    T* p2;           // row partials of the warps: [RC][NVP/32]
    T* vec0;         // nx: row sums of every CTA, gathered after the step's cluster barrier
    T* vec1;         // 2 x RC: this CTA's own row sums, step parity (read by the other CTAs)
    T* ctab;         // 3 nx + 16: ctab[j] = c[(j - nx - 8) mod nx], c = real(ifft(m))
    T* fld;          // W: E (forward) or grho (adjoint) of the local rows
    T* aux;          // nx: H (forward) or g_E (adjoint), global row index
    VShift<T>* vsh;  // W: v shifts of the current step, local rows
    double* feq;     // nv: the f_eq row (x-invariant f_eq)
    T* dfeq;         // nv: f_eq[j+1] - f_eq[j] rounded from float64 (periodic)
    double* eep;     // 4 partial energies of the own rows (step s in slot s % 4; read by CTA 0)
    T* own;          // RC: accumulated g_H of the own rows (adjoint)
    T* po;           // W rows: the v step of the current plane (forward: o), computed once per row
};

__host__ __device__ inline size_t res_align(size_t x) { return (x + 15) & ~(size_t)15; }

// Launch bound of the resident kernels by rows per thread: 1024 threads, or 512 from 8 rows per
// thread up (their register arrays need more than the 64 registers a 1024-thread CTA allows).
__host__ __device__ constexpr int res_max_threads(int rpt) { return rpt >= 8 ? 512 : 1024; }

// po: with the plane of phase-A results (forward float32 with an x-invariant f_eq).
__host__ __device__ inline size_t res_smem_bytes(int nx, int nv, int RC, int W, size_t rs, bool po) {
    size_t b = 0;
    b += res_align((size_t)W * nv * rs) * 2;
    b += res_align((size_t)RC * nv * rs);
    b += res_align((size_t)nx * rs) * 3;
    b += res_align((size_t)(3 * nx + 16) * rs);
    b += res_align((size_t)W * rs);
    b += res_align((size_t)W * (rs == 8 ? 16 : 8));
    b += res_align((size_t)nv * 8);
    b += res_align((size_t)nv * rs);
    b += res_align((size_t)4 * 8);
    b += res_align((size_t)RC * rs);
    if (po) b += res_align((size_t)W * nv * rs);
    return b;
}

template <typename T>
__device__ ResSmem<T> res_carve(unsigned char* smem, int nx, int nv, int RC, int W, bool po) {
    ResSmem<T> s;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = smem + off;
        off += res_align(bytes);
        return p;
    };
    s.p0 = reinterpret_cast<T*>(take((size_t)W * nv * sizeof(T)));
    s.p1 = reinterpret_cast<T*>(take((size_t)W * nv * sizeof(T)));
    s.p2 = reinterpret_cast<T*>(take((size_t)RC * nv * sizeof(T)));
    s.vec0 = reinterpret_cast<T*>(take((size_t)nx * sizeof(T)));
    s.vec1 = reinterpret_cast<T*>(take((size_t)nx * sizeof(T)));
    s.aux = reinterpret_cast<T*>(take((size_t)nx * sizeof(T)));
    s.ctab = reinterpret_cast<T*>(take((size_t)(3 * nx + 16) * sizeof(T)));
    s.fld = reinterpret_cast<T*>(take((size_t)W * sizeof(T)));
    s.vsh = reinterpret_cast<VShift<T>*>(take((size_t)W * sizeof(VShift<T>)));
    s.feq = reinterpret_cast<double*>(take((size_t)nv * sizeof(double)));
    s.dfeq = reinterpret_cast<T*>(take((size_t)nv * sizeof(T)));
    s.eep = reinterpret_cast<double*>(take((size_t)4 * sizeof(double)));
    s.own = reinterpret_cast<T*>(take((size_t)RC * sizeof(T)));
    s.po = po ? reinterpret_cast<T*>(take((size_t)W * nv * sizeof(T))) : nullptr;
    return s;
}

// Global row of local row l: gr0 - h_lo + l (mod nx). The halo is shorter than nx in total, so
// gr0 - h_lo + l lies in [-nx, 2nx) and one conditional correction suffices (no division: integer
// division by a runtime value costs tens of instructions, and these helpers run every step).
__device__ __forceinline__ int res_grow(int gr0, int h_lo, int l, int nx) {
    int q = gr0 - h_lo + l;
    q += q < 0 ? nx : 0;
    return q >= nx ? q - nx : q;
}

// Unreduced x offset of a column from its table entry m in [0, nx): the offset lies in
// [mx_lo, mx_hi] with mx_hi - mx_lo < nx, so it is mx_lo + ((m - mx_lo) mod nx).
__device__ __forceinline__ int res_signed(int m, int mx_lo, int nx) {
    int r = (m - mx_lo) % nx;
    r = r < 0 ? r + nx : r;
    return mx_lo + r;
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
// f_eq rounded from float64; other shifts use the float64 values. i: global row (x-dependent f_eq).
template <typename T, bool FEQ2D>
__device__ __forceinline__ T res_vcorr(const ResSmem<T>& S, const double* __restrict__ feq, int rs,
                                       int i, int j, int c0, int c1, const VShift<T> v, int nv) {
    if (!FEQ2D) {
        // m = 0: c0 = j, t*D[j]; m = nv-1: c0 = j-1, (t-1)*D[j-1] (= -(1-t)*D[j-1] exactly)
        if (v.m == 0 || v.m == nv - 1) return (v.m == 0 ? v.t : v.t - T(1)) * S.dfeq[c0];
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

// Split cluster barrier: arrive (release: this thread's earlier shared/global writes become
// visible cluster-wide) ... wait (acquire). Work placed between the two overlaps the barrier;
// the global writes of the outputs go there so the release does not wait for them.
__device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

template <typename T> struct Vec16Of {
    using type = float4;
};
template <> struct Vec16Of<double> {
    using type = double2;
};

// Fills the halo rows of `plane` (this CTA's copy) from the owners' own rows of the same plane:
// one row per warp at a time, 16-byte loads when a row is a whole number of them.
template <typename T, int RC>
__device__ __forceinline__ void res_fill_halo(cg::cluster_group& cluster, T* plane, int nx, int nv,
                                              int gr0, int h_lo, int h_hi) {
    const int nh = h_lo + h_hi;
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    using V = typename Vec16Of<T>::type;
    constexpr int VE = 16 / (int)sizeof(T);
    for (int h = (int)(threadIdx.x >> 5); h < nh; h += nw) {
        const int l = h < h_lo ? h : h + RC;
        const int q = res_grow(gr0, h_lo, l, nx);
        const int c = q / RC;   // RC is a power of two known at compile time
        const T* src = cluster.map_shared_rank(plane, c) + (size_t)(h_lo + q - c * RC) * nv;
        T* dst = plane + l * nv;   // shared-memory offsets in 32-bit arithmetic
        if (nv % VE == 0) {
            for (int v = lane; v < nv / VE; v += 32) reinterpret_cast<V*>(dst)[v] = reinterpret_cast<const V*>(src)[v];
        } else {
            for (int v = lane; v < nv; v += 32) dst[v] = src[v];
        }
    }
}

// Row sums in three fixed-order stages. (1) Each warp reduces its RPT rows over its 32 columns
// with a transposed butterfly (RPT values in log2(RPT) halving exchanges, then a plain xor tree)
// and writes one partial per row to red[row][column group] (no block barrier). (2) After a block
// barrier, res_rows_local sums each row's column-group partials in ascending order into the CTA's
// own row-sum slot. (3) After the cluster barrier that publishes the slots, every CTA gathers all
// nx row sums from the owners. Only local shared-memory stores precede the
// barrier; the exchange is one distributed-shared-memory load per row after it (res_exchange).
template <int N> struct ILog2 { static constexpr int value = 1 + ILog2<N / 2>::value; };
template <> struct ILog2<1> { static constexpr int value = 0; };

template <typename T, int RPT>
__device__ __forceinline__ void res_warp_rows(T (&v)[RPT], T* red, int rt, int cw, int ncw) {
    constexpr int LG = ILog2<RPT>::value;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int st = 0; st < LG; ++st) {
        const int o = 16 >> st;
        const int n = RPT >> (st + 1);
        const bool upper = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < (RPT >> 1); ++i) {
            if (i < n) {
                const T send = upper ? v[i] : v[i + n];
                const T keep = upper ? v[i + n] : v[i];
                v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
            }
        }
    }
    T r = v[0];
#pragma unroll
    for (int o = 16 >> LG; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    // lane L holds the sum of row L >> (5 - LG) of the thread's RPT rows
    if ((lane & ((32 >> LG) - 1)) == 0) red[(rt + (lane >> (5 - LG))) * ncw + cw] = r;
}

template <typename T>
__device__ __forceinline__ void res_rows_local(const T* red, T* slot, int ncw, int RC) {
    for (int r = threadIdx.x; r < RC; r += blockDim.x) {
        T s = T(0);
        for (int w = 0; w < ncw; ++w) s += red[r * ncw + w];
        slot[r] = s;
    }
}

// The two exchanges after a step's cluster barrier: the halo rows of `plane` (res_fill_halo) and
// the row sums, out[i] = scale * (row sum of row i) read from slot `par` of the owning CTA. The
// first row sum of each thread is loaded before the halo rows move and stored after them, so that
// the two remote round trips overlap instead of following one another (the halo stores could
// alias the row-sum slots as far as the compiler knows, so it would not hoist the load itself).
template <typename T, int RC>
__device__ __forceinline__ void res_exchange(cg::cluster_group& cluster, T* plane, int nx, int nv, int gr0,
                                             int h_lo, int h_hi, T* own_slots, int par, T* out, T scale) {
    const int i0 = threadIdx.x;
    T first = T(0);
    if (i0 < nx) {
        const int c = i0 / RC;
        first = cluster.map_shared_rank(own_slots, c)[par * RC + (i0 - c * RC)];
    }
    res_fill_halo<T, RC>(cluster, plane, nx, nv, gr0, h_lo, h_hi);
    if (i0 < nx) out[i0] = scale * first;
    for (int i = i0 + (int)blockDim.x; i < nx; i += blockDim.x) {
        const int c = i / RC;
        out[i] = scale * cluster.map_shared_rank(own_slots, c)[par * RC + (i - c * RC)];
    }
}

// out[r] = sum_k c[(i-k) mod nx] x[k] (adjoint: c[(k-i) mod nx]) for the n_rows rows
// i = (first + r) mod nx, r < n_rows. A warp takes 4 consecutive rows at a time; lane g sums
// k = g, g + 32, ... in order for the 4 rows at once: the 4 coefficients of one k are
// consecutive table entries, and consecutive lanes read consecutive entries of x and of the
// table (no shared-memory bank conflicts). The 4 x 32 partial sums are combined by a transposed
// butterfly (fixed order). With `vsh`, the lane that writes out[r] also writes the v shift of
// row r from out[r] + aux[global row] (the forward field). No integer division; starts with a
// block barrier, and the caller places one after it before out or vsh are read.
template <typename T>
__device__ __forceinline__ void res_circ_rows(const T* ctab, const T* x, T* out, int nx, int first,
                                              int n_rows, bool adjoint, VShift<T>* vsh = nullptr,
                                              const T* aux = nullptr, T dtdv = T(0), int nv = 0) {
    __syncthreads();
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int off = nx + 8;
    const int ngrp = (n_rows + 3) >> 2;
    for (int grp = (int)(threadIdx.x >> 5); grp < ngrp; grp += nw) {
        int i0 = first + 4 * grp;
        while (i0 >= nx) i0 -= nx;
        // rows i0 + q (q < 4, not reduced mod nx: the table covers the overhang); coefficient of
        // row q at k: forward ctab[off + i0 + q - k], adjoint ctab[off + k - i0 - q]
        T acc[4] = {T(0), T(0), T(0), T(0)};
        const int sgn = adjoint ? -1 : 1;
        const T* cp = adjoint ? ctab + off + lane - i0 : ctab + off + i0 - lane;
        const int cstep = adjoint ? 32 : -32;
#pragma unroll 4
        for (int k = lane; k < nx; k += 32) {
            const T xk = x[k];
            acc[0] += cp[0] * xk;
            acc[1] += cp[sgn] * xk;
            acc[2] += cp[2 * sgn] * xk;
            acc[3] += cp[3 * sgn] * xk;
            cp += cstep;
        }
        // transposed butterfly: lane l ends with the sum of row l >> 3
#pragma unroll
        for (int st = 0; st < 2; ++st) {
            const int o = 16 >> st;
            const int n = 2 >> st;
            const bool upper = (lane & o) != 0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (q < n) {
                    const T send = upper ? acc[q] : acc[q + n];
                    const T keep = upper ? acc[q + n] : acc[q];
                    acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, o);
                }
            }
        }
        T sum = acc[0];
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        const int r = 4 * grp + (lane >> 3);
        if ((lane & 7) == 0 && r < n_rows) {
            out[r] = sum;
            if (vsh != nullptr) {
                int q = first + r;
                while (q >= nx) q -= nx;
                vsh[r] = res_vshift<T>(sum + aux[q], dtdv, nv);
            }
        }
    }
}

template <typename T>
__device__ void res_init_tables(ResSmem<T>& S, const PoissonTables<T>& P, const double* feq,
                                bool feq2d, int nx, int nv) {
    for (int j = threadIdx.x; j < 3 * nx + 16; j += blockDim.x) {
        int d = (j - nx - 8) % nx;   // once per launch
        d += d < 0 ? nx : 0;
        S.ctab[j] = __ldg(P.circ + d);
    }
    if (!feq2d) {
        for (int j = threadIdx.x; j < nv; j += blockDim.x) {
            const double f = __ldg(feq + j);
            S.feq[j] = f;
            S.dfeq[j] = (T)(__ldg(feq + (j + 1 == nv ? 0 : j + 1)) - f);
        }
    }
}

// Phase A of a float32 step with an x-invariant f_eq: o = V(h) + [V(f_eq) - f_eq] of every local
// row of `cur` into S.po, computed once per (row, column) instead of once per thread window, so a
// warp works on one row (one shift) at a time. The arithmetic is the per-cell form of the
// thread-window code (lerp of the two source cells plus res_vcorr), so the results are the same
// bits. Needs nv % 4 == 0 (and, for res_v_rows, blockDim.x a multiple of nv / 4).
// v step of one local row l (shift v) on four columns j0 .. j0+3 of the plane `cur`, into the
// phase-A plane: o = V(h) + [V(f_eq) - f_eq] (the fast forms for shifts 0 and -1).
__device__ __forceinline__ void res_v_quad(const ResSmem<float>& S, const float* cur, int nv, int l, int j0,
                                           const VShift<float> v) {
    const int jm = j0 == 0 ? nv - 1 : j0 - 1, jp = j0 + 4 == nv ? 0 : j0 + 4;
    const float* hr = cur + l * nv;
    float4 o;
    if (v.m == 0) {
        const float4 h = *reinterpret_cast<const float4*>(hr + j0);
        const float4 dd = *reinterpret_cast<const float4*>(S.dfeq + j0);
        const float t = v.t;
        o.x = lerp(h.x, h.y, t) + t * dd.x;
        o.y = lerp(h.y, h.z, t) + t * dd.y;
        o.z = lerp(h.z, h.w, t) + t * dd.z;
        o.w = lerp(h.w, hr[jp], t) + t * dd.w;
    } else if (v.m == nv - 1) {
        const float4 h = *reinterpret_cast<const float4*>(hr + j0);
        const float4 dd = *reinterpret_cast<const float4*>(S.dfeq + j0);
        const float t = v.t, tm = v.t - 1.f;
        o.x = lerp(hr[jm], h.x, t) + tm * S.dfeq[jm];
        o.y = lerp(h.x, h.y, t) + tm * dd.x;
        o.z = lerp(h.y, h.z, t) + tm * dd.y;
        o.w = lerp(h.z, h.w, t) + tm * dd.z;
    } else {
        float r[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int j = j0 + e;
            const int c0 = wrap1(j + v.m, nv);
            const int c1 = c0 + 1 == nv ? 0 : c0 + 1;
            r[e] = lerp(hr[c0], hr[c1], v.t) + res_vcorr<float, false>(S, nullptr, 0, 0, j, c0, c1, v, nv);
        }
        o = make_float4(r[0], r[1], r[2], r[3]);
    }
    *reinterpret_cast<float4*>(S.po + (l * nv + j0)) = o;
}

// Phase A of a step as its own pass: the v step once per (local row, column) of the plane `cur`
// into S.po, four columns per thread, one row per thread group at a time (blockDim.x a multiple
// of nv / 4).
__device__ __forceinline__ void res_v_rows(const ResSmem<float>& S, const float* cur, int nv, int W) {
    const int nq = nv >> 2;
    const int q = threadIdx.x % nq, j0 = 4 * q;
    const int lstep = blockDim.x / nq;
#pragma unroll 1
    for (int l = threadIdx.x / nq; l < W; l += lstep) res_v_quad(S, cur, nv, l, j0, S.vsh[l]);
}

// The forward field of the W local rows and phase A of the next step in one pass, one row per warp
// at a time: the warp sums E of its row over k (each lane k = lane, lane + 32, ... in order, then
// an xor tree), derives the row's v shift from E + H, stores both and applies the v step to the
// row's columns of the plane `cur` into S.po. A row stays with one warp from the field to the
// plane, so no block barrier separates the two. Used for CTAs of at most 8 own rows, whose W
// local rows number about as many as the CTA's warps (128^2: 11 % faster per forward loop);
// with 16 own rows and more the rows' uneven split over the warps cost more than the barrier
// saved (256^2: 4.6 % slower), and phase A stays a pass of its own there.
// rho in S.vec0; starts and ends with a block barrier.
__device__ __forceinline__ void res_field_vrows(const ResSmem<float>& S, const float* cur, int nx, int nv,
                                                int first, int W, float dtdv) {
    __syncthreads();
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int off = nx + 8;
    for (int l = (int)(threadIdx.x >> 5); l < W; l += nw) {
        int i = first + l;
        while (i >= nx) i -= nx;
        const float* cp = S.ctab + off + i - lane;   // coefficient of row i at k: ctab[off + i - k]
        float acc = 0.f;
#pragma unroll 4
        for (int k = lane; k < nx; k += 32) {
            acc += cp[0] * S.vec0[k];
            cp -= 32;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        const VShift<float> v = res_vshift<float>(acc + S.aux[i], dtdv, nv);
        if (lane == 0) {
            S.fld[l] = acc;
            S.vsh[l] = v;
        }
        for (int j0 = 4 * lane; j0 < nv; j0 += 128) res_v_quad(S, cur, nv, l, j0, v);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------------------------
// Forward
// ---------------------------------------------------------------------------------------------

// Field of step k: fills the halo of `plane` (holding h_k), gathers the row sums of h_k published
// in slot `par` of every CTA into rho, evaluates Poisson on the W local rows and their v shifts.
// CTA 0 also sums the partial energies of step k - 2 (published by the barrier before this call)
// into ee_hist[k - 2]; the remote reads go here, with the other exchanges of the step, because
// every CTA is between the same two barriers. Ends with a block barrier.
template <typename T, int RC>
__device__ void res_fwd_field(const ResFwdArgs<T>& a, ResSmem<T>& S, cg::cluster_group& cluster, T* plane,
                              int par, int gr0, int k, int me, int CN) {
    const int nx = a.nx, nv = a.nv;
    const int W = a.h_lo + RC + a.h_hi;
    // warp 0 of CTA 0: the energy partials are loaded before the exchanges and summed after them
    const bool ee = me == 0 && k >= 2 && a.ee_hist != nullptr && threadIdx.x < 32;
    const int lane = threadIdx.x & 31;
    double eev = 0.0;
    if (ee && lane < CN) eev = cluster.map_shared_rank(S.eep, lane)[(k - 2) & 3];
    res_exchange<T, RC>(cluster, plane, nx, nv, gr0, a.h_lo, a.h_hi, S.vec1, par, S.vec0, -a.dv);   // halo, rho
    if (ee) {
        double tot = 0.0;
        for (int c = 0; c < CN; ++c) tot += __shfl_sync(0xffffffffu, eev, c);
        if (lane == 0) a.ee_hist[k - 2] = (T)(0.5 * tot * (double)a.dx);
    }
    const int first = res_grow(gr0, a.h_lo, 0, nx);
    if constexpr (sizeof(T) == 4 && RC <= 8) {
        if (S.po != nullptr) {   // float32, x-invariant f_eq, plane present: field + phase A of the next step
            res_field_vrows(S, plane, nx, nv, first, W, a.dtdv);
            return;
        }
    }
    res_circ_rows<T>(S.ctab, S.vec0, S.fld, nx, first, W, false, S.vsh, S.aux, a.dtdv, nv);
    __syncthreads();
}

// One warp, for step s (S.fld holds E_s): E_hist, E_tape and vsh_tape of the own rows, and the
// partial energy of the own rows into its slot s % 4 (the next cluster barrier publishes it; CTA 0
// sums the partials in the field of step s + 2). Runs between a cluster arrive and wait.
template <typename T>
__device__ void res_fwd_outputs(const ResFwdArgs<T>& a, ResSmem<T>& S, int s, int gr0, int RC) {
    const int nx = a.nx, nv = a.nv;
    const int lane = threadIdx.x & 31;
    double e2 = 0.0;
    for (int r = lane; r < RC; r += 32) {
        const int i = gr0 + r;
        const T E = S.fld[a.h_lo + r];
        const T Et = E + S.aux[i];
        if (a.E_hist != nullptr) a.E_hist[(size_t)s * nx + i] = Et;
        if (a.E_tape != nullptr) a.E_tape[(size_t)s * nx + i] = E;
        if (a.vsh_tape != nullptr) a.vsh_tape[(size_t)s * nx + i] = res_vshift<T>(Et, a.dtdv, nv);
        e2 += (double)(trap_w<T>(i, nx) * E * E);
    }
    e2 = warp_sum(e2);
    if (lane == 0) S.eep[s & 3] = e2;
}

template <typename T, int RC, int RPT, bool FEQ2D>
__global__ void __launch_bounds__(res_max_threads(RPT)) vp_res_fwd_kernel(const ResFwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int nx = a.nx, nv = a.nv;
    const int me = (int)cluster.block_rank();
    const int CN = (int)cluster.num_blocks();
    const int gr0 = me * RC;
    const int hl = a.h_lo;
    constexpr int G = RC / RPT;
    const int NVP = blockDim.x / G;
    const int j = threadIdx.x % NVP;
    const int rt = (threadIdx.x / NVP) * RPT;   // first own row of this thread (CTA-local)
    const int g = gr0 + rt;                      // first own row of this thread (global)
    const bool colv = j < nv;
    const int cw = j >> 5, ncw = NVP >> 5;      // warp column group, groups per row
    const bool out_warp = (int)(threadIdx.x >> 5) == (int)(blockDim.x >> 5) - 1;
    const int W = hl + RC + a.h_hi;
    // the v step by rows (phase A) when the host gave the block the plane for it
    const bool vrows = a.vrows != 0;
    ResSmem<T> S = res_carve<T>(smem, nx, nv, RC, W, vrows);
    T* Hb[2] = {S.p0, S.p1};   // h of even / odd steps, local rows (own rows read remotely)
    T* red = S.p2;             // row partials of the warps
    res_init_tables<T>(S, a.P, a.feq, FEQ2D, nx, nv);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) S.aux[i] = __ldg(a.H + i);

    // per-column constants of the x half-step
    int m = 0, sm = 0;
    T t = T(0), wj = T(0);
    double t64 = 0.0, feq_j = 0.0;
    if (colv) {
        m = __ldg(a.mx + j);
        sm = res_signed(m, a.mx_lo, nx);
        t = __ldg(a.tx + j);
        t64 = __ldg(a.tx64 + j);
        wj = trap_w<T>(j, nv);
        feq_j = FEQ2D ? 0.0 : __ldg(a.feq + j);
    }
    __syncthreads();

    // ---- prologue: h_0 = X(f_iv - f_eq) + corr for the own rows, straight from global memory ----
    {
        T wv[RPT];
#pragma unroll
        for (int k = 0; k < RPT; ++k) wv[k] = T(0);
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
                Hb[0][(hl + rt + k) * nv + j] = h;
                wv[k] = wj * h;
                if (a.h_tape != nullptr) a.h_tape[(size_t)i * nv + j] = h;
            }
        }
        res_warp_rows<T, RPT>(wv, red, rt, cw, ncw);
    }
    __syncthreads();
    res_rows_local<T>(red, S.vec1, ncw, RC);
    cluster.sync();
    res_fwd_field<T, RC>(a, S, cluster, Hb[0], 0, gr0, 0, me, CN);

    for (int n = 0; n < a.n_steps; ++n) {
        const T* cur = Hb[n & 1];
        T* nxt = Hb[(n + 1) & 1];
        const bool last = (n == a.n_steps - 1);
        T d[RPT + 1];
        T hv[RPT];
        T wv[RPT];
#pragma unroll
        for (int k = 0; k < RPT; ++k) wv[k] = T(0);
        int dq = 0;
        if constexpr (sizeof(T) == 4 && !FEQ2D && RC > 8) {
            if (vrows) {
                res_v_rows(S, cur, nv, W);   // phase A: the v step once per (row, column)
                __syncthreads();
            }
        }
        if (colv) {
            // o on rows g+2m .. g+2m+RPT+1: local rows l0 .. l0+RPT+1 (own or halo)
            T o[RPT + 2];
            const int l0 = hl + rt + 2 * sm;
            bool from_plane = false;
            if constexpr (sizeof(T) == 4 && !FEQ2D) from_plane = vrows;
            if (from_plane) {
                const T* op = S.po + (l0 * nv + j);
#pragma unroll
                for (int k = 0; k < RPT + 2; ++k) o[k] = op[k * nv];
            } else {
#pragma unroll
                for (int k = 0; k < RPT + 2; ++k) {
                    const int l = l0 + k;
                    const VShift<T> v = S.vsh[l];
                    const T* hr = cur + l * nv;
                    const int c0 = wrap1(j + v.m, nv);
                    const int c1 = c0 + 1 == nv ? 0 : c0 + 1;
                    const int q = FEQ2D ? res_grow(gr0, hl, l, nx) : 0;
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
                    nxt[(hl + rt + k) * nv + j] = h;
                    wv[k] = wj * h;
                }
            }
        }
        const int par = (n + 1) & 1;
        if (!last) {
            res_warp_rows<T, RPT>(wv, red, rt, cw, ncw);
            __syncthreads();
            res_rows_local<T>(red, S.vec1 + par * RC, ncw, RC);
        }
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
        if (out_warp) res_fwd_outputs<T>(a, S, n, gr0, RC);
        cluster_wait();
        if (!last) res_fwd_field<T, RC>(a, S, cluster, nxt, par, gr0, n + 1, me, CN);
    }
    // energies of the last two steps (their partials are published by this barrier); the second
    // barrier keeps every CTA's shared memory alive until CTA 0 has read it
    cluster.sync();
    if (me == 0 && threadIdx.x == 0 && a.ee_hist != nullptr) {
        for (int s = a.n_steps >= 2 ? a.n_steps - 2 : 0; s < a.n_steps; ++s) {
            double tot = 0.0;
            for (int c = 0; c < CN; ++c) tot += cluster.map_shared_rank(S.eep, c)[s & 3];
            a.ee_hist[s] = (T)(0.5 * tot * (double)a.dx);
        }
    }
    cluster.sync();
}

// ---------------------------------------------------------------------------------------------
// Adjoint
// ---------------------------------------------------------------------------------------------

// Tape values that the adjoint field of step s reads, loaded into registers ahead of their use:
// g_E_hist and E_tape of row threadIdx.x and the v shift of local row threadIdx.x. Rows beyond
// blockDim.x are read in the field itself.
template <typename T> struct ResBwdPre {
    T gEh, Etp, gee;
    VShift<T> vs;
};

template <typename T>
__device__ __forceinline__ ResBwdPre<T> res_bwd_prefetch(const ResBwdArgs<T>& a, int s, int gr0, int W) {
    const int nx = a.nx, i = threadIdx.x;
    ResBwdPre<T> p;
    p.gee = a.g_ee != nullptr ? __ldg(a.g_ee + s) : T(0);
    p.gEh = (a.g_Eh != nullptr && i < nx) ? __ldg(a.g_Eh + (size_t)s * nx + i) : T(0);
    p.Etp = i < nx ? __ldg(a.E_tape + (size_t)s * nx + i) : T(0);
    p.vs.m = 0;
    p.vs.t = T(0);
    if (i < W) p.vs = a.vsh_tape[(size_t)s * nx + res_grow(gr0, a.h_lo, i, nx)];
    return p;
}

// Tail of the adjoint for step s (every CTA): fills the halo of `plane` (holding w_s), gathers the
// row sums published in slot `par`; g_E_total = -dt/dv * rowsum + g_E_hist[s]; g_H += g_E_total
// (own rows); g_E = g_E_total + ee^T; grho = Poisson^T(g_E) and the v shifts of step s on the W
// local rows. `pre` holds this thread's tape values of step s.
template <typename T, int RC>
__device__ void res_bwd_field(const ResBwdArgs<T>& a, ResSmem<T>& S, cg::cluster_group& cluster, T* plane,
                              int par, int s, int gr0, const ResBwdPre<T>& pre) {
    const int nx = a.nx;
    const int W = a.h_lo + RC + a.h_hi;
    const int me_i = threadIdx.x;
    T* sums = S.vec0;
    res_exchange<T, RC>(cluster, plane, nx, a.nv, gr0, a.h_lo, a.h_hi, S.vec1, par, sums, T(1));
    const T gee = pre.gee;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const bool own = i == me_i;
        T gEt = a.neg_dt_dv * sums[i];
        if (a.g_Eh != nullptr) gEt += own ? pre.gEh : __ldg(a.g_Eh + (size_t)s * nx + i);
        if (i >= gr0 && i < gr0 + RC) S.own[i - gr0] += gEt;
        const T Et = own ? pre.Etp : __ldg(a.E_tape + (size_t)s * nx + i);
        S.aux[i] = gEt + a.dx * trap_w<T>(i, nx) * Et * gee;
    }
    for (int l = threadIdx.x; l < W; l += blockDim.x)
        S.vsh[l] = l == me_i ? pre.vs : a.vsh_tape[(size_t)s * nx + res_grow(gr0, a.h_lo, l, nx)];
    res_circ_rows<T>(S.ctab, S.aux, S.fld, nx, res_grow(gr0, a.h_lo, 0, nx), W, true);
    __syncthreads();
}

// Slope inputs of step np at the own rows g .. g+RPT-1, column j: the v shifts of those rows
// (vs, loaded one step ahead) select the two h_tape values (h0, h1) that the slope
// (h + f_eq)[d1] - (h + f_eq)[d0] needs. The loads are issued a step before their use.
template <typename T, int RPT>
__device__ __forceinline__ void res_bwd_load_shifts(const ResBwdArgs<T>& a, int np, int g,
                                                    VShift<T> (&vs)[RPT]) {
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        vs[k].m = 0;
        vs[k].t = T(0);
    }
    if (np < 0) return;
#pragma unroll
    for (int k = 0; k < RPT; ++k) vs[k] = a.vsh_tape[(size_t)np * a.nx + g + k];
}

// With an x-invariant f_eq the f_eq slope D[d0] of each row is read here too (fd), so that the
// step that uses the slopes needs no shifts and no index wraps.
template <typename T, int RPT, bool FEQ2D>
__device__ __forceinline__ void res_bwd_load_h(const ResBwdArgs<T>& a, const ResSmem<T>& S, int np, int g, int j,
                                               const VShift<T> (&vs)[RPT], T (&h0)[RPT], T (&h1)[RPT],
                                               T (&fd)[RPT]) {
    const int nv = a.nv;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        h0[k] = T(0);
        h1[k] = T(0);
        fd[k] = T(0);
    }
    if (np < 0) return;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        const int d0 = wrap1(j + vs[k].m, nv);
        const int d1 = d0 + 1 == nv ? 0 : d0 + 1;
        const T* hr = a.h_tape + ((size_t)np * a.nx + g + k) * nv;
        h0[k] = __ldg(hr + d0);
        h1[k] = __ldg(hr + d1);
        if (!FEQ2D) fd[k] = S.dfeq[d0];
    }
}

// w on the own rows g .. g+RPT-1 (stored at own_rows, the plane's first own row) from c on rows
// g-m-1 .. g-m+RPT-1 (held in registers), and the slope * w products for the dE row sums (slope
// inputs of step np from res_bwd_load_*).
template <typename T, int RPT, bool FEQ2D>
__device__ __forceinline__ void res_bwd_w(const ResBwdArgs<T>& a, const ResSmem<T>& S,
                                          const T (&c)[RPT + 1], T* own_rows, T (&prod)[RPT],
                                          const VShift<T> (&vs)[RPT], const T (&h0)[RPT],
                                          const T (&h1)[RPT], const T (&fd)[RPT], int g, int rt, int j, T t) {
    const int nv = a.nv;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        const T wv = lerp(c[k + 1], c[k], t);
        own_rows[(rt + k) * nv + j] = wv;
        T sl = h1[k] - h0[k];
        if constexpr (FEQ2D) {
            const int i = g + k;
            const int d0 = wrap1(j + vs[k].m, nv);
            const int d1 = d0 + 1 == nv ? 0 : d0 + 1;
            sl += (T)(__ldg(a.feq + (size_t)i * a.feq_rs + d1) - __ldg(a.feq + (size_t)i * a.feq_rs + d0));
        } else {
            sl += fd[k];
        }
        prod[k] = sl * wv;
    }
}

template <typename T, int RC, int RPT, bool FEQ2D>
__global__ void __launch_bounds__(res_max_threads(RPT)) vp_res_bwd_kernel(const ResBwdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int nx = a.nx, nv = a.nv, T_steps = a.n_steps;
    const int me = (int)cluster.block_rank();
    const int CN = (int)cluster.num_blocks();
    const int gr0 = me * RC;
    const int hl = a.h_lo;
    const int W = hl + RC + a.h_hi;
    constexpr int G = RC / RPT;
    const int NVP = blockDim.x / G;
    const int j = threadIdx.x % NVP;
    const int rt = (threadIdx.x / NVP) * RPT;
    const int g = gr0 + rt;
    const bool colv = j < nv;
    const int cw = j >> 5, ncw = NVP >> 5;
    ResSmem<T> S = res_carve<T>(smem, nx, nv, RC, W, false);
    T* Wb[2] = {S.p0, S.p1};   // cotangent on the v-step output of even / odd steps, local rows
    T* red = S.p2;             // row partials of the warps
    res_init_tables<T>(S, a.P, a.feq, FEQ2D, nx, nv);
    for (int r = threadIdx.x; r < RC; r += blockDim.x) S.own[r] = T(0);
    __syncthreads();   // S.dfeq is complete before the first slope loads read it
    int m = 0, sm = 0;
    T t = T(0), wr = T(0);
    if (colv) {
        m = __ldg(a.mx + j);
        sm = res_signed(m, a.mx_lo, nx);
        t = __ldg(a.tx + j);
        wr = -a.dv * trap_w<T>(j, nv);   // rho^T weight (warp_vp_solver/kernels.py:292-299)
    }
    // slope inputs: vA/hA of the step whose slopes come next, vB the shifts of the step after it
    VShift<T> vA[RPT], vB[RPT];
    T hA0[RPT], hA1[RPT], fdA[RPT];
    ResBwdPre<T> pre = res_bwd_prefetch<T>(a, T_steps - 1, gr0, W);
    if (colv) {
        res_bwd_load_shifts<T, RPT>(a, T_steps - 1, g, vA);
        res_bwd_load_h<T, RPT, FEQ2D>(a, S, T_steps - 1, g, j, vA, hA0, hA1, fdA);
        res_bwd_load_shifts<T, RPT>(a, T_steps - 2, g, vB);
    }
    __syncthreads();

    // ---- prologue (n = T): c = g_f_final + g_f_hist[T-1] on rows g-m-1 .. g-m+RPT-1 ----
    {
        T* nxt = Wb[(T_steps - 1) & 1];
        T prod[RPT];
#pragma unroll
        for (int k = 0; k < RPT; ++k) prod[k] = T(0);
        if (colv) {
            T c[RPT + 1];
            const int cb = wrapneg(g - m - 1, nx);   // g - m - 1 >= -nx
#pragma unroll
            for (int k = 0; k <= RPT; ++k) {
                const int q = wrap1(cb + k, nx);
                T v = T(0);
                if (a.g_ff != nullptr) v += __ldg(a.g_ff + (size_t)q * nv + j);
                if (a.g_fh != nullptr) v += __ldg(a.g_fh + ((size_t)(T_steps - 1) * nx + q) * nv + j);
                c[k] = v;
            }
            res_bwd_w<T, RPT, FEQ2D>(a, S, c, nxt + hl * nv, prod, vA, hA0, hA1, fdA, g, rt, j, t);
            // next: slopes of step T-2
#pragma unroll
            for (int k = 0; k < RPT; ++k) vA[k] = vB[k];
            res_bwd_load_h<T, RPT, FEQ2D>(a, S, T_steps - 2, g, j, vA, hA0, hA1, fdA);
            res_bwd_load_shifts<T, RPT>(a, T_steps - 3, g, vB);
        }
        res_warp_rows<T, RPT>(prod, red, rt, cw, ncw);
        __syncthreads();
        const int par = (T_steps - 1) & 1;
        res_rows_local<T>(red, S.vec1 + par * RC, ncw, RC);
        cluster.sync();
        res_bwd_field<T, RC>(a, S, cluster, nxt, par, T_steps - 1, gr0, pre);
    }

    for (int n = T_steps - 1; n >= 0; --n) {
        const T* cur = Wb[n & 1];
        T* nxt = Wb[(n + 1) & 1];   // == Wb[(n-1) & 1]
        if (n > 0) pre = res_bwd_prefetch<T>(a, n - 1, gr0, W);
        T prod[RPT];
#pragma unroll
        for (int k = 0; k < RPT; ++k) prod[k] = T(0);
        if (colv) {
            // gh = V^T(w_n) + rho^T(grho_n) on rows g-2m-2 .. g-2m+RPT-1 (n = 0: g-m-1 ..), local rows
            const int ng = n == 0 ? RPT + 1 : RPT + 2;   // rows of gh needed
            T gh[RPT + 2];
            const int l0 = n == 0 ? hl + rt - sm - 1 : hl + rt - 2 * sm - 2;
#pragma unroll
            for (int k = 0; k < RPT + 2; ++k) {
                if (k < ng) {
                    const int l = l0 + k;
                    const VShift<T> v = S.vsh[l];
                    const T* wrow = cur + l * nv;
                    const int c0 = wrapneg(j - v.m, nv);
                    const int c1 = wrapneg(c0 - 1, nv);
                    gh[k] = lerp(wrow[c0], wrow[c1], v.t) + wr * S.fld[l];
                }
            }
            if (n == 0) {
                // gradient on f_iv: c on the own rows from gh on rows g-m-1 .. g-m+RPT-1
#pragma unroll
                for (int k = 0; k < RPT; ++k) a.g_fiv[(size_t)(g + k) * nv + j] = lerp(gh[k + 1], gh[k], t);
            } else {
                // c on rows g-m-1 .. g-m+RPT-1 (+ g_f_hist[n-1]), then w_{n-1} on the own rows
                T c[RPT + 1];
                const int cb = wrapneg(g - m - 1, nx);
#pragma unroll
                for (int k = 0; k <= RPT; ++k) {
                    c[k] = lerp(gh[k + 1], gh[k], t);
                    if (a.g_fh != nullptr)
                        c[k] += __ldg(a.g_fh + ((size_t)(n - 1) * nx + wrap1(cb + k, nx)) * nv + j);
                }
                res_bwd_w<T, RPT, FEQ2D>(a, S, c, nxt + hl * nv, prod, vA, hA0, hA1, fdA, g, rt, j, t);
                // next: slopes of step n-2 (h loads now, shifts of step n-3 for the one after)
#pragma unroll
                for (int k = 0; k < RPT; ++k) vA[k] = vB[k];
                res_bwd_load_h<T, RPT, FEQ2D>(a, S, n - 2, g, j, vA, hA0, hA1, fdA);
                res_bwd_load_shifts<T, RPT>(a, n - 3, g, vB);
            }
        }
        const int par = (n - 1) & 1;
        if (n > 0) {
            res_warp_rows<T, RPT>(prod, red, rt, cw, ncw);
            __syncthreads();
            res_rows_local<T>(red, S.vec1 + par * RC, ncw, RC);
        }
        cluster_arrive();
        cluster_wait();
        if (n > 0) res_bwd_field<T, RC>(a, S, cluster, nxt, par, n - 1, gr0, pre);
    }
    for (int r = threadIdx.x; r < RC; r += blockDim.x) a.g_H[gr0 + r] = S.own[r];
    // no other CTA reads this CTA's shared memory after the last barrier
}

// ---------------------------------------------------------------------------------------------
// Host-side launch helpers
// ---------------------------------------------------------------------------------------------

// Rows per thread for RC rows per CTA: among the powers of two in [RC/8, RC] whose CTA fits the
// launch bound, the most rows per thread that still gives at least 512 threads (16 warps), or the
// largest CTA when none reaches 512; 0 when none fits. More rows per thread means fewer window
// rows per cell ((RPT+2)/RPT) and fewer per-step overheads; 16 warps keep the latency covered
// (measured on 128x128 and 256x256 grids: 10-20% faster than the 1024-thread shapes).
int res_rows_per_thread(int RC, int nv) {
    const int nvp = ((nv + 31) / 32) * 32;
    int best = 0;
    for (int rpt = RC / 8 > 1 ? RC / 8 : 1; rpt <= RC; rpt *= 2) {
        const int th = (RC / rpt) * nvp;
        if (th > res_max_threads(rpt)) continue;
        if (best == 0 || th >= 512) best = rpt;
    }
    return best;
}

// Threads of the resident CTA for RC rows per CTA (0 when no shape fits).
int res_threads(int RC, int nv) {
    const int nvp = ((nv + 31) / 32) * 32;
    const int rpt = res_rows_per_thread(RC, nv);
    return rpt > 0 ? (RC / rpt) * nvp : 0;
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
    if (RPT == 0 || threads == 0) return 0;
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

size_t res_smem_size(int nx, int nv, int Rc, int halo_rows, size_t real_size, bool vrows) {
    return res_smem_bytes(nx, nv, Rc, Rc + halo_rows, real_size, vrows);
}

template int res_max_clusters<float>(bool, int, int, int, size_t);
template int res_max_clusters<double>(bool, int, int, int, size_t);
template cudaError_t launch_res_fwd<float>(const ResFwdArgs<float>&, bool, int, int, size_t, cudaStream_t);
template cudaError_t launch_res_fwd<double>(const ResFwdArgs<double>&, bool, int, int, size_t, cudaStream_t);
template cudaError_t launch_res_bwd<float>(const ResBwdArgs<float>&, bool, int, int, size_t, cudaStream_t);
template cudaError_t launch_res_bwd<double>(const ResBwdArgs<double>&, bool, int, int, size_t, cudaStream_t);

}  // namespace vpb
