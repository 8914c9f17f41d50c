// Device helpers shared by the fused step kernels and the single-stage operators:
// periodic index arithmetic, lerp, block reductions and the in-block radix-2 FFT Poisson solve.
#pragma once

#include "vp_internal.h"

namespace vpb {

__device__ __forceinline__ float vfloor(float x) { return floorf(x); }
__device__ __forceinline__ double vfloor(double x) { return floor(x); }
__device__ __forceinline__ float vabs(float x) { return fabsf(x); }
__device__ __forceinline__ double vabs(double x) { return fabs(x); }

template <typename T>
__device__ __forceinline__ T lerp(T a, T b, T t) {
    return (T(1) - t) * a + t * b;
}

// x in [0, 2n) -> [0, n)
__device__ __forceinline__ int wrap1(int x, int n) { return x >= n ? x - n : x; }
// x in [0, 3n) -> [0, n)
__device__ __forceinline__ int wrap2(int x, int n) {
    x = x >= n ? x - n : x;
    return x >= n ? x - n : x;
}
// x in [-n, n) -> [0, n)
__device__ __forceinline__ int wrapneg(int x, int n) { return x < 0 ? x + n : x; }
// x in [-2n, n) -> [0, n)
__device__ __forceinline__ int wrapneg2(int x, int n) {
    x = x < 0 ? x + n : x;
    return x < 0 ? x + n : x;
}
// x in [-2n, 2n) -> [0, n)
__device__ __forceinline__ int wrapboth(int x, int n) {
    x = x < 0 ? x + n : x;
    x = x < 0 ? x + n : x;
    return x >= n ? x - n : x;
}
// These replace % n in per-tile index arithmetic: integer division by a runtime value costs
// tens of instructions.

// Trapezoid weight of index k in [0, n): 0.5 at both ends, 1 inside
// (warp_vp_solver/kernels.py:167-172 and 192-197).
template <typename T>
__device__ __forceinline__ T trap_w(int k, int n) {
    return (k == 0 || k == n - 1) ? T(0.5) : T(1);
}

// v-step shift of one row from the total field: s = E_total*dt/dv cells, m = floor(-s) reduced
// mod nv, t = -s - floor(-s). This is the index-space form of the foot v_j - E_total*dt of
// warp_vp_solver/kernels.py:150 and _periodic_indices (kernels.py:47-69).
// A non-finite field gives m = 0 and a NaN weight: the NaN propagates into the results the way
// it does in the reference, and every index stays in bounds.
template <typename T>
__device__ __forceinline__ VShift<T> make_vshift(T Et, T dtdv, int nv) {
    const T s = Et * dtdv;
    const T mf = vfloor(-s);
    const T t = -s - mf;
    int m = 0;
    if (vabs(mf) < T(1.0e9)) {
        long long r = ((long long)mf) % (long long)nv;
        if (r < 0) r += nv;
        m = (int)r;
    }
    VShift<T> v;
    v.m = m;
    v.t = t;
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the block in a fixed order (deterministic). red: >= 32 elements of shared memory.
template <typename T>
__device__ T block_sum(T v, T* red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        T s = lane < nw ? red[lane] : T(0);
        s = warp_sum(s);
        if (lane == 0) red[0] = s;
    }
    __syncthreads();
    return red[0];
}

// ---------------------------------------------------------------------------------------------
// Poisson solve E = real(ifft(m * fft(rho))) (or its transpose with conj(m)) inside one CTA.
// Power-of-two nx: iterative radix-2 decimation-in-time FFT on a complex buffer. The inverse
// transform is a forward transform of the conjugated spectrum, so one twiddle table serves both.
// Other nx: the equivalent real circulant product E_i = sum_k c[(i-k) mod nx] rho_k with
// c = real(ifft(m)) (and c[(k-i) mod nx] for the transpose).
// ---------------------------------------------------------------------------------------------

template <typename C>
__device__ __forceinline__ C cmake(decltype(C::x) a, decltype(C::x) b) {
    C c;
    c.x = a;
    c.y = b;
    return c;
}

__device__ __forceinline__ int bitrev(int i, int L) {
    return L == 0 ? 0 : (int)(__brev((unsigned)i) >> (32 - L));
}

// tw: the nx/2 twiddles exp(-2 pi i q / n), read at q = k * (n >> s) in stage s; or, with
// `staged`, the same values laid out stage after stage (stage s at [2^(s-1) - 1, 2^s - 1)), so
// that the lanes of a warp read consecutive entries instead of one shared-memory bank.
template <typename T>
__device__ void fft_radix2(typename Cplx<T>::type* z, const typename Cplx<T>::type* tw, int n,
                           int L, bool staged = false) {
    using C = typename Cplx<T>::type;
    for (int s = 1; s <= L; ++s) {
        const int half = 1 << (s - 1);
        const int stride = n >> s;
        for (int b = threadIdx.x; b < (n >> 1); b += blockDim.x) {
            const int k = b & (half - 1);
            const int i0 = ((b >> (s - 1)) << s) + k;
            const int i1 = i0 + half;
            const C w = staged ? tw[half - 1 + k] : tw[k * stride];
            const C u = z[i0];
            const C v = z[i1];
            const T vr = v.x * w.x - v.y * w.y;
            const T vi = v.x * w.y + v.y * w.x;
            z[i0] = cmake<C>(u.x + vr, u.y + vi);
            z[i1] = cmake<C>(u.x - vr, u.y - vi);
        }
        __syncthreads();
    }
}

// In-place Poisson transform on a complex work buffer z (nx entries). The caller stores the
// input with poisson_put and reads the result with poisson_get; poisson_core runs between them.
// Power-of-two nx: the input goes to bit-reversed positions, z = fft(x); z = conj(m*z) (or
// conj(conj(m)*z) for the transpose) written back in bit-reversed order; z = fft(z). The result
// is real(z)/nx = real(ifft(m*fft(x))). Other nx: z[i].y = sum_k c[(i-k) mod nx] z[k].x.
// All threads of the block must call poisson_core; it begins and ends with __syncthreads().
template <typename T>
__device__ __forceinline__ void poisson_put(const PoissonTables<T>& P, typename Cplx<T>::type* z,
                                            int i, T v) {
    using C = typename Cplx<T>::type;
    z[P.pow2 ? bitrev(i, P.log2nx) : i] = cmake<C>(v, T(0));
}

template <typename T>
__device__ __forceinline__ T poisson_get(const PoissonTables<T>& P, const typename Cplx<T>::type* z,
                                         int i) {
    return P.pow2 ? z[i].x * (T(1) / T(P.nx)) : z[i].y;
}

template <typename T>
__device__ void poisson_core(const PoissonTables<T>& P, typename Cplx<T>::type* z,
                             const typename Cplx<T>::type* tw_s, bool adjoint) {
    using C = typename Cplx<T>::type;
    const int nx = P.nx;
    __syncthreads();
    if (P.pow2) {
        const int L = P.log2nx;
        const bool staged = P.tw_stage != 0 && P.use_smem != 0;
        fft_radix2<T>(z, tw_s, nx, L, staged);
        const T sgn = adjoint ? T(-1) : T(1);
        for (int i = threadIdx.x; i < nx; i += blockDim.x) {
            const int r = bitrev(i, L);
            if (i <= r) {
                const C a = z[i];
                const C b = z[r];
                const T mi = sgn * P.mult_im[i];
                const T mr = sgn * P.mult_im[r];
                // conj(m * z) with m purely imaginary: (0 + i*mi)(a.x + i*a.y) = (-mi*a.y, mi*a.x)
                z[r] = cmake<C>(-mi * a.y, -mi * a.x);
                z[i] = cmake<C>(-mr * b.y, -mr * b.x);
            }
        }
        __syncthreads();
        fft_radix2<T>(z, tw_s, nx, L, staged);
    } else {
        for (int i = threadIdx.x; i < nx; i += blockDim.x) {
            T s = T(0);
            for (int k = 0; k < nx; ++k) {
                int d = adjoint ? (k - i) : (i - k);
                d = wrapneg(d, nx);
                s += P.circ[d] * z[k].x;
            }
            z[i].y = s;
        }
        __syncthreads();
    }
}

template <typename T>
struct PoissonArea {
    typename Cplx<T>::type* z;
    const typename Cplx<T>::type* tw;
};

// Work area in shared memory (when P.use_smem) or in the global scratch of the workspace.
// Copies the twiddles into shared memory; the copy is complete after poisson_core's first barrier.
template <typename T>
__device__ PoissonArea<T> poisson_area(const PoissonTables<T>& P, unsigned char* smem) {
    using C = typename Cplx<T>::type;
    PoissonArea<T> w;
    if (P.use_smem) {
        C* z = reinterpret_cast<C*>(smem);
        C* tw = z + P.nx;
        if (P.pow2 && P.tw_stage) {
            // entry e = 2^(s-1) - 1 + k of stage s holds twiddle k * (nx >> s)
            for (int e = threadIdx.x; e < P.nx - 1; e += blockDim.x) {
                const int s = 32 - __clz(e + 1);
                const int k = e + 1 - (1 << (s - 1));
                tw[e] = P.tw[(size_t)k * (P.nx >> s)];
            }
        } else if (P.pow2) {
            for (int i = threadIdx.x; i < (P.nx >> 1); i += blockDim.x) tw[i] = P.tw[i];
        }
        w.z = z;
        w.tw = tw;
    } else {
        w.z = reinterpret_cast<C*>(P.gscratch);
        w.tw = P.tw;
    }
    return w;
}

}  // namespace vpb
