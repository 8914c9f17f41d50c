// Single-stage operators: the building blocks of the step exposed on their own, as the
// reference exposes its kernels and helper methods (warp_vp_solver/kernels.py,
// warp_vp_solver/solver.py:393-412, warp_vp_solver/poisson.py:48-99). They share the index
// arithmetic and the in-block FFT with the fused kernels in vp_kernels.cu.

#include "../../include/vp_b200.h"
#include "vp_device.cuh"

#include <algorithm>

namespace vpb {

// rho[i] = dv * trapz_j(f_eq[i,j] - f[i,j]), accumulated in float64 (one CTA per row).
template <typename T>
__global__ void __launch_bounds__(256) rho_kernel(int nv, const double* __restrict__ f,
                                                  const double* __restrict__ feq, int feq_rs,
                                                  double dv, T* __restrict__ rho) {
    __shared__ double red[32];
    const int i = blockIdx.x;
    double s = 0.0;
    for (int j = threadIdx.x; j < nv; j += blockDim.x) {
        const double d = feq[(size_t)i * feq_rs + j] - f[(size_t)i * nv + j];
        s += trap_w<double>(j, nv) * d;
    }
    s = block_sum<double>(s, red);
    if (threadIdx.x == 0) rho[i] = (T)(s * dv);
}

template <typename T>
__global__ void __launch_bounds__(1024) poisson_kernel(const PoissonTables<T> P, const T* in,
                                                      T* out, int adjoint) {
    extern __shared__ __align__(16) unsigned char smem[];
    PoissonArea<T> w = poisson_area<T>(P, smem);
    for (int i = threadIdx.x; i < P.nx; i += blockDim.x) poisson_put<T>(P, w.z, i, in[i]);
    poisson_core<T>(P, w.z, w.tw, adjoint != 0);
    for (int i = threadIdx.x; i < P.nx; i += blockDim.x) out[i] = poisson_get<T>(P, w.z, i);
}

template <typename T>
__global__ void __launch_bounds__(256) ee_kernel(int nx, double dx, const T* E, T* ee) {
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const double e = (double)E[i];
        s += trap_w<double>(i, nx) * e * e;
    }
    s = block_sum<double>(s, red);
    if (threadIdx.x == 0) *ee = (T)(0.5 * s * dx);
}

// x half-step by dt/2 (or its transpose) of an arbitrary array, shift computed per column in
// float64: s = 0.5*v_j*dt/dx (warp_vp_solver/kernels.py:127).
template <typename T>
__global__ void __launch_bounds__(256) semilag_x_kernel(int nx, int nv, const double* __restrict__ vs,
                                                        double dx, double dt, const T* __restrict__ in,
                                                        T* __restrict__ out, int adjoint) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= nv) return;
    const double s = 0.5 * vs[j] * dt / dx;
    const double mf = floor(-s);
    const T t = (T)(-s - mf);
    long long mm = ((long long)mf) % nx;
    if (mm < 0) mm += nx;
    const int m = (int)mm;
    if (!adjoint) {
        const int q0 = wrap1(i + m, nx);
        const int q1 = wrap1(q0 + 1, nx);
        out[(size_t)i * nv + j] = lerp(in[(size_t)q0 * nv + j], in[(size_t)q1 * nv + j], t);
    } else {
        const int q0 = wrapneg(i - m, nx);
        const int q1 = wrapneg(q0 - 1, nx);
        out[(size_t)i * nv + j] = lerp(in[(size_t)q0 * nv + j], in[(size_t)q1 * nv + j], t);
    }
}

// v step (or its transpose plus the field cotangent) of an arbitrary array, one CTA per row.
template <typename T>
__global__ void __launch_bounds__(256) semilag_v_kernel(int nv, T dtdv, const T* __restrict__ in,
                                                        const T* __restrict__ Et,
                                                        T* __restrict__ out, int adjoint,
                                                        const T* __restrict__ f_in,
                                                        T* __restrict__ g_E) {
    __shared__ T red[32];
    const int i = blockIdx.x;
    const VShift<T> vs = make_vshift<T>(Et[i], dtdv, nv);
    const T* row = in + (size_t)i * nv;
    T acc = T(0);
    for (int j = threadIdx.x; j < nv; j += blockDim.x) {
        if (!adjoint) {
            const int c0 = wrap1(j + vs.m, nv);
            const int c1 = wrap1(c0 + 1, nv);
            out[(size_t)i * nv + j] = lerp(row[c0], row[c1], vs.t);
        } else {
            const int c0 = wrapneg(j - vs.m, nv);
            const int c1 = wrapneg(c0 - 1, nv);
            out[(size_t)i * nv + j] = lerp(row[c0], row[c1], vs.t);
            if (g_E != nullptr) {
                const int d0 = wrap1(j + vs.m, nv);
                const int d1 = wrap1(d0 + 1, nv);
                const T* fr = f_in + (size_t)i * nv;
                acc += (fr[d1] - fr[d0]) * row[j];
            }
        }
    }
    if (adjoint && g_E != nullptr) {
        acc = block_sum<T>(acc, red);
        if (threadIdx.x == 0) g_E[i] = -dtdv * acc;
    }
}

template <typename T>
cudaError_t launch_compute_rho(int nx, int nv, const double* f, const double* feq, int feq_rs,
                               double dv, T* rho, cudaStream_t s) {
    if (feq_rs == 0) {
        // broadcast one row of f_eq: index with stride 0
        rho_kernel<T><<<nx, 256, 0, s>>>(nv, f, feq, 0, dv, rho);
    } else {
        rho_kernel<T><<<nx, 256, 0, s>>>(nv, f, feq, feq_rs, dv, rho);
    }
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_poisson(const PoissonTables<T>& P, const T* in, T* out, int adjoint,
                           cudaStream_t s) {
    int threads = P.nx >= 2048 ? 1024 : (P.nx >= 64 ? P.nx / 2 : 32);
    const size_t smem = poisson_area_size(P.nx, sizeof(T));
    poisson_kernel<T><<<1, threads, smem, s>>>(P, in, out, adjoint);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_electric_energy(int nx, double dx, const T* E, T* ee, cudaStream_t s) {
    ee_kernel<T><<<1, 256, 0, s>>>(nx, dx, E, ee);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_semilag_x(int nx, int nv, const double* vs, double dx, double dt,
                             const T* in, T* out, int adjoint, cudaStream_t s) {
    dim3 grid((nv + 127) / 128, nx);
    semilag_x_kernel<T><<<grid, 128, 0, s>>>(nx, nv, vs, dx, dt, in, out, adjoint);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_semilag_v(int nx, int nv, double dv, double dt, const T* in,
                             const T* E_total, T* out, int adjoint, const T* f_in, T* g_E,
                             cudaStream_t s) {
    semilag_v_kernel<T><<<nx, 256, 0, s>>>(nv, (T)(dt / dv), in, E_total, out, adjoint, f_in, g_E);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// KL(f || f_eq) cost, warp_vp_solver/utils.py:53-76, and its gradient with respect to f, in float64:
//   W_ij = wx_i wv_j (trapezoid weights over xs and vs), Z = sum W f + eps,
//   Z_eq = sum W f_eq + eps (host), p = f / Z, q = f_eq / Z_eq + eps,
//   KL = sum W rel_entr(p, q)   (rel_entr: p log(p/q) for p, q > 0; 0 for p = 0, q >= 0; +inf else)
//   dKL/df_ij = (W_ij / Z) (r_ij - S),  r = log(p/q) + 1 where p, q > 0 (0 elsewhere),
//   S = sum W r p.
// Each reduction writes one partial per block and a one-block kernel sums them in block order, so
// the result is deterministic.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double kl_w(int i, int n, double d) { return (i == 0 || i == n - 1) ? 0.5 * d : d; }

__device__ __forceinline__ double block_sum_d(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    __syncthreads();
    return s;
}

// MODE 0: partial[b] = sum W f. MODE 1: partial[b] = sum W rel_entr(p, q), partial[B + b] = sum W r p.
template <int MODE>
__global__ void __launch_bounds__(256) kl_partial_kernel(int nx, int nv, const double* __restrict__ f,
                                                         const double* __restrict__ feq, int feq_rs, double dx,
                                                         double dv, double eps, double zeq,
                                                         const double* __restrict__ zf, double* partial) {
    __shared__ double red[8];
    const long long n = (long long)nx * nv;
    const double Z = MODE == 1 ? *zf : 1.0;
    double a = 0.0, b = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k / nv), j = (int)(k - (long long)i * nv);
        const double W = kl_w(i, nx, dx) * kl_w(j, nv, dv);
        const double fv = f[k];
        if (MODE == 0) {
            a += W * fv;
        } else {
            const double p = fv / Z;
            const double q = feq[(size_t)i * feq_rs + j] / zeq + eps;
            double re;
            if (p > 0.0 && q > 0.0) {
                const double l = log(p / q);
                re = p * l;
                b += W * (l + 1.0) * p;
            } else if (p == 0.0 && q >= 0.0) {
                re = 0.0;
            } else {
                re = INFINITY;
            }
            a += W * re;
        }
    }
    const double sa = block_sum_d(a, red);
    if (MODE == 1) {
        const double sb = block_sum_d(b, red);
        if (threadIdx.x == 0) partial[gridDim.x + blockIdx.x] = sb;
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sa;
}

// out[0] = sum of partial[0..nb) + add0; with two outputs also out[1] = sum partial[nb..2nb).
__global__ void kl_finish_kernel(const double* partial, int nb, int two, double add0, double* out0, double* out1) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += partial[b];
        *out0 = s + add0;
        if (two) {
            double t = 0.0;
            for (int b = 0; b < nb; ++b) t += partial[nb + b];
            *out1 = t;
        }
    }
}

__global__ void __launch_bounds__(256) kl_grad_kernel(int nx, int nv, const double* __restrict__ f,
                                                      const double* __restrict__ feq, int feq_rs, double dx,
                                                      double dv, double eps, double zeq,
                                                      const double* __restrict__ zs, double* grad) {
    const double Z = zs[0], S = zs[1];
    const long long n = (long long)nx * nv;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(k / nv), j = (int)(k - (long long)i * nv);
        const double W = kl_w(i, nx, dx) * kl_w(j, nv, dv);
        const double p = f[k] / Z;
        const double q = feq[(size_t)i * feq_rs + j] / zeq + eps;
        const double r = (p > 0.0 && q > 0.0) ? log(p / q) + 1.0 : 0.0;
        grad[k] = (W / Z) * (r - S);
    }
}

// scratch: [2 * kKlBlocks partials][Z, S]
cudaError_t launch_kl_divergence(int nx, int nv, const double* f, const double* feq, int feq_rs, double dx,
                                 double dv, double eps, double zeq, double* scratch, double* value, double* grad,
                                 cudaStream_t s) {
    const int nb = kKlBlocks;
    double* partial = scratch;
    double* zs = scratch + 2 * nb;
    kl_partial_kernel<0><<<nb, 256, 0, s>>>(nx, nv, f, feq, feq_rs, dx, dv, eps, zeq, nullptr, partial);
    count_launch();
    kl_finish_kernel<<<1, 32, 0, s>>>(partial, nb, 0, eps, zs, nullptr);
    count_launch();
    kl_partial_kernel<1><<<nb, 256, 0, s>>>(nx, nv, f, feq, feq_rs, dx, dv, eps, zeq, zs, partial);
    count_launch();
    kl_finish_kernel<<<1, 32, 0, s>>>(partial, nb, 1, 0.0, value, zs + 1);
    count_launch();
    if (grad != nullptr) {
        const long long n = (long long)nx * nv;
        const int blocks = (int)std::min<long long>(4096, (n + 255) / 256);
        kl_grad_kernel<<<blocks, 256, 0, s>>>(nx, nv, f, feq, feq_rs, dx, dv, eps, zeq, zs, grad);
        count_launch();
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t set_poisson_smem_limit(size_t bytes) {
    return cudaFuncSetAttribute(poisson_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}
template cudaError_t set_poisson_smem_limit<float>(size_t);
template cudaError_t set_poisson_smem_limit<double>(size_t);

// Finite-input check of a forward call: raises VP_STATUS_NONFINITE_INPUT in *status when f (n
// doubles) or H (nx reals) holds a NaN or an infinity. Grid-stride over 16-byte loads of f (its
// base is 16-byte aligned when it comes from a torch allocation; otherwise 8-byte loads).
__global__ void __launch_bounds__(256) check_finite_kernel(const double* __restrict__ f, size_t n,
                                                           const void* __restrict__ H, int nx, int h64,
                                                           unsigned* status) {
    bool bad = false;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    if ((reinterpret_cast<uintptr_t>(f) & 15) == 0) {
        const double2* f2 = reinterpret_cast<const double2*>(f);
        for (size_t i = tid; i < n / 2; i += stride) {
            const double2 v = __ldg(f2 + i);
            bad |= !isfinite(v.x) || !isfinite(v.y);
        }
        if (tid == 0 && (n & 1)) bad |= !isfinite(__ldg(f + n - 1));
    } else {
        for (size_t i = tid; i < n; i += stride) bad |= !isfinite(__ldg(f + i));
    }
    for (size_t i = tid; i < (size_t)nx; i += stride)
        bad |= h64 ? !isfinite(__ldg(static_cast<const double*>(H) + i))
                   : !isfinite(__ldg(static_cast<const float*>(H) + i));
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status, VP_STATUS_NONFINITE_INPUT);
}

cudaError_t launch_check_finite(const double* f, size_t n, const void* H, int nx, bool h64, unsigned* status,
                                cudaStream_t s) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t want = (n / 2 + 255) / 256;
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>(want, (size_t)sms * 8));
    check_finite_kernel<<<blocks, 256, 0, s>>>(f, n, H, nx, h64 ? 1 : 0, status);
    count_launch();
    return cudaGetLastError();
}

// ---- x-slab decomposition: per-row records of a slab's rows, and its owned rows' sums --------
// A slab's arrays hold ext_rows rows; array row k is grid row (row_first + k) mod nx. This copies
// the per-row records the step kernels read (v shifts of step n and n-1, cotangent on rho) from
// the full-grid arrays every rank holds into the slab's own row order. Null pairs are skipped.
template <typename T>
__global__ void __launch_bounds__(256) slab_gather_rows_kernel(int nx, int row_first, int ext_rows,
                                                               const VShift<T>* __restrict__ vsh,
                                                               VShift<T>* __restrict__ vsh_out,
                                                               const VShift<T>* __restrict__ vsh2,
                                                               VShift<T>* __restrict__ vsh2_out,
                                                               const T* __restrict__ grho,
                                                               T* __restrict__ grho_out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ext_rows) return;
    const int r = (row_first + k) % nx;   // row_first in [0, nx)
    if (vsh != nullptr) vsh_out[k] = vsh[r];
    if (vsh2 != nullptr) vsh2_out[k] = vsh2[r];
    if (grho != nullptr) grho_out[k] = grho[r];
}

// out[i] = sum over column chunks c (ascending) of part[c][ghost + i], i < n_rows: the owned rows'
// trapezoid sums, added in the order the single-grid tails add the same partials.
template <typename T>
__global__ void __launch_bounds__(256) slab_row_sums_kernel(const T* __restrict__ part, int n_chunks,
                                                            int ext_rows, int ghost, int n_rows,
                                                            T* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rows) return;
    const T* p = part + ghost + i;
    T s = p[0];
    for (int c = 1; c < n_chunks; ++c) s += p[(size_t)c * ext_rows];
    out[i] = s;
}

template <typename T>
cudaError_t launch_slab_gather_rows(int nx, int row_first, int ext_rows, const VShift<T>* vsh, VShift<T>* vsh_out,
                                    const VShift<T>* vsh2, VShift<T>* vsh2_out, const T* grho, T* grho_out,
                                    cudaStream_t s) {
    slab_gather_rows_kernel<T><<<(ext_rows + 255) / 256, 256, 0, s>>>(nx, row_first, ext_rows, vsh, vsh_out,
                                                                      vsh2, vsh2_out, grho, grho_out);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_slab_row_sums(const T* part, int n_chunks, int ext_rows, int ghost, int n_rows, T* out,
                                 cudaStream_t s) {
    slab_row_sums_kernel<T><<<(n_rows + 255) / 256, 256, 0, s>>>(part, n_chunks, ext_rows, ghost, n_rows, out);
    count_launch();
    return cudaGetLastError();
}

#define VP_INST(T)                                                                              \
    template cudaError_t launch_slab_gather_rows<T>(int, int, int, const VShift<T>*, VShift<T>*, \
                                                    const VShift<T>*, VShift<T>*, const T*, T*, \
                                                    cudaStream_t);                              \
    template cudaError_t launch_slab_row_sums<T>(const T*, int, int, int, int, T*, cudaStream_t); \
    template cudaError_t launch_compute_rho<T>(int, int, const double*, const double*, int,     \
                                               double, T*, cudaStream_t);                       \
    template cudaError_t launch_poisson<T>(const PoissonTables<T>&, const T*, T*, int,          \
                                           cudaStream_t);                                       \
    template cudaError_t launch_electric_energy<T>(int, double, const T*, T*, cudaStream_t);    \
    template cudaError_t launch_semilag_x<T>(int, int, const double*, double, double, const T*, \
                                             T*, int, cudaStream_t);                            \
    template cudaError_t launch_semilag_v<T>(int, int, double, double, const T*, const T*, T*,  \
                                             int, const T*, T*, cudaStream_t);
VP_INST(float)
VP_INST(double)

}  // namespace vpb
