/*
 * C restatement of the reference's Vlasov-Poisson step and discrete adjoint, float64.
 *
 * TEST INFRASTRUCTURE ONLY (the CPU baseline and a fast checker): nothing in the product package
 * links or calls it. It follows the reference's loop structure: one iteration per (i, j) cell for
 * the semi-Lagrangian kernels (warp_vp_solver/kernels.py:109-153), one sequential trapezoid per
 * row for rho (kernels.py:156-172), a sequential trapezoid for ee (kernels.py:175-197), the legacy
 * forward loop (warp_vp_solver/solver.py:470-524) and the legacy adjoint (solver.py:778-932).
 * The per-cell loops are parallelised with OpenMP the way the reference's Warp launches are data
 * parallel. The adjoint scatters (kernels.py:215-273) are done per column (X^T) or per row (V^T),
 * which touches only that column or row, so no atomics are needed and the result is deterministic.
 * The Poisson step (warp_vp_solver/poisson.py:34-99, NumPy FFT in the reference) uses a textbook
 * iterative radix-2 FFT for power-of-two nx and a direct DFT otherwise, in float64.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int nx, nv;
    const double* xs;
    const double* vs;
    double dx, dv, period_x, period_v;
} grid_t;

/* kernels.py:47-69 */
static inline void periodic_indices(double xq, double x0, double h, int n, double period, int* i0,
                                    int* i1, double* t) {
    double x_rel = xq - x0;
    double x_wrapped = x_rel - floor(x_rel / period) * period;
    double idx_f = x_wrapped / h;
    int a = ((int)floor(idx_f)) % n;
    if (a < 0) a += n;
    *i0 = a;
    *i1 = (a + 1) % n;
    *t = idx_f - floor(idx_f);
}

static void semilag_x(const grid_t* g, double dt, const double* fin, double* fout) {
    const int nx = g->nx, nv = g->nv;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < (long)nx * nv; ++c) {
        const int i = (int)(c / nv), j = (int)(c % nv);
        const double x_foot = g->xs[i] - 0.5 * g->vs[j] * dt;
        int i0, i1;
        double t;
        periodic_indices(x_foot, g->xs[0], g->dx, nx, g->period_x, &i0, &i1, &t);
        fout[c] = (1.0 - t) * fin[(long)i0 * nv + j] + t * fin[(long)i1 * nv + j];
    }
}

static void semilag_v(const grid_t* g, double dt, const double* fin, const double* Etot, double* fout) {
    const int nx = g->nx, nv = g->nv;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < (long)nx * nv; ++c) {
        const int i = (int)(c / nv), j = (int)(c % nv);
        const double v_foot = g->vs[j] - Etot[i] * dt;
        int i0, i1;
        double t;
        periodic_indices(v_foot, g->vs[0], g->dv, nv, 2.0 * g->period_v, &i0, &i1, &t);
        fout[c] = (1.0 - t) * fin[(long)i * nv + i0] + t * fin[(long)i * nv + i1];
    }
}

static void compute_rho(const grid_t* g, const double* feq, const double* f, double* rho) {
    const int nx = g->nx, nv = g->nv;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        const double* a = feq + (long)i * nv;
        const double* b = f + (long)i * nv;
        double acc = 0.5 * (a[0] - b[0]);
        for (int k = 1; k < nv - 1; ++k) acc = acc + (a[k] - b[k]);
        acc = acc + 0.5 * (a[nv - 1] - b[nv - 1]);
        rho[i] = acc * g->dv;
    }
}

static double compute_ee(const grid_t* g, const double* E) {
    const int nx = g->nx;
    double acc = 0.5 * E[0] * E[0];
    for (int k = 1; k < nx - 1; ++k) acc = acc + E[k] * E[k];
    acc = acc + 0.5 * E[nx - 1] * E[nx - 1];
    return 0.5 * acc * g->dx;
}

/* ---- Poisson: E = real(ifft(m * fft(rho))), m_k = -1/(i 2 pi f_k) (poisson.py:34-69) ---- */

static void fft_inplace(double* re, double* im, int n, int inverse) {
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = re[i]; re[i] = re[j]; re[j] = tr;
            double ti = im[i]; im[i] = im[j]; im[j] = ti;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const double ang = (inverse ? 2.0 : -2.0) * M_PI / len;
        for (int s = 0; s < n; s += len) {
            for (int k = 0; k < len / 2; ++k) {
                const double wr = cos(ang * k), wi = sin(ang * k);
                const int a = s + k, b = s + k + len / 2;
                const double xr = re[b] * wr - im[b] * wi;
                const double xi = re[b] * wi + im[b] * wr;
                re[b] = re[a] - xr; im[b] = im[a] - xi;
                re[a] += xr; im[a] += xi;
            }
        }
    }
    if (inverse)
        for (int i = 0; i < n; ++i) { re[i] /= n; im[i] /= n; }
}

static void mult_imag(const grid_t* g, double* mi) {
    const int nx = g->nx;
    const double val = 1.0 / (nx * (g->period_x / nx));
    const int npos = (nx - 1) / 2 + 1;
    mi[0] = 0.0;
    for (int k = 1; k < nx; ++k) {
        const double f = (k < npos ? (double)k : (double)(k - nx)) * val;
        mi[k] = 1.0 / ((2.0 * M_PI) * f);
    }
}

/* out = real(ifft(m * fft(x))) (adjoint: conj(m)) */
static void poisson(const grid_t* g, const double* x, double* out, int adjoint) {
    const int nx = g->nx;
    double* re = (double*)malloc(sizeof(double) * nx * 3);
    double* im = re + nx;
    double* mi = im + nx;
    mult_imag(g, mi);
    const double sgn = adjoint ? -1.0 : 1.0;
    if ((nx & (nx - 1)) == 0) {
        for (int i = 0; i < nx; ++i) { re[i] = x[i]; im[i] = 0.0; }
        fft_inplace(re, im, nx, 0);
        for (int k = 0; k < nx; ++k) {   /* (0 + i*m)(a + i*b) = (-m*b, m*a) */
            const double a = re[k], b = im[k], m = sgn * mi[k];
            re[k] = -m * b;
            im[k] = m * a;
        }
        fft_inplace(re, im, nx, 1);
        for (int i = 0; i < nx; ++i) out[i] = re[i];
    } else {
        for (int k = 0; k < nx; ++k) {   /* direct DFT */
            double sr = 0.0, si = 0.0;
            for (int i = 0; i < nx; ++i) {
                const double ang = -2.0 * M_PI * (double)((long)k * i % nx) / nx;
                sr += x[i] * cos(ang);
                si += x[i] * sin(ang);
            }
            const double m = sgn * mi[k];
            re[k] = -m * si;
            im[k] = m * sr;
        }
        for (int i = 0; i < nx; ++i) {
            double s = 0.0;
            for (int k = 0; k < nx; ++k) {
                const double ang = 2.0 * M_PI * (double)((long)k * i % nx) / nx;
                s += re[k] * cos(ang) - im[k] * sin(ang);
            }
            out[i] = s / nx;
        }
    }
    free(re);
}

/* ---- adjoint kernels (kernels.py:215-322), deterministic ---- */

static void semilag_x_adjoint(const grid_t* g, double dt, const double* gout, double* gin) {
    const int nx = g->nx, nv = g->nv;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nv; ++j) {
        for (int i = 0; i < nx; ++i) gin[(long)i * nv + j] = 0.0;
        for (int i = 0; i < nx; ++i) {
            const double x_foot = g->xs[i] - 0.5 * g->vs[j] * dt;
            int i0, i1;
            double t;
            periodic_indices(x_foot, g->xs[0], g->dx, nx, g->period_x, &i0, &i1, &t);
            const double go = gout[(long)i * nv + j];
            gin[(long)i0 * nv + j] += (1.0 - t) * go;
            gin[(long)i1 * nv + j] += t * go;
        }
    }
}

static void semilag_v_adjoint(const grid_t* g, double dt, const double* gout, const double* fin,
                              const double* Etot, double* gin, double* gE) {
    const int nx = g->nx, nv = g->nv;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        double* gr = gin + (long)i * nv;
        const double* fr = fin + (long)i * nv;
        for (int j = 0; j < nv; ++j) gr[j] = 0.0;
        double acc = 0.0;
        for (int j = 0; j < nv; ++j) {
            const double v_foot = g->vs[j] - Etot[i] * dt;
            int i0, i1;
            double t;
            periodic_indices(v_foot, g->vs[0], g->dv, nv, 2.0 * g->period_v, &i0, &i1, &t);
            const double go = gout[(long)i * nv + j];
            gr[i0] += (1.0 - t) * go;
            gr[i1] += t * go;
            acc += -dt * ((fr[i1] - fr[i0]) / g->dv) * go;
        }
        gE[i] = acc;
    }
}

/* ---- time loops ---- */

int vpo_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Legacy forward (solver.py:470-524). f_hist: T*nx*nv (required), E_hist: T*nx, ee_hist: T. */
int vpo_forward(const grid_t* g, double dt, const double* feq, const double* f_iv, const double* H,
                int T, double* f_final, double* f_hist, double* E_hist, double* ee_hist) {
    const int nx = g->nx, nv = g->nv;
    const long nn = (long)nx * nv;
    double* fa = (double*)malloc(sizeof(double) * nn * 3 + sizeof(double) * nx * 3);
    if (!fa) return 1;
    double* fb = fa + nn;
    double* fc = fb + nn;
    double* rho = fc + nn;
    double* E = rho + nx;
    double* Et = E + nx;
    memcpy(fa, f_iv, sizeof(double) * nn);
    for (int t = 0; t < T; ++t) {
        semilag_x(g, dt, fa, fb);
        compute_rho(g, feq, fb, rho);
        poisson(g, rho, E, 0);
        const double ee = compute_ee(g, E);
        for (int i = 0; i < nx; ++i) Et[i] = E[i] + H[i];
        semilag_v(g, dt, fb, Et, fc);
        semilag_x(g, dt, fc, fa);
        memcpy(f_hist + (long)t * nn, fa, sizeof(double) * nn);
        if (E_hist) memcpy(E_hist + (long)t * nx, Et, sizeof(double) * nx);
        if (ee_hist) ee_hist[t] = ee;
    }
    if (f_final) memcpy(f_final, fa, sizeof(double) * nn);
    free(fa);
    return 0;
}

/* Legacy adjoint (solver.py:778-932). Cotangents may be NULL (zero). */
int vpo_backward(const grid_t* g, double dt, const double* feq, const double* f_iv, const double* H,
                 int T, const double* f_hist, const double* g_ff, const double* g_fh,
                 const double* g_Eh, const double* g_ee, double* g_fiv, double* g_H) {
    const int nx = g->nx, nv = g->nv;
    const long nn = (long)nx * nv;
    double* gf = (double*)malloc(sizeof(double) * nn * 4 + sizeof(double) * nx * 6);
    if (!gf) return 1;
    double* fh = gf + nn;
    double* g1 = fh + nn;
    double* g2 = g1 + nn;
    double* rho = g2 + nn;
    double* E = rho + nx;
    double* Et = E + nx;
    double* gEt = Et + nx;
    double* gE = gEt + nx;
    double* grho = gE + nx;
    if (g_ff) memcpy(gf, g_ff, sizeof(double) * nn); else memset(gf, 0, sizeof(double) * nn);
    memset(g_H, 0, sizeof(double) * nx);
    for (int t = T - 1; t >= 0; --t) {
        const double* fin = t == 0 ? f_iv : f_hist + (long)(t - 1) * nn;
        if (g_fh)
            for (long c = 0; c < nn; ++c) gf[c] += g_fh[(long)t * nn + c];
        semilag_x(g, dt, fin, fh);
        compute_rho(g, feq, fh, rho);
        poisson(g, rho, E, 0);
        for (int i = 0; i < nx; ++i) Et[i] = E[i] + H[i];
        semilag_x_adjoint(g, dt, gf, g1);
        semilag_v_adjoint(g, dt, g1, fh, Et, g2, gEt);
        for (int i = 0; i < nx; ++i) {
            gEt[i] += g_Eh ? g_Eh[(long)t * nx + i] : 0.0;
            g_H[i] += gEt[i];
            const double w = (i == 0 || i == nx - 1) ? 0.5 * g->dx : g->dx;
            gE[i] = gEt[i] + w * E[i] * (g_ee ? g_ee[t] : 0.0);
        }
        poisson(g, gE, grho, 1);
#pragma omp parallel for schedule(static)
        for (long c = 0; c < nn; ++c) {
            const int i = (int)(c / nv), j = (int)(c % nv);
            const double w = (j == 0 || j == nv - 1) ? -0.5 * g->dv : -g->dv;
            g2[c] += w * grho[i];
        }
        semilag_x_adjoint(g, dt, g2, gf);
    }
    memcpy(g_fiv, gf, sizeof(double) * nn);
    free(gf);
    return 0;
}
