// Strip step kernels for large grids (float32, x-invariant f_eq, Strang scheme).
//
// A time step of the forward loop (warp_vp_solver/solver.py:573-609) or of the discrete adjoint
// (solver.py:814-929) is two launches here: a strip kernel that advances the state and sums its
// rows, then a field kernel that solves Poisson for every row at once.
//
// Strip kernel. A CTA is one column group: 64 threads, each owning the 4 columns of a quad (the
// quads, their x weights, f_eq differences and smallest shifts are the persistent path's tables,
// vp_pst.cuh). The work of a step is the n_chunks x n_bands tiles of R rows x 256 columns; the
// bands of every chunk are split into the same `runs` runs of consecutive bands, one CTA per (chunk,
// run), so CTAs of neighbouring chunks work on the same rows at the same time and read each other's
// 4-column halos from L2. Walking down a run, consecutive bands' windows overlap
// in all but R rows, so the CTA keeps the window rows in a shared-memory ring: while band i
// computes, the R rows that band i + 1 adds are in flight (16-byte cp.async, one commit group per
// band), and each row of the state is read from HBM once per chunk (the 4-column halo on each side
// is 3 % extra). The tile arithmetic is the persistent loop's (same operation order, so the two
// paths agree to rounding of the field only).
//
// Row sums. A tile's R row sums go to part[chunk][row]; a per-run counter tells the CTA that
// finishes the run's last chunk, which sums the chunks in ascending order (deterministic) into rho
// (forward) or g_E of the previous step (adjoint) for the run's rows and resets the counter for the
// next launch.
//
// Field kernel. E_i = sum_k c[(i - k) mod nx] rho_k (c = real(ifft(m)), the circulant form of
// warp_vp_solver/poisson.py:34-69; Poisson^T uses c[(k - i) mod nx], poisson.py:72-99): a CTA
// computes 32 rows; thread t takes blocks of 8 k values (t, t + 256, ...) and accumulates all 32
// rows from a window of 40 coefficients in registers (256 multiply-adds per 12 vector loads), then a
// fixed-order butterfly and a fixed-order sum over the 8 warps. The forward kernel also writes
// E_hist, the tape's E and v shifts, and the energy: per-CTA partials in float64 that the last CTA
// sums in ascending order.

#include "vp_pst.cuh"

#include <algorithm>
#include <vector>

namespace vpb {

namespace {

constexpr int kFieldThreads = 256;
constexpr int kFieldWarps = kFieldThreads / 32;
constexpr int kStripMaxSmem = 200 * 1024;   // dynamic shared memory cap of a strip CTA

__device__ __forceinline__ void strip_cp8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(pst_smem(dst)), "l"(src) : "memory");
}

// Ring row of a column group of GT threads: 4 GT columns and 4 halo columns on each side.
__host__ __device__ constexpr int strip_row(int GT) { return 4 * GT + 8; }

// Shared memory of a forward CTA: NR ring rows, their shift records, the row-sum scratch.
constexpr size_t strip_fwd_bytes(int NR, int R, int GT) {
    return (size_t)NR * strip_row(GT) * 4 + (size_t)NR * 8 + (size_t)2 * R * 4;
}

// Adjoint CTA: NR ring rows of w_n with their shift records and rho cotangents, two buffers of the
// band's R own rows of h_{n-1} with their shifts, the row-sum scratch.
constexpr size_t strip_bwd_bytes(int NR, int R, int GT) {
    return (size_t)NR * strip_row(GT) * 4 + (size_t)2 * R * strip_row(GT) * 4 + (size_t)NR * 8 + (size_t)NR * 4 +
           (size_t)2 * R * 4 + (size_t)2 * R * 4;
}

// acc[R] summed over each warp (transposed butterfly) into red[warp][row]; after the next block
// barrier, thread r < R forms the row's sum over the NW warps in order (strip_rows_total).
template <int R>
__device__ __forceinline__ void strip_rows_stage(float (&acc)[R], float* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
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
}

template <int R, int NW>
__device__ __forceinline__ float strip_rows_total(const float* red) {
    if (threadIdx.x >= R) return 0.f;
    float s = red[threadIdx.x];
#pragma unroll
    for (int w = 1; w < NW; ++w) s += red[w * R + threadIdx.x];
    return s;
}

// After a CTA has written the row partials of all bands of its run: returns true in every thread
// of the CTA that completed the run's last chunk (every chunk's run i covers the same bands), after
// which the partials of all chunks are visible to it; the counter is reset for the next launch.
// One fence and one atomic per run (the grid-barrier pattern: block barrier, then one thread).
__device__ __forceinline__ bool strip_run_done(unsigned* run_ctr, int n_chunks, int* s_last) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const bool last = atomicAdd(run_ctr, 1u) == (unsigned)(n_chunks - 1);
        if (last) {
            *run_ctr = 0u;
            __threadfence();
        }
        *s_last = last ? 1 : 0;
    }
    __syncthreads();
    return *s_last != 0;
}

// Run i of a chunk: bands [i n_bands / runs, (i + 1) n_bands / runs). A single-instance launch
// gives CTA blockIdx.x run blockIdx.x mod runs of chunk blockIdx.x / runs, so the CTAs of one run in
// neighbouring chunks work on the same rows at the same time and the 4-column halos they read from
// each other stay in L2.
__device__ __forceinline__ void strip_run_bands(int run, int runs, int n_bands, int* b0, int* nb) {
    *b0 = (int)((long long)run * n_bands / runs);
    *nb = (int)((long long)(run + 1) * n_bands / runs) - *b0;
}

// In-halo shift forms. A thread holds the 8 staged cells w[i] = row[j0 + base + i] (two aligned
// 16-byte loads, base = -4 or 0) and the f_eq differences Dw[i] = D[j0 - 4 + i], i < 12, of its
// quad (D[j] = f_eq[j + 1] - f_eq[j], rounded once from float64). For a shift M in [-4, 3]:
//   forward V:  o_e = (h[j + M] + A) + t ((h[j + M + 1] - h[j + M]) + D[j + M]),
//               A = f_eq[j + M] - f_eq[j] = sum of D over [j, j + M) (negated for M < 0)
//               (for M = 0 and -1 this is the same arithmetic as the fast forms);
//   adjoint V^T: g_e = w[j - M] + t (w[j - M - 1] - w[j - M]);
//   slope:       s_e = (h[j + M + 1] - h[j + M]) + D[j + M]   (the f_eq slope table B_M exactly).
template <int M>
__device__ __forceinline__ void strip_v_form(const float (&w)[8], const float (&Dw)[12], float tv, float (&o)[4]) {
    constexpr int S = M < 0 ? M + 4 : M;   // index of h[j0 + M] in w
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        float A = 0.f;
        if constexpr (M > 0) {
#pragma unroll
            for (int i = 0; i < M; ++i) A += Dw[4 + e + i];
        } else if constexpr (M < 0) {
#pragma unroll
            for (int i = M; i < 0; ++i) A -= Dw[4 + e + i];
        }
        o[e] = (w[S + e] + A) + tv * ((w[S + e + 1] - w[S + e]) + Dw[4 + e + M]);
    }
}

template <int M>
__device__ __forceinline__ void strip_vt_form(const float (&w)[8], float tv, float (&o)[4]) {
    constexpr int base = M >= 0 ? -4 : 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float a = w[e - M - base], b = w[e - M - 1 - base];
        o[e] = a + tv * (b - a);
    }
}

template <int M>
__device__ __forceinline__ void strip_slope_form(const float (&w)[8], const float (&Dw)[12], float (&o)[4]) {
    constexpr int S = M < 0 ? M + 4 : M;
#pragma unroll
    for (int e = 0; e < 4; ++e) o[e] = (w[S + e + 1] - w[S + e]) + Dw[4 + e + M];
}

// The 8 cells of a staged row at j0 + base .. j0 + base + 7 (sr points at j0).
__device__ __forceinline__ void strip_load8(const float* sr, int base, float (&w)[8]) {
    const float4 u = *reinterpret_cast<const float4*>(sr + base);
    const float4 v = *reinterpret_cast<const float4*>(sr + base + 4);
    w[0] = u.x; w[1] = u.y; w[2] = u.z; w[3] = u.w;
    w[4] = v.x; w[5] = v.y; w[6] = v.z; w[7] = v.w;
}

// Forward V of one quad row for a shift in [-4, 3] other than 0 and -1.
__device__ __forceinline__ void strip_v_general(const float* sr, int ms, const float (&Dw)[12], float tv,
                                                float (&o)[4]) {
    float w[8];
    strip_load8(sr, ms < 0 ? -4 : 0, w);
    switch (ms) {
        case -4: strip_v_form<-4>(w, Dw, tv, o); break;
        case -3: strip_v_form<-3>(w, Dw, tv, o); break;
        case -2: strip_v_form<-2>(w, Dw, tv, o); break;
        case 1: strip_v_form<1>(w, Dw, tv, o); break;
        case 2: strip_v_form<2>(w, Dw, tv, o); break;
        default: strip_v_form<3>(w, Dw, tv, o); break;
    }
}

__device__ __forceinline__ void strip_vt_general(const float* sr, int ms, float tv, float (&o)[4]) {
    float w[8];
    strip_load8(sr, ms >= 0 ? -4 : 0, w);
    switch (ms) {
        case -4: strip_vt_form<-4>(w, tv, o); break;
        case -3: strip_vt_form<-3>(w, tv, o); break;
        case -2: strip_vt_form<-2>(w, tv, o); break;
        case 1: strip_vt_form<1>(w, tv, o); break;
        case 2: strip_vt_form<2>(w, tv, o); break;
        default: strip_vt_form<3>(w, tv, o); break;
    }
}

__device__ __forceinline__ void strip_slope_general(const float* hr, int ms, const float (&Dw)[12], float (&o)[4]) {
    float w[8];
    strip_load8(hr, ms < 0 ? -4 : 0, w);
    switch (ms) {
        case -4: strip_slope_form<-4>(w, Dw, o); break;
        case -3: strip_slope_form<-3>(w, Dw, o); break;
        case -2: strip_slope_form<-2>(w, Dw, o); break;
        case 1: strip_slope_form<1>(w, Dw, o); break;
        case 2: strip_slope_form<2>(w, Dw, o); break;
        default: strip_slope_form<3>(w, Dw, o); break;
    }
}

// D[j0 - 4 .. j0 + 7] (periodic in j).
__device__ __forceinline__ void strip_dwin(const float* __restrict__ dfeq, int j0, int nv, float (&Dw)[12]) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(dfeq + (j0 == 0 ? nv - 4 : j0 - 4)));
    const float4 b = __ldg(reinterpret_cast<const float4*>(dfeq + j0));
    const float4 c = __ldg(reinterpret_cast<const float4*>(dfeq + (j0 + 4 == nv ? 0 : j0 + 4)));
    Dw[0] = a.x; Dw[1] = a.y; Dw[2] = a.z; Dw[3] = a.w;
    Dw[4] = b.x; Dw[5] = b.y; Dw[6] = b.z; Dw[7] = b.w;
    Dw[8] = c.x; Dw[9] = c.y; Dw[10] = c.z; Dw[11] = c.w;
}

// a + t (b - a) on two columns at once, each lane rounded exactly as pst_lerp (b - a, then one fma).
__device__ __forceinline__ float2 strip_lerp2(float2 a, float2 b, float2 t) {
    return __ffma2_rn(t, __ffma2_rn(a, make_float2(-1.f, -1.f), b), a);
}

// Stores a quad's 4 values of ring row `slot` into the ring, column e two rows earlier (slot - 2,
// mod NR) when bit e of smask is set. Phase B then reads one row of 4 values per window row for all
// of its columns, whichever of the quad's two x shifts each column has.
template <int SW>
__device__ __forceinline__ void strip_put(float* ring, int NR, int slot, int gt, int smask, float v0, float v1,
                                          float v2, float v3) {
    float* p = ring + (size_t)slot * SW + 4 + 4 * gt;
    if (smask == 0) {
        *reinterpret_cast<float4*>(p) = make_float4(v0, v1, v2, v3);
        return;
    }
    int s2 = slot - 2;
    s2 += s2 < 0 ? NR : 0;
    float* q = ring + (size_t)s2 * SW + 4 + 4 * gt;
    if (smask == 0xF) {
        *reinterpret_cast<float4*>(q) = make_float4(v0, v1, v2, v3);
        return;
    }
    (smask & 1 ? q : p)[0] = v0;
    (smask & 2 ? q : p)[1] = v1;
    (smask & 4 ? q : p)[2] = v2;
    (smask & 8 ? q : p)[3] = v3;
}

// Column index c (in [-4, nv + 4)) reduced mod nv.
__device__ __forceinline__ int strip_col(int c, int nv) { return c < 0 ? c + nv : (c >= nv ? c - nv : c); }

// Sum over the chunks (ascending) of the partials of row i.
__device__ __forceinline__ float strip_chunk_sum(const float* part, int nx, int n_chunks, int i) {
    float sum = 0.f;
    for (int c = 0; c < n_chunks; ++c) sum += __ldcg(part + (size_t)c * nx + i);
    return sum;
}

}  // namespace

template <int R, int GT>
__device__ __forceinline__ void strip_fwd_body(const StripFwdArgs& a, unsigned char* smem, int* s_last, int c, int run_idx) {
    constexpr int SW = strip_row(GT);
    const int nx = a.nx, nv = a.nv, NR = a.ring_rows;   // NR = (L + 1) R ring rows
    const int gt = threadIdx.x;
    float* ring = reinterpret_cast<float*>(smem);                      // [NR][SW]
    int2* rinf = reinterpret_cast<int2*>(ring + (size_t)NR * SW);    // [NR] (m mod nv, t)
    float* red = reinterpret_cast<float*>(rinf + NR);                  // [2][R]
    const bool next = a.h_out != nullptr;
    const bool sums = next && a.part != nullptr;
    const bool fout = a.f_hist_n != nullptr || a.f_final != nullptr;
    int b0, nb;
    strip_run_bands(run_idx, a.runs, a.n_bands, &b0, &nb);
    if (nb <= 0) return;   // (the same run is empty in every chunk: no counter involved)
    const int2 cm = __ldg(a.chunk + c);             // smallest / largest quad shift of the chunk
    const int span = 2 * (cm.y - cm.x) + R + 4;      // window rows of a band
    const int L = (span + R - 1) / R;               // slabs of R rows a window spans
    const int origin = b0 * R + 2 * cm.x;           // global row of ring row 0 (unreduced)
    const int c0 = c * (4 * GT);
    const int q = c * GT + gt, j0 = c0 + 4 * gt;
    const int2 qi = __ldg(a.quad + q);
    const float4 t4 = __ldg(a.tq + q);
    float Dw[12];
    strip_dwin(a.dfeq, j0, nv, Dw);
    const float tt[4] = {t4.x, t4.y, t4.z, t4.w};
    const float w0 = j0 == 0 ? 0.5f : 1.f, w3 = j0 + 3 == nv - 1 ? 0.5f : 1.f;
    const int col0 = strip_col(c0 - 4 + 4 * gt, nv);
    const int col1 = strip_col(c0 - 4 + 4 * (gt + GT), nv);
    const bool two = gt < (GT + 2) - GT;
    const int n_slabs = nb + L - 1;

    // slab g: ring rows g R .. g R + R - 1 (slots (g R + r) mod NR; NR / R >= L + 1 slabs) with their
    // shift records
    // slabs are issued in order: the next one's first slot and global row advance by R
    int is_slot = 0, is_row = pst_wrap(origin, nx);
    auto issue_slab = [&](int g) {
        const int s0 = is_slot;
        int grow = is_row;
        is_slot = is_slot + R == NR ? 0 : is_slot + R;
        is_row += R;
        is_row -= is_row >= nx ? nx : 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float* src = a.h_in + (size_t)grow * nv;
            float* dst = ring + (size_t)(s0 + r) * SW;
            pst_cp16(dst + 4 * gt, src + col0);
            if (two) pst_cp16(dst + 4 * (gt + GT), src + col1);
            if (gt == r) strip_cp8(rinf + s0 + r, a.vsh + grow);
            grow = grow + 1 == nx ? 0 : grow + 1;
        }
        pst_cp_commit();
    };
    issue_slab(0);
    if (n_slabs > 1) issue_slab(1);

    int a_slot = 0, b_slot = 0;   // first slots of slab g and of band g - L + 1
    for (int g = 0; g < n_slabs; ++g) {
        if (g + 1 < n_slabs) pst_cp_wait(1);
        else pst_cp_wait(0);
        __syncthreads();
        // phase A: o = V(h) + V(f_eq) - f_eq on the slab's rows, in place; every thread works on the
        // same row at a time, so the row's shift selects one form for the whole CTA
        const int s0 = a_slot;
        a_slot = a_slot + R == NR ? 0 : a_slot + R;
        float ov[R][4];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int2 ri = rinf[s0 + r];
            const float tv = __int_as_float(ri.y);
            const float* sr = ring + (size_t)(s0 + r) * SW + 4 + 4 * gt;
            float* o = ov[r];
            if (ri.x == 0) {
                const float4 h = *reinterpret_cast<const float4*>(sr);
                const float h4 = sr[4];
                o[0] = h.x + tv * ((h.y - h.x) + Dw[4]);
                o[1] = h.y + tv * ((h.z - h.y) + Dw[5]);
                o[2] = h.z + tv * ((h.w - h.z) + Dw[6]);
                o[3] = h.w + tv * ((h4 - h.w) + Dw[7]);
            } else if (ri.x == nv - 1) {   // shift -1
                const float hm = sr[-1];
                const float4 h = *reinterpret_cast<const float4*>(sr);
                o[0] = (hm - Dw[3]) + tv * ((h.x - hm) + Dw[3]);
                o[1] = (h.x - Dw[4]) + tv * ((h.y - h.x) + Dw[4]);
                o[2] = (h.y - Dw[5]) + tv * ((h.z - h.y) + Dw[5]);
                o[3] = (h.z - Dw[6]) + tv * ((h.w - h.z) + Dw[6]);
            } else {
                const int ms = ri.x > nv / 2 ? ri.x - nv : ri.x;
                if (ms >= -4 && ms <= 3) {
                    strip_v_general(sr, ms, Dw, tv, ov[r]);
                } else {   // beyond the staged halo: float64 form from global memory
                    const float4 r4 = pst_v_rare(a.vtab, a.feq, nv, sr, a.h_in, ms, tv,
                                                 pst_wrap(origin + g * R + r, nx), j0);
                    o[0] = r4.x;
                    o[1] = r4.y;
                    o[2] = r4.z;
                    o[3] = r4.w;
                }
            }
        }
        __syncthreads();   // every thread has read the slab's h (its neighbours' halo cells included)
        // a column whose x shift is bm + 1 reads its window two rows further: its o goes two rows
        // earlier, so that window row k of every column of the quad is ring row zb + k below
#pragma unroll
        for (int r = 0; r < R; ++r) strip_put<SW>(ring, NR, s0 + r, gt, qi.y, ov[r][0], ov[r][1], ov[r][2], ov[r][3]);
        __syncthreads();
        // phase B: band i = g - L + 1, whose window (ring rows i R .. i R + span - 1) is complete
        const int i = g - L + 1;
        const int r0 = (b0 + i) * R;
        if (i >= 0) {
            // this thread's window row k is ring row i R + 2 (bm - cm.x) + k, global r0 + 2 bm + k
            int zb = b_slot + 2 * (qi.x - cm.x);
            b_slot = b_slot + R == NR ? 0 : b_slot + R;
            zb -= zb >= NR ? NR : 0;
            const float2 ta = make_float2(tt[0], tt[1]), tb = make_float2(tt[2], tt[3]);
            const float2 wa = make_float2(w0, 1.f), wb = make_float2(1.f, w3);
            float2 acc2[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc2[r] = make_float2(0.f, 0.f);
            float2 pa, pb, dpa, dpb;
#pragma unroll
            for (int k = 0; k < R + 2; ++k) {
                int sl = zb + k;
                sl -= sl >= NR ? NR : 0;
                const float4 o4 = *reinterpret_cast<const float4*>(ring + (size_t)sl * SW + 4 + 4 * gt);
                const float2 oa = make_float2(o4.x, o4.y), ob = make_float2(o4.z, o4.w);
                if (k >= 1) {
                    // d row qd from window rows qd, qd + 1
                    const int qd = k - 1;
                    const float2 da = strip_lerp2(pa, oa, ta), db = strip_lerp2(pb, ob, tb);
                    const float dn[4] = {da.x, da.y, db.x, db.y};
                    if (fout && qd < R) {
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const int row = pst_wrap(r0 + qi.x + ((qi.y >> e) & 1) + qd, nx);
                            const double f = __ldg(a.feq + j0 + e) + (double)dn[e];
                            if (a.f_hist_n != nullptr) a.f_hist_n[(size_t)row * nv + j0 + e] = (float)f;
                            if (a.f_final != nullptr) a.f_final[(size_t)row * nv + j0 + e] = f;
                        }
                    }
                    if (qd >= 1 && next) {
                        const int r = qd - 1;
                        const float2 ha = strip_lerp2(dpa, da, ta), hb = strip_lerp2(dpb, db, tb);
                        *reinterpret_cast<float4*>(a.h_out + (size_t)(r0 + r) * nv + j0) =
                            make_float4(ha.x, ha.y, hb.x, hb.y);
                        // trapezoid-weighted row sum: (w0 h0 + h2, h1 + w3 h3)
                        acc2[r] = __fadd2_rn(acc2[r], __ffma2_rn(wb, hb, __fmul2_rn(wa, ha)));
                    }
                    dpa = da;
                    dpb = db;
                }
                pa = oa;
                pb = ob;
            }
            if (sums) {
                float acc[R];
#pragma unroll
                for (int r = 0; r < R; ++r) acc[r] = acc2[r].x + acc2[r].y;
                strip_rows_stage<R>(acc, red);
            }
        }
        __syncthreads();   // band i's first slab is free, the row sums staged
        if (g + 2 < n_slabs) issue_slab(g + 2);
        if (i >= 0 && sums && gt < R) a.part[(size_t)c * nx + r0 + gt] = strip_rows_total<R, GT / 32>(red);
    }
    // rho of the run's rows, once every chunk has published them
    if (sums && strip_run_done(a.run_ctr + run_idx, a.n_chunks, s_last))
        for (int row = b0 * R + gt; row < (b0 + nb) * R; row += GT)
            a.rho_out[row] = -a.dv * strip_chunk_sum(a.part, nx, a.n_chunks, row);
}

// 640 / GT CTAs per SM: 10 two-warp CTAs (up to 96 registers) measured 4 % faster on 8192^2 than
// 12 (80 registers), which the shared memory of the ring would also allow
template <int R, int GT>
__global__ void __launch_bounds__(GT, 640 / GT) vp_strip_fwd_kernel(const StripFwdArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_last;
    strip_fwd_body<R, GT>(a, smem, &s_last, blockIdx.x / a.runs, blockIdx.x % a.runs);
}

template <int R, int GT>
__device__ __forceinline__ void strip_bwd_body(const StripBwdArgs& a, unsigned char* smem, int* s_last, int c, int run_idx) {
    constexpr int SW = strip_row(GT);
    const int nx = a.nx, nv = a.nv, NR = a.ring_rows;
    const int gt = threadIdx.x;
    float* ring = reinterpret_cast<float*>(smem);                       // [NR][SW] rows of w_n
    float* hring = ring + (size_t)NR * SW;                           // [2][R][SW] rows of h_{n-1}
    int2* rinf = reinterpret_cast<int2*>(hring + (size_t)2 * R * SW);   // [NR] step n shifts
    float* rgr = reinterpret_cast<float*>(rinf + NR);                   // [NR] rho cotangents
    int* hinf = reinterpret_cast<int*>(rgr + NR);                       // [2][R] step n-1 shifts
    float* red = reinterpret_cast<float*>(hinf + 2 * R);                // [2][R]
    int b0, nb;
    strip_run_bands(run_idx, a.runs, a.n_bands, &b0, &nb);
    if (nb <= 0) return;
    const int2 cm = __ldg(a.chunk + c);
    const int span = 2 * (cm.y - cm.x) + R + 4;
    const int L = (span + R - 1) / R;
    const int origin = b0 * R - 2 * cm.y - 4;       // the thread of shift m reads rows r0 - 2m - 4 + k
    const int c0 = c * (4 * GT);
    const int q = c * GT + gt, j0 = c0 + 4 * gt;
    const int2 qi = __ldg(a.quad + q);
    const float4 t4 = __ldg(a.tq + q);
    float Dw[12];
    strip_dwin(a.dfeq, j0, nv, Dw);
    const float tt[4] = {t4.x, t4.y, t4.z, t4.w};
    const float wr0 = j0 == 0 ? -0.5f * a.dv : -a.dv;   // rho^T weights (kernels.py:276-299)
    const float wr3 = j0 + 3 == nv - 1 ? -0.5f * a.dv : -a.dv;
    const int col0 = strip_col(c0 - 4 + 4 * gt, nv);
    const int col1 = strip_col(c0 - 4 + 4 * (gt + GT), nv);
    const bool two = gt < (GT + 2) - GT;
    const int n_slabs = nb + L - 1;

    // slab g of w_n (ring rows g R .. g R + R - 1) with shifts and rho cotangents, and the own rows of
    // h_{n-1} of band g - L + 1 (buffer band & 1) with their shifts: one commit group
    // slabs are issued in order: the next one's first slot and global row advance by R
    int is_slot = 0, is_row = pst_wrap(origin, nx);
    auto issue_slab = [&](int g) {
        const int s0 = is_slot;
        int grow = is_row;
        is_slot = is_slot + R == NR ? 0 : is_slot + R;
        is_row += R;
        is_row -= is_row >= nx ? nx : 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const float* src = a.w_in + (size_t)grow * nv;
            float* dst = ring + (size_t)(s0 + r) * SW;
            pst_cp16(dst + 4 * gt, src + col0);
            if (two) pst_cp16(dst + 4 * (gt + GT), src + col1);
            if (gt == r) {
                strip_cp8(rinf + s0 + r, a.vsh_n + grow);
                pst_cp4(rgr + s0 + r, a.grho + grow);
            }
            grow = grow + 1 == nx ? 0 : grow + 1;
        }
        const int band = g - L + 1;
        if (band >= 0 && band < nb) {
            const int hr0 = (b0 + band) * R;
            float* hb = hring + (size_t)(band & 1) * R * SW;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float* src = a.h_prev + (size_t)(hr0 + r) * nv;
                pst_cp16(hb + (size_t)r * SW + 4 * gt, src + col0);
                if (two) pst_cp16(hb + (size_t)r * SW + 4 * (gt + GT), src + col1);
            }
            if (gt < R) pst_cp4(hinf + (band & 1) * R + gt, &a.vsh_prev[hr0 + gt].m);
        }
        pst_cp_commit();
    };
    issue_slab(0);
    if (n_slabs > 1) issue_slab(1);

    int a_slot = 0, b_slot = 0;   // first slots of slab g and of band g - L + 1
    for (int g = 0; g < n_slabs; ++g) {
        if (g + 1 < n_slabs) pst_cp_wait(1);
        else pst_cp_wait(0);
        __syncthreads();
        const int s0 = a_slot;
        a_slot = a_slot + R == NR ? 0 : a_slot + R;
        const int i = g - L + 1;                    // band whose window completes with this slab
        float* hb = hring + (size_t)(i & 1) * R * SW + 4 + 4 * gt;
        // phase A: gh = V^T w + rho^T grho on the slab's rows and, for band i, the slopes
        // (h + f_eq)[j + m + 1] - (h + f_eq)[j + m] of its own rows of h_{n-1}; in place, one row
        // (one shift) at a time for the whole CTA
        float gv[R][4], sv[R][4];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int2 ri = rinf[s0 + r];
            const float tv = __int_as_float(ri.y), gr = rgr[s0 + r];
            const float* sr = ring + (size_t)(s0 + r) * SW + 4 + 4 * gt;
            float* o = gv[r];
            if (ri.x == 0) {
                const float hm = sr[-1];
                const float4 h = *reinterpret_cast<const float4*>(sr);
                o[0] = h.x + tv * (hm - h.x);
                o[1] = h.y + tv * (h.x - h.y);
                o[2] = h.z + tv * (h.y - h.z);
                o[3] = h.w + tv * (h.z - h.w);
            } else if (ri.x == nv - 1) {   // shift -1
                const float4 h = *reinterpret_cast<const float4*>(sr);
                const float h4 = sr[4];
                o[0] = h.y + tv * (h.x - h.y);
                o[1] = h.z + tv * (h.y - h.z);
                o[2] = h.w + tv * (h.z - h.w);
                o[3] = h4 + tv * (h.w - h4);
            } else {
                const int ms = ri.x > nv / 2 ? ri.x - nv : ri.x;
                if (ms >= -4 && ms <= 3) {
                    strip_vt_general(sr, ms, tv, gv[r]);
                } else {
                    const float4 v4 = pst_vt_rare(sr, a.w_in, nv, ms, tv, pst_wrap(origin + g * R + r, nx), j0);
                    o[0] = v4.x;
                    o[1] = v4.y;
                    o[2] = v4.z;
                    o[3] = v4.w;
                }
            }
            o[0] += wr0 * gr;
            o[1] -= a.dv * gr;
            o[2] -= a.dv * gr;
            o[3] += wr3 * gr;
        }
        if (i >= 0) {
            const int* hi = hinf + (i & 1) * R;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int mh = hi[r];
                const float* hr = hb + (size_t)r * SW;
                float* o = sv[r];
                if (mh == 0) {
                    const float4 h = *reinterpret_cast<const float4*>(hr);
                    const float h4 = hr[4];
                    o[0] = (h.y - h.x) + Dw[4];
                    o[1] = (h.z - h.y) + Dw[5];
                    o[2] = (h.w - h.z) + Dw[6];
                    o[3] = (h4 - h.w) + Dw[7];
                } else if (mh == nv - 1) {
                    const float hm = hr[-1];
                    const float4 h = *reinterpret_cast<const float4*>(hr);
                    o[0] = (h.x - hm) + Dw[3];
                    o[1] = (h.y - h.x) + Dw[4];
                    o[2] = (h.z - h.y) + Dw[5];
                    o[3] = (h.w - h.z) + Dw[6];
                } else {
                    const int ms = mh > nv / 2 ? mh - nv : mh;
                    if (ms >= -4 && ms <= 3) {
                        strip_slope_general(hr, ms, Dw, sv[r]);
                    } else {
                        const float4 s4 =
                            pst_slope_rare(hr, a.h_prev, a.vtab, a.feq, nv, ms, (b0 + i) * R + r, j0);
                        o[0] = s4.x;
                        o[1] = s4.y;
                        o[2] = s4.z;
                        o[3] = s4.w;
                    }
                }
            }
        }
        __syncthreads();   // every thread has read the rows it converts' neighbours
        // a column whose x shift is bm reads its window two rows further than one of bm + 1: its gh
        // goes two rows earlier, so that window row k of every column is ring row zb + k below
#pragma unroll
        for (int r = 0; r < R; ++r)
            strip_put<SW>(ring, NR, s0 + r, gt, ~qi.y & 0xF, gv[r][0], gv[r][1], gv[r][2], gv[r][3]);
        if (i >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                *reinterpret_cast<float4*>(hb + (size_t)r * SW) = make_float4(sv[r][0], sv[r][1], sv[r][2], sv[r][3]);
        }
        __syncthreads();
        // phase B: band i: c = X^T gh (+ the f_hist cotangent), w_{n-1} = X^T c, slope products
        const int r0 = (b0 + i) * R;
        if (i >= 0) {
            int zb = b_slot + 2 * (cm.y - qi.x);
            b_slot = b_slot + R == NR ? 0 : b_slot + R;
            zb -= zb >= NR ? NR : 0;
            const float2 ta = make_float2(tt[0], tt[1]), tb = make_float2(tt[2], tt[3]);
            float2 acc2[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc2[r] = make_float2(0.f, 0.f);
            float2 ga, gb, cpa, cpb;
#pragma unroll
            for (int k = 0; k < R + 2; ++k) {
                int sl = zb + k;
                sl -= sl >= NR ? NR : 0;
                const float4 g4 = *reinterpret_cast<const float4*>(ring + (size_t)sl * SW + 4 + 4 * gt);
                const float2 xa = make_float2(g4.x, g4.y), xb = make_float2(g4.z, g4.w);
                if (k >= 1) {
                    // c row q2 from window rows q2 (g0) and q2 + 1 (g1): c = g1 + t (g0 - g1)
                    const int q2 = k - 1;
                    float2 ca = strip_lerp2(xa, ga, ta), cb = strip_lerp2(xb, gb, tb);
                    if (a.gfh != nullptr) {
                        const float* gr = a.gfh + j0;
                        ca.x += __ldg(gr + (size_t)pst_wrap(r0 - qi.x - (qi.y & 1) - 1 + q2, nx) * nv);
                        ca.y += __ldg(gr + (size_t)pst_wrap(r0 - qi.x - ((qi.y >> 1) & 1) - 1 + q2, nx) * nv + 1);
                        cb.x += __ldg(gr + (size_t)pst_wrap(r0 - qi.x - ((qi.y >> 2) & 1) - 1 + q2, nx) * nv + 2);
                        cb.y += __ldg(gr + (size_t)pst_wrap(r0 - qi.x - ((qi.y >> 3) & 1) - 1 + q2, nx) * nv + 3);
                    }
                    if (q2 >= 1) {
                        // w row r = q2 - 1 (own row r0 + r) and its slope products
                        const int r = q2 - 1;
                        const float2 wa = strip_lerp2(ca, cpa, ta), wb = strip_lerp2(cb, cpb, tb);
                        if (a.w_out != nullptr)
                            *reinterpret_cast<float4*>(a.w_out + (size_t)(r0 + r) * nv + j0) =
                                make_float4(wa.x, wa.y, wb.x, wb.y);
                        const float4 s4 = *reinterpret_cast<const float4*>(hb + (size_t)r * SW);
                        acc2[r] = __ffma2_rn(make_float2(s4.z, s4.w), wb,
                                             __ffma2_rn(make_float2(s4.x, s4.y), wa, acc2[r]));
                    }
                    cpa = ca;
                    cpb = cb;
                }
                ga = xa;
                gb = xb;
            }
            float acc[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = acc2[r].x + acc2[r].y;
            strip_rows_stage<R>(acc, red);
        }
        __syncthreads();   // band i's first slab and its h buffer are free, the row sums staged
        if (g + 2 < n_slabs) issue_slab(g + 2);
        if (i >= 0 && gt < R) a.part[(size_t)c * nx + r0 + gt] = strip_rows_total<R, GT / 32>(red);
    }
    if (strip_run_done(a.run_ctr + run_idx, a.n_chunks, s_last)) {
        // tail of step n - 1 for the run's rows (warp_vp_solver/solver.py:870-929)
        const float gee = a.gee != nullptr ? __ldg(a.gee) : 0.f;
        for (int row = b0 * R + gt; row < (b0 + nb) * R; row += GT) {
            float gEt = a.neg_dt_dv * strip_chunk_sum(a.part, nx, a.n_chunks, row);
            if (a.gE_hist != nullptr) gEt += __ldg(a.gE_hist + row);
            a.gH[row] += gEt;
            a.gE_out[row] = gEt + a.dx * trap_w<float>(row, nx) * __ldg(a.E_prev + row) * gee;
        }
    }
}

template <int R, int GT>
__global__ void __launch_bounds__(GT, 512 / GT) vp_strip_bwd_kernel(const StripBwdArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_last;
    strip_bwd_body<R, GT>(a, smem, &s_last, blockIdx.x / a.runs, blockIdx.x % a.runs);
}

// Rows blk * 32 .. blk * 32 + 31 of the field; nblk CTAs solve the whole field (their energy
// partials are summed by the last of them).
__device__ __forceinline__ void strip_field_body(const StripFieldArgs& a, int blk, int nblk) {
    constexpr int FR = kStripFieldRows;
    __shared__ float red[kFieldWarps][FR];
    __shared__ double s_e[FR];
    __shared__ int s_last;
    const int nx = a.nx;
    const int i0 = blk * FR;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float acc[FR];
#pragma unroll
    for (int r = 0; r < FR; ++r) acc[r] = 0.f;
    // k blocks of 8: forward coefficient (r, k) = c[(i0 + r - k) mod nx] = ctab[nx + i0 + r - k],
    // adjoint c[(k - i0 - r) mod nx] = ctab[nx + k - i0 - r]; a window of 40 table entries covers
    // a block (its first entry is 16-byte aligned: i0, nx and kb are multiples of 8)
    for (int kb = 8 * threadIdx.x; kb < nx; kb += 8 * kFieldThreads) {
        const float4 xa = __ldg(reinterpret_cast<const float4*>(a.x + kb));
        const float4 xb = __ldg(reinterpret_cast<const float4*>(a.x + kb + 4));
        const float xk[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
        const int base = a.adjoint ? nx + kb - i0 - 32 : nx + i0 - kb - 8;
        float cw[40];
#pragma unroll
        for (int v = 0; v < 10; ++v) {
            const float4 t = __ldg(reinterpret_cast<const float4*>(a.ctab + base) + v);
            cw[4 * v] = t.x;
            cw[4 * v + 1] = t.y;
            cw[4 * v + 2] = t.z;
            cw[4 * v + 3] = t.w;
        }
        if (a.adjoint) {
#pragma unroll
            for (int k = 0; k < 8; ++k)
#pragma unroll
                for (int r = 0; r < FR; ++r) acc[r] += cw[32 + k - r] * xk[k];
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k)
#pragma unroll
                for (int r = 0; r < FR; ++r) acc[r] += cw[8 + r - k] * xk[k];
        }
    }
    // transposed butterfly: lane l ends with the warp's sum of row l
#pragma unroll
    for (int st = 0; st < 5; ++st) {
        const int o = 16 >> st;
        const int n = FR >> (st + 1);
        const bool upper = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < FR / 2; ++i) {
            if (i < n) {
                const float send = upper ? acc[i] : acc[i + n];
                const float keep = upper ? acc[i + n] : acc[i];
                acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
            }
        }
    }
    red[wid][lane] = acc[0];
    __syncthreads();
    if (threadIdx.x < FR) {
        const int r = threadIdx.x, i = i0 + r;
        float E = 0.f;
#pragma unroll
        for (int w = 0; w < kFieldWarps; ++w) E += red[w][r];
        if (a.adjoint) {
            a.grho_out[i] = E;
        } else {
            const float Et = E + __ldg(a.H + i);
            a.E_out[i] = E;
            if (a.E_hist_out != nullptr) a.E_hist_out[i] = Et;
            a.vsh_out[i] = make_vshift<float>(Et, a.dtdv, a.nv);
            s_e[r] = (double)(trap_w<float>(i, nx) * E * E);
        }
    }
    if (a.adjoint || a.ee_out == nullptr) return;
    __syncthreads();
    if (threadIdx.x < 32) {
        double e = s_e[lane];
        e = warp_sum(e);
        if (lane == 0) {
            a.eep[blk] = e;
            __threadfence();
            s_last = atomicAdd(a.counter, 1u) == (unsigned)(nblk - 1) ? 1 : 0;
        }
        e = 0.0;
        if (__shfl_sync(0xffffffffu, s_last, 0)) {
            __threadfence();
            for (int g = lane; g < nblk; g += 32) e += __ldcg(a.eep + g);
            e = warp_sum(e);
            if (lane == 0) {
                *a.ee_out = (float)(0.5 * e * (double)a.dx);
                *a.counter = 0u;
            }
        }
    }
}

__global__ void __launch_bounds__(kFieldThreads) vp_strip_field_kernel(const StripFieldArgs a) {
    strip_field_body(a, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------------------------
// Ensembles: the same bodies over all instances of an ensemble in one launch. CTA blockIdx.x works
// on map[blockIdx.x] = (instance, chunk, run) with 128-column groups; the per-step buffers are the
// ensemble's packed ones (BatchStep), the tables and offsets each instance's (StripInst).
// ---------------------------------------------------------------------------------------------

// 20 one-warp CTAs per SM (up to 96 registers): the C4 ensemble's forward step 5 % faster than
// with 24 (80 registers)
__global__ void __launch_bounds__(kStripEnsThreads, 20)
    vp_strip_ens_fwd_kernel(const StripInst* __restrict__ insts, const int4* __restrict__ map,
                            const BatchStep<float> b) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_last;
    const int4 m = __ldg(map + blockIdx.x);
    const StripInst& I = insts[m.x];
    const long long nn = (long long)I.nx * I.nv;
    StripFwdArgs a{};
    a.nx = I.nx;
    a.nv = I.nv;
    a.n_chunks = I.n_chunks;
    a.n_bands = I.n_bands;
    a.ring_rows = I.ring_rows;
    a.runs = I.runs;
    a.quad = I.quad;
    a.tq = I.tq;
    a.chunk = I.chunk;
    a.dfeq = I.dfeq;
    a.vtab = I.vtab;
    a.feq = I.feq;
    a.h_in = b.c_in + b.c_in_mul * I.off_f + (long long)b.c_in_step * nn;
    a.h_out = b.c_out ? b.c_out + b.c_out_mul * I.off_f + (long long)b.c_out_step * nn : nullptr;
    a.vsh = b.vsh_in + (long long)b.vsh_in_mul * I.off_x + (long long)b.vsh_in_step * I.nx;
    a.f_hist_n = nullptr;
    a.f_final = b.f_final ? b.f_final + I.off_f : nullptr;
    a.part = b.part ? b.part + I.off_part : nullptr;
    a.run_ctr = b.counters + I.off_ctr;
    a.rho_out = b.rho + I.off_x;
    a.dv = I.dv;
    strip_fwd_body<kStripEnsRows, kStripEnsThreads>(a, smem, &s_last, m.y, m.z);
}

__global__ void __launch_bounds__(kStripEnsThreads, 16)
    vp_strip_ens_bwd_kernel(const StripInst* __restrict__ insts, const int4* __restrict__ map,
                            const BatchStep<float> b) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_last;
    const int4 m = __ldg(map + blockIdx.x);
    const StripInst& I = insts[m.x];
    const long long nn = (long long)I.nx * I.nv;
    StripBwdArgs a{};
    a.nx = I.nx;
    a.nv = I.nv;
    a.n_chunks = I.n_chunks;
    a.n_bands = I.n_bands;
    a.ring_rows = I.ring_rows;
    a.runs = I.runs;
    a.quad = I.quad;
    a.tq = I.tq;
    a.chunk = I.chunk;
    a.dfeq = I.dfeq;
    a.vtab = I.vtab;
    a.feq = I.feq;
    a.w_in = b.c_in + b.c_in_mul * I.off_f + (long long)b.c_in_step * nn;
    a.w_out = b.c_out ? b.c_out + b.c_out_mul * I.off_f + (long long)b.c_out_step * nn : nullptr;
    a.grho = b.grho + I.off_x;
    a.vsh_n = b.vsh_in + (long long)b.vsh_in_mul * I.off_x + (long long)b.vsh_in_step * I.nx;
    a.vsh_prev = b.vsh_prev + (long long)b.n_steps * I.off_x + (long long)b.vsh_prev_step * I.nx;
    a.h_prev = b.h_prev + (long long)b.n_steps * I.off_f + (long long)b.h_prev_step * nn;
    a.gfh = nullptr;
    a.part = b.part + I.off_part;
    a.run_ctr = b.counters + I.off_ctr;
    a.dv = I.dv;
    a.dx = I.dx;
    a.neg_dt_dv = I.neg_dt_dv;
    a.gE_hist = b.g_Eh ? b.g_Eh + (long long)b.n_steps * I.off_x + (long long)b.g_step * I.nx : nullptr;
    a.gee = b.g_ee ? b.g_ee + (long long)I.index * b.n_steps + b.g_step : nullptr;
    a.E_prev = b.E_prev + (long long)b.n_steps * I.off_x + (long long)b.E_prev_step * I.nx;
    a.gH = b.g_H + I.off_x;
    a.gE_out = b.gE + I.off_x;
    strip_bwd_body<kStripEnsRows, kStripEnsThreads>(a, smem, &s_last, m.y, m.z);
}

__global__ void __launch_bounds__(kFieldThreads)
    vp_strip_ens_field_kernel(const StripInst* __restrict__ insts, const int2* __restrict__ fmap,
                              const BatchStep<float> b, int adjoint) {
    const int2 m = __ldg(fmap + blockIdx.x);   // (instance, 32-row block)
    const StripInst& I = insts[m.x];
    StripFieldArgs f{};
    f.nx = I.nx;
    f.nv = I.nv;
    f.adjoint = adjoint;
    f.ctab = I.ctab;
    f.dx = I.dx;
    if (adjoint) {
        f.x = b.gE + I.off_x;
        f.grho_out = b.grho_out + I.off_x;
    } else {
        f.x = b.rho + I.off_x;
        f.H = b.H + I.off_x;
        f.dtdv = I.dtdv;
        f.E_out = b.E_out + (long long)b.E_out_mul * I.off_x + (long long)b.E_out_step * I.nx;
        f.E_hist_out = b.E_hist ? b.E_hist + (long long)b.n_steps * I.off_x + (long long)b.hist_step * I.nx : nullptr;
        f.vsh_out = b.vsh_out + (long long)b.vsh_out_mul * I.off_x + (long long)b.vsh_out_step * I.nx;
        f.ee_out = b.ee_hist ? b.ee_hist + (long long)I.index * b.n_steps + b.hist_step : nullptr;
        f.eep = b.eep + I.off_eep;
        f.counter = b.fctr + I.index;
    }
    strip_field_body(f, m.y, I.field_ctas);
}

// The field of a whole small instance (nx <= kStripSmallField) in one CTA of 4 x kStripSmallField
// threads: part p = threadIdx.x / kStripSmallField of row i sums k in [p nx / 4, (p + 1) nx / 4) of
// E_i = sum_k c[(i - k) mod nx] x_k (adjoint: c[(k - i) mod nx]) from x and the coefficient table
// ctab[1 .. 2 nx) staged in shared memory, in two interleaved partial sums; the four parts are
// added in a fixed order and the energy is a fixed-order block sum. blockIdx.x is the instance.
__global__ void __launch_bounds__(4 * kStripSmallField)
    vp_strip_ens_field_small_kernel(const StripInst* __restrict__ insts, const BatchStep<float> b, int adjoint) {
    constexpr int NF = kStripSmallField;
    __shared__ float xs[NF];
    __shared__ float cs[2 * NF];
    __shared__ float ps[4][NF];
    __shared__ double red[NF / 32];
    const StripInst& I = insts[blockIdx.x];
    const int nx = I.nx, t = threadIdx.x % NF, part = threadIdx.x / NF;
    const float* x = adjoint ? b.gE + I.off_x : b.rho + I.off_x;
    for (int k = threadIdx.x; k < nx; k += blockDim.x) xs[k] = __ldcg(x + k);
    for (int u = threadIdx.x; u < 2 * nx - 1; u += blockDim.x) cs[u] = __ldg(I.ctab + 1 + u);   // c[(u + 1 - nx) mod nx]
    __syncthreads();
    if (t < nx) {
        // forward: coefficient (t, k) = cs[nx - 1 + t - k]; adjoint: cs[nx - 1 + k - t]
        const int base = nx - 1 + (adjoint ? -t : t), step = adjoint ? 1 : -1;
        const int k0 = part * (nx / 4), k1 = k0 + nx / 4;
        float a0 = 0.f, a1 = 0.f;
#pragma unroll 4
        for (int k = k0; k < k1; k += 2) {
            a0 += cs[base + step * k] * xs[k];
            a1 += cs[base + step * (k + 1)] * xs[k + 1];
        }
        ps[part][t] = a0 + a1;
    }
    __syncthreads();
    if (part != 0) return;
    double e2 = 0.0;
    if (t < nx) {
        const float E = (ps[0][t] + ps[1][t]) + (ps[2][t] + ps[3][t]);
        if (adjoint) {
            b.grho_out[I.off_x + t] = E;
        } else {
            const float Et = E + __ldg(b.H + I.off_x + t);
            b.E_out[(long long)b.E_out_mul * I.off_x + (long long)b.E_out_step * nx + t] = E;
            if (b.E_hist) b.E_hist[(long long)b.n_steps * I.off_x + (long long)b.hist_step * nx + t] = Et;
            b.vsh_out[(long long)b.vsh_out_mul * I.off_x + (long long)b.vsh_out_step * nx + t] =
                make_vshift<float>(Et, I.dtdv, I.nv);
            e2 = (double)(trap_w<float>(t, nx) * E * E);
        }
    }
    if (adjoint || b.ee_hist == nullptr) return;
    e2 = warp_sum(e2);
    if ((t & 31) == 0) red[t >> 5] = e2;
    asm volatile("bar.sync 1, %0;" ::"r"(NF) : "memory");   // the part-0 warps only
    if (t == 0) {
        double sum = 0.0;
        for (int w = 0; w < NF / 32; ++w) sum += red[w];
        b.ee_hist[(long long)I.index * b.n_steps + b.hist_step] = (float)(0.5 * sum * (double)I.dx);
    }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------

template <int R, int GT>
static int strip_occupancy(bool fwd, size_t smem) {
    int n = 0;
    cudaError_t e;
    // the attribute is the largest size any plan uses, so that plans of other grids stay launchable
    if (fwd) {
        e = cudaFuncSetAttribute(vp_strip_fwd_kernel<R, GT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStripMaxSmem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, vp_strip_fwd_kernel<R, GT>, GT, smem);
    } else {
        e = cudaFuncSetAttribute(vp_strip_bwd_kernel<R, GT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStripMaxSmem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, vp_strip_bwd_kernel<R, GT>, GT, smem);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

template <int GT>
static int strip_occupancy_r(int R, bool fwd, size_t smem) {
    if constexpr (GT == 32) {
        return R == 8 ? strip_occupancy<8, 32>(fwd, smem) : R == 4 ? strip_occupancy<4, 32>(fwd, smem) : 0;
    } else {
        return R == 16 ? strip_occupancy<16, GT>(fwd, smem)
                       : R == 8 ? strip_occupancy<8, GT>(fwd, smem) : strip_occupancy<4, GT>(fwd, smem);
    }
}

// Ring rows of a strip CTA: a band's window (2 dmax + R + 4 rows, at most L slabs of R rows) plus the
// slab in flight; dmax is the largest spread of quad shifts within one chunk of the table.
static int strip_ring_rows(const std::vector<int2>& chunk, int R) {
    int dmax = 0;
    for (const int2& c : chunk) dmax = std::max(dmax, c.y - c.x);
    const int span_max = 2 * dmax + R + 4;
    return ((span_max + R - 1) / R + 1) * R;
}

bool strip_prepare(StripHost& sh, int nx, int nv, const std::vector<int2>& chunk, const std::vector<int2>& bchunk,
                   int n_sms, int force_rows, int gt, int bgt) {
    sh = StripHost{};
    if ((gt != 32 && gt != 64) || (bgt != 32 && bgt != 64)) return false;
    const int cols = 4 * gt, bcols = 4 * bgt;
    if (nv % cols != 0 || nv % bcols != 0 || nx % kStripFieldRows != 0 || nx < 64 ||
        (int)chunk.size() != nv / cols || (int)bchunk.size() != nv / bcols)
        return false;
    for (int R : {4, 8, 16}) {   // automatic: the first that fits (4 measured fastest on B200)
        if (force_rows > 0 && R != force_rows) continue;
        if (nx % R != 0 || ((gt == 32 || bgt == 32) && R == 16)) continue;
        const int NR = strip_ring_rows(chunk, R), NRb = strip_ring_rows(bchunk, R);
        const size_t fb = strip_fwd_bytes(NR, R, gt), bb = strip_bwd_bytes(NRb, R, bgt);
        if (fb > (size_t)kStripMaxSmem || bb > (size_t)kStripMaxSmem) continue;
        const int pf = gt == 32 ? strip_occupancy_r<32>(R, true, fb) : strip_occupancy_r<64>(R, true, fb);
        const int pb = bgt == 32 ? strip_occupancy_r<32>(R, false, bb) : strip_occupancy_r<64>(R, false, bb);
        if (pf <= 0 || pb <= 0) continue;
        sh.R = R;
        sh.gt = gt;
        sh.bgt = bgt;
        sh.n_bands = nx / R;
        sh.n_chunks = nv / cols;
        sh.b_n_chunks = nv / bcols;
        sh.span_max = NR - R;
        sh.ring_rows = NR;
        sh.b_ring_rows = NRb;
        sh.fwd_smem = fb;
        sh.bwd_smem = bb;
        // runs per chunk: as many as fill one wave of CTAs (at least one)
        sh.fwd_runs = std::max(1, std::min(nx / R, pf * n_sms / sh.n_chunks));
        sh.bwd_runs = std::max(1, std::min(nx / R, pb * n_sms / sh.b_n_chunks));
        sh.fwd_ctas = sh.n_chunks * sh.fwd_runs;
        sh.bwd_ctas = sh.b_n_chunks * sh.bwd_runs;
        sh.field_ctas = nx / kStripFieldRows;
        return true;
    }
    return false;
}

cudaError_t launch_strip_fwd(const StripFwdArgs& args, const StripHost& sh, cudaStream_t s) {
    StripFwdArgs a = args;
    a.n_chunks = sh.n_chunks;
    a.n_bands = sh.n_bands;
    a.ring_rows = sh.ring_rows;
    a.runs = sh.fwd_runs;
    switch (sh.R * 100 + sh.gt) {
        case 464: vp_strip_fwd_kernel<4, 64><<<sh.fwd_ctas, 64, sh.fwd_smem, s>>>(a); break;
        case 864: vp_strip_fwd_kernel<8, 64><<<sh.fwd_ctas, 64, sh.fwd_smem, s>>>(a); break;
        case 1664: vp_strip_fwd_kernel<16, 64><<<sh.fwd_ctas, 64, sh.fwd_smem, s>>>(a); break;
        case 432: vp_strip_fwd_kernel<4, 32><<<sh.fwd_ctas, 32, sh.fwd_smem, s>>>(a); break;
        case 832: vp_strip_fwd_kernel<8, 32><<<sh.fwd_ctas, 32, sh.fwd_smem, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_strip_bwd(const StripBwdArgs& args, const StripHost& sh, cudaStream_t s) {
    StripBwdArgs a = args;
    a.n_chunks = sh.b_n_chunks;
    a.n_bands = sh.n_bands;
    a.ring_rows = sh.b_ring_rows;
    a.runs = sh.bwd_runs;
    switch (sh.R * 100 + sh.bgt) {
        case 464: vp_strip_bwd_kernel<4, 64><<<sh.bwd_ctas, 64, sh.bwd_smem, s>>>(a); break;
        case 864: vp_strip_bwd_kernel<8, 64><<<sh.bwd_ctas, 64, sh.bwd_smem, s>>>(a); break;
        case 1664: vp_strip_bwd_kernel<16, 64><<<sh.bwd_ctas, 64, sh.bwd_smem, s>>>(a); break;
        case 432: vp_strip_bwd_kernel<4, 32><<<sh.bwd_ctas, 32, sh.bwd_smem, s>>>(a); break;
        case 832: vp_strip_bwd_kernel<8, 32><<<sh.bwd_ctas, 32, sh.bwd_smem, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_strip_field(const StripFieldArgs& a, const StripHost& sh, cudaStream_t s) {
    if (a.nx % kStripFieldRows != 0 || a.nx % 8 != 0) return cudaErrorInvalidValue;
    vp_strip_field_kernel<<<sh.field_ctas, kFieldThreads, 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

size_t strip_ens_fwd_bytes(int ring_rows) { return strip_fwd_bytes(ring_rows, kStripEnsRows, kStripEnsThreads); }
size_t strip_ens_bwd_bytes(int ring_rows) { return strip_bwd_bytes(ring_rows, kStripEnsRows, kStripEnsThreads); }

int strip_ens_occupancy(bool fwd, size_t smem) {
    int n = 0;
    cudaError_t e;
    if (fwd) {
        e = cudaFuncSetAttribute(vp_strip_ens_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kStripMaxSmem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, vp_strip_ens_fwd_kernel, kStripEnsThreads, smem);
    } else {
        e = cudaFuncSetAttribute(vp_strip_ens_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kStripMaxSmem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, vp_strip_ens_bwd_kernel, kStripEnsThreads, smem);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

cudaError_t launch_strip_ens_fwd(const StripInst* insts, const int4* map, int n_ctas, size_t smem,
                                 const BatchStep<float>& b, cudaStream_t s) {
    vp_strip_ens_fwd_kernel<<<n_ctas, kStripEnsThreads, smem, s>>>(insts, map, b);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_strip_ens_bwd(const StripInst* insts, const int4* map, int n_ctas, size_t smem,
                                 const BatchStep<float>& b, cudaStream_t s) {
    vp_strip_ens_bwd_kernel<<<n_ctas, kStripEnsThreads, smem, s>>>(insts, map, b);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_strip_ens_field(const StripInst* insts, const int2* fmap, int n_ctas, const BatchStep<float>& b,
                                   int adjoint, cudaStream_t s) {
    vp_strip_ens_field_kernel<<<n_ctas, kFieldThreads, 0, s>>>(insts, fmap, b, adjoint);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_strip_ens_field_small(const StripInst* insts, int n_inst, const BatchStep<float>& b, int adjoint,
                                         cudaStream_t s) {
    vp_strip_ens_field_small_kernel<<<n_inst, 4 * kStripSmallField, 0, s>>>(insts, b, adjoint);
    count_launch();
    return cudaGetLastError();
}

}  // namespace vpb
