// Internal declarations shared by the host orchestration (vp_capi.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <string>
#include <vector>

namespace vpb {

template <typename T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };

// Per-row v-step shift: integer cell offset m (already reduced mod nv) and lerp weight t.
template <typename T> struct alignas(2 * sizeof(T) >= 8 ? 2 * sizeof(T) : 8) VShift {
    int m;
    T t;
};

// Device tables of the Poisson solve for one nx.
template <typename T> struct PoissonTables {
    int nx;
    int log2nx;        // valid when pow2
    int pow2;
    const typename Cplx<T>::type* tw;   // nx/2 twiddles exp(-2*pi*i*q/nx)        (pow2)
    const T* mult_im;                   // imaginary part of the multiplier m_k   (pow2)
    const T* circ;                      // c = real(ifft(m)): E = c (*) rho       (any nx)
    T* gscratch;                        // nx complex of global scratch, used when the work area
                                        // does not fit in the launch's shared memory
    int use_smem;                       // work area in dynamic shared memory
    int tw_stage;                       // twiddles in shared memory laid out per FFT stage (pow2,
                                        // use_smem; the work area is poisson_area_size_staged)
};

// Arguments of one fused forward launch (see vp_kernels.cu for the phase semantics).
template <typename T> struct FwdArgs {
    int nx, nv, n_chunks, chunk_cols;
    const T* h_in;              // delta after the leading x half-step of step n
    const double* f_iv;         // prologue only
    T* h_out;                   // delta after the leading x half-step of step n+1 (or null)
    const VShift<T>* vsh;       // v shifts of step n
    const int* mx;              // x half-step offsets, reduced mod nx   [nv]
    const T* tx;                // x half-step weights                   [nv]
    const double* tx64;         // x half-step weights in float64        [nv]
    const double* feq;          // f_eq (one row when feq_rs == 0)
    int feq_rs;                 // f_eq row stride: 0 or nv
    T* f_hist_n;                // f after step n, or null
    double* f_final;            // f after the last step, or null
    T* part;                    // rho partial sums [n_chunks][nx], or null (no tail)
    unsigned* counter;
    // tail (last CTA): Poisson for step n+1
    PoissonTables<T> P;
    T dv, dx, dtdv;
    const T* H;
    T* E_out;                   // raw E of step n+1
    T* E_hist_out;              // E + H of step n+1, or null
    T* ee_out;                  // ee of step n+1, or null
    VShift<T>* vsh_out;         // v shifts of step n+1
    const T* vtab;              // staged step: v-step f_eq correction tables A_m, B_m, or null
    int stage_span;             // staged step: rows the staging buffer holds
};

// v halo of the staged step kernels (cells on each side of a CTA's columns), and the shifts the
// correction tables cover: m in [-kStageHalo, kStageHalo).
constexpr int kStageHalo = 4;

// Arguments of one fused backward launch.
template <typename T> struct BwdArgs {
    int nx, nv, n_chunks, chunk_cols;
    const T* w_in;              // cotangent on the v-step output of step n
    const T* grho;              // cotangent on rho of step n
    const VShift<T>* vsh_n;     // v shifts of step n
    const T* gfh;               // cotangent on f_hist[n-1], or null
    const T* c_src;             // prologue: cotangent on f_final, or null
    const T* c_src2;            // prologue: cotangent on f_hist[T-1], or null
    T* w_out;                   // cotangent on the v-step output of step n-1 (or null)
    T* gfiv_out;                // epilogue: cotangent on f_iv
    const T* h_prev;            // delta_half of step n-1
    const VShift<T>* vsh_prev;  // v shifts of step n-1
    const int* mx;
    const T* tx;
    const double* feq;
    int feq_rs;
    T* part;
    unsigned* counter;
    // tail
    PoissonTables<T> P;
    T dv, dx, neg_dt_dv;
    const T* E_prev;            // raw E of step n-1
    const T* gE_hist;           // cotangent on E_hist[n-1], or null
    const T* gee;               // address of the cotangent on ee_hist[n-1], or null
    T* gH;                      // accumulated cotangent on H
    T* grho_out;                // cotangent on rho of step n-1
    const T* vtab;              // staged step: correction tables (B_m is the f_eq slope), or null
    int stage_span;             // staged step: rows of w the staging buffer holds
};

// ---- ensembles: many instances (any nx, nv, dt, f_eq) advanced together -----------------------
// Packed layouts: per-instance (nx, nv) blocks at off_f, nx blocks at off_x. The per-instance
// device tables (shift tables, f_eq, FFT tables) belong to one vp_plan per instance.
template <typename T> struct BatchInst {
    int nx, nv, n_chunks, chunk_cols;
    int tile_begin, n_tiles;    // tiles of this instance in a step launch
    long long off_f;            // offset of the (nx, nv) block in packed cell buffers
    int off_x;                  // offset of the nx block in packed row buffers
    int off_part;               // offset of its n_chunks*nx partial sums
    int index;                  // position of the instance in the caller's order
    const int* mx;
    const T* tx;
    const double* tx64;
    const T* vtab;              // per-shift f_eq correction tables (A, B pairs), or null
    const double* feq;
    int feq_rs;
    PoissonTables<T> P;
    T dv, dx, dtdv, neg_dt_dv;
};

// One step launch of an ensemble. A cell pointer of instance i is base + mul*off_f[i] + step*nx*nv
// (a row pointer: base + mul*off_x[i] + step*nx): mul/step select a ping-pong slot (1, 0) or a
// tape slot (n_steps, n).
template <typename T> struct BatchStep {
    const BatchInst<T>* inst;
    const int4* tiles;          // per tile: instance (index into inst), first row, column chunk
    int n_inst, n_tiles;
    int last;                   // forward: the last step (no h_out, no tail)
    int n_steps;
    const double* f_iv;         // prologue (forward)
    const T* H;
    const T* c_in; int c_in_mul, c_in_step;   // forward h_n / adjoint w_n
    T* c_out; int c_out_mul, c_out_step;      // forward h_{n+1} / adjoint w_{n-1}
    const VShift<T>* vsh_in; int vsh_in_mul, vsh_in_step;     // shifts of step n
    VShift<T>* vsh_out; int vsh_out_mul, vsh_out_step;        // forward: shifts of step n+1
    T* E_out; int E_out_mul, E_out_step;                      // forward: raw E of step n+1
    double* f_final;            // forward, last step
    T* E_hist;                  // forward: [inst][n_steps][nx], row n+1 (or 0 in the prologue)
    T* ee_hist;                 // forward: [inst][n_steps]
    int hist_step;
    T* part;
    unsigned* counters;
    // adjoint
    const T* grho;              // packed rows, cotangent on rho of step n
    T* grho_out;
    const T* h_prev; int h_prev_step;            // tape h of step n-1 (mul = n_steps)
    const VShift<T>* vsh_prev; int vsh_prev_step; // tape shifts of step n-1
    const T* E_prev; int E_prev_step;            // tape E of step n-1
    const double* unused_;
    // strip step kernels of an ensemble: packed rho and g_E rows, per-instance field energy
    // partials and field completion counters
    T* rho;
    T* gE;
    double* eep;
    unsigned* fctr;
    const T* g_ff;              // prologue: cotangent on f_final (packed cells)
    const T* g_Eh;              // [inst][n_steps][nx], row n-1
    const T* g_ee;              // [inst][n_steps], entry n-1
    int g_step;
    T* g_H;
    T* g_fiv;                   // epilogue
};

struct LaunchCfg {
    int R;          // rows per CTA
    int threads;    // threads per CTA (one column each)
    int n_chunks;   // column chunks per row block
    int chunk_cols; // columns per chunk
    size_t smem;    // dynamic shared memory bytes
};

// Launchers (vp_kernels.cu). PHASE: 0 = prologue, 1 = step, 2 = epilogue (backward only).
template <typename T>
cudaError_t launch_fwd(const FwdArgs<T>& a, const LaunchCfg& c, int phase, bool feq2d,
                       cudaStream_t s);
template <typename T>
cudaError_t launch_bwd(const BwdArgs<T>& a, const LaunchCfg& c, int phase, bool feq2d,
                       cudaStream_t s);
// Staged forward step (x-invariant f_eq, C = c.threads in {128, 256} dividing nv, c.chunk_cols
// columns per CTA in blocks of C); c.smem covers the buffers for a.stage_span rows.
template <typename T>
cudaError_t launch_fwd_staged(const FwdArgs<T>& a, const LaunchCfg& c, cudaStream_t s);
template <typename T>
cudaError_t set_staged_smem_limit(size_t bytes);
// Shared memory of the staged kernel's buffers for a staging span of `span` rows and C columns.
size_t staged_smem_bytes(int span, int C, size_t real_size);
// Staged adjoint step (same shape rules as the staged forward step).
template <typename T>
cudaError_t launch_bwd_staged(const BwdArgs<T>& a, const LaunchCfg& c, cudaStream_t s);
template <typename T>
cudaError_t set_staged_bwd_smem_limit(size_t bytes);
size_t staged_bwd_smem_bytes(int span, int R, int C, size_t real_size);

// ---- persistent forward time loop (vp_persist.cu): float32, x-invariant f_eq, Strang scheme ----
// State slot of step n: ckpt + (n / K) * nx * nv when ckpt != null and n % K == 0; otherwise
// hbuf0/hbuf1 by the parity of n (full mode) or seg + (n % K - 1) * nx * nv (replay mode).
struct PersistArgs {
    int nx, nv;
    int n_steps;                // full mode: T; replay mode: the step after the last one replayed
    int n_chunks;               // nv / 256
    int bands_per_cta, span_max, win_lo, win_rows, field_dist;   // launch shape (set by the launcher)
    int stage_floats, fs_alias, stages, field_rows;
    int mode;                   // 0: full forward (prologue from f_iv, field, outputs); 1: replay
                                //    steps first_step .. n_steps - 1 with the tape's v shifts
    int first_step;
    int K;
    float* hbuf0;
    float* hbuf1;
    float* seg;
    float* ckpt;
    const double* f_iv;
    const float* H;
    const int2* quad;           // per 4 columns: smallest x offset bm (signed), bit e set when
                                // column e's offset is bm + 1                     [nv / 4]
    const float4* tq;           // per 4 columns: x weights                        [nv / 4]
    const int2* chunk;          // per 256 columns: (min bm, max bm)               [nv / 256]
    const double* feq;          // the f_eq row                                     [nv]
    const float* dfeq;          // f_eq[j+1] - f_eq[j] (periodic), rounded from float64 [nv]
    const float* vtab;          // A_m, B_m tables of the staged kernels          [2][8][nv]
    const float* ctab;          // ctab[j] = c[(j - nx) mod nx], c = real(ifft(m)) [3 nx + 8]
    float dv, dx, dtdv;
    float* rho;                 // [2][nx]
    VShift<float>* vsh_g;       // [nx] v shifts of the field slices
    const VShift<float>* vsh_tape_in;   // replay: the forward's v shifts [n_steps][nx]
    double* eep;                // [n_steps][G] energy partials
    unsigned* bar;              // grid barrier counter (zeroed by the launcher)
    unsigned* status;
    unsigned long long wait_ns; // limit of each grid barrier wait
    float* f_hist;
    double* f_final;
    float* E_hist;
    float* ee_hist;
    float* E_tape;
    VShift<float>* vsh_tape;
};

// Persistent adjoint steps n_hi .. n_lo (descending, >= 1) of the discrete adjoint (vp_persist.cu).
struct PersistBwdArgs {
    int nx, nv, n_chunks;
    int bands_per_cta, span_max, win_lo, win_rows, field_dist, stage_floats, fs_alias, stages, field_rows;
    int n_hi, n_lo, K;
    float* wbuf0;               // cotangent on the v-step output of step n: wbuf[n & 1]
    float* wbuf1;
    const float* ckpt;          // h_n: ckpt + (n / K) * nx * nv when n % K == 0, else
    const float* seg;           //      seg + (n % K - 1) * nx * nv
    const int2* quad;
    const float4* tq;
    const int2* chunk;
    const float* dfeq;
    const float* vtab;
    const double* feq;
    const float* ctab;
    float dv, dx, neg_dt_dv;
    const VShift<float>* vsh_tape;
    const float* E_tape;
    const float* g_fh;          // [n_steps][nx][nv] or null
    const float* g_Eh;          // [n_steps][nx] or null
    const float* g_ee;          // [n_steps] or null
    float* g_H;                 // accumulated
    float* grho;                // [nx] in: cotangent on rho of step n_hi; out: of step n_lo - 1
    float* gE;                  // [2][nx] scratch
    unsigned* bar;
    unsigned* status;
    unsigned long long wait_ns;
};

struct PersistHost {
    int R = 0, G = 0, bands_per_cta = 0, span_max = 0, win_lo = 0, win_rows = 0, field_dist = 0;
    int stage_floats = 0, fs_alias = 0, stages = 2, field_rows = 0;
    size_t smem = 0;
    // adjoint launch shape (same bands, CTAs and column groups): window, stage area, field rows
    int bwd_ok = 0, bwin_lo = 0, bwin_rows = 0, bstage_floats = 0, bfs_alias = 0, bstages = 1, bfield_rows = 0;
    int bfield_dist = 0;
    size_t bsmem = 0;
    std::vector<int2> quad;
    std::vector<float> tq;
    std::vector<int2> chunk;
};

// Builds the persistent path's tables and launch shape for a grid (force_rows: 0 = automatic, else
// the band height 4, 8 or 16); false when the grid is not eligible. m_signed: the unreduced x
// half-step offsets floor(-s_j); tx their weights.
bool persist_prepare(PersistHost& ph, int nx, int nv, const std::vector<long long>& m_signed,
                     const std::vector<double>& tx, int n_sms, int force_rows);
cudaError_t launch_persist_fwd(const PersistArgs& a, const PersistHost& ph, cudaStream_t s);
cudaError_t launch_persist_bwd(const PersistBwdArgs& a, const PersistHost& ph, cudaStream_t s);
size_t persist_smem_bytes(int span_max, int win_rows, int R, int nx, int nv, int field_rows, int stages,
                          int* stage_floats, int* fs_alias);
// The column-quad tables of the persistent and strip paths (false: some 4 neighbouring columns'
// x shifts differ by more than one cell, or a shift reaches half a period).
bool build_quad_tables(int nx, int nv, const std::vector<long long>& m_signed, const std::vector<double>& tx,
                       std::vector<int2>& quad, std::vector<float>& tq, std::vector<int2>& chunk,
                       int chunk_cols = 256);

// Strip step kernels (vp_strip.cu): per-step launches for large grids. A CTA is one column group
// (64 threads, 256 columns) that walks one run of consecutive bands of R rows of one column chunk,
// keeping the window rows in a shared-memory ring that the next band's rows load into while the
// current band computes. Forward step / replay step:
struct StripFwdArgs {
    int nx, nv, n_chunks, n_bands, ring_rows, runs;
    const float* h_in;          // h_n
    float* h_out;               // h_{n+1}, or null (last step)
    const VShift<float>* vsh;   // v shifts of step n
    const int2* quad;
    const float4* tq;
    const int2* chunk;
    const float* dfeq;
    const float* vtab;
    const double* feq;
    float* f_hist_n;            // f after step n (float), or null
    double* f_final;            // f after the last step, or null
    float* part;                // row partial sums per chunk [n_chunks][nx], or null (replay)
    unsigned* run_ctr;          // [runs], zero between launches
    float* rho_out;             // rho_{n+1}
    float dv;
};

// Adjoint step n: w_{n-1} from w_n, the slope row sums of h_{n-1} and, per band once its last chunk
// is done, g_E of step n-1 (and g_H += g_E_total).
struct StripBwdArgs {
    int nx, nv, n_chunks, n_bands, ring_rows, runs;
    const float* w_in;
    float* w_out;
    const float* grho;          // cotangent on rho of step n
    const VShift<float>* vsh_n;
    const VShift<float>* vsh_prev;
    const float* h_prev;        // h_{n-1}
    const float* gfh;           // cotangent on f_hist[n-1], or null
    const int2* quad;
    const float4* tq;
    const int2* chunk;
    const float* dfeq;
    const float* vtab;
    const double* feq;
    float* part;
    unsigned* run_ctr;
    float dv, dx, neg_dt_dv;
    const float* gE_hist;       // cotangent on E_hist[n-1], or null
    const float* gee;           // address of the cotangent on ee_hist[n-1], or null
    const float* E_prev;        // raw E of step n-1
    float* gH;
    float* gE_out;              // g_E of step n-1 (input of Poisson^T)
};

// Field of all rows by the circulant product, kStripFieldRows rows per CTA: forward E = c * rho
// with E_hist, the v shifts and ee; adjoint grho = c^T * g_E.
struct StripFieldArgs {
    int nx, nv, adjoint;
    const float* x;             // rho (forward) or g_E (adjoint)
    const float* ctab;          // [3 nx + 8]: ctab[j] = c[(j - nx) mod nx]
    const float* H;
    float dtdv, dx;
    float* E_out;               // forward: raw E
    float* E_hist_out;          // forward: E + H, or null
    VShift<float>* vsh_out;     // forward: v shifts
    float* ee_out;              // forward: ee, or null
    double* eep;                // forward: per-CTA energy partials
    unsigned* counter;          // forward: completion counter, zero between launches
    float* grho_out;            // adjoint
};

// One instance of an ensemble on the strip kernels: its tables, launch shape and offsets in the
// ensemble's packed buffers.
struct StripInst {
    int nx, nv, n_chunks, n_bands, ring_rows, runs, index;
    int off_x, off_part, off_ctr, off_eep, field_ctas;
    long long off_f;
    const int2* quad;
    const float4* tq;
    const int2* chunk;
    const float* dfeq;
    const float* vtab;
    const double* feq;
    const float* ctab;
    float dv, dx, dtdv, neg_dt_dv;
};

struct StripHost {
    int R = 0, n_bands = 0, n_chunks = 0, span_max = 0, ring_rows = 0;
    int gt = 0;                 // forward: threads of a column group, 64 (256-column chunks) or 32 (128)
    int bgt = 0, b_n_chunks = 0, b_ring_rows = 0;   // adjoint: its column group, chunks and ring rows
    int fwd_runs = 0, bwd_runs = 0, fwd_ctas = 0, bwd_ctas = 0, field_ctas = 0;
    size_t fwd_smem = 0, bwd_smem = 0;
};
constexpr int kStripFieldRows = 32;

// Launch shape of the strip path (force_rows 0: automatic, else 4, 8 or 16) for forward column
// groups of gt threads and adjoint column groups of bgt threads (64: 256-column chunks, 32:
// 128-column chunks; chunk / bchunk are the quad shift range tables of those widths); false when
// not eligible.
bool strip_prepare(StripHost& sh, int nx, int nv, const std::vector<int2>& chunk, const std::vector<int2>& bchunk,
                   int n_sms, int force_rows, int gt, int bgt);
cudaError_t launch_strip_fwd(const StripFwdArgs& a, const StripHost& sh, cudaStream_t s);
cudaError_t launch_strip_bwd(const StripBwdArgs& a, const StripHost& sh, cudaStream_t s);
cudaError_t launch_strip_field(const StripFieldArgs& a, const StripHost& sh, cudaStream_t s);
// Ensembles: one launch over the CTA map (instance, chunk, run) of all instances, 128-column groups
// and bands of kStripEnsRows rows; field launches over (instance, 32-row block).
constexpr int kStripEnsRows = 4;
constexpr int kStripEnsThreads = 32;
size_t strip_ens_fwd_bytes(int ring_rows);
size_t strip_ens_bwd_bytes(int ring_rows);
int strip_ens_occupancy(bool fwd, size_t smem);
cudaError_t launch_strip_ens_fwd(const StripInst* insts, const int4* map, int n_ctas, size_t smem,
                                 const BatchStep<float>& b, cudaStream_t s);
cudaError_t launch_strip_ens_bwd(const StripInst* insts, const int4* map, int n_ctas, size_t smem,
                                 const BatchStep<float>& b, cudaStream_t s);
cudaError_t launch_strip_ens_field(const StripInst* insts, const int2* fmap, int n_ctas, const BatchStep<float>& b,
                                   int adjoint, cudaStream_t s);
// Ensembles whose instances all have nx <= kStripSmallField: the field of each instance in one CTA.
constexpr int kStripSmallField = 256;
cudaError_t launch_strip_ens_field_small(const StripInst* insts, int n_inst, const BatchStep<float>& b, int adjoint,
                                         cudaStream_t s);

// Raises VP_STATUS_NONFINITE_INPUT in *status when f (n doubles) or H (nx reals, double when h64)
// holds a NaN or an infinity (vp_ops.cu).
cudaError_t launch_check_finite(const double* f, size_t n, const void* H, int nx, bool h64, unsigned* status,
                                cudaStream_t s);

// Single-stage operators (vp_ops.cu).
template <typename T>
cudaError_t launch_compute_rho(int nx, int nv, const double* f, const double* feq, int feq_rs,
                               double dv, T* rho, cudaStream_t s);
template <typename T>
cudaError_t launch_poisson(const PoissonTables<T>& P, const T* in, T* out, int adjoint,
                           cudaStream_t s);
template <typename T>
cudaError_t launch_electric_energy(int nx, double dx, const T* E, T* ee, cudaStream_t s);
template <typename T>
cudaError_t launch_semilag_x(int nx, int nv, const double* vs, double dx, double dt,
                             const T* in, T* out, int adjoint, cudaStream_t s);
template <typename T>
cudaError_t launch_semilag_v(int nx, int nv, double dv, double dt, const T* in,
                             const T* E_total, T* out, int adjoint, const T* f_in, T* g_E,
                             cudaStream_t s);

template <typename T>
cudaError_t launch_fwd_tail(const FwdArgs<T>& a, int threads, size_t smem, bool tw_stage, cudaStream_t s);
template <typename T>
cudaError_t launch_bwd_tail(const BwdArgs<T>& a, int threads, size_t smem, bool tw_stage, cudaStream_t s);
template <typename T>
cudaError_t set_tail_smem_limit(size_t bytes);
template <typename T>
cudaError_t set_poisson_smem_limit(size_t bytes);
// KL(f || f_eq) cost and gradient (float64); scratch holds 2 * kKlBlocks + 2 doubles.
constexpr int kKlBlocks = 512;
cudaError_t launch_kl_divergence(int nx, int nv, const double* f, const double* feq, int feq_rs, double dx,
                                 double dv, double eps, double zeq, double* scratch, double* value, double* grad,
                                 cudaStream_t s);

// x-slab decomposition (vp_ops.cu): per-row records in a slab's row order (array row k = grid row
// (row_first + k) mod nx), and the owned rows' sums over the column-chunk partials.
template <typename T>
cudaError_t launch_slab_gather_rows(int nx, int row_first, int ext_rows, const VShift<T>* vsh, VShift<T>* vsh_out,
                                    const VShift<T>* vsh2, VShift<T>* vsh2_out, const T* grho, T* grho_out,
                                    cudaStream_t s);
template <typename T>
cudaError_t launch_slab_row_sums(const T* part, int n_chunks, int ext_rows, int ghost, int n_rows, T* out,
                                 cudaStream_t s);

// Bytes of the Poisson work area (nx complex values plus nx/2+1 complex twiddles).
inline size_t poisson_area_size(int nx, size_t real_size) {
    return (size_t)nx * 2 * real_size + (size_t)((nx >> 1) + 1) * 2 * real_size;
}

// Bytes of the work area with per-stage twiddles (nx complex values plus nx complex twiddles).
inline size_t poisson_area_size_staged(int nx, size_t real_size) {
    return (size_t)nx * 4 * real_size;
}

// Cluster-resident kernels (vp_resident.cu): one cluster runs a whole time loop.
template <typename T> struct ResFwdArgs {
    int nx, nv, n_steps, Rc;
    const double* f_iv;
    const T* H;
    const int* mx;
    const T* tx;
    const double* tx64;
    const double* feq;
    int feq_rs;
    double* f_final;
    T* f_hist;
    T* E_hist;
    T* ee_hist;
    T* h_tape;              // h_n for every step (or null)
    T* E_tape;              // raw E_n for every step (or null)
    VShift<T>* vsh_tape;    // v shifts for every step (or null)
    PoissonTables<T> P;
    T dv, dx, dtdv;
    int h_lo, h_hi;         // halo rows kept below / above a CTA's own rows
    int mx_lo;              // smallest unreduced x half-step offset (recovers signed offsets)
    int vrows;              // 1: v step once per (row, column) into a shared plane (phase A)
};

template <typename T> struct ResBwdArgs {
    int nx, nv, n_steps, Rc;
    const T* H;
    const int* mx;
    const T* tx;
    const double* feq;
    int feq_rs;
    const T* h_tape;
    const T* E_tape;
    const VShift<T>* vsh_tape;
    const T* g_ff;
    const T* g_fh;
    const T* g_Eh;
    const T* g_ee;
    T* g_fiv;
    T* g_H;
    PoissonTables<T> P;
    T dv, dx, neg_dt_dv;
    int h_lo, h_hi;         // halo rows kept below / above a CTA's own rows
    int mx_lo;              // smallest unreduced x half-step offset (recovers signed offsets)
};

template <typename T>
cudaError_t launch_res_fwd(const ResFwdArgs<T>& a, bool feq2d, int cn, int threads, size_t smem,
                           cudaStream_t s);
template <typename T>
cudaError_t launch_res_bwd(const ResBwdArgs<T>& a, bool feq2d, int cn, int threads, size_t smem,
                           cudaStream_t s);
size_t res_smem_size(int nx, int nv, int Rc, int halo_rows, size_t real_size, bool vrows);
template <typename T>
int res_max_clusters(bool feq2d, int cn, int rc, int nv, size_t smem);
bool res_rows_supported(int rc);
int res_rows_per_thread(int rc, int nv);
int res_threads(int rc, int nv);

template <typename T>
cudaError_t launch_batch_fwd(const BatchStep<T>& b, int R, int phase, bool feq2d, int grid,
                             int threads, size_t smem, cudaStream_t s);
template <typename T>
cudaError_t launch_batch_bwd(const BatchStep<T>& b, int R, int phase, bool feq2d, int grid,
                             int threads, size_t smem, cudaStream_t s);
template <typename T>
int batch_blocks_per_sm(int R, bool fwd, bool feq2d, int threads, size_t smem);

void count_launch(int n = 1);
// Records the message returned by vp_get_last_error and returns code.
int set_err(int code, const char* fmt, ...);

}  // namespace vpb
