/*
 * vp_b200.h - C ABI of the B200 (sm_100a) Vlasov-Poisson step and its discrete adjoint.
 *
 * This is the boundary a host binding (ctypes, cffi, a C/C++ driver) links against. It replaces
 * the device side of Forgotten/warp_vp_solver: the Warp kernels of warp_vp_solver/kernels.py,
 * the host FFT Poisson solve of warp_vp_solver/poisson.py and the per-step launch/transfer
 * loops of warp_vp_solver/solver.py. Each entry point names the reference interface it replaces.
 *
 * Conventions
 *  - Every call returns an int status: VP_OK (0) or one of the VP_ERR_* codes below. The text
 *    of the last error on the calling thread is returned by vp_get_last_error().
 *  - Array arguments are DEVICE pointers owned by the caller (for example torch tensors), laid
 *    out row-major with x (index i, length nx) as rows and v (index j, length nv) as columns,
 *    exactly like the reference's (nx, nv) arrays. "real" below means the plan's compute type:
 *    float when the plan was created with VP_F32, double with VP_F64.
 *  - Calls are asynchronous on the given cudaStream_t (passed as void*; NULL = legacy default
 *    stream). They never synchronise the device and never allocate device memory: scratch space
 *    is a caller-provided workspace of vp_workspace_bytes() bytes, and state kept from the
 *    forward pass for the backward pass lives in a caller-provided tape of vp_tape_bytes()
 *    bytes. Calls are therefore safe to capture in a CUDA graph.
 *  - A plan is bound to the device that was current at vp_plan_create(). One plan must not be
 *    used from two host threads at once, and two calls that share a workspace must not overlap
 *    on the device (the reference's solver object is not re-entrant either,
 *    warp_vp_solver/solver.py:169-203).
 */
#ifndef VP_B200_H
#define VP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VP_ABI_VERSION 7

/* status codes */
#define VP_OK 0
#define VP_ERR_ARG 1          /* invalid argument (shape, pointer, size, value)           */
#define VP_ERR_CUDA 2         /* a CUDA runtime call failed                                */
#define VP_ERR_TIMEOUT 3      /* a bounded device-side wait ran out                        */
#define VP_ERR_UNSUPPORTED 4  /* valid request this build does not implement               */

/* compute types */
#define VP_F32 0
#define VP_F64 1

/* Mesh description: the fields of warp_vp_solver/mesh.py:10-23 (Mesh) that the step uses.
 * xs and vs are HOST arrays of length nx and nv (float64), as produced by make_mesh
 * (warp_vp_solver/mesh.py:26-56). period_v is the half width length_v; the v period of the
 * advection is 2*period_v (warp_vp_solver/solver.py:241). */
typedef struct vp_mesh_desc {
    int32_t nx;
    int32_t nv;
    const double* xs;
    const double* vs;
    double dx;
    double dv;
    double period_x;
    double period_v;
} vp_mesh_desc;

typedef struct vp_plan vp_plan;

/* Builds a plan for one (mesh, dt, f_eq) triple. Replaces WarpVlasovPoissonSolver.__init__
 * (warp_vp_solver/solver.py:92-206): validates the inputs, uploads f_eq, and precomputes the
 * per-column x half-step shifts, the FFT twiddles and the spectral multiplier of
 * fft_inv_multiplier (warp_vp_solver/poisson.py:34-45).
 * f_eq_host: HOST float64 array of nx*nv values (row-major (nx, nv)).
 * dtype: VP_F32 or VP_F64. The plan detects an x-invariant f_eq (every row equal) and then
 * keeps only one row on the device. */
int vp_plan_create(const vp_mesh_desc* mesh, double dt, const double* f_eq_host, int dtype,
                   vp_plan** out_plan);

/* Releases a plan and its device tables. */
/* The same plan from one row of f_eq (nv values) that every x row equals: an x-invariant f_eq
 * without its nx*nv host array, for grids too large for one GPU that x slabs split. No
 * counterpart in the reference, which always builds the full (nx, nv) f_eq
 * (warp_vp_solver/solver.py:170-203). */
int vp_plan_create_from_row(const vp_mesh_desc* mesh, double dt, const double* f_eq_row, int dtype,
                            vp_plan** out_plan);
int vp_plan_destroy(vp_plan* plan);

/* Device-side status of a plan: flags that kernels raise without synchronising the host, read
 * with vp_plan_status and reset with vp_plan_clear_status (both synchronous). They extend the
 * reference's argument validation (warp_vp_solver/solver.py:144-167), which checks shapes only:
 *   VP_STATUS_NONFINITE_INPUT  a vp_forward call's f_iv or H held a NaN or an infinity (checked
 *                              on the device before the loop; the outputs of that call are not
 *                              meaningful);
 *   VP_STATUS_WAIT_TIMEOUT     a bounded device-side wait ran out (for example the grid barrier of
 *                              a persistent time loop); the kernel stopped early and the outputs
 *                              of that call are invalid. */
#define VP_STATUS_NONFINITE_INPUT 1u
#define VP_STATUS_WAIT_TIMEOUT 2u
int vp_plan_status(vp_plan* plan, uint32_t* flags);
int vp_plan_clear_status(vp_plan* plan);
/* Limit, in nanoseconds, of each device-side wait of a plan's persistent launches at their grid
 * barrier (default 1 s; 0: a CTA that is not the last to arrive gives up at once). A wait that
 * gives up raises VP_STATUS_WAIT_TIMEOUT and its CTA returns; every other CTA then gives up at the
 * next barrier, so the launch ends and the CUDA context stays usable. */
int vp_plan_set_wait_limit(vp_plan* plan, uint64_t ns);

/* Number of time steps for t_final: int(t_final / dt), as WarpVlasovPoissonSolver.num_steps
 * (warp_vp_solver/solver.py:212-213). */
int vp_num_steps(const vp_plan* plan, double t_final, int32_t* out_steps);

/* Bytes of caller-provided device workspace a forward or backward call of n_steps steps needs
 * with the given checkpoint interval (0 = automatic). */
int vp_workspace_bytes(const vp_plan* plan, int32_t n_steps, int32_t checkpoint_every,
                       size_t* out_bytes);

/* Bytes of the tape a forward call writes for a later backward call: the delta-f state after
 * the leading x half-step at every checkpoint_every-th step, plus the self-consistent field E
 * and the v-step shift of every step. Replaces the f_hist residual the reference keeps in host
 * memory for its adjoint (warp_vp_solver/solver.py:1379-1392). */
int vp_tape_bytes(const vp_plan* plan, int32_t n_steps, int32_t checkpoint_every,
                  size_t* out_bytes);

/* Checkpoint interval actually used for a request. every > 0 is used as given (capped at
 * n_steps). every == 0 (automatic) keeps the state of every step when that tape is at most
 * 256 MiB and otherwise checkpoints every ceil(sqrt(n_steps)) steps, recomputing the states in
 * between during the adjoint. */
int vp_resolve_checkpoint_every(const vp_plan* plan, int32_t n_steps, int32_t checkpoint_every,
                                int32_t* out_every);

/* Forward time loop of n_steps Strang steps. Replaces WarpVlasovPoissonSolver.run_forward
 * (warp_vp_solver/solver.py:418-464; legacy loop 470-524, fused-E+H loop 530-612).
 *   f_iv      double[nx*nv]     initial distribution (input).
 *   H         real[nx]          external field (input).
 *   f_final   double[nx*nv]     final distribution, or NULL.
 *   f_hist    real[n_steps*nx*nv]  f after every step, or NULL (record_history=False).
 *   E_hist    real[n_steps*nx]  E + H of every step, or NULL.
 *   ee_hist   real[n_steps]     0.5*trapz(E^2)*dx of the self-consistent E, or NULL.
 *   tape      vp_tape_bytes() bytes, or NULL when no backward pass will follow.
 * n_steps == 0 copies f_iv to f_final. */
int vp_forward(vp_plan* plan, const double* f_iv, const void* H, int32_t n_steps,
               double* f_final, void* f_hist, void* E_hist, void* ee_hist,
               void* tape, int32_t checkpoint_every,
               void* workspace, size_t workspace_bytes, void* stream);

/* Discrete adjoint of vp_forward. Replaces WarpVlasovPoissonSolver._run_backward
 * (warp_vp_solver/solver.py:742-772; legacy adjoint 778-932, on-device adjoint 938-1105).
 * Reads the tape written by the vp_forward call with the same (H, n_steps, checkpoint_every)
 * and recomputes the states between checkpoints. Cotangents may be NULL (treated as zero):
 *   g_f_final real[nx*nv], g_f_hist real[n_steps*nx*nv], g_E_hist real[n_steps*nx],
 *   g_ee_hist real[n_steps].
 * Outputs: g_f_iv real[nx*nv] and g_H real[nx] (both overwritten). */
int vp_backward(vp_plan* plan, const void* H, int32_t n_steps,
                const void* tape, int32_t checkpoint_every,
                const void* g_f_final, const void* g_f_hist, const void* g_E_hist,
                const void* g_ee_hist, void* g_f_iv, void* g_H,
                void* workspace, size_t workspace_bytes, void* stream);

/* vp_forward with f_hist streamed to pinned host memory while the loop runs (the reference
 * copies f_hist to the host synchronously every step, warp_vp_solver/solver.py:519, 607):
 * step n's f is written to device slot n % ring_slots of `ring` (ring_slots*nx*nv reals, 2..64
 * slots) and copied from there to f_hist_host + n*nx*nv (pinned, n_steps*nx*nv reals) on
 * copy_stream, overlapping the following steps; the compute stream waits for a slot's copy
 * before reusing it and, at the end, for every copy, so the history is complete once `stream`
 * is. Other arguments as vp_forward (checkpoint_every as given or 0 for automatic); the
 * cluster-resident path is not used. */
int vp_forward_stream_history(vp_plan* plan, const double* f_iv, const void* H, int32_t n_steps, double* f_final,
                              void* f_hist_host, void* ring, int32_t ring_slots, void* E_hist, void* ee_hist,
                              void* tape, int32_t checkpoint_every, void* workspace, size_t workspace_bytes,
                              void* stream, void* copy_stream);

/* Maximum scratch of vp_forward_noalloc: 8 MiB of device memory per GPU that loads the library. */
#define VP_NOALLOC_SCRATCH_BYTES ((size_t)8 << 20)

/* Forward time loop that allocates nothing: the same computation and outputs as vp_forward
 * without a tape, for callers that cannot allocate device memory when they run the solver. Such
 * callers include code recorded into a CUDA graph under a capture mode that forbids cudaMalloc,
 * plug-ins whose host application owns every byte of device memory through its own pool, and
 * time-critical loops that cannot afford the device-wide synchronisation cudaMalloc may cause.
 * No counterpart in the reference, which allocates Warp arrays per solver
 * (warp_vp_solver/solver.py:169-203).
 * The scratch it needs (two delta-f planes of nx*nv reals plus O(nx) vectors) lives in one
 * statically allocated device array of VP_NOALLOC_SCRATCH_BYTES bytes, which every GPU that
 * loads this library holds until the process exits. Requests that need more return VP_ERR_ARG:
 * the two planes take 8*nx*nv bytes in float32 (512x1024 fits, 1024x1024 does not) and 16*nx*nv
 * bytes in float64 (512x512 fits, 512x1024 does not). The first call on a device looks up that
 * array's device address (with the device current), so make the first call on each device
 * before any stream capture. Every call shares the one array and it keeps the previous call's
 * contents: the call clears what must start at zero itself, but two calls whose work overlaps on
 * the GPU (other streams, other host threads, other plans on the same device) race and corrupt
 * each other. */
int vp_forward_noalloc(vp_plan* plan, const double* f_iv, const void* H, int32_t n_steps,
                       double* f_final, void* f_hist, void* E_hist, void* ee_hist, void* stream);

/* --- ensembles ------------------------------------------------------------------------------
 * Many instances (each with its own mesh, dt, f_eq, initial state and field) advanced together:
 * one persistent launch per time step covers every instance. No counterpart in the reference,
 * which advances one WarpVlasovPoissonSolver at a time (warp_vp_solver/solver.py:418-612,
 * 742-1105); each instance's numerics are exactly those of vp_forward / vp_backward.
 * Packed layouts (instance i, in the order given to vp_batch_create):
 *   cell arrays (f_iv, f_final, g_f_final, g_f_iv): the (nx_i, nv_i) block at cell offset i;
 *   row arrays (H, g_H): the nx_i block at row offset i;
 *   E_hist / g_E_hist: the (n_steps, nx_i) block at n_steps * row offset i;
 *   ee_hist / g_ee_hist: the n_steps entries at i * n_steps.
 * Offsets come from vp_batch_offsets. The adjoint needs the tape of the forward call. */
typedef struct vp_batch vp_batch;

int vp_batch_create(int32_t n_instances, const vp_mesh_desc* meshes, const double* dts,
                    const double* const* f_eq_host, int dtype, vp_batch** out_batch);
int vp_batch_destroy(vp_batch* batch);

/* Total packed sizes (cells and rows) and the per-instance offsets (arrays of n_instances;
 * either may be NULL). */
int vp_batch_offsets(const vp_batch* batch, int64_t* total_cells, int64_t* total_rows,
                     int64_t* cell_offsets, int64_t* row_offsets);
int vp_batch_workspace_bytes(const vp_batch* batch, int32_t n_steps, size_t* out_bytes);
int vp_batch_tape_bytes(const vp_batch* batch, int32_t n_steps, size_t* out_bytes);

/* Forward of every instance for n_steps steps (all pointers device memory, packed as above).
 * f_final, E_hist, ee_hist and tape may be NULL. */
int vp_batch_forward(vp_batch* batch, const double* f_iv, const void* H, int32_t n_steps,
                     double* f_final, void* E_hist, void* ee_hist, void* tape,
                     void* workspace, size_t workspace_bytes, void* stream);

/* Adjoint of every instance; cotangents may be NULL (zero). Outputs g_f_iv and g_H. */
int vp_batch_backward(vp_batch* batch, const void* H, int32_t n_steps, const void* tape,
                      const void* g_f_final, const void* g_E_hist, const void* g_ee_hist,
                      void* g_f_iv, void* g_H, void* workspace, size_t workspace_bytes,
                      void* stream);

/* Tile shape of an ensemble's step launches (the autotuner's knobs). */
typedef struct vp_batch_config {
    int32_t rows_per_tile;    /* 1, 2, 4 or 8; divides every instance's nx and is <= nx/2        */
    int32_t chunk_cols;       /* columns per tile: a multiple of 32 in [32, 256]                  */
    int32_t threads;          /* threads per CTA: a multiple of 32 in [32, 256]                   */
    int32_t ctas_per_sm;      /* persistent CTAs per SM (0: as many as fit)                       */
    int32_t n_tiles;          /* derived: tiles per step over all instances                       */
    int32_t grid_fwd;         /* derived: persistent grid of the forward launches                 */
    int32_t grid_bwd;         /* derived: persistent grid of the adjoint launches                 */
    int32_t strip;            /* 1: the steps run on the strip kernels (one launch over all       */
                              /* instances' 128-column groups and runs of bands, then a field     */
                              /* launch); on by default where every instance qualifies (float32,  */
                              /* x-invariant f_eq, nv a multiple of 128, nx of 32); 0: the tile  */
                              /* kernels above                                                    */
    int32_t strip_ctas;       /* derived: CTAs of a strip launch                                  */
} vp_batch_config;

int vp_batch_get_config(const vp_batch* batch, vp_batch_config* out);
/* Sets rows_per_tile, chunk_cols, threads and ctas_per_sm. Workspace sizes depend on chunk_cols
 * (query vp_batch_workspace_bytes again); graphs captured before the call must be re-captured. */
int vp_batch_set_config(vp_batch* batch, const vp_batch_config* cfg);

/* --- surrogate MLP ----------------------------------------------------------------------------
 * Fully connected network widths[0] -> ... -> widths[n_layers] with GELU (erf form) between
 * layers and none on the output: BF16 operands, FP32 accumulation on the tensor cores, FP32
 * master weights and Adam state. No counterpart in the reference, whose control optimisation
 * uses the adjoint gradient alone; the network is the learned surrogate of the map from the
 * external field's Fourier coefficients to the log electric-energy history.
 * Parameters are packed per layer: W_l [widths[l+1], widths[l]] row-major, then b_l
 * [widths[l+1]]. All pointers are device memory; row-major inputs take a leading dimension and
 * an optional row-index array (rows[m] selects the input row of batch entry m). */
typedef struct vp_mlp vp_mlp;

int vp_mlp_create(int32_t n_layers, const int32_t* widths, int32_t max_batch, vp_mlp** out_mlp);
int vp_mlp_destroy(vp_mlp* mlp);
int vp_mlp_param_count(const vp_mlp* mlp, int64_t* count);
/* Copies FP32 parameters in, zeroes the Adam moments and step count, refreshes the BF16 copies. */
int vp_mlp_set_params(vp_mlp* mlp, const float* params, void* stream);
/* Copies the FP32 parameters and/or the last parameter gradients out (either may be NULL). */
int vp_mlp_get_params(const vp_mlp* mlp, float* params, float* grads, void* stream);
/* Y[m, :] = net(X[rows ? rows[m] : m, :]) for m < M; Y may be NULL (activations are kept for a
 * following backward). */
int vp_mlp_forward(vp_mlp* mlp, const float* X, int64_t ldx, const int32_t* rows, int32_t M, float* Y,
                   int64_t ldy, void* stream);
/* Backward of the last forward (same M) from the output cotangent g_Y: parameter gradients
 * when param_grads != 0 and, when g_X is not NULL, the input cotangent. */
int vp_mlp_backward(vp_mlp* mlp, const float* g_Y, int64_t ldg, int32_t M, int32_t param_grads, float* g_X,
                    int64_t ldgx, void* stream);
/* Mean-squared-error loss of the last forward against target rows (gathered like X) and its
 * parameter gradients; loss (one float, device) may be NULL. */
int vp_mlp_mse_backward(vp_mlp* mlp, const float* target, int64_t ldt, const int32_t* rows, int32_t M,
                        float* loss, void* stream);
/* One Adam step (Kingma and Ba) on the last parameter gradients; the step count lives on the
 * device, so the call can be captured in a CUDA graph. */
int vp_mlp_adam(vp_mlp* mlp, float lr, float beta1, float beta2, float eps, void* stream);
/* Adam on one input vector c (length widths[0]) minimising J(c) = sum_n w_n exp(y_mean_n +
 * y_std_n * net(c * x_scale)_n) for `iters` steps in one single-CTA launch (warp GEMVs on the
 * network's BF16 weights, FP32 accumulation; widths up to 512); writes the best iterate and its
 * J (device pointers). The surrogate-warm-started control's search phase. */
int vp_mlp_search(vp_mlp* mlp, const float* c0, int32_t iters, float lr, float beta1, float beta2, float eps,
                  float x_scale, const float* y_mean, const float* y_std, const float* weights, float* best_c,
                  float* best_J, void* stream);
/* Nonzero bit 0: a tensor-core wait gave up (results of that call are invalid). Synchronous. */
int vp_mlp_status(vp_mlp* mlp, uint32_t* flags);
/* Resets the status flags (synchronous). */
int vp_mlp_clear_status(vp_mlp* mlp);
/* Limit, in nanoseconds, of each bounded wait with which the network's tensor-core kernels detect
 * a stalled pipeline (default 1 s; 0 gives up at the first poll that finds the work unfinished).
 * A wait that gives up raises bit 0 of vp_mlp_status; the CTA still waits (up to 1 s) for the
 * tensor-core work it issued, frees its tensor memory and returns. */
int vp_mlp_set_wait_limit(vp_mlp* mlp, uint64_t ns);
/* One BF16 tile GEMM with the MLP's epilogues: C = act(A[M,K] . B[N,K]^T + bias), act 0 none,
 * 1 GELU, 2 multiply by GELU'(aux[m, n]); outputs FP32 C32, BF16 C16 and BF16 transposed C16T
 * (each may be NULL). K, lda, ldb multiples of 8; A, B 16-byte aligned. */
int vp_gemm_bf16(const void* A, int64_t lda, const void* B, int64_t ldb, int32_t M, int32_t N, int32_t K,
                 const float* bias, int32_t act, const float* aux, int64_t ldaux, float* C32, int64_t ldc32,
                 void* C16, int64_t ldc16, void* C16T, int64_t ldc16t, uint32_t* err, void* stream);

/* --- single-stage operators (the reference's helper methods and unit-tested kernels) ------ */

/* KL(f || f_eq) integrated over phase space (warp_vp_solver/utils.py:53-76, the cost of
 * make_cost_function_kl, utils.py:79-92) and its gradient with respect to f, in float64 on the
 * device: value (one double) and grad (nx*nv doubles, may be NULL) are device pointers; f is the
 * float64 final state. The first call on a plan allocates an 8 KiB scratch (do it before any
 * stream capture). */
int vp_kl_divergence(vp_plan* plan, const double* f, double eps, double* value, double* grad, void* stream);

/* rho[i] = dv * trapz_j(f_eq[i,j] - f[i,j]). Replaces compute_rho (warp_vp_solver/solver.py:
 * 393-397) and compute_rho_kernel (warp_vp_solver/kernels.py:156-172). f: double[nx*nv],
 * rho: real[nx]. */
int vp_compute_rho(vp_plan* plan, const double* f, void* rho, void* stream);

/* E = real(ifft(m * fft(rho))) (adjoint=0) or real(ifft(conj(m) * fft(rho))) (adjoint=1) with
 * the in-block shared-memory FFT. Replaces solve_poisson_host / solve_poisson_host_adjoint
 * (warp_vp_solver/poisson.py:48-99) and compute_E_from_rho (warp_vp_solver/solver.py:399-404).
 * in, out: real[nx]. */
int vp_poisson(vp_plan* plan, const void* in, void* out, int adjoint, void* stream);

/* ee = 0.5 * dx * trapz(E^2). Replaces compute_electric_energy (warp_vp_solver/solver.py:
 * 409-412) and compute_ee_kernel (warp_vp_solver/kernels.py:175-197). E: real[nx], ee: real[1]. */
int vp_electric_energy(vp_plan* plan, const void* E, void* ee, void* stream);

/* x half-step advection by dt/2 (adjoint=0) or its transpose (adjoint=1) on an arbitrary
 * real[nx*nv] array. Replaces semilag_x_kernel / semilag_x_adjoint_kernel
 * (warp_vp_solver/kernels.py:109-130, 215-241). dt may differ from the plan's dt. */
int vp_semilag_x(vp_plan* plan, const void* in, void* out, double dt, int adjoint, void* stream);

/* v advection by dt with field E_total[nx] on an arbitrary real[nx*nv] array. adjoint=0:
 * out = V(in) (semilag_v_kernel / semilag_v_fused_kernel, warp_vp_solver/kernels.py:133-153,
 * 367-393). adjoint=1: out = V^T(in) and, when f_in and g_E are non-NULL,
 * g_E[i] = sum_j -dt*(f_in[i,i1]-f_in[i,i0])/dv * in[i,j] (semilag_v_adjoint_kernel /
 * semilag_v_fused_adjoint_kernel, warp_vp_solver/kernels.py:244-273, 396-429). */
int vp_semilag_v(vp_plan* plan, const void* in, const void* E_total, void* out, double dt,
                 int adjoint, const void* f_in, void* g_E, void* stream);

/* --- x-slab decomposition ---------------------------------------------------------------- */

/* One grid split into slabs of consecutive x rows, one slab per device (rank), for grids whose
 * state does not fit one GPU. No counterpart in the reference, which keeps every array of a solve
 * on one Warp device (warp_vp_solver/solver.py:170-203); each call below runs one piece of the
 * reference's forward step (solver.py:573-609) or adjoint step (solver.py:814-929) on a slab.
 *
 * A slab owns grid rows [row0, row0 + n_rows). Its state arrays ("_ext", real[ext_rows * nv])
 * hold `ghost` rows copied from the neighbour below, then the owned rows, then `ghost` rows
 * copied from the neighbour above (periodic in x), then pad rows the calls never read for the
 * owned rows: array row k is grid row (row0 - ghost + k) mod nx. Between calls the caller
 * fills the ghost rows of the next call's input state from the neighbours' owned rows (the
 * rows next to the boundary), and gathers every slab's row sums (real[n_rows] each) into one
 * real[nx] array in grid-row order. The field of a step (E, E + H, ee, v shifts) is then solved
 * by every rank on the same gathered sums, into a caller-held "field record" of field_bytes
 * (256-byte aligned); records of past steps feed the adjoint. A slab belongs to its plan: destroy
 * the slab first. Needs an x-invariant f_eq and the Strang scheme; the slab's per-column launch
 * shape is the plan's at vp_slab_create. The calls allocate device memory for the slab's row
 * buffers at vp_slab_create, and for one cell buffer on the first call that returns cells
 * (f_rows, f_final_rows, g_f_iv_rows). */
typedef struct vp_slab vp_slab;
/* n_rows must be at least the ghost width 2 * (largest x half-step offset in cells) + 2. */
int vp_slab_create(vp_plan* plan, int32_t row0, int32_t n_rows, vp_slab** out_slab);
int vp_slab_destroy(vp_slab* slab);
int vp_slab_geometry(const vp_slab* slab, int32_t* ghost_rows, int32_t* ext_rows, size_t* field_bytes);

/* Forward prologue: h_0 = X(f_iv - f_eq) on the owned rows of h_ext and their trapezoid row
 * sums. f_iv_ext: double[ext_rows * nv] with its ghost rows filled. */
int vp_slab_forward_start(vp_slab* slab, const double* f_iv_ext, void* h_ext, void* row_sums, void* stream);
/* Field of step n from the gathered row sums (real[nx]) and H (real[nx]): into field; E + H into
 * E_hist_row (real[nx]) and ee into ee (real[1]) when not NULL. */
int vp_slab_field(vp_slab* slab, const void* row_sums_all, const void* H, void* field, void* E_hist_row, void* ee,
                  void* stream);
/* Step n: from h_ext (h_n, ghost rows filled) and the field record of step n, h_{n+1} on the
 * owned rows of h_out_ext (NULL on the last step) and its row sums (NULL: not needed, e.g. when
 * replaying a checkpoint segment); f_{n+1} of the owned rows into f_rows (real[n_rows * nv]) and
 * f_final_rows (double[n_rows * nv]) when not NULL. */
int vp_slab_forward_step(vp_slab* slab, const void* h_ext, const void* field, void* h_out_ext, void* row_sums,
                         void* f_rows, double* f_final_rows, void* stream);

/* Adjoint prologue (n = T): w_{T-1} = X^T g on the owned rows of w_out_ext from the
 * cotangent on f_final (g_f_ext, ghost rows filled; NULL = zero), and the slope row sums of
 * the v step with h_{T-1} (h_prev_ext) and the field record of step T-1. */
int vp_slab_backward_start(vp_slab* slab, const void* g_f_ext, const void* h_prev_ext, const void* field_prev,
                           void* w_out_ext, void* slope_sums, void* stream);
/* Adjoint field of step n-1 from the gathered slope sums (real[nx]): g_E_total = -dt/dv * sums
 * + gE_hist_row, g_H += g_E_total, and grho (real[nx]) = Poisson^T(g_E_total + ee^T(gee)).
 * gE_hist_row (real[nx]) and gee (real[1], the cotangent on ee of step n-1) may be NULL. */
int vp_slab_backward_field(vp_slab* slab, const void* slope_sums_all, const void* field_prev, const void* gE_hist_row,
                           const void* gee, void* g_H, void* grho, void* stream);
/* Adjoint step n (1 <= n < T): w_{n-1} on the owned rows of w_out_ext and its slope row sums,
 * from w_ext (w_n, ghost rows filled), the cotangent on f_hist[n-1] (g_f_ext, ghost rows
 * filled; NULL = zero), grho of step n (real[nx]), the field records of steps n and n-1 and
 * h_{n-1} (h_prev_ext). */
int vp_slab_backward_step(vp_slab* slab, const void* w_ext, const void* g_f_ext, const void* grho,
                          const void* field_n, const void* field_prev, const void* h_prev_ext, void* w_out_ext,
                          void* slope_sums, void* stream);
/* Adjoint epilogue (n = 0): the cotangent on f_iv's owned rows (real[n_rows * nv]) from w_0
 * (ghost rows filled), grho of step 0 and the field record of step 0. */
int vp_slab_backward_finish(vp_slab* slab, const void* w_ext, const void* grho, const void* field0, void* g_f_iv_rows,
                            void* stream);

/* --- launch configuration (autotuning) ---------------------------------------------------- */

/* Launch shape of a plan's fused step kernels. No reference counterpart: the reference launches
 * one thread per cell (warp_vp_solver/solver.py:215-265) and has no tunables beyond
 * aggressive_tile_size (solver.py:99-167). */
typedef struct vp_launch_config {
    int32_t rows_per_cta;     /* R: 1, 2, 4, 8 or 16; must divide nx and be <= nx/2 (or be 1) */
    int32_t threads;          /* threads per CTA: a multiple of 32 in [32, 256], one column each */
    int32_t n_chunks;         /* column chunks per row block, >= 1                                */
    int32_t chunk_cols;       /* columns per chunk (derived: ceil(nv / n_chunks) rounded to 32)   */
    int32_t tail_inline;      /* 1: the Poisson tail runs in the last CTA of the fused launch     */
    int32_t tail_threads;     /* threads of the separate tail launch (tail_inline == 0)           */
    int64_t fused_smem_bytes; /* dynamic shared memory of the fused launch                        */
    int64_t tail_smem_bytes;  /* dynamic shared memory of the tail launch (0: global scratch)     */
    int32_t cluster_size;     /* > 0: whole time loops run in one launch of one cluster of this   */
                              /* many CTAs with the state in distributed shared memory            */
                              /* (cluster-resident path); 0: one fused launch per step            */
    int32_t cluster_threads;  /* threads per CTA of the cluster-resident kernels                  */
    int64_t cluster_smem_bytes; /* dynamic shared memory per CTA of the cluster-resident kernels  */
    int32_t stage_rows;       /* > 0: per-step forward launches use the staged kernel with this   */
                              /* many rows per CTA (4, 8, 16 or 32; x-invariant f_eq only); 0: off */
    int32_t stage_threads;    /* columns (= threads) per CTA of the staged kernel, dividing nv    */
    int32_t stage_span;       /* rows of its shared-memory staging buffer (derived)               */
    int64_t stage_smem_bytes; /* dynamic shared memory of the staged kernel (derived)             */
    int32_t persist_rows;     /* > 0: float32 forward loops (and the adjoint's recomputation of   */
                              /* checkpoint segments) run as one cooperative launch per loop     */
                              /* whose CTAs own bands of this many rows (4, 8 or 16) and meet at */
                              /* a bounded grid barrier once per step; 0: off. Needs an          */
                              /* x-invariant f_eq, nv a multiple of 256 and nx <= 16384; on by   */
                              /* default where the state is not cluster-resident and each CTA  */
                              /* can solve the field on its own window rows (nx of a few 1000s)  */
    int32_t persist_ctas;     /* CTAs of that launch (derived)                                    */
    int64_t persist_smem_bytes; /* dynamic shared memory per CTA of that launch (derived)        */
    int32_t strip_rows;       /* > 0: float32 Strang steps (forward, recomputation, adjoint) run  */
                              /* as two launches each: a strip kernel whose 64-thread CTAs walk */
                              /* runs of bands of this many rows (4, 8 or 16) down one 256-column*/
                              /* chunk with the window rows in a shared-memory ring, and a field */
                              /* kernel (circulant product, 32 rows per CTA); 0: off. Same      */
                              /* conditions as persist_rows; on by default where the persistent  */
                              /* loop is not (the field would need slices, nx of several 1000s) */
                              /* and the state is not cluster-resident. persist_rows wins when  */
                              /* both are set.                                                   */
    int32_t strip_ctas;       /* CTAs of the forward strip launch (derived)                       */
    int64_t strip_smem_bytes; /* dynamic shared memory per CTA of the forward strip launch        */
    int32_t strip_cols;       /* columns a forward strip CTA walks: 256 (two warps) or 128 (one   */
                              /* warp); 0 in vp_plan_set_config keeps the current width          */
    int32_t strip_adj_cols;   /* the same for the adjoint strip CTAs                              */
} vp_launch_config;

/* Reads the plan's current launch shape. */
int vp_plan_get_config(const vp_plan* plan, vp_launch_config* out);

/* Sets rows_per_cta, threads, n_chunks, cluster_size, stage_rows, stage_threads, persist_rows, strip_rows, strip_cols and strip_adj_cols (the other
 * fields are derived and ignored). cluster_size must be 0 or a power of two in [2, 16] that splits nx into 1, 2, 4, 8,
 * 16 or 32 rows per CTA whose state fits in shared memory; the cluster-resident path is used for forward calls without a tape or with
 * checkpoint interval 1, and for backward calls with checkpoint interval 1. Workspace sizes
 * depend on n_chunks and strip_rows: query vp_workspace_bytes() again after changing them. */
int vp_plan_set_config(vp_plan* plan, const vp_launch_config* cfg);

/* Time-splitting scheme of a plan's forward and adjoint loops.
 * VP_SCHEME_STRANG: X(dt/2) V(dt) X(dt/2) every step (the reference's default path,
 *   warp_vp_solver/solver.py:418-612, 742-1105).
 * VP_SCHEME_MERGED: the reference's aggressive path (`aggressive=True`, solver.py:618-736,
 *   1111-1338): the trailing X(dt/2) of a step and the leading X(dt/2) of the next are one
 *   X(dt); f_hist[t] holds the state after that X(dt) (f_final for the last step). Runs on the
 *   per-column kernels (the cluster-resident and staged paths are Strang only). */
#define VP_SCHEME_STRANG 0
#define VP_SCHEME_MERGED 1
int vp_plan_set_scheme(vp_plan* plan, int32_t scheme);
int vp_plan_get_scheme(const vp_plan* plan, int32_t* scheme);

/* --- diagnostics ------------------------------------------------------------------------ */

/* Copies the last error message of the calling thread into buf (always NUL-terminated). */
int vp_get_last_error(char* buf, size_t buf_len);

/* Kernel launches issued by the calling thread since the last reset (for launch accounting). */
int64_t vp_launch_count(void);
void vp_reset_launch_count(void);

/* ABI version (VP_ABI_VERSION). */
int vp_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* VP_B200_H */
