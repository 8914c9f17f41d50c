// C ABI (include/vp_b200.h): plan set-up, validation, workspace/tape layout and the host-side
// orchestration of the fused forward and adjoint launches. No device allocation and no device
// synchronisation happen inside vp_forward / vp_backward; they only enqueue work on the
// caller's stream.

#include "../../include/vp_b200.h"
#include "vp_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

namespace vpb {

static thread_local char g_err[512] = "";
static thread_local int64_t g_launches = 0;

void count_launch(int n) { g_launches += n; }

int set_err(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

static int cuda_err(cudaError_t e, const char* what) {
    return set_err(VP_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

#define VP_CUDA(call, what)                        \
    do {                                           \
        cudaError_t e_ = (call);                   \
        if (e_ != cudaSuccess) return cuda_err(e_, what); \
    } while (0)

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Poisson work area placement: inside the fused launch up to kInlineTailBytes of shared memory
// (it is requested by every CTA of that launch), else in a separate single-CTA launch with up to
// kTailSmemBytes of shared memory, else in global scratch.
static const size_t kInlineTailBytes = 24 * 1024;
static const size_t kTailSmemBytes = 200 * 1024;

}  // namespace vpb

using namespace vpb;

struct vp_plan {
    int nx = 0, nv = 0, dtype = VP_F32;
    double dx = 0, dv = 0, dt = 0, period_x = 0, period_v = 0;
    int feq2d = 0;
    int device = 0;
    int pow2 = 0, log2nx = 0;
    int tail_inline = 0;       // Poisson tail inside the fused launch (small nx)
    size_t tail_smem = 0;      // dynamic shared memory of the separate tail launch (0: global scratch)
    int tail_tw_stage = 0;     // the separate tail's FFT twiddles are laid out per stage
    int tail_threads = 0;
    LaunchCfg cfg{};
    std::vector<double> host_feq;  // f_eq as given (host), for recognising identical plans
    std::vector<double> host_vs;
    int res_cn = 0;            // cluster size of the cluster-resident path (0: not used)
    long long mx_lo = 0, mx_hi = 0;  // extremes of the unreduced x half-step offsets floor(-s_j)
    int res_threads = 0;
    size_t res_smem = 0;
    int res_vrows = 0;      // the resident forward computes the v step once per (row, column)
    // device tables (owned)
    double* d_feq = nullptr;   // nv (x-invariant) or nx*nv
    double* d_vs = nullptr;    // nv
    int* d_mx = nullptr;       // nv
    void* d_tx = nullptr;      // nv reals
    int* d_mxf = nullptr;      // merged scheme: full-step x offsets (mod nx)      [nv]
    void* d_txf = nullptr;     // merged scheme: full-step x weights               [nv]
    double* d_txf64 = nullptr; // merged scheme: full-step x weights in float64    [nv]
    int merged = 0;            // 1: merged-Strang (aggressive) scheme
    double feq_integral = 0.0; // trapezoid integral of f_eq over xs and vs (for the KL cost)
    double* d_kl = nullptr;    // KL cost scratch: 2 * kKlBlocks + 2 doubles
    unsigned* d_status = nullptr;  // VP_STATUS_* flags raised on the device (vp_plan_status)
    std::vector<cudaEvent_t> ev_written, ev_copied;   // streamed-history slots
    void* d_vtab = nullptr;    // staged step: [2][2*kStageHalo][nv] reals (x-invariant f_eq only)
    LaunchCfg scfg{};          // staged forward step (R rows x threads columns per CTA)
    int stage_span = 0;        // rows its staging buffer holds (0: staged step not used)
    std::vector<int> host_mx;  // x half-step offsets (host copy, for staged shapes)
    size_t sb_smem = 0;        // staged adjoint step's shared memory (0: adjoint not staged)
    double* d_tx64 = nullptr;  // nv
    void* d_tw = nullptr;      // nx/2 complex
    void* d_mult = nullptr;    // nx reals (imaginary part)
    void* d_circ = nullptr;    // nx reals
    // persistent forward path (vp_persist.cu)
    PersistHost pst;           // launch shape and host tables (pst.R == 0: not eligible)
    int pst_on = 0;            // forward loops (and the adjoint's recomputation) use it
    int2* d_pquad = nullptr;   // [nv / 4]
    float4* d_ptq = nullptr;   // [nv / 4]
    int2* d_pchunk = nullptr;  // [nv / 256]
    float* d_dfeq = nullptr;   // [nv]
    float* d_ctab2 = nullptr;  // [3 nx + 8]
    // strip step path (vp_strip.cu): per-step kernels for large grids on the same quad tables
    StripHost strip;           // launch shape (strip.R == 0: not eligible)
    int strip_on = 0;          // per-step forward and adjoint steps (and recomputation) use it
    int2* d_echunk = nullptr;  // ensembles on the strip kernels: quad shift range per 128 columns
    std::vector<long long> host_msigned;   // unreduced x half-step offsets (re-shaping the paths)
    std::vector<double> host_tx;           // their weights
    std::vector<long long> host_mxs;       // unreduced x half-step offsets of every plan (x slabs)
    unsigned long long wait_ns = 1000000000ull;   // limit of each device-side grid barrier wait
};

namespace vpb {

static size_t real_size(const vp_plan* p) { return p->dtype == VP_F64 ? 8 : 4; }
static size_t vshift_size(const vp_plan* p) { return p->dtype == VP_F64 ? 16 : 8; }

// Set while the calling thread's stream is being captured into a CUDA graph: pointer
// attribute queries are skipped then (the same call is validated when run eagerly).
static thread_local bool g_capturing = false;

struct CaptureScope {
    explicit CaptureScope(bool on) { g_capturing = on; }
    ~CaptureScope() { g_capturing = false; }
};

static bool stream_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return st != cudaStreamCaptureStatusNone;
}

static int check_dev_ptr(const void* ptr, const char* name, int device) {
    if (ptr == nullptr) return set_err(VP_ERR_ARG, "%s must not be NULL", name);
    if (g_capturing) return VP_OK;
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(VP_ERR_ARG, "%s is not a CUDA-visible pointer (%s)", name, cudaGetErrorName(e));
    }
    if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
        return set_err(VP_ERR_ARG, "%s must be device memory (got host or unregistered memory)", name);
    if (at.type == cudaMemoryTypeDevice && at.device != device)
        return set_err(VP_ERR_ARG, "%s lives on device %d but the plan is bound to device %d", name,
                       at.device, device);
    return VP_OK;
}

static int check_opt_ptr(const void* ptr, const char* name, int device) {
    return ptr == nullptr ? VP_OK : check_dev_ptr(ptr, name, device);
}

// Launch shape of the fused kernels: R rows per CTA (largest of 16, 8, 4, 2 that divides nx and
// leaves at least two row blocks, else 1), one column per thread, and enough column chunks per
// row block for about eight CTAs per SM; R is lowered while the grid has fewer than two CTAs per
// SM. Halo rows cost (R+2)/R V evaluations per output row, so larger R is preferred.
static LaunchCfg choose_cfg(int nx, int nv, int n_sms) {
    LaunchCfg c{};
    c.threads = nv >= 128 ? 128 : ((nv + 31) / 32) * 32;
    int R = 1;
    for (int r : {16, 8, 4, 2}) {
        if (nx % r == 0 && r <= nx / 2) {
            R = r;
            break;
        }
    }
    const int max_chunks = std::max(1, nv / c.threads);
    auto chunks_for = [&](int rr) {
        const int rows = nx / rr;
        return std::max(1, std::min(max_chunks, (8 * n_sms + rows - 1) / rows));
    };
    int chunks = chunks_for(R);
    while (R > 1 && (nx / R) * chunks < 2 * n_sms) {
        R /= 2;
        chunks = chunks_for(R);
    }
    int chunk_cols = (nv + chunks - 1) / chunks;
    chunk_cols = ((chunk_cols + 31) / 32) * 32;
    c.R = R;
    c.chunk_cols = chunk_cols;
    c.n_chunks = (nv + chunk_cols - 1) / chunk_cols;
    return c;
}

// Largest shared memory a CTA may request on sm_100.
static const size_t kMaxSmemPerCta = 227 * 1024;

// Halo rows that a resident CTA keeps below and above its own rows: the forward reads rows
// g + 2m .. g + 2m + RPT + 1 and the adjoint rows g - 2m - 2 .. g - 2m + RPT - 1 of a step's state
// for x offsets m in [mx_lo, mx_hi] (vp_resident.cu).
static void res_halo_rows(const vp_plan* p, int* lo, int* hi) {
    const long long f_lo = -2 * p->mx_lo, f_hi = 2 * p->mx_hi + 2;
    const long long b_lo = 2 * p->mx_hi + 2, b_hi = -2 * p->mx_lo;
    *lo = (int)std::max(0LL, std::max(f_lo, b_lo));
    *hi = (int)std::max(0LL, std::max(f_hi, b_hi));
}

// Checks that a cluster-resident configuration of cn CTAs can launch; returns its shared memory
// (0 when it cannot). *vrows is set when the forward's phase-A plane (the v step of the local rows,
// float32 with an x-invariant f_eq, 4-column quads tiling the block) fits as well; the shared
// memory returned then includes it.
static size_t res_config_ok(const vp_plan* p, int cn, int* vrows) {
    *vrows = 0;
    if (cn < 2 || cn > 16 || (cn & (cn - 1)) != 0 || p->nx % cn != 0) return 0;
    const int Rc = p->nx / cn;
    if (!res_rows_supported(Rc)) return 0;
    // offsets within one period, with a range short enough to recover them from mx (mod nx)
    if (p->mx_lo < -p->nx || p->mx_hi > p->nx || p->mx_hi - p->mx_lo >= p->nx / 2) return 0;
    int hlo = 0, hhi = 0;
    res_halo_rows(p, &hlo, &hhi);
    if (hlo + hhi >= p->nx) return 0;   // local rows of a CTA span less than two periods
    const size_t smem = res_smem_size(p->nx, p->nv, Rc, hlo + hhi, real_size(p), false);
    if (smem > kMaxSmemPerCta) return 0;
    const int threads = res_threads(Rc, p->nv);
    if (threads == 0) return 0;
    const int n = p->dtype == VP_F64 ? res_max_clusters<double>(p->feq2d != 0, cn, Rc, p->nv, smem)
                                     : res_max_clusters<float>(p->feq2d != 0, cn, Rc, p->nv, smem);
    if (n <= 0) return 0;
    if (p->dtype == VP_F32 && !p->feq2d && p->nv % 4 == 0 && threads % (p->nv / 4) == 0) {
        const size_t smem_v = res_smem_size(p->nx, p->nv, Rc, hlo + hhi, real_size(p), true);
        if (smem_v <= kMaxSmemPerCta && res_max_clusters<float>(false, cn, Rc, p->nv, smem_v) > 0) {
            *vrows = 1;
            return smem_v;
        }
    }
    return smem;
}


static size_t fused_smem(const vp_plan* p, int R) {
    const size_t red = ((size_t)32 * R * real_size(p) + 15) & ~(size_t)15;
    return red + (p->tail_inline ? poisson_area_size(p->nx, real_size(p)) : 0);
}

// Staged forward step with R rows x C columns per CTA (C divides nv): its staging buffer holds
// the widest x window of any column block, R + 2 + 2 * (max - min signed x offset over the
// block's columns) rows. Returns false (and leaves the plan unchanged) when the shape is not
// usable.
static bool staged_config(vp_plan* p, int R, int C, int blocks_per_cta = 0) {
    const int nx = p->nx, nv = p->nv;
    if (p->d_vtab == nullptr || (C != 128 && C != 256) || nv % C != 0) return false;
    if (!(R == 4 || R == 8 || R == 16 || R == 32) || nx % R != 0 || R > nx / 4) return false;
    int dmax = 0;
    for (int c0 = 0; c0 < nv; c0 += C) {
        int lo = 1 << 30, hi = -(1 << 30);
        for (int j = c0; j < c0 + C; ++j) {
            const int sm = p->host_mx[j] > nx / 2 ? p->host_mx[j] - nx : p->host_mx[j];
            lo = std::min(lo, sm);
            hi = std::max(hi, sm);
        }
        dmax = std::max(dmax, hi - lo);
    }
    const int span = R + 2 + 2 * dmax;
    if (span > nx) return false;
    const size_t rs = real_size(p);
    const size_t red = ((size_t)32 * R * rs + 15) & ~(size_t)15;
    const size_t stage = staged_smem_bytes(span, C, rs);
    const size_t tail = p->tail_inline ? poisson_area_size(nx, rs) : 0;
    const size_t smem = red + std::max(stage, tail);
    if (smem > 160 * 1024) return false;
    // column blocks per CTA: enough CTAs for two per SM, at most 8 blocks
    const int n_blocks = nv / C;
    int nb = blocks_per_cta;
    if (nb <= 0) {
        int sms = 148;
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        nb = 1;
        while (nb < 8 && n_blocks % (2 * nb) == 0 && (long long)(nx / R) * (n_blocks / (2 * nb)) >= 2LL * sms)
            nb *= 2;
    }
    if (nb < 1 || n_blocks % nb != 0) return false;
    const cudaError_t e = p->dtype == VP_F64 ? set_staged_smem_limit<double>(smem) : set_staged_smem_limit<float>(smem);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    // the adjoint step stages the same window of w plus the CTA's own rows of h_{n-1}
    size_t sb = red + std::max(staged_bwd_smem_bytes(span, R, C, rs), tail);
    if (sb > 200 * 1024) {
        sb = 0;
    } else {
        const cudaError_t eb = p->dtype == VP_F64 ? set_staged_bwd_smem_limit<double>(sb)
                                                  : set_staged_bwd_smem_limit<float>(sb);
        if (eb != cudaSuccess) {
            cudaGetLastError();
            sb = 0;
        }
    }
    p->scfg.R = R;
    p->scfg.threads = C;
    p->scfg.chunk_cols = C * nb;
    p->scfg.n_chunks = n_blocks / nb;
    p->scfg.smem = smem;
    p->stage_span = span;
    p->sb_smem = sb;
    return true;
}

// Default staged shape: C = 256 (or 128) columns, and the largest R of 16, 8, 4 that still gives
// two CTAs per SM (R = 32 widens the staged window; an autotuned shape may still choose it).
static void choose_staged(vp_plan* p, int n_sms) {
    p->stage_span = 0;
    for (int C : {256, 128}) {
        if (p->nv % C != 0) continue;
        int best = 0;
        for (int r : {16, 8, 4}) {
            if (p->nx % r != 0 || r > p->nx / 4) continue;
            if (best == 0) best = r;
            if ((long long)(p->nx / r) * (p->nv / C) >= 2LL * n_sms) {
                best = r;
                break;
            }
        }
        if (best == 0) continue;
        for (int r = best; r >= 4; r /= 2)
            if (staged_config(p, r, C)) return;
    }
}

// Checkpoint interval. every > 0 is used as given (capped at n_steps). every == 0 (automatic)
// keeps every step's state when that tape fits in kStoreAllBytes, and otherwise checkpoints every
// ceil(sqrt(n_steps)) steps, recomputing the states in between during the adjoint.
static const size_t kStoreAllBytes = (size_t)256 << 20;

static int resolve_every(const vp_plan* p, int n_steps, int every) {
    if (n_steps <= 0) return 1;
    if (every <= 0) {
        const size_t all = (size_t)n_steps * p->nx * p->nv * real_size(p);
        if (all <= kStoreAllBytes) return 1;
        int k = (int)std::ceil(std::sqrt((double)n_steps));
        return std::max(1, std::min(k, n_steps));
    }
    return std::min(every, n_steps);
}

struct WsLayout {
    size_t hbuf0, hbuf1, seg, part, counter, vsh, E, grho, gscratch, prho, pvsh, peep, pbar;
    size_t srho, sgE, seep, sctr, total;
};

static WsLayout ws_layout(const vp_plan* p, int n_steps, int every) {
    const size_t nxnv = (size_t)p->nx * p->nv * real_size(p);
    const int K = resolve_every(p, n_steps, every);
    WsLayout L{};
    size_t off = 0;
    L.hbuf0 = off; off += align256(nxnv);
    L.hbuf1 = off; off += align256(nxnv);
    L.seg = off; off += align256(nxnv * (size_t)std::max(0, K - 1));
    const int part_chunks = std::max({p->cfg.n_chunks, p->stage_span > 0 ? p->scfg.n_chunks : 0,
                                      p->strip.R > 0 ? std::max(p->strip.n_chunks, p->strip.b_n_chunks) : 0});
    L.part = off; off += align256((size_t)part_chunks * p->nx * real_size(p));
    L.counter = off; off += 256;
    L.vsh = off; off += align256((size_t)p->nx * vshift_size(p));
    L.E = off; off += align256((size_t)p->nx * real_size(p));
    L.grho = off; off += align256((size_t)p->nx * real_size(p));
    L.gscratch = off; off += align256((size_t)2 * p->nx * real_size(p));
    if (p->pst.R > 0) {   // persistent path: rho (two steps), field-slice shifts, energy partials, barrier
        L.prho = off; off += align256((size_t)2 * p->nx * sizeof(float));
        L.pvsh = off; off += align256((size_t)p->nx * sizeof(VShift<float>));
        L.peep = off; off += align256((size_t)std::max(1, n_steps) * p->pst.G * sizeof(double));
        L.pbar = off; off += 256;
    }
    if (p->strip.R > 0) {   // strip path: rho, g_E, field energy partials, band and field counters
        L.srho = off; off += align256((size_t)p->nx * sizeof(float));
        L.sgE = off; off += align256((size_t)p->nx * sizeof(float));
        L.seep = off; off += align256((size_t)p->strip.field_ctas * sizeof(double));
        L.sctr = off; off += align256((size_t)(p->strip.n_bands + 1) * sizeof(unsigned));
    }
    L.total = off;
    return L;
}

struct TapeLayout {
    size_t ckpt, E, vsh, total;
    int K, n_ckpt;
};

static TapeLayout tape_layout(const vp_plan* p, int n_steps, int every) {
    TapeLayout L{};
    L.K = resolve_every(p, n_steps, every);
    L.n_ckpt = n_steps > 0 ? (n_steps + L.K - 1) / L.K : 0;
    const size_t nxnv = (size_t)p->nx * p->nv * real_size(p);
    size_t off = 0;
    L.ckpt = off; off += align256(nxnv * (size_t)L.n_ckpt);
    L.E = off; off += align256((size_t)n_steps * p->nx * real_size(p));
    L.vsh = off; off += align256((size_t)n_steps * p->nx * vshift_size(p));
    L.total = off;
    return L;
}

template <typename T>
static PoissonTables<T> poisson_tables(const vp_plan* p, unsigned char* ws, const WsLayout* L,
                                       bool in_smem) {
    PoissonTables<T> P{};
    P.nx = p->nx;
    P.log2nx = p->log2nx;
    P.pow2 = p->pow2;
    P.tw = static_cast<const typename Cplx<T>::type*>(p->d_tw);
    P.mult_im = static_cast<const T*>(p->d_mult);
    P.circ = static_cast<const T*>(p->d_circ);
    P.gscratch = (ws != nullptr && L != nullptr) ? reinterpret_cast<T*>(ws + L->gscratch) : nullptr;
    P.use_smem = in_smem ? 1 : 0;
    return P;
}

// Arguments of a persistent launch common to the forward loop and the adjoint's recomputation.
static PersistArgs persist_args(const vp_plan* p, unsigned char* ws, const WsLayout& L) {
    PersistArgs a{};
    a.nx = p->nx;
    a.nv = p->nv;
    a.n_chunks = p->nv / 256;
    a.quad = p->d_pquad;
    a.tq = p->d_ptq;
    a.chunk = p->d_pchunk;
    a.feq = p->d_feq;
    a.dfeq = p->d_dfeq;
    a.vtab = static_cast<const float*>(p->d_vtab);
    a.ctab = p->d_ctab2;
    a.dv = (float)p->dv;
    a.dx = (float)p->dx;
    a.dtdv = (float)(p->dt / p->dv);
    a.rho = reinterpret_cast<float*>(ws + L.prho);
    a.vsh_g = reinterpret_cast<VShift<float>*>(ws + L.pvsh);
    a.eep = reinterpret_cast<double*>(ws + L.peep);
    a.bar = reinterpret_cast<unsigned*>(ws + L.pbar);
    a.status = p->d_status;
    a.wait_ns = p->wait_ns;
    return a;
}

// Table arguments of a strip step launch (forward, replay or adjoint).
template <typename A>
static void strip_tables(const vp_plan* p, A& a, int gt) {
    a.nx = p->nx;
    a.nv = p->nv;
    a.quad = p->d_pquad;
    a.tq = p->d_ptq;
    a.chunk = gt == 32 ? p->d_echunk : p->d_pchunk;   // quad shift range per chunk of the group width
    a.dfeq = p->d_dfeq;
    a.vtab = static_cast<const float*>(p->d_vtab);
    a.feq = p->d_feq;
}

// The strip step kernels run this plan's float32 Strang steps.
static bool strip_active(const vp_plan* p) { return p->strip_on && p->strip.R > 0 && !p->merged && p->dtype == VP_F32; }

// Field of step n+1 from the strip kernel's rho (forward) into the step's outputs.
static int strip_field_fwd(const vp_plan* p, unsigned char* ws, const WsLayout& L, const float* H, float* E_out,
                           float* E_hist_out, VShift<float>* vsh_out, float* ee_out, cudaStream_t s) {
    StripFieldArgs f{};
    f.nx = p->nx;
    f.nv = p->nv;
    f.adjoint = 0;
    f.x = reinterpret_cast<const float*>(ws + L.srho);
    f.ctab = p->d_ctab2;
    f.H = H;
    f.dtdv = (float)(p->dt / p->dv);
    f.dx = (float)p->dx;
    f.E_out = E_out;
    f.E_hist_out = E_hist_out;
    f.vsh_out = vsh_out;
    f.ee_out = ee_out;
    f.eep = reinterpret_cast<double*>(ws + L.seep);
    f.counter = reinterpret_cast<unsigned*>(ws + L.sctr) + p->strip.n_bands;
    VP_CUDA(launch_strip_field(f, p->strip, s), "strip field launch");
    return VP_OK;
}

// ---------------------------------------------------------------------------------------------
// forward orchestration
// ---------------------------------------------------------------------------------------------
// f_hist streamed to pinned host memory: step n's f goes to device slot n % slots of f_hist (the
// ring) and is copied to host + n*nx*nv on `copy`; the compute stream waits for a slot's previous
// copy before overwriting it, and at the end for every copy.
struct HistRing {
    unsigned char* host;
    int slots;
    cudaStream_t copy;
    cudaEvent_t* written;
    cudaEvent_t* copied;
};

template <typename T>
static int forward_impl(vp_plan* p, const double* f_iv, const T* H, int T_steps, double* f_final,
                        T* f_hist, T* E_hist, T* ee_hist, unsigned char* tape, int every,
                        unsigned char* ws, cudaStream_t s, const HistRing* ring = nullptr) {
    const int nx = p->nx, nv = p->nv;
    const size_t nxnv = (size_t)nx * nv;
    const WsLayout L = ws_layout(p, T_steps, every);
    const TapeLayout TL = tape_layout(p, T_steps, every);
    const int K = TL.K;
    T* hbuf[2] = {reinterpret_cast<T*>(ws + L.hbuf0), reinterpret_cast<T*>(ws + L.hbuf1)};
    unsigned* counter = reinterpret_cast<unsigned*>(ws + L.counter);
    T* part = reinterpret_cast<T*>(ws + L.part);
    VShift<T>* vsh_ws = reinterpret_cast<VShift<T>*>(ws + L.vsh);
    T* E_ws = reinterpret_cast<T*>(ws + L.E);
    T* ckpt = tape ? reinterpret_cast<T*>(tape + TL.ckpt) : nullptr;
    T* E_all = tape ? reinterpret_cast<T*>(tape + TL.E) : nullptr;
    VShift<T>* vsh_all = tape ? reinterpret_cast<VShift<T>*>(tape + TL.vsh) : nullptr;

    if (p->res_cn > 0 && !p->merged && ring == nullptr && (tape == nullptr || K == 1)) {
        ResFwdArgs<T> r{};
        r.nx = nx;
        r.nv = nv;
        r.n_steps = T_steps;
        r.Rc = nx / p->res_cn;
        r.f_iv = f_iv;
        r.H = H;
        r.mx = p->d_mx;
        r.tx = static_cast<const T*>(p->d_tx);
        r.tx64 = p->d_tx64;
        r.feq = p->d_feq;
        r.feq_rs = p->feq2d ? nv : 0;
        r.f_final = f_final;
        r.f_hist = f_hist;
        r.E_hist = E_hist;
        r.ee_hist = ee_hist;
        r.h_tape = ckpt;
        r.E_tape = E_all;
        r.vsh_tape = vsh_all;
        r.P = poisson_tables<T>(p, nullptr, nullptr, true);
        r.dv = (T)p->dv;
        r.dx = (T)p->dx;
        r.dtdv = (T)(p->dt / p->dv);
        res_halo_rows(p, &r.h_lo, &r.h_hi);
        r.mx_lo = (int)p->mx_lo;
        r.vrows = p->res_vrows;
        VP_CUDA(launch_res_fwd<T>(r, p->feq2d != 0, p->res_cn, p->res_threads, p->res_smem, s),
                "cluster-resident forward launch");
        return VP_OK;
    }

    if constexpr (sizeof(T) == 4) {
        if (p->pst_on && !p->merged && ring == nullptr) {
            PersistArgs pa = persist_args(p, ws, L);
            pa.mode = 0;
            pa.n_steps = T_steps;
            pa.K = K;
            pa.hbuf0 = reinterpret_cast<float*>(hbuf[0]);
            pa.hbuf1 = reinterpret_cast<float*>(hbuf[1]);
            pa.ckpt = reinterpret_cast<float*>(ckpt);
            pa.f_iv = f_iv;
            pa.H = reinterpret_cast<const float*>(H);
            pa.f_hist = reinterpret_cast<float*>(f_hist);
            pa.f_final = f_final;
            pa.E_hist = reinterpret_cast<float*>(E_hist);
            pa.ee_hist = reinterpret_cast<float*>(ee_hist);
            pa.E_tape = reinterpret_cast<float*>(E_all);
            pa.vsh_tape = reinterpret_cast<VShift<float>*>(vsh_all);
            VP_CUDA(launch_persist_fwd(pa, p->pst, s), "persistent forward launch");
            return VP_OK;
        }
    }

    VP_CUDA(cudaMemsetAsync(counter, 0, 256, s), "cudaMemsetAsync(counter)");
    const bool strip = sizeof(T) == 4 && strip_active(p);
    if (strip)
        VP_CUDA(cudaMemsetAsync(ws + L.sctr, 0, (size_t)(p->strip.n_bands + 1) * sizeof(unsigned), s),
                "cudaMemsetAsync(strip counters)");

    auto h_slot = [&](int n) -> T* {
        if (ckpt != nullptr && n % K == 0) return ckpt + (size_t)(n / K) * nxnv;
        return hbuf[n & 1];
    };

    FwdArgs<T> a{};
    a.nx = nx;
    a.nv = nv;
    a.n_chunks = p->cfg.n_chunks;
    a.chunk_cols = p->cfg.chunk_cols;
    a.mx = p->d_mx;
    a.tx = static_cast<const T*>(p->d_tx);
    a.tx64 = p->d_tx64;
    a.feq = p->d_feq;
    a.feq_rs = p->feq2d ? nv : 0;
    a.counter = p->tail_inline ? counter : nullptr;
    a.P = poisson_tables<T>(p, ws, &L, p->tail_inline || p->tail_smem > 0);
    a.dv = (T)p->dv;
    a.dx = (T)p->dx;
    a.dtdv = (T)(p->dt / p->dv);
    a.H = H;
    a.vtab = static_cast<const T*>(p->d_vtab);
    a.stage_span = p->stage_span;

    // prologue: h_0, rho_0 -> E_0
    a.f_iv = f_iv;
    a.h_in = nullptr;
    a.h_out = h_slot(0);
    a.vsh = nullptr;
    a.part = part;
    a.E_out = E_all ? E_all : E_ws;
    a.vsh_out = vsh_all ? vsh_all : vsh_ws;
    a.E_hist_out = E_hist;
    a.ee_out = ee_hist;
    a.f_hist_n = nullptr;
    a.f_final = nullptr;
    VP_CUDA(launch_fwd<T>(a, p->cfg, 0, p->feq2d != 0, s), "forward prologue launch");
    if (!p->tail_inline) VP_CUDA(launch_fwd_tail<T>(a, p->tail_threads, p->tail_smem, p->tail_tw_stage != 0, s), "forward tail launch");

    for (int n = 0; n < T_steps; ++n) {
        const bool last = (n == T_steps - 1);
        a.f_iv = nullptr;
        a.h_in = h_slot(n);
        a.h_out = last ? nullptr : h_slot(n + 1);
        a.vsh = vsh_all ? vsh_all + (size_t)n * nx : vsh_ws;
        int slot = 0;
        if (ring != nullptr) {
            slot = n % ring->slots;
            if (n >= ring->slots) VP_CUDA(cudaStreamWaitEvent(s, ring->copied[slot], 0), "wait for history slot");
            a.f_hist_n = f_hist + (size_t)slot * nxnv;
        } else {
            a.f_hist_n = f_hist ? f_hist + (size_t)n * nxnv : nullptr;
        }
        a.f_final = last ? f_final : nullptr;
        a.part = last ? nullptr : part;
        a.E_out = E_all ? E_all + (size_t)(n + 1) * nx : E_ws;
        a.vsh_out = vsh_all ? vsh_all + (size_t)(n + 1) * nx : vsh_ws;
        a.E_hist_out = (E_hist && !last) ? E_hist + (size_t)(n + 1) * nx : nullptr;
        a.ee_out = (ee_hist && !last) ? ee_hist + (n + 1) : nullptr;
        if (p->merged && !last) {
            // merged-Strang inner step: one X(dt) with the full-step tables
            FwdArgs<T> am = a;
            am.mx = p->d_mxf;
            am.tx = static_cast<const T*>(p->d_txf);
            am.tx64 = p->d_txf64;
            VP_CUDA(launch_fwd<T>(am, p->cfg, 3, p->feq2d != 0, s), "forward merged step launch");
        } else if (strip) {
            if constexpr (sizeof(T) == 4) {
                StripFwdArgs sa{};
                strip_tables(p, sa, p->strip.gt);
                sa.h_in = a.h_in;
                sa.h_out = a.h_out;
                sa.vsh = a.vsh;
                sa.f_hist_n = a.f_hist_n;
                sa.f_final = a.f_final;
                sa.part = last ? nullptr : part;
                sa.run_ctr = reinterpret_cast<unsigned*>(ws + L.sctr);
                sa.rho_out = reinterpret_cast<float*>(ws + L.srho);
                sa.dv = (float)p->dv;
                VP_CUDA(launch_strip_fwd(sa, p->strip, s), "strip forward step launch");
                if (!last) {
                    const int rc = strip_field_fwd(p, ws, L, H, a.E_out, a.E_hist_out, a.vsh_out, a.ee_out, s);
                    if (rc != VP_OK) return rc;
                }
            }
        } else if (p->stage_span > 0 && !p->merged) {
            a.n_chunks = p->scfg.n_chunks;
            a.chunk_cols = p->scfg.chunk_cols;
            VP_CUDA(launch_fwd_staged<T>(a, p->scfg, s), "forward step launch");
        } else {
            VP_CUDA(launch_fwd<T>(a, p->cfg, 1, p->feq2d != 0, s), "forward step launch");
        }
        if (!last && !p->tail_inline && !strip)
            VP_CUDA(launch_fwd_tail<T>(a, p->tail_threads, p->tail_smem, p->tail_tw_stage != 0, s), "forward tail launch");
        if (ring != nullptr) {
            VP_CUDA(cudaEventRecord(ring->written[slot], s), "record history slot");
            VP_CUDA(cudaStreamWaitEvent(ring->copy, ring->written[slot], 0), "copy stream wait");
            VP_CUDA(cudaMemcpyAsync(ring->host + (size_t)n * nxnv * sizeof(T), a.f_hist_n, nxnv * sizeof(T),
                                    cudaMemcpyDeviceToHost, ring->copy),
                    "history copy");
            VP_CUDA(cudaEventRecord(ring->copied[slot], ring->copy), "record history copy");
        }
    }
    if (ring != nullptr)
        for (int q = 0; q < std::min(ring->slots, T_steps); ++q)
            VP_CUDA(cudaStreamWaitEvent(s, ring->copied[q], 0), "wait for history copies");
    return VP_OK;
}

// ---------------------------------------------------------------------------------------------
// backward orchestration
// ---------------------------------------------------------------------------------------------
template <typename T>
static int backward_impl(vp_plan* p, const T* H, int T_steps, const unsigned char* tape, int every,
                         const T* g_ff, const T* g_fh, const T* g_Eh, const T* g_ee, T* g_fiv,
                         T* g_H, unsigned char* ws, cudaStream_t s) {
    const int nx = p->nx, nv = p->nv;
    const size_t nxnv = (size_t)nx * nv;
    const WsLayout L = ws_layout(p, T_steps, every);
    const TapeLayout TL = tape_layout(p, T_steps, every);
    const int K = TL.K;
    T* wbuf[2] = {reinterpret_cast<T*>(ws + L.hbuf0), reinterpret_cast<T*>(ws + L.hbuf1)};
    T* seg = reinterpret_cast<T*>(ws + L.seg);
    unsigned* counter = reinterpret_cast<unsigned*>(ws + L.counter);
    T* part = reinterpret_cast<T*>(ws + L.part);
    T* grho = reinterpret_cast<T*>(ws + L.grho);
    const T* ckpt = reinterpret_cast<const T*>(tape + TL.ckpt);
    const T* E_all = reinterpret_cast<const T*>(tape + TL.E);
    const VShift<T>* vsh_all = reinterpret_cast<const VShift<T>*>(tape + TL.vsh);

    if (p->res_cn > 0 && !p->merged && K == 1) {
        ResBwdArgs<T> r{};
        r.nx = nx;
        r.nv = nv;
        r.n_steps = T_steps;
        r.Rc = nx / p->res_cn;
        r.H = H;
        r.mx = p->d_mx;
        r.tx = static_cast<const T*>(p->d_tx);
        r.feq = p->d_feq;
        r.feq_rs = p->feq2d ? nv : 0;
        r.h_tape = ckpt;
        r.E_tape = E_all;
        r.vsh_tape = vsh_all;
        r.g_ff = g_ff;
        r.g_fh = g_fh;
        r.g_Eh = g_Eh;
        r.g_ee = g_ee;
        r.g_fiv = g_fiv;
        r.g_H = g_H;
        r.P = poisson_tables<T>(p, nullptr, nullptr, true);
        r.dv = (T)p->dv;
        r.dx = (T)p->dx;
        r.neg_dt_dv = (T)(-p->dt / p->dv);
        res_halo_rows(p, &r.h_lo, &r.h_hi);
        r.mx_lo = (int)p->mx_lo;
        VP_CUDA(launch_res_bwd<T>(r, p->feq2d != 0, p->res_cn, p->res_threads, p->res_smem, s),
                "cluster-resident backward launch");
        return VP_OK;
    }

    VP_CUDA(cudaMemsetAsync(counter, 0, 256, s), "cudaMemsetAsync(counter)");
    VP_CUDA(cudaMemsetAsync(g_H, 0, (size_t)nx * sizeof(T), s), "cudaMemsetAsync(g_H)");
    const bool strip = sizeof(T) == 4 && strip_active(p);
    if (strip)
        VP_CUDA(cudaMemsetAsync(ws + L.sctr, 0, (size_t)(p->strip.n_bands + 1) * sizeof(unsigned), s),
                "cudaMemsetAsync(strip counters)");

    auto h_ptr = [&](int n) -> const T* {
        if (n % K == 0) return ckpt + (size_t)(n / K) * nxnv;
        return seg + (size_t)((n % K) - 1) * nxnv;
    };
    auto h_mut = [&](int n) -> T* { return seg + (size_t)((n % K) - 1) * nxnv; };

    FwdArgs<T> fa{};
    fa.nx = nx;
    fa.nv = nv;
    fa.n_chunks = p->cfg.n_chunks;
    fa.chunk_cols = p->cfg.chunk_cols;
    fa.mx = p->d_mx;
    fa.tx = static_cast<const T*>(p->d_tx);
    fa.tx64 = p->d_tx64;
    fa.feq = p->d_feq;
    fa.feq_rs = p->feq2d ? nv : 0;
    fa.counter = nullptr;
    fa.P = poisson_tables<T>(p, ws, &L, true);
    fa.dv = (T)p->dv;
    fa.dx = (T)p->dx;
    fa.dtdv = (T)(p->dt / p->dv);
    fa.H = H;
    fa.vtab = static_cast<const T*>(p->d_vtab);
    fa.stage_span = p->stage_span;
    fa.part = nullptr;  // propagation only

    int current_seg = -1;
    auto recompute = [&](int sgi) -> int {
        if (sgi == current_seg) return VP_OK;
        current_seg = sgi;
        const int n0 = sgi * K;
        const int n1 = std::min(n0 + K, T_steps);
        if constexpr (sizeof(T) == 4) {
            if (p->pst_on && !p->merged) {
                // the forward's persistent kernel replays the segment with the tape's shifts:
                // bitwise the states the forward computed
                if (n1 - 1 > n0) {
                    PersistArgs pa = persist_args(p, ws, L);
                    pa.mode = 1;
                    pa.first_step = n0;
                    pa.n_steps = n1 - 1;
                    pa.K = K;
                    pa.seg = reinterpret_cast<float*>(seg);
                    pa.ckpt = const_cast<float*>(reinterpret_cast<const float*>(ckpt));
                    pa.vsh_tape_in = reinterpret_cast<const VShift<float>*>(vsh_all);
                    VP_CUDA(launch_persist_fwd(pa, p->pst, s), "persistent recompute launch");
                }
                return VP_OK;
            }
        }
        for (int n = n0; n < n1 - 1; ++n) {
            fa.h_in = h_ptr(n);
            fa.h_out = h_mut(n + 1);
            fa.vsh = vsh_all + (size_t)n * nx;
            if (strip) {
                // the forward's strip kernel, without row sums: bitwise the states it computed
                if constexpr (sizeof(T) == 4) {
                    StripFwdArgs sa{};
                    strip_tables(p, sa, p->strip.gt);
                    sa.h_in = fa.h_in;
                    sa.h_out = fa.h_out;
                    sa.vsh = fa.vsh;
                    VP_CUDA(launch_strip_fwd(sa, p->strip, s), "strip recompute launch");
                }
            } else if (p->merged) {
                FwdArgs<T> am = fa;
                am.mx = p->d_mxf;
                am.tx = static_cast<const T*>(p->d_txf);
                am.tx64 = p->d_txf64;
                VP_CUDA(launch_fwd<T>(am, p->cfg, 3, p->feq2d != 0, s), "recompute launch");
            } else if (p->stage_span > 0) {
                VP_CUDA(launch_fwd_staged<T>(fa, p->scfg, s), "recompute launch");
            } else {
                VP_CUDA(launch_fwd<T>(fa, p->cfg, 1, p->feq2d != 0, s), "recompute launch");
            }
        }
        return VP_OK;
    };

    BwdArgs<T> b{};
    b.nx = nx;
    b.nv = nv;
    b.n_chunks = p->cfg.n_chunks;
    b.chunk_cols = p->cfg.chunk_cols;
    b.mx = p->d_mx;
    b.tx = static_cast<const T*>(p->d_tx);
    b.feq = p->d_feq;
    b.feq_rs = p->feq2d ? nv : 0;
    b.part = part;
    b.counter = p->tail_inline ? counter : nullptr;
    b.P = poisson_tables<T>(p, ws, &L, p->tail_inline || p->tail_smem > 0);
    b.dv = (T)p->dv;
    b.dx = (T)p->dx;
    b.neg_dt_dv = (T)(-p->dt / p->dv);
    b.gH = g_H;
    b.grho_out = grho;
    b.vtab = static_cast<const T*>(p->d_vtab);
    b.stage_span = p->stage_span;

    int rc;
    // prologue (n = T)
    if ((rc = recompute((T_steps - 1) / K)) != VP_OK) return rc;
    b.c_src = g_ff;
    b.c_src2 = g_fh ? g_fh + (size_t)(T_steps - 1) * nxnv : nullptr;
    b.w_out = wbuf[(T_steps - 1) & 1];
    b.h_prev = h_ptr(T_steps - 1);
    b.vsh_prev = vsh_all + (size_t)(T_steps - 1) * nx;
    b.E_prev = E_all + (size_t)(T_steps - 1) * nx;
    b.gE_hist = g_Eh ? g_Eh + (size_t)(T_steps - 1) * nx : nullptr;
    b.gee = g_ee ? g_ee + (T_steps - 1) : nullptr;
    if (g_ff == nullptr && g_fh == nullptr && !p->tail_inline) {
        // no cotangent on the final state or the history: w_{T-1} = X^T(0) = 0 and the slope row
        // sums are 0, so the prologue is two memsets and the tail
        VP_CUDA(cudaMemsetAsync(b.w_out, 0, nxnv * sizeof(T), s), "cudaMemsetAsync(w)");
        VP_CUDA(cudaMemsetAsync(part, 0, (size_t)b.n_chunks * nx * sizeof(T), s), "cudaMemsetAsync(part)");
    } else {
        VP_CUDA(launch_bwd<T>(b, p->cfg, 0, p->feq2d != 0, s), "backward prologue launch");
    }
    if (!p->tail_inline) VP_CUDA(launch_bwd_tail<T>(b, p->tail_threads, p->tail_smem, p->tail_tw_stage != 0, s), "backward tail launch");

    b.c_src = nullptr;
    b.c_src2 = nullptr;
    bool adj_persist = false;
    if constexpr (sizeof(T) == 4) adj_persist = p->pst_on && p->pst.bwd_ok && !p->merged;
    if (adj_persist) {
        // one persistent launch per checkpoint segment: adjoint steps n with h_{n-1} in the segment,
        // after the segment's states are replayed
        for (int sgi = (T_steps - 2) / K; sgi >= 0 && T_steps >= 2; --sgi) {
            const int n_lo = sgi * K + 1, n_hi = std::min(sgi * K + K, T_steps - 1);
            if (n_hi < n_lo) continue;
            if ((rc = recompute(sgi)) != VP_OK) return rc;
            PersistBwdArgs pb{};
            pb.nx = nx;
            pb.nv = nv;
            pb.n_chunks = nv / 256;
            pb.n_hi = n_hi;
            pb.n_lo = n_lo;
            pb.K = K;
            pb.wbuf0 = reinterpret_cast<float*>(wbuf[0]);
            pb.wbuf1 = reinterpret_cast<float*>(wbuf[1]);
            pb.ckpt = reinterpret_cast<const float*>(ckpt);
            pb.seg = reinterpret_cast<const float*>(seg);
            pb.quad = p->d_pquad;
            pb.tq = p->d_ptq;
            pb.chunk = p->d_pchunk;
            pb.dfeq = p->d_dfeq;
            pb.vtab = static_cast<const float*>(p->d_vtab);
            pb.feq = p->d_feq;
            pb.ctab = p->d_ctab2;
            pb.dv = (float)p->dv;
            pb.dx = (float)p->dx;
            pb.neg_dt_dv = (float)(-p->dt / p->dv);
            pb.vsh_tape = reinterpret_cast<const VShift<float>*>(vsh_all);
            pb.E_tape = reinterpret_cast<const float*>(E_all);
            pb.g_fh = reinterpret_cast<const float*>(g_fh);
            pb.g_Eh = reinterpret_cast<const float*>(g_Eh);
            pb.g_ee = reinterpret_cast<const float*>(g_ee);
            pb.g_H = reinterpret_cast<float*>(g_H);
            pb.grho = reinterpret_cast<float*>(grho);
            pb.gE = reinterpret_cast<float*>(ws + L.gscratch);
            pb.bar = reinterpret_cast<unsigned*>(ws + L.pbar);
            pb.status = p->d_status;
            pb.wait_ns = p->wait_ns;
            VP_CUDA(launch_persist_bwd(pb, p->pst, s), "persistent adjoint launch");
        }
    }
    for (int n = adj_persist ? 0 : T_steps - 1; n >= 1; --n) {
        if ((rc = recompute((n - 1) / K)) != VP_OK) return rc;
        b.w_in = wbuf[n & 1];
        b.grho = grho;
        b.vsh_n = vsh_all + (size_t)n * nx;
        b.gfh = g_fh ? g_fh + (size_t)(n - 1) * nxnv : nullptr;
        b.w_out = wbuf[(n - 1) & 1];
        b.h_prev = h_ptr(n - 1);
        b.vsh_prev = vsh_all + (size_t)(n - 1) * nx;
        b.E_prev = E_all + (size_t)(n - 1) * nx;
        b.gE_hist = g_Eh ? g_Eh + (size_t)(n - 1) * nx : nullptr;
        b.gee = g_ee ? g_ee + (n - 1) : nullptr;
        if (strip) {
            if constexpr (sizeof(T) == 4) {
                StripBwdArgs sb{};
                strip_tables(p, sb, p->strip.bgt);
                sb.w_in = b.w_in;
                sb.w_out = b.w_out;
                sb.grho = grho;
                sb.vsh_n = b.vsh_n;
                sb.vsh_prev = b.vsh_prev;
                sb.h_prev = b.h_prev;
                sb.gfh = b.gfh;
                sb.part = part;
                sb.run_ctr = reinterpret_cast<unsigned*>(ws + L.sctr);
                sb.dv = (float)p->dv;
                sb.dx = (float)p->dx;
                sb.neg_dt_dv = (float)(-p->dt / p->dv);
                sb.gE_hist = b.gE_hist;
                sb.gee = b.gee;
                sb.E_prev = b.E_prev;
                sb.gH = g_H;
                sb.gE_out = reinterpret_cast<float*>(ws + L.sgE);
                VP_CUDA(launch_strip_bwd(sb, p->strip, s), "strip adjoint step launch");
                StripFieldArgs f{};
                f.nx = nx;
                f.nv = nv;
                f.adjoint = 1;
                f.x = sb.gE_out;
                f.ctab = p->d_ctab2;
                f.grho_out = grho;
                VP_CUDA(launch_strip_field(f, p->strip, s), "strip adjoint field launch");
            }
        } else if (p->merged) {
            BwdArgs<T> bm = b;
            bm.mx = p->d_mxf;
            bm.tx = static_cast<const T*>(p->d_txf);
            VP_CUDA(launch_bwd<T>(bm, p->cfg, 3, p->feq2d != 0, s), "backward merged step launch");
        } else if (p->stage_span > 0 && p->sb_smem > 0) {
            LaunchCfg bc = p->scfg;
            bc.smem = p->sb_smem;
            b.n_chunks = bc.n_chunks;
            b.chunk_cols = bc.chunk_cols;
            VP_CUDA(launch_bwd_staged<T>(b, bc, s), "backward step launch");
        } else {
            VP_CUDA(launch_bwd<T>(b, p->cfg, 1, p->feq2d != 0, s), "backward step launch");
        }
        if (!p->tail_inline && !strip)
            VP_CUDA(launch_bwd_tail<T>(b, p->tail_threads, p->tail_smem, p->tail_tw_stage != 0, s), "backward tail launch");
    }
    // epilogue (n = 0)
    b.w_in = wbuf[0];
    b.grho = grho;
    b.vsh_n = vsh_all;
    b.gfh = nullptr;
    b.w_out = nullptr;
    b.gfiv_out = g_fiv;
    VP_CUDA(launch_bwd<T>(b, p->cfg, 2, p->feq2d != 0, s), "backward epilogue launch");
    return VP_OK;
}

static void free_plan(vp_plan* p) {
    if (!p) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    cudaFree(p->d_feq);
    cudaFree(p->d_vs);
    cudaFree(p->d_mx);
    cudaFree(p->d_tx);
    cudaFree(p->d_tx64);
    cudaFree(p->d_mxf);
    cudaFree(p->d_kl);
    cudaFree(p->d_status);
    for (cudaEvent_t e : p->ev_written) cudaEventDestroy(e);
    for (cudaEvent_t e : p->ev_copied) cudaEventDestroy(e);
    cudaFree(p->d_txf);
    cudaFree(p->d_txf64);
    cudaFree(p->d_vtab);
    cudaFree(p->d_tw);
    cudaFree(p->d_mult);
    cudaFree(p->d_circ);
    cudaFree(p->d_pquad);
    cudaFree(p->d_ptq);
    cudaFree(p->d_pchunk);
    cudaFree(p->d_dfeq);
    cudaFree(p->d_ctab2);
    cudaFree(p->d_echunk);
    cudaSetDevice(prev);
    delete p;
}

// Imaginary part of the multiplier of fft_inv_multiplier (poisson.py:34-45): m_k = -1/(i*2*pi*f_k)
// = i/(2*pi*f_k), f_k the FFT frequencies of nx points over the period (m_0 = 0).
static std::vector<double> poisson_mult_im(int nx, double period_x) {
    std::vector<double> mult_im(nx, 0.0);
    const double d = period_x / nx;
    const double val = 1.0 / (nx * d);
    const int npos = (nx - 1) / 2 + 1;
    for (int k = 1; k < nx; ++k) {
        const double kk = k < npos ? (double)k : (double)(k - nx);
        const double f = kk * val;
        mult_im[k] = 1.0 / ((2.0 * M_PI) * f);
    }
    return mult_im;
}

// c = real(ifft(m)) for the spectral multiplier's imaginary part: c[k] = -(1/nx) * sum_q mult_im[q]
// * sin(2*pi*((q*k) mod nx)/nx), q ascending, from a table of the nx sines (O(nx^2) multiply-adds).
static std::vector<double> circulant_of(int nx, const std::vector<double>& mult_im) {
    std::vector<double> sn(nx);
    for (int r = 0; r < nx; ++r) sn[r] = std::sin(2.0 * M_PI * (double)r / (double)nx);
    std::vector<double> c(nx, 0.0);
    for (int k = 0; k < nx; ++k) {
        double acc = 0.0;
        int idx = 0;
        for (int q = 0; q < nx; ++q) {
            acc += mult_im[q] * sn[idx];
            idx += k;
            idx -= idx >= nx ? nx : 0;
        }
        c[k] = -acc / nx;
    }
    return c;
}

template <typename T>
static int upload(void** dst, const std::vector<double>& src) {
    std::vector<T> tmp(src.size());
    for (size_t i = 0; i < src.size(); ++i) tmp[i] = (T)src[i];
    VP_CUDA(cudaMalloc(dst, std::max<size_t>(1, tmp.size()) * sizeof(T)), "cudaMalloc(plan table)");
    if (!tmp.empty())
        VP_CUDA(cudaMemcpy(*dst, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice),
                "cudaMemcpy(plan table)");
    return VP_OK;
}

static int upload_bytes(void** dst, const void* src, size_t bytes) {
    VP_CUDA(cudaMalloc(dst, std::max<size_t>(1, bytes)), "cudaMalloc(plan table)");
    if (bytes) VP_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(plan table)");
    return VP_OK;
}

// Tables of a plan for ensembles on the strip kernels (128-column groups): the quads, their x
// weights, the f_eq differences, the circulant table (built here when the plan's own paths did not
// need them) and the quad shift range per 128 columns. Returns false when the plan is not eligible:
// float32, x-invariant f_eq, nv a multiple of 128, nx a multiple of 32 and at most 16384, the x
// shifts of every 4 neighbouring columns within one cell.
static bool plan_ens_tables(vp_plan* p, int* rc) {
    *rc = VP_OK;
    if (p->d_echunk != nullptr) return true;
    const int nx = p->nx, nv = p->nv;
    if (p->dtype != VP_F32 || p->feq2d || p->d_vtab == nullptr || nv % 128 != 0 || nx % kStripFieldRows != 0 ||
        nx > 16384 || nx % kStripEnsRows != 0)
        return false;
    std::vector<long long> m_signed(nv);
    std::vector<double> tx(nv);
    for (int j = 0; j < nv; ++j) {
        const double sj = 0.5 * p->host_vs[j] * p->dt / p->dx;
        const double mf = std::floor(-sj);
        tx[j] = -sj - mf;
        m_signed[j] = std::fabs(mf) < 1e15 ? (long long)mf : 0;
    }
    std::vector<int2> quad, chunk;
    std::vector<float> tq;
    if (!build_quad_tables(nx, nv, m_signed, tx, quad, tq, chunk, 128)) return false;
    if (p->d_pquad == nullptr) {
        const double* fe = p->host_feq.data();
        std::vector<float> dfeq(nv);
        for (int j = 0; j < nv; ++j) dfeq[j] = (float)(fe[(j + 1) % nv] - fe[j]);
        const std::vector<double> circ = circulant_of(nx, poisson_mult_im(nx, p->period_x));
        std::vector<float> ctab2((size_t)3 * nx + 8);
        for (size_t j = 0; j < ctab2.size(); ++j)
            ctab2[j] = (float)circ[(size_t)((((long long)j - nx) % nx + nx) % nx)];
        if ((*rc = upload_bytes((void**)&p->d_pquad, quad.data(), quad.size() * sizeof(int2))) ||
            (*rc = upload_bytes((void**)&p->d_ptq, tq.data(), tq.size() * sizeof(float))) ||
            (*rc = upload_bytes((void**)&p->d_dfeq, dfeq.data(), dfeq.size() * sizeof(float))) ||
            (*rc = upload_bytes((void**)&p->d_ctab2, ctab2.data(), ctab2.size() * sizeof(float))))
            return false;
    }
    if ((*rc = upload_bytes((void**)&p->d_echunk, chunk.data(), chunk.size() * sizeof(int2)))) return false;
    return true;
}

}  // namespace vpb

// =============================================================================================
// extern "C" entry points
// =============================================================================================

extern "C" {

int vp_abi_version(void) { return VP_ABI_VERSION; }

int vp_get_last_error(char* buf, size_t buf_len) {
    if (buf == nullptr || buf_len == 0) return VP_ERR_ARG;
    std::snprintf(buf, buf_len, "%s", g_err);
    return VP_OK;
}

int64_t vp_launch_count(void) { return g_launches; }
void vp_reset_launch_count(void) { g_launches = 0; }

// Plan set-up from f_eq given either as nx*nv values (row_only == false) or as one row of nv
// values that every row of the grid equals (row_only == true: x-invariant, no nx*nv host array).
static int plan_create(const vp_mesh_desc* mesh, double dt, const double* f_eq_host, bool row_only, int dtype,
                       vp_plan** out_plan) {
    if (out_plan == nullptr) return set_err(VP_ERR_ARG, "out_plan must not be NULL");
    *out_plan = nullptr;
    if (mesh == nullptr || f_eq_host == nullptr || mesh->xs == nullptr || mesh->vs == nullptr)
        return set_err(VP_ERR_ARG, "mesh, mesh->xs, mesh->vs and f_eq must not be NULL");
    const int nx = mesh->nx, nv = mesh->nv;
    if (nx < 2 || nv < 2) return set_err(VP_ERR_ARG, "nx and nv must be >= 2 (got %d, %d)", nx, nv);
    if ((long long)nx * nv > (1LL << 31) - 1)
        return set_err(VP_ERR_ARG, "nx*nv = %lld exceeds 2^31-1 cells", (long long)nx * nv);
    if (!(mesh->dx > 0) || !(mesh->dv > 0) || !std::isfinite(mesh->dx) || !std::isfinite(mesh->dv))
        return set_err(VP_ERR_ARG, "dx and dv must be finite and positive");
    if (!(mesh->period_x > 0) || !(mesh->period_v > 0))
        return set_err(VP_ERR_ARG, "period_x and period_v must be positive");
    if (!std::isfinite(dt)) return set_err(VP_ERR_ARG, "dt must be finite");
    if (dtype != VP_F32 && dtype != VP_F64) return set_err(VP_ERR_ARG, "dtype must be VP_F32 or VP_F64");
    for (int j = 0; j < nv; ++j)
        if (!std::isfinite(mesh->vs[j])) return set_err(VP_ERR_ARG, "vs[%d] is not finite", j);
    for (int i = 0; i < nx; ++i)
        if (!std::isfinite(mesh->xs[i])) return set_err(VP_ERR_ARG, "xs[%d] is not finite", i);
    const size_t feq_given = row_only ? (size_t)nv : (size_t)nx * nv;
    for (size_t c = 0; c < feq_given; ++c)
        if (!std::isfinite(f_eq_host[c]))
            return set_err(VP_ERR_ARG, "f_eq[%zu, %zu] is not finite", row_only ? (size_t)0 : c / (size_t)nv,
                           c % (size_t)nv);

    vp_plan* p = new (std::nothrow) vp_plan();
    if (!p) return set_err(VP_ERR_ARG, "out of host memory");
    p->nx = nx;
    p->nv = nv;
    p->dtype = dtype;
    p->dx = mesh->dx;
    p->dv = mesh->dv;
    p->dt = dt;
    p->period_x = mesh->period_x;
    p->period_v = mesh->period_v;
    cudaError_t ce = cudaGetDevice(&p->device);
    if (ce != cudaSuccess) {
        delete p;
        return cuda_err(ce, "cudaGetDevice");
    }
    int n_sms = 148;
    cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, p->device);

    // f_eq: x-invariant when every row equals the first one exactly
    bool inv = true;
    for (int i = 1; i < nx && inv && !row_only; ++i)
        inv = std::memcmp(f_eq_host + (size_t)i * nv, f_eq_host, (size_t)nv * sizeof(double)) == 0;
    p->feq2d = inv ? 0 : 1;
    p->host_feq.assign(f_eq_host, f_eq_host + feq_given);
    p->host_vs.assign(mesh->vs, mesh->vs + nv);

    // x half-step table: s_j = 0.5*v_j*dt/dx, m_j = floor(-s_j) mod nx, t_j = -s_j - floor(-s_j)
    std::vector<int> mx(nv);
    std::vector<double> tx(nv);
    std::vector<long long> m_signed(nv);
    for (int j = 0; j < nv; ++j) {
        const double sj = 0.5 * mesh->vs[j] * dt / mesh->dx;
        const double mf = std::floor(-sj);
        tx[j] = -sj - mf;
        m_signed[j] = std::fabs(mf) < 1e15 ? (long long)mf : 0;
        if (j == 0 || (long long)mf < p->mx_lo) p->mx_lo = (long long)mf;
        if (j == 0 || (long long)mf > p->mx_hi) p->mx_hi = (long long)mf;
        long long mi = (long long)mf % nx;
        if (mi < 0) mi += nx;
        mx[j] = (int)mi;
    }
    p->host_mxs = m_signed;
    // full step of the merged-Strang scheme: s_j = v_j*dt/dx (semilag_x_full_kernel, kernels.py:535-556)
    std::vector<int> mxf(nv);
    std::vector<double> txf(nv);
    for (int j = 0; j < nv; ++j) {
        const double sj = mesh->vs[j] * dt / mesh->dx;
        const double mf = std::floor(-sj);
        txf[j] = -sj - mf;
        long long mi = (long long)mf % nx;
        if (mi < 0) mi += nx;
        mxf[j] = (int)mi;
    }

    // Poisson: multiplier of fft_inv_multiplier (poisson.py:34-45): m_k = -1/(i*2*pi*f_k) = i/(2*pi*f_k)
    p->pow2 = (nx & (nx - 1)) == 0;
    p->log2nx = 0;
    while ((1 << p->log2nx) < nx) ++p->log2nx;
    const std::vector<double> mult_im = poisson_mult_im(nx, mesh->period_x);
    std::vector<double> tw;  // interleaved (re, im)
    if (p->pow2) {
        tw.resize((size_t)std::max(1, nx / 2) * 2);
        for (int q = 0; q < nx / 2; ++q) {
            const double ang = 2.0 * M_PI * (double)q / (double)nx;
            tw[2 * q] = std::cos(ang);
            tw[2 * q + 1] = -std::sin(ang);
        }
    }
    // circulant kernel c = real(ifft(m)): c[k] = -(1/nx) * sum_q mult_im[q] * sin(2*pi*q*k/nx)
    // (needed by the non-power-of-two FFT fallback and by the cluster-resident path, nx <= 512)
    std::vector<double> circ(nx, 0.0);
    if (!p->pow2 || nx <= 512) circ = circulant_of(nx, mult_im);
    const size_t rs = dtype == VP_F64 ? 8 : 4;
    const size_t area = poisson_area_size(nx, rs);
    p->tail_inline = area <= kInlineTailBytes ? 1 : 0;
    p->tail_smem = (!p->tail_inline && area <= kTailSmemBytes) ? area : 0;
    if (p->tail_smem > 0 && p->pow2 && poisson_area_size_staged(nx, rs) <= kTailSmemBytes) {
        p->tail_smem = poisson_area_size_staged(nx, rs);
        p->tail_tw_stage = 1;
    }
    p->tail_threads = nx >= 2048 ? 1024 : std::max(32, ((nx / 2 + 31) / 32) * 32);
    p->cfg = choose_cfg(nx, nv, n_sms);
    p->cfg.smem = fused_smem(p, p->cfg.R);
    p->host_mx = mx;
    // cluster-resident path: the largest cluster (16, 8, 4, 2 CTAs) whose per-CTA share of the
    // state fits in shared memory and that the occupancy calculator accepts
    for (int cn : {16, 8, 4, 2}) {
        int vrows = 0;
        const size_t smem = res_config_ok(p, cn, &vrows);
        if (smem > 0) {
            p->res_cn = cn;
            p->res_threads = res_threads(nx / cn, nv);
            p->res_smem = smem;
            p->res_vrows = vrows;
            break;
        }
    }
    {
        cudaError_t e1 = dtype == VP_F64 ? set_tail_smem_limit<double>(kTailSmemBytes)
                                         : set_tail_smem_limit<float>(kTailSmemBytes);
        cudaError_t e2 = dtype == VP_F64 ? set_poisson_smem_limit<double>(kTailSmemBytes)
                                         : set_poisson_smem_limit<float>(kTailSmemBytes);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            delete p;
            return cuda_err(e1 != cudaSuccess ? e1 : e2, "cudaFuncSetAttribute(tail shared memory)");
        }
    }

    int rc = VP_OK;
    const size_t feq_count = inv ? (size_t)nv : (size_t)nx * nv;
    std::vector<double> vs(mesh->vs, mesh->vs + nv);
    if ((rc = upload_bytes((void**)&p->d_feq, f_eq_host, feq_count * sizeof(double))) ||
        (rc = upload_bytes((void**)&p->d_vs, vs.data(), nv * sizeof(double))) ||
        (rc = upload_bytes((void**)&p->d_mx, mx.data(), nv * sizeof(int))) ||
        (rc = upload_bytes((void**)&p->d_tx64, tx.data(), nv * sizeof(double))) ||
        (rc = upload_bytes((void**)&p->d_mxf, mxf.data(), nv * sizeof(int))) ||
        (rc = upload_bytes((void**)&p->d_txf64, txf.data(), nv * sizeof(double)))) {
        free_plan(p);
        return rc;
    }
    // staged-step correction tables, m in [-kStageHalo, kStageHalo):
    // A_m[j] = f_eq[j+m] - f_eq[j], B_m[j] = f_eq[j+m+1] - f_eq[j+m] (periodic, float64)
    std::vector<double> vtab;
    const bool stage_tables = inv && nv % 32 == 0;
    if (stage_tables) {
        const int NM = 2 * kStageHalo;
        vtab.assign((size_t)2 * NM * nv, 0.0);
        auto fq = [&](long long c) { return f_eq_host[((c % nv) + nv) % nv]; };
        for (int q = 0; q < NM; ++q) {
            const int m = q - kStageHalo;
            for (int j = 0; j < nv; ++j) {
                vtab[(size_t)q * nv + j] = fq(j + m) - fq(j);
                vtab[(size_t)(NM + q) * nv + j] = fq(j + m + 1) - fq(j + m);
            }
        }
    }
    if (dtype == VP_F64) {
        if (stage_tables) rc = upload<double>(&p->d_vtab, vtab);
        if (!rc) rc = upload<double>(&p->d_tx, tx);
        if (!rc) rc = upload<double>(&p->d_txf, txf);
        if (!rc) rc = upload<double>(&p->d_tw, tw);
        if (!rc) rc = upload<double>(&p->d_mult, mult_im);
        if (!rc) rc = upload<double>(&p->d_circ, circ);
    } else {
        if (stage_tables) rc = upload<float>(&p->d_vtab, vtab);
        if (!rc) rc = upload<float>(&p->d_tx, tx);
        if (!rc) rc = upload<float>(&p->d_txf, txf);
        if (!rc) rc = upload<float>(&p->d_tw, tw);
        if (!rc) rc = upload<float>(&p->d_mult, mult_im);
        if (!rc) rc = upload<float>(&p->d_circ, circ);
    }
    if (!rc) {
        ce = cudaMalloc((void**)&p->d_status, 256);
        if (ce == cudaSuccess) ce = cudaMemset(p->d_status, 0, 256);
        if (ce != cudaSuccess) rc = cuda_err(ce, "cudaMalloc(plan status)");
    }
    if (rc) {
        free_plan(p);
        return rc;
    }
    choose_staged(p, n_sms);
    // persistent and strip paths: float32, x-invariant f_eq, nv a multiple of 256, the x shifts of
    // every 4 neighbouring columns within one cell, nx <= 16384 (the circulant table costs O(nx^2)
    // on the host)
    std::vector<int2> quad, chunk, chunk128;
    std::vector<float> tq;
    if (dtype == VP_F32 && inv && p->d_vtab != nullptr && nx <= 16384 &&
        build_quad_tables(nx, nv, m_signed, tx, quad, tq, chunk)) {
        p->host_msigned = m_signed;
        p->host_tx = tx;
        if (!persist_prepare(p->pst, nx, nv, m_signed, tx, n_sms, 0)) p->pst = PersistHost{};
        // strip shapes measured on B200 (8192^2): forward 256-column CTAs of two warps, adjoint
        // 128-column CTAs of one warp
        std::vector<int2> q2;
        std::vector<float> t2;
        const bool c128 = build_quad_tables(nx, nv, m_signed, tx, q2, t2, chunk128, 128);
        if (!(c128 && strip_prepare(p->strip, nx, nv, chunk, chunk128, n_sms, 0, 64, 32)) &&
            !strip_prepare(p->strip, nx, nv, chunk, chunk, n_sms, 0, 64, 64))
            p->strip = StripHost{};
        if (p->strip.R > 0 && p->strip.bgt == 32 &&
            (rc = upload_bytes((void**)&p->d_echunk, chunk128.data(), chunk128.size() * sizeof(int2)))) {
            free_plan(p);
            return rc;
        }
    }
    if (p->pst.R > 0 || p->strip.R > 0) {
        std::vector<float> dfeq(nv);
        for (int j = 0; j < nv; ++j) dfeq[j] = (float)(f_eq_host[(j + 1) % nv] - f_eq_host[j]);
        if (circ.size() != (size_t)nx || (p->pow2 && nx > 512)) circ = circulant_of(nx, mult_im);
        std::vector<float> ctab2((size_t)3 * nx + 8);
        for (size_t j = 0; j < ctab2.size(); ++j)
            ctab2[j] = (float)circ[(size_t)((((long long)j - nx) % nx + nx) % nx)];
        if ((rc = upload_bytes((void**)&p->d_pquad, quad.data(), quad.size() * sizeof(int2))) ||
            (rc = upload_bytes((void**)&p->d_ptq, tq.data(), tq.size() * sizeof(float))) ||
            (rc = upload_bytes((void**)&p->d_pchunk, chunk.data(), chunk.size() * sizeof(int2))) ||
            (rc = upload_bytes((void**)&p->d_dfeq, dfeq.data(), dfeq.size() * sizeof(float))) ||
            (rc = upload_bytes((void**)&p->d_ctab2, ctab2.data(), ctab2.size() * sizeof(float)))) {
            free_plan(p);
            return rc;
        }
        // defaults, measured on B200: the persistent loop on grids that are not cluster-resident
        // and whose CTAs each solve the field on their own window rows (512x1024 forward + adjoint
        // 2.0e10 cell-steps/s against 1.1e10 per step); the strip step kernels where the field
        // would need slices and a second grid barrier per step (8192x8192)
        p->pst_on = (p->res_cn == 0 && p->pst.R > 0 && p->pst.field_dist == 0) ? 1 : 0;
        p->strip_on = (p->res_cn == 0 && !p->pst_on && p->strip.R > 0) ? 1 : 0;
    }
    {   // trapezoid integral of f_eq (kl_divergence's norm_eq without eps, utils.py:59-64)
        double tot = 0.0;
        for (int i = 0; i < nx; ++i) {
            const double wx = (i == 0 || i == nx - 1) ? 0.5 * mesh->dx : mesh->dx;
            const double* fr = f_eq_host + (row_only ? (size_t)0 : (size_t)i * nv);
            double row = 0.0;
            for (int j = 0; j < nv; ++j) {
                const double wv = (j == 0 || j == nv - 1) ? 0.5 * mesh->dv : mesh->dv;
                row += wv * fr[j];
            }
            tot += wx * row;
        }
        p->feq_integral = tot;
    }
    *out_plan = p;
    return VP_OK;
}

int vp_plan_create(const vp_mesh_desc* mesh, double dt, const double* f_eq_host, int dtype, vp_plan** out_plan) {
    return plan_create(mesh, dt, f_eq_host, false, dtype, out_plan);
}

int vp_plan_create_from_row(const vp_mesh_desc* mesh, double dt, const double* f_eq_row, int dtype,
                            vp_plan** out_plan) {
    return plan_create(mesh, dt, f_eq_row, true, dtype, out_plan);
}

int vp_plan_get_config(const vp_plan* plan, vp_launch_config* out) {
    if (!plan || !out) return set_err(VP_ERR_ARG, "plan and out must not be NULL");
    out->rows_per_cta = plan->cfg.R;
    out->threads = plan->cfg.threads;
    out->n_chunks = plan->cfg.n_chunks;
    out->chunk_cols = plan->cfg.chunk_cols;
    out->tail_inline = plan->tail_inline;
    out->tail_threads = plan->tail_threads;
    out->fused_smem_bytes = (int64_t)plan->cfg.smem;
    out->tail_smem_bytes = (int64_t)plan->tail_smem;
    out->cluster_size = plan->res_cn;
    out->cluster_threads = plan->res_threads;
    out->cluster_smem_bytes = (int64_t)plan->res_smem;
    out->stage_rows = plan->stage_span > 0 ? plan->scfg.R : 0;
    out->stage_threads = plan->stage_span > 0 ? plan->scfg.threads : 0;
    out->stage_span = plan->stage_span;
    out->stage_smem_bytes = plan->stage_span > 0 ? (int64_t)plan->scfg.smem : 0;
    out->persist_rows = plan->pst_on ? plan->pst.R : 0;
    out->persist_ctas = plan->pst_on ? plan->pst.G : 0;
    out->persist_smem_bytes = plan->pst_on ? (int64_t)plan->pst.smem : 0;
    const bool strip = plan->strip_on && !plan->pst_on && plan->strip.R > 0;
    out->strip_rows = strip ? plan->strip.R : 0;
    out->strip_ctas = strip ? plan->strip.fwd_ctas : 0;
    out->strip_smem_bytes = strip ? (int64_t)plan->strip.fwd_smem : 0;
    out->strip_cols = strip ? 4 * plan->strip.gt : 0;
    out->strip_adj_cols = strip ? 4 * plan->strip.bgt : 0;
    return VP_OK;
}

int vp_plan_set_config(vp_plan* plan, const vp_launch_config* cfg) {
    if (!plan || !cfg) return set_err(VP_ERR_ARG, "plan and cfg must not be NULL");
    const int R = cfg->rows_per_cta, th = cfg->threads, ch = cfg->n_chunks;
    if (!(R == 1 || R == 2 || R == 4 || R == 8 || R == 16))
        return set_err(VP_ERR_ARG, "rows_per_cta must be 1, 2, 4, 8 or 16 (got %d)", R);
    if (plan->nx % R != 0 || (R > 1 && R > plan->nx / 2))
        return set_err(VP_ERR_ARG, "rows_per_cta=%d must divide nx=%d and be <= nx/2", R, plan->nx);
    if (th < 32 || th > 256 || th % 32 != 0)
        return set_err(VP_ERR_ARG, "threads must be a multiple of 32 in [32, 256] (got %d)", th);
    if (ch < 1 || ch > plan->nv) return set_err(VP_ERR_ARG, "n_chunks must be in [1, nv] (got %d)", ch);
    const int cn = cfg->cluster_size;
    size_t res_smem = 0;
    int res_vrows = 0;
    if (cn != 0) {
        res_smem = res_config_ok(plan, cn, &res_vrows);
        if (res_smem == 0)
            return set_err(VP_ERR_ARG, "cluster_size=%d is not usable for a %dx%d grid (must be a power of two "
                                       "in [2,16] dividing nx into 1, 2, 4, 8, 16 or 32 rows per CTA whose "
                                       "state fits in shared memory)",
                           cn, plan->nx, plan->nv);
    }
    if (cfg->stage_rows != 0) {
        const LaunchCfg keep = plan->scfg;
        const int keep_span = plan->stage_span;
        if (!staged_config(plan, cfg->stage_rows, cfg->stage_threads)) {
            plan->scfg = keep;
            plan->stage_span = keep_span;
            return set_err(VP_ERR_ARG, "stage_rows=%d, stage_threads=%d is not usable for this plan (needs an "
                                       "x-invariant f_eq, stage_threads a multiple of 32 in [32, 256] dividing nv, "
                                       "stage_rows 4, 8, 16 or 32 dividing nx and <= nx/4, and a staging buffer "
                                       "that fits in shared memory)",
                           cfg->stage_rows, cfg->stage_threads);
        }
    } else {
        plan->stage_span = 0;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cfg->persist_rows != 0) {
        if (plan->d_pquad == nullptr)
            return set_err(VP_ERR_ARG, "persist_rows=%d: the persistent path needs a float32 plan with an "
                                       "x-invariant f_eq, nv a multiple of 256 and nx <= 16384", cfg->persist_rows);
        const PersistHost keep = plan->pst;
        if (!persist_prepare(plan->pst, plan->nx, plan->nv, plan->host_msigned, plan->host_tx, sms,
                             cfg->persist_rows)) {
            plan->pst = keep;
            return set_err(VP_ERR_ARG, "persist_rows=%d is not usable for a %dx%d grid (4, 8 or 16 dividing nx, "
                                       "with every CTA resident at once)",
                           cfg->persist_rows, plan->nx, plan->nv);
        }
    }
    if (cfg->strip_rows != 0) {
        if (plan->d_pquad == nullptr)
            return set_err(VP_ERR_ARG, "strip_rows=%d: the strip path needs a float32 plan with an "
                                       "x-invariant f_eq, nv a multiple of 256 and nx <= 16384", cfg->strip_rows);
        const int keep_f = plan->strip.gt > 0 ? 4 * plan->strip.gt : 256;
        const int cols = cfg->strip_cols != 0 ? cfg->strip_cols : (cfg->strip_rows == 16 ? 256 : keep_f);
        // a width left at 0 keeps the current one where the band height allows it (128-column CTAs
        // exist for bands of 4 and 8 rows), else 256
        const int keep_b = plan->strip.bgt > 0 ? 4 * plan->strip.bgt : 256;
        const int bcols = cfg->strip_adj_cols != 0 ? cfg->strip_adj_cols : (cfg->strip_rows == 16 ? 256 : keep_b);
        if ((cols != 128 && cols != 256) || (bcols != 128 && bcols != 256))
            return set_err(VP_ERR_ARG, "strip_cols and strip_adj_cols must be 0, 128 or 256 (got %d, %d)",
                           cfg->strip_cols, cfg->strip_adj_cols);
        std::vector<int2> quad, chunk, bchunk;
        std::vector<float> tq;
        StripHost sh;
        int rc = VP_OK;
        if ((cols == 128 || bcols == 128) && !plan_ens_tables(plan, &rc))
            return rc != VP_OK ? rc : set_err(VP_ERR_ARG, "128-column strip CTAs are not usable for this plan");
        if (!build_quad_tables(plan->nx, plan->nv, plan->host_msigned, plan->host_tx, quad, tq, chunk, cols) ||
            !build_quad_tables(plan->nx, plan->nv, plan->host_msigned, plan->host_tx, quad, tq, bchunk, bcols) ||
            !strip_prepare(sh, plan->nx, plan->nv, chunk, bchunk, sms, cfg->strip_rows, cols / 4, bcols / 4))
            return set_err(VP_ERR_ARG, "strip_rows=%d with strip_cols=%d, strip_adj_cols=%d is not usable for a %dx%d "
                                       "grid (4, 8 or 16 dividing nx, 16 only with 256 columns, nx a multiple of 32)",
                           cfg->strip_rows, cols, bcols, plan->nx, plan->nv);
        plan->strip = sh;
    }
    plan->pst_on = cfg->persist_rows != 0 ? 1 : 0;
    plan->strip_on = cfg->strip_rows != 0 ? 1 : 0;
    plan->res_cn = cn;
    plan->res_smem = res_smem;
    plan->res_vrows = res_vrows;
    plan->res_threads = cn ? res_threads(plan->nx / cn, plan->nv) : 0;
    LaunchCfg c{};
    c.R = R;
    c.threads = th;
    int cols = (plan->nv + ch - 1) / ch;
    cols = ((cols + 31) / 32) * 32;
    c.chunk_cols = cols;
    c.n_chunks = (plan->nv + cols - 1) / cols;
    plan->cfg = c;
    plan->cfg.smem = fused_smem(plan, R);
    return VP_OK;
}

int vp_plan_set_scheme(vp_plan* plan, int32_t scheme) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    if (scheme != VP_SCHEME_STRANG && scheme != VP_SCHEME_MERGED)
        return set_err(VP_ERR_ARG, "scheme must be VP_SCHEME_STRANG (0) or VP_SCHEME_MERGED (1), got %d", scheme);
    plan->merged = scheme == VP_SCHEME_MERGED ? 1 : 0;
    return VP_OK;
}

int vp_plan_get_scheme(const vp_plan* plan, int32_t* scheme) {
    if (!plan || !scheme) return set_err(VP_ERR_ARG, "plan and scheme must not be NULL");
    *scheme = plan->merged ? VP_SCHEME_MERGED : VP_SCHEME_STRANG;
    return VP_OK;
}

int vp_plan_set_wait_limit(vp_plan* plan, uint64_t ns) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    plan->wait_ns = ns;
    return VP_OK;
}

int vp_plan_status(vp_plan* plan, uint32_t* flags) {
    if (!plan || !flags) return set_err(VP_ERR_ARG, "plan and flags must not be NULL");
    VP_CUDA(cudaMemcpy(flags, plan->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost), "read plan status");
    return VP_OK;
}

int vp_plan_clear_status(vp_plan* plan) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    VP_CUDA(cudaMemset(plan->d_status, 0, sizeof(uint32_t)), "clear plan status");
    VP_CUDA(cudaDeviceSynchronize(), "clear plan status");
    return VP_OK;
}

int vp_plan_destroy(vp_plan* plan) {
    free_plan(plan);
    return VP_OK;
}

int vp_num_steps(const vp_plan* plan, double t_final, int32_t* out_steps) {
    if (!plan || !out_steps) return set_err(VP_ERR_ARG, "plan and out_steps must not be NULL");
    const double r = t_final / plan->dt;
    if (!std::isfinite(r) || r > 2147483647.0 || r < -2147483648.0)
        return set_err(VP_ERR_ARG, "t_final/dt = %g is out of range", r);
    *out_steps = (int32_t)r;  // C truncation == Python int() for finite values
    return VP_OK;
}

int vp_resolve_checkpoint_every(const vp_plan* plan, int32_t n_steps, int32_t every,
                                int32_t* out_every) {
    if (!plan || !out_every) return set_err(VP_ERR_ARG, "plan and out_every must not be NULL");
    if (n_steps < 0) return set_err(VP_ERR_ARG, "n_steps must be >= 0");
    *out_every = resolve_every(plan, n_steps, every);
    return VP_OK;
}

int vp_workspace_bytes(const vp_plan* plan, int32_t n_steps, int32_t every, size_t* out_bytes) {
    if (!plan || !out_bytes) return set_err(VP_ERR_ARG, "plan and out_bytes must not be NULL");
    if (n_steps < 0) return set_err(VP_ERR_ARG, "n_steps must be >= 0");
    *out_bytes = ws_layout(plan, n_steps, every).total;
    return VP_OK;
}

int vp_tape_bytes(const vp_plan* plan, int32_t n_steps, int32_t every, size_t* out_bytes) {
    if (!plan || !out_bytes) return set_err(VP_ERR_ARG, "plan and out_bytes must not be NULL");
    if (n_steps < 0) return set_err(VP_ERR_ARG, "n_steps must be >= 0");
    *out_bytes = tape_layout(plan, n_steps, every).total;
    return VP_OK;
}

static int check_ws(vp_plan* plan, int32_t n_steps, int32_t every, void* ws, size_t ws_bytes) {
    size_t need = ws_layout(plan, n_steps, every).total;
    if (ws_bytes < need)
        return set_err(VP_ERR_ARG, "workspace has %zu bytes, %zu needed", ws_bytes, need);
    if (((uintptr_t)ws & 255) != 0) return set_err(VP_ERR_ARG, "workspace must be 256-byte aligned");
    return check_dev_ptr(ws, "workspace", plan->device);
}

int vp_forward(vp_plan* plan, const double* f_iv, const void* H, int32_t n_steps, double* f_final,
               void* f_hist, void* E_hist, void* ee_hist, void* tape, int32_t every,
               void* workspace, size_t workspace_bytes, void* stream) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    if (n_steps < 0) return set_err(VP_ERR_ARG, "n_steps must be >= 0 (got %d)", n_steps);
    int rc;
    const int dev = plan->device;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CaptureScope capture_scope(stream_capturing(s));
    if ((rc = check_dev_ptr(f_iv, "f_iv", dev)) || (rc = check_opt_ptr(f_final, "f_final", dev)))
        return rc;
    const size_t nxnv = (size_t)plan->nx * plan->nv;
    if (n_steps == 0) {
        if (f_final)
            VP_CUDA(cudaMemcpyAsync(f_final, f_iv, nxnv * sizeof(double), cudaMemcpyDeviceToDevice, s),
                    "cudaMemcpyAsync(f_final)");
        return VP_OK;
    }
    if ((rc = check_dev_ptr(H, "H", dev)) || (rc = check_opt_ptr(f_hist, "f_hist", dev)) ||
        (rc = check_opt_ptr(E_hist, "E_hist", dev)) || (rc = check_opt_ptr(ee_hist, "ee_hist", dev)) ||
        (rc = check_opt_ptr(tape, "tape", dev)) ||
        (rc = check_ws(plan, n_steps, every, workspace, workspace_bytes)))
        return rc;
    if (tape && ((uintptr_t)tape & 255) != 0) return set_err(VP_ERR_ARG, "tape must be 256-byte aligned");
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != dev) return set_err(VP_ERR_ARG, "current device %d differs from the plan's device %d", cur, dev);
    unsigned char* ws = static_cast<unsigned char*>(workspace);
    unsigned char* tp = static_cast<unsigned char*>(tape);
    VP_CUDA(launch_check_finite(f_iv, nxnv, H, plan->nx, plan->dtype == VP_F64, plan->d_status, s),
            "finite-input check launch");
    if (plan->dtype == VP_F64)
        return forward_impl<double>(plan, f_iv, (const double*)H, n_steps, f_final, (double*)f_hist,
                                    (double*)E_hist, (double*)ee_hist, tp, every, ws, s);
    return forward_impl<float>(plan, f_iv, (const float*)H, n_steps, f_final, (float*)f_hist,
                               (float*)E_hist, (float*)ee_hist, tp, every, ws, s);
}

int vp_backward(vp_plan* plan, const void* H, int32_t n_steps, const void* tape, int32_t every,
                const void* g_f_final, const void* g_f_hist, const void* g_E_hist,
                const void* g_ee_hist, void* g_f_iv, void* g_H, void* workspace,
                size_t workspace_bytes, void* stream) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    if (n_steps < 0) return set_err(VP_ERR_ARG, "n_steps must be >= 0 (got %d)", n_steps);
    int rc;
    const int dev = plan->device;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CaptureScope capture_scope(stream_capturing(s));
    if ((rc = check_dev_ptr(g_f_iv, "g_f_iv", dev)) || (rc = check_dev_ptr(g_H, "g_H", dev)) ||
        (rc = check_opt_ptr(g_f_final, "g_f_final", dev)))
        return rc;
    const size_t rsz = real_size(plan);
    const size_t nxnv = (size_t)plan->nx * plan->nv;
    if (n_steps == 0) {
        if (g_f_final)
            VP_CUDA(cudaMemcpyAsync(g_f_iv, g_f_final, nxnv * rsz, cudaMemcpyDeviceToDevice, s), "copy g_f_iv");
        else
            VP_CUDA(cudaMemsetAsync(g_f_iv, 0, nxnv * rsz, s), "zero g_f_iv");
        VP_CUDA(cudaMemsetAsync(g_H, 0, (size_t)plan->nx * rsz, s), "zero g_H");
        return VP_OK;
    }
    if ((rc = check_dev_ptr(H, "H", dev)) || (rc = check_dev_ptr(tape, "tape", dev)) ||
        (rc = check_opt_ptr(g_f_hist, "g_f_hist", dev)) || (rc = check_opt_ptr(g_E_hist, "g_E_hist", dev)) ||
        (rc = check_opt_ptr(g_ee_hist, "g_ee_hist", dev)) ||
        (rc = check_ws(plan, n_steps, every, workspace, workspace_bytes)))
        return rc;
    if (((uintptr_t)tape & 255) != 0) return set_err(VP_ERR_ARG, "tape must be 256-byte aligned");
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != dev) return set_err(VP_ERR_ARG, "current device %d differs from the plan's device %d", cur, dev);
    unsigned char* ws = static_cast<unsigned char*>(workspace);
    const unsigned char* tp = static_cast<const unsigned char*>(tape);
    if (plan->dtype == VP_F64)
        return backward_impl<double>(plan, (const double*)H, n_steps, tp, every, (const double*)g_f_final,
                                     (const double*)g_f_hist, (const double*)g_E_hist,
                                     (const double*)g_ee_hist, (double*)g_f_iv, (double*)g_H, ws, s);
    return backward_impl<float>(plan, (const float*)H, n_steps, tp, every, (const float*)g_f_final,
                                (const float*)g_f_hist, (const float*)g_E_hist, (const float*)g_ee_hist,
                                (float*)g_f_iv, (float*)g_H, ws, s);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// vp_forward_noalloc: the forward loop with its scratch in a static device array, for callers
// that cannot allocate device memory at call time.
// ---------------------------------------------------------------------------------------------
namespace vpb {

static __device__ __align__(256) unsigned char g_noalloc_scratch[VP_NOALLOC_SCRATCH_BYTES];

static const int kMaxDevices = 64;
static std::mutex g_noalloc_mutex;
static void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device. In host code the array's name is
// only a host-side stand-in; the address comes from cudaGetSymbolAddress, called with that device
// current. Only a successful lookup is cached: a lookup that fails (for example during a stream
// capture, or with an earlier error pending) clears the error and is retried by the next call.
static int noalloc_scratch(int device, void** out) {
    if (device < 0 || device >= kMaxDevices) return set_err(VP_ERR_UNSUPPORTED, "device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_ptr[device] == nullptr) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr) {
            cudaGetLastError();
            return cuda_err(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress(noalloc scratch)");
        }
        g_noalloc_ptr[device] = ptr;
    }
    *out = g_noalloc_ptr[device];
    return VP_OK;
}

}  // namespace vpb

extern "C" {

int vp_forward_noalloc(vp_plan* plan, const double* f_iv, const void* H, int32_t n_steps,
                       double* f_final, void* f_hist, void* E_hist, void* ee_hist, void* stream) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    if (n_steps < 0) return set_err(VP_ERR_ARG, "n_steps must be >= 0 (got %d)", n_steps);
    int rc;
    const int dev = plan->device;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != dev) return set_err(VP_ERR_ARG, "current device %d differs from the plan's device %d", cur, dev);
    CaptureScope capture_scope(stream_capturing(s));
    if ((rc = check_dev_ptr(f_iv, "f_iv", dev)) || (rc = check_opt_ptr(f_final, "f_final", dev)))
        return rc;
    const size_t nxnv = (size_t)plan->nx * plan->nv;
    if (n_steps == 0) {
        if (f_final)
            VP_CUDA(cudaMemcpyAsync(f_final, f_iv, nxnv * sizeof(double), cudaMemcpyDeviceToDevice, s),
                    "cudaMemcpyAsync(f_final)");
        return VP_OK;
    }
    if ((rc = check_dev_ptr(H, "H", dev)) || (rc = check_opt_ptr(f_hist, "f_hist", dev)) ||
        (rc = check_opt_ptr(E_hist, "E_hist", dev)) || (rc = check_opt_ptr(ee_hist, "ee_hist", dev)))
        return rc;
    const size_t need = ws_layout(plan, n_steps, 1).total;
    if (need > VP_NOALLOC_SCRATCH_BYTES)
        return set_err(VP_ERR_ARG,
                       "vp_forward_noalloc: a %dx%d %s grid needs %zu bytes of scratch, more than the "
                       "%zu-byte static scratch; use vp_forward with a caller-provided workspace",
                       plan->nx, plan->nv, plan->dtype == VP_F64 ? "float64" : "float32", need,
                       (size_t)VP_NOALLOC_SCRATCH_BYTES);
    void* scratch = nullptr;
    if ((rc = noalloc_scratch(dev, &scratch)) != VP_OK) return rc;
    unsigned char* ws = static_cast<unsigned char*>(scratch);
    if (plan->dtype == VP_F64)
        return forward_impl<double>(plan, f_iv, (const double*)H, n_steps, f_final, (double*)f_hist,
                                    (double*)E_hist, (double*)ee_hist, nullptr, 1, ws, s);
    return forward_impl<float>(plan, f_iv, (const float*)H, n_steps, f_final, (float*)f_hist,
                               (float*)E_hist, (float*)ee_hist, nullptr, 1, ws, s);
}

int vp_compute_rho(vp_plan* plan, const double* f, void* rho, void* stream) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    int rc;
    if ((rc = check_dev_ptr(f, "f", plan->device)) || (rc = check_dev_ptr(rho, "rho", plan->device))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int rs = plan->feq2d ? plan->nv : 0;
    cudaError_t e = plan->dtype == VP_F64
                        ? launch_compute_rho<double>(plan->nx, plan->nv, f, plan->d_feq, rs, plan->dv, (double*)rho, s)
                        : launch_compute_rho<float>(plan->nx, plan->nv, f, plan->d_feq, rs, plan->dv, (float*)rho, s);
    return e == cudaSuccess ? VP_OK : cuda_err(e, "compute_rho launch");
}

int vp_poisson(vp_plan* plan, const void* in, void* out, int adjoint, void* stream) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    int rc;
    if ((rc = check_dev_ptr(in, "in", plan->device)) || (rc = check_dev_ptr(out, "out", plan->device))) return rc;
    if (poisson_area_size(plan->nx, real_size(plan)) > kTailSmemBytes)
        return set_err(VP_ERR_UNSUPPORTED, "standalone Poisson solve needs nx*%zu bytes of shared memory; "
                                           "nx=%d exceeds the %zu-byte limit", 3 * real_size(plan), plan->nx,
                       kTailSmemBytes);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (plan->dtype == VP_F64)
        e = launch_poisson<double>(poisson_tables<double>(plan, nullptr, nullptr, true), (const double*)in, (double*)out, adjoint, s);
    else
        e = launch_poisson<float>(poisson_tables<float>(plan, nullptr, nullptr, true), (const float*)in, (float*)out, adjoint, s);
    return e == cudaSuccess ? VP_OK : cuda_err(e, "poisson launch");
}

int vp_electric_energy(vp_plan* plan, const void* E, void* ee, void* stream) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    int rc;
    if ((rc = check_dev_ptr(E, "E", plan->device)) || (rc = check_dev_ptr(ee, "ee", plan->device))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = plan->dtype == VP_F64
                        ? launch_electric_energy<double>(plan->nx, plan->dx, (const double*)E, (double*)ee, s)
                        : launch_electric_energy<float>(plan->nx, plan->dx, (const float*)E, (float*)ee, s);
    return e == cudaSuccess ? VP_OK : cuda_err(e, "electric energy launch");
}

int vp_forward_stream_history(vp_plan* plan, const double* f_iv, const void* H, int32_t n_steps, double* f_final,
                              void* f_hist_host, void* ring, int32_t ring_slots, void* E_hist, void* ee_hist,
                              void* tape, int32_t checkpoint_every, void* workspace, size_t workspace_bytes,
                              void* stream, void* copy_stream) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    if (n_steps < 1) return set_err(VP_ERR_ARG, "n_steps must be >= 1 (got %d)", n_steps);
    if (ring_slots < 2 || ring_slots > 64) return set_err(VP_ERR_ARG, "ring_slots must be in [2, 64] (got %d)", ring_slots);
    if (copy_stream == nullptr || copy_stream == stream)
        return set_err(VP_ERR_ARG, "copy_stream must be a stream other than the compute stream");
    if (f_hist_host == nullptr) return set_err(VP_ERR_ARG, "f_hist_host must not be NULL");
    {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, f_hist_host) != cudaSuccess || at.type != cudaMemoryTypeHost) {
            cudaGetLastError();
            return set_err(VP_ERR_ARG, "f_hist_host must be pinned host memory (cudaHostAlloc or cudaHostRegister)");
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CaptureScope capture_scope(stream_capturing(s));
    int rc;
    const int dev = plan->device;
    if ((rc = check_dev_ptr(f_iv, "f_iv", dev)) || (rc = check_dev_ptr(H, "H", dev)) ||
        (rc = check_dev_ptr(ring, "ring", dev)) || (rc = check_opt_ptr(f_final, "f_final", dev)) ||
        (rc = check_opt_ptr(E_hist, "E_hist", dev)) || (rc = check_opt_ptr(ee_hist, "ee_hist", dev)) ||
        (rc = check_opt_ptr(tape, "tape", dev)))
        return rc;
    const int K = resolve_every(plan, n_steps, checkpoint_every);
    const size_t need = ws_layout(plan, n_steps, K).total;
    if (workspace_bytes < need) return set_err(VP_ERR_ARG, "workspace has %zu bytes, %zu needed", workspace_bytes, need);
    if ((rc = check_dev_ptr(workspace, "workspace", dev))) return rc;
    while ((int)plan->ev_written.size() < ring_slots) {
        cudaEvent_t a, b;
        VP_CUDA(cudaEventCreateWithFlags(&a, cudaEventDisableTiming), "cudaEventCreate");
        VP_CUDA(cudaEventCreateWithFlags(&b, cudaEventDisableTiming), "cudaEventCreate");
        plan->ev_written.push_back(a);
        plan->ev_copied.push_back(b);
    }
    HistRing hr{static_cast<unsigned char*>(f_hist_host), ring_slots, static_cast<cudaStream_t>(copy_stream),
                plan->ev_written.data(), plan->ev_copied.data()};
    unsigned char* w = static_cast<unsigned char*>(workspace);
    unsigned char* t = static_cast<unsigned char*>(tape);
    if (plan->dtype == VP_F64)
        return forward_impl<double>(plan, f_iv, (const double*)H, n_steps, f_final, (double*)ring,
                                    (double*)E_hist, (double*)ee_hist, t, K, w, s, &hr);
    return forward_impl<float>(plan, f_iv, (const float*)H, n_steps, f_final, (float*)ring, (float*)E_hist,
                               (float*)ee_hist, t, K, w, s, &hr);
}

int vp_kl_divergence(vp_plan* plan, const double* f, double eps, double* value, double* grad, void* stream) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    if (!std::isfinite(eps) || eps < 0.0) return set_err(VP_ERR_ARG, "eps must be finite and >= 0");
    int rc;
    if ((rc = check_dev_ptr(f, "f", plan->device)) || (rc = check_dev_ptr(value, "value", plan->device)) ||
        (rc = check_opt_ptr(grad, "grad", plan->device)))
        return rc;
    if (plan->d_kl == nullptr) {
        if (stream_capturing(static_cast<cudaStream_t>(stream)))
            return set_err(VP_ERR_ARG, "the first vp_kl_divergence call on a plan must not be captured "
                                       "(it allocates the plan's scratch)");
        VP_CUDA(cudaMalloc(&plan->d_kl, (2 * kKlBlocks + 2) * sizeof(double)), "cudaMalloc(kl scratch)");
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const cudaError_t e = launch_kl_divergence(plan->nx, plan->nv, f, plan->d_feq, plan->feq2d ? plan->nv : 0,
                                               plan->dx, plan->dv, eps, plan->feq_integral + eps, plan->d_kl,
                                               value, grad, s);
    return e == cudaSuccess ? VP_OK : cuda_err(e, "kl divergence launch");
}

int vp_semilag_x(vp_plan* plan, const void* in, void* out, double dt, int adjoint, void* stream) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    if (!std::isfinite(dt)) return set_err(VP_ERR_ARG, "dt must be finite");
    int rc;
    if ((rc = check_dev_ptr(in, "in", plan->device)) || (rc = check_dev_ptr(out, "out", plan->device))) return rc;
    if (in == out) return set_err(VP_ERR_ARG, "in and out must not alias");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = plan->dtype == VP_F64
                        ? launch_semilag_x<double>(plan->nx, plan->nv, plan->d_vs, plan->dx, dt, (const double*)in, (double*)out, adjoint, s)
                        : launch_semilag_x<float>(plan->nx, plan->nv, plan->d_vs, plan->dx, dt, (const float*)in, (float*)out, adjoint, s);
    return e == cudaSuccess ? VP_OK : cuda_err(e, "semilag_x launch");
}

int vp_semilag_v(vp_plan* plan, const void* in, const void* E_total, void* out, double dt,
                 int adjoint, const void* f_in, void* g_E, void* stream) {
    if (!plan) return set_err(VP_ERR_ARG, "plan must not be NULL");
    if (!std::isfinite(dt)) return set_err(VP_ERR_ARG, "dt must be finite");
    int rc;
    const int dev = plan->device;
    if ((rc = check_dev_ptr(in, "in", dev)) || (rc = check_dev_ptr(out, "out", dev)) ||
        (rc = check_dev_ptr(E_total, "E_total", dev)) || (rc = check_opt_ptr(f_in, "f_in", dev)) ||
        (rc = check_opt_ptr(g_E, "g_E", dev)))
        return rc;
    if (in == out) return set_err(VP_ERR_ARG, "in and out must not alias");
    if ((g_E == nullptr) != (f_in == nullptr)) return set_err(VP_ERR_ARG, "f_in and g_E must be given together");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = plan->dtype == VP_F64
                        ? launch_semilag_v<double>(plan->nx, plan->nv, plan->dv, dt, (const double*)in, (const double*)E_total,
                                                   (double*)out, adjoint, (const double*)f_in, (double*)g_E, s)
                        : launch_semilag_v<float>(plan->nx, plan->nv, plan->dv, dt, (const float*)in, (const float*)E_total,
                                                  (float*)out, adjoint, (const float*)f_in, (float*)g_E, s);
    return e == cudaSuccess ? VP_OK : cuda_err(e, "semilag_v launch");
}

}  // extern "C"

// =============================================================================================
// Ensembles
// =============================================================================================

struct vp_batch {
    int n = 0, dtype = VP_F32, device = 0, R = 1, threads = 128, feq2d = 0, chunk = 128, per_sm = 0;
    std::vector<vp_plan*> owned;          // distinct plans
    std::vector<vp_plan*> plan_of;        // plan of each instance (caller order)
    std::vector<long long> off_f;         // caller order
    std::vector<long long> off_x;
    long long total_f = 0, total_x = 0, total_part = 0;
    int n_tiles = 0, grid_fwd = 0, grid_bwd = 0;
    size_t smem = 0;
    void* d_inst = nullptr;
    void* d_tiles = nullptr;   // int4 per tile: instance, first row, column chunk (no search on the device)
    // strip step kernels (float32 ensembles whose instances all qualify): instance table, CTA maps,
    // launch shapes and the sizes of their workspace regions
    int strip_ok = 0, strip_on = 0;
    void* d_sinst = nullptr;   // StripInst per instance (caller order)
    void* d_smap = nullptr;    // int4 per strip CTA: instance, chunk, run
    void* d_sfmap = nullptr;   // int2 per field CTA: instance, 32-row block
    int s_ctas = 0, s_fctas = 0, s_small = 0;   // s_small: every nx <= kStripSmallField
    size_t s_fsmem = 0, s_bsmem = 0;
    long long s_part = 0, s_ctr = 0, s_eep = 0;
};

namespace vpb {

struct BatchWs {
    size_t h0, h1, part, counters, vsh, E, grho;
    size_t spart, sctr, srho, sgE, seep;   // strip kernels: row partials, counters, rho, g_E, energies
    size_t total;
};

static BatchWs batch_ws(const vp_batch* b) {
    const size_t rs = b->dtype == VP_F64 ? 8 : 4, vs = b->dtype == VP_F64 ? 16 : 8;
    BatchWs L{};
    size_t off = 0;
    L.h0 = off; off += align256((size_t)b->total_f * rs);
    L.h1 = off; off += align256((size_t)b->total_f * rs);
    L.part = off; off += align256((size_t)b->total_part * rs);
    L.counters = off; off += align256((size_t)b->n * sizeof(unsigned));
    L.vsh = off; off += align256((size_t)b->total_x * vs);
    L.E = off; off += align256((size_t)b->total_x * rs);
    L.grho = off; off += align256((size_t)b->total_x * rs);
    if (b->strip_ok) {
        L.spart = off; off += align256((size_t)b->s_part * sizeof(float));
        L.sctr = off; off += align256((size_t)(b->s_ctr + b->n) * sizeof(unsigned));
        L.srho = off; off += align256((size_t)b->total_x * sizeof(float));
        L.sgE = off; off += align256((size_t)b->total_x * sizeof(float));
        L.seep = off; off += align256((size_t)b->s_eep * sizeof(double));
    }
    L.total = off;
    return L;
}

struct BatchTape {
    size_t h, E, vsh, total;
};

static BatchTape batch_tape(const vp_batch* b, int T) {
    const size_t rs = b->dtype == VP_F64 ? 8 : 4, vs = b->dtype == VP_F64 ? 16 : 8;
    BatchTape L{};
    size_t off = 0;
    L.h = off; off += align256((size_t)T * b->total_f * rs);
    L.E = off; off += align256((size_t)T * b->total_x * rs);
    L.vsh = off; off += align256((size_t)T * b->total_x * vs);
    L.total = off;
    return L;
}

template <typename T>
static void batch_fill(const vp_batch* b, std::vector<BatchInst<T>>& out, const std::vector<int>& order,
                       const std::vector<int>& chunk_cols) {
    out.clear();
    int tile = 0;
    long long part = 0;
    for (int k : order) {
        const vp_plan* p = b->plan_of[k];
        BatchInst<T> I{};
        I.nx = p->nx;
        I.nv = p->nv;
        I.chunk_cols = chunk_cols[k];
        I.n_chunks = (p->nv + I.chunk_cols - 1) / I.chunk_cols;
        I.n_tiles = (p->nx / b->R) * I.n_chunks;
        I.tile_begin = tile;
        tile += I.n_tiles;
        I.off_f = b->off_f[k];
        I.off_x = (int)b->off_x[k];
        I.off_part = (int)part;
        part += (long long)I.n_chunks * p->nx;
        I.index = k;
        I.mx = p->d_mx;
        I.tx = static_cast<const T*>(p->d_tx);
        I.tx64 = p->d_tx64;
        I.feq = p->d_feq;
        I.feq_rs = p->feq2d ? p->nv : 0;
        I.vtab = static_cast<const T*>(p->d_vtab);
        I.P = poisson_tables<T>(p, nullptr, nullptr, true);
        I.dv = (T)p->dv;
        I.dx = (T)p->dx;
        I.dtdv = (T)(p->dt / p->dv);
        I.neg_dt_dv = (T)(-p->dt / p->dv);
        out.push_back(I);
    }
}

static void free_batch(vp_batch* b) {
    if (!b) return;
    for (vp_plan* p : b->owned) free_plan(p);
    if (b->d_inst) {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(b->device);
        cudaFree(b->d_inst);
        if (b->d_tiles) cudaFree(b->d_tiles);
        cudaFree(b->d_sinst);
        cudaFree(b->d_smap);
        cudaFree(b->d_sfmap);
        cudaSetDevice(prev);
    }
    delete b;
}

// Tile shape of an ensemble: R rows x up to `chunk` columns per tile (instances narrower than the
// chunk use their nv rounded up to 32), `threads` per CTA, and a persistent grid of `per_sm`
// CTAs per SM (0: as many as the occupancy calculator allows). Rebuilds the device instance
// table (longest instances first); a CUDA graph captured before this call is stale after it.
static int batch_layout(vp_batch* b, int R, int chunk, int threads, int per_sm) {
    if (!(R == 1 || R == 2 || R == 4 || R == 8)) return set_err(VP_ERR_ARG, "rows_per_tile must be 1, 2, 4 or 8");
    for (vp_plan* p : b->plan_of)
        if (p->nx % R != 0 || (R > 1 && R > p->nx / 2))
            return set_err(VP_ERR_ARG, "rows_per_tile=%d must divide every nx and be <= nx/2 (nx=%d)", R, p->nx);
    if (chunk < 32 || chunk > 256 || chunk % 32 != 0)
        return set_err(VP_ERR_ARG, "chunk_cols must be a multiple of 32 in [32, 256] (got %d)", chunk);
    if (threads < 32 || threads > 256 || threads % 32 != 0)
        return set_err(VP_ERR_ARG, "threads must be a multiple of 32 in [32, 256] (got %d)", threads);
    if (per_sm < 0) return set_err(VP_ERR_ARG, "ctas_per_sm must be >= 0");
    const int n = b->n;
    std::vector<int> chunk_cols(n);
    int max_nx = 0;
    long long part = 0;
    for (int i = 0; i < n; ++i) {
        vp_plan* p = b->plan_of[i];
        chunk_cols[i] = std::min(chunk, ((p->nv + 31) / 32) * 32);
        max_nx = std::max(max_nx, p->nx);
        part += (long long)((p->nv + chunk_cols[i] - 1) / chunk_cols[i]) * p->nx;
    }
    const size_t rs = b->dtype == VP_F64 ? 8 : 4;
    const size_t area = poisson_area_size(max_nx, rs);
    if (area > 40 * 1024)
        return set_err(VP_ERR_UNSUPPORTED, "ensembles support nx up to the in-kernel Poisson limit (got nx=%d)", max_nx);
    const size_t smem = (((size_t)32 * R * rs + 15) & ~(size_t)15) + area;
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return (long long)b->plan_of[a]->nx * b->plan_of[a]->nv > (long long)b->plan_of[c]->nx * b->plan_of[c]->nv;
    });
    const int old_R = b->R;
    b->R = R;   // batch_fill reads it
    size_t bytes = 0;
    int n_tiles = 0;
    std::vector<unsigned char> host;
    std::vector<int4> tiles;
    auto tile_map = [&](const auto& v) {
        for (size_t k = 0; k < v.size(); ++k)
            for (int lt = 0; lt < v[k].n_tiles; ++lt)
                tiles.push_back(make_int4((int)k, (lt / v[k].n_chunks) * R, lt % v[k].n_chunks, 0));
    };
    if (b->dtype == VP_F64) {
        std::vector<BatchInst<double>> v;
        batch_fill<double>(b, v, order, chunk_cols);
        n_tiles = v.back().tile_begin + v.back().n_tiles;
        bytes = v.size() * sizeof(BatchInst<double>);
        host.assign(reinterpret_cast<unsigned char*>(v.data()), reinterpret_cast<unsigned char*>(v.data()) + bytes);
        tile_map(v);
    } else {
        std::vector<BatchInst<float>> v;
        batch_fill<float>(b, v, order, chunk_cols);
        n_tiles = v.back().tile_begin + v.back().n_tiles;
        bytes = v.size() * sizeof(BatchInst<float>);
        host.assign(reinterpret_cast<unsigned char*>(v.data()), reinterpret_cast<unsigned char*>(v.data()) + bytes);
        tile_map(v);
    }
    void* d_inst = nullptr;
    int rc = upload_bytes(&d_inst, host.data(), bytes);
    if (rc != VP_OK) {
        b->R = old_R;
        return rc;
    }
    void* d_tiles = nullptr;
    rc = upload_bytes(&d_tiles, tiles.data(), tiles.size() * sizeof(int4));
    if (rc != VP_OK) {
        cudaFree(d_inst);
        b->R = old_R;
        return rc;
    }
    if (b->d_inst) cudaFree(b->d_inst);
    if (b->d_tiles) cudaFree(b->d_tiles);
    b->d_inst = d_inst;
    b->d_tiles = d_tiles;
    const bool f2 = b->feq2d != 0;
    int n_sms = 148;
    cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, b->device);
    int bf = b->dtype == VP_F64 ? batch_blocks_per_sm<double>(R, true, f2, threads, smem)
                                : batch_blocks_per_sm<float>(R, true, f2, threads, smem);
    int bb = b->dtype == VP_F64 ? batch_blocks_per_sm<double>(R, false, f2, threads, smem)
                                : batch_blocks_per_sm<float>(R, false, f2, threads, smem);
    bf = std::max(1, bf);
    bb = std::max(1, bb);
    if (per_sm > 0) {
        bf = std::min(bf, per_sm);
        bb = std::min(bb, per_sm);
    }
    b->chunk = chunk;
    b->threads = threads;
    b->per_sm = per_sm;
    b->smem = smem;
    b->total_part = part;
    b->n_tiles = n_tiles;
    b->grid_fwd = std::max(1, std::min(n_tiles, bf * n_sms));
    b->grid_bwd = std::max(1, std::min(n_tiles, bb * n_sms));
    return VP_OK;
}

// Instance table and CTA maps of an ensemble on the strip kernels (128-column groups, bands of
// kStripEnsRows rows, runs of about 8 bands). Sets b->strip_ok when every instance qualifies; the
// strip kernels are then used by default.
static int batch_strip_layout(vp_batch* b) {
    b->strip_ok = b->strip_on = 0;
    if (b->dtype != VP_F32) return VP_OK;
    for (vp_plan* p : b->owned) {
        int rc = VP_OK;
        if (!plan_ens_tables(p, &rc)) return rc;   // not eligible (rc VP_OK) or an upload error
    }
    constexpr int RR = kStripEnsRows;
    const int n = b->n;
    std::vector<StripInst> inst(n);
    long long part = 0, ctr = 0, eep = 0;
    int max_nr = 0;
    for (int k = 0; k < n; ++k) {
        vp_plan* p = b->plan_of[k];
        StripInst& I = inst[k];
        I.nx = p->nx;
        I.nv = p->nv;
        I.n_chunks = p->nv / 128;
        I.n_bands = p->nx / RR;
        std::vector<int2> chunk(I.n_chunks);
        VP_CUDA(cudaMemcpy(chunk.data(), p->d_echunk, chunk.size() * sizeof(int2), cudaMemcpyDeviceToHost),
                "cudaMemcpy(chunk table)");
        int dmax = 0;
        for (const int2& c : chunk) dmax = std::max(dmax, c.y - c.x);
        const int span_max = 2 * dmax + RR + 4;
        I.ring_rows = ((span_max + RR - 1) / RR + 1) * RR;
        max_nr = std::max(max_nr, I.ring_rows);
        I.runs = std::max(1, std::min(I.n_bands, (I.n_bands + 7) / 8));
        I.index = k;
        I.off_x = (int)b->off_x[k];
        I.off_f = b->off_f[k];
        I.off_part = (int)part;
        part += (long long)I.n_chunks * p->nx;
        I.off_ctr = (int)ctr;
        ctr += I.runs;
        I.field_ctas = p->nx / kStripFieldRows;
        I.off_eep = (int)eep;
        eep += I.field_ctas;
        I.quad = p->d_pquad;
        I.tq = p->d_ptq;
        I.chunk = p->d_echunk;
        I.dfeq = p->d_dfeq;
        I.vtab = static_cast<const float*>(p->d_vtab);
        I.feq = p->d_feq;
        I.ctab = p->d_ctab2;
        I.dv = (float)p->dv;
        I.dx = (float)p->dx;
        I.dtdv = (float)(p->dt / p->dv);
        I.neg_dt_dv = (float)(-p->dt / p->dv);
    }
    const size_t fsmem = strip_ens_fwd_bytes(max_nr), bsmem = strip_ens_bwd_bytes(max_nr);
    if (strip_ens_occupancy(true, fsmem) <= 0 || strip_ens_occupancy(false, bsmem) <= 0) return VP_OK;
    // CTA maps, largest instances first
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return (long long)inst[a].nx * inst[a].nv > (long long)inst[c].nx * inst[c].nv;
    });
    std::vector<int4> map;
    std::vector<int2> fmap;
    for (int k : order) {
        for (int c = 0; c < inst[k].n_chunks; ++c)
            for (int r = 0; r < inst[k].runs; ++r) map.push_back(make_int4(k, c, r, 0));
        for (int rb = 0; rb < inst[k].field_ctas; ++rb) fmap.push_back(make_int2(k, rb));
    }
    void *d_inst = nullptr, *d_map = nullptr, *d_fmap = nullptr;
    int rc = upload_bytes(&d_inst, inst.data(), inst.size() * sizeof(StripInst));
    if (!rc) rc = upload_bytes(&d_map, map.data(), map.size() * sizeof(int4));
    if (!rc) rc = upload_bytes(&d_fmap, fmap.data(), fmap.size() * sizeof(int2));
    if (rc) {
        cudaFree(d_inst);
        cudaFree(d_map);
        cudaFree(d_fmap);
        return rc;
    }
    cudaFree(b->d_sinst);
    cudaFree(b->d_smap);
    cudaFree(b->d_sfmap);
    b->d_sinst = d_inst;
    b->d_smap = d_map;
    b->d_sfmap = d_fmap;
    b->s_ctas = (int)map.size();
    b->s_small = 1;
    for (const StripInst& I : inst) b->s_small = b->s_small && I.nx <= kStripSmallField;
    b->s_fctas = (int)fmap.size();
    b->s_fsmem = fsmem;
    b->s_bsmem = bsmem;
    b->s_part = part;
    b->s_ctr = ctr;
    b->s_eep = eep;
    b->strip_ok = b->strip_on = 1;
    return VP_OK;
}

template <typename T>
static int batch_forward_impl(vp_batch* b, const double* f_iv, const T* H, int Ts, double* f_final,
                              T* E_hist, T* ee_hist, unsigned char* tape, unsigned char* ws, cudaStream_t s) {
    const BatchWs L = batch_ws(b);
    const BatchTape TL = batch_tape(b, Ts);
    T* hb[2] = {reinterpret_cast<T*>(ws + L.h0), reinterpret_cast<T*>(ws + L.h1)};
    VShift<T>* vsh_ws = reinterpret_cast<VShift<T>*>(ws + L.vsh);
    T* E_ws = reinterpret_cast<T*>(ws + L.E);
    T* th = tape ? reinterpret_cast<T*>(tape + TL.h) : nullptr;
    T* tE = tape ? reinterpret_cast<T*>(tape + TL.E) : nullptr;
    VShift<T>* tv = tape ? reinterpret_cast<VShift<T>*>(tape + TL.vsh) : nullptr;
    VP_CUDA(cudaMemsetAsync(ws + L.counters, 0, (size_t)b->n * sizeof(unsigned), s), "memset(counters)");
    BatchStep<T> st{};
    st.inst = static_cast<const BatchInst<T>*>(b->d_inst);
    st.tiles = static_cast<const int4*>(b->d_tiles);
    st.n_inst = b->n;
    st.n_tiles = b->n_tiles;
    st.n_steps = Ts;
    st.H = H;
    st.part = reinterpret_cast<T*>(ws + L.part);
    st.counters = reinterpret_cast<unsigned*>(ws + L.counters);
    st.E_hist = E_hist;
    st.ee_hist = ee_hist;
    auto set_out = [&](int n) {   // slots written for step n (h_n, shifts/E of step n)
        if (tape) {
            st.c_out = th; st.c_out_mul = Ts; st.c_out_step = n;
            st.vsh_out = tv; st.vsh_out_mul = Ts; st.vsh_out_step = n;
            st.E_out = tE; st.E_out_mul = Ts; st.E_out_step = n;
        } else {
            st.c_out = hb[n & 1]; st.c_out_mul = 1; st.c_out_step = 0;
            st.vsh_out = vsh_ws; st.vsh_out_mul = 1; st.vsh_out_step = 0;
            st.E_out = E_ws; st.E_out_mul = 1; st.E_out_step = 0;
        }
    };
    // prologue
    st.f_iv = f_iv;
    st.last = 0;
    st.hist_step = 0;
    set_out(0);
    VP_CUDA(launch_batch_fwd<T>(st, b->R, 0, b->feq2d != 0, b->grid_fwd, b->threads, b->smem, s), "batch prologue");
    st.f_iv = nullptr;
    if constexpr (sizeof(T) == 4) {
        if (b->strip_on) {
            // the steps on the strip kernels: a strip launch and a field launch per step
            VP_CUDA(cudaMemsetAsync(ws + L.sctr, 0, (size_t)(b->s_ctr + b->n) * sizeof(unsigned), s),
                    "memset(strip counters)");
            st.part = reinterpret_cast<T*>(ws + L.spart);
            st.counters = reinterpret_cast<unsigned*>(ws + L.sctr);
            st.rho = reinterpret_cast<T*>(ws + L.srho);
            st.eep = reinterpret_cast<double*>(ws + L.seep);
            st.fctr = reinterpret_cast<unsigned*>(ws + L.sctr) + b->s_ctr;
            const StripInst* si = static_cast<const StripInst*>(b->d_sinst);
            for (int n = 0; n < Ts; ++n) {
                const bool last = (n == Ts - 1);
                if (tape) {
                    st.c_in = th; st.c_in_mul = Ts; st.c_in_step = n;
                    st.vsh_in = tv; st.vsh_in_mul = Ts; st.vsh_in_step = n;
                } else {
                    st.c_in = hb[n & 1]; st.c_in_mul = 1; st.c_in_step = 0;
                    st.vsh_in = vsh_ws; st.vsh_in_mul = 1; st.vsh_in_step = 0;
                }
                if (last) st.c_out = nullptr;
                else set_out(n + 1);
                st.last = last ? 1 : 0;
                st.hist_step = n + 1;
                st.f_final = last ? f_final : nullptr;
                VP_CUDA(launch_strip_ens_fwd(si, static_cast<const int4*>(b->d_smap), b->s_ctas, b->s_fsmem, st, s),
                        "ensemble strip step");
                if (!last)
                    VP_CUDA(b->s_small ? launch_strip_ens_field_small(si, b->n, st, 0, s)
                                       : launch_strip_ens_field(si, static_cast<const int2*>(b->d_sfmap), b->s_fctas,
                                                                st, 0, s),
                            "ensemble field");
            }
            return VP_OK;
        }
    }
    for (int n = 0; n < Ts; ++n) {
        const bool last = (n == Ts - 1);
        if (tape) {
            st.c_in = th; st.c_in_mul = Ts; st.c_in_step = n;
            st.vsh_in = tv; st.vsh_in_mul = Ts; st.vsh_in_step = n;
        } else {
            st.c_in = hb[n & 1]; st.c_in_mul = 1; st.c_in_step = 0;
            st.vsh_in = vsh_ws; st.vsh_in_mul = 1; st.vsh_in_step = 0;
        }
        if (last) {
            st.c_out = nullptr;
        } else {
            set_out(n + 1);
        }
        st.last = last ? 1 : 0;
        st.hist_step = n + 1;
        st.f_final = last ? f_final : nullptr;
        VP_CUDA(launch_batch_fwd<T>(st, b->R, 1, b->feq2d != 0, b->grid_fwd, b->threads, b->smem, s), "batch step");
    }
    return VP_OK;
}

template <typename T>
static int batch_backward_impl(vp_batch* b, const T* H, int Ts, const unsigned char* tape, const T* g_ff,
                               const T* g_Eh, const T* g_ee, T* g_fiv, T* g_H, unsigned char* ws,
                               cudaStream_t s) {
    const BatchWs L = batch_ws(b);
    const BatchTape TL = batch_tape(b, Ts);
    T* wb[2] = {reinterpret_cast<T*>(ws + L.h0), reinterpret_cast<T*>(ws + L.h1)};
    const T* th = reinterpret_cast<const T*>(tape + TL.h);
    const T* tE = reinterpret_cast<const T*>(tape + TL.E);
    const VShift<T>* tv = reinterpret_cast<const VShift<T>*>(tape + TL.vsh);
    T* grho = reinterpret_cast<T*>(ws + L.grho);
    VP_CUDA(cudaMemsetAsync(ws + L.counters, 0, (size_t)b->n * sizeof(unsigned), s), "memset(counters)");
    VP_CUDA(cudaMemsetAsync(g_H, 0, (size_t)b->total_x * sizeof(T), s), "memset(g_H)");
    BatchStep<T> st{};
    st.inst = static_cast<const BatchInst<T>*>(b->d_inst);
    st.tiles = static_cast<const int4*>(b->d_tiles);
    st.n_inst = b->n;
    st.n_tiles = b->n_tiles;
    st.n_steps = Ts;
    st.H = H;
    st.part = reinterpret_cast<T*>(ws + L.part);
    st.counters = reinterpret_cast<unsigned*>(ws + L.counters);
    st.g_Eh = g_Eh;
    st.g_ee = g_ee;
    st.g_H = g_H;
    st.grho_out = grho;
    // prologue (n = T)
    st.g_ff = g_ff;
    st.c_out = wb[(Ts - 1) & 1]; st.c_out_mul = 1; st.c_out_step = 0;
    st.h_prev = th; st.h_prev_step = Ts - 1;
    st.vsh_prev = tv; st.vsh_prev_step = Ts - 1;
    st.E_prev = tE; st.E_prev_step = Ts - 1;
    st.g_step = Ts - 1;
    VP_CUDA(launch_batch_bwd<T>(st, b->R, 0, b->feq2d != 0, b->grid_bwd, b->threads, b->smem, s), "batch bwd prologue");
    st.g_ff = nullptr;
    st.grho = grho;
    bool strip = false;
    if constexpr (sizeof(T) == 4) strip = b->strip_on != 0;
    if (strip) {
        if constexpr (sizeof(T) == 4) {
            // adjoint steps n = T-1 .. 1 on the strip kernels (strip launch, Poisson^T field launch)
            VP_CUDA(cudaMemsetAsync(ws + L.sctr, 0, (size_t)(b->s_ctr + b->n) * sizeof(unsigned), s),
                    "memset(strip counters)");
            BatchStep<T> ss = st;
            ss.part = reinterpret_cast<T*>(ws + L.spart);
            ss.counters = reinterpret_cast<unsigned*>(ws + L.sctr);
            ss.gE = reinterpret_cast<T*>(ws + L.sgE);
            const StripInst* si = static_cast<const StripInst*>(b->d_sinst);
            for (int n = Ts - 1; n >= 1; --n) {
                ss.c_in = wb[n & 1]; ss.c_in_mul = 1; ss.c_in_step = 0;
                ss.c_out = wb[(n - 1) & 1];
                ss.vsh_in = tv; ss.vsh_in_mul = Ts; ss.vsh_in_step = n;
                ss.h_prev_step = n - 1;
                ss.vsh_prev_step = n - 1;
                ss.E_prev_step = n - 1;
                ss.g_step = n - 1;
                VP_CUDA(launch_strip_ens_bwd(si, static_cast<const int4*>(b->d_smap), b->s_ctas, b->s_bsmem, ss, s),
                        "ensemble strip adjoint step");
                VP_CUDA(b->s_small ? launch_strip_ens_field_small(si, b->n, ss, 1, s)
                                   : launch_strip_ens_field(si, static_cast<const int2*>(b->d_sfmap), b->s_fctas, ss,
                                                            1, s),
                        "ensemble adjoint field");
            }
        }
    }
    for (int n = strip ? 0 : Ts - 1; n >= 1; --n) {
        st.c_in = wb[n & 1]; st.c_in_mul = 1; st.c_in_step = 0;
        st.c_out = wb[(n - 1) & 1];
        st.vsh_in = tv; st.vsh_in_mul = Ts; st.vsh_in_step = n;
        st.h_prev_step = n - 1;
        st.vsh_prev_step = n - 1;
        st.E_prev_step = n - 1;
        st.g_step = n - 1;
        VP_CUDA(launch_batch_bwd<T>(st, b->R, 1, b->feq2d != 0, b->grid_bwd, b->threads, b->smem, s), "batch bwd step");
    }
    st.c_in = wb[0]; st.c_in_mul = 1; st.c_in_step = 0;
    st.c_out = nullptr;
    st.vsh_in = tv; st.vsh_in_mul = Ts; st.vsh_in_step = 0;
    st.g_fiv = g_fiv;
    VP_CUDA(launch_batch_bwd<T>(st, b->R, 2, b->feq2d != 0, b->grid_bwd, b->threads, b->smem, s), "batch bwd epilogue");
    return VP_OK;
}

}  // namespace vpb

extern "C" {

int vp_batch_create(int32_t n, const vp_mesh_desc* meshes, const double* dts,
                    const double* const* f_eq_host, int dtype, vp_batch** out) {
    if (!out) return set_err(VP_ERR_ARG, "out_batch must not be NULL");
    *out = nullptr;
    if (n < 1) return set_err(VP_ERR_ARG, "n_instances must be >= 1 (got %d)", n);
    if (!meshes || !dts || !f_eq_host) return set_err(VP_ERR_ARG, "meshes, dts and f_eq_host must not be NULL");
    vp_batch* b = new (std::nothrow) vp_batch();
    if (!b) return set_err(VP_ERR_ARG, "out of host memory");
    b->n = n;
    b->dtype = dtype;
    cudaGetDevice(&b->device);
    // one plan per distinct (mesh, dt, f_eq)
    for (int i = 0; i < n; ++i) {
        vp_plan* found = nullptr;
        const vp_mesh_desc& m = meshes[i];
        for (vp_plan* p : b->owned) {
            if (p->nx == m.nx && p->nv == m.nv && p->dx == m.dx && p->dv == m.dv && p->dt == dts[i] &&
                p->period_x == m.period_x && p->period_v == m.period_v && p->host_feq.size() == (size_t)m.nx * m.nv &&
                std::memcmp(p->host_feq.data(), f_eq_host[i], sizeof(double) * (size_t)m.nx * m.nv) == 0 &&
                std::memcmp(p->host_vs.data(), m.vs, sizeof(double) * (size_t)m.nv) == 0) {
                found = p;
                break;
            }
        }
        if (!found) {
            int rc = vp_plan_create(&m, dts[i], f_eq_host[i], dtype, &found);
            if (rc != VP_OK) {
                free_batch(b);
                return rc;
            }
            b->owned.push_back(found);
        }
        b->plan_of.push_back(found);
    }
    int R = 8;   // largest common rows-per-tile
    for (;;) {
        bool ok = true;
        for (vp_plan* p : b->plan_of) ok = ok && (p->nx % R == 0) && (R == 1 || R <= p->nx / 2);
        if (ok || R == 1) break;
        R /= 2;
    }
    bool feq2d = false;
    for (int i = 0; i < n; ++i) {
        vp_plan* p = b->plan_of[i];
        feq2d = feq2d || p->feq2d;
        b->off_f.push_back(b->total_f);
        b->off_x.push_back(b->total_x);
        b->total_f += (long long)p->nx * p->nv;
        b->total_x += p->nx;
    }
    if (b->total_x > 2147483647LL) {
        free_batch(b);
        return set_err(VP_ERR_ARG, "ensemble has more than 2^31 rows");
    }
    b->feq2d = feq2d ? 1 : 0;
    int rc = batch_layout(b, R, 128, 128, 0);
    if (rc == VP_OK) rc = batch_strip_layout(b);
    if (rc != VP_OK) {
        free_batch(b);
        return rc;
    }
    *out = b;
    return VP_OK;
}

int vp_batch_get_config(const vp_batch* b, vp_batch_config* out) {
    if (!b || !out) return set_err(VP_ERR_ARG, "batch and out must not be NULL");
    out->rows_per_tile = b->R;
    out->chunk_cols = b->chunk;
    out->threads = b->threads;
    out->ctas_per_sm = b->per_sm;
    out->n_tiles = b->n_tiles;
    out->grid_fwd = b->grid_fwd;
    out->grid_bwd = b->grid_bwd;
    out->strip = b->strip_on;
    out->strip_ctas = b->strip_on ? b->s_ctas : 0;
    return VP_OK;
}

int vp_batch_set_config(vp_batch* b, const vp_batch_config* cfg) {
    if (!b || !cfg) return set_err(VP_ERR_ARG, "batch and cfg must not be NULL");
    if (cfg->strip != 0 && !b->strip_ok)
        return set_err(VP_ERR_ARG, "strip=1: the strip kernels need a float32 ensemble whose instances all have an "
                                   "x-invariant f_eq, nv a multiple of 128 and nx a multiple of 32");
    const int rc = batch_layout(b, cfg->rows_per_tile, cfg->chunk_cols, cfg->threads, cfg->ctas_per_sm);
    if (rc == VP_OK) b->strip_on = cfg->strip != 0 ? 1 : 0;
    return rc;
}

int vp_batch_destroy(vp_batch* b) {
    free_batch(b);
    return VP_OK;
}

int vp_batch_offsets(const vp_batch* b, int64_t* total_cells, int64_t* total_rows, int64_t* cell_offsets,
                     int64_t* row_offsets) {
    if (!b) return set_err(VP_ERR_ARG, "batch must not be NULL");
    if (total_cells) *total_cells = b->total_f;
    if (total_rows) *total_rows = b->total_x;
    for (int i = 0; i < b->n; ++i) {
        if (cell_offsets) cell_offsets[i] = b->off_f[i];
        if (row_offsets) row_offsets[i] = b->off_x[i];
    }
    return VP_OK;
}

int vp_batch_workspace_bytes(const vp_batch* b, int32_t n_steps, size_t* out) {
    if (!b || !out) return set_err(VP_ERR_ARG, "batch and out_bytes must not be NULL");
    if (n_steps < 0) return set_err(VP_ERR_ARG, "n_steps must be >= 0");
    *out = batch_ws(b).total;
    return VP_OK;
}

int vp_batch_tape_bytes(const vp_batch* b, int32_t n_steps, size_t* out) {
    if (!b || !out) return set_err(VP_ERR_ARG, "batch and out_bytes must not be NULL");
    if (n_steps < 0) return set_err(VP_ERR_ARG, "n_steps must be >= 0");
    *out = batch_tape(b, n_steps).total;
    return VP_OK;
}

static int batch_check_ws(vp_batch* b, void* ws, size_t ws_bytes) {
    const size_t need = batch_ws(b).total;
    if (ws_bytes < need) return set_err(VP_ERR_ARG, "workspace has %zu bytes, %zu needed", ws_bytes, need);
    if (((uintptr_t)ws & 255) != 0) return set_err(VP_ERR_ARG, "workspace must be 256-byte aligned");
    return check_dev_ptr(ws, "workspace", b->device);
}

int vp_batch_forward(vp_batch* b, const double* f_iv, const void* H, int32_t n_steps, double* f_final,
                     void* E_hist, void* ee_hist, void* tape, void* ws, size_t ws_bytes, void* stream) {
    if (!b) return set_err(VP_ERR_ARG, "batch must not be NULL");
    if (n_steps < 1) return set_err(VP_ERR_ARG, "ensembles need n_steps >= 1 (got %d)", n_steps);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CaptureScope capture_scope(stream_capturing(s));
    int rc;
    const int dev = b->device;
    if ((rc = check_dev_ptr(f_iv, "f_iv", dev)) || (rc = check_dev_ptr(H, "H", dev)) ||
        (rc = check_opt_ptr(f_final, "f_final", dev)) || (rc = check_opt_ptr(E_hist, "E_hist", dev)) ||
        (rc = check_opt_ptr(ee_hist, "ee_hist", dev)) || (rc = check_opt_ptr(tape, "tape", dev)) ||
        (rc = batch_check_ws(b, ws, ws_bytes)))
        return rc;
    if (tape && ((uintptr_t)tape & 255) != 0) return set_err(VP_ERR_ARG, "tape must be 256-byte aligned");
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != dev) return set_err(VP_ERR_ARG, "current device %d differs from the batch's device %d", cur, dev);
    unsigned char* w = static_cast<unsigned char*>(ws);
    unsigned char* t = static_cast<unsigned char*>(tape);
    if (b->dtype == VP_F64)
        return batch_forward_impl<double>(b, f_iv, (const double*)H, n_steps, f_final, (double*)E_hist,
                                          (double*)ee_hist, t, w, s);
    return batch_forward_impl<float>(b, f_iv, (const float*)H, n_steps, f_final, (float*)E_hist,
                                     (float*)ee_hist, t, w, s);
}

int vp_batch_backward(vp_batch* b, const void* H, int32_t n_steps, const void* tape, const void* g_f_final,
                      const void* g_E_hist, const void* g_ee_hist, void* g_f_iv, void* g_H, void* ws,
                      size_t ws_bytes, void* stream) {
    if (!b) return set_err(VP_ERR_ARG, "batch must not be NULL");
    if (n_steps < 1) return set_err(VP_ERR_ARG, "ensembles need n_steps >= 1 (got %d)", n_steps);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CaptureScope capture_scope(stream_capturing(s));
    int rc;
    const int dev = b->device;
    if ((rc = check_dev_ptr(H, "H", dev)) || (rc = check_dev_ptr(tape, "tape", dev)) ||
        (rc = check_opt_ptr(g_f_final, "g_f_final", dev)) || (rc = check_opt_ptr(g_E_hist, "g_E_hist", dev)) ||
        (rc = check_opt_ptr(g_ee_hist, "g_ee_hist", dev)) || (rc = check_dev_ptr(g_f_iv, "g_f_iv", dev)) ||
        (rc = check_dev_ptr(g_H, "g_H", dev)) || (rc = batch_check_ws(b, ws, ws_bytes)))
        return rc;
    if (((uintptr_t)tape & 255) != 0) return set_err(VP_ERR_ARG, "tape must be 256-byte aligned");
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != dev) return set_err(VP_ERR_ARG, "current device %d differs from the batch's device %d", cur, dev);
    unsigned char* w = static_cast<unsigned char*>(ws);
    const unsigned char* t = static_cast<const unsigned char*>(tape);
    if (b->dtype == VP_F64)
        return batch_backward_impl<double>(b, (const double*)H, n_steps, t, (const double*)g_f_final,
                                           (const double*)g_E_hist, (const double*)g_ee_hist, (double*)g_f_iv,
                                           (double*)g_H, w, s);
    return batch_backward_impl<float>(b, (const float*)H, n_steps, t, (const float*)g_f_final,
                                      (const float*)g_E_hist, (const float*)g_ee_hist, (float*)g_f_iv,
                                      (float*)g_H, w, s);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// x-slab decomposition: one grid split into slabs of rows, one per device. A slab's state arrays
// hold its own rows plus `ghost` copied rows of each neighbour (and pad rows up to a multiple of
// the per-column kernels' rows per CTA). The step kernels are the per-column ones, launched over
// the slab's array as if it were a periodic grid of ext_rows rows with the x offsets reduced mod
// ext_rows: the owned rows read only owned and ghost rows, so they see exactly what the one-grid
// step sees; the ghost and pad rows' results are discarded. The caller exchanges ghost rows and
// gathers the rows' sums between the calls; the field (Poisson, E, ee, v shifts) is solved on the
// whole x grid by every rank on the same gathered sums.
// ---------------------------------------------------------------------------------------------
struct vp_slab {
    vp_plan* plan = nullptr;
    int row0 = 0, n_rows = 0, ghost = 0, ext_rows = 0, row_first = 0;
    LaunchCfg cfg{};            // launch shape of the slab's per-column launches (rows per CTA fixed)
    int tail_threads = 0;
    size_t tail_smem = 0;
    int tail_tw_stage = 0;
    int* d_mx = nullptr;        // x half-step offsets reduced mod ext_rows      [nv]
    void* d_part = nullptr;     // column-chunk partial sums                    [n_chunks][ext_rows]
    void* d_vsh = nullptr;      // v shifts of step n in slab row order          [ext_rows]
    void* d_vsh2 = nullptr;     // v shifts of step n-1 (adjoint)                [ext_rows]
    void* d_grho = nullptr;     // cotangent on rho of step n                    [ext_rows]
    void* d_gscratch = nullptr; // Poisson work area when the tail's is not in shared memory
    void* d_cells = nullptr;    // f_{n+1} or g_f_iv over the slab's rows (allocated on first use)
    double* d_cells64 = nullptr;// f_final over the slab's rows (allocated on first use)
};

namespace vpb {

static size_t slab_field_vsh_bytes(const vp_plan* p) { return align256((size_t)p->nx * vshift_size(p)); }
static size_t slab_field_bytes(const vp_plan* p) {
    return slab_field_vsh_bytes(p) + align256((size_t)p->nx * real_size(p));
}

static void free_slab(vp_slab* sl) {
    if (!sl) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(sl->plan->device);
    for (void* q : {(void*)sl->d_mx, sl->d_part, sl->d_vsh, sl->d_vsh2, sl->d_grho, sl->d_gscratch, sl->d_cells,
                    (void*)sl->d_cells64})
        if (q) cudaFree(q);
    cudaSetDevice(prev);
    delete sl;
}

static int slab_check(vp_slab* sl, cudaStream_t s) {
    if (!sl) return set_err(VP_ERR_ARG, "slab must not be NULL");
    if (sl->plan->merged)
        return set_err(VP_ERR_UNSUPPORTED, "x slabs run the Strang scheme only (the plan is set to the merged scheme)");
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != sl->plan->device)
        return set_err(VP_ERR_ARG, "current device %d differs from the slab's device %d", cur, sl->plan->device);
    (void)s;
    return VP_OK;
}

template <typename T>
static VShift<T>* field_vsh(const vp_plan* p, const void* field) {
    return reinterpret_cast<VShift<T>*>(const_cast<void*>(field));
}
template <typename T>
static T* field_E(const vp_plan* p, const void* field) {
    return reinterpret_cast<T*>(static_cast<unsigned char*>(const_cast<void*>(field)) + slab_field_vsh_bytes(p));
}

template <typename T>
static PoissonTables<T> slab_poisson(const vp_slab* sl) {
    PoissonTables<T> P = poisson_tables<T>(sl->plan, nullptr, nullptr, sl->tail_smem > 0);
    P.gscratch = static_cast<T*>(sl->d_gscratch);
    return P;
}

// FwdArgs of a per-column launch over the slab's rows.
template <typename T>
static FwdArgs<T> slab_fwd_args(const vp_slab* sl) {
    const vp_plan* p = sl->plan;
    FwdArgs<T> a{};
    a.nx = sl->ext_rows;
    a.nv = p->nv;
    a.n_chunks = sl->cfg.n_chunks;
    a.chunk_cols = sl->cfg.chunk_cols;
    a.mx = sl->d_mx;
    a.tx = static_cast<const T*>(p->d_tx);
    a.tx64 = p->d_tx64;
    a.feq = p->d_feq;
    a.feq_rs = 0;
    a.counter = nullptr;   // no tail inside the launch: the field is solved on the gathered sums
    a.dv = (T)p->dv;
    a.dx = (T)p->dx;
    a.dtdv = (T)(p->dt / p->dv);
    return a;
}

template <typename T>
static int slab_lazy_cells(vp_slab* sl, bool f64) {
    const size_t n = (size_t)sl->ext_rows * sl->plan->nv;
    if (f64 && sl->d_cells64 == nullptr)
        VP_CUDA(cudaMalloc((void**)&sl->d_cells64, n * sizeof(double)), "cudaMalloc(slab f_final rows)");
    if (!f64 && sl->d_cells == nullptr) VP_CUDA(cudaMalloc(&sl->d_cells, n * sizeof(T)), "cudaMalloc(slab cells)");
    return VP_OK;
}

// Owned rows of a slab-ordered cell array into a caller's (n_rows, nv) array.
static int slab_copy_owned(const vp_slab* sl, const void* ext, void* out, size_t elem, cudaStream_t s) {
    const size_t row = (size_t)sl->plan->nv * elem;
    VP_CUDA(cudaMemcpyAsync(out, static_cast<const unsigned char*>(ext) + (size_t)sl->ghost * row,
                            (size_t)sl->n_rows * row, cudaMemcpyDeviceToDevice, s),
            "slab owned-row copy");
    return VP_OK;
}

template <typename T>
static int slab_forward_impl(vp_slab* sl, int phase, const void* in_ext, const void* field, void* out_ext,
                             void* row_sums, void* f_rows, double* f_final_rows, cudaStream_t s) {
    const vp_plan* p = sl->plan;
    FwdArgs<T> a = slab_fwd_args<T>(sl);
    int rc;
    if (phase == 0) {
        a.f_iv = static_cast<const double*>(in_ext);
        a.h_out = static_cast<T*>(out_ext);
    } else {
        VP_CUDA(launch_slab_gather_rows<T>(p->nx, sl->row_first, sl->ext_rows, field_vsh<T>(p, field),
                                           static_cast<VShift<T>*>(sl->d_vsh), nullptr, nullptr, nullptr, nullptr, s),
                "slab row gather launch");
        a.h_in = static_cast<const T*>(in_ext);
        a.h_out = static_cast<T*>(out_ext);
        a.vsh = static_cast<const VShift<T>*>(sl->d_vsh);
        if (f_rows != nullptr) {
            if ((rc = slab_lazy_cells<T>(sl, false)) != VP_OK) return rc;
            a.f_hist_n = static_cast<T*>(sl->d_cells);
        }
        if (f_final_rows != nullptr) {
            if ((rc = slab_lazy_cells<T>(sl, true)) != VP_OK) return rc;
            a.f_final = sl->d_cells64;
        }
    }
    a.part = row_sums != nullptr ? static_cast<T*>(sl->d_part) : nullptr;
    VP_CUDA(launch_fwd<T>(a, sl->cfg, phase, false, s), phase == 0 ? "slab forward start launch" : "slab forward step launch");
    if (row_sums != nullptr && (phase == 0 || out_ext != nullptr))
        VP_CUDA(launch_slab_row_sums<T>(static_cast<const T*>(sl->d_part), sl->cfg.n_chunks, sl->ext_rows, sl->ghost,
                                        sl->n_rows, static_cast<T*>(row_sums), s),
                "slab row sums launch");
    if (f_rows != nullptr && (rc = slab_copy_owned(sl, sl->d_cells, f_rows, sizeof(T), s)) != VP_OK) return rc;
    if (f_final_rows != nullptr && (rc = slab_copy_owned(sl, sl->d_cells64, f_final_rows, sizeof(double), s)) != VP_OK)
        return rc;
    return VP_OK;
}

template <typename T>
static int slab_field_impl(vp_slab* sl, const T* sums, const T* H, void* field, T* E_hist_row, T* ee,
                           cudaStream_t s) {
    const vp_plan* p = sl->plan;
    FwdArgs<T> a{};
    a.nx = p->nx;
    a.nv = p->nv;
    a.n_chunks = 1;
    a.part = const_cast<T*>(sums);
    a.P = slab_poisson<T>(sl);
    a.dv = (T)p->dv;
    a.dx = (T)p->dx;
    a.dtdv = (T)(p->dt / p->dv);
    a.H = H;
    a.E_out = field_E<T>(p, field);
    a.E_hist_out = E_hist_row;
    a.ee_out = ee;
    a.vsh_out = field_vsh<T>(p, field);
    VP_CUDA(launch_fwd_tail<T>(a, sl->tail_threads, sl->tail_smem, sl->tail_tw_stage != 0, s), "slab field launch");
    return VP_OK;
}

template <typename T>
static BwdArgs<T> slab_bwd_args(const vp_slab* sl) {
    const vp_plan* p = sl->plan;
    BwdArgs<T> b{};
    b.nx = sl->ext_rows;
    b.nv = p->nv;
    b.n_chunks = sl->cfg.n_chunks;
    b.chunk_cols = sl->cfg.chunk_cols;
    b.mx = sl->d_mx;
    b.tx = static_cast<const T*>(p->d_tx);
    b.feq = p->d_feq;
    b.feq_rs = 0;
    b.part = static_cast<T*>(sl->d_part);
    b.counter = nullptr;
    b.dv = (T)p->dv;
    b.dx = (T)p->dx;
    b.neg_dt_dv = (T)(-p->dt / p->dv);
    b.vtab = static_cast<const T*>(p->d_vtab);
    return b;
}

// phase 0: prologue (n = T), 1: step n, 2: epilogue (n = 0); see vp_bwd_kernel.
template <typename T>
static int slab_backward_impl(vp_slab* sl, int phase, const void* w_ext, const void* g_ext, const T* grho,
                              const void* field_n, const void* field_prev, const void* h_prev_ext, void* w_out_ext,
                              void* slope_sums, void* g_f_iv_rows, cudaStream_t s) {
    const vp_plan* p = sl->plan;
    BwdArgs<T> b = slab_bwd_args<T>(sl);
    int rc;
    VP_CUDA(launch_slab_gather_rows<T>(
                p->nx, sl->row_first, sl->ext_rows, phase != 0 ? field_vsh<T>(p, field_n) : nullptr,
                static_cast<VShift<T>*>(sl->d_vsh), phase != 2 ? field_vsh<T>(p, field_prev) : nullptr,
                static_cast<VShift<T>*>(sl->d_vsh2), phase != 0 ? grho : nullptr, static_cast<T*>(sl->d_grho), s),
            "slab row gather launch");
    b.vsh_n = static_cast<const VShift<T>*>(sl->d_vsh);
    b.vsh_prev = static_cast<const VShift<T>*>(sl->d_vsh2);
    b.grho = static_cast<const T*>(sl->d_grho);
    b.w_in = static_cast<const T*>(w_ext);
    b.h_prev = static_cast<const T*>(h_prev_ext);
    b.w_out = static_cast<T*>(w_out_ext);
    if (phase == 0) {
        b.c_src = static_cast<const T*>(g_ext);
    } else if (phase == 1) {
        b.gfh = static_cast<const T*>(g_ext);
    } else {
        if ((rc = slab_lazy_cells<T>(sl, false)) != VP_OK) return rc;
        b.gfiv_out = static_cast<T*>(sl->d_cells);
    }
    if (phase == 0 && g_ext == nullptr) {
        // no cotangent on the final state: w_{T-1} = X^T(0) = 0 and the slope sums are 0
        VP_CUDA(cudaMemsetAsync(w_out_ext, 0, (size_t)sl->ext_rows * p->nv * sizeof(T), s), "cudaMemsetAsync(w)");
        VP_CUDA(cudaMemsetAsync(slope_sums, 0, (size_t)sl->n_rows * sizeof(T), s), "cudaMemsetAsync(slope sums)");
        return VP_OK;
    }
    VP_CUDA(launch_bwd<T>(b, sl->cfg, phase, false, s), "slab adjoint launch");
    if (phase == 2) return slab_copy_owned(sl, sl->d_cells, g_f_iv_rows, sizeof(T), s);
    VP_CUDA(launch_slab_row_sums<T>(static_cast<const T*>(sl->d_part), sl->cfg.n_chunks, sl->ext_rows, sl->ghost,
                                    sl->n_rows, static_cast<T*>(slope_sums), s),
            "slab row sums launch");
    return VP_OK;
}

template <typename T>
static int slab_backward_field_impl(vp_slab* sl, const T* sums, const void* field_prev, const T* gE_hist_row,
                                    const T* gee, T* g_H, T* grho, cudaStream_t s) {
    const vp_plan* p = sl->plan;
    BwdArgs<T> b{};
    b.nx = p->nx;
    b.nv = p->nv;
    b.n_chunks = 1;
    b.part = const_cast<T*>(sums);
    b.P = slab_poisson<T>(sl);
    b.dv = (T)p->dv;
    b.dx = (T)p->dx;
    b.neg_dt_dv = (T)(-p->dt / p->dv);
    b.E_prev = field_E<T>(p, field_prev);
    b.gE_hist = gE_hist_row;
    b.gee = gee;
    b.gH = g_H;
    b.grho_out = grho;
    VP_CUDA(launch_bwd_tail<T>(b, sl->tail_threads, sl->tail_smem, sl->tail_tw_stage != 0, s), "slab adjoint field launch");
    return VP_OK;
}

}  // namespace vpb

extern "C" {

int vp_slab_create(vp_plan* plan, int32_t row0, int32_t n_rows, vp_slab** out) {
    if (!plan || !out) return set_err(VP_ERR_ARG, "plan and out must not be NULL");
    *out = nullptr;
    if (plan->feq2d)
        return set_err(VP_ERR_UNSUPPORTED, "x slabs need an x-invariant f_eq (one row of nv values)");
    if (n_rows < 1 || row0 < 0 || row0 + (int64_t)n_rows > plan->nx)
        return set_err(VP_ERR_ARG, "slab rows [%d, %d) do not lie in [0, %d)", row0, row0 + n_rows, plan->nx);
    // rows a step reads around its own: x offsets m in [mx_lo, mx_hi]; the forward reads rows r + 2m
    // .. r + 2m + 2 (v-step inputs of the two x half-steps), the adjoint rows r - 2m - 2 .. r - 2m
    const long long g = std::max({-2 * plan->mx_lo, 2 * plan->mx_hi + 2, 1LL});
    if (g > n_rows)
        return set_err(VP_ERR_ARG,
                       "a slab of %d rows is thinner than the %lld ghost rows a step reads from each neighbour "
                       "(x shifts of up to %lld cells); use fewer, thicker slabs",
                       n_rows, g, std::max(-plan->mx_lo, plan->mx_hi + 1));
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(plan->device);
    vp_slab* sl = new (std::nothrow) vp_slab();
    if (!sl) {
        cudaSetDevice(prev);
        return set_err(VP_ERR_ARG, "out of host memory");
    }
    sl->plan = plan;
    sl->row0 = row0;
    sl->n_rows = n_rows;
    sl->ghost = (int)g;
    sl->cfg = plan->cfg;
    const int R = std::max(1, sl->cfg.R);
    sl->ext_rows = (n_rows + 2 * sl->ghost + R - 1) / R * R;
    sl->row_first = (int)(((long long)row0 - sl->ghost) % plan->nx + plan->nx) % plan->nx;
    const size_t rs = real_size(plan);
    if (plan->tail_inline) {
        // the one-grid path solves the field inside the step launch, with the step's block size
        sl->tail_threads = plan->cfg.threads;
        sl->tail_smem = poisson_area_size(plan->nx, rs);
    } else {
        sl->tail_threads = plan->tail_threads;
        sl->tail_smem = plan->tail_smem;
        sl->tail_tw_stage = plan->tail_tw_stage;
    }
    std::vector<int> mx(plan->nv);
    for (int j = 0; j < plan->nv; ++j) {
        const long long m = plan->host_mxs[j];
        mx[j] = (int)(((m % sl->ext_rows) + sl->ext_rows) % sl->ext_rows);
    }
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void** q, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(q, bytes);
    };
    alloc((void**)&sl->d_mx, (size_t)plan->nv * sizeof(int));
    alloc(&sl->d_part, (size_t)sl->cfg.n_chunks * sl->ext_rows * rs);
    alloc(&sl->d_vsh, (size_t)sl->ext_rows * vshift_size(plan));
    alloc(&sl->d_vsh2, (size_t)sl->ext_rows * vshift_size(plan));
    alloc(&sl->d_grho, (size_t)sl->ext_rows * rs);
    if (sl->tail_smem == 0) alloc(&sl->d_gscratch, (size_t)2 * plan->nx * rs);
    if (e == cudaSuccess)
        e = cudaMemcpy(sl->d_mx, mx.data(), mx.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        free_slab(sl);
        return cuda_err(e, "vp_slab_create");
    }
    *out = sl;
    return VP_OK;
}

int vp_slab_destroy(vp_slab* slab) {
    free_slab(slab);
    return VP_OK;
}

int vp_slab_geometry(const vp_slab* slab, int32_t* ghost_rows, int32_t* ext_rows, size_t* field_bytes) {
    if (!slab) return set_err(VP_ERR_ARG, "slab must not be NULL");
    if (ghost_rows) *ghost_rows = slab->ghost;
    if (ext_rows) *ext_rows = slab->ext_rows;
    if (field_bytes) *field_bytes = slab_field_bytes(slab->plan);
    return VP_OK;
}

int vp_slab_forward_start(vp_slab* slab, const double* f_iv_ext, void* h_ext, void* row_sums, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    if ((rc = slab_check(slab, s)) != VP_OK) return rc;
    const int dev = slab->plan->device;
    if ((rc = check_dev_ptr(f_iv_ext, "f_iv_ext", dev)) || (rc = check_dev_ptr(h_ext, "h_ext", dev)) ||
        (rc = check_dev_ptr(row_sums, "row_sums", dev)))
        return rc;
    if (slab->plan->dtype == VP_F64)
        return slab_forward_impl<double>(slab, 0, f_iv_ext, nullptr, h_ext, row_sums, nullptr, nullptr, s);
    return slab_forward_impl<float>(slab, 0, f_iv_ext, nullptr, h_ext, row_sums, nullptr, nullptr, s);
}

int vp_slab_field(vp_slab* slab, const void* row_sums_all, const void* H, void* field, void* E_hist_row, void* ee,
                  void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    if ((rc = slab_check(slab, s)) != VP_OK) return rc;
    const int dev = slab->plan->device;
    if ((rc = check_dev_ptr(row_sums_all, "row_sums_all", dev)) || (rc = check_dev_ptr(H, "H", dev)) ||
        (rc = check_dev_ptr(field, "field", dev)) || (rc = check_opt_ptr(E_hist_row, "E_hist_row", dev)) ||
        (rc = check_opt_ptr(ee, "ee", dev)))
        return rc;
    if (((uintptr_t)field & 255) != 0) return set_err(VP_ERR_ARG, "field must be 256-byte aligned");
    if (slab->plan->dtype == VP_F64)
        return slab_field_impl<double>(slab, (const double*)row_sums_all, (const double*)H, field, (double*)E_hist_row,
                                       (double*)ee, s);
    return slab_field_impl<float>(slab, (const float*)row_sums_all, (const float*)H, field, (float*)E_hist_row,
                                  (float*)ee, s);
}

int vp_slab_forward_step(vp_slab* slab, const void* h_ext, const void* field, void* h_out_ext, void* row_sums,
                         void* f_rows, double* f_final_rows, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    if ((rc = slab_check(slab, s)) != VP_OK) return rc;
    const int dev = slab->plan->device;
    if ((rc = check_dev_ptr(h_ext, "h_ext", dev)) || (rc = check_dev_ptr(field, "field", dev)) ||
        (rc = check_opt_ptr(h_out_ext, "h_out_ext", dev)) || (rc = check_opt_ptr(row_sums, "row_sums", dev)) ||
        (rc = check_opt_ptr(f_rows, "f_rows", dev)) || (rc = check_opt_ptr(f_final_rows, "f_final_rows", dev)))
        return rc;
    if (h_ext == h_out_ext) return set_err(VP_ERR_ARG, "h_ext and h_out_ext must be different arrays");
    if (slab->plan->dtype == VP_F64)
        return slab_forward_impl<double>(slab, 1, h_ext, field, h_out_ext, row_sums, f_rows, f_final_rows, s);
    return slab_forward_impl<float>(slab, 1, h_ext, field, h_out_ext, row_sums, f_rows, f_final_rows, s);
}

int vp_slab_backward_start(vp_slab* slab, const void* g_f_ext, const void* h_prev_ext, const void* field_prev,
                           void* w_out_ext, void* slope_sums, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    if ((rc = slab_check(slab, s)) != VP_OK) return rc;
    const int dev = slab->plan->device;
    if ((rc = check_opt_ptr(g_f_ext, "g_f_ext", dev)) || (rc = check_dev_ptr(h_prev_ext, "h_prev_ext", dev)) ||
        (rc = check_dev_ptr(field_prev, "field_prev", dev)) || (rc = check_dev_ptr(w_out_ext, "w_out_ext", dev)) ||
        (rc = check_dev_ptr(slope_sums, "slope_sums", dev)))
        return rc;
    if (slab->plan->dtype == VP_F64)
        return slab_backward_impl<double>(slab, 0, nullptr, g_f_ext, nullptr, nullptr, field_prev, h_prev_ext,
                                          w_out_ext, slope_sums, nullptr, s);
    return slab_backward_impl<float>(slab, 0, nullptr, g_f_ext, nullptr, nullptr, field_prev, h_prev_ext, w_out_ext,
                                     slope_sums, nullptr, s);
}

int vp_slab_backward_field(vp_slab* slab, const void* slope_sums_all, const void* field_prev, const void* gE_hist_row,
                           const void* gee, void* g_H, void* grho, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    if ((rc = slab_check(slab, s)) != VP_OK) return rc;
    const int dev = slab->plan->device;
    if ((rc = check_dev_ptr(slope_sums_all, "slope_sums_all", dev)) ||
        (rc = check_dev_ptr(field_prev, "field_prev", dev)) || (rc = check_opt_ptr(gE_hist_row, "gE_hist_row", dev)) ||
        (rc = check_opt_ptr(gee, "gee", dev)) || (rc = check_dev_ptr(g_H, "g_H", dev)) ||
        (rc = check_dev_ptr(grho, "grho", dev)))
        return rc;
    if (slab->plan->dtype == VP_F64)
        return slab_backward_field_impl<double>(slab, (const double*)slope_sums_all, field_prev,
                                                (const double*)gE_hist_row, (const double*)gee, (double*)g_H,
                                                (double*)grho, s);
    return slab_backward_field_impl<float>(slab, (const float*)slope_sums_all, field_prev, (const float*)gE_hist_row,
                                           (const float*)gee, (float*)g_H, (float*)grho, s);
}

int vp_slab_backward_step(vp_slab* slab, const void* w_ext, const void* g_f_ext, const void* grho,
                          const void* field_n, const void* field_prev, const void* h_prev_ext, void* w_out_ext,
                          void* slope_sums, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    if ((rc = slab_check(slab, s)) != VP_OK) return rc;
    const int dev = slab->plan->device;
    if ((rc = check_dev_ptr(w_ext, "w_ext", dev)) || (rc = check_opt_ptr(g_f_ext, "g_f_ext", dev)) ||
        (rc = check_dev_ptr(grho, "grho", dev)) || (rc = check_dev_ptr(field_n, "field_n", dev)) ||
        (rc = check_dev_ptr(field_prev, "field_prev", dev)) || (rc = check_dev_ptr(h_prev_ext, "h_prev_ext", dev)) ||
        (rc = check_dev_ptr(w_out_ext, "w_out_ext", dev)) || (rc = check_dev_ptr(slope_sums, "slope_sums", dev)))
        return rc;
    if (w_ext == w_out_ext) return set_err(VP_ERR_ARG, "w_ext and w_out_ext must be different arrays");
    if (slab->plan->dtype == VP_F64)
        return slab_backward_impl<double>(slab, 1, w_ext, g_f_ext, (const double*)grho, field_n, field_prev,
                                          h_prev_ext, w_out_ext, slope_sums, nullptr, s);
    return slab_backward_impl<float>(slab, 1, w_ext, g_f_ext, (const float*)grho, field_n, field_prev, h_prev_ext,
                                     w_out_ext, slope_sums, nullptr, s);
}

int vp_slab_backward_finish(vp_slab* slab, const void* w_ext, const void* grho, const void* field0, void* g_f_iv_rows,
                            void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    if ((rc = slab_check(slab, s)) != VP_OK) return rc;
    const int dev = slab->plan->device;
    if ((rc = check_dev_ptr(w_ext, "w_ext", dev)) || (rc = check_dev_ptr(grho, "grho", dev)) ||
        (rc = check_dev_ptr(field0, "field0", dev)) || (rc = check_dev_ptr(g_f_iv_rows, "g_f_iv_rows", dev)))
        return rc;
    if (slab->plan->dtype == VP_F64)
        return slab_backward_impl<double>(slab, 2, w_ext, nullptr, (const double*)grho, field0, nullptr, nullptr,
                                          nullptr, nullptr, g_f_iv_rows, s);
    return slab_backward_impl<float>(slab, 2, w_ext, nullptr, (const float*)grho, field0, nullptr, nullptr, nullptr,
                                     nullptr, g_f_iv_rows, s);
}

}  // extern "C"
