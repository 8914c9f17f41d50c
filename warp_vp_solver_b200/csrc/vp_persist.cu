// Persistent forward time loop for large grids (float32, x-invariant f_eq, Strang scheme).
//
// One cooperative launch runs a whole forward loop (warp_vp_solver/solver.py:470-612): the
// per-step launches, the one-CTA Poisson tail and the host round trips of the reference (and of
// the per-step kernels in vp_kernels.cu) become one kernel whose CTAs meet at a software grid
// barrier once per step (twice on grids whose field is solved in slices, below).
//
// Work split. CTA g owns `bands_per_cta` consecutive bands of R rows, full width; a band is
// processed as n_chunks tiles of R rows x C = 256 columns. Because a CTA owns whole rows, the row
// sums of h_{n+1} (rho_{n+1}) are complete inside it and need no cross-CTA partials.
//
// Tile. Thread t (64 per CTA) owns the 4 consecutive columns j0 = c0 + 4t .. j0 + 3. The x shifts
// m_j of 4 neighbouring columns differ by at most one cell (checked on the host), so the thread
// walks one window of R + 4 rows of the v-step output o, rows r0 + 2*bm + k (bm = the smallest
// shift of its quad); a column whose shift is bm + 1 reads the same window two rows lower (a
// register select). The window rows of a tile are staged into shared memory by asynchronous
// 16-byte copies of every thread (cp.async.cg through L2, one commit group per tile) into a ring
// of up to 8 stage buffers, so that later tiles' rows arrive while one computes (one-kilobyte
// cp.async.bulk copies per row were measured to be limited by the copy engine's per-copy cost:
// about 80 ns each). Per window row the v step reads its 5 source cells with one
// 16-byte and one 4-byte shared-memory load and forms V(f_eq) - f_eq for the usual shifts m = 0
// and m = -1 from the first differences D of f_eq held in registers:
//   m = 0:  o = h[j] + t*((h[j+1] - h[j]) + D[j])
//   m = -1: o = (h[j-1] - D[j-1]) + t*((h[j] - h[j-1]) + D[j-1])
// (the same value as lerp + correction of the per-step kernels, associated differently); shifts in
// [-4, 4) use the A_m, B_m tables, larger ones the float64 form from global memory.
//
// Field. After the barrier every CTA needs E + H on the rows its next tiles read. On grids where
// that window times nx is small (configuration 3: 28 rows x 512), each CTA evaluates
// E_i = sum_k c[(i-k) mod nx] rho_k for its window rows itself (c = real(ifft(m)), the circulant
// form of warp_vp_solver/poisson.py:34-69); otherwise CTA g solves a slice of nx/G rows, publishes
// their v shifts, and a second barrier precedes the tiles. The energies of the own rows go to
// per-CTA partials that CTA 0 sums in a fixed order one step later, so every result is
// deterministic.
//
// The grid barrier's wait is bounded: a barrier that does not complete within the plan's wait
// limit raises VP_STATUS_WAIT_TIMEOUT in the plan's status word and the CTA returns after waiting
// for its own copies in flight.

#include "vp_pst.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace vpb {

namespace {

// Field inputs up to this size get their own shared memory (the first tiles of a step then load
// while the field is solved); larger ones reuse the stage buffers.
constexpr size_t kPstOwnFieldBytes = 24 * 1024;

}  // namespace

// Shared memory of a launch: the stage area (two stage buffers, or the field inputs when those are
// larger and share it), the row records of the union window, the row-sum scratch, and the field
// inputs when they have their own region.
size_t persist_smem_bytes(int span_max, int win_rows, int R, int nx, int nv, int field_rows, int stages,
                          int* stage_floats, int* fs_alias) {
    const int groups = std::min(kPstGroups, nv / kPstC);   // groups that have chunks to stage
    const size_t st = (size_t)groups * stages * span_max * kPstW;
    const size_t ff = (pst_field_floats(nx, field_rows) + 3) & ~(size_t)3;
    const bool alias = ff * sizeof(float) > kPstOwnFieldBytes;
    const size_t area = alias ? std::max(st, ff) : st;
    size_t b = area * sizeof(float);
    b += ((size_t)win_rows * sizeof(int2) + 15) & ~(size_t)15;
    b += (size_t)kPstWarps * R * sizeof(float) + 16;
    if (!alias) b += ff * sizeof(float);
    const size_t qb = (size_t)(nv / 4) * sizeof(PstQuad);
    if (qb <= kPstQuadSmemBytes) b += qb;
    if (stage_floats) *stage_floats = (int)area;
    if (fs_alias) *fs_alias = alias ? 1 : 0;
    return b;
}

template <int R>
__global__ void __launch_bounds__(kPstThreads, 2) vp_persist_fwd_kernel(const PersistArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_flag;
    __shared__ double s_ee[kPstWarps];

    const int nx = a.nx, nv = a.nv, nch = a.n_chunks;
    const size_t nxnv = (size_t)nx * nv;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int gid = tid / kPstGroup, gt = tid - gid * kPstGroup;   // column group and its thread
    const int g = blockIdx.x, G = gridDim.x;
    // bands g, g + G, g + 2G, ...: at any time the CTAs work on neighbouring rows, so the halo rows
    // a tile reads were just read (or written) by a neighbour and are found in L2
    const int bpc = a.bands_per_cta;
    auto band_row = [&](int bi) { return (g + bi * G) * R; };
    const int S = a.stages;                           // stage buffers per group
    float* stages = reinterpret_cast<float*>(smem);
    int2* rinfo = reinterpret_cast<int2*>(stages + (size_t)a.stage_floats);   // [bpc][win_rows]
    float* red = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(rinfo) +
                                          (((size_t)bpc * a.win_rows * sizeof(int2) + 15) & ~(size_t)15));
    // field inputs: their own region after the row-sum scratch, or the stage area
    float* fs = a.fs_alias ? stages : red + kPstWarps * R + 4;
    const size_t ff = ((size_t)2 * nx + a.field_rows + 8 + 3) & ~(size_t)3;
    const int nq = nv / 4;
    PstQuad* sq = ((size_t)nq * sizeof(PstQuad) <= kPstQuadSmemBytes)
                      ? reinterpret_cast<PstQuad*>(a.fs_alias ? red + kPstWarps * R + 4 : fs + ff)
                      : nullptr;
    const bool replay = a.mode == 1;
    const int n_first = replay ? a.first_step : 0;
    const int n_end = a.n_steps;                      // steps n_first .. n_end - 1
    // chunks of this group: c = gid, gid + 4, ...; its tiles per step: bands x those chunks
    const int cpg = gid < nch ? (nch - gid + kPstGroups - 1) / kPstGroups : 0;
    const int ntile = a.bands_per_cta * cpg;

    auto quad_of = [&](int q) -> PstQuad {
        PstQuad r;
        const int2 qi = __ldg(a.quad + q);
        r.t = __ldg(a.tq + q);
        r.D = __ldg(reinterpret_cast<const float4*>(a.dfeq) + q);
        r.bm = qi.x;
        r.mask = qi.y;
        r.Dm1 = __ldg(a.dfeq + (q == 0 ? nv - 1 : 4 * q - 1));
        r.pad = 0.f;
        return r;
    };
    if (sq != nullptr)
        for (int q = tid; q < nq; q += blockDim.x) sq[q] = quad_of(q);
    __syncthreads();

    auto slot = [&](int n) -> float* {
        if (a.ckpt != nullptr && n % a.K == 0) return a.ckpt + (size_t)(n / a.K) * nxnv;
        if (replay) return a.seg + (size_t)(n % a.K - 1) * nxnv;
        return (n & 1) ? a.hbuf1 : a.hbuf0;
    };

    unsigned bar_index = 0;
    bool alive = true;
    auto barrier = [&]() -> bool {
        if (!pst_grid_barrier(a.bar, bar_index++, (unsigned)G, a.wait_ns, a.status, &s_flag)) alive = false;
        return alive;
    };
    auto group_sync = [&]() { asm volatile("bar.sync %0, %1;" ::"r"(1 + gid), "r"(kPstGroup) : "memory"); };

    // ---- staging: the group's tile j of a step (band j / cpg, chunk gid + 4 (j % cpg)) goes to
    // the group's stage (k % S), k counting the group's tiles over the launch; 16-byte
    // asynchronous copies of the group's threads, one commit group per tile ----
    constexpr int kPieces = kPstW / 4;               // 16-byte pieces of a staged row
    unsigned tiles_issued = 0, tiles_used = 0;
    auto tile_of = [&](int j, int* r0, int* c) {
        const int bi = j / cpg;
        *c = gid + kPstGroups * (j - bi * cpg);
        *r0 = band_row(bi);
    };
    auto stage_ptr = [&](unsigned k) {
        return stages + (gid * S + (int)(k % (unsigned)S)) * a.span_max * kPstW;   // 32-bit shared offsets
    };
    auto issue = [&](int j, const float* src) {
        const unsigned mine = tiles_issued++;
        int r0, c;
        tile_of(j, &r0, &c);
        const int c0 = c * kPstC;
        const int2 cm = __ldg(a.chunk + c);           // (min bm, max bm) over the chunk
        const int span = 2 * (cm.y - cm.x) + R + 4;
        const int lo = r0 + 2 * cm.x;
        float* st = stage_ptr(mine);
        for (int p = gt; p < span * kPieces; p += kPstGroup) {
            const int k = p / kPieces, v = p - k * kPieces;
            int col = c0 - 4 + 4 * v;
            col += col < 0 ? nv : 0;
            col -= col >= nv ? nv : 0;
            pst_cp16(st + (k * kPstW + 4 * v), src + (size_t)pst_wrap(lo + k, nx) * nv + col);
        }
        pst_cp_commit();
    };
    auto issue_first = [&](const float* src) {
        for (int j = 0; j < S && j < ntile; ++j) issue(j, src);
    };

    // ---- field: v shifts of each band's window rows [r0 + win_lo, r0 + win_lo + win_rows) into
    // rinfo[band][.] ----
    auto field_local = [&](int n, const float* tiles_src) {
        // E of every window row from rho_n; the band's own rows also write E_hist, the tape and the
        // energy partial. With tiles_src, the step's first tiles are issued right after the first
        // band's field inputs, so that they load while the field is solved.
        double e2 = 0.0;
        for (int bi = 0; bi < bpc; ++bi) {
            const int wf = band_row(bi) + a.win_lo;
            if (bi > 0) __syncthreads();   // the previous band's circulant has read the inputs
            if (bi == 0 && tiles_src != nullptr) {
                pst_field_issue(fs, a.rho + (size_t)(n & 1) * nx, a.ctab, nx, wf, a.win_rows);
                issue_first(tiles_src);
                pst_cp_wait((int)(tiles_issued - tiles_used));   // the field group only
                __syncthreads();
            } else {
                pst_field_inputs(fs, a.rho + (size_t)(n & 1) * nx, a.ctab, nx, wf, a.win_rows);
            }
            int2* ri = rinfo + (size_t)bi * a.win_rows;
            pst_circ_rows(fs, nx, a.win_rows, [&](int u, float E) {
                const int i = pst_wrap(wf + u, nx);
                const float Et = E + __ldg(a.H + i);
                const VShift<float> vs = make_vshift<float>(Et, a.dtdv, nv);
                ri[u] = pst_rinfo(vs, nv);
                const int own = u + a.win_lo;          // row offset from the band's first row
                if (own >= 0 && own < R) {
                    if (a.E_hist != nullptr) a.E_hist[(size_t)n * nx + i] = Et;
                    if (a.E_tape != nullptr) a.E_tape[(size_t)n * nx + i] = E;
                    if (a.vsh_tape != nullptr) a.vsh_tape[(size_t)n * nx + i] = vs;
                    e2 += (double)(trap_w<float>(i, nx) * E * E);
                }
            });
        }
        return e2;
    };
    auto field_slice = [&](int n) {
        const int Sl = (nx + G - 1) / G;
        const int first = g * Sl;
        const int cnt = max(0, min(Sl, nx - first));
        pst_field_inputs(fs, a.rho + (size_t)(n & 1) * nx, a.ctab, nx, first, cnt);
        double e2 = 0.0;
        pst_circ_rows(fs, nx, cnt, [&](int u, float E) {
            const int i = first + u;
            const float Et = E + __ldg(a.H + i);
            const VShift<float> vs = make_vshift<float>(Et, a.dtdv, nv);
            a.vsh_g[i] = vs;
            if (a.E_hist != nullptr) a.E_hist[(size_t)n * nx + i] = Et;
            if (a.E_tape != nullptr) a.E_tape[(size_t)n * nx + i] = E;
            if (a.vsh_tape != nullptr) a.vsh_tape[(size_t)n * nx + i] = vs;
            e2 += (double)(trap_w<float>(i, nx) * E * E);
        });
        return e2;
    };
    auto rinfo_from = [&](const VShift<float>* vsh) {
        for (int x = tid; x < bpc * a.win_rows; x += blockDim.x) {
            const int bi = x / a.win_rows, u = x - bi * a.win_rows;
            const VShift<float>* p = vsh + pst_wrap(band_row(bi) + a.win_lo + u, nx);
            VShift<float> v;
            v.m = __ldcg(&p->m);
            v.t = __ldcg(&p->t);
            rinfo[x] = pst_rinfo(v, nv);
        }
    };
    auto publish_energy = [&](int n, double e2) {
        e2 = warp_sum(e2);
        if (lane == 0) s_ee[wid] = e2;
        __syncthreads();
        if (tid == 0) {
            double sum = 0.0;
            for (int w = 0; w < kPstWarps; ++w) sum += s_ee[w];
            a.eep[(size_t)n * G + g] = sum;
        }
    };
    // ee_hist[n] from the G partials of step n (after the barrier that published them): lanes sum
    // in a fixed order, then a fixed butterfly. The steps are shared out over the CTAs at the end.
    auto sum_energy = [&](int n) {
        double sum = 0.0;
        for (int c = lane; c < G; c += 32) sum += __ldcg(a.eep + (size_t)n * G + c);
        sum = warp_sum(sum);
        if (lane == 0) a.ee_hist[n] = (float)(0.5 * sum * (double)a.dx);
    };

    // ---- row sums of a band: acc[R] over the CTA's threads in a fixed order -> rho ----
    auto band_rows = [&](float (&acc)[R], int r0, float* rho_out) {
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
        __syncthreads();
        if (tid < R) {
            float sum = 0.f;
            for (int w = 0; w < kPstWarps; ++w) sum += red[w * R + tid];
            rho_out[r0 + tid] = -a.dv * sum;
        }
        __syncthreads();
    };

    // ---- prologue (full mode): h_0 = X(f_iv - f_eq) on the own rows, rho_0 ----
    if (!replay) {
        float* h0 = slot(0);
        for (int bi = 0; bi < bpc; ++bi) {
            const int r0 = band_row(bi);
            float acc[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = 0.f;
            for (int c = gid; c < nch; c += kPstGroups) {
                const int q = c * kPstGroup + gt;
                const int j0 = 4 * q;
                const PstQuad Q = sq != nullptr ? sq[q] : quad_of(q);
                const double2 fa = __ldg(reinterpret_cast<const double2*>(a.feq + j0));
                const double2 fb = __ldg(reinterpret_cast<const double2*>(a.feq + j0 + 2));
                const double fe[4] = {fa.x, fa.y, fb.x, fb.y};
                const float tt[4] = {Q.t.x, Q.t.y, Q.t.z, Q.t.w};
                const float w0 = j0 == 0 ? 0.5f : 1.f, w3 = j0 + 3 == nv - 1 ? 0.5f : 1.f;
                // rolling over the rows of d = f_iv - f_eq: output row r = k - 2 reads d rows
                // r + delta and r + 1 + delta
                float d[3][4];
#pragma unroll
                for (int k = 0; k < R + 2; ++k) {
                    const int row = pst_wrap(r0 + Q.bm + k, nx);
                    const double2* fr = reinterpret_cast<const double2*>(a.f_iv + (size_t)row * nv + j0);
                    const double2 u = __ldg(fr), v = __ldg(fr + 1);
                    d[k % 3][0] = (float)(u.x - fe[0]);
                    d[k % 3][1] = (float)(u.y - fe[1]);
                    d[k % 3][2] = (float)(v.x - fe[2]);
                    d[k % 3][3] = (float)(v.y - fe[3]);
                    if (k >= 2) {
                        const int r = k - 2;
                        float hv[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const bool dl = (Q.mask >> e) & 1;
                            const float p0 = dl ? d[(r + 1) % 3][e] : d[r % 3][e];
                            const float p1 = dl ? d[(r + 2) % 3][e] : d[(r + 1) % 3][e];
                            hv[e] = pst_lerp(p0, p1, tt[e]);
                        }
                        *reinterpret_cast<float4*>(h0 + (size_t)(r0 + r) * nv + j0) =
                            make_float4(hv[0], hv[1], hv[2], hv[3]);
                        acc[r] += w0 * hv[0] + hv[1] + hv[2] + w3 * hv[3];
                    }
                }
            }
            band_rows(acc, r0, a.rho);   // rho_0 in buffer 0
        }
        if (!barrier()) return;
    }

    for (int n = n_first; n < n_end && alive; ++n) {
        const bool last = !replay && n == a.n_steps - 1;
        const float* src = slot(n);
        float* dst = last ? nullptr : slot(n + 1);
        // the first tiles of the step load while the field is solved (after it, when the field's
        // inputs share the stage buffers)
        const bool early = replay || !a.fs_alias;
        if (early && (replay || a.field_dist != 0)) issue_first(src);
        if (replay) {
            rinfo_from(a.vsh_tape_in + (size_t)n * nx);
        } else if (a.field_dist == 0) {
            const double e2 = field_local(n, early ? src : nullptr);
            publish_energy(n, e2);
        } else {
            const double e2 = field_slice(n);
            publish_energy(n, e2);
            if (!early) issue_first(src);
            if (!barrier()) break;
            rinfo_from(a.vsh_g);
        }
        __syncthreads();
        if (!early && a.field_dist == 0) issue_first(src);

        float* rho_next = a.rho + (size_t)((n + 1) & 1) * nx;
        float acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = 0.f;
        for (int bi = 0; bi < bpc; ++bi) {
            const int r0 = band_row(bi);
            for (int jj = 0; jj < cpg; ++jj) {
                const int j = bi * cpg + jj;
                const int c = gid + kPstGroups * jj;
                const int c0 = c * kPstC;
                const int q = c * kPstGroup + gt;
                const int j0 = c0 + 4 * gt;
                const int2 cm = __ldg(a.chunk + c);
                const PstQuad Q = sq != nullptr ? sq[q] : quad_of(q);
                const int2 qi = make_int2(Q.bm, Q.mask);
                const float tt[4] = {Q.t.x, Q.t.y, Q.t.z, Q.t.w};
                const float4 D4 = Q.D;
                const float Dm1 = Q.Dm1;
                pst_cp_wait((int)(tiles_issued - tiles_used - 1));   // groups committed after this tile's
                group_sync();
                const float* st = stage_ptr(tiles_used);
                ++tiles_used;
                // window row k of this thread: stage row 2*(bm - cm.x) + k, global row r0 + 2*bm + k
                const float* sb = st + (2 * (qi.x - cm.x) * kPstW + 4 + 4 * gt);
                const int ib = bi * a.win_rows + 2 * qi.x - a.win_lo;   // rinfo index of window row 0
                // rolling over the window rows: after o row k, d row q = k - 3 (o rows q .. q + 3)
                // and h' row r = k - 4 (d rows r, r + 1) are complete
                float O[4][4], dprev[4];
                float* fh = a.f_hist != nullptr ? a.f_hist + (size_t)(n - n_first) * nxnv : nullptr;
                const bool fout = fh != nullptr || (last && a.f_final != nullptr);
                const float w0 = j0 == 0 ? 0.5f : 1.f, w3 = j0 + 3 == nv - 1 ? 0.5f : 1.f;
#pragma unroll
                for (int k = 0; k < R + 4; ++k) {
                    float* o = O[k & 3];
                    const int2 ri = rinfo[ib + k];
                    const float tv = __int_as_float(ri.y);
                    const float* sr = sb + k * kPstW;
                    if (ri.x == 0) {
                        const float4 h = *reinterpret_cast<const float4*>(sr);
                        const float h4 = sr[4];
                        o[0] = h.x + tv * ((h.y - h.x) + D4.x);
                        o[1] = h.y + tv * ((h.z - h.y) + D4.y);
                        o[2] = h.z + tv * ((h.w - h.z) + D4.z);
                        o[3] = h.w + tv * ((h4 - h.w) + D4.w);
                    } else if (ri.x == -1) {
                        const float hm = sr[-1];
                        const float4 h = *reinterpret_cast<const float4*>(sr);
                        o[0] = (hm - Dm1) + tv * ((h.x - hm) + Dm1);
                        o[1] = (h.x - D4.x) + tv * ((h.y - h.x) + D4.x);
                        o[2] = (h.y - D4.y) + tv * ((h.z - h.y) + D4.y);
                        o[3] = (h.z - D4.z) + tv * ((h.w - h.z) + D4.z);
                    } else {
                        const float4 r4 = pst_v_rare(a.vtab, a.feq, nv, sr, src, ri.x, tv, pst_wrap(r0 + 2 * qi.x + k, nx), j0);
                        o[0] = r4.x;
                        o[1] = r4.y;
                        o[2] = r4.z;
                        o[3] = r4.w;
                    }
                    if (k >= 3) {
                        // d row q per column: window offset 0 or 2 rows (delta bit)
                        const int q = k - 3;
                        float dn[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const bool dl = (qi.y >> e) & 1;
                            const float p0 = dl ? O[(q + 2) & 3][e] : O[q & 3][e];
                            const float p1 = dl ? O[(q + 3) & 3][e] : O[(q + 1) & 3][e];
                            dn[e] = pst_lerp(p0, p1, tt[e]);
                        }
                        if (fout && q < R) {
#pragma unroll
                            for (int e = 0; e < 4; ++e) {
                                const int row = pst_wrap(r0 + qi.x + ((qi.y >> e) & 1) + q, nx);
                                const double f = __ldg(a.feq + j0 + e) + (double)dn[e];
                                if (fh != nullptr) fh[(size_t)row * nv + j0 + e] = (float)f;
                                if (last && a.f_final != nullptr) a.f_final[(size_t)row * nv + j0 + e] = f;
                            }
                        }
                        if (q >= 1 && dst != nullptr) {
                            const int r = q - 1;
                            const float h0v = pst_lerp(dprev[0], dn[0], tt[0]);
                            const float h1v = pst_lerp(dprev[1], dn[1], tt[1]);
                            const float h2v = pst_lerp(dprev[2], dn[2], tt[2]);
                            const float h3v = pst_lerp(dprev[3], dn[3], tt[3]);
                            *reinterpret_cast<float4*>(dst + (size_t)(r0 + r) * nv + j0) =
                                make_float4(h0v, h1v, h2v, h3v);
                            acc[r] += w0 * h0v + h1v + h2v + w3 * h3v;
                        }
#pragma unroll
                        for (int e = 0; e < 4; ++e) dprev[e] = dn[e];
                    }
                }
                group_sync();   // the stage is free
                if (j + S < ntile) issue(j + S, src);
            }
            // every group has finished the band: its row sums
            if (!replay && !last) band_rows(acc, r0, rho_next);
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = 0.f;
        }
        if (!barrier()) break;
    }
    // a CTA that stopped early still owns the copies it issued: wait for them
    pst_cp_wait(0);
    if (alive && !replay && a.ee_hist != nullptr)
        for (int n = g * kPstWarps + wid; n < a.n_steps; n += G * kPstWarps) sum_energy(n);
}

// ---------------------------------------------------------------------------------------------
// Persistent adjoint steps (the per-step phase of the discrete adjoint, warp_vp_solver/solver.py:
// 814-929): for n = n_hi down to n_lo, gh = V^T w_n + rho^T grho_n on a window of R + 4 rows,
// c = X^T gh (+ the f_hist cotangent), w_{n-1} = X^T c on the own rows, and the slope row sums of
// h_{n-1}; after the grid barrier g_E and grho_{n-1} = Poisson^T g_E (transposed circulant). Same
// work split, column groups, staging ring and barrier as the forward loop. The thread of column
// shift m reads the window rows r0 - 2m - 2 + k; a quad's window is rows r0 - 2 bm - 4 + k',
// k' < R + 4, and a column with shift bm reads it two rows higher than one with bm + 1.
// ---------------------------------------------------------------------------------------------


template <int R>
__global__ void __launch_bounds__(kPstThreads, 2) vp_persist_bwd_kernel(const PersistBwdArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_flag;

    const int nx = a.nx, nv = a.nv, nch = a.n_chunks;
    const size_t nxnv = (size_t)nx * nv;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int gid = tid / kPstGroup, gt = tid - gid * kPstGroup;
    const int g = blockIdx.x, G = gridDim.x;
    const int bpc = a.bands_per_cta;
    auto band_row = [&](int bi) { return (g + bi * G) * R; };
    const int S = a.stages;
    const int srows = a.span_max + R;                 // staged rows per stage: w window, then own h rows
    float* stages = reinterpret_cast<float*>(smem);
    int4* rinfo = reinterpret_cast<int4*>(stages + (size_t)a.stage_floats);   // [bpc][win_rows]
    int* hinfo = reinterpret_cast<int*>(rinfo + (size_t)bpc * a.win_rows);   // [bpc][R]
    float* red = reinterpret_cast<float*>(hinfo + (((size_t)bpc * R + 3) & ~(size_t)3));
    float* fs = a.fs_alias ? stages : red + kPstWarps * R + 4;
    const size_t ff = ((size_t)2 * nx + a.field_rows + 8 + 3) & ~(size_t)3;
    const int nq = nv / 4;
    PstQuad* sq = ((size_t)nq * sizeof(PstQuad) <= kPstQuadSmemBytes)
                      ? reinterpret_cast<PstQuad*>(a.fs_alias ? red + kPstWarps * R + 4 : fs + ff)
                      : nullptr;
    const int cpg = gid < nch ? (nch - gid + kPstGroups - 1) / kPstGroups : 0;
    const int ntile = bpc * cpg;

    auto quad_of = [&](int q) -> PstQuad {
        PstQuad r;
        const int2 qi = __ldg(a.quad + q);
        r.t = __ldg(a.tq + q);
        r.D = __ldg(reinterpret_cast<const float4*>(a.dfeq) + q);
        r.bm = qi.x;
        r.mask = qi.y;
        r.Dm1 = __ldg(a.dfeq + (q == 0 ? nv - 1 : 4 * q - 1));
        r.pad = 0.f;
        return r;
    };
    if (sq != nullptr)
        for (int q = tid; q < nq; q += blockDim.x) sq[q] = quad_of(q);

    auto h_slot = [&](int n) -> const float* {
        if (n % a.K == 0) return a.ckpt + (size_t)(n / a.K) * nxnv;
        return a.seg + (size_t)(n % a.K - 1) * nxnv;
    };
    auto rinfo_row = [&](int n, int row, float gr) {
        const VShift<float> v = a.vsh_tape[(size_t)n * nx + row];
        int4 r;
        r.x = v.m > nv / 2 ? v.m - nv : v.m;
        r.y = __float_as_int(v.t);
        r.z = __float_as_int(gr);
        r.w = 0;
        return r;
    };
    auto load_rinfo = [&](int n) {   // step n's shifts and grho (global) on every band's window rows
        for (int x = tid; x < bpc * a.win_rows; x += blockDim.x) {
            const int bi = x / a.win_rows, u = x - bi * a.win_rows;
            const int row = pst_wrap(band_row(bi) + a.win_lo + u, nx);
            rinfo[x] = rinfo_row(n, row, __ldcg(a.grho + row));
        }
    };
    auto load_hinfo = [&](int n) {   // step n's signed shifts of the own rows
        for (int x = tid; x < bpc * R; x += blockDim.x) {
            const int bi = x / R, r = x - bi * R;
            const int m = a.vsh_tape[(size_t)n * nx + band_row(bi) + r].m;
            hinfo[x] = m > nv / 2 ? m - nv : m;
        }
    };

    unsigned bar_index = 0;
    bool alive = true;
    auto barrier = [&]() -> bool {
        if (!pst_grid_barrier(a.bar, bar_index++, (unsigned)G, a.wait_ns, a.status, &s_flag)) alive = false;
        return alive;
    };
    auto group_sync = [&]() { asm volatile("bar.sync %0, %1;" ::"r"(1 + gid), "r"(kPstGroup) : "memory"); };

    constexpr int kPieces = kPstW / 4;
    unsigned tiles_issued = 0, tiles_used = 0;
    auto stage_ptr = [&](unsigned k) {
        return stages + (gid * S + (int)(k % (unsigned)S)) * srows * kPstW;
    };
    auto issue = [&](int j, const float* w_src, const float* h_src) {
        const unsigned mine = tiles_issued++;
        const int bi = j / cpg;
        const int c = gid + kPstGroups * (j - bi * cpg);
        const int r0 = band_row(bi), c0 = c * kPstC;
        const int2 cm = __ldg(a.chunk + c);
        const int span = 2 * (cm.y - cm.x) + R + 4;
        const int lo = r0 - 2 * cm.y - 4;             // w window of the chunk
        float* st = stage_ptr(mine);
        for (int p = gt; p < (span + R) * kPieces; p += kPstGroup) {
            const int k = p / kPieces, v = p - k * kPieces;
            int col = c0 - 4 + 4 * v;
            col += col < 0 ? nv : 0;
            col -= col >= nv ? nv : 0;
            const bool wrow = k < span;
            const float* src = wrow ? w_src + (size_t)pst_wrap(lo + k, nx) * nv + col
                                    : h_src + (size_t)(r0 + k - span) * nv + col;
            const int srow = wrow ? k : a.span_max + (k - span);
            pst_cp16(st + (srow * kPstW + 4 * v), src);
        }
        pst_cp_commit();
    };

    auto band_rows = [&](float (&acc)[R], int r0, int n) {
        constexpr int LG = R >= 32 ? 5 : R >= 16 ? 4 : R >= 8 ? 3 : R >= 4 ? 2 : R >= 2 ? 1 : 0;
#pragma unroll
        for (int st = 0; st < LG; ++st) {
            const int o = 16 >> st;
            const int nn = R >> (st + 1);
            const bool upper = (lane & o) != 0;
#pragma unroll
            for (int i = 0; i < (R >> 1); ++i) {
                if (i < nn) {
                    const float send = upper ? acc[i] : acc[i + nn];
                    const float keep = upper ? acc[i + nn] : acc[i];
                    acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
                }
            }
        }
        float v = acc[0];
#pragma unroll
        for (int o = 16 >> LG; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((lane & ((32 >> LG) - 1)) == 0) red[wid * R + (lane >> (5 - LG))] = v;
        __syncthreads();
        if (tid < R) {
            float sum = 0.f;
            for (int w = 0; w < kPstWarps; ++w) sum += red[w * R + tid];
            // tail of step n - 1 for this row (warp_vp_solver/solver.py:870-929)
            const int i = r0 + tid;
            float gEt = a.neg_dt_dv * sum;
            if (a.g_Eh != nullptr) gEt += __ldg(a.g_Eh + (size_t)(n - 1) * nx + i);
            a.g_H[i] += gEt;
            const float gee = a.g_ee != nullptr ? __ldg(a.g_ee + n - 1) : 0.f;
            a.gE[(size_t)(n & 1) * nx + i] = gEt + a.dx * trap_w<float>(i, nx) * __ldg(a.E_tape + (size_t)(n - 1) * nx + i) * gee;
        }
        __syncthreads();
    };

    load_rinfo(a.n_hi);
    load_hinfo(a.n_hi - 1);
    __syncthreads();

    bool pre_issued = false;   // this step's first tiles were issued during the previous field
    for (int n = a.n_hi; n >= a.n_lo && alive; --n) {
        const float* w_src = (n & 1) ? a.wbuf1 : a.wbuf0;
        float* w_dst = (n & 1) ? a.wbuf0 : a.wbuf1;
        const float* h_src = h_slot(n - 1);
        const float* gfh = a.g_fh != nullptr ? a.g_fh + (size_t)(n - 1) * nxnv : nullptr;
        if (!pre_issued)
            for (int j = 0; j < S && j < ntile; ++j) issue(j, w_src, h_src);
        pre_issued = false;

        float acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = 0.f;
        for (int bi = 0; bi < bpc; ++bi) {
            const int r0 = band_row(bi);
            for (int jj = 0; jj < cpg; ++jj) {
                const int j = bi * cpg + jj;
                const int c = gid + kPstGroups * jj;
                const int q = c * kPstGroup + gt;
                const int j0 = c * kPstC + 4 * gt;
                const int2 cm = __ldg(a.chunk + c);
                const PstQuad Q = sq != nullptr ? sq[q] : quad_of(q);
                const float tt[4] = {Q.t.x, Q.t.y, Q.t.z, Q.t.w};
                const float4 D4 = Q.D;
                const float Dm1 = Q.Dm1;
                const float wr0 = j0 == 0 ? -0.5f * a.dv : -a.dv;          // rho^T weights
                const float wr3 = j0 + 3 == nv - 1 ? -0.5f * a.dv : -a.dv;
                pst_cp_wait((int)(tiles_issued - tiles_used - 1));
                group_sync();
                const float* st = stage_ptr(tiles_used);
                ++tiles_used;
                const float* sb = st + (2 * (cm.y - Q.bm) * kPstW + 4 + 4 * gt);   // window row 0
                const float* hb = st + (a.span_max * kPstW + 4 + 4 * gt);            // own row 0
                const int ib = bi * a.win_rows + (-2 * Q.bm - 4 - a.win_lo);
                float GH[4][4], cprev[4];
#pragma unroll
                for (int k = 0; k < R + 4; ++k) {
                    float* o = GH[k & 3];
                    const int4 ri = rinfo[ib + k];
                    const float tv = __int_as_float(ri.y), gr = __int_as_float(ri.z);
                    const float* sr = sb + k * kPstW;
                    float4 v4;
                    if (ri.x == 0) {
                        const float hm = sr[-1];
                        const float4 h = *reinterpret_cast<const float4*>(sr);
                        v4 = make_float4(h.x + tv * (hm - h.x), h.y + tv * (h.x - h.y), h.z + tv * (h.y - h.z),
                                         h.w + tv * (h.z - h.w));
                    } else if (ri.x == -1) {
                        const float4 h = *reinterpret_cast<const float4*>(sr);
                        const float h4 = sr[4];
                        v4 = make_float4(h.y + tv * (h.x - h.y), h.z + tv * (h.y - h.z), h.w + tv * (h.z - h.w),
                                         h4 + tv * (h.w - h4));
                    } else {
                        v4 = pst_vt_rare(sr, w_src, nv, ri.x, tv, pst_wrap(r0 - 2 * Q.bm - 4 + k, nx), j0);
                    }
                    o[0] = v4.x + wr0 * gr;
                    o[1] = v4.y - a.dv * gr;
                    o[2] = v4.z - a.dv * gr;
                    o[3] = v4.w + wr3 * gr;
                    if (k >= 3) {
                        // c row q per column (column shift bm + delta reads window rows q + 2 - 2 delta ..)
                        const int q2 = k - 3;
                        float cn[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const bool dl = (Q.mask >> e) & 1;
                            const float g0 = dl ? GH[q2 & 3][e] : GH[(q2 + 2) & 3][e];
                            const float g1 = dl ? GH[(q2 + 1) & 3][e] : GH[(q2 + 3) & 3][e];
                            cn[e] = pst_lerp(g1, g0, tt[e]);
                            if (gfh != nullptr) {
                                const int row = pst_wrap(r0 - Q.bm - ((Q.mask >> e) & 1) - 1 + q2, nx);
                                cn[e] += __ldg(gfh + (size_t)row * nv + j0 + e);
                            }
                        }
                        if (q2 >= 1) {
                            // w row r = q2 - 1 (own row r0 + r) and its slope products
                            const int r = q2 - 1;
                            float wv[4];
#pragma unroll
                            for (int e = 0; e < 4; ++e) wv[e] = pst_lerp(cn[e], cprev[e], tt[e]);
                            *reinterpret_cast<float4*>(w_dst + (size_t)(r0 + r) * nv + j0) =
                                make_float4(wv[0], wv[1], wv[2], wv[3]);
                            const int ms = hinfo[bi * R + r];
                            const float* hr = hb + r * kPstW;
                            float4 sl;
                            if (ms == 0) {
                                const float4 h = *reinterpret_cast<const float4*>(hr);
                                const float h4 = hr[4];
                                sl = make_float4((h.y - h.x) + D4.x, (h.z - h.y) + D4.y, (h.w - h.z) + D4.z,
                                                 (h4 - h.w) + D4.w);
                            } else if (ms == -1) {
                                const float hm = hr[-1];
                                const float4 h = *reinterpret_cast<const float4*>(hr);
                                sl = make_float4((h.x - hm) + Dm1, (h.y - h.x) + D4.x, (h.z - h.y) + D4.y,
                                                 (h.w - h.z) + D4.z);
                            } else {
                                sl = pst_slope_rare(hr, h_src, a.vtab, a.feq, nv, ms, r0 + r, j0);
                            }
                            acc[r] += sl.x * wv[0] + sl.y * wv[1] + sl.z * wv[2] + sl.w * wv[3];
                        }
#pragma unroll
                        for (int e = 0; e < 4; ++e) cprev[e] = cn[e];
                    }
                }
                group_sync();   // the stage is free
                if (j + S < ntile) issue(j + S, w_src, h_src);
            }
            band_rows(acc, r0, n);
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = 0.f;
        }
        if (!barrier()) break;
        // grho_{n-1} = Poisson^T g_E: on every band's window rows (and the own rows to global), or
        // in slices with a second barrier
        const float* gE = a.gE + (size_t)(n & 1) * nx;
        const bool more = n - 1 >= a.n_lo;
        if (a.field_dist == 0) {
            for (int bi = 0; bi < bpc; ++bi) {
                const int wf = band_row(bi) + a.win_lo;
                if (bi > 0) __syncthreads();
                if (bi == 0 && more && !a.fs_alias) {
                    // the next step's first tiles (w_{n-1} is complete after the barrier) load while
                    // this field is solved
                    pst_field_issue_t(fs, gE, a.ctab, nx, wf, a.win_rows);
                    for (int j = 0; j < S && j < ntile; ++j) issue(j, w_dst, h_slot(n - 2));
                    pre_issued = true;
                    pst_cp_wait((int)(tiles_issued - tiles_used));   // the field group only
                    __syncthreads();
                } else {
                    pst_field_inputs_t(fs, gE, a.ctab, nx, wf, a.win_rows);
                }
                int4* ri = rinfo + (size_t)bi * a.win_rows;
                pst_circ_rows_t(fs, nx, a.win_rows, [&](int u, float v) {
                    const int row = pst_wrap(wf + u, nx);
                    if (more) ri[u] = rinfo_row(n - 1, row, v);
                    const int own = u + a.win_lo;
                    if (own >= 0 && own < R) a.grho[row] = v;
                });
            }
        } else {
            const int Sl = (nx + G - 1) / G;
            const int first = g * Sl;
            const int cnt = max(0, min(Sl, nx - first));
            pst_field_inputs_t(fs, gE, a.ctab, nx, first, cnt);
            pst_circ_rows_t(fs, nx, cnt, [&](int u, float v) { a.grho[first + u] = v; });
            if (more) {
                if (!barrier()) break;
                load_rinfo(n - 1);
            }
        }
        if (more && n - 2 >= 0) load_hinfo(n - 2);
        __syncthreads();
    }
    pst_cp_wait(0);
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------

static const int kPstRows[] = {16, 8, 4};

template <int R>
static cudaError_t pst_set_smem(size_t smem) {
    return cudaFuncSetAttribute(vp_persist_fwd_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int R>
static int pst_max_blocks(size_t smem) {
    int n = 0;
    if (pst_set_smem<R>(smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, vp_persist_fwd_kernel<R>, kPstThreads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

template <int R>
static int pst_bwd_max_blocks(size_t smem) {
    int n = 0;
    if (cudaFuncSetAttribute(vp_persist_bwd_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, vp_persist_bwd_kernel<R>, kPstThreads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

static int pst_bwd_max_blocks_r(int R, size_t smem) {
    switch (R) {
        case 4: return pst_bwd_max_blocks<4>(smem);
        case 8: return pst_bwd_max_blocks<8>(smem);
        case 16: return pst_bwd_max_blocks<16>(smem);
        default: return 0;
    }
}

static int pst_max_blocks_r(int R, size_t smem) {
    switch (R) {
        case 4: return pst_max_blocks<4>(smem);
        case 8: return pst_max_blocks<8>(smem);
        case 16: return pst_max_blocks<16>(smem);
        default: return 0;
    }
}

// Host tables and launch shape of the persistent path for one grid. Returns false when the grid
// is not eligible: nv a multiple of 256, the x shifts of every 4 neighbouring columns within one
// cell of each other, windows shorter than a period.
bool build_quad_tables(int nx, int nv, const std::vector<long long>& m_signed, const std::vector<double>& tx,
                       std::vector<int2>& quad, std::vector<float>& tq, std::vector<int2>& chunk, int chunk_cols) {
    if (chunk_cols % 4 != 0 || nv % chunk_cols != 0 || nx < 8) return false;
    const int nq = nv / 4;
    quad.assign(nq, make_int2(0, 0));
    tq.assign((size_t)4 * nq, 0.f);
    for (int q = 0; q < nq; ++q) {
        long long lo = m_signed[4 * q], hi = lo;
        for (int e = 1; e < 4; ++e) {
            lo = std::min(lo, m_signed[4 * q + e]);
            hi = std::max(hi, m_signed[4 * q + e]);
        }
        if (hi - lo > 1 || 2 * std::llabs(lo) > nx || 2 * std::llabs(hi) > nx) return false;
        int mask = 0;
        for (int e = 0; e < 4; ++e) mask |= (m_signed[4 * q + e] - lo == 1 ? 1 : 0) << e;
        quad[q] = make_int2((int)lo, mask);
        for (int e = 0; e < 4; ++e) tq[(size_t)4 * q + e] = (float)tx[4 * q + e];
    }
    const int nch = nv / chunk_cols, qpc = chunk_cols / 4;
    chunk.assign(nch, make_int2(0, 0));
    for (int c = 0; c < nch; ++c) {
        int lo = 1 << 30, hi = -(1 << 30);
        for (int q = c * qpc; q < (c + 1) * qpc; ++q) {
            lo = std::min(lo, quad[q].x);
            hi = std::max(hi, quad[q].x);
        }
        chunk[c] = make_int2(lo, hi);
    }
    return true;
}

bool persist_prepare(PersistHost& ph, int nx, int nv, const std::vector<long long>& m_signed,
                     const std::vector<double>& tx, int n_sms, int force_rows) {
    ph = PersistHost{};
    if (!build_quad_tables(nx, nv, m_signed, tx, ph.quad, ph.tq, ph.chunk)) return false;
    int all_lo = 1 << 30, all_hi = -(1 << 30), dmax = 0;
    for (const int2& c : ph.chunk) {
        all_lo = std::min(all_lo, c.x);
        all_hi = std::max(all_hi, c.y);
        dmax = std::max(dmax, c.y - c.x);
    }
    // rows per band: the largest R of 16, 8, 4 that gives at least 0.8 bands per SM (or forced)
    int R = 0;
    for (int r : kPstRows) {
        if (nx % r != 0) continue;
        if (force_rows > 0 && r != force_rows) continue;
        R = r;
        if (force_rows > 0 || nx / r >= (4 * n_sms) / 5) break;
    }
    if (R == 0) return false;
    const int span_max = 2 * dmax + R + 4;
    if (span_max > nx) return false;
    const int bands = nx / R;
    // CTAs: bands / bands_per_cta, the smallest bands_per_cta that fits on the device at once
    for (int bpc = 1; bpc <= bands; ++bpc) {
        if (bands % bpc != 0) continue;
        const int G = bands / bpc;
        // the window of a band's tiles (offsets from its first row), widened to cover its own rows
        const int win_lo = std::min(2 * (int)all_lo, 0);
        const int win_end = std::max(R + 2 * (int)all_hi + 4, R);
        const int win_rows = win_end - win_lo;
        if (win_rows > nx - 8) return false;   // the coefficient slices of the fields cover at most nx - 8 rows
        const int fdist = (long long)bpc * win_rows * nx > (1LL << 17) ? 1 : 0;
        const int field_rows = fdist ? (nx + G - 1) / G : win_rows;
        // stages per column group: up to all of the group's tiles of a step, within about 96 KB
        // for the four groups
        const int ntile = bpc * ((nv / kPstC + kPstGroups - 1) / kPstGroups);
        const size_t stage_bytes = (size_t)span_max * kPstW * sizeof(float);
        const int fit = (int)((96 * 1024) / (std::min(kPstGroups, nv / kPstC) * stage_bytes));
        const int stages = std::max(1, std::min({kPstMaxStages, ntile, fit}));
        int stage_floats = 0, fs_alias = 0;
        const size_t smem = persist_smem_bytes(span_max, bpc * win_rows, R, nx, nv, field_rows, stages, &stage_floats,
                                               &fs_alias);
        if (smem > 200 * 1024) continue;
        const int per_sm = pst_max_blocks_r(R, smem);
        if (per_sm <= 0) return false;
        if ((long long)per_sm * n_sms < G) continue;
        ph.R = R;
        ph.G = G;
        ph.bands_per_cta = bpc;
        ph.span_max = span_max;
        ph.win_lo = win_lo;
        ph.win_rows = win_rows;
        ph.smem = smem;
        // the field on each CTA's own window when that costs little, else in slices + a barrier
        ph.field_dist = fdist;
        ph.stage_floats = stage_floats;
        ph.fs_alias = fs_alias;
        ph.stages = stages;
        ph.field_rows = field_rows;
        // the adjoint: window rows r0 - 2m - 4 .. r0 - 2m + R per column quad, widened to the own
        // rows; each stage holds the chunk's window of w and the band's own rows of h_{n-1}
        const int bwin_lo = std::min(-2 * (int)all_hi - 4, 0);
        const int bwin_end = std::max(R - 2 * (int)all_lo, R);
        const int bwin_rows = bwin_end - bwin_lo;
        if (bwin_rows <= nx - 8) {
            const int bfdist = (long long)bpc * bwin_rows * nx > (1LL << 17) ? 1 : 0;
            const int bfield_rows = bfdist ? (nx + G - 1) / G : bwin_rows;
            const int groups = std::min(kPstGroups, nv / kPstC);
            const size_t bstage_bytes = (size_t)(span_max + R) * kPstW * sizeof(float);
            const int bfit = (int)((96 * 1024) / (groups * bstage_bytes));
            const int bstages = std::max(1, std::min({kPstMaxStages, ntile, bfit}));
            const size_t st = (size_t)groups * bstages * (span_max + R) * kPstW;
            const size_t ff = (pst_field_floats(nx, bfield_rows) + 3) & ~(size_t)3;
            const bool alias = ff * sizeof(float) > kPstOwnFieldBytes;
            const size_t area = alias ? std::max(st, ff) : st;
            size_t b = area * sizeof(float) + (size_t)bpc * bwin_rows * 16 + (((size_t)bpc * R + 3) & ~(size_t)3) * 4;
            b += (size_t)kPstWarps * R * sizeof(float) + 16;
            if (!alias) b += ff * sizeof(float);
            const size_t qb = (size_t)(nv / 4) * sizeof(PstQuad);
            if (qb <= kPstQuadSmemBytes) b += qb;
            const int bper_sm = b <= 200 * 1024 ? pst_bwd_max_blocks_r(R, b) : 0;
            if (bper_sm > 0 && (long long)bper_sm * n_sms >= G) {
                ph.bwd_ok = 1;
                ph.bwin_lo = bwin_lo;
                ph.bwin_rows = bwin_rows;
                ph.bstage_floats = (int)area;
                ph.bfs_alias = alias ? 1 : 0;
                ph.bstages = bstages;
                ph.bfield_rows = bfield_rows;
                ph.bfield_dist = bfdist;
                ph.bsmem = b;
            }
        }
        return true;
    }
    return false;
}

cudaError_t launch_persist_fwd(const PersistArgs& args, const PersistHost& ph, cudaStream_t s) {
    PersistArgs a = args;
    a.bands_per_cta = ph.bands_per_cta;
    a.span_max = ph.span_max;
    a.win_lo = ph.win_lo;
    a.win_rows = ph.win_rows;
    a.field_dist = ph.field_dist;
    a.stage_floats = ph.stage_floats;
    a.fs_alias = ph.fs_alias;
    a.stages = ph.stages;
    a.field_rows = ph.field_rows;
    cudaError_t e = cudaMemsetAsync(a.bar, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ph.G, 1, 1);
    cfg.blockDim = dim3(kPstThreads, 1, 1);
    cfg.dynamicSmemBytes = ph.smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    switch (ph.R) {
        case 4: e = cudaLaunchKernelEx(&cfg, vp_persist_fwd_kernel<4>, a); break;
        case 8: e = cudaLaunchKernelEx(&cfg, vp_persist_fwd_kernel<8>, a); break;
        case 16: e = cudaLaunchKernelEx(&cfg, vp_persist_fwd_kernel<16>, a); break;
        default: return cudaErrorInvalidValue;
    }
    count_launch();
    return e;
}

cudaError_t launch_persist_bwd(const PersistBwdArgs& args, const PersistHost& ph, cudaStream_t s) {
    if (!ph.bwd_ok) return cudaErrorInvalidValue;
    PersistBwdArgs a = args;
    a.bands_per_cta = ph.bands_per_cta;
    a.span_max = ph.span_max;
    a.win_lo = ph.bwin_lo;
    a.win_rows = ph.bwin_rows;
    a.field_dist = ph.bfield_dist;
    a.stage_floats = ph.bstage_floats;
    a.fs_alias = ph.bfs_alias;
    a.stages = ph.bstages;
    a.field_rows = ph.bfield_rows;
    cudaError_t e = cudaMemsetAsync(a.bar, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ph.G, 1, 1);
    cfg.blockDim = dim3(kPstThreads, 1, 1);
    cfg.dynamicSmemBytes = ph.bsmem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    switch (ph.R) {
        case 4: e = cudaLaunchKernelEx(&cfg, vp_persist_bwd_kernel<4>, a); break;
        case 8: e = cudaLaunchKernelEx(&cfg, vp_persist_bwd_kernel<8>, a); break;
        case 16: e = cudaLaunchKernelEx(&cfg, vp_persist_bwd_kernel<16>, a); break;
        default: return cudaErrorInvalidValue;
    }
    count_launch();
    return e;
}

}  // namespace vpb
