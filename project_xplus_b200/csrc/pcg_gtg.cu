// pcg_gtg.cu -- persistent PCG with the factorized preconditioner M^-1 = G^T G (G lower-
// triangular on A's lower pattern in the matrix's given order, e.g. predicted by the learned
// network of gnn.cu).  Applying M^-1 is two more sliced SpMVs and no triangular solve.
//
// One cooperative launch, one 512-thread CTA per SM, contiguous slice ranges per CTA as in
// pcg_kernels.cu.  Per iteration three grid barriers:
//   A   p' = z + beta p (neighbours recomputed from their {z, p} records), Ap', p'.Ap'
//   BC  x += alpha p' (FP64), r' = r - alpha Ap' (into the other r buffer), r'.r' partial,
//       t_i = sum_j G_ij r'_j with every neighbour's r'_j recomputed from its r_j and Ap'_j by
//       the same fused multiply-add as the owner's, so t needs no barrier of its own
//   D   z = G^T t, record z, r'.z partial
// FP64 residual replacement as in pcg_kernels.cu (the refreshed r is preconditioned by two
// more phases).  Jacobi fallback inside the launch: when the learned preconditioner stagnates
// (8 replacements without a 10% gain of the true residual) or passes the iteration cap, the
// kernel switches to z = M^-1 r with the Jacobi inverse, refreshes r from x in FP64 and
// restarts the search direction; the iteration of the switch is reported.
// Control flow, breakdown tests and status codes: kernels/cuper_pcg_control_kernel.cpp:1069-1235.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "../../include/xplus_b200.h"
#include "device_common.cuh"
#include "pcg_device.cuh"
#include "pcg_kernels.cuh"

namespace xplus {
namespace {

using namespace dev;

constexpr int kGtgSlices = 1024;  // slice table capacity per CTA
constexpr int kGChunk = 2;        // G / G^T SELL chunk (FP32 values, int32 columns)

// NB rows (32 sl[k] + lane) of G or G^T in SELL form times x (sl[k] < 0: no row); st is the
// CTA's shared slice table {first slot, width} starting at slice s_first.  With RECOMP the
// operand is r'_j = fma(-alpha, Ap'_j, r_j), recomputed exactly as the owner of row j
// computes it.  The slot loads of all
// rows are issued first, then all the gathers, then the arithmetic, so a warp keeps
// NB * 2 * kGChunk loads in flight instead of walking its slices one dependent chain at a time.
template <int NB, bool RECOMP>
__device__ __forceinline__ void g_rows(const int2* __restrict__ st, int s_first, const int* __restrict__ col,
                                       const float* __restrict__ val, const int (&sl)[NB], int lane, const float* x,
                                       const float* ap, float nal, float (&out)[NB]) {
    int base[NB], w[NB], wmax = 0;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        out[k] = 0.0f;
        const int2 e = sl[k] >= 0 ? st[sl[k] - s_first] : make_int2(0, 0);
        base[k] = e.x;
        w[k] = e.y;
        wmax = max(wmax, w[k]);
    }
    // two chunk steps per pass: every slot load of both steps before any gather, so a row of
    // up to 2 * kGChunk entries costs one load-then-gather round trip instead of two (the
    // products still add in slot order, as one step at a time would)
    for (int c = 0; c < wmax; c += 2 * kGChunk) {
        float2 v[NB][2];
        int2 cc[NB][2];
#pragma unroll
        for (int k = 0; k < NB; ++k)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (c + h * kGChunk < w[k]) {
                    const int off = base[k] + (c + h * kGChunk) * 32 + lane * kGChunk;
                    v[k][h] = __ldg(reinterpret_cast<const float2*>(val + off));
                    cc[k][h] = __ldg(reinterpret_cast<const int2*>(col + off));
                } else {
                    v[k][h] = make_float2(0.0f, 0.0f);
                    cc[k][h] = make_int2(-1, -1);
                }
            }
        float x0[NB][2], x1[NB][2];
#pragma unroll
        for (int k = 0; k < NB; ++k)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                x0[k][h] = cc[k][h].x >= 0 ? x[cc[k][h].x] : 0.0f;
                x1[k][h] = cc[k][h].y >= 0 ? x[cc[k][h].y] : 0.0f;
                if (RECOMP) {
                    if (cc[k][h].x >= 0) x0[k][h] = __fmaf_rn(nal, ap[cc[k][h].x], x0[k][h]);
                    if (cc[k][h].y >= 0) x1[k][h] = __fmaf_rn(nal, ap[cc[k][h].y], x1[k][h]);
                }
            }
#pragma unroll
        for (int k = 0; k < NB; ++k)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                out[k] = fmaf(v[k][h].x, x0[k][h], out[k]);
                out[k] = fmaf(v[k][h].y, x1[k][h], out[k]);
            }
    }
}

constexpr int kGRows = 4;  // G rows of one warp in flight

template <typename VT, int CHUNK, typename IT>
__global__ void __launch_bounds__(512, 1) pcg_gtg_kernel(PcgArgs a) {
    constexpr int NS = 2;
    __shared__ double s_red[32 * 4];
    __shared__ double s_tot[4];
    __shared__ int s_flag;
    __shared__ int2 s_slice[kGtgSlices];
    __shared__ int2 s_gslice[kGtgSlices];   // G and G^T slice tables {first slot, width}
    __shared__ int2 s_gtslice[kGtgSlices];
    __shared__ long long s_clk[6];
    GridBarrier bar{a.bar, a.err, a.timeout_ns, 0u, a.debug_skip_block};
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int per_block = (a.n_slices + gridDim.x - 1) / gridDim.x;
    const int sb = blockIdx.x * per_block;
    const int se = min(a.n_slices, sb + per_block);
    const VT* __restrict__ val = static_cast<const VT*>(a.val);
    const float* __restrict__ minv = static_cast<const float*>(a.minv);
    const float* __restrict__ rowsum = static_cast<const float*>(a.rowsum);
    const float* __restrict__ gval = static_cast<const float*>(a.g_val);
    const float* __restrict__ gtval = static_cast<const float*>(a.gt_val);
    NodeRec<float>* rec = static_cast<NodeRec<float>*>(a.rec);
    float* ap = static_cast<float*>(a.ap);
    float* r_cur = static_cast<float*>(a.r);
    float* r_nxt = static_cast<float*>(a.r2);
    float* t = static_cast<float*>(a.t);
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const bool true_mode = a.tau_true_rr >= 0.0;
    for (int k = threadIdx.x; k < se - sb; k += blockDim.x) {
        const long long b0 = a.slice_ptr[sb + k];
        s_slice[k] = make_int2(static_cast<int>(b0), static_cast<int>((a.slice_ptr[sb + k + 1] - b0) >> 5));
        const long long g0 = a.g_slice_ptr[sb + k];
        s_gslice[k] = make_int2(static_cast<int>(g0), static_cast<int>((a.g_slice_ptr[sb + k + 1] - g0) >> 5));
        const long long t0 = a.gt_slice_ptr[sb + k];
        s_gtslice[k] = make_int2(static_cast<int>(t0), static_cast<int>((a.gt_slice_ptr[sb + k + 1] - t0) >> 5));
    }
    // phase clock (per CTA, thread 0): {A work, grid-barrier waits, BC work, D work}
    if (threadIdx.x == 0) {
        for (int k = 0; k < 5; ++k) s_clk[k] = 0;
        s_clk[5] = globaltimer_ns();
        if (lead) a.out->t_start_ns = s_clk[5];
    }
    __syncthreads();
    auto clock = [&](int slot) {
        if (threadIdx.x == 0) {
            const long long t = globaltimer_ns();
            s_clk[slot] += t - s_clk[5];
            s_clk[5] = t;
        }
    };
    int bank = 0;
    auto next_bank = [&]() {
        double* b = a.partial + static_cast<size_t>(bank) * 4 * gridDim.x;
        bank ^= 1;
        return b;
    };
    double* cur_bank = nullptr;
    bool jac = false;
    int fell_back = -1;

    // r = b - A x in FP64 (stored rounded); with Jacobi also z = M^-1 r into the record.
    // Partials: r.z (Jacobi only), r.r, ||b - A x||^2, and ||b||^2 in the first pass or
    // z_new . Ap' at a replacement (Jacobi only).
    auto residual_phase = [&](bool init) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int s = sb + warp; s < se; s += wpb) {
            const int row = s * 32 + lane;
            const double y = row_fp64<VT, float, CHUNK, true, IT>(a, s, lane, row);
            const double bv = a.b64[row];
            const double rt = bv - y;
            if (init) acc[3] += bv * bv;
            const float rv = static_cast<float>(rt);
            r_cur[row] = rv;
            if (jac) {
                const float zv = minv[row] * rv;
                if (init) {
                    store_rec(rec + row, zv, 0.0f);
                } else {
                    rec[row].z = zv;
                    acc[3] += static_cast<double>(zv) * static_cast<double>(ap[row]);
                }
                acc[0] += static_cast<double>(rv) * static_cast<double>(zv);
            } else if (init) {
                store_rec(rec + row, 0.0f, 0.0f);
            }
            acc[1] += static_cast<double>(rv) * static_cast<double>(rv);
            acc[2] += rt * rt;
        }
        cur_bank = next_bank();
        publish<4>(acc, s_red, cur_bank);
    };
    // z = G^T t into the record, partials r.z (r = r_cur) and, with zap_too (a replacement), z.Ap'
    auto z_phase = [&](bool zap_too) {
        double acc[2] = {0.0, 0.0};
        for (int s0 = sb + warp; s0 < se; s0 += kGRows * wpb) {
            int sl[kGRows];
            float zv[kGRows], rv[kGRows];
#pragma unroll
            for (int k = 0; k < kGRows; ++k) {
                const int s = s0 + k * wpb;
                sl[k] = s < se ? s : -1;
                rv[k] = s < se ? r_cur[s * 32 + lane] : 0.0f;
            }
            g_rows<kGRows, false>(s_gtslice, sb, a.gt_col, gtval, sl, lane, t, nullptr, 0.0f, zv);
#pragma unroll
            for (int k = 0; k < kGRows; ++k) {
                if (sl[k] < 0) continue;
                rec[sl[k] * 32 + lane].z = zv[k];
                acc[0] += static_cast<double>(rv[k]) * static_cast<double>(zv[k]);
                if (zap_too) acc[1] += static_cast<double>(zv[k]) * static_cast<double>(ap[sl[k] * 32 + lane]);
            }
        }
        cur_bank = next_bank();
        publish<2>(acc, s_red, cur_bank);
    };
    double rz = 0.0, rr = 0.0, true_rr = 0.0, bb = 0.0, zap = 0.0;
    // FP64 residual and its preconditioning (the first one also sums ||b||^2); false when
    // a barrier gave up
    auto refresh = [&](bool init) -> bool {
        residual_phase(init);
        if (!bar.sync(&s_flag)) return false;
        grid_totals(cur_bank, 4, s_tot);
        rz = s_tot[0];
        rr = s_tot[1];
        true_rr = s_tot[2];
        if (init) bb = s_tot[3];
        else zap = s_tot[3];
        if (!jac) {
            for (int s0 = sb + warp; s0 < se; s0 += kGRows * wpb) {
                int sl[kGRows];
                float tv[kGRows];
#pragma unroll
                for (int k = 0; k < kGRows; ++k) sl[k] = s0 + k * wpb < se ? s0 + k * wpb : -1;
                g_rows<kGRows, false>(s_gslice, sb, a.g_col, gval, sl, lane, r_cur, nullptr, 0.0f, tv);
#pragma unroll
                for (int k = 0; k < kGRows; ++k)
                    if (sl[k] >= 0) t[sl[k] * 32 + lane] = tv[k];
            }
            if (!bar.sync(&s_flag)) return false;
            z_phase(!init);
            if (!bar.sync(&s_flag)) return false;
            grid_totals(cur_bank, 2, s_tot);
            rz = s_tot[0];
            if (!init) zap = s_tot[1];
        }
        return true;
    };

    if (!refresh(true)) return;
    const double tau_true_rr = a.tau2_rel > 0.0 ? a.tau2_rel * bb : a.tau_true_rr;
    if (lead) a.out->bb = bb;
    double rr_at_replace = rr;
    double pap = 0.0, alpha = 0.0, beta = 0.0;
    int status = XPLUS_MAX_ITER, iterations = 0, replacements = 0, stagnated = 0;
    ReplacePolicy pol(a.restart_on_replace, true_rr);
    const bool converged_now = true_mode ? (true_rr <= tau_true_rr) : (rr <= a.tau_rr);

    if (converged_now) {
        status = XPLUS_CONVERGED;
    } else {
        for (int it = 0; it < a.max_iters; ++it) {
            if (bad(rz) || bad(rr) || fabs(rz) <= kBreakdownEps) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            const float be = static_cast<float>(beta);
            // ---- A: p', Ap', p'.Ap' ----
            {
                double acc[1] = {0.0};
                for (int s0 = sb + warp; s0 < se; s0 += NS * wpb) {
                    int2 sl[NS];
                    int row[NS];
                    float pi[NS], y[NS];
#pragma unroll
                    for (int k = 0; k < NS; ++k) {
                        const int s = s0 + k * wpb;
                        const bool on = s < se;
                        sl[k] = on ? s_slice[s - sb] : make_int2(0, 0);
                        row[k] = on ? s * 32 + lane : -1;
                    }
#pragma unroll
                    for (int k = 0; k < NS; ++k) {
                        const NodeRec<float> me = row[k] >= 0 ? load_rec(rec + row[k]) : NodeRec<float>{0.0f, 0.0f};
                        pi[k] = node_pnew(me.z, be, me.p);
                    }
                    sell_rows_pnew<VT, CHUNK, true, IT, float, NS>(sl, row, lane, static_cast<const IT*>(a.col), val, rec,
                                                                   be, pi, y);
#pragma unroll
                    for (int k = 0; k < NS; ++k) {
                        if (row[k] < 0) continue;
                        y[k] = y[k] * a.val_scale + rowsum[row[k]] * pi[k];
                        ap[row[k]] = y[k];
                        acc[0] += static_cast<double>(pi[k]) * static_cast<double>(y[k]);
                    }
                }
                cur_bank = next_bank();
                publish<1>(acc, s_red, cur_bank);
            }
            clock(0);
            if (!bar.sync(&s_flag)) return;
            clock(1);
            grid_totals(cur_bank, 1, s_tot);
            pap = s_tot[0];
            if (bad(pap) || fabs(pap) <= kBreakdownEps) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            const double rz_old = rz;
            alpha = rz / pap;
            if (bad(alpha)) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            // ---- BC: x, r' (other buffer), r'.r'; t = G r' (or z = M^-1 r' with Jacobi) ----
            double rz_new = 0.0, rr_new = 0.0;
            {
                double acc[2] = {0.0, 0.0};
                const float nal = -static_cast<float>(alpha);
                for (int s0 = sb + warp; s0 < se; s0 += kGRows * wpb) {
                    int sl[kGRows];
                    NodeRec<float> me[kGRows];
                    float apv[kGRows], rv[kGRows];
                    double xv[kGRows];
#pragma unroll
                    for (int k = 0; k < kGRows; ++k) {
                        const int s = s0 + k * wpb;
                        sl[k] = s < se ? s : -1;
                        const int row = (s < se ? s : s0) * 32 + lane;
                        me[k] = load_rec(rec + row);
                        apv[k] = ap[row];
                        rv[k] = r_cur[row];
                        xv[k] = a.x64[row];
                    }
#pragma unroll
                    for (int k = 0; k < kGRows; ++k) {
                        if (sl[k] < 0) continue;
                        const int row = sl[k] * 32 + lane;
                        const float pv = node_pnew(me[k].z, be, me[k].p);
                        a.x64[row] = xv[k] + alpha * static_cast<double>(pv);
                        const float rn = __fmaf_rn(nal, apv[k], rv[k]);
                        r_nxt[row] = rn;
                        if (jac) {
                            const float zv = minv[row] * rn;
                            store_rec(rec + row, zv, pv);
                            acc[0] += static_cast<double>(rn) * static_cast<double>(zv);
                        } else {
                            rec[row].p = pv;
                        }
                        acc[1] += static_cast<double>(rn) * static_cast<double>(rn);
                    }
                    if (!jac) {
                        float tv[kGRows];
                        g_rows<kGRows, true>(s_gslice, sb, a.g_col, gval, sl, lane, r_cur, ap, nal, tv);
#pragma unroll
                        for (int k = 0; k < kGRows; ++k)
                            if (sl[k] >= 0) t[sl[k] * 32 + lane] = tv[k];
                    }
                }
                cur_bank = next_bank();
                publish<2>(acc, s_red, cur_bank);
            }
            clock(2);
            if (!bar.sync(&s_flag)) return;
            clock(1);
            grid_totals(cur_bank, 2, s_tot);
            rz_new = s_tot[0];
            rr_new = s_tot[1];
            {
                float* tmp = r_cur;
                r_cur = r_nxt;
                r_nxt = tmp;
            }
            if (!jac) {
                // ---- D: z = G^T t, r'.z ----
                z_phase(false);
                clock(3);
                if (!bar.sync(&s_flag)) return;
                clock(1);
                grid_totals(cur_bank, 1, s_tot);
                rz_new = s_tot[0];
            }
            iterations = it + 1;
            if (bad(rz_new) || bad(rr_new)) {
                rz = rz_new;
                rr = rr_new;
                status = XPLUS_BREAKDOWN;
                break;
            }
            bool do_replace = false, drop_replace = false, restart = false;
            if (true_mode) {
                if (rr_new <= tau_true_rr) do_replace = drop_replace = true;
                if (a.replace_every > 0 && iterations % a.replace_every == 0) do_replace = true;
                if (a.replace_drop > 0.0 && rr_new <= a.replace_drop * rr_at_replace) do_replace = drop_replace = true;
            }
            // Jacobi fallback: the learned preconditioner stagnated or used up its iterations
            if (!jac && (stagnated || (a.g_fallback_iters > 0 && iterations >= a.g_fallback_iters))) {
                jac = true;
                fell_back = iterations;
                stagnated = 0;
                pol.stagnant = 0;
                do_replace = true;
                restart = true;
            }
            if (do_replace) {
                if (!refresh(false)) return;
                rz_new = rz;
                rr_new = rr;
                ++replacements;
                rr_at_replace = rr_new;
                if (restart) {
                    // the switch to Jacobi: the refreshed residual is the new reference
                    if (a.restart_on_replace == 3 && pol.mode == 2 && true_rr > 4.0 * pol.best) pol.mode = 1;
                    pol.best = true_rr;
                } else if (pol.after(a.restart_on_replace, true_rr, a.stag_factor, a.stag_window)) {
                    stagnated = 1;
                }
            }
            if (lead && a.trace && it < a.trace_cap) {
                double* tr = a.trace + 5 * static_cast<size_t>(it);
                tr[0] = alpha;
                tr[1] = rz_new / rz_old;
                tr[2] = rz_new;
                tr[3] = rr_new;
                tr[4] = sqrt(rr_new > 0.0 ? rr_new : 0.0);
            }
            rz = rz_new;
            rr = rr_new;
            if (true_mode ? (do_replace && true_rr <= tau_true_rr) : (rr <= a.tau_rr)) {
                status = XPLUS_CONVERGED;
                break;
            }
            if (stagnated && jac) break;
            if (fabs(rz_old) <= kBreakdownEps) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            beta = restart ? 0.0 : pol.beta(do_replace, drop_replace, rz, rz_old, zap, pap);
            if (bad(beta)) {
                status = XPLUS_BREAKDOWN;
                break;
            }
        }
    }
    if (status == XPLUS_MAX_ITER && !true_mode && rr <= a.tau_rr) status = XPLUS_CONVERGED;

    // exit: FP64 true residual of the final x
    {
        double acc[1] = {0.0};
        for (int s = sb + warp; s < se; s += wpb) {
            const int row = s * 32 + lane;
            const double y = row_fp64<VT, float, CHUNK, true, IT>(a, s, lane, row);
            const double rt = a.b64[row] - y;
            acc[0] += rt * rt;
        }
        cur_bank = next_bank();
        publish<1>(acc, s_red, cur_bank);
    }
    if (threadIdx.x == 0 && a.block_clk)
        for (int k = 0; k < 4; ++k) a.block_clk[4 * static_cast<size_t>(blockIdx.x) + k] = s_clk[k];
    if (!bar.sync(&s_flag)) return;
    if (blockIdx.x == 0) {
        grid_totals(cur_bank, 1, s_tot);
        if (threadIdx.x == 0) {
            PcgOut* o = a.out;
            o->status = status;
            o->iterations = iterations;
            o->replacements = replacements;
            o->stagnated = stagnated;
            o->rz = rz;
            o->rr = rr;
            o->pap = pap;
            o->alpha = alpha;
            o->true_rr = s_tot[0];
            o->reserved = static_cast<double>(fell_back);
            o->t_end_ns = globaltimer_ns();
            for (int k = 0; k < 4; ++k) o->t_phase[k] = s_clk[k];
        }
    }
}

using GtgKernel = void (*)(PcgArgs);

template <typename VT, typename IT>
GtgKernel gtg_pick_chunk(int chunk) {
    switch (chunk) {
        case 1: return pcg_gtg_kernel<VT, 1, IT>;
        case 2: return pcg_gtg_kernel<VT, 2, IT>;
        case 4: return pcg_gtg_kernel<VT, 4, IT>;
    }
    return nullptr;
}

GtgKernel gtg_kernel(const KernelKey& k) {
    if (k.xt != XPLUS_F32 || !k.diag) return nullptr;
    switch (k.vt) {
        case XPLUS_F32: return k.idx16 ? gtg_pick_chunk<float, short>(k.chunk) : gtg_pick_chunk<float, int>(k.chunk);
        case XPLUS_F16: return k.idx16 ? gtg_pick_chunk<__half, short>(k.chunk) : gtg_pick_chunk<__half, int>(k.chunk);
        case XPLUS_BF16:
            return k.idx16 ? gtg_pick_chunk<__nv_bfloat16, short>(k.chunk) : gtg_pick_chunk<__nv_bfloat16, int>(k.chunk);
    }
    return nullptr;
}

__global__ void k_gtg_fill(const double* __restrict__ glow, const int* __restrict__ map, float* __restrict__ val,
                           long long slots) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q < slots) {
        const int m = map[q];
        val[q] = m >= 0 ? static_cast<float>(glow[m]) : 0.0f;
    }
}

}  // namespace

cudaError_t gtg_fill_values(const double* d_glow, const int* d_map, float* d_val, long long slots, cudaStream_t s) {
    k_gtg_fill<<<static_cast<unsigned>((slots + 255) / 256), 256, 0, s>>>(d_glow, d_map, d_val, slots);
    return cudaGetLastError();
}

cudaError_t gtg_grid(const KernelKey& k, int device, int n_slices, int* grid, int* tpb) {
    GtgKernel f = gtg_kernel(k);
    if (!f) return cudaErrorInvalidValue;
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, 512, 0);
    if (e != cudaSuccess) return e;
    if (per_sm <= 0) return cudaErrorInvalidConfiguration;
    int blocks = per_sm * sms;
    const int need = (n_slices + 15) / 16;
    if (blocks > need) blocks = need > 0 ? need : 1;
    if ((n_slices + blocks - 1) / blocks > kGtgSlices) return cudaErrorInvalidConfiguration;
    *grid = blocks;
    *tpb = 512;
    return cudaSuccess;
}

cudaError_t gtg_launch(const KernelKey& k, const PcgArgs& a, int grid, int tpb, cudaStream_t s,
                       const cudaAccessPolicyWindow& window) {
    GtgKernel f = gtg_kernel(k);
    if (!f) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(tpb);
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    int na = 0;
    attr[na].id = cudaLaunchAttributeCooperative;
    attr[na].val.cooperative = 1;
    ++na;
    if (window.num_bytes > 0) {
        attr[na].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[na].val.accessPolicyWindow = window;
        ++na;
    }
    cfg.attrs = attr;
    cfg.numAttrs = na;
    return cudaLaunchKernelEx(&cfg, f, a);
}

}  // namespace xplus
