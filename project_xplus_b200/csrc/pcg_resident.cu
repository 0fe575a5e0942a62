// pcg_resident.cu -- the SM-resident persistent Jacobi-PCG kernel (FP32 vectors, row-sum form).
//
// One CTA per SM owns a contiguous band of rows [R0, R0 + nb).  Every iteration it copies the
// records {z, p} of its band plus the bandwidth halo [W0, W0 + wn) into shared memory as the
// new search direction p' = z + beta p, so the SpMV gathers p' from shared memory and the only
// global stream of phase A is the matrix itself.  The per-row state that no other CTA reads --
// r, Ap, the FP32 solution increment dx, M^-1 and the row sums -- lives in shared memory for
// the whole solve; dx is folded into the FP64 solution x every `flush_every` iterations and
// before every FP64 residual (which needs x of neighbouring rows).  Two grid barriers per
// iteration, as in the global-memory kernel (pcg_kernels.cu), with the same control flow,
// breakdown tests and status codes (kernels/cuper_pcg_control_kernel.cpp:1069-1235).
// pcg_resident1_kernel below needs one grid barrier per iteration instead of two.
//
// Shared memory (floats): pw[wn] | r[nb] | ap[nb] | dx[nb] | minv[nb] | rowsum[nb].
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

constexpr int kResSlices = 1024;  // slice table capacity per CTA
constexpr int kResNS = 4;         // slices of one warp in flight together in phase A

template <typename VT, int CHUNK, typename IT>
__global__ void __launch_bounds__(512, 1) pcg_resident_kernel(PcgArgs a) {
    constexpr int NS = kResNS;
    extern __shared__ float smem[];
    __shared__ double s_red[32 * 4];
    __shared__ double s_tot[4];
    __shared__ int s_flag;
    __shared__ int2 s_slice[kResSlices];
    __shared__ long long s_clk[6];
    GridBarrier bar{a.bar, a.err, a.timeout_ns, 0u, a.debug_skip_block};
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int per_block = (a.n_slices + gridDim.x - 1) / gridDim.x;
    const int sb = blockIdx.x * per_block;
    const int se = min(a.n_slices, sb + per_block);
    const int r0 = sb * 32;
    const int nb = max(0, se - sb) * 32;
    const int2 win = a.win[blockIdx.x];
    const int w0 = win.x, wn = win.y;
    float* pw = smem;
    float* rv = pw + wn;
    float* apv = rv + nb;
    float* dxv = apv + nb;
    float* mi = dxv + nb;
    float* rsv = mi + nb;
    const VT* __restrict__ val = static_cast<const VT*>(a.val);
    const IT* __restrict__ col = static_cast<const IT*>(a.col);
    const float* __restrict__ minv_g = static_cast<const float*>(a.minv);
    const float* __restrict__ rowsum_g = static_cast<const float*>(a.rowsum);
    NodeRec<float>* rec = static_cast<NodeRec<float>*>(a.rec);
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const bool true_mode = a.tau_true_rr >= 0.0;
    for (int k = threadIdx.x; k < se - sb; k += blockDim.x) {
        const long long b0 = a.slice_ptr[sb + k];
        s_slice[k] = make_int2(static_cast<int>(b0), static_cast<int>((a.slice_ptr[sb + k + 1] - b0) >> 5));
    }
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
        mi[t] = minv_g[r0 + t];
        rsv[t] = rowsum_g[r0 + t];
        dxv[t] = 0.0f;
    }
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

    // x += dx for the band (FP64 accumulation of the FP32 increments), dx = 0
    auto flush_dx = [&]() {
        for (int t = threadIdx.x; t < nb; t += blockDim.x) {
            a.x64[r0 + t] += static_cast<double>(dxv[t]);
            dxv[t] = 0.0f;
        }
    };

    // ---- residual phase: r = b - A x in FP64 (x of neighbours from global memory), rounded
    //      into shared r; z = M^-1 r into the record (init also clears p) ----
    auto residual_phase = [&](bool init) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int s = sb + warp; s < se; s += wpb) {
            const int row = s * 32 + lane;
            const double y = row_fp64<VT, float, CHUNK, true, IT>(a, s, lane, row);
            const double bv = a.b64[row];
            const double rt = bv - y;
            const float r_ = static_cast<float>(rt);
            const float z_ = mi[row - r0] * r_;
            // slot 3: ||b||^2 in the first pass, z_new . Ap' at a replacement
            acc[3] += init ? bv * bv : static_cast<double>(z_) * static_cast<double>(apv[row - r0]);
            rv[row - r0] = r_;
            if (init) store_rec(rec + row, z_, 0.0f);
            else rec[row].z = z_;
            acc[0] += static_cast<double>(r_) * static_cast<double>(z_);
            acc[1] += static_cast<double>(r_) * static_cast<double>(r_);
            acc[2] += rt * rt;
        }
        cur_bank = next_bank();
        publish<4>(acc, s_red, cur_bank);
    };

    residual_phase(true);
    if (!bar.sync(&s_flag)) return;
    grid_totals(cur_bank, 4, s_tot);
    double rz = s_tot[0], rr = s_tot[1], true_rr = s_tot[2];
    const double tau_true_rr = a.tau2_rel > 0.0 ? a.tau2_rel * s_tot[3] : a.tau_true_rr;
    if (lead) a.out->bb = s_tot[3];
    double rr_at_replace = rr;
    double pap = 0.0, alpha = 0.0, beta = 0.0;
    int status = XPLUS_MAX_ITER, iterations = 0, replacements = 0, stagnated = 0;
    ReplacePolicy pol(a.restart_on_replace, true_rr);
    const bool converged_now = true_mode ? (true_rr <= tau_true_rr) : (rr <= a.tau_rr);
    const int flush_every = a.flush_every > 0 ? a.flush_every : 16;
    clock(4);

    if (converged_now) {
        status = XPLUS_CONVERGED;
    } else {
        for (int it = 0; it < a.max_iters; ++it) {
            if (bad(rz) || bad(rr) || fabs(rz) <= kBreakdownEps) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            const float be = static_cast<float>(beta);
            // ---- phase A: window p' = z + beta p, then Ap' from shared memory ----
            {
                for (int t = threadIdx.x; t < wn; t += blockDim.x) {
                    const NodeRec<float> nr = load_rec(rec + w0 + t);
                    pw[t] = node_pnew(nr.z, be, nr.p);
                }
                __syncthreads();
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
                        pi[k] = on ? pw[row[k] - w0] : 0.0f;
                    }
                    sell_rows_smem<VT, CHUNK, IT, NS>(sl, row, lane, col, val, pw, w0, pi, y);
#pragma unroll
                    for (int k = 0; k < NS; ++k) {
                        if (row[k] < 0) continue;
                        const int t = row[k] - r0;
                        const float yy = y[k] * a.val_scale + rsv[t] * pi[k];
                        apv[t] = yy;
                        acc[0] += static_cast<double>(pi[k]) * static_cast<double>(yy);
                    }
                }
                cur_bank = next_bank();
                publish<1>(acc, s_red, cur_bank);
            }
            clock(0);
            if (!bar.sync(&s_flag)) return;
            grid_totals(cur_bank, 1, s_tot);
            clock(1);
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
            // ---- phase B: dx += alpha p', r -= alpha Ap', z = M^-1 r, record {z, p'} ----
            {
                double acc[2] = {0.0, 0.0};
                const float al = static_cast<float>(alpha);
                const bool flush = (it + 1) % flush_every == 0;
                for (int t = threadIdx.x; t < nb; t += blockDim.x) {
                    const float pv = pw[r0 + t - w0];
                    const float d = __fmaf_rn(al, pv, dxv[t]);
                    const float r_ = rv[t] - al * apv[t];
                    const float z_ = mi[t] * r_;
                    rv[t] = r_;
                    if (flush) {
                        a.x64[r0 + t] += static_cast<double>(d);
                        dxv[t] = 0.0f;
                    } else {
                        dxv[t] = d;
                    }
                    store_rec(rec + r0 + t, z_, pv);
                    acc[0] += static_cast<double>(r_) * static_cast<double>(z_);
                    acc[1] += static_cast<double>(r_) * static_cast<double>(r_);
                }
                cur_bank = next_bank();
                publish<2>(acc, s_red, cur_bank);
            }
            clock(2);
            if (!bar.sync(&s_flag)) return;
            grid_totals(cur_bank, 2, s_tot);
            clock(3);
            double rz_new = s_tot[0], rr_new = s_tot[1];
            iterations = it + 1;
            if (bad(rz_new) || bad(rr_new)) {
                rz = rz_new;
                rr = rr_new;
                status = XPLUS_BREAKDOWN;
                break;
            }
            bool do_replace = false, drop_replace = false;
            double zap = 0.0;  // z_new . Ap' of a replacement
            if (true_mode) {
                if (rr_new <= tau_true_rr) do_replace = drop_replace = true;
                if (a.replace_every > 0 && iterations % a.replace_every == 0) do_replace = true;
                if (a.replace_drop > 0.0 && rr_new <= a.replace_drop * rr_at_replace) do_replace = drop_replace = true;
            }
            if (do_replace) {
                flush_dx();
                if (!bar.sync(&s_flag)) return;
                residual_phase(false);
                if (!bar.sync(&s_flag)) return;
                grid_totals(cur_bank, 4, s_tot);
                clock(4);
                rz_new = s_tot[0];
                rr_new = s_tot[1];
                true_rr = s_tot[2];
                zap = s_tot[3];
                ++replacements;
                rr_at_replace = rr_new;
                if (pol.after(a.restart_on_replace, true_rr, a.stag_factor, a.stag_window)) stagnated = 1;
            }
            if (lead && a.trace && it < a.trace_cap) {
                double* t = a.trace + 5 * static_cast<size_t>(it);
                t[0] = alpha;
                t[1] = rz_new / rz_old;
                t[2] = rz_new;
                t[3] = rr_new;
                t[4] = sqrt(rr_new > 0.0 ? rr_new : 0.0);
            }
            rz = rz_new;
            rr = rr_new;
            if (true_mode ? (do_replace && true_rr <= tau_true_rr) : (rr <= a.tau_rr)) {
                status = XPLUS_CONVERGED;
                break;
            }
            if (stagnated) break;
            if (fabs(rz_old) <= kBreakdownEps) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            beta = pol.beta(do_replace, drop_replace, rz, rz_old, zap, pap);
            if (bad(beta)) {
                status = XPLUS_BREAKDOWN;
                break;
            }
        }
    }
    if (status == XPLUS_MAX_ITER && !true_mode && rr <= a.tau_rr) status = XPLUS_CONVERGED;

    // ---- exit: fold dx into x, then the FP64 true residual of the final x ----
    flush_dx();
    if (!bar.sync(&s_flag)) return;
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
            o->t_end_ns = globaltimer_ns();
            for (int k = 0; k < 4; ++k) o->t_phase[k] = s_clk[k];
        }
    }
}

// ---------------------------------------------------------------------------------------
// One grid barrier per iteration.  Phase A of iteration k publishes, next to p'.Ap', the six
// FP64 sums that give the NEXT r.z and r.r in closed form once alpha is known:
//   r_{k+1} = r_k - alpha Ap'_k  =>  r.z = S(m r r) - 2 alpha S(m r Ap') + alpha^2 S(m Ap' Ap')
//                                     r.r = S(r r)   - 2 alpha S(r Ap')   + alpha^2 S(Ap' Ap')
// (m = M^-1), so alpha, beta and the convergence test all come out of one reduction.  Instead
// of exchanging z_{k+1} through a second barrier, each row publishes {m r_k, m Ap'_k, p'_k}
// (double-buffered by generation) and every reader rebuilds p'_{k+1} = (m r_k - alpha m Ap'_k)
// + beta p'_k for its window with the same fused multiply-adds, bit-identical to the owner's.
// ---------------------------------------------------------------------------------------
constexpr int kPartials1 = 7;

template <typename VT, int CHUNK, typename IT>
__global__ void __launch_bounds__(512, 1) pcg_resident1_kernel(PcgArgs a) {
    constexpr int NS = kResNS;
    // halo float4 groups per thread loaded ahead, per record array: as many as fit the
    // 128-register budget without spills (-Xptxas -v)
    constexpr int kHaloU = std::is_same<VT, float>::value ? 3 : 2;
    extern __shared__ float smem[];
    __shared__ double s_red[32 * kPartials1];
    __shared__ double s_tot[kPartials1 + 1];
    __shared__ int s_flag;
    __shared__ int2 s_slice[kResSlices];
    __shared__ long long s_clk[6];
    __shared__ int s_exp[2];
    GridBarrier bar{a.bar, a.err, a.timeout_ns, 0u, a.debug_skip_block};
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int per_block = (a.n_slices + gridDim.x - 1) / gridDim.x;
    const int sb = blockIdx.x * per_block;
    const int se = min(a.n_slices, sb + per_block);
    const int r0 = sb * 32;
    const int nb = max(0, se - sb) * 32;
    const int2 win = a.win[blockIdx.x];
    const int w0 = win.x, wn = win.y;  // w0 and wn are multiples of 4
    float* pw = smem;
    float* rv = pw + wn;
    float* apv = rv + nb;
    float* dxv = apv + nb;
    float* mi = dxv + nb;
    float* rsv = mi + nb;
    const VT* __restrict__ val = static_cast<const VT*>(a.val);
    const IT* __restrict__ col = static_cast<const IT*>(a.col);
    const float* __restrict__ minv_g = static_cast<const float*>(a.minv);
    const float* __restrict__ rowsum_g = static_cast<const float*>(a.rowsum);
    float* recs = static_cast<float*>(a.rec);  // [gen][{m r, m Ap, p}][n_pad]
    const size_t np = static_cast<size_t>(a.n_pad);
    auto rec_zr = [&](int g) { return recs + (3 * static_cast<size_t>(g) + 0) * np; };
    auto rec_za = [&](int g) { return recs + (3 * static_cast<size_t>(g) + 1) * np; };
    auto rec_p = [&](int g) { return recs + (3 * static_cast<size_t>(g) + 2) * np; };
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const bool true_mode = a.tau_true_rr >= 0.0;
    for (int k = threadIdx.x; k < se - sb; k += blockDim.x) {
        const long long b0 = a.slice_ptr[sb + k];
        s_slice[k] = make_int2(static_cast<int>(b0), static_cast<int>((a.slice_ptr[sb + k + 1] - b0) >> 5));
    }
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
        mi[t] = minv_g[r0 + t];
        rsv[t] = rowsum_g[r0 + t];
        dxv[t] = 0.0f;
        apv[t] = 0.0f;
    }
    // the band's p' is rebuilt from its own previous value (beta = 0 the first time)
    for (int t = threadIdx.x; t < wn; t += blockDim.x) pw[t] = 0.0f;
    // The rows of this band that another CTA's window covers: [r0, s_exp[0]) for the CTAs
    // below, [s_exp[1], r0 + nb) for those above.  Only these rows' records are ever read by
    // anyone but their owner, so the hot loop writes no others.
    if (warp == 0) {
        int lo = r0, hi = r0 + nb;
        for (int c = lane; c < static_cast<int>(gridDim.x); c += 32) {
            const int2 wc = a.win[c];
            if (wc.y <= 0) continue;
            if (c < static_cast<int>(blockIdx.x)) lo = max(lo, wc.x + wc.y);
            else if (c > static_cast<int>(blockIdx.x)) hi = min(hi, wc.x);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = max(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = min(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            s_exp[0] = min(lo, r0 + nb);
            s_exp[1] = max(hi, r0);
        }
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < 5; ++k) s_clk[k] = 0;
        s_clk[5] = globaltimer_ns();
        if (lead) a.out->t_start_ns = s_clk[5];
    }
    __syncthreads();
    const int exp_lo = s_exp[0], exp_hi = s_exp[1];
    auto clock = [&](int slot) {
        if (threadIdx.x == 0) {
            const long long t = globaltimer_ns();
            s_clk[slot] += t - s_clk[5];
            s_clk[5] = t;
        }
    };
    int bank = 0;
    auto next_bank = [&]() {
        double* b = a.partial + static_cast<size_t>(bank) * 8 * gridDim.x;
        bank ^= 1;
        return b;
    };
    double* cur_bank = nullptr;
    auto flush_dx = [&]() {
        for (int t = threadIdx.x; t < nb; t += blockDim.x) {
            a.x64[r0 + t] += static_cast<double>(dxv[t]);
            dxv[t] = 0.0f;
        }
    };
    // r = b - A x in FP64 into shared r; records of generation g get {m r, 0, p (kept, or 0)}
    auto residual_phase = [&](bool init, int g) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int s = sb + warp; s < se; s += wpb) {
            const int row = s * 32 + lane;
            const double y = row_fp64<VT, float, CHUNK, true, IT>(a, s, lane, row);
            const double bv = a.b64[row];
            const double rt = bv - y;
            const float r_ = static_cast<float>(rt);
            const float z_ = mi[row - r0] * r_;
            if (init) acc[3] += bv * bv;
            rv[row - r0] = r_;
            rec_zr(g)[row] = z_;
            rec_za(g)[row] = 0.0f;
            if (init) rec_p(g)[row] = 0.0f;
            acc[0] += static_cast<double>(r_) * static_cast<double>(z_);
            acc[1] += static_cast<double>(r_) * static_cast<double>(r_);
            acc[2] += rt * rt;
        }
        cur_bank = next_bank();
        publish<4>(acc, s_red, cur_bank);
    };
    // the pending update of the previous iteration: dx += alpha p', r -= alpha Ap'
    auto apply_update = [&](float al) {
        for (int t = threadIdx.x; t < nb; t += blockDim.x) {
            const float pv = pw[r0 + t - w0];
            dxv[t] = __fmaf_rn(al, pv, dxv[t]);
            rv[t] = rv[t] - al * apv[t];
        }
    };

    // The halo's records, in float4 groups of the window [w0, w0 + wn) without the own band
    // (w0, r0, nb and wn are multiples of 4): group u < nlo lies below the band, the others
    // above it.  The first kHaloU groups of each thread are loaded into registers as soon as
    // the grid barrier has made the records final (issue_halo), so the loads overlap the
    // dot-product totals, the scalar updates and the own band's update.
    const int nlo = (r0 - w0) >> 2;
    const int hi0 = (r0 + nb - w0) >> 2;
    const int nh = nlo + (wn >> 2) - hi0;
    const int hbd = static_cast<int>(blockDim.x);
    auto qof = [&](int u) { return u < nlo ? u : hi0 + (u - nlo); };
    float4 hz[kHaloU], hq[kHaloU], hp[kHaloU];
    auto issue_halo = [&](int g) {
        const float4* zr4 = reinterpret_cast<const float4*>(rec_zr(g) + w0);
        const float4* za4 = reinterpret_cast<const float4*>(rec_za(g) + w0);
        const float4* p4 = reinterpret_cast<const float4*>(rec_p(g) + w0);
#pragma unroll
        for (int v = 0; v < kHaloU; ++v) {
            const int u = threadIdx.x + v * hbd;
            if (u < nh) {
                const int qq = qof(u);
                hz[v] = zr4[qq];
                hq[v] = za4[qq];
                hp[v] = p4[qq];
            }
        }
    };
    bool halo_ready = false;  // hz, hq, hp hold generation gen's halo records

    int gen = 0;
    residual_phase(true, gen);
    if (!bar.sync(&s_flag)) return;
    issue_halo(gen);
    halo_ready = true;
    grid_totals(cur_bank, 4, s_tot);
    double rz = s_tot[0], rr = s_tot[1], true_rr = s_tot[2];
    const double tau_true_rr = a.tau2_rel > 0.0 ? a.tau2_rel * s_tot[3] : a.tau_true_rr;
    if (lead) a.out->bb = s_tot[3];
    double rr_at_replace = rr;
    double pap = 0.0, alpha = 0.0, beta = 0.0;
    double pend = 0.0;  // alpha of the update not yet applied to x and r (0: none)
    int status = XPLUS_MAX_ITER, iterations = 0, replacements = 0, stagnated = 0;
    ReplacePolicy pol(a.restart_on_replace, true_rr);
    const bool converged_now = true_mode ? (true_rr <= tau_true_rr) : (rr <= a.tau_rr);
    const int flush_every = a.flush_every > 0 ? a.flush_every : 16;
    clock(4);

    if (converged_now) {
        status = XPLUS_CONVERGED;
    } else {
        for (int it = 0; it < a.max_iters; ++it) {
            if (bad(rz) || bad(rr) || fabs(rz) <= kBreakdownEps) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            // ---- the previous update and the new p' ----
            // Own band, from shared memory: the records this CTA published last iteration are
            // {m r, m Ap', p'} of these very values, so p'_new = fma(beta, p', fma(-alpha, m Ap',
            // m r)) here is bit-identical to what the neighbours rebuild from the records; then
            // the pending update dx += alpha p', r -= alpha Ap'.  Only the halo reads records.
            if (!halo_ready) issue_halo(gen);
            halo_ready = false;
            const float al_prev = static_cast<float>(pend);
            const bool upd = pend != 0.0;
            const bool flush = upd && it % flush_every == 0;
            const float be = static_cast<float>(beta);
            {
                // four rows per thread and step (float4: pw + r0 - w0, rv, apv, mi and dxv all
                // start on 16-byte boundaries, w0 being a multiple of 4 and nb of 32); each row's
                // arithmetic is the scalar form's
                float4* pw4o = reinterpret_cast<float4*>(pw + (r0 - w0));
                float4* rv4 = reinterpret_cast<float4*>(rv);
                const float4* ap4 = reinterpret_cast<const float4*>(apv);
                const float4* mi4 = reinterpret_cast<const float4*>(mi);
                float4* dx4 = reinterpret_cast<float4*>(dxv);
                // p' (new), r and dx of one row; d is read and written only with upd
                auto row_update = [&](float& pv, float& r_, float ap_, float m, float& d) {
                    const float mr = m * r_;
                    const float ma = upd ? m * ap_ : 0.0f;  // the records' m Ap' is 0 after a residual
                    const float pn = __fmaf_rn(be, pv, __fmaf_rn(-al_prev, ma, mr));
                    if (upd) {
                        d = __fmaf_rn(al_prev, pv, d);
                        r_ = r_ - al_prev * ap_;
                    }
                    pv = pn;
                };
                for (int t4 = threadIdx.x; t4 < (nb >> 2); t4 += blockDim.x) {
                    float4 pv = pw4o[t4];
                    float4 r4 = rv4[t4];
                    const float4 a4 = ap4[t4], m4 = mi4[t4];
                    float4 d4 = upd ? dx4[t4] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    row_update(pv.x, r4.x, a4.x, m4.x, d4.x);
                    row_update(pv.y, r4.y, a4.y, m4.y, d4.y);
                    row_update(pv.z, r4.z, a4.z, m4.z, d4.z);
                    row_update(pv.w, r4.w, a4.w, m4.w, d4.w);
                    pw4o[t4] = pv;
                    if (upd) {
                        rv4[t4] = r4;
                        if (flush) {
                            double* xr = a.x64 + r0 + 4 * t4;
                            xr[0] += static_cast<double>(d4.x);
                            xr[1] += static_cast<double>(d4.y);
                            xr[2] += static_cast<double>(d4.z);
                            xr[3] += static_cast<double>(d4.w);
                            d4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        }
                        dx4[t4] = d4;
                    }
                }
            }
            pend = 0.0;
            {
                // halo [w0, r0) and [r0 + nb, w0 + wn) from the records, in float4 groups:
                // the first U groups of each thread were loaded right after the grid barrier
                // (issue_halo), the rest (halos above U * 4 * blockDim.x rows) load here
                const float4* zr4 = reinterpret_cast<const float4*>(rec_zr(gen) + w0);
                const float4* za4 = reinterpret_cast<const float4*>(rec_za(gen) + w0);
                const float4* p4 = reinterpret_cast<const float4*>(rec_p(gen) + w0);
                float4* pw4 = reinterpret_cast<float4*>(pw);
                auto fill = [&](const float4& z, const float4& q, const float4& p) {
                    float4 o;
                    o.x = __fmaf_rn(be, p.x, __fmaf_rn(-al_prev, q.x, z.x));
                    o.y = __fmaf_rn(be, p.y, __fmaf_rn(-al_prev, q.y, z.y));
                    o.z = __fmaf_rn(be, p.z, __fmaf_rn(-al_prev, q.z, z.z));
                    o.w = __fmaf_rn(be, p.w, __fmaf_rn(-al_prev, q.w, z.w));
                    return o;
                };
#pragma unroll
                for (int v = 0; v < kHaloU; ++v) {
                    const int u = threadIdx.x + v * hbd;
                    if (u < nh) pw4[qof(u)] = fill(hz[v], hq[v], hp[v]);
                }
                constexpr int U = kHaloU;
                const int bd = hbd;
                int u = threadIdx.x + U * bd;
                for (; u + (U - 1) * bd < nh; u += U * bd) {
                    float4 z[U], q[U], p[U];
#pragma unroll
                    for (int v = 0; v < U; ++v) {
                        const int qq = qof(u + v * bd);
                        z[v] = zr4[qq];
                        q[v] = za4[qq];
                        p[v] = p4[qq];
                    }
#pragma unroll
                    for (int v = 0; v < U; ++v) pw4[qof(u + v * bd)] = fill(z[v], q[v], p[v]);
                }
                for (; u < nh; u += bd) {
                    const int qq = qof(u);
                    pw4[qq] = fill(zr4[qq], za4[qq], p4[qq]);
                }
                __syncthreads();
            }
            clock(2);
            // ---- Ap' from shared memory, then each row's records of the next generation and
            // its terms of the seven sums (the row's own values only: no CTA barrier between) ----
            {
                double acc[kPartials1] = {0, 0, 0, 0, 0, 0, 0};
                const int g1 = gen ^ 1;
                float* zr1 = rec_zr(g1);
                float* za1 = rec_za(g1);
                float* p1 = rec_p(g1);
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
                        pi[k] = on ? pw[row[k] - w0] : 0.0f;
                    }
                    sell_rows_smem<VT, CHUNK, IT, NS>(sl, row, lane, col, val, pw, w0, pi, y);
#pragma unroll
                    for (int k = 0; k < NS; ++k) {
                        if (row[k] < 0) continue;
                        const int t = row[k] - r0;
                        const float ap_ = y[k] * a.val_scale + rsv[t] * pi[k];
                        apv[t] = ap_;
                        const float r_ = rv[t], m = mi[t];
                        if (row[k] < exp_lo || row[k] >= exp_hi) {
                            zr1[row[k]] = m * r_;
                            za1[row[k]] = m * ap_;
                            p1[row[k]] = pi[k];
                        }
                        const double dr = r_, da = ap_, dm = m;
                        acc[0] += static_cast<double>(pi[k]) * da;
                        acc[1] += dm * dr * dr;
                        acc[2] += dm * dr * da;
                        acc[3] += dm * da * da;
                        acc[4] += dr * dr;
                        acc[5] += dr * da;
                        acc[6] += da * da;
                    }
                }
                clock(3);
                cur_bank = next_bank();
                publish_scatter<kPartials1>(acc, s_red, cur_bank);
            }
            clock(0);
            if (!bar.sync(&s_flag)) return;
            issue_halo(gen ^ 1);  // the generation just published
            halo_ready = true;
            grid_totals(cur_bank, kPartials1, s_tot);
            clock(1);
            gen ^= 1;
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
            pend = alpha;
            double rz_new = s_tot[1] - 2.0 * alpha * s_tot[2] + alpha * alpha * s_tot[3];
            double rr_new = s_tot[4] - 2.0 * alpha * s_tot[5] + alpha * alpha * s_tot[6];
            iterations = it + 1;
            if (bad(rz_new) || bad(rr_new)) {
                rz = rz_new;
                rr = rr_new;
                status = XPLUS_BREAKDOWN;
                break;
            }
            bool do_replace = false, drop_replace = false;
            double zap = 0.0;  // z_new . Ap' of a replacement
            if (true_mode) {
                if (rr_new <= tau_true_rr) do_replace = drop_replace = true;
                if (a.replace_every > 0 && iterations % a.replace_every == 0) do_replace = true;
                if (a.replace_drop > 0.0 && rr_new <= a.replace_drop * rr_at_replace) do_replace = drop_replace = true;
            }
            if (do_replace) {
                halo_ready = false;  // the residual phase rewrites this generation's records
                apply_update(static_cast<float>(pend));
                pend = 0.0;
                __syncthreads();
                flush_dx();
                if (!bar.sync(&s_flag)) return;
                residual_phase(false, gen);
                if (!bar.sync(&s_flag)) return;
                grid_totals(cur_bank, 3, s_tot);
                clock(4);
                rz_new = s_tot[0];
                rr_new = s_tot[1];
                true_rr = s_tot[2];
                ++replacements;
                rr_at_replace = rr_new;
                if (pol.after(a.restart_on_replace, true_rr, a.stag_factor, a.stag_window)) stagnated = 1;
                if (pol.mode == 4) {
                    // z_new . Ap' for the flexible coefficient: a pass of its own, so the
                    // residual phase (and the hot loop around it) stays as in the other modes;
                    // every thread reads back only the records it wrote
                    double acc[1] = {0.0};
                    for (int s = sb + warp; s < se; s += wpb) {
                        const int row = s * 32 + lane;
                        acc[0] += static_cast<double>(rec_zr(gen)[row]) * static_cast<double>(apv[row - r0]);
                    }
                    cur_bank = next_bank();
                    publish<1>(acc, s_red, cur_bank);
                    if (!bar.sync(&s_flag)) return;
                    grid_totals(cur_bank, 1, s_tot);
                    zap = s_tot[0];
                }
            }
            if (lead && a.trace && it < a.trace_cap) {
                double* t = a.trace + 5 * static_cast<size_t>(it);
                t[0] = alpha;
                t[1] = rz_new / rz_old;
                t[2] = rz_new;
                t[3] = rr_new;
                t[4] = sqrt(rr_new > 0.0 ? rr_new : 0.0);
            }
            rz = rz_new;
            rr = rr_new;
            if (true_mode ? (do_replace && true_rr <= tau_true_rr) : (rr <= a.tau_rr)) {
                status = XPLUS_CONVERGED;
                break;
            }
            if (stagnated) break;
            if (fabs(rz_old) <= kBreakdownEps) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            beta = pol.beta(do_replace, drop_replace, rz, rz_old, zap, pap);
            if (bad(beta)) {
                status = XPLUS_BREAKDOWN;
                break;
            }
        }
    }
    if (status == XPLUS_MAX_ITER && !true_mode && rr <= a.tau_rr) status = XPLUS_CONVERGED;

    // ---- exit: the pending update, dx into x, then the FP64 true residual ----
    if (pend != 0.0) {
        apply_update(static_cast<float>(pend));
        __syncthreads();
    }
    flush_dx();
    if (!bar.sync(&s_flag)) return;
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
            o->t_end_ns = globaltimer_ns();
            for (int k = 0; k < 4; ++k) o->t_phase[k] = s_clk[k];
        }
    }
}

template <typename F>
bool resident_dispatch(const KernelKey& k, F&& f) {
    if (k.xt != XPLUS_F32 || !k.diag || k.gtg) return false;
    auto with_it = [&](auto* vt, auto chunk) {
        if (k.idx16) f(vt, chunk, static_cast<short*>(nullptr));
        else f(vt, chunk, static_cast<int*>(nullptr));
        return true;
    };
    auto with_chunk = [&](auto* vt) {
        switch (k.chunk) {
            case 1: return with_it(vt, std::integral_constant<int, 1>());
            case 2: return with_it(vt, std::integral_constant<int, 2>());
            case 4: return with_it(vt, std::integral_constant<int, 4>());
        }
        return false;
    };
    if (k.vt == XPLUS_F32) return with_chunk(static_cast<float*>(nullptr));
    if (k.vt == XPLUS_BF16) return with_chunk(static_cast<__nv_bfloat16*>(nullptr));
    if (k.vt == XPLUS_F16) return with_chunk(static_cast<__half*>(nullptr));
    return false;
}

}  // namespace

bool resident_supported(const KernelKey& k) {
    return resident_dispatch(k, [](auto*, auto, auto*) {});
}

template <typename VT, int CHUNK, typename IT>
auto resident_fn(bool one_sync) {
    return one_sync ? pcg_resident1_kernel<VT, CHUNK, IT> : pcg_resident_kernel<VT, CHUNK, IT>;
}

cudaError_t resident_prepare(const KernelKey& k, int device, size_t smem_bytes, int tpb, bool one_sync,
                             bool* fits) {
    *fits = false;
    int optin = 0;
    cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa{};
    bool ok = resident_dispatch(k, [&](auto* vt, auto chunk, auto* it) {
        using VT = std::remove_pointer_t<decltype(vt)>;
        using IT = std::remove_pointer_t<decltype(it)>;
        e = cudaFuncGetAttributes(&fa, resident_fn<VT, decltype(chunk)::value, IT>(one_sync));
    });
    if (!ok) return cudaSuccess;
    if (e != cudaSuccess) return e;
    if (smem_bytes + fa.sharedSizeBytes > static_cast<size_t>(optin)) return cudaSuccess;
    if (tpb > fa.maxThreadsPerBlock) return cudaSuccess;
    resident_dispatch(k, [&](auto* vt, auto chunk, auto* it) {
        using VT = std::remove_pointer_t<decltype(vt)>;
        using IT = std::remove_pointer_t<decltype(it)>;
        e = cudaFuncSetAttribute(resident_fn<VT, decltype(chunk)::value, IT>(one_sync),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_bytes));
    });
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    resident_dispatch(k, [&](auto* vt, auto chunk, auto* it) {
        using VT = std::remove_pointer_t<decltype(vt)>;
        using IT = std::remove_pointer_t<decltype(it)>;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, resident_fn<VT, decltype(chunk)::value, IT>(one_sync), tpb, smem_bytes);
    });
    if (e != cudaSuccess) return e;
    *fits = per_sm >= 1;
    return cudaSuccess;
}

cudaError_t resident_launch(const KernelKey& k, const PcgArgs& a, int grid, int tpb, size_t smem_bytes,
                            bool one_sync, cudaStream_t s, const cudaAccessPolicyWindow& window) {
    cudaError_t e = cudaErrorInvalidValue;
    resident_dispatch(k, [&](auto* vt, auto chunk, auto* it) {
        using VT = std::remove_pointer_t<decltype(vt)>;
        using IT = std::remove_pointer_t<decltype(it)>;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(tpb);
        cfg.dynamicSmemBytes = smem_bytes;
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
        e = cudaLaunchKernelEx(&cfg, resident_fn<VT, decltype(chunk)::value, IT>(one_sync), a);
    });
    return e;
}

int resident_max_slices() { return kResSlices; }

}  // namespace xplus
