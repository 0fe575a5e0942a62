// pcg_kernels.cu -- the persistent Jacobi-PCG kernel (the role of cuper_pcg_control_kernel,
// kernels/cuper_pcg_control_kernel.cpp:972-1235) and the SELL-C-sigma SpMV.
//
// One cooperative launch runs the whole solve.  Work is owned per SELL slice: warp w of
// the grid owns slices w, w + W, w + 2W, ... and lane l of that warp owns row 32*s + l in
// every phase, so Ap is consumed by the thread that produced it and every vector access is
// a coalesced 32-row segment.  Per iteration (two grid barriers):
//   phase A  p' = z + beta p and Ap' (neighbours' p' recomputed from their {z, p} records,
//            so p' needs no exchange of its own), p'.Ap' partial        -> grid barrier
//   phase B  x += alpha p' (FP64), r -= alpha Ap', z = M^-1 r, r.z and r.r partials,
//            record {z, p'}                                             -> grid barrier
// Dot products are reduced in FP64 with a fixed order (warp tree, block tree, then the
// per-block partials summed identically by every block), so every block takes the same
// control decisions.  FP64 true residuals r = b - A x (FP64 matrix copy) replace the
// recurrence residual on demand: at convergence in true-residual mode, every k
// iterations, or when ||r|| fell by a set factor.  The control flow, breakdown tests and
// status codes follow kernels/cuper_pcg_control_kernel.cpp:1069-1235.
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

constexpr int kMaxSlicesPerBlock = 1024;  // shared slice table capacity (host checks the fit)
constexpr int kSlicesInFlight = 2;

// One iteration needs two grid barriers: the update p' = z + beta p is folded into the next
// SpMV (each row recomputes its neighbours' p' from their records), so the search direction
// is never exchanged through a barrier of its own.
//   phase A  p'_i, Ap'_i (neighbours' p' recomputed), p'.Ap'   -> grid barrier
//   phase B  x += alpha p' (FP64), r -= alpha Ap', z = M^-1 r, r.z, r.r, record {z, p'}
//                                                               -> grid barrier
// Block b owns the contiguous slice range [b*S, (b+1)*S): with a bandwidth-reducing order the
// rows a block gathers from are mostly its own band, which stays in its L1.
template <typename VT, typename XT, int CHUNK, bool DIFF, typename IT>
__global__ void __launch_bounds__(512, 1) pcg_persistent_kernel(PcgArgs a) {
    constexpr int NS = kSlicesInFlight;
    __shared__ double s_red[32 * 4];
    __shared__ double s_tot[4];
    __shared__ int s_flag;
    __shared__ int2 s_slice[kMaxSlicesPerBlock];  // {first slot, width} of the block's slices
    __shared__ long long s_clk[6];
    GridBarrier bar{a.bar, a.err, a.timeout_ns, 0u, a.debug_skip_block};
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int per_block = (a.n_slices + gridDim.x - 1) / gridDim.x;
    const int sb = blockIdx.x * per_block;
    const int se = min(a.n_slices, sb + per_block);
    const VT* __restrict__ val = static_cast<const VT*>(a.val);
    const XT* __restrict__ minv = static_cast<const XT*>(a.minv);
    const XT* __restrict__ rowsum = static_cast<const XT*>(a.rowsum);
    NodeRec<XT>* rec = static_cast<NodeRec<XT>*>(a.rec);
    XT* r = static_cast<XT*>(a.r);
    XT* ap = static_cast<XT*>(a.ap);
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const bool true_mode = a.tau_true_rr >= 0.0;
    for (int k = threadIdx.x; k < se - sb; k += blockDim.x) {
        const long long b0 = a.slice_ptr[sb + k];
        s_slice[k] = make_int2(static_cast<int>(b0), static_cast<int>((a.slice_ptr[sb + k + 1] - b0) >> 5));
    }
    // phase clock of block 0 (globaltimer, in shared memory): work of phase A / B incl. the
    // block reduction, and the grid-barrier waits after each.  Slot 5 is the last mark.
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
    // Two banks of 4 partial slots: consecutive publishes alternate banks, so a block that
    // runs ahead can never overwrite partials another block has not read yet (a barrier
    // separates any two publishes, and a bank is reused only two publishes later).
    int bank = 0;
    auto next_bank = [&]() {
        double* b = a.partial + static_cast<size_t>(bank) * 4 * gridDim.x;
        bank ^= 1;
        return b;
    };
    double* cur_bank = nullptr;

    // ---- residual phase: r = b - A x in FP64, stored rounded, z = M^-1 r into the record
    //      (init also clears p); partials r.z, r.r, true r.r, and ||b||^2 (init) or z.Ap' ----
    auto residual_phase = [&](bool init) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int s = sb + warp; s < se; s += wpb) {
            const int row = s * 32 + lane;
            const double y = row_fp64<VT, XT, CHUNK, DIFF, IT>(a, s, lane, row);
            const double bv = a.b64[row];
            const double rt = bv - y;
            const XT rv = static_cast<XT>(rt);
            const XT zv = minv[row] * rv;
            // slot 3: ||b||^2 in the first pass, z_new . Ap' at a replacement
            acc[3] += init ? bv * bv : static_cast<double>(zv) * static_cast<double>(ap[row]);
            r[row] = rv;
            if (init) store_rec(rec + row, zv, XT(0));
            else rec[row].z = zv;
            acc[0] += static_cast<double>(rv) * static_cast<double>(zv);
            acc[1] += static_cast<double>(rv) * static_cast<double>(rv);
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
    clock(4);

    if (converged_now) {
        status = XPLUS_CONVERGED;
    } else {
        for (int it = 0; it < a.max_iters; ++it) {
            if (bad(rz) || bad(rr) || fabs(rz) <= kBreakdownEps) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            const XT be = static_cast<XT>(beta);
            // ---- phase A: p' = z + beta p (own row), Ap' with recomputed neighbours, p'.Ap' ----
            {
                double acc[1] = {0.0};
                for (int s0 = sb + warp; s0 < se; s0 += NS * wpb) {
                    int2 sl[NS];
                    int row[NS];
                    XT pi[NS], y[NS];
#pragma unroll
                    for (int k = 0; k < NS; ++k) {
                        const int s = s0 + k * wpb;
                        const bool on = s < se;
                        sl[k] = on ? s_slice[s - sb] : make_int2(0, 0);
                        row[k] = on ? s * 32 + lane : -1;
                    }
#pragma unroll
                    for (int k = 0; k < NS; ++k) {
                        const NodeRec<XT> me = row[k] >= 0 ? load_rec(rec + row[k]) : NodeRec<XT>{XT(0), XT(0)};
                        pi[k] = node_pnew(me.z, be, me.p);
                    }
                    sell_rows_pnew<VT, CHUNK, DIFF, IT, XT, NS>(sl, row, lane, static_cast<const IT*>(a.col), val,
                                                                rec, be, pi, y);
#pragma unroll
                    for (int k = 0; k < NS; ++k) {
                        if (row[k] < 0) continue;
                        if (DIFF) y[k] = y[k] * static_cast<XT>(a.val_scale) + rowsum[row[k]] * pi[k];
                        ap[row[k]] = y[k];
                        acc[0] += static_cast<double>(pi[k]) * static_cast<double>(y[k]);
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
            // ---- phase B: x, r, z and the two dots; the record becomes {z_new, p'}; four
            //      slices per step so the loads of all are in flight together ----
            {
                double acc[2] = {0.0, 0.0};
                const XT al = static_cast<XT>(alpha);
                constexpr int NB = 4;  // slices of one warp whose loads are in flight together
                for (int s0 = sb + warp; s0 < se; s0 += NB * wpb) {
                    int row[NB];
                    NodeRec<XT> me[NB];
                    XT apv[NB], rv0[NB], mv[NB];
                    double xv[NB];
#pragma unroll
                    for (int k = 0; k < NB; ++k) {
                        const int s = s0 + k * wpb;
                        row[k] = s < se ? s * 32 + lane : -1;
                        const int rr_ = row[k] >= 0 ? row[k] : s0 * 32 + lane;
                        me[k] = load_rec(rec + rr_);
                        apv[k] = ap[rr_];
                        rv0[k] = r[rr_];
                        mv[k] = minv[rr_];
                        xv[k] = a.x64[rr_];
                    }
#pragma unroll
                    for (int k = 0; k < NB; ++k) {
                        if (row[k] < 0) continue;
                        const XT pv = node_pnew(me[k].z, be, me[k].p);
                        a.x64[row[k]] = xv[k] + alpha * static_cast<double>(pv);
                        const XT rv = rv0[k] - al * apv[k];
                        const XT zv = mv[k] * rv;
                        r[row[k]] = rv;
                        store_rec(rec + row[k], zv, pv);
                        acc[0] += static_cast<double>(rv) * static_cast<double>(zv);
                        acc[1] += static_cast<double>(rv) * static_cast<double>(rv);
                    }
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

    // ---- exit: FP64 true residual of the final x ----
    {
        double acc[1] = {0.0};
        for (int s = sb + warp; s < se; s += wpb) {
            const int row = s * 32 + lane;
            const double y = row_fp64<VT, XT, CHUNK, DIFF, IT>(a, s, lane, row);
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

template <typename VT, typename XT, int CHUNK, bool DIFF, typename IT>
__global__ void __launch_bounds__(256) sell_spmv_kernel(SpmvArgs a, const XT* __restrict__ x,
                                                        XT* __restrict__ y) {
    const int s = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= a.n_slices) return;
    const int row = s * 32 + lane;
    const XT xi = x[row];
    XT acc = sell_row<VT, CHUNK, DIFF, IT, XT, XT>(a.slice_ptr, static_cast<const IT*>(a.col),
                                                   static_cast<const VT*>(a.val), s, lane, x, xi);
    if (DIFF) acc = acc * static_cast<XT>(a.val_scale) + static_cast<const XT*>(a.rowsum)[row] * xi;
    y[row] = acc;
}

template <typename T>
__global__ void gather_kernel(const double* __restrict__ src, T* __restrict__ dst,
                              const int* __restrict__ perm, int n, int n_pad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_pad) dst[i] = i < n ? static_cast<T>(src[perm[i]]) : T(0);
}

__global__ void scatter_kernel(const double* __restrict__ src, double* __restrict__ dst,
                               const int* __restrict__ perm, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[perm[i]] = src[i];
}

// ---- dispatch over (value type, vector type, chunk, row-sum form, index width) ----
// Instantiated combinations: FP32 values in either form, BF16 and FP16 values in the row-sum
// form only, FP64 values in the plain form only.
template <typename XT, int CHUNK, bool DIFF, typename IT, typename F>
bool with_vt(int vt, F&& f) {
    using C = std::integral_constant<int, CHUNK>;
    using D = std::integral_constant<bool, DIFF>;
    switch (vt) {
        case XPLUS_F32: f(static_cast<float*>(nullptr), static_cast<XT*>(nullptr), C(), D(), static_cast<IT*>(nullptr)); return true;
        case XPLUS_BF16:
            if constexpr (DIFF) { f(static_cast<__nv_bfloat16*>(nullptr), static_cast<XT*>(nullptr), C(), D(), static_cast<IT*>(nullptr)); return true; }
            return false;
        case XPLUS_F16:
            if constexpr (DIFF) { f(static_cast<__half*>(nullptr), static_cast<XT*>(nullptr), C(), D(), static_cast<IT*>(nullptr)); return true; }
            return false;
        case XPLUS_F64:
            if constexpr (!DIFF) { f(static_cast<double*>(nullptr), static_cast<XT*>(nullptr), C(), D(), static_cast<IT*>(nullptr)); return true; }
            return false;
    }
    return false;
}
template <typename XT, int CHUNK, bool DIFF, typename F>
bool with_idx(const KernelKey& k, F&& f) {
    return k.idx16 ? with_vt<XT, CHUNK, DIFF, short>(k.vt, f) : with_vt<XT, CHUNK, DIFF, int>(k.vt, f);
}
template <typename XT, int CHUNK, typename F>
bool with_diag(const KernelKey& k, F&& f) {
    return k.diag ? with_idx<XT, CHUNK, true>(k, f) : with_idx<XT, CHUNK, false>(k, f);
}
template <typename XT, typename F>
bool with_chunk(const KernelKey& k, F&& f) {
    switch (k.chunk) {
        case 1: return with_diag<XT, 1>(k, f);
        case 2: return with_diag<XT, 2>(k, f);
        case 4: return with_diag<XT, 4>(k, f);
    }
    return false;
}
template <typename F>
bool dispatch(const KernelKey& k, F&& f) {
    if (k.gtg) return false;
    if (k.xt == XPLUS_F32) return with_chunk<float>(k, f);
    if (k.xt == XPLUS_F64) return with_chunk<double>(k, f);
    return false;
}

}  // namespace

cudaError_t pcg_grid(const KernelKey& k, int device, int n_slices, int want_tpb, int want_bps,
                     int* grid, int* tpb) {
    int sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    const int threads = want_tpb > 0 ? want_tpb : 512;
    int per_sm = 0;
    const bool ok = dispatch(k, [&](auto* vt, auto* xt, auto chunk, auto diag, auto* it) {
        using VT = std::remove_pointer_t<decltype(vt)>;
        using XT = std::remove_pointer_t<decltype(xt)>;
        using IT = std::remove_pointer_t<decltype(it)>;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, pcg_persistent_kernel<VT, XT, decltype(chunk)::value, decltype(diag)::value, IT>,
            threads, 0);
    });
    if (!ok) return cudaErrorInvalidValue;
    if (e != cudaSuccess) return e;
    if (per_sm <= 0) return cudaErrorInvalidConfiguration;
    if (want_bps > 0 && want_bps < per_sm) per_sm = want_bps;
    int blocks = per_sm * sms;
    const int warps_per_block = threads / 32;
    const int need = (n_slices + warps_per_block - 1) / warps_per_block;
    if (blocks > need) blocks = need > 0 ? need : 1;
    // a system of at most four slices per warp runs on one CTA, whose grid barrier is a CTA
    // barrier (n = 1024: 7.3 us per iteration on two CTAs)
    if (n_slices <= 4 * warps_per_block) blocks = 1;
    // every block's contiguous slice range must fit its shared slice table
    if ((n_slices + blocks - 1) / blocks > kMaxSlicesPerBlock) return cudaErrorInvalidConfiguration;
    *grid = blocks;
    *tpb = threads;
    return cudaSuccess;
}

cudaError_t pcg_launch(const KernelKey& k, const PcgArgs& a, int grid, int tpb, cudaStream_t s,
                       const cudaAccessPolicyWindow& window) {
    cudaError_t e = cudaErrorInvalidValue;
    dispatch(k, [&](auto* vt, auto* xt, auto chunk, auto diag, auto* it) {
        using VT = std::remove_pointer_t<decltype(vt)>;
        using XT = std::remove_pointer_t<decltype(xt)>;
        using IT = std::remove_pointer_t<decltype(it)>;
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
        e = cudaLaunchKernelEx(&cfg, pcg_persistent_kernel<VT, XT, decltype(chunk)::value, decltype(diag)::value, IT>, a);
    });
    return e;
}

cudaError_t spmv_launch(const KernelKey& k, const SpmvArgs& a, const void* x, void* y,
                        cudaStream_t s) {
    cudaError_t e = cudaErrorInvalidValue;
    dispatch(k, [&](auto* vt, auto* xt, auto chunk, auto diag, auto* it) {
        using VT = std::remove_pointer_t<decltype(vt)>;
        using XT = std::remove_pointer_t<decltype(xt)>;
        using IT = std::remove_pointer_t<decltype(it)>;
        const int threads = 256;
        const int blocks = (a.n_slices * 32 + threads - 1) / threads;
        sell_spmv_kernel<VT, XT, decltype(chunk)::value, decltype(diag)::value, IT>
            <<<blocks, threads, 0, s>>>(a, static_cast<const XT*>(x), static_cast<XT*>(y));
        e = cudaGetLastError();
    });
    return e;
}

cudaError_t gather_to_sell(int xt, const double* src, void* dst, const int* perm, int n, int n_pad,
                           cudaStream_t s) {
    const int threads = 256, blocks = (n_pad + threads - 1) / threads;
    if (xt == XPLUS_F32)
        gather_kernel<float><<<blocks, threads, 0, s>>>(src, static_cast<float*>(dst), perm, n, n_pad);
    else
        gather_kernel<double><<<blocks, threads, 0, s>>>(src, static_cast<double*>(dst), perm, n, n_pad);
    return cudaGetLastError();
}

cudaError_t scatter_from_sell(const double* src, double* dst, const int* perm, int n,
                              cudaStream_t s) {
    const int threads = 256, blocks = (n + threads - 1) / threads;
    scatter_kernel<<<blocks, threads, 0, s>>>(src, dst, perm, n);
    return cudaGetLastError();
}

}  // namespace xplus
