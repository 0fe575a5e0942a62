// pcg_kernels.cu -- the persistent Jacobi-PCG kernel (the role of cuper_pcg_control_kernel,
// kernels/cuper_pcg_control_kernel.cpp:972-1235) and the SELL-C-sigma SpMV.
//
// One cooperative launch runs the whole solve.  Work is owned per SELL slice: warp w of
// the grid owns slices w, w + W, w + 2W, ... and lane l of that warp owns row 32*s + l in
// every phase, so the SpMV result Ap never leaves the thread that uses it and every vector
// access is a coalesced 32-row segment.  Per iteration:
//   phase A  Ap = A p (SELL, chunked vector loads), p.Ap partial   -> grid barrier
//   phase B  x += alpha p (FP64), r -= alpha Ap, z = M^-1 r, r.z and r.r partials
//                                                                    -> grid barrier
//   phase C  p = z + beta p                                          -> grid barrier
// Dot products are reduced in FP64 with a fixed order (warp tree, block tree, then the
// per-block partials summed identically by every block), so every block takes the same
// control decisions.  FP64 true residuals r = b - A x (FP64 matrix copy) replace the
// recurrence residual on demand: at convergence in true-residual mode, every k
// iterations, or when ||r|| fell by a set factor.  The control flow, breakdown tests and
// status codes follow kernels/cuper_pcg_control_kernel.cpp:1069-1235.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "../../include/xplus_b200.h"
#include "device_common.cuh"
#include "pcg_kernels.cuh"

namespace xplus {
namespace {

using namespace dev;

constexpr double kBreakdownEps = 1.0e-30;  // include/cg_common.hpp:13

template <typename T> struct TypeOf;
template <> struct TypeOf<float> { static constexpr int id = XPLUS_F32; };
template <> struct TypeOf<double> { static constexpr int id = XPLUS_F64; };
template <> struct TypeOf<__nv_bfloat16> { static constexpr int id = XPLUS_BF16; };

// Row `32*s + lane` of the SELL matrix times x, accumulated in AT.
template <typename VT, int CHUNK, typename XV, typename AT>
__device__ __forceinline__ AT sell_row(const long long* __restrict__ slice_ptr,
                                       const int* __restrict__ col, const VT* __restrict__ val,
                                       int s, int lane, const XV* x) {
    const long long base = slice_ptr[s];
    const int w = static_cast<int>((slice_ptr[s + 1] - base) >> 5);
    const VT* vp = val + base + lane * CHUNK;
    const int* cp = col + base + lane * CHUNK;
    AT acc = AT(0);
    int c = 0;
    // two chunks in flight per step
    for (; c + 2 * CHUNK <= w; c += 2 * CHUNK) {
        typename ValArith<VT>::type v0[CHUNK], v1[CHUNK];
        int c0[CHUNK], c1[CHUNK];
        ChunkLoad<VT, CHUNK>::run(vp, v0);
        ColLoad<CHUNK>::run(cp, c0);
        ChunkLoad<VT, CHUNK>::run(vp + 32 * CHUNK, v1);
        ColLoad<CHUNK>::run(cp + 32 * CHUNK, c1);
        AT xv0[CHUNK], xv1[CHUNK];
#pragma unroll
        for (int q = 0; q < CHUNK; ++q) xv0[q] = static_cast<AT>(x[c0[q]]);
#pragma unroll
        for (int q = 0; q < CHUNK; ++q) xv1[q] = static_cast<AT>(x[c1[q]]);
#pragma unroll
        for (int q = 0; q < CHUNK; ++q) acc += static_cast<AT>(v0[q]) * xv0[q];
#pragma unroll
        for (int q = 0; q < CHUNK; ++q) acc += static_cast<AT>(v1[q]) * xv1[q];
        vp += 64 * CHUNK;
        cp += 64 * CHUNK;
    }
    if (c < w) {
        typename ValArith<VT>::type v0[CHUNK];
        int c0[CHUNK];
        ChunkLoad<VT, CHUNK>::run(vp, v0);
        ColLoad<CHUNK>::run(cp, c0);
#pragma unroll
        for (int q = 0; q < CHUNK; ++q) acc += static_cast<AT>(v0[q]) * static_cast<AT>(x[c0[q]]);
    }
    return acc;
}

// FP64 row of A (FP64 copy when present, else the stored values widened) times x64.
template <typename VT, typename XT, int CHUNK, bool DIAG>
__device__ __forceinline__ double row_fp64(const PcgArgs& a, int s, int lane, int row) {
    double y;
    if (a.val64) {
        y = sell_row<double, CHUNK, double, double>(a.slice_ptr, a.col, a.val64, s, lane, a.x64);
        if (DIAG) y += a.diag64[row] * a.x64[row];
    } else {
        y = sell_row<VT, CHUNK, double, double>(a.slice_ptr, a.col, static_cast<const VT*>(a.val),
                                                s, lane, a.x64);
        if (DIAG) y += static_cast<double>(static_cast<const XT*>(a.diag)[row]) * a.x64[row];
    }
    return y;
}

// Sum of the per-block partials of slot q (fixed order, same in every block).
__device__ __forceinline__ void grid_totals(const double* partial, int nq, double* s_tot) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        for (int q = 0; q < nq; ++q) {
            double v = 0.0;
            for (int b = lane; b < static_cast<int>(gridDim.x); b += 32)
                v += __ldcg(partial + static_cast<size_t>(q) * gridDim.x + b);
            v = warp_sum(v);
            if (lane == 0) s_tot[q] = v;
        }
    }
    __syncthreads();
}

template <int NV>
__device__ __forceinline__ void publish(double (&v)[NV], double* s_red, double* partial) {
    block_sum<NV>(v, s_red);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) partial[static_cast<size_t>(q) * gridDim.x + blockIdx.x] = v[q];
}

inline __device__ bool bad(double v) { return v != v; }

template <typename VT, typename XT, int CHUNK, bool DIAG>
__global__ void __launch_bounds__(512) pcg_persistent_kernel(PcgArgs a) {
    __shared__ double s_red[32 * 3];
    __shared__ double s_tot[4];
    __shared__ int s_flag;
    GridBarrier bar{a.bar, a.err, a.timeout_ns, 0u, a.debug_skip_block};
    const int lane = threadIdx.x & 31;
    const int gwarp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
    const VT* __restrict__ val = static_cast<const VT*>(a.val);
    const XT* __restrict__ minv = static_cast<const XT*>(a.minv);
    const XT* __restrict__ diag = static_cast<const XT*>(a.diag);
    XT* r = static_cast<XT*>(a.r);
    XT* p = static_cast<XT*>(a.p);
    XT* ap = static_cast<XT*>(a.ap);
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const bool true_mode = a.tau_true_rr >= 0.0;
    // Two banks of 4 partial slots: consecutive publishes alternate banks, so a block that
    // runs ahead can never overwrite partials another block has not read yet (a barrier
    // separates any two publishes, and a bank is reused only two publishes later).
    int bank = 0;
    auto next_bank = [&]() {
        double* b = a.partial + static_cast<size_t>(bank) * 4 * gridDim.x;
        bank ^= 1;
        return b;
    };
    double* cur = nullptr;
    if (lead) a.out->t_start_ns = globaltimer_ns();

    // ---- residual phase: r = b - A x (FP64), z = M^-1 r, optionally p = z ----
    // partial slots: 0 = r.z, 1 = r.r (of the stored r), 2 = true r.r (FP64)
    auto residual_phase = [&](bool set_p) {
        double acc[3] = {0.0, 0.0, 0.0};
        for (int s = gwarp; s < a.n_slices; s += nwarps) {
            const int row = s * 32 + lane;
            const double y = row_fp64<VT, XT, CHUNK, DIAG>(a, s, lane, row);
            const double rt = a.b64[row] - y;
            const XT rv = static_cast<XT>(rt);
            const XT zv = minv[row] * rv;
            r[row] = rv;
            if (set_p) p[row] = zv;
            acc[0] += static_cast<double>(rv) * static_cast<double>(zv);
            acc[1] += static_cast<double>(rv) * static_cast<double>(rv);
            acc[2] += rt * rt;
        }
        cur = next_bank();
        publish<3>(acc, s_red, cur);
    };

    residual_phase(true);
    if (!bar.sync(&s_flag)) return;
    grid_totals(cur, 3, s_tot);
    double rz = s_tot[0], rr = s_tot[1], true_rr = s_tot[2];
    double rr_at_replace = rr, best_true = true_rr;
    double pap = 0.0, alpha = 0.0;
    int status = XPLUS_MAX_ITER, iterations = 0, replacements = 0, stagnant = 0, stagnated = 0;
    bool converged_now = true_mode ? (true_rr <= a.tau_true_rr) : (rr <= a.tau_rr);

    if (converged_now) {
        status = XPLUS_CONVERGED;
    } else {
        for (int it = 0; it < a.max_iters; ++it) {
            if (bad(rz) || bad(rr) || fabs(rz) <= kBreakdownEps) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            // ---- phase A: Ap = A p, p.Ap ----
            {
                double acc[1] = {0.0};
                for (int s = gwarp; s < a.n_slices; s += nwarps) {
                    const int row = s * 32 + lane;
                    XT y = sell_row<VT, CHUNK, XT, XT>(a.slice_ptr, a.col, val, s, lane, p);
                    const XT pv = p[row];
                    if (DIAG) y += diag[row] * pv;
                    ap[row] = y;
                    acc[0] += static_cast<double>(pv) * static_cast<double>(y);
                }
                cur = next_bank();
                publish<1>(acc, s_red, cur);
            }
            if (!bar.sync(&s_flag)) return;
            grid_totals(cur, 1, s_tot);
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
            // ---- phase B: x, r, z and the two dots ----
            {
                double acc[2] = {0.0, 0.0};
                const XT al = static_cast<XT>(alpha);
                for (int s = gwarp; s < a.n_slices; s += nwarps) {
                    const int row = s * 32 + lane;
                    const XT pv = p[row];
                    a.x64[row] += alpha * static_cast<double>(pv);
                    const XT rv = r[row] - al * ap[row];
                    const XT zv = minv[row] * rv;
                    r[row] = rv;
                    acc[0] += static_cast<double>(rv) * static_cast<double>(zv);
                    acc[1] += static_cast<double>(rv) * static_cast<double>(rv);
                }
                cur = next_bank();
                publish<2>(acc, s_red, cur);
            }
            if (!bar.sync(&s_flag)) return;
            grid_totals(cur, 2, s_tot);
            double rz_new = s_tot[0], rr_new = s_tot[1];
            iterations = it + 1;
            if (bad(rz_new) || bad(rr_new)) {
                rz = rz_new;
                rr = rr_new;
                status = XPLUS_BREAKDOWN;
                break;
            }
            bool do_replace = false;
            if (true_mode) {
                if (rr_new <= a.tau_true_rr) do_replace = true;
                if (a.replace_every > 0 && iterations % a.replace_every == 0) do_replace = true;
                if (a.replace_drop > 0.0 && rr_new <= a.replace_drop * rr_at_replace) do_replace = true;
            }
            if (do_replace) {
                residual_phase(false);
                if (!bar.sync(&s_flag)) return;
                grid_totals(cur, 3, s_tot);
                rz_new = s_tot[0];
                rr_new = s_tot[1];
                true_rr = s_tot[2];
                ++replacements;
                rr_at_replace = rr_new;
                if (true_rr < 0.9 * best_true) {
                    best_true = true_rr;
                    stagnant = 0;
                } else if (++stagnant >= 8) {
                    stagnated = 1;
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
            if (true_mode ? (do_replace && true_rr <= a.tau_true_rr) : (rr <= a.tau_rr)) {
                status = XPLUS_CONVERGED;
                break;
            }
            if (stagnated) break;
            if (fabs(rz_old) <= kBreakdownEps) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            const double beta = rz / rz_old;
            if (bad(beta)) {
                status = XPLUS_BREAKDOWN;
                break;
            }
            // ---- phase C: p = z + beta p ----
            {
                const XT be = static_cast<XT>(beta);
                for (int s = gwarp; s < a.n_slices; s += nwarps) {
                    const int row = s * 32 + lane;
                    p[row] = minv[row] * r[row] + be * p[row];
                }
            }
            if (!bar.sync(&s_flag)) return;
        }
    }
    if (status == XPLUS_MAX_ITER && !true_mode && rr <= a.tau_rr) status = XPLUS_CONVERGED;

    // ---- exit: FP64 true residual of the final x ----
    {
        double acc[1] = {0.0};
        for (int s = gwarp; s < a.n_slices; s += nwarps) {
            const int row = s * 32 + lane;
            const double y = row_fp64<VT, XT, CHUNK, DIAG>(a, s, lane, row);
            const double rt = a.b64[row] - y;
            acc[0] += rt * rt;
        }
        cur = next_bank();
        publish<1>(acc, s_red, cur);
    }
    if (!bar.sync(&s_flag)) return;
    if (blockIdx.x == 0) {
        grid_totals(cur, 1, s_tot);
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
        }
    }
}

template <typename VT, typename XT, int CHUNK, bool DIAG>
__global__ void __launch_bounds__(256) sell_spmv_kernel(SpmvArgs a, const XT* __restrict__ x,
                                                        XT* __restrict__ y) {
    const int s = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= a.n_slices) return;
    const int row = s * 32 + lane;
    XT acc = sell_row<VT, CHUNK, XT, XT>(a.slice_ptr, a.col, static_cast<const VT*>(a.val), s, lane, x);
    if (DIAG) acc += static_cast<const XT*>(a.diag)[row] * x[row];
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

// ---- dispatch over (value type, vector type, chunk, diag) ----
template <typename XT, int CHUNK, bool DIAG, typename F>
bool with_vt(int vt, F&& f) {
    switch (vt) {
        case XPLUS_F32: f(static_cast<float*>(nullptr), static_cast<XT*>(nullptr), std::integral_constant<int, CHUNK>(), std::integral_constant<bool, DIAG>()); return true;
        case XPLUS_BF16: f(static_cast<__nv_bfloat16*>(nullptr), static_cast<XT*>(nullptr), std::integral_constant<int, CHUNK>(), std::integral_constant<bool, DIAG>()); return true;
        case XPLUS_F64: f(static_cast<double*>(nullptr), static_cast<XT*>(nullptr), std::integral_constant<int, CHUNK>(), std::integral_constant<bool, DIAG>()); return true;
    }
    return false;
}
template <typename XT, int CHUNK, typename F>
bool with_diag(const KernelKey& k, F&& f) {
    return k.diag ? with_vt<XT, CHUNK, true>(k.vt, f) : with_vt<XT, CHUNK, false>(k.vt, f);
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
    const bool ok = dispatch(k, [&](auto* vt, auto* xt, auto chunk, auto diag) {
        using VT = std::remove_pointer_t<decltype(vt)>;
        using XT = std::remove_pointer_t<decltype(xt)>;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, pcg_persistent_kernel<VT, XT, decltype(chunk)::value, decltype(diag)::value>,
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
    *grid = blocks;
    *tpb = threads;
    return cudaSuccess;
}

cudaError_t pcg_launch(const KernelKey& k, const PcgArgs& a, int grid, int tpb, cudaStream_t s) {
    cudaError_t e = cudaErrorInvalidValue;
    dispatch(k, [&](auto* vt, auto* xt, auto chunk, auto diag) {
        using VT = std::remove_pointer_t<decltype(vt)>;
        using XT = std::remove_pointer_t<decltype(xt)>;
        void* args[] = {const_cast<PcgArgs*>(&a)};
        e = cudaLaunchCooperativeKernel(
            reinterpret_cast<const void*>(
                pcg_persistent_kernel<VT, XT, decltype(chunk)::value, decltype(diag)::value>),
            dim3(grid), dim3(tpb), args, 0, s);
    });
    return e;
}

cudaError_t spmv_launch(const KernelKey& k, const SpmvArgs& a, const void* x, void* y,
                        cudaStream_t s) {
    cudaError_t e = cudaErrorInvalidValue;
    dispatch(k, [&](auto* vt, auto* xt, auto chunk, auto diag) {
        using VT = std::remove_pointer_t<decltype(vt)>;
        using XT = std::remove_pointer_t<decltype(xt)>;
        const int threads = 256;
        const int blocks = (a.n_slices * 32 + threads - 1) / threads;
        sell_spmv_kernel<VT, XT, decltype(chunk)::value, decltype(diag)::value>
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
