// batch.cu -- many independent SPD systems solved by one persistent launch.
//
// The systems' SELL-C-sigma images are concatenated into one slice list (each system keeps
// its own sigma-sort and padding; columns are global rows, or int16 offsets from the row).
// A launch of thread-block clusters takes systems from a device work queue, largest first
// (nnz * sqrt(n), a proxy for work = nnz x iterations): rank 0 of a cluster pops the next
// system id with one atomicAdd and the cluster's CTAs split that system's slices.  Each
// system runs the Jacobi-PCG iteration of pcg_kernels.cu (row-sum form, FP32 vectors, FP64
// solution and FP64 residual replacement) with cluster barriers in place of grid barriers
// and dot products reduced through distributed shared memory in cluster-rank order, so every
// CTA of the cluster takes the same control decisions.  No wait spans two clusters, so the
// launch needs no co-residency: clusters that start late simply find the queue shorter.
// Control flow, breakdown tests and status codes: kernels/cuper_pcg_control_kernel.cpp:1069-1235.
#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>
#include <type_traits>
#include <vector>

#include "batch_common.cuh"
#include "common.hpp"
#include "device_common.cuh"
#include "pcg_device.cuh"

namespace xplus {
namespace {

using namespace dev;

// MAXT / MINB: the 512-thread form for launches of 256 and 512 threads (126 registers), and a
// 128-thread form held to 80 registers so that six CTAs share an SM (24 warps instead of 16;
// no spills) for launches of 128 threads
template <typename VT, int CHUNK, typename IT, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) pcg_batch_kernel(BatchArgs a) {
    constexpr int NS = 2;  // slices of one warp in flight together
    cg::cluster_group cl = cg::this_cluster();
    __shared__ double s_red[32 * 4];
    __shared__ double s_part[2][4];
    __shared__ double s_tot[4];
    __shared__ int s_item[2];
    const int crank = static_cast<int>(cl.block_rank());
    const int csize = static_cast<int>(cl.num_blocks());
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const VT* __restrict__ val = static_cast<const VT*>(a.val);
    const IT* __restrict__ col = static_cast<const IT*>(a.col);
    int pbank = 0, ibank = 0;

    for (;;) {
        if (crank == 0 && threadIdx.x == 0) s_item[ibank] = a.q_begin + atomicAdd(a.head, 1);
        cl.sync();
        const int qi = *cl.map_shared_rank(&s_item[ibank], 0);
        ibank ^= 1;
        if (qi >= a.q_end) {
            // every CTA has read rank 0's queue item before any CTA of the cluster exits: a
            // CTA's shared memory must outlive all distributed-shared-memory reads of it
            cl.sync();
            break;
        }
        const long long t_begin = globaltimer_ns();
        const int sys = a.order[qi];
        const int S0 = a.sys_slice0[sys];
        const int ns = a.sys_slice0[sys + 1] - S0;
        const int per = (ns + csize - 1) / csize;
        const int sb = S0 + min(ns, crank * per);
        const int se = S0 + min(ns, (crank + 1) * per);
        const int n = a.sys_n[sys];
        const float vscale = a.sys_scale[sys];
        const int max_iters = a.max_iters > 0 ? a.max_iters : max(4 * n, 1000);
        const bool true_mode = a.tau_mode == XPLUS_TAU_REL_TRUE;

        // residual phase: r = b - A x in FP64 rounded to FP32, z = M^-1 r into the record
        // (init also clears p); totals r.z, r.r, ||b - A x||^2, and ||b||^2 (init) or z.Ap'
        auto residual_phase = [&](bool init, double (&acc)[4]) {
            acc[0] = acc[1] = acc[2] = acc[3] = 0.0;
            for (int s = sb + warp; s < se; s += wpb) {
                const int row = s * 32 + lane;
                const double bv = a.b64[row];
                const double rt = bv - batch_row64<CHUNK, IT>(a, s, lane);
                const float rv = static_cast<float>(rt);
                const float zv = a.minv[row] * rv;
                a.r[row] = rv;
                if (init) store_rec(a.rec + row, zv, 0.0f);
                else a.rec[row].z = zv;
                acc[0] += static_cast<double>(rv) * static_cast<double>(zv);
                acc[1] += static_cast<double>(rv) * static_cast<double>(rv);
                acc[2] += rt * rt;
                acc[3] += init ? bv * bv : static_cast<double>(zv) * static_cast<double>(a.ap[row]);
            }
            cluster_sum<4>(cl, acc, s_red, s_part, s_tot, pbank);
        };

        double tot[4];
        residual_phase(true, tot);
        double rz = tot[0], rr = tot[1], true_rr = tot[2];
        const double bb = tot[3];
        const double tau_true_rr = a.tau * a.tau * bb;
        double rr_at_replace = rr;
        double pap = 0.0, alpha = 0.0, beta = 0.0;
        int status = XPLUS_MAX_ITER, iterations = 0, replacements = 0;
        ReplacePolicy pol(a.restart_on_replace, true_rr);
        bool stagnated = false;
        const bool converged_now = true_mode ? (true_rr <= tau_true_rr) : (rr <= a.tau);

        if (converged_now) {
            status = XPLUS_CONVERGED;
        } else {
            for (int it = 0; it < max_iters; ++it) {
                if (bad(rz) || bad(rr) || fabs(rz) <= kBreakdownEps) {
                    status = XPLUS_BREAKDOWN;
                    break;
                }
                const float be = static_cast<float>(beta);
                // ---- phase A: p' = z + beta p (neighbours' p' recomputed), Ap', p'.Ap' ----
                {
                    double acc[1] = {0.0};
                    for (int s0 = sb + warp; s0 < se; s0 += NS * wpb) {
                        int2 sl[NS];
                        int row[NS];
                        float pi[NS], y[NS];
                        int wmax = 0;
#pragma unroll
                        for (int k = 0; k < NS; ++k) {
                            const int s = s0 + k * wpb;
                            const bool on = s < se;
                            const long long p0 = on ? a.slice_ptr[s] : 0;
                            sl[k] = on ? make_int2(static_cast<int>(p0), static_cast<int>((a.slice_ptr[s + 1] - p0) >> 5))
                                       : make_int2(0, 0);
                            row[k] = on ? s * 32 + lane : -1;
                            wmax = max(wmax, sl[k].y);
                            const NodeRec<float> me = on ? ldcg_rec(a.rec + row[k]) : NodeRec<float>{0.0f, 0.0f};
                            pi[k] = node_pnew(me.z, be, me.p);
                            y[k] = 0.0f;
                        }
                        for (int c = 0; c < wmax; c += 2 * CHUNK) {
                            float v[NS][2][CHUNK];
                            int cc[NS][2][CHUNK];
#pragma unroll
                            for (int k = 0; k < NS; ++k)
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                    if (c + h * CHUNK < sl[k].y) {
                                        const int off = sl[k].x + (c + h * CHUNK) * 32 + lane * CHUNK;
                                        // slots bypass L1 (streamed once per iteration), so L1 keeps
                                        // the records gathered below (measured 8% faster batch)
                                        ChunkLoad<VT, CHUNK, kLdNoAlloc>::run(val + off, v[k][h]);
                                        ColLoad<CHUNK, IT, kLdNoAlloc>::run(col + off, row[k], cc[k][h]);
                                    } else {
#pragma unroll
                                        for (int q = 0; q < CHUNK; ++q) {
                                            v[k][h][q] = 0.0f;
                                            cc[k][h][q] = -1;
                                        }
                                    }
                                }
                            NodeRec<float> nb[NS][2][CHUNK];
#pragma unroll
                            for (int k = 0; k < NS; ++k)
#pragma unroll
                                for (int h = 0; h < 2; ++h)
#pragma unroll
                                    for (int q = 0; q < CHUNK; ++q)
                                        nb[k][h][q] = cc[k][h][q] >= 0 ? ldcg_rec(a.rec + cc[k][h][q])
                                                                       : NodeRec<float>{0.0f, 0.0f};
#pragma unroll
                            for (int k = 0; k < NS; ++k)
#pragma unroll
                                for (int h = 0; h < 2; ++h)
#pragma unroll
                                    for (int q = 0; q < CHUNK; ++q)
                                        y[k] += v[k][h][q] * (node_pnew(nb[k][h][q].z, be, nb[k][h][q].p) - pi[k]);
                        }
#pragma unroll
                        for (int k = 0; k < NS; ++k) {
                            if (row[k] < 0) continue;
                            const float yk = y[k] * vscale + a.rowsum[row[k]] * pi[k];
                            a.ap[row[k]] = yk;
                            acc[0] += static_cast<double>(pi[k]) * static_cast<double>(yk);
                        }
                    }
                    cluster_sum<1>(cl, acc, s_red, s_part, s_tot, pbank);
                    pap = acc[0];
                }
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
                // ---- phase B: x += alpha p' (FP64), r -= alpha Ap', z = M^-1 r, r.z, r.r ----
                double rz_new, rr_new;
                {
                    double acc[2] = {0.0, 0.0};
                    const float al = static_cast<float>(alpha);
                    // four slices of the warp at once: every load before any arithmetic
                    constexpr int NB = 4;
                    for (int s0 = sb + warp; s0 < se; s0 += NB * wpb) {
                        NodeRec<float> me[NB];
                        double xv[NB];
                        float r0[NB], apv[NB], mv[NB];
                        int row[NB];
#pragma unroll
                        for (int k = 0; k < NB; ++k) {
                            const int s = s0 + k * wpb;
                            row[k] = s < se ? s * 32 + lane : -1;
                            const int rr_ = row[k] >= 0 ? row[k] : s0 * 32 + lane;
                            me[k] = ldcg_rec(a.rec + rr_);
                            xv[k] = a.x64[rr_];
                            r0[k] = a.r[rr_];
                            apv[k] = a.ap[rr_];
                            mv[k] = a.minv[rr_];
                        }
#pragma unroll
                        for (int k = 0; k < NB; ++k) {
                            if (row[k] < 0) continue;
                            const float pv = node_pnew(me[k].z, be, me[k].p);
                            a.x64[row[k]] = xv[k] + alpha * static_cast<double>(pv);
                            const float rv = r0[k] - al * apv[k];
                            const float zv = mv[k] * rv;
                            a.r[row[k]] = rv;
                            store_rec(a.rec + row[k], zv, pv);
                            acc[0] += static_cast<double>(rv) * static_cast<double>(zv);
                            acc[1] += static_cast<double>(rv) * static_cast<double>(rv);
                        }
                    }
                    cluster_sum<2>(cl, acc, s_red, s_part, s_tot, pbank);
                    rz_new = acc[0];
                    rr_new = acc[1];
                }
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
                    if (a.replace_drop2 > 0.0 && rr_new <= a.replace_drop2 * rr_at_replace) do_replace = drop_replace = true;
                }
                if (do_replace) {
                    double t4[4];
                    residual_phase(false, t4);
                    rz_new = t4[0];
                    rr_new = t4[1];
                    true_rr = t4[2];
                    zap = t4[3];
                    ++replacements;
                    rr_at_replace = rr_new;
                    if (pol.after(a.restart_on_replace, true_rr, a.stag_factor, a.stag_window)) stagnated = true;
                }
                rz = rz_new;
                rr = rr_new;
                if (true_mode ? (do_replace && true_rr <= tau_true_rr) : (rr <= a.tau)) {
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
        if (status == XPLUS_MAX_ITER && !true_mode && rr <= a.tau) status = XPLUS_CONVERGED;

        // exit: FP64 true residual of the final x
        double fin[1] = {0.0};
        for (int s = sb + warp; s < se; s += wpb) {
            const int row = s * 32 + lane;
            const double rt = a.b64[row] - batch_row64<CHUNK, IT>(a, s, lane);
            fin[0] += rt * rt;
        }
        cluster_sum<1>(cl, fin, s_red, s_part, s_tot, pbank);
        if (crank == 0 && threadIdx.x == 0) {
            a.out_status[sys] = status;
            a.out_iters[sys] = iterations;
            a.out_repl[sys] = replacements;
            a.out_true_rel[sys] = bb > 0.0 ? sqrt(fin[0] / bb) : sqrt(fin[0]);
            a.out_ns[sys] = globaltimer_ns() - t_begin;
        }
    }
}

// dst[i] = src[map[i]] (0 where map[i] < 0: padding rows)
__global__ void batch_gather_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                    const int* __restrict__ map, int rows) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < rows) {
        const int m = map[i];
        dst[i] = m >= 0 ? src[m] : 0.0;
    }
}

__global__ void batch_scatter_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                     const int* __restrict__ map, int rows) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < rows) {
        const int m = map[i];
        if (m >= 0) dst[m] = src[i];
    }
}

template <typename VT, typename IT, int MAXT, int MINB>
BatchKernel pick_chunk(int chunk) {
    switch (chunk) {
        case 1: return pcg_batch_kernel<VT, 1, IT, MAXT, MINB>;
        case 2: return pcg_batch_kernel<VT, 2, IT, MAXT, MINB>;
        case 4: return pcg_batch_kernel<VT, 4, IT, MAXT, MINB>;
    }
    return nullptr;
}
template <typename IT, int MAXT, int MINB>
BatchKernel pick_vt(int vt, int chunk) {
    switch (vt) {
        case XPLUS_F32: return pick_chunk<float, IT, MAXT, MINB>(chunk);
        case XPLUS_BF16: return pick_chunk<__nv_bfloat16, IT, MAXT, MINB>(chunk);
        case XPLUS_F16: return pick_chunk<__half, IT, MAXT, MINB>(chunk);
    }
    return nullptr;
}
// small: the 128-thread form
BatchKernel pick_kernel(int vt, int chunk, bool idx16, bool small) {
    if (small) return idx16 ? pick_vt<short, 128, 6>(vt, chunk) : pick_vt<int, 128, 6>(vt, chunk);
    return idx16 ? pick_vt<short, 512, 1>(vt, chunk) : pick_vt<int, 512, 1>(vt, chunk);
}

}  // namespace
}  // namespace xplus

struct xplus_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    xplus_opts opts{};
    int nsys = 0;
    int rows = 0;          // concatenated SELL rows (padding included)
    int n_slices = 0;
    int64_t total_n = 0, total_nnz = 0, slots = 0;
    bool idx16 = true;
    xplus::BatchKernel kernel = nullptr;        // launches of 256 or 512 threads
    xplus::BatchKernel kernel_small = nullptr;  // launches of 128 threads
    int cluster = 4, tpb = 512, grid = 0;
    // the `split` largest systems in a launch of their own (clusters of cluster2 CTAs of tpb2
    // threads, one cluster per system) on a second stream, beside the launch of the rest
    int split = 0, cluster2 = 16, tpb2 = 512, grid2 = 0;
    // the cluster-resident kernel (both lanes): vectors and the p' window in shared memory,
    // each launch sized for the largest need of the systems it takes
    xplus::BatchKernel res_kernel = nullptr;
    bool resident = false;
    int res_max_dyn = 0;             // dynamic shared memory a CTA may have (bytes)
    int res_half = 0;                // dynamic shared memory at which two CTAs share an SM
    int res_smem = 0, res_smem2 = 0; // the main and the split launch's dynamic shared memory
    // stage each band's matrix in the shared memory a launch has beyond its vectors (each
    // launch widened to the most that keeps its occupancy)
    bool stage_matrix = true;
    std::vector<int> order;          // host copy of the queue (system ids, largest first)
    std::vector<int> need[5];        // [log2 cluster][system]: resident bytes per CTA
    float* d_rec3 = nullptr;
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::vector<int> sys_n;
    std::vector<int64_t> sys_off;   // original-order offsets of each system in b / x
    // device data
    int* d_order = nullptr;
    int* d_head = nullptr;
    int* d_slice0 = nullptr;
    int* d_sysn = nullptr;
    float* d_scale = nullptr;
    long long* d_slice_ptr = nullptr;
    void* d_col = nullptr;
    void* d_val = nullptr;
    double* d_val64 = nullptr;
    double* d_diag64 = nullptr;
    float* d_rowsum = nullptr;
    float* d_minv = nullptr;
    int* d_map = nullptr;
    double* d_b64 = nullptr;
    double* d_x64 = nullptr;
    void* d_rec = nullptr;
    float* d_r = nullptr;
    float* d_ap = nullptr;
    double* d_bio = nullptr;
    double* d_xio = nullptr;
    int* d_status = nullptr;
    int* d_iters = nullptr;
    int* d_repl = nullptr;
    double* d_true_rel = nullptr;
    long long* d_ns = nullptr;
    int* d_staged = nullptr;        // resident kernel: CTAs per system that staged their matrix
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // CUDA graph of the last device solve, replayed while its arguments stay the same
    cudaGraphExec_t gexec = nullptr;
    const double* g_b = nullptr;
    double* g_x = nullptr;
    double g_tau = 0.0;
    int g_mode = -1, g_iters = 0, g_cluster = 0, g_tpb = 0, g_split = -1, g_cluster2 = 0, g_tpb2 = 0;
    bool g_resident = false, g_stage = false;
    bool pending = false;
    bool have_b = false;   // d_b64 holds the (gathered) right-hand side of a solve
    double last_ms = 0.0;
    std::vector<void*> allocations;
};

namespace xplus {
namespace {

void bcheck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

template <typename T>
T* balloc(xplus_batch* h, size_t count) {
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, std::max<size_t>(count * sizeof(T), 256));
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    h->allocations.push_back(p);
    return static_cast<T*>(p);
}

template <typename T>
void upload(xplus_batch* h, T* dst, const std::vector<T>& src) {
    bcheck(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream), "H2D");
}

void batch_destroy(xplus_batch* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    for (void* p : h->allocations) cudaFree(p);
    if (h->stream2) cudaStreamSynchronize(h->stream2);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->stream2) cudaStreamDestroy(h->stream2);
    if (h->stream) cudaStreamDestroy(h->stream);
    cudaGetLastError();
    delete h;
}

int log2_cluster(int c) { return c <= 1 ? 0 : c == 2 ? 1 : c == 4 ? 2 : c == 8 ? 3 : 4; }

BatchKernel kernel_for(const xplus_batch* h, int tpb) {
    if (h->resident) return h->res_kernel;
    return tpb <= 128 ? h->kernel_small : h->kernel;
}

// Largest resident-kernel need (bytes of dynamic shared memory per CTA) of the systems at queue
// positions [q0, q1) on clusters of `cluster` CTAs.
int lane_need(const xplus_batch* h, int q0, int q1, int cluster) {
    const std::vector<int>& nd = h->need[log2_cluster(cluster)];
    int m = 0;
    for (int q = q0; q < q1; ++q) m = std::max(m, nd[static_cast<size_t>(h->order[static_cast<size_t>(q)])]);
    return m;
}

// Clusters of `cluster` CTAs of `tpb` threads (and `smem` bytes of dynamic shared memory) that
// the device holds at once (0: not launchable).
int active_clusters(xplus_batch* h, int cluster, int tpb, int smem = 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster);
    cfg.blockDim = dim3(tpb);
    cfg.dynamicSmemBytes = static_cast<size_t>(smem);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int num = 0;
    if (cudaOccupancyMaxActiveClusters(&num, kernel_for(h, tpb), &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return num;
}

// The dynamic shared memory of a resident launch whose systems need `need` bytes per CTA: with
// matrix staging, the most (all a CTA may have, or what lets two CTAs share an SM) at which
// clusters of `cluster` CTAs of `tpb` threads are as many on the device as at `need`.
int widen_budget(xplus_batch* h, int cluster, int tpb, int need) {
    if (!h->stage_matrix) return need;
    const int num = active_clusters(h, cluster, tpb, need);
    for (int b : {h->res_max_dyn, h->res_half})
        if (b >= need && active_clusters(h, cluster, tpb, b) == num) return b;
    return need;
}

// Grids of the two launches (and, for the resident kernel, their dynamic shared memory) for
// the handle's current kernel and shapes; throws when a shape cannot launch or a system does
// not fit the resident kernel's shared memory at its lane's cluster size.
void plan(xplus_batch* h) {
    const int split = std::min(h->split, h->nsys);
    if (h->resident) {
        h->res_smem = lane_need(h, split, h->nsys, h->cluster);
        require(h->res_smem <= h->res_max_dyn, XPLUS_ERR_ARG,
                "a system of the main launch does not fit the resident kernel's shared memory at cluster " +
                    std::to_string(h->cluster) + " (" + std::to_string(h->res_smem) + " bytes per CTA)");
        h->res_smem2 = split > 0 ? lane_need(h, 0, split, h->cluster2) : 0;
        require(h->res_smem2 <= h->res_max_dyn, XPLUS_ERR_ARG,
                "a system of the split launch does not fit the resident kernel's shared memory at cluster " +
                    std::to_string(h->cluster2) + " (" + std::to_string(h->res_smem2) + " bytes per CTA)");
        if (split < h->nsys) h->res_smem = widen_budget(h, h->cluster, h->tpb, h->res_smem);
        if (split > 0) h->res_smem2 = widen_budget(h, h->cluster2, h->tpb2, h->res_smem2);
    }
    if (split < h->nsys) {
        const int num = active_clusters(h, h->cluster, h->tpb, h->resident ? h->res_smem : 0);
        require(num > 0, XPLUS_ERR_CUDA, "cluster shape not launchable on this device");
        h->grid = num * h->cluster;
    } else {
        h->grid = 0;
    }
    if (split > 0) {
        const int num2 = active_clusters(h, h->cluster2, h->tpb2, h->resident ? h->res_smem2 : 0);
        require(num2 > 0, XPLUS_ERR_CUDA, "split cluster shape not launchable on this device");
        h->grid2 = std::min(num2, split) * h->cluster2;
    } else {
        h->grid2 = 0;
    }
}

// Runs `change` on the handle's launch settings and plans them; restores the previous
// settings when the new ones cannot launch.
template <typename F>
void replan(xplus_batch* h, F&& change) {
    const bool res0 = h->resident;
    const int c0 = h->cluster, t0 = h->tpb, s0 = h->split, c20 = h->cluster2, t20 = h->tpb2;
    change();
    try {
        plan(h);
    } catch (...) {
        h->resident = res0;
        h->cluster = c0;
        h->tpb = t0;
        h->split = s0;
        h->cluster2 = c20;
        h->tpb2 = t20;
        try {
            plan(h);
        } catch (...) {
        }
        throw;
    }
}

void set_split(xplus_batch* h, int count, int cluster, int tpb) {
    require(count >= 0 && count <= h->nsys, XPLUS_ERR_ARG, "split count must be in [0, nsys]");
    require(cluster == 4 || cluster == 8 || cluster == 16, XPLUS_ERR_ARG, "split cluster must be 4, 8 or 16");
    require(tpb == 128 || tpb == 256 || tpb == 512, XPLUS_ERR_ARG, "block_threads must be 128, 256 or 512");
    replan(h, [&] {
        h->split = count;
        if (count > 0) {
            h->cluster2 = cluster;
            h->tpb2 = tpb;
        }
    });
}

void set_launch(xplus_batch* h, int cluster, int tpb) {
    require(cluster == 1 || cluster == 2 || cluster == 4 || cluster == 8, XPLUS_ERR_ARG,
            "cluster must be 1, 2, 4 or 8");
    require(tpb == 128 || tpb == 256 || tpb == 512, XPLUS_ERR_ARG, "block_threads must be 128, 256 or 512");
    replan(h, [&] {
        h->cluster = cluster;
        h->tpb = tpb;
    });
}

// The resident kernel's records: [generation][{M r, M Ap', p'}][rows], allocated on first use.
void ensure_rec3(xplus_batch* h) {
    if (h->d_rec3) return;
    void* p = nullptr;
    const size_t bytes = 6 * sizeof(float) * static_cast<size_t>(h->rows);
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_NOMEM, "cudaMalloc (resident records)");
    }
    h->allocations.push_back(p);
    h->d_rec3 = static_cast<float*>(p);
    bcheck(cudaMemset(h->d_rec3, 0, bytes), "memset");
}

void set_resident(xplus_batch* h, bool on) {
    require(!on || h->res_kernel, XPLUS_ERR_ARG, "no resident batch kernel for these options");
    if (on) ensure_rec3(h);
    replan(h, [&] { h->resident = on; });
}

// f(k) for every system k, on the host's threads (system k on thread k mod T, which balances
// systems of mixed size); every call writes only system k's own output ranges.
template <typename F>
void for_each_system(int count, F&& f) {
    const int nt = std::max(1, std::min(count, std::min(32, static_cast<int>(std::thread::hardware_concurrency()))));
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&f, t, nt, count] {
            for (int k = t; k < count; k += nt) f(k);
        });
    for (auto& th : pool) th.join();
}

void batch_create(int nsys, const int* const* row_ptrs, const int* const* col_idxs,
                  const double* const* values, const int* ns, const xplus_opts* opts_in, xplus_batch** out) {
    require(nsys > 0 && row_ptrs && col_idxs && values && ns && out, XPLUS_ERR_ARG, "null argument or nsys <= 0");
    xplus_opts o;
    xplus_opts_default(&o);
    if (opts_in) o = *opts_in;
    require(o.value_type == XPLUS_F32 || o.value_type == XPLUS_BF16 || o.value_type == XPLUS_F16, XPLUS_ERR_ARG,
            "batch value_type must be F32, BF16 or F16");
    require(o.vector_type == XPLUS_F32, XPLUS_ERR_ARG, "batch vectors are FP32");
    require(o.slice_height == 32, XPLUS_ERR_ARG, "slice_height must be 32");
    require(o.chunk == 1 || o.chunk == 2 || o.chunk == 4, XPLUS_ERR_ARG, "chunk must be 1, 2 or 4");
    require(o.sigma >= 1, XPLUS_ERR_ARG, "sigma must be >= 1");
    require(o.restart_on_replace >= -1 && o.restart_on_replace <= 4, XPLUS_ERR_ARG, "restart_on_replace must be -1..4");
    for (int k = 0; k < nsys; ++k) {
        require(row_ptrs[k] && col_idxs[k] && values[k] && ns[k] > 0, XPLUS_ERR_ARG, "bad system " + std::to_string(k));
        validate_csr(ns[k], row_ptrs[k], col_idxs[k], row_ptrs[k][ns[k]]);
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_CUDA, "no CUDA device available (the solver has no CPU path)");
    }
    require(o.device >= 0 && o.device < count, XPLUS_ERR_ARG, "device ordinal out of range");
    cudaDeviceProp prop;
    bcheck(cudaGetDeviceProperties(&prop, o.device), "cudaGetDeviceProperties");
    require(prop.major == 10, XPLUS_ERR_CUDA, "this build targets sm_100 (B200) devices only");
    bcheck(cudaSetDevice(o.device), "cudaSetDevice");

    // per-system SELL images in parallel (row-sum form: off-diagonals in the slots)
    std::vector<SellHost> S(static_cast<size_t>(nsys));
    std::vector<std::vector<double>> diag(static_cast<size_t>(nsys));
    std::vector<double> scale16(static_cast<size_t>(nsys), 1.0);  // FP16: a_ij / scale16 stored
    const double split_ratio = split_ratio_of(o);
    std::vector<std::string> errs(static_cast<size_t>(nsys));
    std::vector<int> codes(static_cast<size_t>(nsys), 0);
    {
        const int nt = std::max(1, std::min<int>(nsys, static_cast<int>(std::thread::hardware_concurrency())));
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&, t] {
                for (int k = t; k < nsys; k += nt) {
                    try {
                        const size_t K = static_cast<size_t>(k);
                        diag[K].resize(static_cast<size_t>(ns[k]));
                        jacobi_diag(ns[k], row_ptrs[k], col_idxs[k], values[k], diag[K].data());
                        for (double d : diag[K])
                            require(std::fabs(d) > 1.0e-30, XPLUS_ERR_DATA, "zero diagonal entry while building Jacobi inverse");
                        if (o.value_type == XPLUS_F16)
                            scale16[K] = f16_offdiag_scale(ns[k], row_ptrs[k], col_idxs[k], values[k]);
                        // two-term entries for the large weights of cancelling rows (16-bit values)
                        TwoTermCsr two;
                        if (split_ratio > 0.0)
                            two_term_entries(ns[k], row_ptrs[k], col_idxs[k], values[k], o.value_type, scale16[K],
                                             split_ratio, two);
                        if (two.row_ptr.empty())
                            sell_build(ns[k], row_ptrs[k], col_idxs[k], values[k], 32, o.sigma, o.chunk, 1, S[K]);
                        else
                            sell_build(ns[k], two.row_ptr.data(), two.col_idx.data(), two.values.data(), 32, o.sigma,
                                       o.chunk, 1, S[K]);
                    } catch (const Error& e) {
                        codes[static_cast<size_t>(k)] = e.code;
                        errs[static_cast<size_t>(k)] = e.what();
                    } catch (const std::exception& e) {
                        codes[static_cast<size_t>(k)] = XPLUS_ERR_ARG;
                        errs[static_cast<size_t>(k)] = e.what();
                    }
                }
            });
        for (auto& th : pool) th.join();
        for (int k = 0; k < nsys; ++k)
            if (codes[static_cast<size_t>(k)]) throw Error(codes[static_cast<size_t>(k)], "system " + std::to_string(k) + ": " + errs[static_cast<size_t>(k)]);
    }

    auto* h = new xplus_batch();
    h->device = o.device;
    try {
        h->opts = o;
        h->nsys = nsys;
        h->sys_n.assign(ns, ns + nsys);
        h->sys_off.assign(static_cast<size_t>(nsys) + 1, 0);
        std::vector<int> slice0(static_cast<size_t>(nsys) + 1, 0);
        int64_t slots = 0;
        for (int k = 0; k < nsys; ++k) {
            const size_t K = static_cast<size_t>(k);
            h->sys_off[K + 1] = h->sys_off[K] + ns[k];
            require(static_cast<int64_t>(slice0[K]) + S[K].n_slices < (1LL << 26), XPLUS_ERR_ARG, "batch too large");
            slice0[K + 1] = slice0[K] + S[K].n_slices;
            slots += S[K].slots;
            h->total_nnz += row_ptrs[k][ns[k]];
        }
        h->total_n = h->sys_off[static_cast<size_t>(nsys)];
        h->n_slices = slice0[static_cast<size_t>(nsys)];
        h->rows = h->n_slices * 32;
        h->slots = slots;
        require(slots < (1LL << 31) && h->total_n < (1LL << 31), XPLUS_ERR_ARG, "batch too large (2^31 slots)");
        // int16 offsets when every system's ordered bandwidth allows
        bool idx16 = o.index16 != 0;
        const int ch = o.chunk;
        // slot (j/chunk) 32 chunk + lane chunk + j%chunk of slice sl belongs to row 32 sl + lane
        auto for_each_slot = [ch](const SellHost& s, auto&& g) {
            for (int sl = 0; sl < s.n_slices; ++sl) {
                const int64_t b0 = s.slice_ptr[static_cast<size_t>(sl)];
                const int64_t groups = (s.slice_ptr[static_cast<size_t>(sl) + 1] - b0) / (32 * ch);
                for (int64_t jg = 0; jg < groups; ++jg)
                    for (int lane = 0; lane < 32; ++lane)
                        for (int q = 0; q < ch; ++q) g(sl, lane, b0 + jg * 32 * ch + lane * ch + q);
            }
        };
        if (idx16) {
            std::vector<unsigned char> far(static_cast<size_t>(nsys), 0);
            for_each_system(nsys, [&](int k) {
                const SellHost& s = S[static_cast<size_t>(k)];
                for_each_slot(s, [&](int sl, int lane, int64_t pos) {
                    const int d = s.col[static_cast<size_t>(pos)] - (sl * 32 + lane);
                    if (d < -32768 || d > 32767) far[static_cast<size_t>(k)] = 1;
                });
            });
            for (unsigned char f : far)
                if (f) idx16 = false;
        }
        h->idx16 = idx16;
        h->kernel = pick_kernel(o.value_type, o.chunk, idx16, false);
        h->kernel_small = pick_kernel(o.value_type, o.chunk, idx16, true);
        require(h->kernel != nullptr && h->kernel_small != nullptr, XPLUS_ERR_ARG, "no batch kernel for these options");
        // clusters of 16 CTAs (beyond the portable 8) for the lane of the largest systems
        for (BatchKernel k : {h->kernel, h->kernel_small})
            if (cudaFuncSetAttribute(reinterpret_cast<const void*>(k), cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                cudaSuccess)
                cudaGetLastError();  // then 16 is simply not launchable (active_clusters returns 0)
        // the cluster-resident kernel: as much dynamic shared memory as a CTA may have
        h->res_kernel = batch_resident_kernel(o.value_type, o.chunk, idx16);
        if (h->res_kernel) {
            int optin = 0;
            const int st = batch_resident_static_smem(h->res_kernel);
            const void* fk = reinterpret_cast<const void*>(h->res_kernel);
            if (st < 0 || cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, o.device) != cudaSuccess ||
                cudaFuncSetAttribute(fk, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - st) != cudaSuccess) {
                cudaGetLastError();
                h->res_kernel = nullptr;
            } else {
                h->res_max_dyn = optin - st;
                int per_sm = 0;
                if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, o.device) == cudaSuccess)
                    h->res_half = std::max(0, per_sm / 2 - st - 1024);  // 1 KB per CTA is the system's
                else
                    cudaGetLastError();
                if (cudaFuncSetAttribute(fk, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
                    cudaGetLastError();
            }
        }
        // the resident kernel's shared memory per CTA for every system and cluster size of 1 to
        // 16: the band split and the column window (every slot's column, padding included,
        // widened to float4 groups) that the kernel itself computes
        for (auto& v : h->need) v.assign(static_cast<size_t>(nsys), 0);
        for_each_system(nsys, [&](int k) {
            const SellHost& s = S[static_cast<size_t>(k)];
            const int nsl_all = s.n_slices;
            std::vector<int> smin(static_cast<size_t>(nsl_all)), smax(static_cast<size_t>(nsl_all));
            for (int sl = 0; sl < nsl_all; ++sl) {
                int lo = sl * 32, hi = sl * 32 + 32;
                for (int64_t pos = s.slice_ptr[static_cast<size_t>(sl)]; pos < s.slice_ptr[static_cast<size_t>(sl) + 1]; ++pos) {
                    lo = std::min(lo, s.col[static_cast<size_t>(pos)]);
                    hi = std::max(hi, s.col[static_cast<size_t>(pos)] + 1);
                }
                smin[static_cast<size_t>(sl)] = lo;
                smax[static_cast<size_t>(sl)] = hi;
            }
            for (int li = 0; li < 5; ++li) {
                const int cs = 1 << li;
                const int per = (nsl_all + cs - 1) / cs;
                long long worst = 0;
                for (int rk = 0; rk < cs; ++rk) {
                    const int sb = std::min(nsl_all, rk * per), se = std::min(nsl_all, (rk + 1) * per);
                    const int nsl = se - sb, r0 = sb * 32, nb = nsl * 32;
                    int cmin = r0, cmax = r0 + nb;
                    for (int sl = sb; sl < se; ++sl) {
                        cmin = std::min(cmin, smin[static_cast<size_t>(sl)]);
                        cmax = std::max(cmax, smax[static_cast<size_t>(sl)]);
                    }
                    const int w0 = std::max(0, cmin & ~3);
                    const int wend = std::min(nsl_all * 32, (cmax + 3) & ~3);
                    const long long need = ((nsl * 8LL + 15) & ~15LL) + 4LL * ((wend - w0) + 5LL * nb);
                    worst = std::max(worst, need);
                }
                h->need[li][static_cast<size_t>(k)] = static_cast<int>(std::min<long long>(worst, 1LL << 30));
            }
        });

        // concatenated host image
        const size_t R = static_cast<size_t>(h->rows);
        std::vector<long long> sp(static_cast<size_t>(h->n_slices) + 1, 0);
        std::vector<int> col32;
        std::vector<short> col16;
        if (idx16) col16.resize(static_cast<size_t>(slots));
        else col32.resize(static_cast<size_t>(slots));
        std::vector<double> v64(static_cast<size_t>(slots));
        std::vector<double> d64(R, 0.0), rs(R, 0.0), mi(R, 0.0);
        std::vector<int> map(R, -1);
        std::vector<float> scale(static_cast<size_t>(nsys), 1.0f);
        std::vector<unsigned char> vbytes(static_cast<size_t>(slots) * (o.value_type == XPLUS_F32 ? 4 : 2));
        std::vector<int64_t> sys_base(static_cast<size_t>(nsys) + 1, 0);
        for (int k = 0; k < nsys; ++k) sys_base[static_cast<size_t>(k) + 1] = sys_base[static_cast<size_t>(k)] + S[static_cast<size_t>(k)].slots;
        const int64_t base = sys_base[static_cast<size_t>(nsys)];
        for_each_system(nsys, [&](int k) {
            const size_t K = static_cast<size_t>(k);
            const SellHost& s = S[K];
            const int64_t b0 = sys_base[K];
            const int r0 = slice0[K] * 32;
            for (int sl = 0; sl < s.n_slices; ++sl)
                sp[static_cast<size_t>(slice0[K] + sl)] = b0 + s.slice_ptr[static_cast<size_t>(sl)];
            const double sc = scale16[K];
            scale[K] = static_cast<float>(sc);
            for_each_slot(s, [&](int sl, int lane, int64_t pos) {
                const size_t gpos = static_cast<size_t>(b0 + pos);
                const int c = s.col[static_cast<size_t>(pos)];
                if (idx16) col16[gpos] = static_cast<short>(c - (sl * 32 + lane));
                else col32[gpos] = r0 + c;
                const double v = s.val[static_cast<size_t>(pos)];
                v64[gpos] = v;
                if (o.value_type == XPLUS_F32) reinterpret_cast<float*>(vbytes.data())[gpos] = static_cast<float>(v);
                else if (o.value_type == XPLUS_F16) reinterpret_cast<__half*>(vbytes.data())[gpos] = __double2half(v / sc);
                else reinterpret_cast<__nv_bfloat16*>(vbytes.data())[gpos] = __double2bfloat16(v);
            });
            for (int i = 0; i < s.n; ++i) {
                const int old = s.perm[static_cast<size_t>(i)];
                const size_t gi = static_cast<size_t>(r0 + i);
                const double d = diag[K][static_cast<size_t>(old)];
                d64[gi] = d;
                mi[gi] = 1.0 / d;
                double acc = 0.0;
                for (int q = row_ptrs[k][old]; q < row_ptrs[k][old + 1]; ++q) acc += values[k][q];
                rs[gi] = acc;
                map[gi] = static_cast<int>(h->sys_off[K] + old);
            }
        });
        sp[static_cast<size_t>(h->n_slices)] = base;
        // queue: largest first by nnz * sqrt(n) (PCG iterations grow like sqrt(n) on these grids)
        std::vector<int> order(static_cast<size_t>(nsys));
        for (int k = 0; k < nsys; ++k) order[static_cast<size_t>(k)] = k;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            const double wa = static_cast<double>(row_ptrs[a][ns[a]]) * std::sqrt(static_cast<double>(ns[a]));
            const double wb = static_cast<double>(row_ptrs[b][ns[b]]) * std::sqrt(static_cast<double>(ns[b]));
            return wa > wb;
        });

        h->order = order;
        bcheck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        bcheck(cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking), "cudaStreamCreate");
        bcheck(cudaEventCreate(&h->ev0), "cudaEventCreate");
        bcheck(cudaEventCreate(&h->ev1), "cudaEventCreate");
        bcheck(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming), "cudaEventCreate");
        bcheck(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming), "cudaEventCreate");
        std::vector<int> sysn(ns, ns + nsys);
        std::vector<float> rsf(rs.begin(), rs.end()), mif(mi.begin(), mi.end());
        h->d_order = balloc<int>(h, order.size());
        h->d_head = balloc<int>(h, 2);
        h->d_slice0 = balloc<int>(h, slice0.size());
        h->d_sysn = balloc<int>(h, sysn.size());
        h->d_scale = balloc<float>(h, scale.size());
        h->d_slice_ptr = balloc<long long>(h, sp.size());
        h->d_col = balloc<unsigned char>(h, static_cast<size_t>(slots) * (idx16 ? 2 : 4));
        h->d_val = balloc<unsigned char>(h, vbytes.size());
        h->d_val64 = balloc<double>(h, v64.size());
        h->d_diag64 = balloc<double>(h, R);
        h->d_rowsum = balloc<float>(h, R);
        h->d_minv = balloc<float>(h, R);
        h->d_map = balloc<int>(h, R);
        h->d_b64 = balloc<double>(h, R);
        h->d_x64 = balloc<double>(h, R);
        h->d_rec = balloc<NodeRec<float>>(h, R);
        h->d_r = balloc<float>(h, R);
        h->d_ap = balloc<float>(h, R);
        h->d_bio = balloc<double>(h, static_cast<size_t>(h->total_n));
        h->d_xio = balloc<double>(h, static_cast<size_t>(h->total_n));
        h->d_status = balloc<int>(h, static_cast<size_t>(nsys));
        h->d_iters = balloc<int>(h, static_cast<size_t>(nsys));
        h->d_repl = balloc<int>(h, static_cast<size_t>(nsys));
        h->d_true_rel = balloc<double>(h, static_cast<size_t>(nsys));
        h->d_ns = balloc<long long>(h, static_cast<size_t>(nsys));
        h->d_staged = balloc<int>(h, static_cast<size_t>(nsys));
        upload(h, h->d_order, order);
        upload(h, h->d_slice0, slice0);
        upload(h, h->d_sysn, sysn);
        upload(h, h->d_scale, scale);
        upload(h, h->d_slice_ptr, sp);
        if (idx16) upload(h, static_cast<short*>(h->d_col), col16);
        else upload(h, static_cast<int*>(h->d_col), col32);
        upload(h, static_cast<unsigned char*>(h->d_val), vbytes);
        upload(h, h->d_val64, v64);
        upload(h, h->d_diag64, d64);
        upload(h, h->d_rowsum, rsf);
        upload(h, h->d_minv, mif);
        upload(h, h->d_map, map);
        bcheck(cudaMemsetAsync(h->d_x64, 0, R * sizeof(double), h->stream), "memset");
        bcheck(cudaMemsetAsync(h->d_rec, 0, R * sizeof(NodeRec<float>), h->stream), "memset");
        bcheck(cudaMemsetAsync(h->d_staged, 0, static_cast<size_t>(nsys) * sizeof(int), h->stream), "memset");
        bcheck(cudaStreamSynchronize(h->stream), "sync");
        set_launch(h, 4, 512);
        *out = h;
    } catch (...) {
        batch_destroy(h);
        throw;
    }
}

// Enqueues head reset, the persistent launch (no gather / scatter): b64 and x64 are set.
void enqueue_kernel(xplus_batch* h, double tau, int tau_mode, int max_iters, int cluster, int tpb, int grid,
                    cudaStream_t st) {
    BatchArgs a{};
    a.nsys = h->nsys;
    a.order = h->d_order;
    a.head = h->d_head;
    a.sys_slice0 = h->d_slice0;
    a.sys_n = h->d_sysn;
    a.sys_scale = h->d_scale;
    a.slice_ptr = h->d_slice_ptr;
    a.col = h->d_col;
    a.val = h->d_val;
    a.val64 = h->d_val64;
    a.diag64 = h->d_diag64;
    a.rowsum = h->d_rowsum;
    a.minv = h->d_minv;
    a.b64 = h->d_b64;
    a.x64 = h->d_x64;
    a.rec = static_cast<NodeRec<float>*>(h->d_rec);
    a.r = h->d_r;
    a.ap = h->d_ap;
    a.rec3 = h->d_rec3;
    a.rows = h->rows;
    a.tau = tau;
    a.tau_mode = tau_mode;
    a.max_iters = max_iters;
    a.replace_every = h->opts.replace_every;
    a.replace_drop2 = h->opts.replace_drop > 0.0 ? h->opts.replace_drop * h->opts.replace_drop : 0.0;
    const bool low = h->opts.value_type != XPLUS_F32;
    a.restart_on_replace = h->opts.restart_on_replace < 0 ? (low ? 4 : 0) : h->opts.restart_on_replace;
    stagnation_args(h->opts, &a.stag_factor, &a.stag_window);
    a.out_status = h->d_status;
    a.out_iters = h->d_iters;
    a.out_repl = h->d_repl;
    a.out_true_rel = h->d_true_rel;
    a.out_ns = h->d_ns;
    a.stage_matrix = h->stage_matrix ? 1 : 0;
    a.out_staged = h->d_staged;
    bcheck(cudaMemsetAsync(h->d_head, 0, 2 * sizeof(int), st), "memset");
    auto launch = [&](const BatchArgs& args, int c, int t, int g, cudaStream_t s, int priority, const char* what) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(g);
        cfg.blockDim = dim3(t);
        cfg.dynamicSmemBytes = h->resident ? static_cast<size_t>(args.res_smem) : 0;
        cfg.stream = s;
        cudaLaunchAttribute attr[2];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        attr[1].id = cudaLaunchAttributePriority;
        attr[1].val.priority = priority;
        cfg.attrs = attr;
        cfg.numAttrs = 2;
        bcheck(cudaLaunchKernelEx(&cfg, kernel_for(h, t), args), what);
    };
    int prio_low = 0, prio_high = 0;  // numerically lower is higher priority
    bcheck(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high), "priority range");
    const int split = std::min(h->split, h->nsys);
    if (split > 0) {
        // the largest systems first, on the second stream (fork / join through events, which
        // stream capture turns into parallel graph branches); no wait crosses the launches
        BatchArgs big = a;
        big.q_begin = 0;
        big.q_end = split;
        big.head = h->d_head + 1;
        big.res_smem = h->res_smem2;
        bcheck(cudaEventRecord(h->ev_fork, st), "event");
        bcheck(cudaStreamWaitEvent(h->stream2, h->ev_fork, 0), "wait");
        // the highest priority: when SMs free up, the CTA scheduler places this launch's
        // clusters before the main launch's, so the largest systems get SMs of their own early
        launch(big, h->cluster2, h->tpb2, h->grid2, h->stream2, prio_high, "batch PCG launch (largest systems)");
        bcheck(cudaEventRecord(h->ev_join, h->stream2), "event");
    }
    a.q_begin = split;
    a.q_end = h->nsys;
    a.res_smem = h->res_smem;
    if (split < h->nsys) launch(a, cluster, tpb, grid, st, prio_low, "batch PCG launch");
    if (split > 0) bcheck(cudaStreamWaitEvent(st, h->ev_join, 0), "wait");
}

void check_tau(double tau, int tau_mode) {
    require(tau > 0.0 && tau == tau, XPLUS_ERR_ARG, "tau must be positive");
    require(tau_mode == XPLUS_TAU_ABS_RR || tau_mode == XPLUS_TAU_REL_TRUE, XPLUS_ERR_ARG, "bad tau_mode");
}

// gather b and x (device, original order), solve, scatter x back
void enqueue_solve(xplus_batch* h, const double* d_b, double* d_x, double tau, int tau_mode, int max_iters,
                   cudaStream_t st) {
    const int threads = 256, blocks = (h->rows + threads - 1) / threads;
    batch_gather_kernel<<<blocks, threads, 0, st>>>(d_b, h->d_b64, h->d_map, h->rows);
    bcheck(cudaGetLastError(), "gather");
    batch_gather_kernel<<<blocks, threads, 0, st>>>(d_x, h->d_x64, h->d_map, h->rows);
    bcheck(cudaGetLastError(), "gather");
    enqueue_kernel(h, tau, tau_mode, max_iters, h->cluster, h->tpb, h->grid, st);
    batch_scatter_kernel<<<blocks, threads, 0, st>>>(h->d_x64, d_x, h->d_map, h->rows);
    bcheck(cudaGetLastError(), "scatter");
}

void collect(xplus_batch* h) {
    if (!h->pending) return;
    bcheck(cudaEventSynchronize(h->ev1), "sync");
    float ms = 0.0f;
    bcheck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "event");
    h->last_ms = ms;
    h->pending = false;
}

}  // namespace
}  // namespace xplus

using namespace xplus;

extern "C" {

int xplus_batch_create(int nsys, const int* const* row_ptrs, const int* const* col_idxs,
                       const double* const* values, const int* ns, const xplus_opts* opts,
                       xplus_batch** out) {
    return guarded([&] { batch_create(nsys, row_ptrs, col_idxs, values, ns, opts, out); });
}

int xplus_batch_destroy(xplus_batch* h) {
    return guarded([&] { batch_destroy(h); });
}

int xplus_batch_set_launch(xplus_batch* h, int cluster, int block_threads) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        bcheck(cudaSetDevice(h->device), "cudaSetDevice");
        set_launch(h, cluster, block_threads);
    });
}

int xplus_batch_set_split(xplus_batch* h, int count, int cluster, int block_threads) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        bcheck(cudaSetDevice(h->device), "cudaSetDevice");
        set_split(h, count, cluster, block_threads);
    });
}

int xplus_batch_solve(xplus_batch* h, const double* b, const double* x0, double tau, int tau_mode,
                      int max_iters, double* x_out) {
    return guarded([&] {
        require(h && b && x_out, XPLUS_ERR_ARG, "null argument");
        check_tau(tau, tau_mode);
        bcheck(cudaSetDevice(h->device), "cudaSetDevice");
        cudaStream_t st = h->stream;
        const size_t nb = sizeof(double) * static_cast<size_t>(h->total_n);
        bcheck(cudaMemcpyAsync(h->d_bio, b, nb, cudaMemcpyHostToDevice, st), "H2D");
        if (x0) bcheck(cudaMemcpyAsync(h->d_xio, x0, nb, cudaMemcpyHostToDevice, st), "H2D");
        else bcheck(cudaMemsetAsync(h->d_xio, 0, nb, st), "memset");
        bcheck(cudaEventRecord(h->ev0, st), "event");
        enqueue_solve(h, h->d_bio, h->d_xio, tau, tau_mode, max_iters, st);
        h->have_b = true;
        bcheck(cudaEventRecord(h->ev1, st), "event");
        h->pending = true;
        bcheck(cudaMemcpyAsync(x_out, h->d_xio, nb, cudaMemcpyDeviceToHost, st), "D2H");
        bcheck(cudaStreamSynchronize(st), "sync");
        collect(h);
    });
}

int xplus_batch_solve_device(xplus_batch* h, const double* d_b, double* d_x, double tau, int tau_mode,
                             int max_iters, void* stream) {
    return guarded([&] {
        require(h && d_b && d_x, XPLUS_ERR_ARG, "null argument");
        check_tau(tau, tau_mode);
        bcheck(cudaSetDevice(h->device), "cudaSetDevice");
        require_device_memory(d_b, h->device, "d_b");
        require_device_memory(d_x, h->device, "d_x");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : h->stream;
        const bool same = h->gexec && h->g_b == d_b && h->g_x == d_x && h->g_tau == tau && h->g_mode == tau_mode &&
                          h->g_iters == max_iters && h->g_cluster == h->cluster && h->g_tpb == h->tpb &&
                          h->g_split == h->split && h->g_cluster2 == h->cluster2 && h->g_tpb2 == h->tpb2 &&
                          h->g_resident == h->resident && h->g_stage == h->stage_matrix;
        if (!same) {
            if (h->gexec) {
                bcheck(cudaGraphExecDestroy(h->gexec), "graph destroy");
                h->gexec = nullptr;
            }
            // capture on the handle's own stream; the executable graph runs on any stream
            bcheck(cudaStreamSynchronize(h->stream), "sync");
            bcheck(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            cudaGraph_t graph = nullptr;
            try {
                enqueue_solve(h, d_b, d_x, tau, tau_mode, max_iters, h->stream);
            } catch (...) {
                cudaStreamEndCapture(h->stream, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            bcheck(cudaStreamEndCapture(h->stream, &graph), "end capture");
            const cudaError_t e = cudaGraphInstantiate(&h->gexec, graph, 0);
            cudaGraphDestroy(graph);
            bcheck(e, "graph instantiate");
            h->g_b = d_b;
            h->g_x = d_x;
            h->g_tau = tau;
            h->g_mode = tau_mode;
            h->g_iters = max_iters;
            h->g_cluster = h->cluster;
            h->g_tpb = h->tpb;
            h->g_split = h->split;
            h->g_cluster2 = h->cluster2;
            h->g_tpb2 = h->tpb2;
            h->g_resident = h->resident;
            h->g_stage = h->stage_matrix;
        }
        bcheck(cudaEventRecord(h->ev0, st), "event");
        bcheck(cudaGraphLaunch(h->gexec, st), "graph launch");
        h->have_b = true;
        bcheck(cudaEventRecord(h->ev1, st), "event");
        h->pending = true;
    });
}

int xplus_batch_results(xplus_batch* h, int* status, int* iterations, int* replacements, double* true_rel,
                        double* system_ms, double* kernel_ms) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        bcheck(cudaSetDevice(h->device), "cudaSetDevice");
        collect(h);
        const size_t K = static_cast<size_t>(h->nsys);
        std::vector<int> its(K);
        bcheck(cudaMemcpy(its.data(), h->d_iters, K * sizeof(int), cudaMemcpyDeviceToHost), "D2H");
        for (size_t k = 0; k < K; ++k)
            require(its[k] >= 0, XPLUS_ERR_CUDA,
                    "system " + std::to_string(k) + " did not fit the resident launch's shared memory (not solved)");
        if (status) bcheck(cudaMemcpy(status, h->d_status, K * sizeof(int), cudaMemcpyDeviceToHost), "D2H");
        if (iterations) std::copy(its.begin(), its.end(), iterations);
        if (replacements) bcheck(cudaMemcpy(replacements, h->d_repl, K * sizeof(int), cudaMemcpyDeviceToHost), "D2H");
        if (true_rel) bcheck(cudaMemcpy(true_rel, h->d_true_rel, K * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
        if (system_ms) {
            std::vector<long long> t(K);
            bcheck(cudaMemcpy(t.data(), h->d_ns, K * sizeof(long long), cudaMemcpyDeviceToHost), "D2H");
            for (size_t k = 0; k < K; ++k) system_ms[k] = static_cast<double>(t[k]) * 1e-6;
        }
        if (kernel_ms) *kernel_ms = h->last_ms;
    });
}

int xplus_batch_autotune(xplus_batch* h, int iters, double tau, int* cluster, int* block_threads,
                         double* best_ms) {
    return guarded([&] {
        require(h && (iters > 0 || (tau > 0.0 && tau < 1.0)), XPLUS_ERR_ARG, "bad argument");
        bcheck(cudaSetDevice(h->device), "cudaSetDevice");
        cudaStream_t st = h->stream;
        // x = 0 for every system; either a fixed number of iterations per system on b = 1 (an
        // absolute tolerance no system reaches, so every shape does the same work), or every
        // system solved to the FP64 true relative residual tau (the makespan that matters), on
        // the right-hand side of the last solve when there was one (b = 1 otherwise): how fast
        // each system converges depends on b, and so does the best shape
        const bool fixed = iters > 0;
        const bool last_b = !fixed && h->have_b;
        std::vector<double> ones(static_cast<size_t>(h->rows), 0.0), saved;
        std::vector<int> map(static_cast<size_t>(h->rows));
        bcheck(cudaMemcpy(map.data(), h->d_map, map.size() * sizeof(int), cudaMemcpyDeviceToHost), "D2H");
        for (size_t i = 0; i < map.size(); ++i) ones[i] = map[i] >= 0 ? 1.0 : 0.0;
        if (last_b) {
            bcheck(cudaStreamSynchronize(st), "sync");
            bcheck(cudaMemcpy(ones.data(), h->d_b64, ones.size() * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
        }
        // best of two launches with the handle's current settings
        auto time_current = [&]() {
            double ms_min = 1e300;
            for (int rep = 0; rep < 2; ++rep) {
                bcheck(cudaMemcpyAsync(h->d_b64, ones.data(), ones.size() * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
                bcheck(cudaMemsetAsync(h->d_x64, 0, ones.size() * sizeof(double), st), "memset");
                bcheck(cudaEventRecord(h->ev0, st), "event");
                if (fixed) enqueue_kernel(h, 1e-300, XPLUS_TAU_ABS_RR, iters, h->cluster, h->tpb, h->grid, st);
                else enqueue_kernel(h, tau, XPLUS_TAU_REL_TRUE, 0, h->cluster, h->tpb, h->grid, st);
                bcheck(cudaEventRecord(h->ev1, st), "event");
                bcheck(cudaEventSynchronize(h->ev1), "sync");
                float ms = 0.0f;
                bcheck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "event");
                ms_min = std::min(ms_min, static_cast<double>(ms));
            }
            return ms_min;
        };
        struct Cfg {
            bool res;
            int c, t, k, c2, t2;
        };
        auto apply = [&](const Cfg& q) {
            try {
                replan(h, [&] {
                    h->resident = q.res;
                    h->cluster = q.c;
                    h->tpb = q.t;
                    h->split = q.k;
                    if (q.k > 0) {
                        h->cluster2 = q.c2;
                        h->tpb2 = q.t2;
                    }
                });
                return true;
            } catch (const Error&) {
                return false;  // not launchable, or a system does not fit: not a candidate
            }
        };
        double best = 1e300;
        Cfg bestc{false, h->cluster, h->tpb, 0, h->cluster2, h->tpb2};
        auto trial = [&](const Cfg& q) {
            if (!apply(q)) return;
            const double ms = time_current();
            if (ms < best) {
                best = ms;
                bestc = q;
            }
        };
        // stage 1: the global-memory kernel's main shape, every system in the main launch
        for (int c : {1, 2, 4, 8})
            for (int t : {128, 256, 512}) trial(Cfg{false, c, t, 0, 16, 512});
        require(best < 1e300, XPLUS_ERR_CUDA, "no launchable cluster shape");
        // stage 2: on that shape, the largest systems in a lane of their own with bigger clusters
        // (the largest system otherwise sets the makespan on its own)
        {
            const Cfg g = bestc;
            for (int k : {1, 2, 4, 8, 16}) {
                if (k > h->nsys / 4) break;
                for (const auto& sh : {std::make_pair(16, 512), std::make_pair(8, 512), std::make_pair(16, 256)})
                    trial(Cfg{false, g.c, g.t, k, sh.first, sh.second});
            }
        }
        // stage 3: the cluster-resident kernel.  Main launches of 2, 4 or 8 CTAs; the systems
        // whose bands do not fit the main launch's shared-memory budget (all a CTA may have, or
        // what lets two CTAs share an SM) go to a split launch of 16-CTA clusters, largest first
        if (h->res_kernel) {
            ensure_rec3(h);
            const int half = h->res_half;
            for (int c : {2, 4, 8}) {
                // suffix maxima of the needs in queue order: the main launch takes [k, nsys)
                const std::vector<int>& nd = h->need[log2_cluster(c)];
                std::vector<int> suf(static_cast<size_t>(h->nsys) + 1, 0);
                for (int q = h->nsys - 1; q >= 0; --q)
                    suf[static_cast<size_t>(q)] = std::max(suf[static_cast<size_t>(q) + 1],
                                                           nd[static_cast<size_t>(h->order[static_cast<size_t>(q)])]);
                int last_k = -1;
                for (int budget : {h->res_max_dyn, half}) {
                    int k = 0;
                    while (k < h->nsys && suf[static_cast<size_t>(k)] > budget) ++k;
                    if (k == last_k || k >= h->nsys) continue;
                    last_k = k;
                    for (int t : {256, 512}) {
                        if (k == 0) trial(Cfg{true, c, t, 0, 16, 512});
                        else
                            for (int t2 : {256, 512}) trial(Cfg{true, c, t, k, 16, t2});
                    }
                }
            }
        }
        require(apply(bestc), XPLUS_ERR_CUDA, "the autotuner's best shape no longer launches");
        const int bc = bestc.c, bt = bestc.t;
        if (cluster) *cluster = bc;
        if (block_threads) *block_threads = bt;
        if (best_ms) *best_ms = best;
    });
}

int xplus_batch_set_resident(xplus_batch* h, int on) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        bcheck(cudaSetDevice(h->device), "cudaSetDevice");
        set_resident(h, on != 0);
    });
}

int xplus_batch_set_stage_matrix(xplus_batch* h, int on) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        bcheck(cudaSetDevice(h->device), "cudaSetDevice");
        const bool s0 = h->stage_matrix;
        try {
            replan(h, [&] { h->stage_matrix = on != 0; });
        } catch (...) {
            h->stage_matrix = s0;
            throw;
        }
    });
}

int xplus_batch_staged_info(xplus_batch* h, int* on, int* systems_all, int* systems_some) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        bcheck(cudaSetDevice(h->device), "cudaSetDevice");
        if (on) *on = h->stage_matrix ? 1 : 0;
        int all = 0, some = 0;
        if (h->resident) {
            collect(h);
            std::vector<int> st(static_cast<size_t>(h->nsys));
            bcheck(cudaMemcpy(st.data(), h->d_staged, st.size() * sizeof(int), cudaMemcpyDeviceToHost), "D2H");
            const int split = std::min(h->split, h->nsys);
            for (int q = 0; q < h->nsys; ++q) {
                const int k = st[static_cast<size_t>(h->order[static_cast<size_t>(q)])];
                const int cs = q < split ? h->cluster2 : h->cluster;
                if (k >= cs) ++all;
                else if (k > 0) ++some;
            }
        }
        if (systems_all) *systems_all = all;
        if (systems_some) *systems_some = some;
    });
}

int xplus_batch_resident_info(xplus_batch* h, int* on, int* smem, int* smem_split) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        if (on) *on = h->resident ? 1 : 0;
        if (smem) *smem = h->resident ? h->res_smem : 0;
        if (smem_split) *smem_split = h->resident && h->split > 0 ? h->res_smem2 : 0;
    });
}

int xplus_batch_split_info(xplus_batch* h, int* count, int* cluster, int* block_threads, int* grid) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        if (count) *count = h->split;
        if (cluster) *cluster = h->cluster2;
        if (block_threads) *block_threads = h->tpb2;
        if (grid) *grid = h->split > 0 ? h->grid2 : 0;
    });
}

int xplus_batch_info(xplus_batch* h, int64_t* total_n, int64_t* total_nnz, int* cluster, int* block_threads,
                     int* grid, int64_t* spmv_bytes) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        if (total_n) *total_n = h->total_n;
        if (total_nnz) *total_nnz = h->total_nnz;
        if (cluster) *cluster = h->cluster;
        if (block_threads) *block_threads = h->tpb;
        if (grid) *grid = h->grid;
        if (spmv_bytes) {
            // one SpMV over every system in the stored format, padding excluded: off-diagonal
            // entries (value + index), row sums, x read and y written
            const int64_t sv = h->opts.value_type == XPLUS_F32 ? 4 : 2;
            const int64_t si = h->idx16 ? 2 : 4;
            *spmv_bytes = (h->total_nnz - h->total_n) * (sv + si) + h->total_n * 12;
        }
    });
}

}  // extern "C"
