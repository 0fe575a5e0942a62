// batch_common.cuh -- what the batched solver's two kernels share: the launch arguments, the
// cluster-wide sums and the FP64 row product of the residual replacement.
//   pcg_batch_kernel      (batch.cu): vectors in global memory, two cluster barriers per iteration
//   pcg_batch_res_kernel  (batch_resident.cu): each CTA keeps its band's vectors and the search
//                         direction's window in shared memory, one cluster barrier per iteration
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "pcg_device.cuh"

namespace xplus {

namespace cg = cooperative_groups;

struct BatchArgs {
    int nsys;
    int q_begin, q_end;       // this launch takes queue positions [q_begin, q_end)
    const int* order;         // queue: system ids in the order they are taken
    int* head;                // this launch's queue head (atomic), zero at launch
    const int* sys_slice0;    // [nsys + 1] first global slice of each system
    const int* sys_n;         // rows of each system
    const float* sys_scale;   // stored off-diagonal value = a_ij / scale (FP16), else 1
    const long long* slice_ptr;
    const void* col;          // int32 global rows or int16 offsets from the row
    const void* val;          // off-diagonal weights (row-sum form), VT
    const double* val64;      // FP64 copy of the off-diagonals, same layout
    const double* diag64;     // FP64 diagonal
    const float* rowsum;      // s_i = sum_j a_ij
    const float* minv;        // 1 / a_ii
    const double* b64;
    double* x64;
    dev::NodeRec<float>* rec; // {z, p} per row (global-memory kernel)
    float* r;
    float* ap;
    float* rec3;              // resident kernel: [generation][{M r, M Ap', p'}][rows]
    int rows;                 // concatenated SELL rows (padding included)
    int res_smem;             // resident kernel: dynamic shared memory of the launch (bytes)
    int stage_matrix;         // resident kernel: copy a band's matrix into shared memory when it fits
    int* out_staged;          // resident kernel: CTAs of the system's cluster that staged their band
    double tau;
    int tau_mode;             // XPLUS_TAU_ABS_RR | XPLUS_TAU_REL_TRUE
    int max_iters;            // <= 0: max(4n, 1000) per system
    int replace_every;
    double replace_drop2;     // squared ||r|| drop that triggers a replacement (0: off)
    int restart_on_replace;   // ReplacePolicy: 0 keep p, 1 / 2 restart, 3 / 4 adaptive
    double stag_factor;
    int stag_window;
    int* out_status;
    int* out_iters;           // -1: the system did not fit the resident launch (not solved)
    int* out_repl;
    double* out_true_rel;
    long long* out_ns;        // device time of each system (first pop to exit residual)
};

using BatchKernel = void (*)(BatchArgs);

__device__ __forceinline__ dev::NodeRec<float> ldcg_rec(const dev::NodeRec<float>* q) {
    const float2 v = __ldcg(reinterpret_cast<const float2*>(q));
    return dev::NodeRec<float>{v.x, v.y};
}

// Sum of NV per-thread values over the cluster: block tree, then the per-CTA partials read
// through distributed shared memory in rank order (same result in every CTA).  Two banks of
// partials: a CTA that runs ahead writes the other bank, and a bank is rewritten only after
// the next cluster barrier, by which time every reader has finished with it.
template <int NV>
__device__ __forceinline__ void cluster_sum(cg::cluster_group& cl, double (&v)[NV], double* s_red,
                                            double (*s_part)[4], double* s_tot, int& pbank) {
    dev::block_sum<NV>(v, s_red);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) s_part[pbank][q] = v[q];
    cl.sync();
    if (threadIdx.x < NV) {
        const int cs = static_cast<int>(cl.num_blocks());
        double t = 0.0;
        for (int rk = 0; rk < cs; ++rk) t += *cl.map_shared_rank(&s_part[pbank][threadIdx.x], rk);
        s_tot[threadIdx.x] = t;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = s_tot[q];
    pbank ^= 1;
}

// FP64 row of A times x: stored off-diagonals (FP64 copy) plus the exact diagonal.  x of
// neighbouring rows is read through L2 (another CTA of the cluster wrote it).
template <int CHUNK, typename IT>
__device__ __forceinline__ double batch_row64(const BatchArgs& a, int s, int lane) {
    const long long base = a.slice_ptr[s];
    const int w = static_cast<int>((a.slice_ptr[s + 1] - base) >> 5);
    const int row = s * 32 + lane;
    const double* vp = a.val64 + base + lane * CHUNK;
    const IT* cp = static_cast<const IT*>(a.col) + base + lane * CHUNK;
    double acc = 0.0;
    for (int c = 0; c < w; c += CHUNK) {
        double v[CHUNK];
        int cc[CHUNK];
        dev::ChunkLoad<double, CHUNK, dev::kLdNoAlloc>::run(vp, v);
        dev::ColLoad<CHUNK, IT, dev::kLdNoAlloc>::run(cp, row, cc);
#pragma unroll
        for (int q = 0; q < CHUNK; ++q) acc += v[q] * __ldcg(a.x64 + cc[q]);
        vp += 32 * CHUNK;
        cp += 32 * CHUNK;
    }
    return acc + a.diag64[row] * __ldcg(a.x64 + row);
}

// The cluster-resident kernel for (value type, chunk, int16 columns); nullptr when none.
BatchKernel batch_resident_kernel(int vt, int chunk, bool idx16);
// Static shared memory of that kernel (bytes): the launch's dynamic part is what is left.
int batch_resident_static_smem(BatchKernel k);

}  // namespace xplus
