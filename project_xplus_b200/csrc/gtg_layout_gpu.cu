// gtg_layout_gpu.cu -- the SELL images of G and G^T for the factorized preconditioner
// M^-1 = G^T G, built on the GPU, bit-identical to the host construction in solver.cu
// (gtg_layout_host).
//
// G lives on A's lower pattern (entries j <= i of every CSR row, the g_low order: row by row,
// CSR order within a row).  Both images are in the matrix's SELL row order (perm[new] = old),
// chunk 2, int32 columns, with `map` taking every slot to its g_low entry (-1: padding, whose
// column is the row itself).  G row perm^-1(i) lists row i's lower entries in CSR order; G^T
// row perm^-1(j) lists the entries (i, j) in increasing g_low index, which a stable radix sort
// of the g_low entries by their G^T row gives.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "common.hpp"
#include "gtg_layout_gpu.hpp"

namespace xplus {
namespace {

constexpr int kCh = 2;  // slots per lane per step (chunk)

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

struct Tmp {
    std::vector<void*> p;
    template <typename T>
    T* get(size_t count) {
        void* q = nullptr;
        const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 256));
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error(XPLUS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        p.push_back(q);
        return static_cast<T*>(q);
    }
    ~Tmp() {
        for (void* q : p) cudaFree(q);
    }
};

__global__ void k_iperm(const int* __restrict__ perm, int n, int* __restrict__ iperm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) iperm[perm[i]] = i;
}

// lower entries of original row i, and each one's contribution to the G^T row lengths
// (a row range or column outside [0, n) sets *bad and is skipped: checked before any fill)
__global__ void k_low_count(const int* __restrict__ rp, const int* __restrict__ ci, const int* __restrict__ iperm,
                            int n, int nnz, int* __restrict__ cnt, int* __restrict__ tlen, int* __restrict__ bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int q0 = rp[i], q1 = rp[i + 1];
    if (q0 < 0 || q1 < q0 || q1 > nnz) {
        atomicOr(bad, 1);
        cnt[i] = 0;
        return;
    }
    int c = 0;
    for (int q = q0; q < q1; ++q) {
        const int j = ci[q];
        if (j < 0 || j >= n) {
            atomicOr(bad, 1);
            continue;
        }
        if (j > i) continue;
        ++c;
        atomicAdd(&tlen[iperm[j]], 1);
    }
    cnt[i] = c;
}

__global__ void k_glen(const int* __restrict__ cnt, const int* __restrict__ perm, int n, int n_pad,
                       int* __restrict__ glen) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n_pad) glen[r] = r < n ? cnt[perm[r]] : 0;
}

// per slice: 32 x (the longest row rounded up to the chunk)
__global__ void k_slice_slots(const int* __restrict__ len, int ns, long long* __restrict__ slots) {
    const int s = static_cast<int>((static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= ns) return;
    int w = len[s * 32 + lane];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w = max(w, __shfl_xor_sync(0xffffffffu, w, o));
    if (lane == 0) slots[s] = 32LL * ((w + kCh - 1) / kCh * kCh);
}

__device__ __forceinline__ long long gslot(const long long* sp, int r, int j) {
    return sp[r >> 5] + static_cast<long long>(j / kCh) * 32 * kCh + (r & 31) * kCh + (j % kCh);
}

__global__ void k_g_fill(const int* __restrict__ rp, const int* __restrict__ ci, const int* __restrict__ perm,
                         const int* __restrict__ iperm, const int* __restrict__ gptr, const long long* __restrict__ sp,
                         int n, int n_pad, int* __restrict__ col, int* __restrict__ map, int* __restrict__ gl_row,
                         int* __restrict__ gl_key) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_pad) return;
    const int w = static_cast<int>((sp[(r >> 5) + 1] - sp[r >> 5]) / 32);
    int jj = 0;
    if (r < n) {
        const int i = perm[r];
        const int g0 = gptr[i];
        for (int q = rp[i]; q < rp[i + 1]; ++q) {
            const int j = ci[q];
            if (j > i) continue;
            const long long pos = gslot(sp, r, jj);
            const int rj = iperm[j];
            col[pos] = rj;
            map[pos] = g0 + jj;
            gl_row[g0 + jj] = r;
            gl_key[g0 + jj] = rj;
            ++jj;
        }
    }
    for (; jj < w; ++jj) {
        const long long pos = gslot(sp, r, jj);
        col[pos] = r;
        map[pos] = -1;
    }
}

__global__ void k_gt_fill(const int* __restrict__ tptr, const int* __restrict__ sorted_gl, const int* __restrict__ gl_row,
                          const long long* __restrict__ sp, int n_pad, int* __restrict__ col, int* __restrict__ map) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_pad) return;
    const int w = static_cast<int>((sp[(r >> 5) + 1] - sp[r >> 5]) / 32);
    const int e0 = tptr[r], e1 = tptr[r + 1];
    int jj = 0;
    for (int e = e0; e < e1; ++e, ++jj) {
        const int gl = sorted_gl[e];
        const long long pos = gslot(sp, r, jj);
        col[pos] = gl_row[gl];
        map[pos] = gl;
    }
    for (; jj < w; ++jj) {
        const long long pos = gslot(sp, r, jj);
        col[pos] = r;
        map[pos] = -1;
    }
}

__global__ void k_iota(int* __restrict__ v, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

template <typename T, typename O>
void exclusive_sum(const T* in, O* out, int count, Tmp& tmp, cudaStream_t st) {
    size_t bytes = 0;
    ck(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, count, st), "scan size");
    void* ws = tmp.get<unsigned char>(bytes);
    ck(cub::DeviceScan::ExclusiveSum(ws, bytes, in, out, count, st), "scan");
}

}  // namespace

GtgImages gtg_layout_device(int n, int n_pad, const int* row_ptr, const int* col_idx, const int* d_perm,
                            const std::function<void*(size_t)>& alloc, cudaStream_t st) {
    Tmp tmp;
    const int nnz = row_ptr[n];
    const int tb = 256;
    const int ns = n_pad / 32;
    int* rp = tmp.get<int>(static_cast<size_t>(n) + 1);
    int* ci = tmp.get<int>(static_cast<size_t>(nnz));
    ck(cudaMemcpyAsync(rp, row_ptr, (static_cast<size_t>(n) + 1) * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    ck(cudaMemcpyAsync(ci, col_idx, static_cast<size_t>(nnz) * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    int* iperm = tmp.get<int>(static_cast<size_t>(n));
    k_iperm<<<(n + tb - 1) / tb, tb, 0, st>>>(d_perm, n, iperm);
    int* cnt = tmp.get<int>(static_cast<size_t>(n) + 1);
    int* tlen = tmp.get<int>(static_cast<size_t>(n_pad) + 1);
    ck(cudaMemsetAsync(cnt, 0, (static_cast<size_t>(n) + 1) * sizeof(int), st), "memset");
    ck(cudaMemsetAsync(tlen, 0, (static_cast<size_t>(n_pad) + 1) * sizeof(int), st), "memset");
    int* bad = tmp.get<int>(1);
    ck(cudaMemsetAsync(bad, 0, sizeof(int), st), "memset");
    k_low_count<<<(n + tb - 1) / tb, tb, 0, st>>>(rp, ci, iperm, n, nnz, cnt, tlen, bad);
    ck(cudaGetLastError(), "gtg counts");
    int h_bad = 0;
    ck(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    require(h_bad == 0, XPLUS_ERR_DATA, "column index out of range");
    int* gptr = tmp.get<int>(static_cast<size_t>(n) + 1);
    exclusive_sum(cnt, gptr, n + 1, tmp, st);  // gptr[n] = n_glow (cnt[n] = 0)
    int* tptr = tmp.get<int>(static_cast<size_t>(n_pad) + 1);
    exclusive_sum(tlen, tptr, n_pad + 1, tmp, st);
    int* glen = tmp.get<int>(static_cast<size_t>(n_pad));
    k_glen<<<(n_pad + tb - 1) / tb, tb, 0, st>>>(cnt, d_perm, n, n_pad, glen);
    long long* gss = tmp.get<long long>(static_cast<size_t>(ns) + 1);
    long long* tss = tmp.get<long long>(static_cast<size_t>(ns) + 1);
    ck(cudaMemsetAsync(gss + ns, 0, sizeof(long long), st), "memset");
    ck(cudaMemsetAsync(tss + ns, 0, sizeof(long long), st), "memset");
    k_slice_slots<<<(ns * 32 + tb - 1) / tb, tb, 0, st>>>(glen, ns, gss);
    k_slice_slots<<<(ns * 32 + tb - 1) / tb, tb, 0, st>>>(tlen, ns, tss);
    ck(cudaGetLastError(), "gtg widths");
    GtgImages out;
    out.g_slice_ptr = static_cast<long long*>(alloc((static_cast<size_t>(ns) + 1) * sizeof(long long)));
    out.gt_slice_ptr = static_cast<long long*>(alloc((static_cast<size_t>(ns) + 1) * sizeof(long long)));
    exclusive_sum(gss, out.g_slice_ptr, ns + 1, tmp, st);
    exclusive_sum(tss, out.gt_slice_ptr, ns + 1, tmp, st);
    int n_glow = 0;
    long long g_slots = 0, gt_slots = 0;
    ck(cudaMemcpyAsync(&n_glow, gptr + n, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaMemcpyAsync(&g_slots, out.g_slice_ptr + ns, sizeof(long long), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaMemcpyAsync(&gt_slots, out.gt_slice_ptr + ns, sizeof(long long), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    require(g_slots < (1LL << 31) && gt_slots < (1LL << 31), XPLUS_ERR_ARG, "G too large (2^31 slots)");
    out.n_glow = n_glow;
    out.g_slots = g_slots;
    out.gt_slots = gt_slots;
    out.g_col = static_cast<int*>(alloc(static_cast<size_t>(g_slots) * sizeof(int)));
    out.g_map = static_cast<int*>(alloc(static_cast<size_t>(g_slots) * sizeof(int)));
    out.gt_col = static_cast<int*>(alloc(static_cast<size_t>(gt_slots) * sizeof(int)));
    out.gt_map = static_cast<int*>(alloc(static_cast<size_t>(gt_slots) * sizeof(int)));
    int* gl_row = tmp.get<int>(static_cast<size_t>(n_glow));
    int* gl_key = tmp.get<int>(static_cast<size_t>(n_glow));
    k_g_fill<<<(n_pad + tb - 1) / tb, tb, 0, st>>>(rp, ci, d_perm, iperm, gptr, out.g_slice_ptr, n, n_pad, out.g_col,
                                                   out.g_map, gl_row, gl_key);
    ck(cudaGetLastError(), "gtg G fill");
    // the g_low entries by G^T row, stably (each G^T row in increasing g_low index)
    int* vals_in = tmp.get<int>(static_cast<size_t>(n_glow));
    int* keys_out = tmp.get<int>(static_cast<size_t>(n_glow));
    int* vals_out = tmp.get<int>(static_cast<size_t>(n_glow));
    k_iota<<<(n_glow + tb - 1) / tb, tb, 0, st>>>(vals_in, n_glow);
    int bits = 1;
    while ((1LL << bits) < n_pad) ++bits;
    size_t bytes = 0;
    ck(cub::DeviceRadixSort::SortPairs(nullptr, bytes, gl_key, keys_out, vals_in, vals_out, n_glow, 0, bits, st), "sort size");
    void* ws = tmp.get<unsigned char>(bytes);
    ck(cub::DeviceRadixSort::SortPairs(ws, bytes, gl_key, keys_out, vals_in, vals_out, n_glow, 0, bits, st), "sort");
    k_gt_fill<<<(n_pad + tb - 1) / tb, tb, 0, st>>>(tptr, vals_out, gl_row, out.gt_slice_ptr, n_pad, out.gt_col,
                                                    out.gt_map);
    ck(cudaGetLastError(), "gtg G^T fill");
    ck(cudaStreamSynchronize(st), "sync");  // the temporaries go next
    return out;
}

}  // namespace xplus
