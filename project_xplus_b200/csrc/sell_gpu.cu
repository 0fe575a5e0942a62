// sell_gpu.cu -- the SELL-C-sigma builder on the GPU, bit-exact with the host builder (sell.cpp).
//
// Same layout rules, as integer work on device arrays:
//   len     row lengths (minus the first diagonal entry when diag_split)       thread per row
//   perm    stable sort of every window of sigma rows by decreasing length,     one CTA per window:
//           ties by increasing row index: row i goes to rank #{j in window :    rank by counting in
//           len_j > len_i or (len_j == len_i and j < i)}                        shared memory
//   width   per slice of C = 32 rows, the longest row rounded up to chunk      warp per slice
//   ptr     exclusive scan of width x 32                                        one-CTA scan
//   fill    entry j of new row r = 32 s + l at ptr[s] + (j/chunk) 32 chunk +    thread per row
//           l chunk + j%chunk, columns renumbered by iperm; padding: own row, 0
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.hpp"

namespace xplus {
namespace {

constexpr int kMaxSigmaGpu = 4096;

__global__ void k_lengths(const int* __restrict__ rp, const int* __restrict__ ci, int n, int split,
                          int* __restrict__ len) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int l = rp[i + 1] - rp[i];
    if (split)
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) {
                --l;
                break;
            }
    len[i] = l;
}

// CSR structure checks before anything is indexed: row_ptr[0] == 0, non-decreasing, and every
// column in [0, n).  Sets *bad (the caller zeroes it) instead of reading out of bounds.
__global__ void k_check_rows(const int* __restrict__ rp, int n, int* __restrict__ bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && rp[0] != 0) atomicOr(bad, 1);
    if (i < n && rp[i + 1] < rp[i]) atomicOr(bad, 1);
}

__global__ void k_check_cols(const int* __restrict__ ci, long long nnz, int n, int* __restrict__ bad) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < nnz) {
        const int c = ci[k];
        if (c < 0 || c >= n) atomicOr(bad, 2);
    }
}

// one CTA per window of sigma rows
__global__ void k_sigma_rank(const int* __restrict__ len, int n, int sigma, int* __restrict__ perm) {
    __shared__ int s_len[kMaxSigmaGpu];
    const int w0 = blockIdx.x * sigma;
    const int w1 = min(n, w0 + sigma);
    const int m = w1 - w0;
    for (int t = threadIdx.x; t < m; t += blockDim.x) s_len[t] = len[w0 + t];
    __syncthreads();
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
        const int li = s_len[t];
        int rank = 0;
        for (int j = 0; j < m; ++j) {
            const int lj = s_len[j];
            rank += (lj > li) || (lj == li && j < t);
        }
        perm[w0 + rank] = w0 + t;
    }
}

__global__ void k_iota(int* __restrict__ perm, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) perm[i] = i;
}

__global__ void k_inverse(const int* __restrict__ perm, int* __restrict__ iperm, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) iperm[perm[i]] = i;
}

// warp per slice: width = max length of its (existing) rows, rounded up to chunk
__global__ void k_widths(const int* __restrict__ perm, const int* __restrict__ len, int n, int n_slices, int chunk,
                         int* __restrict__ width) {
    const int s = static_cast<int>((static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= n_slices) return;
    const int i = s * 32 + lane;
    int w = i < n ? len[perm[i]] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w = max(w, __shfl_xor_sync(0xffffffffu, w, o));
    if (lane == 0) width[s] = (w + chunk - 1) / chunk * chunk;
}

// ptr[0] = 0, ptr[s + 1] = ptr[s] + 32 width[s]: one CTA, each thread a contiguous chunk
__global__ void __launch_bounds__(1024) k_scan_ptr(const int* __restrict__ width, int n_slices,
                                                   long long* __restrict__ ptr) {
    __shared__ long long s_sum[1024];
    const int t = threadIdx.x;
    const int per = (n_slices + blockDim.x - 1) / blockDim.x;
    const int b = min(n_slices, t * per), e = min(n_slices, b + per);
    long long acc = 0;
    for (int s = b; s < e; ++s) acc += 32LL * width[s];
    s_sum[t] = acc;
    __syncthreads();
    // inclusive Hillis-Steele scan of the per-thread sums
    for (int o = 1; o < static_cast<int>(blockDim.x); o <<= 1) {
        const long long v = t >= o ? s_sum[t - o] : 0;
        __syncthreads();
        s_sum[t] += v;
        __syncthreads();
    }
    long long run = t > 0 ? s_sum[t - 1] : 0;
    if (t == 0) ptr[0] = 0;
    for (int s = b; s < e; ++s) {
        run += 32LL * width[s];
        ptr[s + 1] = run;
    }
}

__global__ void k_fill(const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ vals,
                       const int* __restrict__ perm, const int* __restrict__ iperm, const long long* __restrict__ ptr,
                       const int* __restrict__ width, int n, int n_pad, int chunk, int split, int* __restrict__ col,
                       double* __restrict__ val, double* __restrict__ diag) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_pad) return;
    const int s = r >> 5, l = r & 31;
    const long long base = ptr[s];
    const int w = width[s];
    int j = 0;
    if (r < n) {
        const int old = perm[r];
        bool diag_taken = false;
        for (int k = rp[old]; k < rp[old + 1]; ++k) {
            if (split && !diag_taken && ci[k] == old) {
                if (diag) diag[r] = vals[k];
                diag_taken = true;
                continue;
            }
            const long long pos = base + static_cast<long long>(j / chunk) * 32 * chunk + l * chunk + (j % chunk);
            if (col) col[pos] = iperm[ci[k]];
            if (val) val[pos] = vals[k];
            ++j;
        }
    }
    for (; j < w; ++j) {
        const long long pos = base + static_cast<long long>(j / chunk) * 32 * chunk + l * chunk + (j % chunk);
        if (col) col[pos] = r;
        if (val) val[pos] = 0.0;
    }
}

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

struct DevTmp {
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
    ~DevTmp() {
        for (void* q : p) cudaFree(q);
    }
};

void sell_build_device(int n, const int* d_rp, const int* d_ci, const double* d_vals, int C, int sigma, int chunk,
                       int diag_split, int* n_slices, int64_t* slots, int* d_perm, int64_t* d_slice_ptr,
                       int* d_slice_width, int* d_col, double* d_val, double* d_diag, cudaStream_t st) {
    require(n > 0 && d_rp && d_ci && d_vals && n_slices && slots, XPLUS_ERR_ARG, "invalid argument");
    require(C == 32, XPLUS_ERR_ARG, "sell (gpu): slice height must be 32");
    require(chunk == 1 || chunk == 2 || chunk == 4 || chunk == 8, XPLUS_ERR_ARG, "sell: chunk must be 1, 2, 4 or 8");
    require(sigma >= 1 && sigma <= kMaxSigmaGpu, XPLUS_ERR_ARG, "sell (gpu): sigma must be in [1, 4096]");
    const int ns = (n + 31) / 32, n_pad = ns * 32;
    DevTmp tmp;
    int* len = tmp.get<int>(static_cast<size_t>(n));
    int* perm = d_perm ? d_perm : tmp.get<int>(static_cast<size_t>(n));
    int* width = d_slice_width ? d_slice_width : tmp.get<int>(static_cast<size_t>(ns));
    long long* ptr = d_slice_ptr ? reinterpret_cast<long long*>(d_slice_ptr) : tmp.get<long long>(static_cast<size_t>(ns) + 1);
    const int tb = 256;
    {
        int* bad = tmp.get<int>(1);
        int h_bad = 0, h_nnz = 0;
        ck(cudaMemsetAsync(bad, 0, sizeof(int), st), "memset");
        k_check_rows<<<(n + tb - 1) / tb, tb, 0, st>>>(d_rp, n, bad);
        ck(cudaGetLastError(), "sell check");
        ck(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaMemcpyAsync(&h_nnz, d_rp + n, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaStreamSynchronize(st), "sync");
        require(h_bad == 0, XPLUS_ERR_DATA, "row_ptr must start at 0 and be non-decreasing");
        if (h_nnz > 0) {
            k_check_cols<<<static_cast<unsigned>((static_cast<long long>(h_nnz) + tb - 1) / tb), tb, 0, st>>>(d_ci, h_nnz, n, bad);
            ck(cudaGetLastError(), "sell check");
            ck(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
            ck(cudaStreamSynchronize(st), "sync");
            require(h_bad == 0, XPLUS_ERR_DATA, "column index out of range");
        }
    }
    k_lengths<<<(n + tb - 1) / tb, tb, 0, st>>>(d_rp, d_ci, n, diag_split ? 1 : 0, len);
    ck(cudaGetLastError(), "sell lengths");
    if (sigma > 1)
        k_sigma_rank<<<(n + sigma - 1) / sigma, 256, 0, st>>>(len, n, sigma, perm);
    else
        k_iota<<<(n + tb - 1) / tb, tb, 0, st>>>(perm, n);
    ck(cudaGetLastError(), "sell sort");
    k_widths<<<static_cast<unsigned>((static_cast<long long>(ns) * 32 + tb - 1) / tb), tb, 0, st>>>(perm, len, n, ns, chunk, width);
    ck(cudaGetLastError(), "sell widths");
    k_scan_ptr<<<1, 1024, 0, st>>>(width, ns, ptr);
    ck(cudaGetLastError(), "sell scan");
    long long total = 0;
    ck(cudaMemcpyAsync(&total, ptr + ns, sizeof(long long), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    *n_slices = ns;
    *slots = total;
    if (!d_col && !d_val && !d_diag) return;
    int* iperm = tmp.get<int>(static_cast<size_t>(n));
    k_inverse<<<(n + tb - 1) / tb, tb, 0, st>>>(perm, iperm, n);
    ck(cudaGetLastError(), "sell inverse");
    if (d_diag && diag_split) ck(cudaMemsetAsync(d_diag, 0, static_cast<size_t>(n) * sizeof(double), st), "memset");
    // the diagonal output holds n values (rows beyond n are padding)
    double* diag_full = nullptr;
    if (d_diag && diag_split) diag_full = tmp.get<double>(static_cast<size_t>(n_pad));
    if (diag_full) ck(cudaMemsetAsync(diag_full, 0, static_cast<size_t>(n_pad) * sizeof(double), st), "memset");
    k_fill<<<(n_pad + tb - 1) / tb, tb, 0, st>>>(d_rp, d_ci, d_vals, perm, iperm, ptr, width, n, n_pad, chunk,
                                                 diag_split ? 1 : 0, d_col, d_val, diag_full);
    ck(cudaGetLastError(), "sell fill");
    if (diag_full) ck(cudaMemcpyAsync(d_diag, diag_full, static_cast<size_t>(n) * sizeof(double), cudaMemcpyDeviceToDevice, st), "D2D");
    ck(cudaStreamSynchronize(st), "sync");
}

}  // namespace

void sell_build_via_gpu(int n, const int* row_ptr, const int* col_idx, const double* values, int C, int sigma,
                        int chunk, int diag_split, SellHost& S) {
    const int64_t nnz = row_ptr[n];
    cudaStream_t st = nullptr;
    ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
    try {
        DevTmp tmp;
        int* rp = tmp.get<int>(static_cast<size_t>(n) + 1);
        int* ci = tmp.get<int>(static_cast<size_t>(nnz));
        double* v = tmp.get<double>(static_cast<size_t>(nnz));
        ck(cudaMemcpyAsync(rp, row_ptr, (static_cast<size_t>(n) + 1) * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
        ck(cudaMemcpyAsync(ci, col_idx, static_cast<size_t>(nnz) * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
        ck(cudaMemcpyAsync(v, values, static_cast<size_t>(nnz) * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
        int ns = 0;
        int64_t slots = 0;
        sell_build_device(n, rp, ci, v, C, sigma, chunk, diag_split, &ns, &slots, nullptr, nullptr, nullptr, nullptr,
                          nullptr, nullptr, st);
        int* perm = tmp.get<int>(static_cast<size_t>(n));
        int64_t* sp = tmp.get<int64_t>(static_cast<size_t>(ns) + 1);
        int* sw = tmp.get<int>(static_cast<size_t>(ns));
        int* col = tmp.get<int>(static_cast<size_t>(slots));
        double* val = tmp.get<double>(static_cast<size_t>(slots));
        double* dg = diag_split ? tmp.get<double>(static_cast<size_t>(n)) : nullptr;
        sell_build_device(n, rp, ci, v, C, sigma, chunk, diag_split, &ns, &slots, perm, sp, sw, col, val, dg, st);
        S.n = n;
        S.C = C;
        S.sigma = sigma;
        S.chunk = chunk;
        S.diag_split = diag_split;
        S.n_slices = ns;
        S.n_pad = ns * C;
        S.slots = slots;
        S.perm.resize(static_cast<size_t>(n));
        S.slice_ptr.resize(static_cast<size_t>(ns) + 1);
        S.slice_width.resize(static_cast<size_t>(ns));
        S.col.resize(static_cast<size_t>(slots));
        S.val.resize(static_cast<size_t>(slots));
        ck(cudaMemcpyAsync(S.perm.data(), perm, S.perm.size() * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaMemcpyAsync(S.slice_ptr.data(), sp, S.slice_ptr.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaMemcpyAsync(S.slice_width.data(), sw, S.slice_width.size() * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaMemcpyAsync(S.col.data(), col, S.col.size() * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaMemcpyAsync(S.val.data(), val, S.val.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        if (diag_split) {
            S.diag.assign(static_cast<size_t>(S.n_pad), 0.0);
            ck(cudaMemcpyAsync(S.diag.data(), dg, static_cast<size_t>(n) * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        }
        ck(cudaStreamSynchronize(st), "sync");
        S.iperm.resize(static_cast<size_t>(n));
        for (int i = 0; i < n; ++i) S.iperm[static_cast<size_t>(S.perm[static_cast<size_t>(i)])] = i;
    } catch (...) {
        cudaStreamDestroy(st);
        throw;
    }
    cudaStreamDestroy(st);
}

}  // namespace xplus

extern "C" int xplus_sell_build_device(int n, const int* d_row_ptr, const int* d_col_idx, const double* d_values,
                                       int C, int sigma, int chunk, int diag_split, int* n_slices, int64_t* slots,
                                       int* d_perm, int64_t* d_slice_ptr, int* d_slice_width, int* d_col,
                                       double* d_val, double* d_diag, void* stream) {
    return xplus::guarded([&] {
        xplus::sell_build_device(n, d_row_ptr, d_col_idx, d_values, C, sigma, chunk, diag_split, n_slices, slots,
                                 d_perm, d_slice_ptr, d_slice_width, d_col, d_val, d_diag,
                                 static_cast<cudaStream_t>(stream));
    });
}
