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

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cfloat>

#include "common.hpp"
#include "layout_gpu.hpp"

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

// ---------------------------------------------------------------------------------------
// The rest of the device-side create (layout_gpu.hpp)
// ---------------------------------------------------------------------------------------
namespace {

// first diagonal entry of each row; bad[0] = rows without one, bad[1] = rows whose entry is
// zero (|a_ii| <= DBL_MIN, the host test)
__global__ void k_diag_first(const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                             int n, double* __restrict__ diag, int* __restrict__ bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 0.0;
    bool found = false;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
        if (ci[k] == i) {
            d = v[k];
            found = true;
            break;
        }
    diag[i] = d;
    if (!found) atomicAdd(bad, 1);
    else if (fabs(d) <= DBL_MIN) atomicAdd(bad + 1, 1);
}

// slot positions of SELL row r: pos(j) = ptr[s] + (j / chunk) 32 chunk + l chunk + j % chunk
__device__ __forceinline__ long long slot_of(const long long* ptr, int r, int j, int chunk) {
    return ptr[r >> 5] + static_cast<long long>(j / chunk) * 32 * chunk + (r & 31) * chunk + (j % chunk);
}

__global__ void k_pack16(const long long* __restrict__ ptr, const int* __restrict__ width, int n_pad, int chunk,
                         const int* __restrict__ col, short* __restrict__ col16, int* __restrict__ far) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_pad) return;
    const int w = width[r >> 5];
    for (int j = 0; j < w; ++j) {
        const long long pos = slot_of(ptr, r, j, chunk);
        const int d = col[pos] - r;
        if (d < -32768 || d > 32767) atomicOr(far, 1);
        col16[pos] = static_cast<short>(d);
    }
}

__global__ void k_convert(const double* __restrict__ in, long long count, int type, double scale, void* __restrict__ out) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const double x = in[q];
    if (type == XPLUS_F32) static_cast<float*>(out)[q] = __double2float_rn(x);
    else if (type == XPLUS_F16) static_cast<__half*>(out)[q] = __double2half(x / scale);
    else if (type == XPLUS_BF16) static_cast<__nv_bfloat16*>(out)[q] = __double2bfloat16(x);
    else static_cast<double*>(out)[q] = x;
}

__device__ __forceinline__ void store_vec(void* out, int i, int type, double x) {
    if (type == XPLUS_F64) static_cast<double*>(out)[i] = x;
    else static_cast<float*>(out)[i] = __double2float_rn(x);
}

__global__ void k_row_vectors(const int* __restrict__ rp, const double* __restrict__ v, const int* __restrict__ perm,
                              const double* __restrict__ diag_csr, int n, int n_pad, int vtype,
                              double* __restrict__ diag64, void* __restrict__ minv, void* __restrict__ rowsum) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pad) return;
    double d = 0.0, m = 0.0, rs = 0.0;
    if (i < n) {
        const int old = perm[i];
        d = diag_csr[old];
        m = 1.0 / d;
        if (rowsum)
            for (int k = rp[old]; k < rp[old + 1]; ++k) rs += v[k];
    }
    if (diag64) diag64[i] = d;
    store_vec(minv, i, vtype, m);
    if (rowsum) store_vec(rowsum, i, vtype, rs);
}

__global__ void k_count_below(const double* __restrict__ v, int n, double eps, int* __restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && fabs(v[i]) <= eps) atomicAdd(count, 1);
}

// one CTA per resident block: min / max column of its slots
__global__ void k_windows(const long long* __restrict__ ptr, const int* __restrict__ col, int n_slices, int n_pad,
                          int per, int2* __restrict__ win) {
    __shared__ int s_lo[32], s_hi[32];
    const int b = blockIdx.x;
    const int sb = b * per, se = min(n_slices, sb + per);
    if (se <= sb) {
        if (threadIdx.x == 0) win[b] = make_int2(0, 0);
        return;
    }
    int lo = sb * 32, hi = se * 32;
    for (long long pos = ptr[sb] + threadIdx.x; pos < ptr[se]; pos += blockDim.x) {
        const int c = col[pos];
        lo = min(lo, c);
        hi = max(hi, c + 1);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        s_lo[threadIdx.x >> 5] = lo;
        s_hi[threadIdx.x >> 5] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) {
            lo = min(lo, s_lo[w]);
            hi = max(hi, s_hi[w]);
        }
        lo &= ~3;  // 16-byte aligned window
        hi = min(n_pad, (hi + 3) & ~3);
        win[b] = make_int2(lo, hi - lo);
    }
}

}  // namespace

DeviceCsr::~DeviceCsr() {
    for (void* p : owned) cudaFree(p);
}

void upload_csr(int n, const int* row_ptr, const int* col_idx, const double* values, DeviceCsr& csr, cudaStream_t st) {
    csr.n = n;
    csr.nnz = row_ptr[n];
    require(csr.nnz >= 0, XPLUS_ERR_DATA, "row_ptr[n] must equal nnz");
    auto get = [&](size_t bytes) {
        void* p = nullptr;
        const cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 256));
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error(XPLUS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        csr.owned.push_back(p);
        return p;
    };
    csr.rp = static_cast<int*>(get((static_cast<size_t>(n) + 1) * sizeof(int)));
    csr.ci = static_cast<int*>(get(static_cast<size_t>(csr.nnz) * sizeof(int)));
    csr.v = static_cast<double*>(get(static_cast<size_t>(csr.nnz) * sizeof(double)));
    ck(cudaMemcpyAsync(csr.rp, row_ptr, (static_cast<size_t>(n) + 1) * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    ck(cudaMemcpyAsync(csr.ci, col_idx, static_cast<size_t>(csr.nnz) * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    ck(cudaMemcpyAsync(csr.v, values, static_cast<size_t>(csr.nnz) * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
    // structure checks on the device; the host validator supplies the message of a failure
    DevTmp tmp;
    int* bad = tmp.get<int>(1);
    int h_bad = 0;
    const int tb = 256;
    ck(cudaMemsetAsync(bad, 0, sizeof(int), st), "memset");
    k_check_rows<<<(n + tb - 1) / tb, tb, 0, st>>>(csr.rp, n, bad);
    ck(cudaGetLastError(), "csr check");
    ck(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    if (h_bad == 0 && csr.nnz > 0) {
        k_check_cols<<<static_cast<unsigned>((csr.nnz + tb - 1) / tb), tb, 0, st>>>(csr.ci, csr.nnz, n, bad);
        ck(cudaGetLastError(), "csr check");
        ck(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaStreamSynchronize(st), "sync");
    }
    if (h_bad != 0) {
        validate_csr(n, row_ptr, col_idx, csr.nnz);
        throw Error(XPLUS_ERR_DATA, "invalid CSR structure");
    }
}

void jacobi_diag_device(const DeviceCsr& csr, const int* row_ptr, const int* col_idx, const double* values,
                        double* d_diag, cudaStream_t st) {
    DevTmp tmp;
    int* bad = tmp.get<int>(2);
    int h_bad[2] = {0, 0};
    ck(cudaMemsetAsync(bad, 0, 2 * sizeof(int), st), "memset");
    k_diag_first<<<(csr.n + 255) / 256, 256, 0, st>>>(csr.rp, csr.ci, csr.v, csr.n, d_diag, bad);
    ck(cudaGetLastError(), "jacobi diag");
    ck(cudaMemcpyAsync(h_bad, bad, sizeof(h_bad), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    if (h_bad[0] || h_bad[1]) {
        std::vector<double> d(static_cast<size_t>(csr.n));
        jacobi_diag(csr.n, row_ptr, col_idx, values, d.data());  // throws the reference's message
        throw Error(XPLUS_ERR_DATA, "missing or zero diagonal entry");
    }
}

void sell_layout_device(const DeviceCsr& csr, int sigma, int chunk, int diag_split, int* n_slices, int64_t* slots,
                        int* d_perm, long long* d_slice_ptr, int* d_width, int* d_col32, double* d_val64,
                        double* d_diag_sell, cudaStream_t st) {
    sell_build_device(csr.n, csr.rp, csr.ci, csr.v, 32, sigma, chunk, diag_split, n_slices, slots, d_perm,
                      reinterpret_cast<int64_t*>(d_slice_ptr), d_width, d_col32, d_val64, d_diag_sell, st);
}

bool pack_index16_device(const long long* d_slice_ptr, const int* d_width, int n_slices, int chunk,
                         const int* d_col32, short* d_col16, cudaStream_t st) {
    DevTmp tmp;
    int* far = tmp.get<int>(1);
    int h_far = 0;
    const int n_pad = n_slices * 32;
    ck(cudaMemsetAsync(far, 0, sizeof(int), st), "memset");
    k_pack16<<<(n_pad + 255) / 256, 256, 0, st>>>(d_slice_ptr, d_width, n_pad, chunk, d_col32, d_col16, far);
    ck(cudaGetLastError(), "pack int16");
    ck(cudaMemcpyAsync(&h_far, far, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    return h_far == 0;
}

void count_below(const double* d_v, int n, double eps, int* d_count, cudaStream_t st) {
    k_count_below<<<(n + 255) / 256, 256, 0, st>>>(d_v, n, eps, d_count);
    ck(cudaGetLastError(), "count below");
}

void convert_device(const double* d_in, int64_t count, int type, double scale, void* d_out, cudaStream_t st) {
    if (count <= 0) return;
    k_convert<<<static_cast<unsigned>((count + 255) / 256), 256, 0, st>>>(d_in, count, type, scale, d_out);
    ck(cudaGetLastError(), "convert values");
}

void row_vectors_device(const DeviceCsr& csr, const int* d_perm, const double* d_diag_csr, int n_pad, int vtype,
                        double* d_diag64, void* d_minv, void* d_rowsum, cudaStream_t st) {
    k_row_vectors<<<(n_pad + 255) / 256, 256, 0, st>>>(csr.rp, csr.v, d_perm, d_diag_csr, csr.n, n_pad, vtype, d_diag64,
                                                        d_minv, d_rowsum);
    ck(cudaGetLastError(), "row vectors");
}

std::vector<int2> resident_windows_device(const long long* d_slice_ptr, const int* d_col32, int n_slices, int n_pad,
                                          int grid, cudaStream_t st) {
    DevTmp tmp;
    int2* win = tmp.get<int2>(static_cast<size_t>(grid));
    const int per = (n_slices + grid - 1) / grid;
    k_windows<<<grid, 256, 0, st>>>(d_slice_ptr, d_col32, n_slices, n_pad, per, win);
    ck(cudaGetLastError(), "resident windows");
    std::vector<int2> out(static_cast<size_t>(grid));
    ck(cudaMemcpyAsync(out.data(), win, out.size() * sizeof(int2), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    return out;
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
