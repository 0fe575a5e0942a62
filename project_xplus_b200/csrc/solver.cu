// solver.cu -- the single-system handle behind the C ABI: builds the SELL-C-sigma matrix,
// keeps it and the solve vectors resident on one GPU, launches the persistent PCG kernel.
//
// Replaces the XRT host of the reference's single-launch solver
// (host/cuper_control_xrt_host.cpp:163-337): there the host packs the 16-channel stream,
// allocates 26 buffers and launches cuper_pcg_control_kernel once; here the host builds
// SELL-C-sigma, uploads it once per handle and launches one cooperative kernel per solve.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <set>
#include <vector>

#include "common.hpp"
#include "gnn.hpp"
#include "gtg_layout_gpu.hpp"
#include "layout_gpu.hpp"
#include "pcg_kernels.cuh"

struct xplus_pcg {
    int device = 0;
    cudaStream_t stream = nullptr;
    xplus_opts opts{};
    xplus::KernelKey key{};
    int n = 0, n_pad = 0, n_slices = 0;
    int64_t nnz = 0, slots = 0;
    // device matrix
    long long* d_slice_ptr = nullptr;
    void* d_col = nullptr;     // int32 columns or int16 row offsets, followed by the values
    cudaAccessPolicyWindow window{};
    void* d_val = nullptr;
    double* d_val64 = nullptr;
    void* d_rowsum = nullptr;
    double* d_diag64 = nullptr;
    int* d_perm = nullptr;
    // device vectors (SELL order, n_pad)
    void* d_minv = nullptr;
    double* d_b64 = nullptr;
    double* d_x64 = nullptr;
    void* d_rec = nullptr;  // node records {z, p}
    void* d_r = nullptr;
    void* d_ap = nullptr;
    void* d_sx = nullptr;   // scratch SpMV in/out (vector type)
    void* d_sy = nullptr;
    // original-order FP64 staging
    double* d_bio = nullptr;
    double* d_xio = nullptr;
    // control
    double* d_partial = nullptr;
    unsigned* d_bar = nullptr;
    int* d_err = nullptr;
    xplus::PcgOut* d_out = nullptr;
    double* d_trace = nullptr;
    int trace_cap = 0;
    int grid = 0, tpb = 0;
    bool resident = false;     // SM-resident kernel (pcg_resident.cu)
    bool one_sync = false;     // its one-barrier-per-iteration form
    double val_scale = 1.0;    // stored value = a_ij / val_scale (FP16)
    size_t smem_bytes = 0;
    int2* d_win = nullptr;
    long long* d_block_clk = nullptr;  // per-CTA phase clock [grid][4]
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    xplus_metrics last{};
    bool pending = false;
    int debug_skip_block = -1;
    long long phase_ns[4] = {0, 0, 0, 0};
    std::vector<void*> allocations;
    std::vector<int> perm;     // SELL row -> original row
    bool l2_user = false;      // holds a persisting-L2 request (l2_want bytes) in g_l2_wants
    size_t mat_bytes = 0;      // matrix columns + values (one allocation at d_col)
    size_t l2_want = 0;
    // M^-1 = G^T G: G on A's lower pattern (original order), SELL images of G and G^T in the
    // matrix's SELL order, and the map from each SELL slot to its entry of g_low
    bool gtg = false;
    int gtg_grid = 0;
    int g_fallback_iters = 0;
    int64_t n_glow = 0, g_slots = 0, gt_slots = 0;
    long long *d_g_slice_ptr = nullptr, *d_gt_slice_ptr = nullptr;
    int *d_g_col = nullptr, *d_gt_col = nullptr, *d_g_map = nullptr, *d_gt_map = nullptr;
    float *d_g_val = nullptr, *d_gt_val = nullptr, *d_t = nullptr, *d_r2 = nullptr;
    double* d_glow = nullptr;
};

namespace xplus {

namespace {

double round16(double v, int type, double scale) {
    if (type == XPLUS_F16) return static_cast<double>(__half2float(__double2half(v / scale))) * scale;
    return static_cast<double>(__bfloat162float(__double2bfloat16(v)));
}

}  // namespace

void two_term_entries(int n, const int* row_ptr, const int* col_idx, const double* values, int type,
                      double scale, double ratio, TwoTermCsr& out) {
    std::vector<unsigned char> wide(static_cast<size_t>(n), 0);
    std::vector<double> dabs(static_cast<size_t>(n), 0.0);
    parallel_for(n, [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            double off = 0.0, d = 0.0;
            for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
                if (col_idx[k] == i) d += values[k];
                else off += std::fabs(values[k]);
            }
            dabs[static_cast<size_t>(i)] = std::fabs(d);
            wide[static_cast<size_t>(i)] = off > ratio * std::fabs(d);
        }
    });
    auto selected = [&](int64_t i, int k) {
        const int j = col_idx[k];
        return j != i && (wide[static_cast<size_t>(i)] || wide[static_cast<size_t>(j)]) &&
               std::fabs(values[k]) > 0.5 * std::min(dabs[static_cast<size_t>(i)], dabs[static_cast<size_t>(j)]);
    };
    std::vector<int> extra(static_cast<size_t>(n) + 1, 0);
    parallel_for(n, [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            int c = 0;
            for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
                if (selected(i, k)) ++c;
            extra[static_cast<size_t>(i) + 1] = c;
        }
    });
    for (int i = 0; i < n; ++i) extra[static_cast<size_t>(i) + 1] += extra[static_cast<size_t>(i)];
    if (extra[static_cast<size_t>(n)] == 0) return;
    const int64_t total = static_cast<int64_t>(row_ptr[n]) + extra[static_cast<size_t>(n)];
    require(total <= std::numeric_limits<int>::max(), XPLUS_ERR_ARG, "two-term entries overflow int32 row pointers");
    out.row_ptr.resize(static_cast<size_t>(n) + 1);
    for (int i = 0; i <= n; ++i) out.row_ptr[static_cast<size_t>(i)] = row_ptr[i] + extra[static_cast<size_t>(i)];
    out.col_idx.resize(static_cast<size_t>(total));
    out.values.resize(static_cast<size_t>(total));
    parallel_for(n, [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            int q = out.row_ptr[static_cast<size_t>(i)];
            for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
                const int j = col_idx[k];
                if (selected(i, k)) {
                    const double hi = round16(values[k], type, scale);
                    out.col_idx[static_cast<size_t>(q)] = j;
                    out.values[static_cast<size_t>(q++)] = hi;
                    out.col_idx[static_cast<size_t>(q)] = j;
                    out.values[static_cast<size_t>(q++)] = values[k] - hi;
                } else {
                    out.col_idx[static_cast<size_t>(q)] = j;
                    out.values[static_cast<size_t>(q++)] = values[k];
                }
            }
        }
    });
}


double f16_offdiag_scale(int n, const int* row_ptr, const int* col_idx, const double* values) {
    double m = 0.0;
    for (int i = 0; i < n; ++i)
        for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
            if (col_idx[k] != i) m = std::max(m, std::fabs(values[k]));
    return m > 0.0 ? std::ldexp(1.0, static_cast<int>(std::ceil(std::log2(m))) - 15) : 1.0;
}

double split_ratio_of(const xplus_opts& o) {
    if (o.value_type != XPLUS_BF16 && o.value_type != XPLUS_F16) return 0.0;
    return o.split_ratio >= 0.0 ? o.split_ratio : (o.value_type == XPLUS_BF16 ? 1.5 : 2.0);
}

}  // namespace xplus

namespace xplus {
namespace {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

template <typename T>
T* dalloc(xplus_pcg* h, size_t count) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count * sizeof(T), 256);
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    h->allocations.push_back(p);
    return static_cast<T*>(p);
}

size_t elem_size(int t) { return t == XPLUS_F64 ? 8 : ((t == XPLUS_BF16 || t == XPLUS_F16) ? 2 : 4); }

void require_device(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_CUDA, "no CUDA device available (the solver has no CPU path)");
    }
    require(device >= 0 && device < count, XPLUS_ERR_ARG, "device ordinal out of range");
    cudaDeviceProp prop;
    cuda_check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    require(prop.major == 10, XPLUS_ERR_CUDA, "this build targets sm_100 (B200) devices only");
    int coop = 0;
    cuda_check(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device), "attr");
    require(coop != 0, XPLUS_ERR_CUDA, "device does not support cooperative launch");
}

// Converts FP64 values to the storage type into a host byte buffer (FP16: v / scale).
std::vector<unsigned char> convert(const std::vector<double>& v, int type, double scale = 1.0) {
    std::vector<unsigned char> out(v.size() * elem_size(type));
    if (type == XPLUS_F64) {
        std::memcpy(out.data(), v.data(), out.size());
    } else if (type == XPLUS_F32) {
        float* o = reinterpret_cast<float*>(out.data());
        for (size_t i = 0; i < v.size(); ++i) o[i] = static_cast<float>(v[i]);
    } else if (type == XPLUS_F16) {
        __half* o = reinterpret_cast<__half*>(out.data());
        for (size_t i = 0; i < v.size(); ++i) o[i] = __double2half(v[i] / scale);
    } else {
        __nv_bfloat16* o = reinterpret_cast<__nv_bfloat16*>(out.data());
        for (size_t i = 0; i < v.size(); ++i) o[i] = __double2bfloat16(v[i]);
    }
    return out;
}

// The persisting-L2 requests of the live handles, and the limit before the first: the limit
// is the largest live request (never below the one found), so a handle that goes does not
// leave a larger set-aside behind for the others (measured: a destroyed 200 MB-matrix
// handle's limit left in place slowed the 1108^2 solve from 108 to 119 ms), and the last
// one to go restores the limit it found.
std::mutex g_l2_mutex;
std::multiset<size_t> g_l2_wants;
size_t g_l2_limit_before = 0;

void destroy(xplus_pcg* h) {
    if (!h) return;
    if (h->device >= 0) cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->l2_user) {
        // the matrix's lines stay persisting in L2 until reset: hand the cache back
        cudaCtxResetPersistingL2Cache();
        std::lock_guard<std::mutex> lk(g_l2_mutex);
        const auto it = g_l2_wants.find(h->l2_want);
        if (it != g_l2_wants.end()) g_l2_wants.erase(it);
        const size_t keep = g_l2_wants.empty() ? g_l2_limit_before : std::max(g_l2_limit_before, *g_l2_wants.rbegin());
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, keep);
    }
    for (void* p : h->allocations) cudaFree(p);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    cudaGetLastError();
    delete h;
}

// Columns and values in one allocation, so one L2 access-policy window covers both.
unsigned char* alloc_matrix(xplus_pcg* h, const xplus_opts& o, size_t col_bytes, size_t val_bytes) {
    (void)o;
    unsigned char* mat = dalloc<unsigned char>(h, col_bytes + val_bytes);
    h->d_col = mat;
    h->d_val = mat + col_bytes;
    h->mat_bytes = col_bytes + val_bytes;
    return mat;
}

// The persisting-L2 set-aside and access-policy window over the matrix, for the kernels whose
// working set can exceed L2 (the global-memory and the G^T G kernel); requested once per
// handle when such a kernel is first chosen.  The SM-resident kernel does without: its matrix
// stays in L2 anyway, and changing the device's persisting limit at create and destroy took
// from 30 ms up to 2.7 s per call on a shared B200 (1108^2 system, creates without it: 28-29 ms).
void request_l2(xplus_pcg* h) {
    if (h->l2_user || !h->opts.l2_persist || h->mat_bytes == 0) return;
    int max_window = 0;
    cudaDeviceProp prop;
    cuda_check(cudaGetDeviceProperties(&prop, h->device), "props");
    cuda_check(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, h->device), "attr");
    const size_t bytes = std::min(h->mat_bytes, static_cast<size_t>(max_window));
    size_t limit = 0;
    const size_t want = std::min(bytes, static_cast<size_t>(prop.persistingL2CacheMaxSize));
    {
        std::lock_guard<std::mutex> lk(g_l2_mutex);
        cuda_check(cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize), "limit");
        if (g_l2_wants.empty()) g_l2_limit_before = limit;
        if (limit < want) cuda_check(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want), "set L2 limit");
        g_l2_wants.insert(want);
        h->l2_want = want;
        h->l2_user = true;
    }
    cuda_check(cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize), "limit");
    if (bytes > 0 && limit > 0) {
        h->window.base_ptr = h->d_col;
        h->window.num_bytes = bytes;
        h->window.hitRatio = std::min(1.0f, static_cast<float>(limit) / static_cast<float>(bytes));
        h->window.hitProp = cudaAccessPropertyPersisting;
        h->window.missProp = cudaAccessPropertyStreaming;
    }
}

// Device temporaries of one create call, freed when it returns.
struct CreateTmp {
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
    ~CreateTmp() {
        for (void* q : p) cudaFree(q);
    }
};

// The layout on the GPU from one device copy of the CSR: checks, Jacobi diagonal, SELL image,
// int16 offsets, value conversion, FP64 copy, row vectors and the resident windows, every
// array bit-identical to the host path (create_layout_host).  `grid` > 0: windows for that
// many resident blocks.
void create_layout_device(xplus_pcg* h, const xplus_opts& o, bool split, int n, const int* row_ptr,
                          const int* col_idx, const double* values, int grid, std::vector<int2>& win) {
    cudaStream_t st = h->stream;
    CreateTmp tmp;
    DeviceCsr csr;
    upload_csr(n, row_ptr, col_idx, values, csr, st);
    double* d_diag_csr = tmp.get<double>(static_cast<size_t>(n));
    jacobi_diag_device(csr, row_ptr, col_idx, values, d_diag_csr, st);
    {
        // the host path's second test (kBreakdownEps), with its message
        int tiny = 0;
        const double eps = 1.0e-30;
        int* d_tiny = tmp.get<int>(1);
        cuda_check(cudaMemsetAsync(d_tiny, 0, sizeof(int), st), "memset");
        count_below(d_diag_csr, n, eps, d_tiny, st);
        cuda_check(cudaMemcpyAsync(&tiny, d_tiny, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        cuda_check(cudaStreamSynchronize(st), "sync");
        require(tiny == 0, XPLUS_ERR_DATA, "zero diagonal entry while building Jacobi inverse");
    }
    int ns = 0;
    int64_t slots = 0;
    sell_layout_device(csr, o.sigma, o.chunk, split ? 1 : 0, &ns, &slots, nullptr, nullptr, nullptr, nullptr, nullptr,
                       nullptr, st);
    h->n_slices = ns;
    h->n_pad = ns * 32;
    h->slots = slots;
    const size_t np = static_cast<size_t>(h->n_pad);
    const size_t xs = elem_size(o.vector_type);
    h->d_perm = dalloc<int>(h, static_cast<size_t>(n));
    h->d_slice_ptr = dalloc<long long>(h, static_cast<size_t>(ns) + 1);
    int* width = tmp.get<int>(static_cast<size_t>(ns));
    int* col32 = tmp.get<int>(static_cast<size_t>(slots));
    const bool keep64 = o.keep_fp64 != 0 && o.value_type != XPLUS_F64;
    double* val64 = keep64 ? dalloc<double>(h, static_cast<size_t>(slots)) : tmp.get<double>(static_cast<size_t>(slots));
    sell_layout_device(csr, o.sigma, o.chunk, split ? 1 : 0, &ns, &slots, h->d_perm, h->d_slice_ptr, width, col32,
                       val64, nullptr, st);
    // int16 offsets from the row when the ordered bandwidth allows (lossless)
    bool idx16 = o.index16 != 0;
    short* col16 = nullptr;
    if (idx16) {
        col16 = tmp.get<short>(static_cast<size_t>(slots));
        idx16 = pack_index16_device(h->d_slice_ptr, width, ns, o.chunk, col32, col16, st);
    }
    h->key.idx16 = idx16 ? 1 : 0;
    const size_t col_bytes = (static_cast<size_t>(slots) * (idx16 ? 2 : 4) + 255) / 256 * 256;
    const size_t val_bytes = static_cast<size_t>(slots) * elem_size(o.value_type);
    alloc_matrix(h, o, col_bytes, val_bytes);
    cuda_check(cudaMemcpyAsync(h->d_col, idx16 ? static_cast<const void*>(col16) : static_cast<const void*>(col32),
                               static_cast<size_t>(slots) * (idx16 ? 2 : 4), cudaMemcpyDeviceToDevice, st), "D2D");
    h->val_scale = o.value_type == XPLUS_F16 ? f16_offdiag_scale(n, row_ptr, col_idx, values) : 1.0;
    convert_device(val64, slots, o.value_type, h->val_scale, h->d_val, st);
    if (keep64) h->d_val64 = val64;
    else if (o.value_type == XPLUS_F64) h->d_val64 = static_cast<double*>(h->d_val);
    // Jacobi inverse in SELL order (host/pcg_common.hpp:42-54: m_inv = 1 / diag), from the exact
    // FP64 diagonal; in the row-sum form also the row sums and the FP64 diagonal
    h->d_minv = dalloc<unsigned char>(h, np * xs);
    if (split) {
        h->d_rowsum = dalloc<unsigned char>(h, np * xs);
        h->d_diag64 = dalloc<double>(h, np);
    }
    row_vectors_device(csr, h->d_perm, d_diag_csr, h->n_pad, o.vector_type, split ? h->d_diag64 : nullptr, h->d_minv,
                       split ? h->d_rowsum : nullptr, st);
    h->perm.resize(static_cast<size_t>(n));
    cuda_check(cudaMemcpyAsync(h->perm.data(), h->d_perm, static_cast<size_t>(n) * sizeof(int), cudaMemcpyDeviceToHost, st),
               "D2H");
    if (grid > 0) win = resident_windows_device(h->d_slice_ptr, col32, ns, h->n_pad, grid, st);
    cuda_check(cudaStreamSynchronize(st), "sync");  // the temporaries go next
}

// The layout on the host (the reference for create_layout_device): the 16-bit two-term
// rewrite, sort windows above 4096, or build_on_gpu = 0.  diag: the CSR's Jacobi diagonal.
void create_layout_host(xplus_pcg* h, const xplus_opts& o, bool split, int n, const int* row_ptr,
                        const int* col_idx, const double* values, const std::vector<double>& diag, int grid,
                        std::vector<int2>& win) {
    const double scale16 = o.value_type == XPLUS_F16 ? f16_offdiag_scale(n, row_ptr, col_idx, values) : 1.0;
    const double split_ratio = split_ratio_of(o);
    TwoTermCsr two;
    if (split_ratio > 0.0) two_term_entries(n, row_ptr, col_idx, values, o.value_type, scale16, split_ratio, two);
    const bool use_two = !two.row_ptr.empty();
    const int* rp_s = use_two ? two.row_ptr.data() : row_ptr;
    const int* ci_s = use_two ? two.col_idx.data() : col_idx;
    const double* va_s = use_two ? two.values.data() : values;
    SellHost S;
    if (o.build_on_gpu && o.sigma <= 4096)
        sell_build_via_gpu(n, rp_s, ci_s, va_s, 32, o.sigma, o.chunk, split ? 1 : 0, S);
    else
        sell_build(n, rp_s, ci_s, va_s, 32, o.sigma, o.chunk, split ? 1 : 0, S);
    h->n_pad = S.n_pad;
    h->n_slices = S.n_slices;
    h->slots = S.slots;
    h->perm = S.perm;
    cudaStream_t st = h->stream;
    const size_t np = static_cast<size_t>(S.n_pad);
    const size_t xs = elem_size(o.vector_type);
    h->d_slice_ptr = dalloc<long long>(h, S.slice_ptr.size());
    // int16 offsets from the row when the ordered bandwidth allows (lossless)
    bool idx16 = o.index16 != 0;
    std::vector<short> col16;
    if (idx16) {
        col16.resize(static_cast<size_t>(S.slots));
        // slot (j/chunk) 32 chunk + lane chunk + j%chunk of slice sl belongs to row 32 sl + lane
        std::vector<unsigned char> far(static_cast<size_t>(S.n_slices), 0);
        const int ch = o.chunk;
        parallel_for(S.n_slices, [&](int64_t b, int64_t e) {
            for (int64_t sl = b; sl < e; ++sl) {
                const int64_t base = S.slice_ptr[static_cast<size_t>(sl)];
                const int64_t groups = (S.slice_ptr[static_cast<size_t>(sl) + 1] - base) / (32 * ch);
                for (int64_t jg = 0; jg < groups; ++jg)
                    for (int lane = 0; lane < 32; ++lane) {
                        const int row = static_cast<int>(sl) * 32 + lane;
                        const int64_t p0 = base + jg * 32 * ch + lane * ch;
                        for (int q = 0; q < ch; ++q) {
                            const int d = S.col[static_cast<size_t>(p0 + q)] - row;
                            if (d < -32768 || d > 32767) far[static_cast<size_t>(sl)] = 1;
                            col16[static_cast<size_t>(p0 + q)] = static_cast<short>(d);
                        }
                    }
            }
        });
        for (unsigned char f : far)
            if (f) idx16 = false;
    }
    h->key.idx16 = idx16 ? 1 : 0;
    const size_t col_bytes = (static_cast<size_t>(S.slots) * (idx16 ? 2 : 4) + 255) / 256 * 256;
    const size_t val_bytes = static_cast<size_t>(S.slots) * elem_size(o.value_type);
    alloc_matrix(h, o, col_bytes, val_bytes);
    h->d_perm = dalloc<int>(h, static_cast<size_t>(n));
    h->d_minv = dalloc<unsigned char>(h, np * xs);
    std::vector<long long> sp(S.slice_ptr.begin(), S.slice_ptr.end());
    cuda_check(cudaMemcpyAsync(h->d_slice_ptr, sp.data(), sp.size() * sizeof(long long), cudaMemcpyHostToDevice, st), "H2D");
    if (h->key.idx16)
        cuda_check(cudaMemcpyAsync(h->d_col, col16.data(), col16.size() * sizeof(short), cudaMemcpyHostToDevice, st), "H2D");
    else
        cuda_check(cudaMemcpyAsync(h->d_col, S.col.data(), S.col.size() * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    cuda_check(cudaMemcpyAsync(h->d_perm, S.perm.data(), S.perm.size() * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    h->val_scale = o.value_type == XPLUS_F16 ? scale16 : 1.0;
    std::vector<unsigned char> vbytes = convert(S.val, o.value_type, h->val_scale);
    cuda_check(cudaMemcpyAsync(h->d_val, vbytes.data(), vbytes.size(), cudaMemcpyHostToDevice, st), "H2D");
    const bool keep64 = o.keep_fp64 != 0 && o.value_type != XPLUS_F64;
    if (keep64) {
        h->d_val64 = dalloc<double>(h, static_cast<size_t>(S.slots));
        cuda_check(cudaMemcpyAsync(h->d_val64, S.val.data(), S.val.size() * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
    } else if (o.value_type == XPLUS_F64) {
        h->d_val64 = static_cast<double*>(h->d_val);
    }
    // Jacobi inverse in SELL order (host/pcg_common.hpp:42-54: m_inv = 1 / diag), from
    // the exact FP64 diagonal.
    std::vector<double> dsell(np, 0.0), minv(np, 0.0);
    for (int i = 0; i < n; ++i) {
        dsell[static_cast<size_t>(i)] = diag[static_cast<size_t>(S.perm[static_cast<size_t>(i)])];
        minv[static_cast<size_t>(i)] = 1.0 / dsell[static_cast<size_t>(i)];
    }
    if (split) {
        std::vector<double> rs(np, 0.0);
        parallel_for(n, [&](int64_t b, int64_t e) {
            for (int64_t i = b; i < e; ++i) {
                const int old = S.perm[static_cast<size_t>(i)];
                double acc = 0.0;
                for (int k = row_ptr[old]; k < row_ptr[old + 1]; ++k) acc += values[k];
                rs[static_cast<size_t>(i)] = acc;
            }
        });
        std::vector<unsigned char> rb = convert(rs, o.vector_type);
        h->d_rowsum = dalloc<unsigned char>(h, np * xs);
        cuda_check(cudaMemcpyAsync(h->d_rowsum, rb.data(), rb.size(), cudaMemcpyHostToDevice, st), "H2D");
        h->d_diag64 = dalloc<double>(h, np);
        cuda_check(cudaMemcpyAsync(h->d_diag64, dsell.data(), np * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
    }
    std::vector<unsigned char> mb = convert(minv, o.vector_type);
    cuda_check(cudaMemcpyAsync(h->d_minv, mb.data(), mb.size(), cudaMemcpyHostToDevice, st), "H2D");
    if (grid > 0) {
        const int per_block = (S.n_slices + grid - 1) / grid;
        win.assign(static_cast<size_t>(grid), make_int2(0, 0));
        for (int b = 0; b < grid; ++b) {
            const int sb = b * per_block, se = std::min(S.n_slices, sb + per_block);
            if (se <= sb) continue;
            int lo = sb * 32, hi = se * 32;
            for (int64_t pos = S.slice_ptr[static_cast<size_t>(sb)]; pos < S.slice_ptr[static_cast<size_t>(se)]; ++pos) {
                lo = std::min(lo, S.col[static_cast<size_t>(pos)]);
                hi = std::max(hi, S.col[static_cast<size_t>(pos)] + 1);
            }
            lo &= ~3;  // 16-byte aligned window
            hi = std::min(S.n_pad, (hi + 3) & ~3);
            win[static_cast<size_t>(b)] = make_int2(lo, hi - lo);
        }
    }
    cuda_check(cudaStreamSynchronize(st), "sync");  // the host images go next
}

void create(const int* row_ptr, const int* col_idx, const double* values, int n,
            const xplus_opts* opts_in, xplus_pcg** out) {
    require(row_ptr && col_idx && values && out, XPLUS_ERR_ARG, "null argument");
    require(n > 0, XPLUS_ERR_ARG, "n must be positive");
    const auto t0 = std::chrono::steady_clock::now();
    xplus_opts o;
    xplus_opts_default(&o);
    if (opts_in) o = *opts_in;
    require(o.value_type == XPLUS_F32 || o.value_type == XPLUS_BF16 || o.value_type == XPLUS_F16 ||
                o.value_type == XPLUS_F64, XPLUS_ERR_ARG, "bad value_type");
    require(o.vector_type == XPLUS_F32 || o.vector_type == XPLUS_F64, XPLUS_ERR_ARG, "bad vector_type");
    require(o.slice_height == 32, XPLUS_ERR_ARG, "slice_height must be 32");
    require(o.chunk == 1 || o.chunk == 2 || o.chunk == 4, XPLUS_ERR_ARG, "chunk must be 1, 2 or 4");
    require(o.sigma >= 1, XPLUS_ERR_ARG, "sigma must be >= 1");
    require(o.restart_on_replace >= -1 && o.restart_on_replace <= 4, XPLUS_ERR_ARG, "restart_on_replace must be -1..4");
    // Row-sum form for FP32/BF16 values: slots hold the off-diagonal weights, the row sums
    // s_i = sum_j a_ij (FP64 sum) are kept apart in the vector type, and the FP64 diagonal
    // stays apart for the true residual.
    const bool split = (o.value_type != XPLUS_F64) && o.row_sum_form;
    require((o.value_type != XPLUS_BF16 && o.value_type != XPLUS_F16) || split, XPLUS_ERR_ARG,
            "16-bit values need row_sum_form");
    // Everything is derived on the GPU from one device copy of the CSR, unless the 16-bit
    // two-term rewrite (a host CSR transformation) or a sort window beyond the device
    // builder's 4096 asks for the host layout.
    const bool on_device = o.build_on_gpu && o.sigma <= 4096 && split_ratio_of(o) <= 0.0;
    std::vector<double> diag;
    if (!on_device) {
        validate_csr(n, row_ptr, col_idx, row_ptr[n]);
        diag.resize(static_cast<size_t>(n));
        jacobi_diag(n, row_ptr, col_idx, values, diag.data());
        for (int i = 0; i < n; ++i)
            require(std::fabs(diag[static_cast<size_t>(i)]) > 1.0e-30, XPLUS_ERR_DATA,
                    "zero diagonal entry while building Jacobi inverse");
    }
    require_device(o.device);
    cuda_check(cudaSetDevice(o.device), "cudaSetDevice");

    auto* h = new xplus_pcg();
    h->device = o.device;
    try {
        h->opts = o;
        h->key = KernelKey{o.value_type, o.vector_type, o.chunk, split ? 1 : 0, 0, 0};
        h->n = n;
        h->nnz = row_ptr[n];
        cuda_check(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_check(cudaEventCreate(&h->ev0), "cudaEventCreate");
        cuda_check(cudaEventCreate(&h->ev1), "cudaEventCreate");
        // SM-resident kernel candidate: one block per SM, windows computed with the layout
        int sms = 0;
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o.device), "attr");
        const int res_grid = o.resident && resident_supported(h->key) ? sms : 0;
        std::vector<int2> win;
        if (on_device) create_layout_device(h, o, split, n, row_ptr, col_idx, values, res_grid, win);
        else create_layout_host(h, o, split, n, row_ptr, col_idx, values, diag, res_grid, win);
        const size_t np = static_cast<size_t>(h->n_pad);
        const size_t xs = elem_size(o.vector_type);
        h->d_b64 = dalloc<double>(h, np);
        h->d_x64 = dalloc<double>(h, np);
        // {z, p} records, or for the one-barrier resident kernel {m r, m Ap, p} x 2 generations
        h->d_rec = dalloc<unsigned char>(h, np * std::max<size_t>(xs * 2, 6 * sizeof(float)));
        h->d_r = dalloc<unsigned char>(h, np * xs);
        h->d_ap = dalloc<unsigned char>(h, np * xs);
        h->d_sx = dalloc<unsigned char>(h, np * xs);
        h->d_sy = dalloc<unsigned char>(h, np * xs);
        h->d_bio = dalloc<double>(h, static_cast<size_t>(n));
        h->d_xio = dalloc<double>(h, static_cast<size_t>(n));
        h->d_bar = dalloc<unsigned>(h, 1);
        h->d_err = dalloc<int>(h, 1);
        h->d_out = dalloc<PcgOut>(h, 1);
        cudaStream_t st = h->stream;
        const int want_tpb = o.block_threads > 0 ? o.block_threads : 512;
        // SM-resident kernel when its shared-memory band + halo fits one CTA per SM
        if (res_grid > 0) {
            const int per_block = (h->n_slices + res_grid - 1) / res_grid;
            if (per_block <= resident_max_slices()) {
                int max_wn = 0, max_nb = 0;
                for (int b = 0; b < res_grid; ++b) {
                    const int sb = b * per_block, se = std::min(h->n_slices, sb + per_block);
                    if (se <= sb) continue;
                    max_wn = std::max(max_wn, win[static_cast<size_t>(b)].y);
                    max_nb = std::max(max_nb, (se - sb) * 32);
                }
                const size_t smem = sizeof(float) * (static_cast<size_t>(max_wn) + 5 * static_cast<size_t>(max_nb));
                bool fits = false;
                h->one_sync = o.barriers_per_iter != 2;
                cuda_check(resident_prepare(h->key, o.device, smem, want_tpb, h->one_sync, &fits), "resident_prepare");
                if (fits) {
                    h->resident = true;
                    h->smem_bytes = smem;
                    h->grid = res_grid;
                    h->tpb = want_tpb;
                    h->d_win = dalloc<int2>(h, win.size());
                    cuda_check(cudaMemcpyAsync(h->d_win, win.data(), win.size() * sizeof(int2), cudaMemcpyHostToDevice, st), "H2D");
                }
            }
        }
        if (!h->resident) {
            cuda_check(pcg_grid(h->key, o.device, h->n_slices, want_tpb, o.blocks_per_sm, &h->grid, &h->tpb), "pcg_grid");
            request_l2(h);
        }
        h->d_partial = dalloc<double>(h, static_cast<size_t>(16) * h->grid);
        h->d_block_clk = dalloc<long long>(h, static_cast<size_t>(4) * h->grid);
        cuda_check(cudaMemsetAsync(h->d_x64, 0, np * sizeof(double), st), "memset");
        cuda_check(cudaStreamSynchronize(st), "sync");
        h->last.setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        *out = h;
    } catch (...) {
        destroy(h);
        throw;
    }
}

void ensure_trace(xplus_pcg* h, int cap) {
    if (cap <= h->trace_cap) return;
    if (h->d_trace) {
        cudaFree(h->d_trace);
        h->allocations.erase(std::remove(h->allocations.begin(), h->allocations.end(), static_cast<void*>(h->d_trace)), h->allocations.end());
        h->d_trace = nullptr;
    }
    h->d_trace = dalloc<double>(h, static_cast<size_t>(cap) * 5);
    h->trace_cap = cap;
}

// Enqueue one solve on stream st: b64/x64 already in SELL order on the device.
void enqueue_solve(xplus_pcg* h, double tau, int tau_mode, int max_iters_in, int trace_rows, cudaStream_t st) {
    require(tau > 0.0 && tau == tau, XPLUS_ERR_ARG, "tau must be positive");
    require(tau_mode == XPLUS_TAU_ABS_RR || tau_mode == XPLUS_TAU_REL_TRUE, XPLUS_ERR_ARG, "bad tau_mode");
    const int max_iters = max_iters_in > 0 ? max_iters_in : std::max(4 * h->n, 1000);
    PcgArgs a{};
    a.n = h->n;
    a.n_pad = h->n_pad;
    a.n_slices = h->n_slices;
    a.slice_ptr = h->d_slice_ptr;
    a.col = h->d_col;
    a.val = h->d_val;
    a.val_scale = static_cast<float>(h->val_scale);
    a.val64 = h->d_val64;
    a.rowsum = h->d_rowsum;
    a.diag64 = h->d_diag64;
    a.minv = h->d_minv;
    a.b64 = h->d_b64;
    a.x64 = h->d_x64;
    a.rec = h->d_rec;
    a.r = h->d_r;
    a.ap = h->d_ap;
    a.partial = h->d_partial;
    a.bar = h->d_bar;
    a.err = h->d_err;
    a.out = h->d_out;
    a.trace = trace_rows > 0 ? h->d_trace : nullptr;
    a.trace_cap = trace_rows;
    a.max_iters = max_iters;
    a.debug_skip_block = h->debug_skip_block;
    a.win = h->d_win;
    a.block_clk = h->d_block_clk;
    a.flush_every = 16;
    a.timeout_ns = static_cast<long long>((h->opts.barrier_timeout_s > 0 ? h->opts.barrier_timeout_s : 2.0) * 1e9);
    stagnation_args(h->opts, &a.stag_factor, &a.stag_window);
    if (tau_mode == XPLUS_TAU_ABS_RR) {
        a.tau_rr = tau;
        a.tau_true_rr = -1.0;
    } else {
        require(h->d_val64 != nullptr, XPLUS_ERR_ARG, "TAU_REL_TRUE needs keep_fp64 (the FP64 matrix copy)");
        a.tau_true_rr = 0.0;
        a.tau2_rel = tau * tau;  // the kernel scales it by ||b||^2 of the b on the device
        a.tau_rr = 0.0;
        a.replace_every = h->opts.replace_every;
        a.replace_drop = h->opts.replace_drop > 0.0 ? h->opts.replace_drop * h->opts.replace_drop : 0.0;
        const bool low = h->opts.value_type == XPLUS_BF16 || h->opts.value_type == XPLUS_F16;
        a.restart_on_replace = h->opts.restart_on_replace < 0 ? (low ? 4 : 0) : h->opts.restart_on_replace;
    }
    cuda_check(cudaMemsetAsync(h->d_bar, 0, sizeof(unsigned), st), "memset");
    cuda_check(cudaMemsetAsync(h->d_err, 0, sizeof(int), st), "memset");
    cuda_check(cudaMemsetAsync(h->d_out, 0, sizeof(PcgOut), st), "memset");
    cuda_check(cudaEventRecord(h->ev0, st), "event");
    if (h->gtg) {
        a.g_slice_ptr = h->d_g_slice_ptr;
        a.g_col = h->d_g_col;
        a.g_val = h->d_g_val;
        a.gt_slice_ptr = h->d_gt_slice_ptr;
        a.gt_col = h->d_gt_col;
        a.gt_val = h->d_gt_val;
        a.t = h->d_t;
        a.r2 = h->d_r2;
        a.g_fallback_iters = h->g_fallback_iters;
        cuda_check(gtg_launch(h->key, a, h->gtg_grid, 512, st, h->window), "GTG PCG launch");
    } else if (h->resident)
        // no access-policy window: the resident kernel's only global stream is a matrix that L2
        // holds anyway, and the launch attribute cost time (1108^2 system: 97.1 ms with it,
        // 95.9 ms without, and ~3 ms more on the host per solve call)
        cuda_check(resident_launch(h->key, a, h->grid, h->tpb, h->smem_bytes, h->one_sync, st,
                                   cudaAccessPolicyWindow{}),
                   "resident PCG launch");
    else
        cuda_check(pcg_launch(h->key, a, h->grid, h->tpb, st, h->window), "persistent PCG launch");
    cuda_check(cudaEventRecord(h->ev1, st), "event");
    h->pending = true;
}

void collect(xplus_pcg* h, xplus_metrics* m) {
    if (h->pending) {
        cuda_check(cudaEventSynchronize(h->ev1), "sync");
        PcgOut o{};
        int err = 0;
        cuda_check(cudaMemcpy(&o, h->d_out, sizeof(PcgOut), cudaMemcpyDeviceToHost), "D2H");
        cuda_check(cudaMemcpy(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost), "D2H");
        float ms = 0.0f;
        cuda_check(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "event");
        xplus_metrics& L = h->last;
        L.status = err ? XPLUS_TIMEOUT : o.status;
        L.iterations = o.iterations;
        L.replacements = o.replacements;
        L.rz = o.rz;
        L.rr = o.rr;
        L.pap = o.pap;
        L.alpha = o.alpha;
        L.true_rel_residual = o.bb > 0 ? std::sqrt(o.true_rr / o.bb) : std::sqrt(o.true_rr);
        L.kernel_ms = ms;
        L.reserved[0] = o.stagnated;
        L.reserved[1] = static_cast<double>(o.t_end_ns - o.t_start_ns) * 1e-6;
        L.reserved[2] = h->gtg ? 3.0 : (h->resident ? (h->one_sync ? 2.0 : 1.0) : 0.0);
        L.reserved[3] = h->gtg ? o.reserved : -1.0;
        h->phase_ns[0] = o.t_phase[0];
        h->phase_ns[1] = o.t_phase[1];
        h->phase_ns[2] = o.t_phase[2];
        h->phase_ns[3] = o.t_phase[3];
        h->pending = false;
    }
    if (m) *m = h->last;
}

// SELL image (C = 32, chunk 2) of a matrix given by rows in SELL order: rows[r] lists
// (column in SELL order, source index into g_low).  Padding slots: own row, source -1.
void gtg_sell(const std::vector<std::vector<std::pair<int, int>>>& rows, int n_pad, std::vector<long long>& sp,
              std::vector<int>& col, std::vector<int>& map) {
    const int ns = n_pad / 32;
    sp.assign(static_cast<size_t>(ns) + 1, 0);
    for (int s = 0; s < ns; ++s) {
        size_t w = 0;
        for (int l = 0; l < 32; ++l) w = std::max(w, rows[static_cast<size_t>(s * 32 + l)].size());
        w = (w + 1) / 2 * 2;
        sp[static_cast<size_t>(s) + 1] = sp[static_cast<size_t>(s)] + static_cast<long long>(w) * 32;
    }
    col.assign(static_cast<size_t>(sp.back()), 0);
    map.assign(static_cast<size_t>(sp.back()), -1);
    for (int s = 0; s < ns; ++s) {
        const size_t w = static_cast<size_t>((sp[static_cast<size_t>(s) + 1] - sp[static_cast<size_t>(s)]) / 32);
        for (int l = 0; l < 32; ++l) {
            const int r = s * 32 + l;
            const auto& e = rows[static_cast<size_t>(r)];
            for (size_t j = 0; j < w; ++j) {
                const size_t pos = static_cast<size_t>(sp[static_cast<size_t>(s)]) + (j / 2) * 64 + static_cast<size_t>(l) * 2 + j % 2;
                if (j < e.size()) {
                    col[pos] = e[j].first;
                    map[pos] = e[j].second;
                } else {
                    col[pos] = r;
                }
            }
        }
    }
}

// Builds the G / G^T SELL images for the pattern of the CSR given to xplus_pcg_create (once).
// The host construction of the G / G^T images (the reference for gtg_layout_device).
void gtg_layout_host(xplus_pcg* h, const int* row_ptr, const int* col_idx) {
    const int n = h->n;
    std::vector<int> iperm(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) iperm[static_cast<size_t>(h->perm[static_cast<size_t>(i)])] = i;
    std::vector<std::vector<std::pair<int, int>>> g(static_cast<size_t>(h->n_pad)), gt(static_cast<size_t>(h->n_pad));
    int gl = 0;
    for (int i = 0; i < n; ++i)
        for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
            const int j = col_idx[q];
            require(j >= 0 && j < n, XPLUS_ERR_DATA, "column index out of range");
            if (j > i) continue;
            const int ri = iperm[static_cast<size_t>(i)], rj = iperm[static_cast<size_t>(j)];
            g[static_cast<size_t>(ri)].push_back({rj, gl});
            gt[static_cast<size_t>(rj)].push_back({ri, gl});
            ++gl;
        }
    h->n_glow = gl;
    std::vector<long long> sp, tsp;
    std::vector<int> col, map, tcol, tmap;
    gtg_sell(g, h->n_pad, sp, col, map);
    gtg_sell(gt, h->n_pad, tsp, tcol, tmap);
    require(col.size() < (1ULL << 31) && tcol.size() < (1ULL << 31), XPLUS_ERR_ARG, "G too large (2^31 slots)");
    h->g_slots = static_cast<int64_t>(col.size());
    h->gt_slots = static_cast<int64_t>(tcol.size());
    cudaStream_t st = h->stream;
    h->d_g_slice_ptr = dalloc<long long>(h, sp.size());
    h->d_gt_slice_ptr = dalloc<long long>(h, tsp.size());
    h->d_g_col = dalloc<int>(h, col.size());
    h->d_gt_col = dalloc<int>(h, tcol.size());
    h->d_g_map = dalloc<int>(h, map.size());
    h->d_gt_map = dalloc<int>(h, tmap.size());
    cuda_check(cudaMemcpyAsync(h->d_g_slice_ptr, sp.data(), sp.size() * sizeof(long long), cudaMemcpyHostToDevice, st), "H2D");
    cuda_check(cudaMemcpyAsync(h->d_gt_slice_ptr, tsp.data(), tsp.size() * sizeof(long long), cudaMemcpyHostToDevice, st), "H2D");
    cuda_check(cudaMemcpyAsync(h->d_g_col, col.data(), col.size() * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    cuda_check(cudaMemcpyAsync(h->d_gt_col, tcol.data(), tcol.size() * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    cuda_check(cudaMemcpyAsync(h->d_g_map, map.data(), map.size() * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    cuda_check(cudaMemcpyAsync(h->d_gt_map, tmap.data(), tmap.size() * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    cuda_check(cudaStreamSynchronize(st), "sync");  // the host images go next
}

// The G / G^T images and the vectors of the G^T G kernel for the pattern of the CSR given to
// xplus_pcg_create (once per handle): on the GPU unless the handle was built on the host.
void gtg_layout(xplus_pcg* h, const int* row_ptr, const int* col_idx) {
    require(h->opts.vector_type == XPLUS_F32 && h->key.diag && h->opts.value_type != XPLUS_F64,
            XPLUS_ERR_ARG, "G^T G preconditioning needs FP32 vectors, FP32, BF16 or FP16 values and row_sum_form");
    require(h->d_val64 != nullptr, XPLUS_ERR_ARG, "G^T G preconditioning needs keep_fp64");
    if (h->d_g_slice_ptr) return;
    const int n = h->n;
    require(row_ptr && col_idx && row_ptr[0] == 0 && row_ptr[n] == h->nnz, XPLUS_ERR_ARG,
            "pattern differs from the matrix of the handle");
    if (h->opts.build_on_gpu) {
        const GtgImages im = gtg_layout_device(n, h->n_pad, row_ptr, col_idx, h->d_perm,
                                               [h](size_t bytes) { return static_cast<void*>(dalloc<unsigned char>(h, bytes)); },
                                               h->stream);
        h->n_glow = im.n_glow;
        h->g_slots = im.g_slots;
        h->gt_slots = im.gt_slots;
        h->d_g_slice_ptr = im.g_slice_ptr;
        h->d_gt_slice_ptr = im.gt_slice_ptr;
        h->d_g_col = im.g_col;
        h->d_g_map = im.g_map;
        h->d_gt_col = im.gt_col;
        h->d_gt_map = im.gt_map;
    } else {
        gtg_layout_host(h, row_ptr, col_idx);
    }
    cudaStream_t st = h->stream;
    h->d_g_val = dalloc<float>(h, static_cast<size_t>(h->g_slots));
    h->d_gt_val = dalloc<float>(h, static_cast<size_t>(h->gt_slots));
    h->d_t = dalloc<float>(h, static_cast<size_t>(h->n_pad));
    h->d_r2 = dalloc<float>(h, static_cast<size_t>(h->n_pad));
    h->d_glow = dalloc<double>(h, static_cast<size_t>(h->n_glow));
    cuda_check(cudaMemsetAsync(h->d_r2, 0, static_cast<size_t>(h->n_pad) * sizeof(float), st), "memset");
    cuda_check(cudaMemsetAsync(h->d_t, 0, static_cast<size_t>(h->n_pad) * sizeof(float), st), "memset");
    int gtg_tpb = 0;
    cuda_check(gtg_grid(h->key, h->device, h->n_slices, &h->gtg_grid, &gtg_tpb), "gtg grid");
    if (h->gtg_grid > h->grid) {
        // partial sums and the per-CTA clock are sized by the grid
        h->d_partial = dalloc<double>(h, static_cast<size_t>(16) * h->gtg_grid);
        h->d_block_clk = dalloc<long long>(h, static_cast<size_t>(4) * h->gtg_grid);
    }
    cuda_check(cudaStreamSynchronize(st), "sync");
}

// G values (device, g_low order) -> the two SELL images; switches the handle to G^T G
void gtg_enable(xplus_pcg* h, int fallback_iters) {
    cudaStream_t st = h->stream;
    cuda_check(gtg_fill_values(h->d_glow, h->d_g_map, h->d_g_val, h->g_slots, st), "gtg fill");
    cuda_check(gtg_fill_values(h->d_glow, h->d_gt_map, h->d_gt_val, h->gt_slots, st), "gtg fill");
    cuda_check(cudaStreamSynchronize(st), "sync");
    h->g_fallback_iters = fallback_iters;
    h->gtg = true;
    request_l2(h);
}

}  // namespace
}  // namespace xplus

using namespace xplus;

extern "C" {

const char* xplus_version(void) { return "xplus-b200 0.1 (sm_100a)"; }

void xplus_opts_default(xplus_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->value_type = XPLUS_F32;
    o->vector_type = XPLUS_F32;
    o->slice_height = 32;
    o->sigma = 256;
    o->chunk = 4;
    o->keep_fp64 = 1;
    o->replace_every = 0;
    o->replace_drop = 1.0e-2;
    o->block_threads = 0;
    o->blocks_per_sm = 0;
    o->barrier_timeout_s = 2.0;
    o->device = 0;
    o->row_sum_form = 1;
    o->index16 = 1;
    o->l2_persist = 1;
    o->resident = 1;
    o->barriers_per_iter = 1;
    o->restart_on_replace = -1;
    o->stagnation_gain = 0.05;
    o->stagnation_window = 8;
    o->build_on_gpu = 1;
    o->split_ratio = -1.0;
}

int xplus_device_count(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int good = 0;
    for (int d = 0; d < count; ++d) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10) ++good;
    }
    cudaGetLastError();
    return good;
}

int xplus_pcg_create(const int* row_ptr, const int* col_idx, const double* values, int n,
                     const xplus_opts* opts, xplus_pcg** out) {
    return guarded([&] { create(row_ptr, col_idx, values, n, opts, out); });
}

int xplus_pcg_destroy(xplus_pcg* h) {
    return guarded([&] { destroy(h); });
}

int xplus_pcg_solve(xplus_pcg* h, const double* b, const double* x0, double tau, int tau_mode,
                    int max_iters, double* x_out, int* iters_out, double* resid_hist, int hist_len,
                    xplus_metrics* metrics) {
    return guarded([&] {
        require(h && b && x_out, XPLUS_ERR_ARG, "null argument");
        cuda_check(cudaSetDevice(h->device), "cudaSetDevice");
        cudaStream_t st = h->stream;
        const size_t nb = sizeof(double) * static_cast<size_t>(h->n);
        cuda_check(cudaMemcpyAsync(h->d_bio, b, nb, cudaMemcpyHostToDevice, st), "H2D");
        if (x0) cuda_check(cudaMemcpyAsync(h->d_xio, x0, nb, cudaMemcpyHostToDevice, st), "H2D");
        else cuda_check(cudaMemsetAsync(h->d_xio, 0, nb, st), "memset");
        cuda_check(gather_to_sell(XPLUS_F64, h->d_bio, h->d_b64, h->d_perm, h->n, h->n_pad, st), "gather");
        cuda_check(gather_to_sell(XPLUS_F64, h->d_xio, h->d_x64, h->d_perm, h->n, h->n_pad, st), "gather");
        const int rows = resid_hist && hist_len > 0 ? hist_len : 0;
        if (rows > 0) ensure_trace(h, rows);
        enqueue_solve(h, tau, tau_mode, max_iters, rows, st);
        cuda_check(scatter_from_sell(h->d_x64, h->d_xio, h->d_perm, h->n, st), "scatter");
        cuda_check(cudaMemcpyAsync(x_out, h->d_xio, nb, cudaMemcpyDeviceToHost, st), "D2H");
        std::vector<double> tr;
        if (rows > 0) {
            tr.resize(static_cast<size_t>(rows) * 5);
            cuda_check(cudaMemcpyAsync(tr.data(), h->d_trace, tr.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        }
        cuda_check(cudaStreamSynchronize(st), "sync");
        xplus_metrics m;
        collect(h, &m);
        if (iters_out) *iters_out = m.iterations;
        if (rows > 0)
            for (int k = 0; k < rows; ++k) resid_hist[k] = k < m.iterations ? tr[static_cast<size_t>(k) * 5 + 4] : 0.0;
        if (metrics) *metrics = m;
    });
}

int xplus_pcg_last_trace(xplus_pcg* h, double* trace, int rows) {
    return guarded([&] {
        require(h && trace && rows > 0 && rows <= h->trace_cap, XPLUS_ERR_ARG, "bad trace request");
        collect(h, nullptr);  // waits for a pending solve
        cuda_check(cudaMemcpyAsync(trace, h->d_trace, static_cast<size_t>(rows) * 5 * sizeof(double), cudaMemcpyDeviceToHost,
                                   h->stream), "D2H");
        cuda_check(cudaStreamSynchronize(h->stream), "sync");
    });
}

int xplus_pcg_solve_device(xplus_pcg* h, const double* d_b, double* d_x, double tau, int tau_mode,
                           int max_iters, void* stream) {
    return guarded([&] {
        require(h && d_b && d_x, XPLUS_ERR_ARG, "null argument");
        cuda_check(cudaSetDevice(h->device), "cudaSetDevice");
        require_device_memory(d_b, h->device, "d_b");
        require_device_memory(d_x, h->device, "d_x");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : h->stream;
        cuda_check(gather_to_sell(XPLUS_F64, d_b, h->d_b64, h->d_perm, h->n, h->n_pad, st), "gather");
        cuda_check(gather_to_sell(XPLUS_F64, d_x, h->d_x64, h->d_perm, h->n, h->n_pad, st), "gather");
        // stream-ordered: the kernel sums ||b||^2 for the relative test itself, so nothing
        // here waits for the device
        enqueue_solve(h, tau, tau_mode, max_iters, 0, st);
        cuda_check(scatter_from_sell(h->d_x64, d_x, h->d_perm, h->n, st), "scatter");
    });
}

int xplus_pcg_debug_skip_arrival(xplus_pcg* h, int block) {
    return guarded([&] {
        require(h && block >= -1, XPLUS_ERR_ARG, "bad argument");
        h->debug_skip_block = block;
    });
}

int xplus_pcg_last_phase_times(xplus_pcg* h, double* ms4) {
    return guarded([&] {
        require(h && ms4, XPLUS_ERR_ARG, "null argument");
        collect(h, nullptr);
        for (int k = 0; k < 4; ++k) ms4[k] = static_cast<double>(h->phase_ns[k]) * 1e-6;
    });
}

int xplus_pcg_last_block_times(xplus_pcg* h, double* ms, int max_blocks, int* blocks) {
    return guarded([&] {
        require(h && blocks, XPLUS_ERR_ARG, "null argument");
        collect(h, nullptr);
        const int grid = h->gtg ? h->gtg_grid : h->grid;
        *blocks = grid;
        if (!ms) return;
        const int nb = std::min(max_blocks, grid);
        std::vector<long long> t(static_cast<size_t>(4) * grid);
        cuda_check(cudaMemcpy(t.data(), h->d_block_clk, t.size() * sizeof(long long), cudaMemcpyDeviceToHost), "D2H");
        for (int k = 0; k < 4 * nb; ++k) ms[k] = static_cast<double>(t[static_cast<size_t>(k)]) * 1e-6;
    });
}

int xplus_pcg_last_metrics(xplus_pcg* h, xplus_metrics* metrics) {
    return guarded([&] {
        require(h && metrics, XPLUS_ERR_ARG, "null argument");
        collect(h, metrics);
    });
}

int xplus_pcg_spmv(xplus_pcg* h, const double* x, double* y) {
    return guarded([&] {
        require(h && x && y, XPLUS_ERR_ARG, "null argument");
        cuda_check(cudaSetDevice(h->device), "cudaSetDevice");
        cudaStream_t st = h->stream;
        const size_t nb = sizeof(double) * static_cast<size_t>(h->n);
        cuda_check(cudaMemcpyAsync(h->d_xio, x, nb, cudaMemcpyHostToDevice, st), "H2D");
        cuda_check(gather_to_sell(h->opts.vector_type, h->d_xio, h->d_sx, h->d_perm, h->n, h->n_pad, st), "gather");
        SpmvArgs a{h->n_pad, h->n_slices, h->d_slice_ptr, h->d_col, h->d_val, h->d_rowsum,
                   static_cast<float>(h->val_scale)};
        cuda_check(spmv_launch(h->key, a, h->d_sx, h->d_sy, st), "spmv");
        // widen the SELL-order result to FP64 and scatter to original order
        std::vector<unsigned char> ys(static_cast<size_t>(h->n_pad) * elem_size(h->opts.vector_type));
        cuda_check(cudaMemcpyAsync(ys.data(), h->d_sy, ys.size(), cudaMemcpyDeviceToHost, st), "D2H");
        std::vector<int> perm(static_cast<size_t>(h->n));
        cuda_check(cudaMemcpyAsync(perm.data(), h->d_perm, perm.size() * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        cuda_check(cudaStreamSynchronize(st), "sync");
        for (int i = 0; i < h->n; ++i) {
            const double v = h->opts.vector_type == XPLUS_F64 ? reinterpret_cast<double*>(ys.data())[i]
                                                              : static_cast<double>(reinterpret_cast<float*>(ys.data())[i]);
            y[perm[static_cast<size_t>(i)]] = v;
        }
    });
}

int xplus_pcg_spmv_device(xplus_pcg* h, const void* d_x, void* d_y, void* stream) {
    return guarded([&] {
        require(h && d_x && d_y, XPLUS_ERR_ARG, "null argument");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : h->stream;
        SpmvArgs a{h->n_pad, h->n_slices, h->d_slice_ptr, h->d_col, h->d_val, h->d_rowsum,
                   static_cast<float>(h->val_scale)};
        cuda_check(spmv_launch(h->key, a, d_x, d_y, st), "spmv");
    });
}

int xplus_pcg_info(xplus_pcg* h, int64_t* n, int64_t* n_pad, int64_t* nnz, int64_t* slots,
                   int64_t* spmv_bytes) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        if (n) *n = h->n;
        if (n_pad) *n_pad = h->n_pad;
        if (nnz) *nnz = h->nnz;
        if (slots) *slots = h->slots;
        if (spmv_bytes) {
            // bytes of one SpMV in the stored format, padding excluded: every stored entry
            // (value + column index), the row sums when kept apart, x read once, y written once
            const bool split = h->key.diag != 0;
            const int64_t entries = split ? h->nnz - h->n : h->nnz;
            const int64_t sv = static_cast<int64_t>(elem_size(h->opts.value_type));
            const int64_t si = h->key.idx16 ? 2 : 4;
            const int64_t sx = static_cast<int64_t>(elem_size(h->opts.vector_type));
            *spmv_bytes = entries * (sv + si) + static_cast<int64_t>(h->n) * (2 * sx + (split ? sx : 0));
        }
    });
}

int xplus_pcg_scratch_vectors(xplus_pcg* h, void** d_x, void** d_y) {
    return guarded([&] {
        require(h && d_x && d_y, XPLUS_ERR_ARG, "null argument");
        *d_x = h->d_sx;
        *d_y = h->d_sy;
    });
}

int xplus_pcg_control(xplus_pcg* h, const double* b, const double* m_inv, double* x, double* r,
                      double* z, double* p, double* ap, double* metrics, int* status, double tau,
                      int max_iters, int n, void* stream) {
    return guarded([&] {
        require(h && b && x && metrics && status, XPLUS_ERR_ARG, "null argument");
        cuda_check(cudaSetDevice(h->device), "cudaSetDevice");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : h->stream;
        (void)m_inv; (void)r; (void)z; (void)p; (void)ap;
        // Parameter check of kernels/cuper_pcg_control_kernel.cpp:1078-1087.
        if (n != h->n || n <= 0 || max_iters < 0 || !(tau > 0.0)) {
            const int st_bad[2] = {XPLUS_BREAKDOWN, 0};
            const double zero[4] = {0, 0, 0, 0};
            cuda_check(cudaMemcpyAsync(status, st_bad, sizeof(st_bad), cudaMemcpyHostToDevice, st), "H2D");
            cuda_check(cudaMemcpyAsync(metrics, zero, sizeof(zero), cudaMemcpyHostToDevice, st), "H2D");
            cuda_check(cudaStreamSynchronize(st), "sync");
            return;
        }
        cuda_check(gather_to_sell(XPLUS_F64, b, h->d_b64, h->d_perm, h->n, h->n_pad, st), "gather");
        cuda_check(gather_to_sell(XPLUS_F64, x, h->d_x64, h->d_perm, h->n, h->n_pad, st), "gather");
        enqueue_solve(h, tau, XPLUS_TAU_ABS_RR, max_iters > 0 ? max_iters : std::max(4 * n, 1000), 0, st);
        cuda_check(scatter_from_sell(h->d_x64, x, h->d_perm, h->n, st), "scatter");
        xplus_metrics m;
        collect(h, &m);
        const int st_out[2] = {m.status, m.iterations};
        const double met[4] = {m.rz, m.rr, m.pap, m.alpha};
        cuda_check(cudaMemcpyAsync(status, st_out, sizeof(st_out), cudaMemcpyHostToDevice, st), "H2D");
        cuda_check(cudaMemcpyAsync(metrics, met, sizeof(met), cudaMemcpyHostToDevice, st), "H2D");
        cuda_check(cudaStreamSynchronize(st), "sync");
    });
}

int xplus_pcg_set_gtg(xplus_pcg* h, const int* row_ptr, const int* col_idx, const double* g_low,
                      int fallback_iters) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        cuda_check(cudaSetDevice(h->device), "cudaSetDevice");
        if (!g_low) {
            h->gtg = false;
            return;
        }
        require(fallback_iters >= 0, XPLUS_ERR_ARG, "fallback_iters must be >= 0");
        gtg_layout(h, row_ptr, col_idx);
        cuda_check(cudaMemcpyAsync(h->d_glow, g_low, static_cast<size_t>(h->n_glow) * sizeof(double),
                                   cudaMemcpyHostToDevice, h->stream), "H2D");
        gtg_enable(h, fallback_iters);
    });
}

int xplus_pcg_set_gnn(xplus_pcg* h, const int* row_ptr, const int* col_idx, const double* values,
                      const float* params, int fallback_iters, double* infer_ms) {
    return xplus_pcg_set_gnn_ex(h, row_ptr, col_idx, values, params, fallback_iters, 4, infer_ms);
}

int xplus_pcg_set_gnn_ex(xplus_pcg* h, const int* row_ptr, const int* col_idx, const double* values,
                         const float* params, int fallback_iters, int refine_sweeps, double* infer_ms) {
    return guarded([&] {
        require(h && values && params, XPLUS_ERR_ARG, "null argument");
        require(fallback_iters >= 0, XPLUS_ERR_ARG, "fallback_iters must be >= 0");
        require(refine_sweeps >= 0 && refine_sweeps <= 16, XPLUS_ERR_ARG, "refine_sweeps must be in [0, 16]");
        cuda_check(cudaSetDevice(h->device), "cudaSetDevice");
        gtg_layout(h, row_ptr, col_idx);
        const auto t0 = std::chrono::steady_clock::now();
        gnn::Arena ar;
        try {
            cudaStream_t st = h->stream;
            gnn::DevGraph dg;
            if (h->opts.build_on_gpu) {
                DeviceCsr csr;
                upload_csr(h->n, row_ptr, col_idx, values, csr, st);
                dg.build_on_device(h->n, csr.rp, csr.ci, csr.v, row_ptr, col_idx, values, ar, st);
            } else {
                gnn::HostGraph hg;
                hg.build(h->n, row_ptr, col_idx, values);
                dg.upload(hg, ar, st);
            }
            require(dg.n_glow == h->n_glow, XPLUS_ERR_DATA, "matrix pattern needs every diagonal entry");
            gnn::Work w;
            w.alloc(ar, dg.n, std::max(1, dg.n_low), 1, false);
            const int P = gnn::param_offsets().total;
            float* master = ar.get<float>(static_cast<size_t>(P));
            float* wr = ar.get<float>(static_cast<size_t>(P));
            cuda_check(cudaMemcpyAsync(master, params, static_cast<size_t>(P) * sizeof(float), cudaMemcpyHostToDevice, st), "H2D");
            gnn::round_params(master, wr, P, st);
            gnn::forward(dg, wr, w, false, st);
            gnn::refine_rows(dg, w, refine_sweeps, st);
            gnn::normalize_rows(dg, w, st);  // (G A G^T)_ii = 1: the network fixes only each row's direction
            gnn::g_to_low(dg, w, h->d_glow, st);
            gtg_enable(h, fallback_iters);
        } catch (...) {
            cudaStreamSynchronize(h->stream);
            ar.release();
            throw;
        }
        cudaStreamSynchronize(h->stream);
        ar.release();
        if (infer_ms) *infer_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    });
}

int xplus_pcg_scale_gtg(xplus_pcg* h, const int* row_ptr, const int* col_idx, const double* values) {
    return guarded([&] {
        require(h && row_ptr && col_idx && values, XPLUS_ERR_ARG, "null argument");
        require(h->gtg && h->d_glow != nullptr, XPLUS_ERR_ARG, "no G set on this handle");
        const int n = h->n;
        require(row_ptr[0] == 0 && row_ptr[n] == h->nnz, XPLUS_ERR_ARG, "pattern differs from the matrix of the handle");
        cuda_check(cudaSetDevice(h->device), "cudaSetDevice");
        // every copy on the handle's stream: it is a non-blocking stream, so a copy on the legacy
        // stream would not be ordered with the fill kernels that read d_glow
        std::vector<double> g(static_cast<size_t>(h->n_glow));
        cuda_check(cudaMemcpyAsync(g.data(), h->d_glow, g.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "D2H");
        cuda_check(cudaStreamSynchronize(h->stream), "sync");
        // g_low order: row by row, the entries j <= i of the CSR in their CSR order
        std::vector<int64_t> g0(static_cast<size_t>(n) + 1, 0);
        for (int i = 0; i < n; ++i) {
            int c = 0;
            for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q) c += col_idx[q] <= i;
            g0[static_cast<size_t>(i) + 1] = g0[static_cast<size_t>(i)] + c;
        }
        require(g0[static_cast<size_t>(n)] == h->n_glow, XPLUS_ERR_ARG, "pattern differs from the G of the handle");
        std::vector<int> bad(static_cast<size_t>(n), 0);
        parallel_for(n, [&](int64_t b, int64_t e) {
            std::vector<int> slot(static_cast<size_t>(n), -1);  // column -> position in row i's pattern
            for (int64_t i = b; i < e; ++i) {
                const int64_t gb = g0[static_cast<size_t>(i)];
                int t = 0;
                for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q)
                    if (col_idx[q] <= i) slot[static_cast<size_t>(col_idx[q])] = t++;
                // (G A G^T)_ii = sum over k, l in the pattern of g_ik a_kl g_il
                double d = 0.0;
                for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
                    const int k = col_idx[q];
                    if (k > i) continue;
                    const double gk = g[static_cast<size_t>(gb + slot[static_cast<size_t>(k)])];
                    if (gk == 0.0) continue;
                    double acc = 0.0;
                    for (int r = row_ptr[k]; r < row_ptr[k + 1]; ++r) {
                        const int l = col_idx[r];
                        if (l <= i && slot[static_cast<size_t>(l)] >= 0)
                            acc += values[r] * g[static_cast<size_t>(gb + slot[static_cast<size_t>(l)])];
                    }
                    d += gk * acc;
                }
                for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q)
                    if (col_idx[q] <= i) slot[static_cast<size_t>(col_idx[q])] = -1;
                if (!(d > 0.0)) {
                    bad[static_cast<size_t>(i)] = 1;
                    continue;
                }
                const double s = 1.0 / std::sqrt(d);
                for (int64_t u = gb; u < g0[static_cast<size_t>(i) + 1]; ++u) g[static_cast<size_t>(u)] *= s;
            }
        });
        for (int i = 0; i < n; ++i)
            require(!bad[static_cast<size_t>(i)], XPLUS_ERR_DATA, "a row of G has (G A G^T)_ii <= 0");
        cuda_check(cudaMemcpyAsync(h->d_glow, g.data(), g.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream), "H2D");
        gtg_enable(h, h->g_fallback_iters);  // fills G and G^T on the same stream, then waits
    });
}

int xplus_pcg_get_gtg(xplus_pcg* h, double* g_low, int64_t* n_glow) {
    return guarded([&] {
        require(h, XPLUS_ERR_ARG, "null handle");
        if (n_glow) *n_glow = h->n_glow;
        if (!g_low) return;
        require(h->d_glow != nullptr, XPLUS_ERR_ARG, "no G set on this handle");
        cuda_check(cudaMemcpyAsync(g_low, h->d_glow, static_cast<size_t>(h->n_glow) * sizeof(double), cudaMemcpyDeviceToHost,
                                   h->stream), "D2H");
        cuda_check(cudaStreamSynchronize(h->stream), "sync");
    });
}

}  // extern "C"
