// multikernel.cu -- the five "kernel functions" of the reference's multi-kernel path
// (archived/include/cg_kernels.hpp:9-54, archived/kernels/cg_kernels.cpp:43-159) on the GPU,
// same names and arguments, so the reference host loop
// (archived/host/multi_kernel_solver.hpp:100-234) links against this library unchanged.
//
// Arithmetic: every product and sum is rounded on its own (__dmul_rn/__dadd_rn: no FMA
// contraction), which is what the reference's x86-64 build computes.  The SpMV and the
// element-wise updates are therefore bit-identical to the reference.  The dot products
// (dot_kernel, and r.z, r.r of init_pcg_kernel / update_xrz_kernel) are summed in the
// reference's order, one element after the other from index 0, for n <= kSeqMaxN, so the
// whole path is bit-identical there (the reference itself stops at n <= 1024,
// include/cg_common.hpp:11); above that they use a fixed two-level tree (deterministic,
// within a few ulps of the sequential sum).
// Pointers may be device pointers or plain host pointers (staged).  Calls block until the
// results are in place, as the reference's calls do.
#include <cuda.h>  // CUcontext only: cuCtxGetCurrent is reached through cudaGetDriverEntryPoint
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "common.hpp"

namespace xplus {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 1024;
// Largest n whose dot products are summed sequentially (one dependent FP64 add per element,
// about 0.1 ms at this size); larger n use the tree.
constexpr int kSeqMaxN = 65536;

__global__ void csr_spmv_f64_kernel(const int* __restrict__ rp, const int* __restrict__ ci,
                                    const double* __restrict__ v, const double* __restrict__ x,
                                    double* __restrict__ y, int n) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    double acc = 0.0;
    for (int k = rp[row]; k < rp[row + 1]; ++k) acc = __dadd_rn(acc, __dmul_rn(v[k], x[ci[k]]));
    y[row] = acc;
}

__device__ __forceinline__ void block_reduce2(double& a, double& b, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sh[warp] = a;
        sh[32 + warp] = b;
    }
    __syncthreads();
    if (warp == 0) {
        a = lane < (blockDim.x >> 5) ? sh[lane] : 0.0;
        b = lane < (blockDim.x >> 5) ? sh[32 + lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
    }
}

// mode 0: dot(a, b) -> partial[2*blk]
// mode 1: init  r = b - ax, z = m_inv r, p = z; partials (r.z, r.r)
// mode 2: xrz   x += alpha p, r -= alpha ap, z = m_inv r; partials (r.z, r.r)
__global__ void vec_kernel(int mode, int n, double alpha, double* x, const double* p, double* r,
                           const double* ap, const double* m_inv, double* z, double* pp,
                           const double* b, double* partial) {
    __shared__ double sh[64];
    double s0 = 0.0, s1 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (mode == 0) {
            s0 = __dadd_rn(s0, __dmul_rn(x[i], p[i]));
        } else if (mode == 1) {
            const double rv = __dsub_rn(b[i], ap[i]);
            const double zv = __dmul_rn(m_inv[i], rv);
            r[i] = rv;
            z[i] = zv;
            pp[i] = zv;
            s0 = __dadd_rn(s0, __dmul_rn(rv, zv));
            s1 = __dadd_rn(s1, __dmul_rn(rv, rv));
        } else {
            x[i] = __dadd_rn(x[i], __dmul_rn(alpha, p[i]));
            const double rv = __dsub_rn(r[i], __dmul_rn(alpha, ap[i]));
            const double zv = __dmul_rn(m_inv[i], rv);
            r[i] = rv;
            z[i] = zv;
            s0 = __dadd_rn(s0, __dmul_rn(rv, zv));
            s1 = __dadd_rn(s1, __dmul_rn(rv, rv));
        }
    }
    block_reduce2(s0, s1, sh);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = s0;
        partial[2 * blockIdx.x + 1] = s1;
    }
}

// Sequential sums in the reference's order: lane 0 sums a_i * b_i, lane 1 sums c_i * d_i
// (nout == 2), each product and each sum rounded on its own.  The products are recomputed
// from the vectors the element-wise kernel wrote, exactly as that kernel computed them.
__global__ void seq_dot_kernel(const double* __restrict__ a, const double* __restrict__ b,
                               const double* __restrict__ c, const double* __restrict__ d, int n,
                               double* __restrict__ out, int nout) {
    const int lane = threadIdx.x;
    if (lane >= nout) return;
    const double* u = lane == 0 ? a : c;
    const double* v = lane == 0 ? b : d;
    double acc = 0.0;
    int i = 0;
    for (; i + 8 <= n; i += 8) {
        double q[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) q[k] = __dmul_rn(u[i + k], v[i + k]);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc = __dadd_rn(acc, q[k]);
    }
    for (; i < n; ++i) acc = __dadd_rn(acc, __dmul_rn(u[i], v[i]));
    out[lane] = acc;
}

__global__ void finish_kernel(const double* partial, int nparts, double* out, int nout) {
    __shared__ double sh[64];
    double s0 = 0.0, s1 = 0.0;
    for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
        s0 += partial[2 * k];
        s1 += partial[2 * k + 1];
    }
    block_reduce2(s0, s1, sh);
    if (threadIdx.x == 0) {
        out[0] = s0;
        if (nout > 1) out[1] = s1;
    }
}

__global__ void update_p_kernel_dev(const double* __restrict__ z, double* __restrict__ p,
                                    double beta, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = __dadd_rn(z[i], __dmul_rn(beta, p[i]));
}

// ---- staging of host pointers ----
struct Context {
    std::mutex mu;
    cudaStream_t stream = nullptr;
    std::vector<std::pair<void*, size_t>> bufs;  // slot -> device buffer
    double* partial = nullptr;
    bool ready = false;
};
Context& ctx() {
    static Context c;
    return c;
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(XPLUS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void ensure_ready(Context& c) {
    if (c.ready) return;
    check(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaMalloc(&c.partial, sizeof(double) * 2 * kMaxBlocks), "cudaMalloc");
    c.ready = true;
}

bool device_accessible(const void* p, const void** dev) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) {
        *dev = p;
        return true;
    }
    if (attr.type == cudaMemoryTypeHost && attr.devicePointer) {
        *dev = attr.devicePointer;
        return true;
    }
    return false;
}

}  // namespace

void require_device_memory(const void* p, int device, const char* what) {
    cudaPointerAttributes attr;
    const cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();  // this call's own error
        throw Error(XPLUS_ERR_ARG, std::string(what) + ": not a pointer CUDA knows (" + cudaGetErrorString(e) + ")");
    }
    if (attr.type == cudaMemoryTypeManaged) return;
    if (attr.type != cudaMemoryTypeDevice)
        throw Error(XPLUS_ERR_ARG, std::string(what) + ": host memory; this entry point takes device memory of GPU " +
                                       std::to_string(device));
    if (attr.device != device)
        throw Error(XPLUS_ERR_ARG, std::string(what) + ": memory of GPU " + std::to_string(attr.device) +
                                       ", not of GPU " + std::to_string(device));
}

void require_no_pending_cuda_error(const char* entry) {
    const cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess)
        throw Error(XPLUS_ERR_CUDA, std::string(entry) + ": an earlier CUDA error is pending on this thread (" +
                                        cudaGetErrorString(e) + "); nothing was launched");
}

namespace {

// One argument of a call: device view of a caller pointer, copied in/out when staged.
struct Arg {
    void* host = nullptr;
    void* dev = nullptr;
    size_t bytes = 0;
    bool staged = false, out = false;
};

void* slot_buffer(Context& c, size_t slot, size_t bytes) {
    if (c.bufs.size() <= slot) c.bufs.resize(slot + 1, {nullptr, 0});
    auto& b = c.bufs[slot];
    if (b.second < bytes) {
        if (b.first) cudaFree(b.first);
        b.first = nullptr;
        b.second = 0;
        check(cudaMalloc(&b.first, bytes < 256 ? 256 : bytes), "cudaMalloc");
        b.second = bytes < 256 ? 256 : bytes;
    }
    return b.first;
}

Arg bind(Context& c, size_t slot, const void* p, size_t bytes, bool in, bool out) {
    Arg a;
    a.host = const_cast<void*>(p);
    a.bytes = bytes;
    a.out = out;
    const void* d = nullptr;
    if (device_accessible(p, &d)) {
        a.dev = const_cast<void*>(d);
        return a;
    }
    a.staged = true;
    a.dev = slot_buffer(c, slot, bytes);
    if (in && bytes) check(cudaMemcpyAsync(a.dev, p, bytes, cudaMemcpyHostToDevice, c.stream), "H2D");
    return a;
}

void unbind(Context& c, const Arg& a) {
    if (a.staged && a.out && a.bytes)
        check(cudaMemcpyAsync(a.host, a.dev, a.bytes, cudaMemcpyDeviceToHost, c.stream), "D2H");
}

int blocks_for(int n) {
    int b = (n + kThreads - 1) / kThreads;
    return b < 1 ? 1 : (b > kMaxBlocks ? kMaxBlocks : b);
}

int nnz_of(Context& c, const int* row_ptr, int n) {
    const void* d = nullptr;
    int nnz = 0;
    if (device_accessible(row_ptr + n, &d))
        check(cudaMemcpyAsync(&nnz, d, sizeof(int), cudaMemcpyDeviceToHost, c.stream), "D2H");
    else
        nnz = row_ptr[n];
    check(cudaStreamSynchronize(c.stream), "sync");
    if (nnz < 0) throw Error(XPLUS_ERR_DATA, "row_ptr[n] must equal nnz");
    return nnz;
}

void run_spmv(const int* row_ptr, const int* col_idx, const double* values, const double* x,
              double* y, int n) {
    require_no_pending_cuda_error("spmv_csr_kernel");
    Context& c = ctx();
    std::lock_guard<std::mutex> g(c.mu);
    ensure_ready(c);
    const int nnz = nnz_of(c, row_ptr, n);
    Arg a0 = bind(c, 0, row_ptr, sizeof(int) * (static_cast<size_t>(n) + 1), true, false);
    Arg a1 = bind(c, 1, col_idx, sizeof(int) * static_cast<size_t>(nnz), true, false);
    Arg a2 = bind(c, 2, values, sizeof(double) * static_cast<size_t>(nnz), true, false);
    Arg a3 = bind(c, 3, x, sizeof(double) * static_cast<size_t>(n), true, false);
    Arg a4 = bind(c, 4, y, sizeof(double) * static_cast<size_t>(n), false, true);
    csr_spmv_f64_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, c.stream>>>(
        static_cast<const int*>(a0.dev), static_cast<const int*>(a1.dev),
        static_cast<const double*>(a2.dev), static_cast<const double*>(a3.dev),
        static_cast<double*>(a4.dev), n);
    check(cudaGetLastError(), "spmv launch");
    unbind(c, a4);
    check(cudaStreamSynchronize(c.stream), "sync");
}

// ---- scratch of the no-allocation update_xrz variant ----
// One FP64 pair (r.z, r.r) per block of the reduction, compiled into the library: every
// device that loads the library holds these 16 KiB until the process exits.
constexpr int kNoallocBlocks = 1024;
static __device__ __align__(256) double g_noalloc_partial[2 * kNoallocBlocks];
static_assert(kNoallocBlocks >= kMaxBlocks, "blocks_for() may use up to kMaxBlocks blocks");

// The current context, through the driver entry point (the library links only the runtime).
CUcontext current_context() {
    using Fn = CUresult (*)(CUcontext*);
    static Fn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            f = nullptr;
        }
        return reinterpret_cast<Fn>(f);
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) throw Error(XPLUS_ERR_CUDA, "cuCtxGetCurrent is not available");
    return c;
}

// Device address of g_noalloc_partial in the current context.  In host code the symbol is
// only a host-side stand-in, so the kernels get this address.  It is looked up again whenever
// the device's context changed (after cudaDeviceReset the old address is stale).
double* noalloc_scratch() {
    static std::mutex mu;
    static CUcontext ctx_of[64] = {};
    static double* addr[64] = {};
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) throw Error(XPLUS_ERR_ARG, "device ordinal out of range");
    const CUcontext cur = current_context();
    std::lock_guard<std::mutex> g(mu);
    if (!addr[dev] || ctx_of[dev] != cur) {
        void* p = nullptr;
        check(cudaGetSymbolAddress(&p, g_noalloc_partial), "cudaGetSymbolAddress");
        addr[dev] = static_cast<double*>(p);
        ctx_of[dev] = cur;
    }
    return addr[dev];
}

// The dot products of a call: summed in the reference's order from the vectors (a.b, and
// a.a with nout == 2: r.z and r.r) when n <= kSeqMaxN, else the tree over the element-wise
// kernel's block partials.
void finish_dots(const double* partial, int blocks, const double* a, const double* b, int n, double* out, int nout,
                 cudaStream_t st) {
    if (n <= kSeqMaxN)
        seq_dot_kernel<<<1, 32, 0, st>>>(a, b, a, a, n, out, nout);
    else
        finish_kernel<<<1, kThreads, 0, st>>>(partial, blocks, out, nout);
    check(cudaGetLastError(), "dot finish launch");
}

template <typename F>
void abi_call(F&& f) {
    const int rc = guarded(f);
    (void)rc;  // void ABI: the error text stays in xplus_last_error_string()
}

}  // namespace
}  // namespace xplus

using namespace xplus;

extern "C" {

void spmv_csr_kernel(const int* row_ptr, const int* col_idx, const double* values, const double* x,
                     double* y, int n) {
    if (n <= 0) return;
    abi_call([&] { run_spmv(row_ptr, col_idx, values, x, y, n); });
}

void spmv_blocked_kernel(const int* row_ptr, const int* col_idx, const double* values,
                         const double* x, double* y, int n) {
    // The reference's blocked entry degenerates to the CSR body
    // (archived/kernels/cg_kernels.cpp:58-71); so does this one.
    if (n <= 0) return;
    abi_call([&] { run_spmv(row_ptr, col_idx, values, x, y, n); });
}

void init_pcg_kernel(const double* b, const double* ax, const double* m_inv, double* r, double* z,
                     double* p, double* metrics, int n) {
    if (n < 0) return;
    abi_call([&] {
        require_no_pending_cuda_error("init_pcg_kernel");
        Context& c = ctx();
        std::lock_guard<std::mutex> g(c.mu);
        ensure_ready(c);
        const size_t vb = sizeof(double) * static_cast<size_t>(n);
        Arg ab = bind(c, 0, b, vb, true, false), aax = bind(c, 1, ax, vb, true, false);
        Arg am = bind(c, 2, m_inv, vb, true, false), ar = bind(c, 3, r, vb, false, true);
        Arg az = bind(c, 4, z, vb, false, true), ap = bind(c, 5, p, vb, false, true);
        Arg amet = bind(c, 6, metrics, 2 * sizeof(double), false, true);
        const int blocks = blocks_for(n);
        vec_kernel<<<blocks, kThreads, 0, c.stream>>>(
            1, n, 0.0, nullptr, nullptr, static_cast<double*>(ar.dev), static_cast<const double*>(aax.dev),
            static_cast<const double*>(am.dev), static_cast<double*>(az.dev), static_cast<double*>(ap.dev),
            static_cast<const double*>(ab.dev), c.partial);
        check(cudaGetLastError(), "init_pcg launch");
        finish_dots(c.partial, blocks, static_cast<const double*>(ar.dev), static_cast<const double*>(az.dev), n,
                    static_cast<double*>(amet.dev), 2, c.stream);
        unbind(c, ar); unbind(c, az); unbind(c, ap); unbind(c, amet);
        check(cudaStreamSynchronize(c.stream), "sync");
    });
}

void dot_kernel(const double* a, const double* b, double* out, int n) {
    if (n < 0) return;
    abi_call([&] {
        require_no_pending_cuda_error("dot_kernel");
        Context& c = ctx();
        std::lock_guard<std::mutex> g(c.mu);
        ensure_ready(c);
        const size_t vb = sizeof(double) * static_cast<size_t>(n);
        Arg aa = bind(c, 0, a, vb, true, false), ab = bind(c, 1, b, vb, true, false);
        Arg ao = bind(c, 2, out, sizeof(double), false, true);
        const int blocks = blocks_for(n);
        if (n > kSeqMaxN) {
            vec_kernel<<<blocks, kThreads, 0, c.stream>>>(
                0, n, 0.0, static_cast<double*>(aa.dev), static_cast<const double*>(ab.dev), nullptr,
                nullptr, nullptr, nullptr, nullptr, nullptr, c.partial);
            check(cudaGetLastError(), "dot launch");
        }
        finish_dots(c.partial, blocks, static_cast<const double*>(aa.dev), static_cast<const double*>(ab.dev), n,
                    static_cast<double*>(ao.dev), 1, c.stream);
        unbind(c, ao);
        check(cudaStreamSynchronize(c.stream), "sync");
    });
}

void update_xrz_kernel(double* x, const double* p, double* r, const double* ap,
                       const double* m_inv, double* z, double* metrics, double alpha, int n) {
    if (n < 0) return;
    abi_call([&] {
        require_no_pending_cuda_error("update_xrz_kernel");
        Context& c = ctx();
        std::lock_guard<std::mutex> g(c.mu);
        ensure_ready(c);
        const size_t vb = sizeof(double) * static_cast<size_t>(n);
        Arg ax = bind(c, 0, x, vb, true, true), ap_ = bind(c, 1, p, vb, true, false);
        Arg ar = bind(c, 2, r, vb, true, true), aap = bind(c, 3, ap, vb, true, false);
        Arg am = bind(c, 4, m_inv, vb, true, false), az = bind(c, 5, z, vb, false, true);
        Arg amet = bind(c, 6, metrics, 2 * sizeof(double), false, true);
        const int blocks = blocks_for(n);
        vec_kernel<<<blocks, kThreads, 0, c.stream>>>(
            2, n, alpha, static_cast<double*>(ax.dev), static_cast<const double*>(ap_.dev),
            static_cast<double*>(ar.dev), static_cast<const double*>(aap.dev),
            static_cast<const double*>(am.dev), static_cast<double*>(az.dev), nullptr, nullptr, c.partial);
        check(cudaGetLastError(), "update_xrz launch");
        finish_dots(c.partial, blocks, static_cast<const double*>(ar.dev), static_cast<const double*>(az.dev), n,
                    static_cast<double*>(amet.dev), 2, c.stream);
        unbind(c, ax); unbind(c, ar); unbind(c, az); unbind(c, amet);
        check(cudaStreamSynchronize(c.stream), "sync");
    });
}

int xplus_update_xrz_noalloc(double* x, const double* p, double* r, const double* ap,
                             const double* m_inv, double* z, double* metrics, double alpha, int n,
                             void* stream) {
    return guarded([&] {
        require(n >= 0 && n <= XPLUS_NOALLOC_MAX_N, XPLUS_ERR_ARG,
                "n exceeds the no-allocation limit of " + std::to_string(XPLUS_NOALLOC_MAX_N) + " rows");
        require(metrics != nullptr && (n == 0 || (x && p && r && ap && m_inv && z)), XPLUS_ERR_ARG,
                "null argument");
        require_no_pending_cuda_error("xplus_update_xrz_noalloc");
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        // every pointer must be memory the kernels can address on this device: a host array
        // (which update_xrz_kernel would stage) is an argument error here, not a GPU fault
        require_device_memory(metrics, dev, "metrics");
        if (n > 0) {
            require_device_memory(x, dev, "x");
            require_device_memory(p, dev, "p");
            require_device_memory(r, dev, "r");
            require_device_memory(ap, dev, "ap");
            require_device_memory(m_inv, dev, "m_inv");
            require_device_memory(z, dev, "z");
        }
        double* scratch = noalloc_scratch();
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        // at most kNoallocBlocks blocks, so the partials fit the fixed scratch
        const int blocks = blocks_for(n);
        vec_kernel<<<blocks, kThreads, 0, st>>>(2, n, alpha, x, p, r, ap, m_inv, z, nullptr, nullptr, scratch);
        check(cudaGetLastError(), "update_xrz_noalloc launch");
        finish_dots(scratch, blocks, r, z, n, metrics, 2, st);
    });
}

void update_p_kernel(const double* z, double* p, double beta, int n) {
    if (n <= 0) return;
    abi_call([&] {
        require_no_pending_cuda_error("update_p_kernel");
        Context& c = ctx();
        std::lock_guard<std::mutex> g(c.mu);
        ensure_ready(c);
        const size_t vb = sizeof(double) * static_cast<size_t>(n);
        Arg az = bind(c, 0, z, vb, true, false), ap = bind(c, 1, p, vb, true, true);
        update_p_kernel_dev<<<(n + kThreads - 1) / kThreads, kThreads, 0, c.stream>>>(
            static_cast<const double*>(az.dev), static_cast<double*>(ap.dev), beta, n);
        check(cudaGetLastError(), "update_p launch");
        unbind(c, ap);
        check(cudaStreamSynchronize(c.stream), "sync");
    });
}

}  // extern "C"
