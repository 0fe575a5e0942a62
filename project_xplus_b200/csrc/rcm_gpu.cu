// rcm_gpu.cu -- reverse Cuthill-McKee and the symmetric permutation on the GPU, bit-identical
// to rcm_order / permute_symmetric (rcm.cpp), which the oracle restates (sell_rcm_oracle.py).
//
// The host order is sequential: components by lowest unplaced index; start node the component's
// minimum-(degree, index) node refined by the George-Liu pseudo-peripheral search; Cuthill-McKee
// BFS appending each node's unvisited neighbours sorted by (degree, index); reversed.
// The GPU computes the same order level by level.  When the nodes of level L sit at queue
// positions [lb, le), the host gives each node u of level L + 1 to the first node of level L
// (lowest position) adjacent to it, and lists level L + 1 parent by parent, each parent's
// children by (degree, index).  So one persistent cooperative launch per BFS does, per level:
//   claim   every unvisited neighbour u of frontier node p: claim[u] = min(claim[u], p)
//   count   children of p = #{u in adj(p) : claim[u] == p}
//   write   exclusive scan of the counts in frontier order gives every parent its offset;
//           it writes its children sorted by (degree, index) there
// with a bounded grid barrier between the steps.  The pseudo-peripheral search uses the same
// BFS (only its level count and last level matter there).  A node with more than kMaxChildren
// claimed children, or a row with a repeated column, sends the whole ordering to the host
// function instead (same result, host speed).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "common.hpp"
#include "device_common.cuh"

namespace xplus {

void rcm_order(int n, const int* row_ptr, const int* col_idx, int* perm);  // rcm.cpp

namespace {

using namespace dev;

constexpr int kFree = 0x7F7F7F7F;  // claim of a node no frontier node has claimed (memset 0x7F)
constexpr int kMaxChildren = 64;
constexpr int kBfsThreads = 512;

struct BfsArgs {
    const int* rp;
    const int* ci;
    const int* deg;
    const int* placed;  // 1: ordered by an earlier component
    int* vis;           // == stamp: reached by this BFS
    int* claim;         // kFree, or the lowest frontier position that reached the node
    int* order;         // BFS order
    int* cnt;           // children of each frontier node (frontier-relative)
    int* block_sum;     // per CTA
    int* out;           // {visited, levels, first position of the last level, too many children}
    int stamp;
    int root;
    unsigned* bar;
    int* err;
    long long timeout_ns;
};

__device__ __forceinline__ bool before(const int* deg, int a, int b) {
    const int da = deg[a], db = deg[b];
    return da < db || (da == db && a < b);
}

__global__ void __launch_bounds__(kBfsThreads) k_bfs(BfsArgs a) {
    __shared__ int s_flag;
    __shared__ int s_scan[kBfsThreads];
    __shared__ int s_run;
    GridBarrier bar{a.bar, a.err, a.timeout_ns, 0u, -1};
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.order[0] = a.root;
        a.vis[a.root] = a.stamp;
    }
    if (!bar.sync(&s_flag)) return;
    int lb = 0, le = 1, levels = 0, last_b = 0;
    const int gthreads = gridDim.x * blockDim.x;
    while (le > lb) {
        ++levels;
        last_b = lb;
        const int fs = le - lb;
        // claim
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < fs; q += gthreads) {
            const int p = lb + q, x = a.order[p];
            for (int k = a.rp[x]; k < a.rp[x + 1]; ++k) {
                const int u = a.ci[k];
                if (u != x && !a.placed[u] && a.vis[u] != a.stamp) atomicMin(&a.claim[u], p);
            }
        }
        if (!bar.sync(&s_flag)) return;
        // count, over contiguous frontier chunks per CTA
        const int chunk = (fs + gridDim.x - 1) / gridDim.x;
        const int c0 = min(fs, static_cast<int>(blockIdx.x) * chunk), c1 = min(fs, c0 + chunk);
        int mine = 0;
        for (int q = c0 + threadIdx.x; q < c1; q += blockDim.x) {
            const int p = lb + q, x = a.order[p];
            int c = 0;
            for (int k = a.rp[x]; k < a.rp[x + 1]; ++k) {
                const int u = a.ci[k];
                c += (u != x && a.claim[u] == p);
            }
            if (c > kMaxChildren) atomicExch(a.out + 3, 1);
            a.cnt[q] = c;
            mine += c;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
        if ((threadIdx.x & 31) == 0) s_scan[threadIdx.x >> 5] = mine;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += s_scan[w];
            a.block_sum[blockIdx.x] = t;
        }
        if (!bar.sync(&s_flag)) return;
        if (ld_volatile_int(a.out + 3) != 0) return;  // every block sees it: the host takes over
        // offsets: blocks before this one, then a running scan of this block's chunk
        if (threadIdx.x == 0) {
            int base = 0;
            for (int b = 0; b < static_cast<int>(blockIdx.x); ++b) base += a.block_sum[b];
            s_run = base;
        }
        __syncthreads();
        int total = 0;
        for (int b = 0; b < static_cast<int>(gridDim.x); ++b) total += a.block_sum[b];
        for (int t0 = c0; t0 < c1; t0 += blockDim.x) {
            const int q = t0 + threadIdx.x;
            const int c = q < c1 ? a.cnt[q] : 0;
            s_scan[threadIdx.x] = c;
            __syncthreads();
            for (int o = 1; o < static_cast<int>(blockDim.x); o <<= 1) {
                const int v = threadIdx.x >= static_cast<unsigned>(o) ? s_scan[threadIdx.x - o] : 0;
                __syncthreads();
                s_scan[threadIdx.x] += v;
                __syncthreads();
            }
            const int off = s_run + s_scan[threadIdx.x] - c;
            if (q < c1 && c > 0) {
                const int p = lb + q, x = a.order[p];
                int kids[kMaxChildren];
                int m = 0;
                for (int k = a.rp[x]; k < a.rp[x + 1]; ++k) {
                    const int u = a.ci[k];
                    if (u != x && a.claim[u] == p) {
                        int j = m++;  // insertion by (degree, index)
                        while (j > 0 && before(a.deg, u, kids[j - 1])) {
                            kids[j] = kids[j - 1];
                            --j;
                        }
                        kids[j] = u;
                    }
                }
                for (int j = 0; j < m; ++j) {
                    a.order[le + off + j] = kids[j];
                    a.vis[kids[j]] = a.stamp;
                    a.claim[kids[j]] = kFree;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) s_run += s_scan[blockDim.x - 1];
            __syncthreads();
        }
        if (!bar.sync(&s_flag)) return;
        lb = le;
        le += total;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = le;
        a.out[1] = levels;
        a.out[2] = last_b;
    }
}

__global__ void k_degree(const int* __restrict__ rp, const int* __restrict__ ci, int n, int* __restrict__ deg,
                         int* __restrict__ dup) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int d = 0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const int u = ci[k];
        if (u == i) continue;
        ++d;
        for (int q = rp[i]; q < k; ++q)
            if (ci[q] == u) atomicOr(dup, 1);
    }
    deg[i] = d;
}

// minimum (degree, index) over order[b, e) into *best (the caller sets it to ULLONG_MAX)
__global__ void k_argmin(const int* __restrict__ order, int b, int e, const int* __restrict__ deg,
                         unsigned long long* __restrict__ best) {
    const int q = b + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= e) return;
    const int v = order[q];
    atomicMin(best, (static_cast<unsigned long long>(deg[v]) << 32) | static_cast<unsigned>(v));
}

__global__ void k_place(const int* __restrict__ order, int count, int* __restrict__ placed, int* __restrict__ result,
                        int pos) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    placed[order[q]] = 1;
    result[pos + q] = order[q];
}

__global__ void k_first_unplaced(const int* __restrict__ placed, int from, int n, int* __restrict__ first) {
    const int i = from + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !placed[i]) atomicMin(first, i);
}

__global__ void k_reverse(const int* __restrict__ result, int n, int* __restrict__ perm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) perm[i] = result[n - 1 - i];
}

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

}  // namespace

// Reverse Cuthill-McKee of the device CSR (d_rp, d_ci; n rows) into d_perm (perm[new] = old).
// Returns false, with nothing written, when the graph needs the host ordering (a node with more
// than kMaxChildren children claimed at once, or a repeated column); the caller runs it then.
bool rcm_device(int n, const int* d_rp, const int* d_ci, int* d_perm, cudaStream_t st) {
    Tmp tmp;
    int* deg = tmp.get<int>(static_cast<size_t>(n));
    int* placed = tmp.get<int>(static_cast<size_t>(n));
    int* vis = tmp.get<int>(static_cast<size_t>(n));
    int* claim = tmp.get<int>(static_cast<size_t>(n));
    int* order = tmp.get<int>(static_cast<size_t>(n));
    int* result = tmp.get<int>(static_cast<size_t>(n));
    int* cnt = tmp.get<int>(static_cast<size_t>(n));
    int* small = tmp.get<int>(8);  // {dup, first unplaced}
    unsigned long long* best = tmp.get<unsigned long long>(1);
    int dev = 0, sms = 0, per_sm = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attr");
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bfs, kBfsThreads, 0), "occupancy");
    require(per_sm > 0, XPLUS_ERR_CUDA, "rcm: the BFS kernel cannot be resident");
    const int grid = sms;  // one block per SM, co-resident
    int* block_sum = tmp.get<int>(static_cast<size_t>(grid));
    int* out = tmp.get<int>(4);
    unsigned* bar = tmp.get<unsigned>(1);
    int* err = tmp.get<int>(1);
    const int tb = 256;
    ck(cudaMemsetAsync(small, 0, 8 * sizeof(int), st), "memset");
    k_degree<<<(n + tb - 1) / tb, tb, 0, st>>>(d_rp, d_ci, n, deg, small);
    ck(cudaGetLastError(), "rcm degree");
    int h_small[2] = {0, 0};
    ck(cudaMemcpyAsync(h_small, small, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    if (h_small[0]) return false;
    ck(cudaMemsetAsync(placed, 0, static_cast<size_t>(n) * sizeof(int), st), "memset");
    ck(cudaMemsetAsync(vis, 0, static_cast<size_t>(n) * sizeof(int), st), "memset");
    ck(cudaMemsetAsync(claim, 0x7F, static_cast<size_t>(n) * sizeof(int), st), "memset");
    int stamp = 0;
    // one BFS from root over the unplaced nodes: {visited, levels, last level begin}
    auto bfs = [&](int root, int (&res)[3]) -> bool {
        ++stamp;
        BfsArgs a{};
        a.rp = d_rp;
        a.ci = d_ci;
        a.deg = deg;
        a.placed = placed;
        a.vis = vis;
        a.claim = claim;
        a.order = order;
        a.cnt = cnt;
        a.block_sum = block_sum;
        a.out = out;
        a.stamp = stamp;
        a.root = root;
        a.bar = bar;
        a.err = err;
        a.timeout_ns = 2000000000LL;
        ck(cudaMemsetAsync(out, 0, 4 * sizeof(int), st), "memset");
        ck(cudaMemsetAsync(bar, 0, sizeof(unsigned), st), "memset");
        ck(cudaMemsetAsync(err, 0, sizeof(int), st), "memset");
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(kBfsThreads);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        ck(cudaLaunchKernelEx(&cfg, k_bfs, a), "rcm BFS launch");
        int h_out[4], h_err = 0;
        ck(cudaMemcpyAsync(h_out, out, sizeof(h_out), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaStreamSynchronize(st), "sync");
        require(h_err == 0, XPLUS_ERR_CUDA, "rcm: a grid barrier timed out");
        if (h_out[3]) return false;
        res[0] = h_out[0];
        res[1] = h_out[1];
        res[2] = h_out[2];
        return true;
    };
    auto argmin = [&](int b, int e) {
        const unsigned long long init = ~0ull;
        ck(cudaMemcpyAsync(best, &init, sizeof(init), cudaMemcpyHostToDevice, st), "H2D");
        k_argmin<<<(e - b + tb - 1) / tb, tb, 0, st>>>(order, b, e, deg, best);
        ck(cudaGetLastError(), "rcm argmin");
        unsigned long long h = 0;
        ck(cudaMemcpyAsync(&h, best, sizeof(h), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaStreamSynchronize(st), "sync");
        return static_cast<int>(h & 0xFFFFFFFFull);
    };
    int pos = 0, seed = 0;
    while (pos < n) {
        // the lowest unplaced node
        const int big = INT_MAX;
        ck(cudaMemcpyAsync(small + 1, &big, sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
        k_first_unplaced<<<(n - seed + tb - 1) / tb, tb, 0, st>>>(placed, seed, n, small + 1);
        ck(cudaGetLastError(), "rcm seed");
        ck(cudaMemcpyAsync(&seed, small + 1, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaStreamSynchronize(st), "sync");
        int r[3];
        if (!bfs(seed, r)) return false;
        int v = argmin(0, r[0]);  // the component's minimum-(degree, index) node
        if (!bfs(v, r)) return false;
        int ecc = r[1], last_b = r[2], last_e = r[0];
        while (true) {  // George-Liu pseudo-peripheral node
            const int u = argmin(last_b, last_e);
            int r2[3];
            if (!bfs(u, r2)) return false;
            if (r2[1] > ecc) {
                v = u;
                ecc = r2[1];
                last_b = r2[2];
                last_e = r2[0];
            } else {
                break;
            }
        }
        if (!bfs(v, r)) return false;  // Cuthill-McKee from v
        k_place<<<(r[0] + tb - 1) / tb, tb, 0, st>>>(order, r[0], placed, result, pos);
        ck(cudaGetLastError(), "rcm place");
        pos += r[0];
    }
    k_reverse<<<(n + tb - 1) / tb, tb, 0, st>>>(result, n, d_perm);
    ck(cudaGetLastError(), "rcm reverse");
    ck(cudaStreamSynchronize(st), "sync");
    return true;
}

namespace {

__global__ void k_inverse_perm(const int* __restrict__ perm, int n, int* __restrict__ iperm, int* __restrict__ bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = perm[i];
    if (p < 0 || p >= n || atomicExch(&iperm[p], i) != -1) atomicOr(bad, 1);
}

__global__ void k_perm_lengths(const int* __restrict__ rp, const int* __restrict__ perm, int n, int* __restrict__ len) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) len[i] = rp[perm[i] + 1] - rp[perm[i]];
}

// out[0] = 0, out[i + 1] = out[i] + len[i]: one CTA, each thread a contiguous chunk
__global__ void __launch_bounds__(1024) k_scan_int(const int* __restrict__ len, int n, int* __restrict__ out) {
    __shared__ int s_sum[1024];
    const int t = threadIdx.x;
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int b = min(n, t * per), e = min(n, b + per);
    int acc = 0;
    for (int i = b; i < e; ++i) acc += len[i];
    s_sum[t] = acc;
    __syncthreads();
    for (int o = 1; o < static_cast<int>(blockDim.x); o <<= 1) {
        const int v = t >= o ? s_sum[t - o] : 0;
        __syncthreads();
        s_sum[t] += v;
        __syncthreads();
    }
    int run = t > 0 ? s_sum[t - 1] : 0;
    if (t == 0) out[0] = 0;
    for (int i = b; i < e; ++i) {
        run += len[i];
        out[i + 1] = run;
    }
}

// new row i = old row perm[i], columns renumbered by iperm and stably sorted ascending (the
// host's stable_sort of (column, value) pairs)
__global__ void k_perm_fill(const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                            const int* __restrict__ perm, const int* __restrict__ iperm, const int* __restrict__ orp,
                            int n, int* __restrict__ oci, double* __restrict__ ov) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int old = perm[i];
    const int o0 = orp[i];
    int m = 0;
    for (int k = rp[old]; k < rp[old + 1]; ++k, ++m) {
        const int c = iperm[ci[k]];
        const double x = v[k];
        int j = o0 + m;  // insertion: shift only strictly greater columns (stable)
        while (j > o0 && oci[j - 1] > c) {
            oci[j] = oci[j - 1];
            ov[j] = ov[j - 1];
            --j;
        }
        oci[j] = c;
        ov[j] = x;
    }
}

}  // namespace

void permute_symmetric_device(int n, const int* d_rp, const int* d_ci, const double* d_v, const int* d_perm,
                              int* d_orp, int* d_oci, double* d_ov, cudaStream_t st) {
    Tmp tmp;
    int* iperm = tmp.get<int>(static_cast<size_t>(n));
    int* len = tmp.get<int>(static_cast<size_t>(n));
    int* bad = tmp.get<int>(1);
    const int tb = 256;
    ck(cudaMemsetAsync(iperm, 0xFF, static_cast<size_t>(n) * sizeof(int), st), "memset");
    ck(cudaMemsetAsync(bad, 0, sizeof(int), st), "memset");
    k_inverse_perm<<<(n + tb - 1) / tb, tb, 0, st>>>(d_perm, n, iperm, bad);
    ck(cudaGetLastError(), "inverse permutation");
    int h_bad = 0;
    ck(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    require(h_bad == 0, XPLUS_ERR_ARG, "perm is not a permutation");
    k_perm_lengths<<<(n + tb - 1) / tb, tb, 0, st>>>(d_rp, d_perm, n, len);
    k_scan_int<<<1, 1024, 0, st>>>(len, n, d_orp);
    k_perm_fill<<<(n + tb - 1) / tb, tb, 0, st>>>(d_rp, d_ci, d_v, d_perm, iperm, d_orp, n, d_oci, d_ov);
    ck(cudaGetLastError(), "permute");
    ck(cudaStreamSynchronize(st), "sync");
}

}  // namespace xplus

using namespace xplus;

namespace {

// the device CSR's structure, checked before anything is indexed (XPLUS_ERR_DATA)
void check_device_csr(int n, const int* d_rp, const int* d_ci, cudaStream_t st) {
    require(n > 0 && d_rp && d_ci, XPLUS_ERR_ARG, "invalid argument");
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    require_device_memory(d_rp, dev, "d_row_ptr");
    require_device_memory(d_ci, dev, "d_col_idx");
    std::vector<int> rp(static_cast<size_t>(n) + 1);
    ck(cudaMemcpyAsync(rp.data(), d_rp, rp.size() * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    require(rp[0] == 0, XPLUS_ERR_DATA, "row_ptr[0] must be 0");
    for (int i = 0; i < n; ++i) require(rp[static_cast<size_t>(i)] <= rp[static_cast<size_t>(i) + 1], XPLUS_ERR_DATA, "row_ptr must be nondecreasing");
    std::vector<int> ci(static_cast<size_t>(rp[static_cast<size_t>(n)]));
    if (!ci.empty()) {
        ck(cudaMemcpyAsync(ci.data(), d_ci, ci.size() * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaStreamSynchronize(st), "sync");
        for (int c : ci) require(c >= 0 && c < n, XPLUS_ERR_DATA, "col_idx out of range");
    }
}

}  // namespace

extern "C" {

int xplus_rcm_device(int n, const int* d_row_ptr, const int* d_col_idx, int* d_perm, int* used_gpu, void* stream) {
    return guarded([&] {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        check_device_csr(n, d_row_ptr, d_col_idx, st);
        int dev = 0;
        ck(cudaGetDevice(&dev), "cudaGetDevice");
        require_device_memory(d_perm, dev, "d_perm");
        const bool on_gpu = rcm_device(n, d_row_ptr, d_col_idx, d_perm, st);
        if (!on_gpu) {
            // the host ordering (same result): a node with many children at once, or a repeated column
            std::vector<int> rp(static_cast<size_t>(n) + 1), perm(static_cast<size_t>(n));
            ck(cudaMemcpy(rp.data(), d_row_ptr, rp.size() * sizeof(int), cudaMemcpyDeviceToHost), "D2H");
            std::vector<int> ci(static_cast<size_t>(rp[static_cast<size_t>(n)]));
            ck(cudaMemcpy(ci.data(), d_col_idx, ci.size() * sizeof(int), cudaMemcpyDeviceToHost), "D2H");
            rcm_order(n, rp.data(), ci.data(), perm.data());
            ck(cudaMemcpy(d_perm, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice), "H2D");
        }
        if (used_gpu) *used_gpu = on_gpu ? 1 : 0;
    });
}

int xplus_permute_symmetric_device(int n, const int* d_row_ptr, const int* d_col_idx, const double* d_values,
                                   const int* d_perm, int* d_out_row_ptr, int* d_out_col_idx, double* d_out_values,
                                   void* stream) {
    return guarded([&] {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        check_device_csr(n, d_row_ptr, d_col_idx, st);
        int dev = 0;
        ck(cudaGetDevice(&dev), "cudaGetDevice");
        for (const void* p : {static_cast<const void*>(d_values), static_cast<const void*>(d_perm),
                              static_cast<const void*>(d_out_row_ptr), static_cast<const void*>(d_out_col_idx),
                              static_cast<const void*>(d_out_values)})
            require_device_memory(p, dev, "device array");
        permute_symmetric_device(n, d_row_ptr, d_col_idx, d_values, d_perm, d_out_row_ptr, d_out_col_idx, d_out_values,
                                 st);
    });
}

}  // extern "C"
