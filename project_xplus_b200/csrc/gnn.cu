// gnn.cu -- the learned preconditioner M^-1 = G^T G: a 3-layer message-passing network over
// A's graph predicts G on A's lower pattern; forward, probe loss, backward and Adam are the
// kernels below, all hand-written (FP32 arithmetic, parameters rounded to BF16 for the forward).
//
// Network (H = 32), in the row order of the system:
//   x_i = [log a_ii - mean log a_kk, sum_j |a_ij| / a_ii - 1],  e_ij = a_ij / sqrt(a_ii a_jj)
//   h = relu(W0 x + b0)
//   3 x: s_i = Wa h_i + ba + sum_{j<i} e_ij Wl h_j + sum_{j>i} e_ij Wu h_j ; h_i += relu(s_i)
//   lower edge (i, j<i): Ghat_ij = w . relu(P h_i + bp + Q h_j + c e_ij + c2 f_ij) + bw,
//     f_ij = sum_{m < i, m != j} e_jm e_mi: the two-step paths from j to i through i's other
//     lower neighbours (the coupling inside row i's pattern that the exact FSAI row solves)
//   diagonal:            Ghat_ii = exp(wd . h_i + bwd)
//   G = Ghat D^-1/2 (an untrained network with a zero output layer gives Jacobi)
// The node products W h (and D W in the backward pass) run on the tensor cores with the node
// activations rounded to BF16 (BF16 weights, FP32 accumulation); the rest is FP32.
// Losses: over K probes v ~ N(0, I), L = sum ||G A G^T v - v||^2 / (K n); or the row-normalized
// Kaporin loss L = (1/n) sum_i [log (G A G^T)_ii - 2 log Ghat_ii].
// Lower and upper neighbours have their own message weights because G is lower-triangular in
// the given order: what G_ij should be depends on which neighbours precede row i.
//
// Layouts: node arrays are [n][32] row-major (one warp per node, lane = feature, 128-byte
// rows); probe arrays are [n][K].  Weight-gradient sums over nodes or edges go through fixed
// per-block partials and a fixed-order final sum, so gradients are deterministic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "common.hpp"
#include "gnn.hpp"

namespace xplus {
namespace gnn {
namespace {

constexpr int H = kHidden;
constexpr int kRedBlocks = 256;  // blocks of every deterministic reduction (upper bound)

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void k_round_params(const float* __restrict__ master, float* __restrict__ wr, int P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P) wr[i] = __bfloat162float(__float2bfloat16_rn(master[i]));
}

// h0 = relu(W0 x + b0): thread per (node, feature)
__global__ void k_input(const float* __restrict__ x, const float* __restrict__ W0, const float* __restrict__ b0,
                        float* __restrict__ h0, int n) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<long long>(n) * H) return;
    const int i = static_cast<int>(t / H), f = static_cast<int>(t % H);
    const float v = fmaf(W0[2 * f], x[2 * i], fmaf(W0[2 * f + 1], x[2 * i + 1], b0[f]));
    h0[t] = fmaxf(v, 0.0f);
}

// ---- node products on the tensor cores ----
// A warp takes 16 nodes at a time: mma.sync m16n8k16 (BF16 operands, FP32 accumulation), the
// 16 x 32 node block as A (two k-steps of 16 features), a weight matrix as B, four n-tiles of
// 8 outputs.  Node activations are rounded to BF16 as they enter the product (the weights are
// BF16 already); sums, biases and everything outside these products stay FP32.
// Fragment layout of m16n8k16 (g = lane / 4, t = lane % 4):
//   A regs {A[g][2t..+1], A[g+8][2t..+1], A[g][2t+8..+9], A[g+8][2t+8..+9]}
//   B regs {B[2t..+1][g], B[2t+8..+9][g]},  C {C[g][2t..+1], C[g+8][2t..+1]}
constexpr int HP = H + 8;  // row stride (BF16) of the staged weights: conflict-free B loads

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float2 ld_row2(const float* src, int r, int n, int c) {
    return r < n ? *reinterpret_cast<const float2*>(src + static_cast<size_t>(r) * H + c) : make_float2(0.0f, 0.0f);
}

// A fragments of rows [r0, r0 + 16), features [16 s, 16 s + 16) of src ([n][H] FP32)
__device__ __forceinline__ void load_a(const float* __restrict__ src, int r0, int n, int s, int g, int t,
                                       uint32_t (&a)[4]) {
    const int c = 16 * s + 2 * t;
    const float2 x0 = ld_row2(src, r0 + g, n, c), x1 = ld_row2(src, r0 + g + 8, n, c);
    const float2 x2 = ld_row2(src, r0 + g, n, c + 8), x3 = ld_row2(src, r0 + g + 8, n, c + 8);
    a[0] = pack_bf16(x0.x, x0.y);
    a[1] = pack_bf16(x1.x, x1.y);
    a[2] = pack_bf16(x2.x, x2.y);
    a[3] = pack_bf16(x3.x, x3.y);
}

// acc[j] += A (16 x 16, k-step s) times B = staged[n][k] for the n-tile j (n = 8 j + g)
__device__ __forceinline__ void mma_row(float (&acc)[4][4], const uint32_t (&a)[4], const __nv_bfloat16* ws, int s,
                                        int g, int t) {
    const uint32_t* w32 = reinterpret_cast<const uint32_t*>(ws);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int base = ((8 * j + g) * HP + 16 * s + 2 * t) >> 1;
        mma_bf16(acc[j], a, w32[base], w32[base + 4]);
    }
}

// Up to three products Y_m = W_m h (+ b_m) per node; W_m [H][H] row-major (out, in) is B with
// B[k][n] = W_m[n][k], staged as Ws[n][k] (BF16).
struct Lin3 {
    const float* W[3];
    const float* b[3];
    float* Y[3];
    int count;
};

__global__ void __launch_bounds__(256) k_node_lin(const float* __restrict__ h, Lin3 L, int n) {
    __shared__ __align__(16) __nv_bfloat16 Ws[3][H * HP];
#pragma unroll
    for (int m = 0; m < 3; ++m)  // compile-time m: the parameter struct stays out of local memory
        if (m < L.count)
            for (int r = threadIdx.x; r < H * H; r += blockDim.x) Ws[m][(r / H) * HP + r % H] = __float2bfloat16_rn(L.W[m][r]);
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int warps = blockDim.x >> 5;
    for (int r0 = (blockIdx.x * warps + (threadIdx.x >> 5)) * 16; r0 < n; r0 += gridDim.x * warps * 16) {
        uint32_t a[2][4];
        load_a(h, r0, n, 0, g, t, a[0]);
        load_a(h, r0, n, 1, g, t, a[1]);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            if (m >= L.count) continue;
            float acc[4][4] = {};
            mma_row(acc, a[0], Ws[m], 0, g, t);
            mma_row(acc, a[1], Ws[m], 1, g, t);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = 8 * j + 2 * t;
                const float b0 = L.b[m] ? L.b[m][c] : 0.0f, b1 = L.b[m] ? L.b[m][c + 1] : 0.0f;
                if (r0 + g < n)
                    *reinterpret_cast<float2*>(L.Y[m] + static_cast<size_t>(r0 + g) * H + c) =
                        make_float2(acc[j][0] + b0, acc[j][1] + b1);
                if (r0 + g + 8 < n)
                    *reinterpret_cast<float2*>(L.Y[m] + static_cast<size_t>(r0 + g + 8) * H + c) =
                        make_float2(acc[j][2] + b0, acc[j][3] + b1);
            }
        }
    }
}

// Transposed products for the backward pass: dX = sum_m D_m W_m (+ dexp (x) wd), i.e. B with
// B[k][n] = W_m[k][n] (k = output feature, n = input feature), staged as Ws[n][k] (BF16).
// dX = accumulate ? dX + . : .
struct BackLin {
    const float* W[3];
    const float* D[3];
    int count;
    const float* dexp;  // optional per-node scalar times wd
    const float* wd;
    int accumulate;
};

__global__ void __launch_bounds__(256) k_node_backlin(BackLin B, float* __restrict__ dX, int n) {
    __shared__ __align__(16) __nv_bfloat16 Ws[3][H * HP];
#pragma unroll
    for (int m = 0; m < 3; ++m)
        if (m < B.count)
            for (int r = threadIdx.x; r < H * H; r += blockDim.x) Ws[m][(r % H) * HP + r / H] = __float2bfloat16_rn(B.W[m][r]);
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int warps = blockDim.x >> 5;
    for (int r0 = (blockIdx.x * warps + (threadIdx.x >> 5)) * 16; r0 < n; r0 += gridDim.x * warps * 16) {
        float acc[4][4] = {};
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            if (m >= B.count) continue;
            uint32_t a[4];
            load_a(B.D[m], r0, n, 0, g, t, a);
            mma_row(acc, a, Ws[m], 0, g, t);
            load_a(B.D[m], r0, n, 1, g, t, a);
            mma_row(acc, a, Ws[m], 1, g, t);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = 8 * j + 2 * t;
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int r = r0 + g + 8 * half;
                if (r >= n) continue;
                float2 v = make_float2(acc[j][2 * half], acc[j][2 * half + 1]);
                float2* out = reinterpret_cast<float2*>(dX + static_cast<size_t>(r) * H + c);
                if (B.accumulate) {
                    const float2 o = *out;
                    v.x += o.x;
                    v.y += o.y;
                }
                if (B.dexp) {
                    v.x = fmaf(B.dexp[r], B.wd[c], v.x);
                    v.y = fmaf(B.dexp[r], B.wd[c + 1], v.y);
                }
                *out = v;
            }
        }
    }
}

// s_i = a_i + sum_{j<i} e_ij hl_j + sum_{j>i} e_ij hu_j ;  h_out = h_in + relu(s)
__global__ void k_aggregate(const int* __restrict__ adj_ptr, const int* __restrict__ adj_col,
                            const float* __restrict__ adj_e, const float* __restrict__ a,
                            const float* __restrict__ hl, const float* __restrict__ hu,
                            const float* __restrict__ h_in, float* __restrict__ s, float* __restrict__ h_out, int n) {
    const int lane = threadIdx.x & 31;
    const int i = static_cast<int>((static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    float acc = a[static_cast<size_t>(i) * H + lane];
    for (int q = adj_ptr[i]; q < adj_ptr[i + 1]; ++q) {
        const int j = adj_col[q];
        const float* src = j < i ? hl : hu;
        acc = fmaf(adj_e[q], src[static_cast<size_t>(j) * H + lane], acc);
    }
    if (s) s[static_cast<size_t>(i) * H + lane] = acc;
    h_out[static_cast<size_t>(i) * H + lane] = h_in[static_cast<size_t>(i) * H + lane] + fmaxf(acc, 0.0f);
}

// Edge head and diagonal: warp per row i; lower edges of row i in CSR order.
__global__ void k_head(const int* __restrict__ low_ptr, const int* __restrict__ low_col,
                       const float* __restrict__ low_e, const float* __restrict__ low_f, const float* __restrict__ ph,
                       const float* __restrict__ qh,
                       const float* __restrict__ h, const float* __restrict__ isq, const float* __restrict__ wr,
                       ParamOffsets off, float* __restrict__ zpre, float* __restrict__ go, float* __restrict__ gval,
                       float* __restrict__ gd, float* __restrict__ td, float* __restrict__ gdiag, int n) {
    const int lane = threadIdx.x & 31;
    const int i = static_cast<int>((static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    const float c = wr[off.c + lane], c2 = wr[off.c2 + lane], w = wr[off.w + lane], bw = wr[off.bw];
    const float phv = ph[static_cast<size_t>(i) * H + lane];
    for (int k = low_ptr[i]; k < low_ptr[i + 1]; ++k) {
        const int j = low_col[k];
        const float zp = phv + qh[static_cast<size_t>(j) * H + lane] + c * low_e[k] + c2 * low_f[k];
        if (zpre) zpre[static_cast<size_t>(k) * H + lane] = zp;
        const float g = warp_sum_f(w * fmaxf(zp, 0.0f)) + bw;
        if (lane == 0) {
            go[k] = g;
            gval[k] = g * isq[j];
        }
    }
    const float t = warp_sum_f(wr[off.wd + lane] * h[static_cast<size_t>(i) * H + lane]) + wr[off.bwd];
    if (lane == 0) {
        const float e = expf(t);
        gd[i] = e;
        td[i] = t;
        gdiag[i] = e * isq[i];
    }
}

// ---- row-normalized Kaporin loss and the row normalization of G ----
// Row i's pattern P_i = {lower neighbours j < i (ascending), i}; Ghat_i on it is
// (go[low_ptr[i]..], gd[i]).  With A^ = D^-1/2 A D^-1/2 (unit diagonal, off-diagonals adj_e):
//   u_j = (A^ ghat_i)_j = ghat_ij + sum_{m in adj(j), m in P_i} adj_e(j,m) ghat_im   (j in P_i)
//   B_i = (G A G^T)_ii = sum_{j in P_i} ghat_ij u_j
// adj(j) and P_i are both ascending, so the membership test is a merge.  Warp per row, lane
// per pattern entry (loops for rows with more than 32).
__device__ __forceinline__ float kap_u(int i, int pos, int m, int lp, const int* __restrict__ low_col,
                                       const float* __restrict__ go, const float* __restrict__ gd,
                                       const int* __restrict__ adj_ptr, const int* __restrict__ adj_col,
                                       const float* __restrict__ adj_e) {
    const int j = pos < m - 1 ? low_col[lp + pos] : i;
    float u = pos < m - 1 ? go[lp + pos] : gd[i];  // the unit diagonal of A^
    int t = 0;                                      // cursor in P_i
    for (int q = adj_ptr[j]; q < adj_ptr[j + 1]; ++q) {
        const int c = adj_col[q];
        if (c > i) break;  // P_i has nothing above i
        while (t < m - 1 && low_col[lp + t] < c) ++t;
        const int pc = t < m - 1 ? low_col[lp + t] : i;
        if (pc == c) u = fmaf(adj_e[q], t < m - 1 ? go[lp + t] : gd[i], u);
    }
    return u;
}

// One Gauss-Seidel sweep on each row's quadratic form g^T A^[P_i, P_i] g with Ghat_ii held:
// for the lower entries j of row i in ascending order, ghat_ij -= (A^ ghat_i)_j, the exact
// minimizer in that coordinate (A^_jj = 1).  Every step lowers (G A G^T)_ii at a fixed Ghat_ii,
// so every row's Kaporin term log (G A G^T)_ii - 2 log Ghat_ii decreases (or stays): a strongly
// coupled pair (a_ij^2 close to a_ii a_jj), whose best ratio ghat_ij / ghat_ii = -e_ij the
// network cannot resolve to the precision the near-singular block needs, is set exactly.
// Thread per row; the row's values are read back after this thread's own writes, so they go
// through plain (coherent) loads.  gval follows go (gval = go / sqrt(a_jj)).
__device__ __forceinline__ float kap_u_rw(int i, int pos, int m, int lp, const int* __restrict__ low_col,
                                          const float* go, float gdi, const int* __restrict__ adj_ptr,
                                          const int* __restrict__ adj_col, const float* __restrict__ adj_e) {
    const int j = pos < m - 1 ? low_col[lp + pos] : i;
    float u = pos < m - 1 ? go[lp + pos] : gdi;
    int t = 0;
    for (int q = adj_ptr[j]; q < adj_ptr[j + 1]; ++q) {
        const int c = adj_col[q];
        if (c > i) break;
        while (t < m - 1 && low_col[lp + t] < c) ++t;
        const int pc = t < m - 1 ? low_col[lp + t] : i;
        if (pc == c) u = fmaf(adj_e[q], t < m - 1 ? go[lp + t] : gdi, u);
    }
    return u;
}

__global__ void k_row_sweep(const int* __restrict__ low_ptr, const int* __restrict__ low_col,
                            const int* __restrict__ adj_ptr, const int* __restrict__ adj_col,
                            const float* __restrict__ adj_e, const float* __restrict__ isq, float* go,
                            const float* __restrict__ gd, float* __restrict__ gval, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int lp = low_ptr[i];
    const int m = low_ptr[i + 1] - lp + 1;
    const float gdi = gd[i];
    for (int pos = 0; pos < m - 1; ++pos) {
        const float v = go[lp + pos] - kap_u_rw(i, pos, m, lp, low_col, go, gdi, adj_ptr, adj_col, adj_e);
        go[lp + pos] = v;
        gval[lp + pos] = v * isq[low_col[lp + pos]];
    }
}

// mode 0 (training): rowloss_i = log B_i - 2 t_i; dgo_k = 2 u_j / (n B_i) on the lower edges,
//   dexp_i = 2 u_i gd_i / (n B_i) - 2 / n on the diagonal (dL/dt_i).
// mode 1 (inference): rows of G (gval, gdiag) scaled by 1 / sqrt(B_i), so (G A G^T)_ii = 1.
// A row with B_i <= 0 or not finite counts in *bad and is left as it is.
__global__ void k_kaporin(const int* __restrict__ low_ptr, const int* __restrict__ low_col,
                          const int* __restrict__ adj_ptr, const int* __restrict__ adj_col,
                          const float* __restrict__ adj_e, const float* __restrict__ go,
                          const float* __restrict__ gd, const float* __restrict__ td, int n, int mode,
                          float* __restrict__ rowloss, float* __restrict__ dgo, float* __restrict__ dexp,
                          float* __restrict__ gval, float* __restrict__ gdiag, int* __restrict__ bad) {
    const int lane = threadIdx.x & 31;
    const int i = static_cast<int>((static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    const int lp = low_ptr[i];
    const int m = low_ptr[i + 1] - lp + 1;
    float part = 0.0f;
    float u0 = 0.0f;  // u of this lane's first entry (rows of at most 32 entries need no recompute)
    for (int pos = lane; pos < m; pos += 32) {
        const float u = kap_u(i, pos, m, lp, low_col, go, gd, adj_ptr, adj_col, adj_e);
        if (pos == lane) u0 = u;
        part = fmaf(pos < m - 1 ? go[lp + pos] : gd[i], u, part);
    }
    const float B = warp_sum_f(part);
    const bool ok = B > 0.0f && isfinite(B);
    if (!ok) {
        if (lane == 0) atomicAdd(bad, 1);
        if (mode == 0) {
            for (int pos = lane; pos < m - 1; pos += 32) dgo[lp + pos] = 0.0f;
            if (lane == 0) {
                rowloss[i] = 0.0f;
                dexp[i] = 0.0f;
            }
        }
        return;
    }
    if (mode == 1) {
        const float s = rsqrtf(B);
        for (int pos = lane; pos < m - 1; pos += 32) gval[lp + pos] *= s;
        if (lane == 0) gdiag[i] *= s;
        return;
    }
    const float inv_n = 1.0f / static_cast<float>(n);
    const float c = 2.0f * inv_n / B;
    for (int pos = lane; pos < m; pos += 32) {
        const float u = pos == lane ? u0 : kap_u(i, pos, m, lp, low_col, go, gd, adj_ptr, adj_col, adj_e);
        if (pos < m - 1) dgo[lp + pos] = c * u;
        else dexp[i] = c * u * gd[i] - 2.0f * inv_n;
    }
    if (lane == 0) rowloss[i] = logf(B) - 2.0f * td[i];
}

// sum partials of v over [count] (FP64 per block, fixed order)
__global__ void __launch_bounds__(256) k_sum_partial(const float* __restrict__ v, long long count,
                                                     double* __restrict__ partial) {
    __shared__ double red[8];
    double s = 0.0;
    for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < count;
         t += static_cast<long long>(gridDim.x) * blockDim.x)
        s += static_cast<double>(v[t]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < 8; ++q) t += red[q];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_dsum_final(const double* __restrict__ partial, int blocks, double scale, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < blocks; ++b) s += partial[b];
        *out = s * scale;
    }
}

// ---- probe-vector products (thread per (row, probe)) ----
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    unsigned long long z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void k_probes(float* __restrict__ v, long long count, unsigned long long seed) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const unsigned long long s = seed * 0xD1B54A32D192ED03ull;
    const unsigned long long a = splitmix64(s ^ (2ull * static_cast<unsigned long long>(q)));
    const unsigned long long b = splitmix64(s ^ (2ull * static_cast<unsigned long long>(q) + 1ull));
    const double u1 = (static_cast<double>(a >> 11) + 1.0) * (1.0 / 9007199254740992.0);
    const double u2 = (static_cast<double>(b >> 11) + 1.0) * (1.0 / 9007199254740992.0);
    v[q] = static_cast<float>(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
}

// out = G in (- sub):  row i: gdiag_i in_i + sum_{k in low(i)} gval_k in_{col k}
__global__ void k_g_apply(const int* __restrict__ low_ptr, const int* __restrict__ low_col,
                          const float* __restrict__ gval, const float* __restrict__ gdiag,
                          const float* __restrict__ in, const float* __restrict__ sub, float* __restrict__ out,
                          int n, int K) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<long long>(n) * K) return;
    const int i = static_cast<int>(t / K), p = static_cast<int>(t % K);
    float acc = gdiag[i] * in[t];
    for (int k = low_ptr[i]; k < low_ptr[i + 1]; ++k) acc = fmaf(gval[k], in[static_cast<size_t>(low_col[k]) * K + p], acc);
    out[t] = sub ? acc - sub[t] : acc;
}

// out = G^T in:  row j: gdiag_j in_j + sum_{k in up(j)} gval_k in_{row k}
__global__ void k_gt_apply(const int* __restrict__ up_ptr, const int* __restrict__ up_k,
                           const int* __restrict__ up_row, const float* __restrict__ gval,
                           const float* __restrict__ gdiag, const float* __restrict__ in, float* __restrict__ out,
                           int n, int K) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<long long>(n) * K) return;
    const int j = static_cast<int>(t / K), p = static_cast<int>(t % K);
    float acc = gdiag[j] * in[t];
    for (int q = up_ptr[j]; q < up_ptr[j + 1]; ++q)
        acc = fmaf(gval[up_k[q]], in[static_cast<size_t>(up_row[q]) * K + p], acc);
    out[t] = acc;
}

__global__ void k_a_apply(const int* __restrict__ a_ptr, const int* __restrict__ a_col, const float* __restrict__ a_val,
                          const float* __restrict__ in, float* __restrict__ out, int n, int K) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<long long>(n) * K) return;
    const int i = static_cast<int>(t / K), p = static_cast<int>(t % K);
    float acc = 0.0f;
    for (int q = a_ptr[i]; q < a_ptr[i + 1]; ++q) acc = fmaf(a_val[q], in[static_cast<size_t>(a_col[q]) * K + p], acc);
    out[t] = acc;
}

// dL/dGhat: lower edge k = (i, j): dgo_k = scale isq_j sum_p (r_ip w2_jp + v_ip y_jp);
// diagonal: dexp_i = dgd_i * gd_i with dgd_i = scale isq_i sum_p (r_ip w2_ip + v_ip y_ip)
__global__ void k_dG(const int* __restrict__ low_row, const int* __restrict__ low_col, const float* __restrict__ isq,
                     const float* __restrict__ r, const float* __restrict__ w2, const float* __restrict__ v,
                     const float* __restrict__ y, const float* __restrict__ gd, float* __restrict__ dgo,
                     float* __restrict__ dexp, int n_low, int n, int K, float scale) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n_low) {
        const int i = low_row[t], j = low_col[t];
        float acc = 0.0f;
        for (int p = 0; p < K; ++p)
            acc += r[static_cast<size_t>(i) * K + p] * w2[static_cast<size_t>(j) * K + p] +
                   v[static_cast<size_t>(i) * K + p] * y[static_cast<size_t>(j) * K + p];
        dgo[t] = scale * isq[j] * acc;
    } else if (t < n_low + n) {
        const int i = t - n_low;
        float acc = 0.0f;
        for (int p = 0; p < K; ++p)
            acc += r[static_cast<size_t>(i) * K + p] * w2[static_cast<size_t>(i) * K + p] +
                   v[static_cast<size_t>(i) * K + p] * y[static_cast<size_t>(i) * K + p];
        dexp[i] = scale * isq[i] * acc * gd[i];
    }
}

// dph_i = sum_{k in low(i)} dgo_k w .* [zpre_k > 0] ; dqh_j = sum_{k in up(j)} (same)
__global__ void k_head_back(const int* __restrict__ low_ptr, const int* __restrict__ up_ptr, const int* __restrict__ up_k,
                            const float* __restrict__ zpre, const float* __restrict__ dgo, const float* __restrict__ wr,
                            ParamOffsets off, float* __restrict__ dph, float* __restrict__ dqh, int n) {
    const int lane = threadIdx.x & 31;
    const int i = static_cast<int>((static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (i >= n) return;
    const float w = wr[off.w + lane];
    float a = 0.0f, b = 0.0f;
    for (int k = low_ptr[i]; k < low_ptr[i + 1]; ++k)
        if (zpre[static_cast<size_t>(k) * H + lane] > 0.0f) a = fmaf(dgo[k], w, a);
    for (int q = up_ptr[i]; q < up_ptr[i + 1]; ++q) {
        const int k = up_k[q];
        if (zpre[static_cast<size_t>(k) * H + lane] > 0.0f) b = fmaf(dgo[k], w, b);
    }
    dph[static_cast<size_t>(i) * H + lane] = a;
    dqh[static_cast<size_t>(i) * H + lane] = b;
}

// Layer backward through the aggregation: ds = dh .* [s > 0] for the own row, and
// dhl_j = sum_{i in N(j), i > j} e_ij ds_i ; dhu_j = sum_{i in N(j), i < j} e_ij ds_i.
__global__ void k_agg_back(const int* __restrict__ adj_ptr, const int* __restrict__ adj_col,
                           const float* __restrict__ adj_e, const float* __restrict__ dh, const float* __restrict__ s,
                           float* __restrict__ ds, float* __restrict__ dhl, float* __restrict__ dhu, int n) {
    const int lane = threadIdx.x & 31;
    const int j = static_cast<int>((static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (j >= n) return;
    const size_t oj = static_cast<size_t>(j) * H + lane;
    ds[oj] = s[oj] > 0.0f ? dh[oj] : 0.0f;
    float l = 0.0f, u = 0.0f;
    for (int q = adj_ptr[j]; q < adj_ptr[j + 1]; ++q) {
        const int i = adj_col[q];
        const size_t oi = static_cast<size_t>(i) * H + lane;
        const float d = s[oi] > 0.0f ? dh[oi] : 0.0f;
        if (i > j) l = fmaf(adj_e[q], d, l);
        else u = fmaf(adj_e[q], d, u);
    }
    dhl[oj] = l;
    dhu[oj] = u;
}

// dX_in = dX .* [X > 0]  (relu of the input layer: h0 > 0 iff its pre-activation > 0)
__global__ void k_relu_mask(const float* __restrict__ d, const float* __restrict__ x, float* __restrict__ out, long long count) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < count) out[t] = x[t] > 0.0f ? d[t] : 0.0f;
}

// ---- deterministic reductions ----
// partial[b][o*KB + k] = sum_{i in chunk b} D[i][o] X[i][k]; partial[b][32*KB + o] = sum D[i][o]
template <int KB>
__global__ void __launch_bounds__(256) k_outer_partial(const float* __restrict__ D, const float* __restrict__ X,
                                                       int n, int chunk, float* __restrict__ partial) {
    __shared__ float Ds[32][H + 1];
    __shared__ float Xs[32][KB + 1];
    constexpr int NOUT = H * KB + H;
    constexpr int PER = (NOUT + 255) / 256;
    float acc[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) acc[q] = 0.0f;
    const int i0 = blockIdx.x * chunk, i1 = min(n, i0 + chunk);
    for (int base = i0; base < i1; base += 32) {
        __syncthreads();
        for (int q = threadIdx.x; q < 32 * H; q += 256) {
            const int r = q / H, f = q % H, i = base + r;
            Ds[r][f] = i < i1 ? D[static_cast<size_t>(i) * H + f] : 0.0f;
        }
        for (int q = threadIdx.x; q < 32 * KB; q += 256) {
            const int r = q / KB, f = q % KB, i = base + r;
            Xs[r][f] = i < i1 ? X[static_cast<size_t>(i) * KB + f] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int o = threadIdx.x + 256 * q;
            if (o < H * KB) {
                const int a = o / KB, k = o % KB;
                float s = acc[q];
#pragma unroll 8
                for (int r = 0; r < 32; ++r) s = fmaf(Ds[r][a], Xs[r][k], s);
                acc[q] = s;
            } else if (o < NOUT) {
                const int a = o - H * KB;
                float s = acc[q];
#pragma unroll 8
                for (int r = 0; r < 32; ++r) s += Ds[r][a];
                acc[q] = s;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int o = threadIdx.x + 256 * q;
        if (o < NOUT) partial[static_cast<size_t>(blockIdx.x) * NOUT + o] = acc[q];
    }
}

// grad[dst_w + o] = sum_b partial[b][o] for o < nw ; grad[dst_b + o] = sum_b partial[b][nw + o] (dst_b >= 0)
__global__ void k_partial_final(const float* __restrict__ partial, int blocks, int stride, int nw, int nb,
                                float* __restrict__ grad, int dst_w, int dst_b) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nw + nb) return;
    float s = 0.0f;
    for (int b = 0; b < blocks; ++b) s += partial[static_cast<size_t>(b) * stride + o];
    if (o < nw) grad[dst_w + o] = s;
    else if (dst_b >= 0) grad[dst_b + (o - nw)] = s;
}

// Edge-head parameter partials over lower edges (warp per edge, grid-stride):
//   dw[f] += dgo relu(zpre_f), dc[f] += dgo w_f [zpre_f > 0] e, dc2[f] += dgo w_f [zpre_f > 0] f,
//   dbw += dgo;  partial row layout [dw (H) | dc (H) | dc2 (H) | dbw (1)]
constexpr int kEdgeRow = 3 * H + 1;
__global__ void __launch_bounds__(256) k_edge_partial(const float* __restrict__ zpre, const float* __restrict__ dgo,
                                                      const float* __restrict__ low_e, const float* __restrict__ low_f,
                                                      const float* __restrict__ wr, ParamOffsets off, int n_low,
                                                      float* __restrict__ partial) {
    __shared__ float red[8][kEdgeRow];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float w = wr[off.w + lane];
    float aw = 0.0f, ac = 0.0f, ac2 = 0.0f, ab = 0.0f;
    for (int k = blockIdx.x * 8 + warp; k < n_low; k += gridDim.x * 8) {
        const float z = zpre[static_cast<size_t>(k) * H + lane];
        const float d = dgo[k];
        aw = fmaf(d, fmaxf(z, 0.0f), aw);
        if (z > 0.0f) {
            ac = fmaf(d * w, low_e[k], ac);
            ac2 = fmaf(d * w, low_f[k], ac2);
        }
        ab += d;
    }
    red[warp][lane] = aw;
    red[warp][H + lane] = ac;
    red[warp][2 * H + lane] = ac2;
    if (lane == 0) red[warp][3 * H] = ab;
    __syncthreads();
    for (int o = threadIdx.x; o < kEdgeRow; o += blockDim.x) {
        float s = 0.0f;
        for (int q = 0; q < 8; ++q) s += red[q][o];
        partial[static_cast<size_t>(blockIdx.x) * kEdgeRow + o] = s;
    }
}

// Node partials of a weighted column sum: out[f] = sum_i coef_i X[i][f], out[H] = sum_i coef_i
__global__ void __launch_bounds__(256) k_vec_partial(const float* __restrict__ coef, const float* __restrict__ X, int n,
                                                     float* __restrict__ partial) {
    __shared__ float red[8][H + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float aw = 0.0f, ab = 0.0f;
    for (int i = blockIdx.x * 8 + warp; i < n; i += gridDim.x * 8) {
        const float c = coef[i];
        aw = fmaf(c, X[static_cast<size_t>(i) * H + lane], aw);
        ab += c;
    }
    red[warp][lane] = aw;
    if (lane == 0) red[warp][H] = ab;
    __syncthreads();
    for (int o = threadIdx.x; o < H + 1; o += blockDim.x) {
        float s = 0.0f;
        for (int q = 0; q < 8; ++q) s += red[q][o];
        partial[static_cast<size_t>(blockIdx.x) * (H + 1) + o] = s;
    }
}

// loss partials: sum of squares of r over [count]
__global__ void __launch_bounds__(256) k_sumsq_partial(const float* __restrict__ r, long long count, float* __restrict__ partial) {
    __shared__ float red[8];
    float s = 0.0f;
    for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < count;
         t += static_cast<long long>(gridDim.x) * blockDim.x)
        s = fmaf(r[t], r[t], s);
    s = warp_sum_f(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int q = 0; q < 8; ++q) t += red[q];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_loss_final(const float* __restrict__ partial, int blocks, double scale, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < blocks; ++b) s += static_cast<double>(partial[b]);
        *out = s * scale;
    }
}

__global__ void k_adam(float* __restrict__ theta, const float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, int P, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    theta[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_to_glow(const float* __restrict__ gval, const float* __restrict__ gdiag, const int* __restrict__ pos_low,
                          const int* __restrict__ pos_diag, double* __restrict__ g_low, int n_low, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n_low) g_low[pos_low[t]] = gval[t];
    else if (t < n_low + n) g_low[pos_diag[t - n_low]] = gdiag[t - n_low];
}

inline int blocks_for(long long count, int threads) {
    return static_cast<int>((count + threads - 1) / threads);
}

}  // namespace

ParamOffsets param_offsets() {
    ParamOffsets o{};
    int p = 0;
    o.W0 = p; p += H * 2;
    o.b0 = p; p += H;
    for (int l = 0; l < kLayers; ++l) {
        o.Wa[l] = p; p += H * H;
        o.ba[l] = p; p += H;
        o.Wl[l] = p; p += H * H;
        o.Wu[l] = p; p += H * H;
    }
    o.P = p; p += H * H;
    o.bp = p; p += H;
    o.Q = p; p += H * H;
    o.c = p; p += H;
    o.c2 = p; p += H;
    o.w = p; p += H;
    o.bw = p; p += 1;
    o.wd = p; p += H;
    o.bwd = p; p += 1;
    o.total = p;
    return o;
}

// ---------------------------------------------------------------------------------------
// Host: graph construction (the single builder for training and for the solver's inference)
// ---------------------------------------------------------------------------------------
// Runs f(begin, end) over [0, count) split into contiguous chunks on the host's threads.
template <typename F>
static void parallel_rows(int count, F&& f) {
    const int nt = std::max(1, std::min(32, static_cast<int>(std::thread::hardware_concurrency())));
    if (count < 4096 || nt == 1) {
        f(0, count);
        return;
    }
    std::vector<std::thread> pool;
    const int per = (count + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        const int b = t * per, e = std::min(count, b + per);
        if (b < e) pool.emplace_back([&f, b, e] { f(b, e); });
    }
    for (auto& th : pool) th.join();
}

void HostGraph::build(int n_, const int* row_ptr, const int* col_idx, const double* values) {
    n = n_;
    const size_t N = static_cast<size_t>(n);
    std::vector<double> d(N, 0.0), rowabs(N, 0.0), logd(N, 0.0);
    std::vector<int> adj_cnt(N, 0), low_cnt(N, 0), glow_cnt(N, 0);
    std::vector<unsigned char> dup(N, 0);
    // pass 1 (rows in parallel): diagonal, row abs-sum, how many entries each output takes
    parallel_rows(n, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            int diag_seen = 0;
            for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
                const int j = col_idx[q];
                rowabs[static_cast<size_t>(i)] += std::fabs(values[q]);
                if (j == i) {
                    d[static_cast<size_t>(i)] += values[q];
                    ++diag_seen;
                } else {
                    ++adj_cnt[static_cast<size_t>(i)];
                    if (j < i) ++low_cnt[static_cast<size_t>(i)];
                }
                if (j <= i) ++glow_cnt[static_cast<size_t>(i)];
            }
            dup[static_cast<size_t>(i)] = diag_seen > 1;
            logd[static_cast<size_t>(i)] = d[static_cast<size_t>(i)] > 0.0 ? std::log(d[static_cast<size_t>(i)]) : 0.0;
        }
    });
    for (int i = 0; i < n; ++i) {
        require(d[static_cast<size_t>(i)] > 0.0, XPLUS_ERR_DATA, "learned preconditioner needs a positive diagonal");
        require(!dup[static_cast<size_t>(i)], XPLUS_ERR_DATA, "duplicate diagonal entry");
    }
    double mean_ld = 0.0;
    for (double v : logd) mean_ld += v;
    mean_ld /= n;
    adj_ptr.assign(N + 1, 0);
    low_ptr.assign(N + 1, 0);
    std::vector<int> glow_ptr(N + 1, 0);
    for (int i = 0; i < n; ++i) {
        adj_ptr[static_cast<size_t>(i) + 1] = adj_ptr[static_cast<size_t>(i)] + adj_cnt[static_cast<size_t>(i)];
        low_ptr[static_cast<size_t>(i) + 1] = low_ptr[static_cast<size_t>(i)] + low_cnt[static_cast<size_t>(i)];
        glow_ptr[static_cast<size_t>(i) + 1] = glow_ptr[static_cast<size_t>(i)] + glow_cnt[static_cast<size_t>(i)];
    }
    n_adj = adj_ptr[N];
    n_low = low_ptr[N];
    n_glow = glow_ptr[N];
    const int64_t nnz = row_ptr[n];
    x.resize(N * 2);
    isq.resize(N);
    adj_col.resize(static_cast<size_t>(n_adj));
    adj_e.resize(static_cast<size_t>(n_adj));
    low_col.resize(static_cast<size_t>(n_low));
    low_row.resize(static_cast<size_t>(n_low));
    low_e.resize(static_cast<size_t>(n_low));
    pos_low.assign(static_cast<size_t>(n_low), -1);
    pos_diag.assign(N, -1);
    a_ptr.assign(row_ptr, row_ptr + n + 1);
    a_col.assign(col_idx, col_idx + nnz);
    a_val.resize(static_cast<size_t>(nnz));
    // pass 2 (rows in parallel): every row writes its own ranges of the outputs
    parallel_rows(n, [&](int b, int e) {
        std::vector<int> idx, kq;
        for (int i = b; i < e; ++i) {
            const size_t I = static_cast<size_t>(i);
            x[2 * I] = static_cast<float>(logd[I] - mean_ld);
            x[2 * I + 1] = static_cast<float>(rowabs[I] / d[I] - 1.0);
            isq[I] = static_cast<float>(1.0 / std::sqrt(d[I]));
            for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q) a_val[static_cast<size_t>(q)] = static_cast<float>(values[q]);
            // columns of row i in ascending order (stable for equal columns); kq[q - row_ptr[i]]
            // is the lower-edge index of CSR entry q (-1 for the diagonal and the upper entries)
            const int len = row_ptr[i + 1] - row_ptr[i];
            idx.resize(static_cast<size_t>(len));
            kq.assign(static_cast<size_t>(len), -1);
            std::iota(idx.begin(), idx.end(), row_ptr[i]);
            std::stable_sort(idx.begin(), idx.end(), [&](int a2, int b2) { return col_idx[a2] < col_idx[b2]; });
            int wa = adj_ptr[I], wl = low_ptr[I];
            for (int q : idx) {
                const int j = col_idx[q];
                if (j == i) continue;
                const float ev = static_cast<float>(values[q] / std::sqrt(d[I] * d[static_cast<size_t>(j)]));
                adj_col[static_cast<size_t>(wa)] = j;
                adj_e[static_cast<size_t>(wa)] = ev;
                ++wa;
                if (j < i) {
                    kq[static_cast<size_t>(q - row_ptr[i])] = wl;
                    low_col[static_cast<size_t>(wl)] = j;
                    low_row[static_cast<size_t>(wl)] = i;
                    low_e[static_cast<size_t>(wl)] = ev;
                    ++wl;
                }
            }
            // positions of this row's G entries in A's CSR order of the entries with col <= row
            int g = glow_ptr[I];
            for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
                const int j = col_idx[q];
                if (j > i) continue;
                if (j == i) pos_diag[I] = g++;
                else pos_low[static_cast<size_t>(kq[static_cast<size_t>(q - row_ptr[i])])] = g++;
            }
        }
    });
    // f_ij = sum over i's other lower neighbours m of e_jm e_mi (rows in parallel; adj(j) is
    // ascending, so each e_jm is a binary search)
    low_f.assign(static_cast<size_t>(n_low), 0.0f);
    parallel_rows(n, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            const int l0 = low_ptr[static_cast<size_t>(i)], l1 = low_ptr[static_cast<size_t>(i) + 1];
            for (int k = l0; k < l1; ++k) {
                const int j = low_col[static_cast<size_t>(k)];
                const int* a0 = adj_col.data() + adj_ptr[static_cast<size_t>(j)];
                const int* a1 = adj_col.data() + adj_ptr[static_cast<size_t>(j) + 1];
                double f = 0.0;
                for (int q = l0; q < l1; ++q) {
                    if (q == k) continue;
                    const int m = low_col[static_cast<size_t>(q)];
                    const int* at = std::lower_bound(a0, a1, m);
                    if (at != a1 && *at == m)
                        f += static_cast<double>(adj_e[static_cast<size_t>(at - adj_col.data())]) *
                             static_cast<double>(low_e[static_cast<size_t>(q)]);
                }
                low_f[static_cast<size_t>(k)] = static_cast<float>(f);
            }
        }
    });
    // lower edges grouped by column: up(j) = {k : low_col[k] == j}, by increasing row
    up_ptr.assign(N + 1, 0);
    for (int k = 0; k < n_low; ++k) ++up_ptr[static_cast<size_t>(low_col[static_cast<size_t>(k)]) + 1];
    for (int i = 0; i < n; ++i) up_ptr[static_cast<size_t>(i) + 1] += up_ptr[static_cast<size_t>(i)];
    up_k.assign(static_cast<size_t>(n_low), 0);
    up_row.assign(static_cast<size_t>(n_low), 0);
    std::vector<int> fill(up_ptr.begin(), up_ptr.end() - 1);
    for (int k = 0; k < n_low; ++k) {
        const int j = low_col[static_cast<size_t>(k)];
        const int at = fill[static_cast<size_t>(j)]++;
        up_k[static_cast<size_t>(at)] = k;
        up_row[static_cast<size_t>(at)] = low_row[static_cast<size_t>(k)];
    }
}

// ---------------------------------------------------------------------------------------
// Device graph + workspace
// ---------------------------------------------------------------------------------------
namespace {
template <typename T>
T* up(Arena& ar, const std::vector<T>& v, cudaStream_t st) {
    T* p = ar.get<T>(std::max<size_t>(v.size(), 1));
    if (!v.empty()) {
        const cudaError_t e = cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) throw Error(XPLUS_ERR_CUDA, std::string("H2D: ") + cudaGetErrorString(e));
    }
    return p;
}
}  // namespace

void* Arena::raw(size_t bytes) {
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 256));
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    ptrs.push_back(p);
    return p;
}
void Arena::release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
}

// ---------------------------------------------------------------------------------------
// The same graph built on the GPU for inference (forward, refinement, normalization and the
// g_low map): HostGraph::build's arrays, each CSR entry placed by its rank within its row
// (column order, CSR order between equal columns), so no row needs a sort buffer.  The only
// difference is the order of the FP64 sum behind the centring of log a_ii.
// ---------------------------------------------------------------------------------------
namespace {

// per row: diagonal (sum of its entries), |a| row sum, entry counts; bad: 1 no positive
// diagonal, 2 more than one diagonal entry
__global__ void k_gg_rows(const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v, int n,
                          double* __restrict__ d, double* __restrict__ rowabs, double* __restrict__ logd,
                          int* __restrict__ n_adj, int* __restrict__ n_low, int* __restrict__ n_glow, int* __restrict__ bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double di = 0.0, ra = 0.0;
    int seen = 0, a = 0, l = 0, gl = 0;
    for (int q = rp[i]; q < rp[i + 1]; ++q) {
        const int j = ci[q];
        ra += fabs(v[q]);
        if (j == i) {
            di += v[q];
            ++seen;
        } else {
            ++a;
            if (j < i) ++l;
        }
        if (j <= i) ++gl;
    }
    d[i] = di;
    rowabs[i] = ra;
    logd[i] = di > 0.0 ? log(di) : 0.0;
    n_adj[i] = a;
    n_low[i] = l;
    n_glow[i] = gl;
    if (!(di > 0.0)) atomicOr(bad, 1);
    if (seen > 1) atomicOr(bad, 2);
}

__global__ void k_gg_fill(const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v, int n,
                          const double* __restrict__ d, const double* __restrict__ rowabs, const double* __restrict__ logd,
                          const double* __restrict__ mean, const int* __restrict__ adj_ptr, const int* __restrict__ low_ptr,
                          const int* __restrict__ glow_ptr, int* __restrict__ adj_col, float* __restrict__ adj_e,
                          int* __restrict__ low_col, float* __restrict__ low_e, int* __restrict__ pos_low,
                          int* __restrict__ pos_diag, float* __restrict__ x, float* __restrict__ isq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double di = d[i];
    x[2 * i] = static_cast<float>(logd[i] - *mean);
    x[2 * i + 1] = static_cast<float>(rowabs[i] / di - 1.0);
    isq[i] = static_cast<float>(1.0 / sqrt(di));
    const int q0 = rp[i], q1 = rp[i + 1];
    int g = glow_ptr[i];
    for (int q = q0; q < q1; ++q) {
        const int j = ci[q];
        if (j != i) {
            int ra = 0, rl = 0;  // rank among the row's off-diagonal / lower entries
            for (int p = q0; p < q1; ++p) {
                const int c = ci[p];
                if (c == i) continue;
                const bool ahead = c < j || (c == j && p < q);
                ra += ahead;
                rl += ahead && c < i;
            }
            const float ev = static_cast<float>(v[q] / sqrt(di * d[j]));
            adj_col[adj_ptr[i] + ra] = j;
            adj_e[adj_ptr[i] + ra] = ev;
            if (j < i) {
                low_col[low_ptr[i] + rl] = j;
                low_e[low_ptr[i] + rl] = ev;
                pos_low[low_ptr[i] + rl] = g++;
            }
        } else {
            pos_diag[i] = g++;
        }
    }
}

// f_ij over the lower edges of row i (after the adjacency is complete)
__global__ void k_gg_f(const int* __restrict__ adj_ptr, const int* __restrict__ adj_col, const float* __restrict__ adj_e,
                       const int* __restrict__ low_ptr, const int* __restrict__ low_col, const float* __restrict__ low_e,
                       int n, float* __restrict__ low_f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int l0 = low_ptr[i], l1 = low_ptr[i + 1];
    for (int k = l0; k < l1; ++k) {
        const int j = low_col[k];
        const int a0 = adj_ptr[j], a1 = adj_ptr[j + 1];
        double f = 0.0;
        for (int q = l0; q < l1; ++q) {
            if (q == k) continue;
            const int m = low_col[q];
            int lo = a0, hi = a1;  // first adjacency entry >= m
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (adj_col[mid] < m) lo = mid + 1;
                else hi = mid;
            }
            if (lo < a1 && adj_col[lo] == m) f += static_cast<double>(adj_e[lo]) * static_cast<double>(low_e[q]);
        }
        low_f[k] = static_cast<float>(f);
    }
}

void gg_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

}  // namespace

void DevGraph::build_on_device(int n_, const int* d_rp, const int* d_ci, const double* d_v, const int* row_ptr,
                               const int* col_idx, const double* values, Arena& ar, cudaStream_t st) {
    n = n_;
    const int tb = 256;
    Arena tmp;
    try {
        double* d = tmp.get<double>(static_cast<size_t>(n));
        double* rowabs = tmp.get<double>(static_cast<size_t>(n));
        double* logd = tmp.get<double>(static_cast<size_t>(n));
        int* cnt = tmp.get<int>(3 * (static_cast<size_t>(n) + 1));
        int* bad = tmp.get<int>(1);
        double* mean = tmp.get<double>(1);
        gg_check(cudaMemsetAsync(cnt, 0, 3 * (static_cast<size_t>(n) + 1) * sizeof(int), st), "memset");
        gg_check(cudaMemsetAsync(bad, 0, sizeof(int), st), "memset");
        int* c_adj = cnt;
        int* c_low = cnt + (n + 1);
        int* c_glow = cnt + 2 * (n + 1);
        k_gg_rows<<<(n + tb - 1) / tb, tb, 0, st>>>(d_rp, d_ci, d_v, n, d, rowabs, logd, c_adj, c_low, c_glow, bad);
        gg_check(cudaGetLastError(), "graph rows");
        int h_bad = 0;
        gg_check(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        gg_check(cudaStreamSynchronize(st), "sync");
        if (h_bad) {
            HostGraph hg;  // the host builder throws the message of the first failing row
            hg.build(n, row_ptr, col_idx, values);
            throw Error(XPLUS_ERR_DATA, "learned preconditioner needs a positive, single diagonal entry per row");
        }
        adj_ptr = ar.get<int>(static_cast<size_t>(n) + 1);
        low_ptr = ar.get<int>(static_cast<size_t>(n) + 1);
        int* glow_ptr = tmp.get<int>(static_cast<size_t>(n) + 1);
        size_t bytes = 0;
        gg_check(cub::DeviceScan::ExclusiveSum(nullptr, bytes, c_adj, adj_ptr, n + 1, st), "scan size");
        void* ws = tmp.raw(std::max<size_t>(bytes, 1));
        gg_check(cub::DeviceScan::ExclusiveSum(ws, bytes, c_adj, adj_ptr, n + 1, st), "scan");
        gg_check(cub::DeviceScan::ExclusiveSum(ws, bytes, c_low, low_ptr, n + 1, st), "scan");
        gg_check(cub::DeviceScan::ExclusiveSum(ws, bytes, c_glow, glow_ptr, n + 1, st), "scan");
        size_t rbytes = 0;
        gg_check(cub::DeviceReduce::Sum(nullptr, rbytes, logd, mean, n, st), "reduce size");
        void* rws = tmp.raw(std::max<size_t>(rbytes, 1));
        gg_check(cub::DeviceReduce::Sum(rws, rbytes, logd, mean, n, st), "reduce");
        int sizes[3];
        gg_check(cudaMemcpyAsync(&sizes[0], adj_ptr + n, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        gg_check(cudaMemcpyAsync(&sizes[1], low_ptr + n, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        gg_check(cudaMemcpyAsync(&sizes[2], glow_ptr + n, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        double h_sum = 0.0;
        gg_check(cudaMemcpyAsync(&h_sum, mean, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        gg_check(cudaStreamSynchronize(st), "sync");
        n_adj = sizes[0];
        n_low = sizes[1];
        n_glow = sizes[2];
        const double h_mean = h_sum / static_cast<double>(n);  // the host builder's mean
        gg_check(cudaMemcpyAsync(mean, &h_mean, sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
        adj_col = ar.get<int>(std::max(1, n_adj));
        adj_e = ar.get<float>(std::max(1, n_adj));
        low_col = ar.get<int>(std::max(1, n_low));
        low_e = ar.get<float>(std::max(1, n_low));
        low_f = ar.get<float>(std::max(1, n_low));
        pos_low = ar.get<int>(std::max(1, n_low));
        pos_diag = ar.get<int>(static_cast<size_t>(n));
        x = ar.get<float>(2 * static_cast<size_t>(n));
        isq = ar.get<float>(static_cast<size_t>(n));
        k_gg_fill<<<(n + tb - 1) / tb, tb, 0, st>>>(d_rp, d_ci, d_v, n, d, rowabs, logd, mean, adj_ptr, low_ptr, glow_ptr,
                                                    adj_col, adj_e, low_col, low_e, pos_low, pos_diag, x, isq);
        gg_check(cudaGetLastError(), "graph fill");
        k_gg_f<<<(n + tb - 1) / tb, tb, 0, st>>>(adj_ptr, adj_col, adj_e, low_ptr, low_col, low_e, n, low_f);
        gg_check(cudaGetLastError(), "graph two-step paths");
        gg_check(cudaStreamSynchronize(st), "sync");
    } catch (...) {
        cudaStreamSynchronize(st);
        tmp.release();
        throw;
    }
    tmp.release();
}

void DevGraph::upload(const HostGraph& g, Arena& ar, cudaStream_t st) {
    n = g.n;
    n_low = g.n_low;
    n_adj = g.n_adj;
    n_glow = g.n_glow;
    adj_ptr = up(ar, g.adj_ptr, st);
    adj_col = up(ar, g.adj_col, st);
    adj_e = up(ar, g.adj_e, st);
    low_ptr = up(ar, g.low_ptr, st);
    low_col = up(ar, g.low_col, st);
    low_row = up(ar, g.low_row, st);
    low_e = up(ar, g.low_e, st);
    low_f = up(ar, g.low_f, st);
    up_ptr = up(ar, g.up_ptr, st);
    up_k = up(ar, g.up_k, st);
    up_row = up(ar, g.up_row, st);
    a_ptr = up(ar, g.a_ptr, st);
    a_col = up(ar, g.a_col, st);
    a_val = up(ar, g.a_val, st);
    x = up(ar, g.x, st);
    isq = up(ar, g.isq, st);
    pos_low = up(ar, g.pos_low, st);
    pos_diag = up(ar, g.pos_diag, st);
}

void Work::alloc(Arena& ar, int max_n, int max_low, int K_, bool train) {
    K = K_;
    const size_t nH = static_cast<size_t>(max_n) * H, lH = static_cast<size_t>(max_low) * H;
    for (int l = 0; l <= kLayers; ++l) h[l] = ar.get<float>(nH);
    for (int l = 0; l < kLayers; ++l) s[l] = train ? ar.get<float>(nH) : nullptr;
    a = ar.get<float>(nH);
    hl = ar.get<float>(nH);
    hu = ar.get<float>(nH);
    ph = ar.get<float>(nH);
    qh = ar.get<float>(nH);
    gval = ar.get<float>(static_cast<size_t>(max_low));
    gdiag = ar.get<float>(static_cast<size_t>(max_n));
    go = ar.get<float>(static_cast<size_t>(max_low));
    gd = ar.get<float>(static_cast<size_t>(max_n));
    td = ar.get<float>(static_cast<size_t>(max_n));
    bad = ar.get<int>(1);
    if (!train) return;
    zpre = ar.get<float>(lH);
    const size_t nK = static_cast<size_t>(max_n) * std::max(K, 1);
    v = ar.get<float>(nK);
    w1 = ar.get<float>(nK);
    w2 = ar.get<float>(nK);
    r = ar.get<float>(nK);
    t = ar.get<float>(nK);
    y = ar.get<float>(nK);
    dgo = ar.get<float>(static_cast<size_t>(max_low));
    dexp = ar.get<float>(static_cast<size_t>(max_n));
    dh = ar.get<float>(nH);
    dh2 = ar.get<float>(nH);
    ds = ar.get<float>(nH);
    dhl = ar.get<float>(nH);
    dhu = ar.get<float>(nH);
    dph = ar.get<float>(nH);
    dqh = ar.get<float>(nH);
    partial = ar.get<float>(static_cast<size_t>(kRedBlocks) * (H * H + H));
    dpartial = ar.get<double>(static_cast<size_t>(kRedBlocks));
    loss = ar.get<double>(1);
}

static void kcheck(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error(XPLUS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

static void kcheck_status(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(XPLUS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

void forward(const DevGraph& g, const float* wr, Work& w, bool train, cudaStream_t st) {
    const ParamOffsets off = param_offsets();
    const int n = g.n;
    const int nodes_blocks = blocks_for(static_cast<long long>(n) * 32, 256);
    const int lin_blocks = std::min(blocks_for(n, 8 * 16), 148 * 8);  // 8 warps of 16-node tiles
    k_input<<<blocks_for(static_cast<long long>(n) * H, 256), 256, 0, st>>>(g.x, wr + off.W0, wr + off.b0, w.h[0], n);
    kcheck("gnn input");
    for (int l = 0; l < kLayers; ++l) {
        Lin3 L{{wr + off.Wa[l], wr + off.Wl[l], wr + off.Wu[l]}, {wr + off.ba[l], nullptr, nullptr}, {w.a, w.hl, w.hu}, 3};
        k_node_lin<<<lin_blocks, 256, 0, st>>>(w.h[l], L, n);
        kcheck("gnn layer");
        k_aggregate<<<nodes_blocks, 256, 0, st>>>(g.adj_ptr, g.adj_col, g.adj_e, w.a, w.hl, w.hu, w.h[l],
                                                  train ? w.s[l] : nullptr, w.h[l + 1], n);
        kcheck("gnn aggregate");
    }
    Lin3 L{{wr + off.P, wr + off.Q, nullptr}, {wr + off.bp, nullptr, nullptr}, {w.ph, w.qh, nullptr}, 2};
    k_node_lin<<<lin_blocks, 256, 0, st>>>(w.h[kLayers], L, n);
    kcheck("gnn head lin");
    k_head<<<nodes_blocks, 256, 0, st>>>(g.low_ptr, g.low_col, g.low_e, g.low_f, w.ph, w.qh, w.h[kLayers], g.isq, wr, off,
                                         train ? w.zpre : nullptr, w.go, w.gval, w.gd, w.td, w.gdiag, n);
    kcheck("gnn head");
}

void refine_rows(const DevGraph& g, Work& w, int sweeps, cudaStream_t st) {
    for (int k = 0; k < sweeps; ++k) {
        k_row_sweep<<<blocks_for(g.n, 128), 128, 0, st>>>(g.low_ptr, g.low_col, g.adj_ptr, g.adj_col, g.adj_e, g.isq,
                                                          w.go, w.gd, w.gval, g.n);
        kcheck("gnn row sweep");
    }
}

void normalize_rows(const DevGraph& g, Work& w, cudaStream_t st) {
    const int nodes_blocks = blocks_for(static_cast<long long>(g.n) * 32, 256);
    kcheck_status(cudaMemsetAsync(w.bad, 0, sizeof(int), st), "gnn memset");
    k_kaporin<<<nodes_blocks, 256, 0, st>>>(g.low_ptr, g.low_col, g.adj_ptr, g.adj_col, g.adj_e, w.go, w.gd, w.td,
                                            g.n, 1, nullptr, nullptr, nullptr, w.gval, w.gdiag, w.bad);
    kcheck("gnn normalize rows");
    int bad = 0;
    kcheck_status(cudaMemcpyAsync(&bad, w.bad, sizeof(int), cudaMemcpyDeviceToHost, st), "gnn D2H");
    kcheck_status(cudaStreamSynchronize(st), "gnn sync");
    require(bad == 0, XPLUS_ERR_DATA, "a row of the predicted G has (G A G^T)_ii <= 0 or not finite");
}

void g_to_low(const DevGraph& g, const Work& w, double* d_glow, cudaStream_t st) {
    k_to_glow<<<blocks_for(static_cast<long long>(g.n_low) + g.n, 256), 256, 0, st>>>(w.gval, w.gdiag, g.pos_low, g.pos_diag,
                                                                                    d_glow, g.n_low, g.n);
    kcheck("gnn g_low");
}

static void outer_grad(const float* D, const float* X, int kb, int n, Work& w, float* grad, int dst_w, int dst_b,
                       cudaStream_t st) {
    const int chunk = std::max(32, ((n + kRedBlocks - 1) / kRedBlocks + 31) / 32 * 32);
    const int blocks = (n + chunk - 1) / chunk;
    const int nw = H * kb;
    if (kb == H) k_outer_partial<H><<<blocks, 256, 0, st>>>(D, X, n, chunk, w.partial);
    else k_outer_partial<2><<<blocks, 256, 0, st>>>(D, X, n, chunk, w.partial);
    kcheck("gnn outer partial");
    k_partial_final<<<blocks_for(nw + H, 128), 128, 0, st>>>(w.partial, blocks, nw + H, nw, dst_b >= 0 ? H : 0, grad,
                                                              dst_w, dst_b);
    kcheck("gnn outer final");
}

static void wd_grad(const float* coef, const float* X, int n, Work& w, float* grad, int dst_w, int dst_b,
                    cudaStream_t st) {
    const int blocks = std::max(1, std::min(kRedBlocks, blocks_for(n, 8)));
    k_vec_partial<<<blocks, 256, 0, st>>>(coef, X, n, w.partial);
    kcheck("gnn vec partial");
    k_partial_final<<<1, 64, 0, st>>>(w.partial, blocks, H + 1, H, 1, grad, dst_w, dst_b);
    kcheck("gnn vec final");
}

void loss_backward(const DevGraph& g, const float* wr, Work& w, float* grad, unsigned long long seed, cudaStream_t st) {
    if (w.loss_kind == kLossKaporin) {
        const int n = g.n;
        const int nodes_blocks = blocks_for(static_cast<long long>(n) * 32, 256);
        kcheck_status(cudaMemsetAsync(w.bad, 0, sizeof(int), st), "gnn memset");
        k_kaporin<<<nodes_blocks, 256, 0, st>>>(g.low_ptr, g.low_col, g.adj_ptr, g.adj_col, g.adj_e, w.go, w.gd, w.td,
                                                n, 0, w.r, w.dgo, w.dexp, nullptr, nullptr, w.bad);
        kcheck("gnn kaporin");
        const int lb = std::min(kRedBlocks, blocks_for(n, 256));
        k_sum_partial<<<lb, 256, 0, st>>>(w.r, n, w.dpartial);
        k_dsum_final<<<1, 32, 0, st>>>(w.dpartial, lb, 1.0 / static_cast<double>(n), w.loss);
        kcheck("gnn kaporin loss");
        if (grad) backward_from_dg(g, wr, w, grad, st);
        return;
    }
    const int n = g.n, K = w.K;
    const long long nK = static_cast<long long>(n) * K;
    const int pb = blocks_for(nK, 256);
    k_probes<<<pb, 256, 0, st>>>(w.v, nK, seed);
    kcheck("gnn probes");
    // r = G A G^T v - v ; y = A G^T r
    k_gt_apply<<<pb, 256, 0, st>>>(g.up_ptr, g.up_k, g.up_row, w.gval, w.gdiag, w.v, w.w1, n, K);
    k_a_apply<<<pb, 256, 0, st>>>(g.a_ptr, g.a_col, g.a_val, w.w1, w.w2, n, K);
    k_g_apply<<<pb, 256, 0, st>>>(g.low_ptr, g.low_col, w.gval, w.gdiag, w.w2, w.v, w.r, n, K);
    k_gt_apply<<<pb, 256, 0, st>>>(g.up_ptr, g.up_k, g.up_row, w.gval, w.gdiag, w.r, w.t, n, K);
    k_a_apply<<<pb, 256, 0, st>>>(g.a_ptr, g.a_col, g.a_val, w.t, w.y, n, K);
    kcheck("gnn probe products");
    const int lb = std::min(kRedBlocks, blocks_for(nK, 256));
    k_sumsq_partial<<<lb, 256, 0, st>>>(w.r, nK, w.partial);
    k_loss_final<<<1, 32, 0, st>>>(w.partial, lb, 1.0 / static_cast<double>(nK), w.loss);
    kcheck("gnn loss");
    if (!grad) return;
    const float scale = 2.0f / static_cast<float>(nK);
    k_dG<<<blocks_for(static_cast<long long>(g.n_low) + n, 256), 256, 0, st>>>(g.low_row, g.low_col, g.isq, w.r, w.w2, w.v,
                                                                              w.y, w.gd, w.dgo, w.dexp, g.n_low, n, K, scale);
    kcheck("gnn dG");
    backward_from_dg(g, wr, w, grad, st);
}

// Parameter gradient from dL/dGhat on the lower edges (w.dgo) and dL/dt on the diagonal
// (w.dexp): the chain every loss shares.
void backward_from_dg(const DevGraph& g, const float* wr, Work& w, float* grad, cudaStream_t st) {
    const ParamOffsets off = param_offsets();
    const int n = g.n;
    const int nodes_blocks = blocks_for(static_cast<long long>(n) * 32, 256);
    const int lin_blocks = std::min(blocks_for(n, 8 * 16), 148 * 8);  // 8 warps of 16-node tiles
    k_head_back<<<nodes_blocks, 256, 0, st>>>(g.low_ptr, g.up_ptr, g.up_k, w.zpre, w.dgo, wr, off, w.dph, w.dqh, n);
    kcheck("gnn head back");
    // edge-head parameters w, c, bw
    {
        const int eb = std::max(1, std::min(kRedBlocks, blocks_for(g.n_low, 8)));
        k_edge_partial<<<eb, 256, 0, st>>>(w.zpre, w.dgo, g.low_e, g.low_f, wr, off, g.n_low, w.partial);
        kcheck("gnn edge partial");
        // partial rows: [dw (H) | dc (H) | dc2 (H) | dbw (1)]
        k_partial_final<<<1, 128, 0, st>>>(w.partial, eb, kEdgeRow, H, 0, grad, off.w, -1);
        k_partial_final<<<1, 128, 0, st>>>(w.partial + H, eb, kEdgeRow, H, 0, grad, off.c, -1);
        k_partial_final<<<1, 128, 0, st>>>(w.partial + 2 * H, eb, kEdgeRow, H, 0, grad, off.c2, -1);
        k_partial_final<<<1, 32, 0, st>>>(w.partial + 3 * H, eb, kEdgeRow, 1, 0, grad, off.bw, -1);
        kcheck("gnn edge final");
    }
    const float* hL = w.h[kLayers];
    outer_grad(w.dph, hL, H, n, w, grad, off.P, off.bp, st);
    outer_grad(w.dqh, hL, H, n, w, grad, off.Q, -1, st);
    // dh = dph P + dqh Q + dexp wd
    BackLin B{{wr + off.P, wr + off.Q, nullptr}, {w.dph, w.dqh, nullptr}, 2, w.dexp, wr + off.wd, 0};
    k_node_backlin<<<lin_blocks, 256, 0, st>>>(B, w.dh, n);
    kcheck("gnn head backlin");
    wd_grad(w.dexp, hL, n, w, grad, off.wd, off.bwd, st);
    for (int l = kLayers - 1; l >= 0; --l) {
        k_agg_back<<<nodes_blocks, 256, 0, st>>>(g.adj_ptr, g.adj_col, g.adj_e, w.dh, w.s[l], w.ds, w.dhl, w.dhu, n);
        kcheck("gnn agg back");
        const float* hin = w.h[l];
        outer_grad(w.ds, hin, H, n, w, grad, off.Wa[l], off.ba[l], st);
        outer_grad(w.dhl, hin, H, n, w, grad, off.Wl[l], -1, st);
        outer_grad(w.dhu, hin, H, n, w, grad, off.Wu[l], -1, st);
        // dh <- dh + ds Wa + dhl Wl + dhu Wu
        BackLin Bl{{wr + off.Wa[l], wr + off.Wl[l], wr + off.Wu[l]}, {w.ds, w.dhl, w.dhu}, 3, nullptr, nullptr, 1};
        k_node_backlin<<<lin_blocks, 256, 0, st>>>(Bl, w.dh, n);
        kcheck("gnn layer backlin");
    }
    k_relu_mask<<<blocks_for(static_cast<long long>(n) * H, 256), 256, 0, st>>>(w.dh, w.h[0], w.dh2,
                                                                              static_cast<long long>(n) * H);
    kcheck("gnn input mask");
    outer_grad(w.dh2, g.x, 2, n, w, grad, off.W0, off.b0, st);
}

void adam_step(float* theta, const float* grad, float* m, float* v, int P, float lr, int step, cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, static_cast<float>(step));
    const float c2 = 1.0f - std::pow(b2, static_cast<float>(step));
    k_adam<<<blocks_for(P, 256), 256, 0, st>>>(theta, grad, m, v, P, lr, b1, b2, 1e-8f, c1, c2);
    kcheck("gnn adam");
}

void round_params(const float* master, float* wr, int P, cudaStream_t st) {
    k_round_params<<<blocks_for(P, 256), 256, 0, st>>>(master, wr, P);
    kcheck("gnn round");
}

}  // namespace gnn
}  // namespace xplus
