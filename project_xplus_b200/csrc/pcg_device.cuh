// pcg_device.cuh -- device helpers shared by the persistent PCG kernels: SELL row products,
// the FP64 residual row, deterministic grid reductions and the {z, p} node records.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/xplus_b200.h"
#include "device_common.cuh"
#include "pcg_kernels.cuh"

namespace xplus {
namespace dev {

constexpr double kBreakdownEps = 1.0e-30;  // include/cg_common.hpp:13

// Search direction after an FP64 residual replacement (xplus_opts.restart_on_replace), and
// the stagnation test, for one solve.  Modes: 0 keeps p (beta = rz_new / rz_old); 1 restarts
// it (beta = 0) at every replacement; 2 restarts it only at drop- or convergence-triggered
// replacements; 4 re-conjugates it to the replaced residual with the flexible-CG coefficient
// beta = -(z_new . Ap') / (p' . Ap') (Notay's FCG(1); equal to rz_new / rz_old when the
// replaced residual is the recurrence one), which survives the gap an inexact low-precision
// operator opens between the two residuals.  Policy 3 starts in mode 2 and policy 4 in mode 4;
// both drop to mode 1 for the rest of the solve when a replacement finds ||b - A x|| above
// twice its best (CG's residual is not monotone, so a smaller rise is no signal) or the
// stagnation window runs out.
// The policy itself stays in the kernel arguments (read where needed, no register held).
struct ReplacePolicy {
    int mode, stagnant;
    double best;
    __device__ ReplacePolicy(int policy, double true_rr)
        : mode(policy == 3 ? 2 : policy), stagnant(0), best(true_rr) {}
    // After a replacement that measured true_rr = ||b - A x||^2: true when the solve stagnated.
    __device__ bool after(int policy, double true_rr, double stag_factor, int stag_window) {
        if (((policy == 3 && mode == 2) || mode == 4) && true_rr > 4.0 * best) mode = 1;
        if (true_rr < stag_factor * best) {
            best = true_rr;
            stagnant = 0;
        } else if (++stagnant >= stag_window) {
            if ((policy == 3 && mode == 2) || mode == 4) {
                mode = 1;  // no progress keeping p: restart it at every replacement from now on
                stagnant = 0;
            } else {
                return true;
            }
        }
        return false;
    }
    // zap = z_new . Ap' (taken by the replacement), pap = p' . Ap' of the iteration
    // (one division site: a second one would cost the hot loop registers)
    __device__ double beta(bool replaced, bool drop_replaced, double rz, double rz_old, double zap,
                           double pap) const {
        double num = rz, den = rz_old;
        if (replaced && mode == 4) {
            num = -zap;
            den = pap;
        } else if ((mode == 1 && replaced) || (mode == 2 && drop_replaced)) {
            num = 0.0;
            den = 1.0;
        }
        return num / den;
    }
};

// Row `32*s + lane` of the SELL matrix times x, accumulated in AT.  With DIFF the slots hold
// the off-diagonal weights w_ij only and the row computes sum_j w_ij (x_j - x_i); the caller
// adds s_i x_i with the row sum s_i = sum_j a_ij.  That form is exact algebra, and it keeps
// the operator a weighted graph Laplacian plus a diagonal when w and s are rounded to low
// precision: every stored number carries only its own relative rounding error, whereas
// rounding a_ii itself shifts the near-null space of a stiffness matrix.
template <typename VT, int CHUNK, bool DIFF, typename IT, typename XV, typename AT>
__device__ __forceinline__ AT sell_row(const long long* __restrict__ slice_ptr,
                                       const IT* __restrict__ col, const VT* __restrict__ val,
                                       int s, int lane, const XV* x, AT xi) {
    const long long base = slice_ptr[s];
    const int w = static_cast<int>((slice_ptr[s + 1] - base) >> 5);
    const int row = s * 32 + lane;
    const VT* vp = val + base + lane * CHUNK;
    const IT* cp = col + base + lane * CHUNK;
    AT acc = AT(0);
    int c = 0;
    // two chunks in flight per step
    for (; c + 2 * CHUNK <= w; c += 2 * CHUNK) {
        typename ValArith<VT>::type v0[CHUNK], v1[CHUNK];
        int c0[CHUNK], c1[CHUNK];
        ChunkLoad<VT, CHUNK>::run(vp, v0);
        ColLoad<CHUNK, IT>::run(cp, row, c0);
        ChunkLoad<VT, CHUNK>::run(vp + 32 * CHUNK, v1);
        ColLoad<CHUNK, IT>::run(cp + 32 * CHUNK, row, c1);
        AT xv0[CHUNK], xv1[CHUNK];
#pragma unroll
        for (int q = 0; q < CHUNK; ++q) xv0[q] = static_cast<AT>(x[c0[q]]);
#pragma unroll
        for (int q = 0; q < CHUNK; ++q) xv1[q] = static_cast<AT>(x[c1[q]]);
        if (DIFF) {
#pragma unroll
            for (int q = 0; q < CHUNK; ++q) {
                xv0[q] -= xi;
                xv1[q] -= xi;
            }
        }
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
        ColLoad<CHUNK, IT>::run(cp, row, c0);
#pragma unroll
        for (int q = 0; q < CHUNK; ++q) {
            AT xv = static_cast<AT>(x[c0[q]]);
            if (DIFF) xv -= xi;
            acc += static_cast<AT>(v0[q]) * xv;
        }
    }
    return acc;
}

// FP64 row of A times x64: the FP64 copy when present (off-diagonals + exact diagonal in
// the split layout), else the stored values widened.
template <typename VT, typename XT, int CHUNK, bool DIFF, typename IT>
__device__ __forceinline__ double row_fp64(const PcgArgs& a, int s, int lane, int row) {
    const double xi = a.x64[row];
    const IT* col = static_cast<const IT*>(a.col);
    double y;
    if (a.val64) {
        y = sell_row<double, CHUNK, false, IT, double, double>(a.slice_ptr, col, a.val64, s, lane, a.x64, 0.0);
        if (DIFF) y += a.diag64[row] * xi;
    } else {
        y = sell_row<VT, CHUNK, DIFF, IT, double, double>(a.slice_ptr, col, static_cast<const VT*>(a.val),
                                                          s, lane, a.x64, xi);
        if (DIFF) y = y * static_cast<double>(a.val_scale) +
                      static_cast<double>(static_cast<const XT*>(a.rowsum)[row]) * xi;
    }
    return y;
}

// Sum of the per-block partials of each slot q < nq (fixed order, same in every block).  Warp
// q sums slot q, and each lane issues all its loads before adding, so the whole reduction is
// one L2 round trip however many slots there are (nq <= number of warps).
__device__ __forceinline__ void grid_totals(const double* partial, int nq, double* s_tot) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < nq) {
        const double* src = partial + static_cast<size_t>(warp) * gridDim.x;
        double v = 0.0;
        for (int base = 0; base < static_cast<int>(gridDim.x); base += 256) {
            double t[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int b = base + lane + 32 * k;
                t[k] = b < static_cast<int>(gridDim.x) ? __ldcg(src + b) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) v += t[k];
        }
        v = warp_sum(v);
        if (lane == 0) s_tot[warp] = v;
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

// The warp sums of eight values with 9 double shuffles instead of 40: three levels of
// reduce-scatter (partners swap the half of the values that the other keeps, each adding
// what it receives to what it keeps), then two plain levels.  Lane l returns the total of
// value 4*bit4(l) + 2*bit3(l) + bit2(l); the four lanes that share those bits return the
// same bits (a + b == b + a in floating point).
__device__ __forceinline__ double warp_sum8_scatter(const double (&v)[8], int lane) {
    const bool b = (lane >> 4) & 1, c = (lane >> 3) & 1, d = (lane >> 2) & 1;
    double w[4], u[2];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double keep = b ? v[4 + j] : v[j];
        const double give = b ? v[j] : v[4 + j];
        w[j] = keep + __shfl_xor_sync(0xffffffffu, give, 16);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const double keep = c ? w[2 + j] : w[j];
        const double give = c ? w[j] : w[2 + j];
        u[j] = keep + __shfl_xor_sync(0xffffffffu, give, 8);
    }
    double t = (d ? u[1] : u[0]) + __shfl_xor_sync(0xffffffffu, d ? u[0] : u[1], 4);
    t += __shfl_xor_sync(0xffffffffu, t, 2);
    t += __shfl_xor_sync(0xffffffffu, t, 1);
    return t;
}

// Block sums of up to eight values at a fraction of block_sum's shuffles: warp sums by
// warp_sum8_scatter, then warp q sums value q over the warps and lane 0 of warp q calls
// store(q, total).  Every call must be separated from the previous user of s_red by a
// __syncthreads (in the persistent kernels a grid or cluster barrier always is).  Fixed
// combination order.
template <int NV, typename Store>
__device__ __forceinline__ void block_sum_scatter(const double (&v)[NV], double* s_red, Store&& store) {
    static_assert(NV <= 8, "block_sum_scatter sums at most eight values");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double v8[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v8[q] = q < NV ? v[q] : 0.0;
    const double t = warp_sum8_scatter(v8, lane);
    const int q = (((lane >> 4) & 1) << 2) | (((lane >> 3) & 1) << 1) | ((lane >> 2) & 1);
    if ((lane & 3) == 0 && q < NV) s_red[q * 32 + warp] = t;
    __syncthreads();
    if (warp < NV) {
        const double x = warp_sum(lane < nwarps ? s_red[warp * 32 + lane] : 0.0);
        if (lane == 0) store(warp, x);
    }
}

// publish() for up to eight values through block_sum_scatter.
template <int NV>
__device__ __forceinline__ void publish_scatter(const double (&v)[NV], double* s_red, double* partial) {
    block_sum_scatter<NV>(v, s_red, [&](int q, double x) {
        partial[static_cast<size_t>(q) * gridDim.x + blockIdx.x] = x;
    });
}

inline __device__ bool bad(double v) { return v != v; }

// What the SpMV needs from a neighbour j: z_j = M^-1 r_j and the previous search direction
// p_j, packed so one 8-byte (FP32) or 16-byte (FP64) load fetches both.  The new direction
// p'_j = z_j + beta p_j is recomputed by every reader with the same node_pnew(), so all copies
// are bit-identical to the owner's; the owner stores {z_new, p'} only in phase B, after the
// barrier that ends every read of the old pair, so one buffer suffices.
template <typename XT>
struct alignas(2 * sizeof(XT)) NodeRec {
    XT z, p;
};

__device__ __forceinline__ float node_pnew(float z, float beta, float p) { return __fmaf_rn(beta, p, z); }
__device__ __forceinline__ double node_pnew(double z, double beta, double p) { return __fma_rn(beta, p, z); }

__device__ __forceinline__ NodeRec<float> load_rec(const NodeRec<float>* q) {
    const float2 v = *reinterpret_cast<const float2*>(q);
    return NodeRec<float>{v.x, v.y};
}
__device__ __forceinline__ NodeRec<double> load_rec(const NodeRec<double>* q) {
    const double2 v = *reinterpret_cast<const double2*>(q);
    return NodeRec<double>{v.x, v.y};
}
__device__ __forceinline__ void store_rec(NodeRec<float>* q, float z, float p) {
    *reinterpret_cast<float2*>(q) = make_float2(z, p);
}
__device__ __forceinline__ void store_rec(NodeRec<double>* q, double z, double p) {
    *reinterpret_cast<double2*>(q) = make_double2(z, p);
}

// NS slices of one warp at a time (lane = row within each): for every pair of chunks, the
// value/column loads of all NS rows are issued, then all their neighbour-record gathers,
// then the arithmetic -- so NS * 2 * CHUNK gathers per thread are in flight together.  The slot
// loads bypass L1 (the matrix streams once per iteration); the record gathers keep it.
// Returns y_k = (A p')_row_k without the row-sum term; pi[k] = p'_row_k.
template <typename VT, int CHUNK, bool DIFF, typename IT, typename XT, int NS>
__device__ __forceinline__ void sell_rows_pnew(const int2 (&sl)[NS], const int (&row)[NS], int lane,
                                               const IT* __restrict__ col, const VT* __restrict__ val,
                                               const NodeRec<XT>* rec, XT beta, const XT (&pi)[NS],
                                               XT (&y)[NS]) {
    int wmax = 0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        y[k] = XT(0);
        wmax = max(wmax, sl[k].y);
    }
    for (int c = 0; c < wmax; c += 2 * CHUNK) {
        typename ValArith<VT>::type v[NS][2][CHUNK];
        int cc[NS][2][CHUNK];
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (c + h * CHUNK < sl[k].y) {
                    const int off = sl[k].x + (c + h * CHUNK) * 32 + lane * CHUNK;
                    ChunkLoad<VT, CHUNK, true>::run(val + off, v[k][h]);
                    ColLoad<CHUNK, IT, true>::run(col + off, row[k], cc[k][h]);
                } else {
#pragma unroll
                    for (int q = 0; q < CHUNK; ++q) {
                        v[k][h][q] = 0;
                        cc[k][h][q] = -1;
                    }
                }
            }
        NodeRec<XT> nb[NS][2][CHUNK];
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int q = 0; q < CHUNK; ++q)
                    nb[k][h][q] = cc[k][h][q] >= 0 ? load_rec(rec + cc[k][h][q]) : NodeRec<XT>{XT(0), XT(0)};
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int q = 0; q < CHUNK; ++q) {
                    XT pj = node_pnew(nb[k][h][q].z, beta, nb[k][h][q].p);
                    if (DIFF) pj -= pi[k];
                    y[k] += static_cast<XT>(v[k][h][q]) * pj;
                }
    }
}


// NS slices of one warp: all value/column loads of the group first (the only global traffic,
// or shared-memory loads with LD = kLdPlain when the matrix itself is staged there), then the
// products with p' gathered from the shared-memory window.  y_k excludes s_i p'_i.
template <typename VT, int CHUNK, typename IT, int NS, int LD = kLdg>
__device__ __forceinline__ void sell_rows_smem(const int2 (&sl)[NS], const int (&row)[NS], int lane,
                                               const IT* __restrict__ col, const VT* __restrict__ val,
                                               const float* pw, int w0, const float (&pi)[NS],
                                               float (&y)[NS]) {
    int wmax = 0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        y[k] = 0.0f;
        wmax = max(wmax, sl[k].y);
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
                    ChunkLoad<VT, CHUNK, LD>::run(val + off, v[k][h]);
                    ColLoad<CHUNK, IT, LD>::run(col + off, row[k], cc[k][h]);
                } else {
#pragma unroll
                    for (int q = 0; q < CHUNK; ++q) {
                        v[k][h][q] = 0.0f;
                        cc[k][h][q] = row[k] >= 0 ? row[k] : w0;
                    }
                }
            }
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int q = 0; q < CHUNK; ++q) y[k] += v[k][h][q] * (pw[cc[k][h][q] - w0] - pi[k]);
    }
}

}  // namespace dev
}  // namespace xplus
