// gtg_layout_gpu.hpp -- the G / G^T SELL images of the factorized preconditioner built on the
// GPU (gtg_layout_gpu.cu), bit-identical to the host construction in solver.cu.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>

namespace xplus {

struct GtgImages {
    int64_t n_glow = 0, g_slots = 0, gt_slots = 0;
    long long *g_slice_ptr = nullptr, *gt_slice_ptr = nullptr;
    int *g_col = nullptr, *g_map = nullptr, *gt_col = nullptr, *gt_map = nullptr;
};

// row_ptr / col_idx: the host CSR given to xplus_pcg_create (original order); d_perm: its SELL
// order (perm[new] = old); alloc(bytes) returns device memory that outlives the call (the
// handle's).  Blocks until the images are complete.
GtgImages gtg_layout_device(int n, int n_pad, const int* row_ptr, const int* col_idx, const int* d_perm,
                            const std::function<void*(size_t)>& alloc, cudaStream_t st);

}  // namespace xplus
