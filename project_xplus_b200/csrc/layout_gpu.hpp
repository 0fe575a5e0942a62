// layout_gpu.hpp -- the arrays xplus_pcg_create derives from the CSR, built on the GPU from a
// device copy of the CSR (sell_gpu.cu).  The host path of solver.cu computes the same arrays
// and is the reference for each one: every function here is bit-identical to it.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace xplus {

// The CSR uploaded once; the structure checks run on the device and, when one fails, the host
// validator is run to throw the reference's own message.
struct DeviceCsr {
    int n = 0;
    int64_t nnz = 0;
    int* rp = nullptr;
    int* ci = nullptr;
    double* v = nullptr;
    std::vector<void*> owned;
    ~DeviceCsr();
};
void upload_csr(int n, const int* row_ptr, const int* col_idx, const double* values, DeviceCsr& csr, cudaStream_t st);

// diag[i] = a_ii of the first diagonal entry of row i (src/CsrDataset.hpp:92-116); a missing or
// zero entry throws the host function's message.
void jacobi_diag_device(const DeviceCsr& csr, const int* row_ptr, const int* col_idx, const double* values,
                        double* d_diag, cudaStream_t st);

// *d_count += #{i < n : |v_i| <= eps} (the caller zeroes it).
void count_below(const double* d_v, int n, double eps, int* d_count, cudaStream_t st);

// SELL-C-sigma (C = 32) into caller buffers: perm[n], slice_ptr[ns + 1], col32[slots],
// val64[slots], and with diag_split the diagonal in SELL order (n).  First call (col32 null):
// sizes only.
void sell_layout_device(const DeviceCsr& csr, int sigma, int chunk, int diag_split, int* n_slices, int64_t* slots,
                        int* d_perm, long long* d_slice_ptr, int* d_width, int* d_col32, double* d_val64,
                        double* d_diag_sell, cudaStream_t st);

// int16 offsets col - row of every slot; false (nothing written) when one is out of range.
bool pack_index16_device(const long long* d_slice_ptr, const int* d_width, int n_slices, int chunk,
                         const int* d_col32, short* d_col16, cudaStream_t st);

// FP64 values to the value type (XPLUS_F32 / BF16 / F16 divided by scale / F64): out[slots].
void convert_device(const double* d_in, int64_t count, int type, double scale, void* d_out, cudaStream_t st);

// Per SELL row i (padding rows 0): diag64[i] = a of row perm[i] (SELL order, FP64), minv[i] =
// 1 / diag64[i], and with row sums rowsum[i] = sum over CSR row perm[i] in CSR order (FP64);
// minv and rowsum converted to the vector type.  diag_csr: the CSR-order diagonal.
void row_vectors_device(const DeviceCsr& csr, const int* d_perm, const double* d_diag_csr, int n_pad, int vtype,
                        double* d_diag64, void* d_minv, void* d_rowsum, cudaStream_t st);

// Shared-memory windows of the SM-resident kernel: block b of `grid` owns slices
// [b per, (b + 1) per); its window covers its rows and every column its slots read, widened to
// multiples of 4 and clipped to n_pad.  Returns {first row, length} per block (host).
std::vector<int2> resident_windows_device(const long long* d_slice_ptr, const int* d_col32, int n_slices, int n_pad,
                                          int grid, cudaStream_t st);

}  // namespace xplus
