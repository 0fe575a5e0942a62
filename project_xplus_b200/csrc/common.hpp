// common.hpp -- error reporting and small helpers shared by the host and CUDA sources.
#pragma once
#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/xplus_b200.h"

namespace xplus {

// Last error text on the calling thread (xplus_last_error_string).
void set_error(const std::string& msg);
const char* last_error();

// An error that maps to an XPLUS_ERR_* code at the C boundary.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Runs f(); converts exceptions to codes and records the message.
template <typename F>
int guarded(F&& f) {
    try {
        f();
        return XPLUS_OK;
    } catch (const Error& e) {
        set_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return XPLUS_ERR_NOMEM;
    } catch (const std::exception& e) {
        set_error(e.what());
        return XPLUS_ERR_ARG;
    }
}

inline void require(bool cond, int code, const std::string& msg) {
    if (!cond) throw Error(code, msg);
}
// The same for a literal message: no string is built unless the check fails (hot host loops).
inline void require(bool cond, int code, const char* msg) {
    if (!cond) throw Error(code, std::string(msg));
}

// Runs f(begin, end) over [0, count) in contiguous chunks on the host's threads (at most 32).
template <typename F>
void parallel_for(int64_t count, F&& f);

// Device-pointer arguments of the entry points that launch on caller memory (*_solve_device,
// *_noalloc): p must be device memory of `device` or managed memory.  Host memory (pageable or
// pinned) and another GPU's memory are rejected with XPLUS_ERR_ARG before anything is launched,
// so a wrong pointer is an error code, not a GPU fault.  (multikernel.cu)
void require_device_memory(const void* p, int device, const char* what);
// Throws XPLUS_ERR_CUDA if earlier asynchronous work left an error pending on this thread.  The
// error is left in place (cudaPeekAtLastError) for its owner, and the calling entry point
// launches nothing, so a later launch check reports only the entry point's own launches.
void require_no_pending_cuda_error(const char* entry);

// CSR structure checks of src/CsrDataset.hpp:29-52, same messages.
void validate_csr(int n, const int* row_ptr, const int* col_idx, int64_t nnz_expected);

// Jacobi diagonal of src/CsrDataset.hpp:92-116 (throws Error(XPLUS_ERR_DATA, ...)).
void jacobi_diag(int n, const int* row_ptr, const int* col_idx, const double* values,
                 double* diag);

struct SellHost {
    int n = 0, n_pad = 0, C = 32, sigma = 1, chunk = 1, diag_split = 0;
    int n_slices = 0;
    int64_t slots = 0;
    std::vector<int> perm;        // perm[new] = old
    std::vector<int> iperm;       // iperm[old] = new
    std::vector<int64_t> slice_ptr;
    std::vector<int> slice_width;
    std::vector<int> col;
    std::vector<double> val;
    std::vector<double> diag;     // only with diag_split (new order)
};

// Stagnation test of the FP64 replacement loop from the options: a replacement is progress when
// ||b - A x||^2 falls below factor x best (factor = (1 - gain)^2); `window` replacements in a
// row without progress stop the solve.
inline void stagnation_args(const xplus_opts& o, double* factor, int* window) {
    const double g = o.stagnation_gain > 0.0 && o.stagnation_gain < 1.0 ? o.stagnation_gain : 0.05;
    *factor = (1.0 - g) * (1.0 - g);
    *window = o.stagnation_window > 0 ? o.stagnation_window : 8;
}

// SELL-C-sigma builder (the single implementation behind xplus_sell_build).
void sell_build(int n, const int* row_ptr, const int* col_idx, const double* values, int C,
                int sigma, int chunk, int diag_split, SellHost& out);
// The same layout built on the current GPU (sell_gpu.cu, bit-identical) and copied back.
void sell_build_via_gpu(int n, const int* row_ptr, const int* col_idx, const double* values, int C,
                        int sigma, int chunk, int diag_split, SellHost& out);

// 16-bit value storage (xplus_opts.split_ratio): a CSR whose selected off-diagonal entries
// appear twice in a row, first the value rounded to the 16-bit type, then the remainder
// a_ij - round(a_ij), exact in FP64, so the two terms sum to a_ij exactly and the second,
// rounded in turn, carries the bits the first lost.  An entry
// (i, j) is selected when row i or row j has sum_k |a_ik| / a_ii above `ratio` (a row whose
// weights of both signs cancel in A, where independent rounding errors of the weights do not
// cancel and can leave the stored operator indefinite) and |a_ij| is above half the smaller of
// a_ii and a_jj (the weights whose errors matter there).  Empty when nothing is selected.
struct TwoTermCsr {
    std::vector<int> row_ptr, col_idx;
    std::vector<double> values;
};
// type XPLUS_BF16 or XPLUS_F16 (FP16 values are stored divided by `scale`)
void two_term_entries(int n, const int* row_ptr, const int* col_idx, const double* values, int type,
                      double scale, double ratio, TwoTermCsr& out);
// FP16 stores a_ij / scale: the power of two that puts the largest off-diagonal |a_ij| just
// below 2^15, inside FP16's range with a ~1e9 dynamic range still normal
double f16_offdiag_scale(int n, const int* row_ptr, const int* col_idx, const double* values);
// the ratio in effect for these options (0: no two-term entries)
double split_ratio_of(const xplus_opts& o);

template <typename F>
void parallel_for(int64_t count, F&& f) {
    const int nt = static_cast<int>(std::max<unsigned>(1u, std::min(32u, std::thread::hardware_concurrency())));
    if (count < 65536 || nt == 1) {
        f(int64_t{0}, count);
        return;
    }
    std::vector<std::thread> pool;
    const int64_t per = (count + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        const int64_t b = t * per, e = std::min(count, b + per);
        if (b < e) pool.emplace_back([&f, b, e] { f(b, e); });
    }
    for (auto& th : pool) th.join();
}

}  // namespace xplus
