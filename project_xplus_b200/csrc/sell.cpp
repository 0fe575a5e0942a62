// sell.cpp -- SELL-C-sigma construction (host side; the product's only builder).
//
// Layout (restated by oracle/sell_rcm_oracle.py, bit-exact):
//   * row lengths len[i] (minus the diagonal when diag_split);
//   * sigma-sort: inside each window of sigma consecutive rows, rows are ordered by
//     decreasing len, ties by increasing original index (stable); perm[new] = old;
//   * n_pad = ceil(n / C) * C rows in n_slices = n_pad / C slices of C rows;
//   * width[s] = max len in slice s rounded up to a multiple of `chunk`;
//     slice_ptr[s+1] = slice_ptr[s] + width[s] * C;
//   * entry j of the row in lane l of slice s (CSR order, diagonal skipped when split)
//     sits at slice_ptr[s] + (j / chunk) * C * chunk + l * chunk + (j % chunk), so one
//     warp reads C * chunk consecutive slots per step and each lane's `chunk` entries are
//     contiguous (one 8/16-byte load);
//   * columns are renumbered by the same permutation (y and x live in the new order);
//   * padding slots hold col = own (new) row and value 0.
#include <algorithm>
#include <numeric>
#include <vector>

#include "common.hpp"

namespace xplus {

void sell_build(int n, const int* row_ptr, const int* col_idx, const double* values, int C,
                int sigma, int chunk, int diag_split, SellHost& S) {
    require(n > 0, XPLUS_ERR_ARG, "sell: n must be positive");
    require(C > 0 && C <= 1024, XPLUS_ERR_ARG, "sell: bad slice height");
    require(chunk == 1 || chunk == 2 || chunk == 4 || chunk == 8, XPLUS_ERR_ARG, "sell: chunk must be 1, 2, 4 or 8");
    require(sigma >= 1, XPLUS_ERR_ARG, "sell: sigma must be >= 1");
    S.n = n;
    S.C = C;
    S.sigma = sigma;
    S.chunk = chunk;
    S.diag_split = diag_split;
    std::vector<int> len(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) {
        int l = row_ptr[i + 1] - row_ptr[i];
        if (diag_split)
            for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
                if (col_idx[k] == i) {
                    --l;
                    break;
                }
        len[static_cast<size_t>(i)] = l;
    }
    S.perm.resize(static_cast<size_t>(n));
    std::iota(S.perm.begin(), S.perm.end(), 0);
    if (sigma > 1)
        for (int w0 = 0; w0 < n; w0 += sigma) {
            const int w1 = std::min(n, w0 + sigma);
            std::stable_sort(S.perm.begin() + w0, S.perm.begin() + w1, [&](int a, int b) {
                return len[static_cast<size_t>(a)] > len[static_cast<size_t>(b)];
            });
        }
    S.iperm.resize(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) S.iperm[static_cast<size_t>(S.perm[static_cast<size_t>(i)])] = i;
    S.n_slices = (n + C - 1) / C;
    S.n_pad = S.n_slices * C;
    S.slice_ptr.assign(static_cast<size_t>(S.n_slices) + 1, 0);
    S.slice_width.assign(static_cast<size_t>(S.n_slices), 0);
    for (int s = 0; s < S.n_slices; ++s) {
        int w = 0;
        for (int l = 0; l < C; ++l) {
            const int i = s * C + l;
            if (i < n) w = std::max(w, len[static_cast<size_t>(S.perm[static_cast<size_t>(i)])]);
        }
        w = (w + chunk - 1) / chunk * chunk;
        S.slice_width[static_cast<size_t>(s)] = w;
        S.slice_ptr[static_cast<size_t>(s) + 1] = S.slice_ptr[static_cast<size_t>(s)] + static_cast<int64_t>(w) * C;
    }
    S.slots = S.slice_ptr[static_cast<size_t>(S.n_slices)];
    S.col.assign(static_cast<size_t>(S.slots), 0);
    S.val.assign(static_cast<size_t>(S.slots), 0.0);
    if (diag_split) S.diag.assign(static_cast<size_t>(S.n_pad), 0.0);
    for (int s = 0; s < S.n_slices; ++s) {
        const int64_t base = S.slice_ptr[static_cast<size_t>(s)];
        const int w = S.slice_width[static_cast<size_t>(s)];
        for (int l = 0; l < C; ++l) {
            const int i = s * C + l;
            int j = 0;
            if (i < n) {
                const int old = S.perm[static_cast<size_t>(i)];
                bool diag_taken = false;
                for (int k = row_ptr[old]; k < row_ptr[old + 1]; ++k) {
                    if (diag_split && !diag_taken && col_idx[k] == old) {
                        S.diag[static_cast<size_t>(i)] = values[k];
                        diag_taken = true;
                        continue;
                    }
                    const int64_t pos = base + static_cast<int64_t>(j / chunk) * C * chunk + l * chunk + (j % chunk);
                    S.col[static_cast<size_t>(pos)] = S.iperm[static_cast<size_t>(col_idx[k])];
                    S.val[static_cast<size_t>(pos)] = values[k];
                    ++j;
                }
            }
            for (; j < w; ++j) {
                const int64_t pos = base + static_cast<int64_t>(j / chunk) * C * chunk + l * chunk + (j % chunk);
                S.col[static_cast<size_t>(pos)] = i;
                S.val[static_cast<size_t>(pos)] = 0.0;
            }
        }
    }
}

}  // namespace xplus

using namespace xplus;

extern "C" {

int xplus_sell_build(int n, const int* row_ptr, const int* col_idx, const double* values, int C,
                     int sigma, int chunk, int diag_split, int* n_slices, int64_t* slots,
                     int* perm, int64_t* slice_ptr, int* slice_width, int* col, double* val,
                     double* diag) {
    return guarded([&] {
        require(n > 0 && row_ptr && col_idx && values && n_slices && slots, XPLUS_ERR_ARG, "invalid argument");
        validate_csr(n, row_ptr, col_idx, row_ptr[n]);
        SellHost S;
        sell_build(n, row_ptr, col_idx, values, C, sigma, chunk, diag_split, S);
        *n_slices = S.n_slices;
        *slots = S.slots;
        if (perm) std::copy(S.perm.begin(), S.perm.end(), perm);
        if (slice_ptr) std::copy(S.slice_ptr.begin(), S.slice_ptr.end(), slice_ptr);
        if (slice_width) std::copy(S.slice_width.begin(), S.slice_width.end(), slice_width);
        if (col) std::copy(S.col.begin(), S.col.end(), col);
        if (val) std::copy(S.val.begin(), S.val.end(), val);
        if (diag && diag_split) std::copy(S.diag.begin(), S.diag.begin() + n, diag);
    });
}

}  // extern "C"
