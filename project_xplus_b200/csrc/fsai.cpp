// fsai.cpp -- exact factorized sparse approximate inverse on A's lower pattern (host).
//
// The non-learned counterpart of the network's G (Kolotilina & Yeremin, "Factorized sparse
// approximate inverse preconditionings I", 1993): row i of G solves A[P_i, P_i] g = e_i over
// P_i = {j <= i : a_ij != 0} and is scaled so that (G A G^T)_ii = 1.  Each row is one small
// dense SPD solve (Cholesky).  Output in A's CSR order of the entries with col <= row, the
// layout xplus_pcg_set_gtg takes.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.hpp"

namespace xplus {
namespace {

void fsai_lower(int n, const int* row_ptr, const int* col_idx, const double* values, double* g_low) {
    require(n > 0 && row_ptr && col_idx && values && g_low, XPLUS_ERR_ARG, "null argument");
    validate_csr(n, row_ptr, col_idx, row_ptr[n]);
    int64_t out = 0;
    std::vector<int> pat;
    std::vector<double> M, y;
    for (int i = 0; i < n; ++i) {
        pat.clear();
        for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q)
            if (col_idx[q] <= i) pat.push_back(col_idx[q]);
        const int m = static_cast<int>(pat.size());
        require(m > 0 && std::find(pat.begin(), pat.end(), i) != pat.end(), XPLUS_ERR_DATA,
                "missing diagonal entry while building the factorized approximate inverse");
        // A[P, P] (dense, m x m): entries looked up in the CSR rows of the pattern
        M.assign(static_cast<size_t>(m) * m, 0.0);
        for (int a = 0; a < m; ++a) {
            const int ra = pat[static_cast<size_t>(a)];
            for (int q = row_ptr[ra]; q < row_ptr[ra + 1]; ++q)
                for (int b = 0; b < m; ++b)
                    if (col_idx[q] == pat[static_cast<size_t>(b)]) M[static_cast<size_t>(a) * m + b] += values[q];
        }
        // Cholesky M = L L^T (in place, lower part)
        for (int c = 0; c < m; ++c) {
            double d = M[static_cast<size_t>(c) * m + c];
            for (int k = 0; k < c; ++k) d -= M[static_cast<size_t>(c) * m + k] * M[static_cast<size_t>(c) * m + k];
            require(d > 0.0, XPLUS_ERR_DATA, "local matrix not positive definite (A is not SPD)");
            const double l = std::sqrt(d);
            M[static_cast<size_t>(c) * m + c] = l;
            for (int r = c + 1; r < m; ++r) {
                double v = M[static_cast<size_t>(r) * m + c];
                for (int k = 0; k < c; ++k) v -= M[static_cast<size_t>(r) * m + k] * M[static_cast<size_t>(c) * m + k];
                M[static_cast<size_t>(r) * m + c] = v / l;
            }
        }
        // solve L L^T y = e_i (position of i in the pattern)
        y.assign(static_cast<size_t>(m), 0.0);
        for (int a = 0; a < m; ++a) y[static_cast<size_t>(a)] = pat[static_cast<size_t>(a)] == i ? 1.0 : 0.0;
        for (int r = 0; r < m; ++r) {
            double v = y[static_cast<size_t>(r)];
            for (int k = 0; k < r; ++k) v -= M[static_cast<size_t>(r) * m + k] * y[static_cast<size_t>(k)];
            y[static_cast<size_t>(r)] = v / M[static_cast<size_t>(r) * m + r];
        }
        for (int r = m - 1; r >= 0; --r) {
            double v = y[static_cast<size_t>(r)];
            for (int k = r + 1; k < m; ++k) v -= M[static_cast<size_t>(k) * m + r] * y[static_cast<size_t>(k)];
            y[static_cast<size_t>(r)] = v / M[static_cast<size_t>(r) * m + r];
        }
        double yii = 0.0;
        for (int a = 0; a < m; ++a)
            if (pat[static_cast<size_t>(a)] == i) yii = y[static_cast<size_t>(a)];
        require(yii > 0.0, XPLUS_ERR_DATA, "factorized approximate inverse: non-positive pivot");
        const double sc = 1.0 / std::sqrt(yii);
        for (int a = 0; a < m; ++a) g_low[out++] = y[static_cast<size_t>(a)] * sc;
    }
}

}  // namespace
}  // namespace xplus

extern "C" int xplus_fsai_lower(int n, const int* row_ptr, const int* col_idx, const double* values, double* g_low) {
    return xplus::guarded([&] { xplus::fsai_lower(n, row_ptr, col_idx, values, g_low); });
}
