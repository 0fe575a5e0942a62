// ref_shim_common.hpp -- TEST INFRASTRUCTURE ONLY (part of the oracle).
// Builds a reference CsrDataset (src/CsrDataset.hpp:17-135) straight from arrays so
// that the reference's own golden and host solvers, compiled from the reference
// sources, can be driven from Python without writing text files.  The reference class
// keeps its arrays private and only fills them in load(); the shim opens the class
// for this translation unit alone.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include <chrono>
#include <queue>
#define private public
#include "CsrDataset.hpp"
#undef private

namespace refshim {
using project_xplus::cgsolver::CsrDataset;

inline CsrDataset make_dataset(int n, const int* row_ptr, const int* col_idx, const double* val,
                               const double* b, const double* x0) {
    CsrDataset d;
    const int nnz = row_ptr[n];
    d.n_ = n;
    d.nnz_ = nnz;
    d.row_ptr_.assign(row_ptr, row_ptr + n + 1);
    d.col_idx_.assign(col_idx, col_idx + nnz);
    d.values_.assign(val, val + nnz);
    d.b_.assign(b, b + n);
    d.x0_.assign(x0, x0 + n);
    return d;
}

inline thread_local std::string last_error;
}  // namespace refshim
