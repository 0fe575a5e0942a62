// dataset_io.cpp -- the CsrDataset text format (src/CsrDataset.hpp:19-67), a binary cache
// of the same arrays, and the Jacobi diagonal (src/CsrDataset.hpp:92-116).
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>

#include "common.hpp"

namespace xplus {

namespace {
thread_local std::string g_last_error;

// Whole-file read; text parsing below is a strtol/strtod scan (the reference reads with
// operator>>, which accepts the same whitespace-separated decimal tokens).
std::string read_file(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw Error(XPLUS_ERR_IO, "failed to open " + path);
    std::string s;
    std::fseek(f, 0, SEEK_END);
    long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (len > 0) {
        s.resize(static_cast<size_t>(len));
        size_t got = std::fread(&s[0], 1, static_cast<size_t>(len), f);
        s.resize(got);
    }
    std::fclose(f);
    return s;
}

// Parses values until the first token that does not parse (operator>> stops there too).
template <typename T>
std::vector<T> parse_array(const std::string& path) {
    const std::string text = read_file(path);
    std::vector<T> out;
    const char* p = text.c_str();
    const char* end = p + text.size();
    while (p < end) {
        char* q = nullptr;
        if constexpr (std::is_same<T, int>::value) {
            errno = 0;
            long v = std::strtol(p, &q, 10);
            if (q == p || errno == ERANGE || v > std::numeric_limits<int>::max() ||
                v < std::numeric_limits<int>::min())
                break;
            out.push_back(static_cast<int>(v));
        } else {
            double v = std::strtod(p, &q);
            if (q == p) break;
            out.push_back(v);
        }
        p = q;
    }
    if (out.empty()) throw Error(XPLUS_ERR_IO, "empty array file: " + path);
    return out;
}

struct Loaded {
    std::vector<int> row_ptr, col_idx;
    std::vector<double> values, b, x0;
};

Loaded load_text(const std::string& dir) {
    Loaded d;
    const std::string base = dir.empty() || dir.back() == '/' ? dir : dir + "/";
    d.row_ptr = parse_array<int>(base + "row_ptr.txt");
    d.col_idx = parse_array<int>(base + "col_idx.txt");
    d.values = parse_array<double>(base + "values.txt");
    require(d.row_ptr.size() >= 2, XPLUS_ERR_DATA, "row_ptr.txt must contain at least 2 entries");
    const int n = static_cast<int>(d.row_ptr.size()) - 1;
    require(d.values.size() == d.col_idx.size(), XPLUS_ERR_DATA,
            "col_idx.txt and values.txt size mismatch");
    validate_csr(n, d.row_ptr.data(), d.col_idx.data(), static_cast<int64_t>(d.col_idx.size()));
    d.b = parse_array<double>(base + "b.txt");
    d.x0 = parse_array<double>(base + "x0.txt");
    require(static_cast<int>(d.b.size()) == n, XPLUS_ERR_DATA, "b.txt length must equal n");
    require(static_cast<int>(d.x0.size()) == n, XPLUS_ERR_DATA, "x0.txt length must equal n");
    return d;
}

constexpr char kMagic[8] = {'X', 'P', 'C', 'S', 'R', 'B', '0', '1'};
}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

void validate_csr(int n, const int* row_ptr, const int* col_idx, int64_t nnz) {
    require(row_ptr[0] == 0, XPLUS_ERR_DATA, "row_ptr[0] must be 0");
    require(static_cast<int64_t>(row_ptr[n]) == nnz, XPLUS_ERR_DATA, "row_ptr[n] must equal nnz");
    for (int row = 0; row < n; ++row) {
        require(row_ptr[row] <= row_ptr[row + 1], XPLUS_ERR_DATA, "row_ptr must be nondecreasing");
        for (int k = row_ptr[row]; k < row_ptr[row + 1]; ++k)
            require(col_idx[k] >= 0 && col_idx[k] < n, XPLUS_ERR_DATA, "col_idx out of range");
    }
}

void jacobi_diag(int n, const int* row_ptr, const int* col_idx, const double* values,
                 double* diag) {
    for (int row = 0; row < n; ++row) {
        bool found = false;
        diag[row] = 0.0;
        for (int k = row_ptr[row]; k < row_ptr[row + 1]; ++k) {
            if (col_idx[k] == row) {
                diag[row] = values[k];
                found = true;
                break;
            }
        }
        if (!found) throw Error(XPLUS_ERR_DATA, "missing diagonal entry at row " + std::to_string(row));
        if (std::fabs(diag[row]) <= std::numeric_limits<double>::min())
            throw Error(XPLUS_ERR_DATA, "zero diagonal entry at row " + std::to_string(row));
    }
}

}  // namespace xplus

using namespace xplus;

extern "C" {

const char* xplus_last_error_string(void) { return last_error(); }

int xplus_dataset_load_text(const char* dir, int* n, int* nnz, int* row_ptr, int* col_idx,
                            double* values, double* b, double* x0) {
    return guarded([&] {
        require(dir && n && nnz, XPLUS_ERR_ARG, "null argument");
        Loaded d = load_text(dir);
        *n = static_cast<int>(d.row_ptr.size()) - 1;
        *nnz = static_cast<int>(d.col_idx.size());
        if (row_ptr) std::memcpy(row_ptr, d.row_ptr.data(), d.row_ptr.size() * sizeof(int));
        if (col_idx) std::memcpy(col_idx, d.col_idx.data(), d.col_idx.size() * sizeof(int));
        if (values) std::memcpy(values, d.values.data(), d.values.size() * sizeof(double));
        if (b) std::memcpy(b, d.b.data(), d.b.size() * sizeof(double));
        if (x0) std::memcpy(x0, d.x0.data(), d.x0.size() * sizeof(double));
    });
}

int xplus_dataset_save_binary(const char* path, int n, int nnz, const int* row_ptr,
                              const int* col_idx, const double* values, const double* b,
                              const double* x0) {
    return guarded([&] {
        require(path && row_ptr && col_idx && values && b && x0 && n > 0 && nnz >= 0,
                XPLUS_ERR_ARG, "invalid argument");
        validate_csr(n, row_ptr, col_idx, nnz);
        FILE* f = std::fopen(path, "wb");
        require(f != nullptr, XPLUS_ERR_IO, std::string("failed to open ") + path);
        const int64_t hdr[2] = {n, nnz};
        bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(hdr, sizeof(hdr), 1, f) == 1 &&
                  std::fwrite(row_ptr, sizeof(int), static_cast<size_t>(n) + 1, f) == static_cast<size_t>(n) + 1 &&
                  std::fwrite(col_idx, sizeof(int), static_cast<size_t>(nnz), f) == static_cast<size_t>(nnz) &&
                  std::fwrite(values, sizeof(double), static_cast<size_t>(nnz), f) == static_cast<size_t>(nnz) &&
                  std::fwrite(b, sizeof(double), static_cast<size_t>(n), f) == static_cast<size_t>(n) &&
                  std::fwrite(x0, sizeof(double), static_cast<size_t>(n), f) == static_cast<size_t>(n);
        ok = (std::fclose(f) == 0) && ok;
        require(ok, XPLUS_ERR_IO, std::string("short write to ") + path);
    });
}

int xplus_dataset_load_binary(const char* path, int* n, int* nnz, int* row_ptr, int* col_idx,
                              double* values, double* b, double* x0) {
    return guarded([&] {
        require(path && n && nnz, XPLUS_ERR_ARG, "null argument");
        FILE* f = std::fopen(path, "rb");
        require(f != nullptr, XPLUS_ERR_IO, std::string("failed to open ") + path);
        char magic[8];
        int64_t hdr[2];
        bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kMagic, 8) == 0 &&
                  std::fread(hdr, sizeof(hdr), 1, f) == 1 && hdr[0] > 0 && hdr[1] >= 0 &&
                  hdr[0] < (int64_t(1) << 31) && hdr[1] < (int64_t(1) << 31);
        if (!ok) {
            std::fclose(f);
            throw Error(XPLUS_ERR_IO, std::string("not an xplus binary CSR file: ") + path);
        }
        *n = static_cast<int>(hdr[0]);
        *nnz = static_cast<int>(hdr[1]);
        if (!row_ptr) {
            std::fclose(f);
            return;
        }
        if (!(col_idx && values && b && x0)) {
            std::fclose(f);
            throw Error(XPLUS_ERR_ARG, "all five output arrays are required");
        }
        const size_t N = static_cast<size_t>(*n), NZ = static_cast<size_t>(*nnz);
        ok = std::fread(row_ptr, sizeof(int), N + 1, f) == N + 1 &&
             std::fread(col_idx, sizeof(int), NZ, f) == NZ &&
             std::fread(values, sizeof(double), NZ, f) == NZ &&
             std::fread(b, sizeof(double), N, f) == N && std::fread(x0, sizeof(double), N, f) == N;
        std::fclose(f);
        require(ok, XPLUS_ERR_IO, std::string("truncated binary CSR file: ") + path);
        validate_csr(*n, row_ptr, col_idx, *nnz);
    });
}

int xplus_jacobi_diag(int n, const int* row_ptr, const int* col_idx, const double* values,
                      double* diag) {
    return guarded([&] {
        require(n > 0 && row_ptr && col_idx && values && diag, XPLUS_ERR_ARG, "invalid argument");
        jacobi_diag(n, row_ptr, col_idx, values, diag);
    });
}

}  // extern "C"
