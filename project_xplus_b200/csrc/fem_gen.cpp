// fem_gen.cpp -- synthetic SPD systems: P1 finite-element stiffness matrices of
// -div(k grad u) = f with homogeneous Dirichlet boundary, on jittered structured meshes.
//
//   2D: (g+2) x (g+2) nodes on the unit square, the outer ring is Dirichlet (eliminated),
//       each cell split into two triangles along a random diagonal.  n = g^2, ~7 nnz/row.
//   3D: (g+2)^3 nodes on the unit cube, each cube split into the 6 Kuhn tetrahedra
//       (one per axis permutation; the split is conforming across cubes).  n = g^3,
//       15 nnz/row in the interior.
// Per-element conductivity k = exp(sigma * N(0,1)).  Interior nodes move by U(-j h, j h)
// per coordinate.  All randomness is splitmix64 with one independent stream per purpose:
// 1 = node jitter, 2 = triangle diagonals, 3 = conductivity, 4 = x_true, 5 = permutation.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.hpp"

namespace xplus {

struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
    // Box-Muller, one value per call (the second of the pair is dropped: simpler to restate).
    double normal() {
        const double u1 = 1.0 - uniform();  // (0, 1]
        const double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

inline uint64_t stream_seed(uint64_t seed, uint64_t stream) {
    SplitMix64 m(seed ^ (stream * 0xD1B54A32D192ED03ull));
    m.next();
    return m.next();
}

struct CsrBuild {
    int n = 0;
    std::vector<int> row_ptr, col_idx;
    std::vector<double> values;
};

void rcm_order(int n, const int* row_ptr, const int* col_idx, int* perm);
void permute_symmetric(int n, const int* row_ptr, const int* col_idx, const double* values,
                       const int* perm, std::vector<int>& orp, std::vector<int>& oci,
                       std::vector<double>& ov);

namespace {

// Assembly into a fixed stencil per interior node: slot s of row u is the coupling with
// the neighbour at stencil offset s.  touched marks structural non-zeros.
struct StencilMatrix {
    int n, slots;
    std::vector<double> a;
    std::vector<unsigned char> touched;
    StencilMatrix(int n_, int slots_)
        : n(n_), slots(slots_), a(static_cast<size_t>(n_) * slots_, 0.0),
          touched(static_cast<size_t>(n_) * slots_, 0) {}
    void add(int row, int slot, double v) {
        const size_t k = static_cast<size_t>(row) * slots + slot;
        a[k] += v;
        touched[k] = 1;
    }
};

CsrBuild fem2d(int g, double sigma, double jitter, uint64_t seed) {
    require(g >= 1 && g <= 46340, XPLUS_ERR_ARG, "fem2d: g out of range");
    const int m = g + 2;  // nodes per side incl. boundary
    const double h = 1.0 / (g + 1);
    std::vector<double> X(static_cast<size_t>(m) * m), Y(static_cast<size_t>(m) * m);
    SplitMix64 rj(stream_seed(seed, 1)), rd(stream_seed(seed, 2)), rk(stream_seed(seed, 3));
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            double x = j * h, y = i * h;
            if (i > 0 && i < m - 1 && j > 0 && j < m - 1) {
                x += (2.0 * rj.uniform() - 1.0) * jitter * h;
                y += (2.0 * rj.uniform() - 1.0) * jitter * h;
            }
            X[static_cast<size_t>(i) * m + j] = x;
            Y[static_cast<size_t>(i) * m + j] = y;
        }
    StencilMatrix S(g * g, 9);
    auto unknown = [&](int i, int j) { return (i - 1) * g + (j - 1); };
    auto interior = [&](int i, int j) { return i > 0 && i < m - 1 && j > 0 && j < m - 1; };
    for (int ci = 0; ci < m - 1; ++ci)
        for (int cj = 0; cj < m - 1; ++cj) {
            const int ni[4] = {ci, ci, ci + 1, ci + 1};
            const int nj[4] = {cj, cj + 1, cj, cj + 1};  // a b c d
            const bool flip = (rd.next() >> 63) != 0;
            const int tris[2][3] = {{0, 1, flip ? 3 : 2}, {flip ? 0 : 1, 3, 2}};
            for (int t = 0; t < 2; ++t) {
                const double kappa = std::exp(sigma * rk.normal());
                int vi[3], vj[3];
                double px[3], py[3];
                for (int q = 0; q < 3; ++q) {
                    vi[q] = ni[tris[t][q]];
                    vj[q] = nj[tris[t][q]];
                    px[q] = X[static_cast<size_t>(vi[q]) * m + vj[q]];
                    py[q] = Y[static_cast<size_t>(vi[q]) * m + vj[q]];
                }
                const double det = (px[1] - px[0]) * (py[2] - py[0]) - (px[2] - px[0]) * (py[1] - py[0]);
                const double area = 0.5 * std::fabs(det);
                double gx[3], gy[3];
                for (int q = 0; q < 3; ++q) {
                    const int a1 = (q + 1) % 3, a2 = (q + 2) % 3;
                    gx[q] = (py[a1] - py[a2]) / det;
                    gy[q] = (px[a2] - px[a1]) / det;
                }
                for (int k = 0; k < 3; ++k) {
                    if (!interior(vi[k], vj[k])) continue;
                    const int row = unknown(vi[k], vj[k]);
                    for (int l = 0; l < 3; ++l) {
                        if (!interior(vi[l], vj[l])) continue;
                        const int slot = (vi[l] - vi[k] + 1) * 3 + (vj[l] - vj[k] + 1);
                        S.add(row, slot, kappa * area * (gx[k] * gx[l] + gy[k] * gy[l]));
                    }
                }
            }
        }
    CsrBuild out;
    out.n = g * g;
    out.row_ptr.assign(static_cast<size_t>(out.n) + 1, 0);
    out.col_idx.reserve(static_cast<size_t>(out.n) * 7);
    out.values.reserve(static_cast<size_t>(out.n) * 7);
    for (int i = 1; i <= g; ++i)
        for (int j = 1; j <= g; ++j) {
            const int row = unknown(i, j);
            for (int s = 0; s < 9; ++s) {
                const size_t k = static_cast<size_t>(row) * 9 + s;
                if (!S.touched[k]) continue;
                const int ii = i + s / 3 - 1, jj = j + s % 3 - 1;
                out.col_idx.push_back(unknown(ii, jj));
                out.values.push_back(S.a[k]);
            }
            out.row_ptr[static_cast<size_t>(row) + 1] = static_cast<int>(out.col_idx.size());
        }
    return out;
}

// 3x3 determinant and inverse rows (gradients of the barycentric functions 1..3).
CsrBuild fem3d(int g, double sigma, double jitter, uint64_t seed) {
    require(g >= 1 && g <= 1200, XPLUS_ERR_ARG, "fem3d: g out of range");
    const int m = g + 2;
    const double h = 1.0 / (g + 1);
    const size_t nn = static_cast<size_t>(m) * m * m;
    std::vector<double> P(nn * 3);
    SplitMix64 rj(stream_seed(seed, 1)), rk(stream_seed(seed, 3));
    auto nid = [&](int k, int i, int j) { return (static_cast<size_t>(k) * m + i) * m + j; };
    for (int k = 0; k < m; ++k)
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                double c[3] = {j * h, i * h, k * h};
                if (k > 0 && k < m - 1 && i > 0 && i < m - 1 && j > 0 && j < m - 1)
                    for (int d = 0; d < 3; ++d) c[d] += (2.0 * rj.uniform() - 1.0) * jitter * h;
                for (int d = 0; d < 3; ++d) P[nid(k, i, j) * 3 + d] = c[d];
            }
    const int n = g * g * g;
    StencilMatrix S(n, 27);
    auto interior = [&](int k, int i, int j) {
        return k > 0 && k < m - 1 && i > 0 && i < m - 1 && j > 0 && j < m - 1;
    };
    auto unknown = [&](int k, int i, int j) { return ((k - 1) * g + (i - 1)) * g + (j - 1); };
    static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    for (int ck = 0; ck < m - 1; ++ck)
        for (int ci = 0; ci < m - 1; ++ci)
            for (int cj = 0; cj < m - 1; ++cj)
                for (int t = 0; t < 6; ++t) {
                    const double kappa = std::exp(sigma * rk.normal());
                    int vk[4], vi[4], vj[4];
                    int off[3] = {0, 0, 0};  // x(j), y(i), z(k) offsets
                    for (int q = 0; q < 4; ++q) {
                        if (q > 0) off[perms[t][q - 1]] = 1;
                        vj[q] = cj + off[0];
                        vi[q] = ci + off[1];
                        vk[q] = ck + off[2];
                    }
                    double p[4][3];
                    for (int q = 0; q < 4; ++q)
                        for (int d = 0; d < 3; ++d) p[q][d] = P[nid(vk[q], vi[q], vj[q]) * 3 + d];
                    double J[3][3];  // columns: p1-p0, p2-p0, p3-p0
                    for (int d = 0; d < 3; ++d)
                        for (int c = 0; c < 3; ++c) J[d][c] = p[c + 1][d] - p[0][d];
                    const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                                       J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                                       J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
                    const double vol = std::fabs(det) / 6.0;
                    // rows of J^{-1} = gradients of barycentric functions 1..3
                    double inv[3][3];
                    inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
                    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
                    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
                    inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
                    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
                    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
                    inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
                    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
                    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
                    double gr[4][3];
                    for (int d = 0; d < 3; ++d) {
                        gr[1][d] = inv[0][d];
                        gr[2][d] = inv[1][d];
                        gr[3][d] = inv[2][d];
                        gr[0][d] = -(inv[0][d] + inv[1][d] + inv[2][d]);
                    }
                    for (int a = 0; a < 4; ++a) {
                        if (!interior(vk[a], vi[a], vj[a])) continue;
                        const int row = unknown(vk[a], vi[a], vj[a]);
                        for (int b = 0; b < 4; ++b) {
                            if (!interior(vk[b], vi[b], vj[b])) continue;
                            const int slot = (vk[b] - vk[a] + 1) * 9 + (vi[b] - vi[a] + 1) * 3 +
                                             (vj[b] - vj[a] + 1);
                            const double dotg =
                                gr[a][0] * gr[b][0] + gr[a][1] * gr[b][1] + gr[a][2] * gr[b][2];
                            S.add(row, slot, kappa * vol * dotg);
                        }
                    }
                }
    CsrBuild out;
    out.n = n;
    out.row_ptr.assign(static_cast<size_t>(n) + 1, 0);
    out.col_idx.reserve(static_cast<size_t>(n) * 15);
    out.values.reserve(static_cast<size_t>(n) * 15);
    for (int k = 1; k <= g; ++k)
        for (int i = 1; i <= g; ++i)
            for (int j = 1; j <= g; ++j) {
                const int row = unknown(k, i, j);
                for (int s = 0; s < 27; ++s) {
                    const size_t q = static_cast<size_t>(row) * 27 + s;
                    if (!S.touched[q]) continue;
                    out.col_idx.push_back(unknown(k + s / 9 - 1, i + (s / 3) % 3 - 1, j + s % 3 - 1));
                    out.values.push_back(S.a[q]);
                }
                out.row_ptr[static_cast<size_t>(row) + 1] = static_cast<int>(out.col_idx.size());
            }
    return out;
}

void finish(CsrBuild& A, int64_t perm_seed, int rcm, uint64_t x_seed, int* n, int* nnz,
            int* row_ptr, int* col_idx, double* values, double* b, double* x_true) {
    if (perm_seed >= 0) {
        std::vector<int> perm(static_cast<size_t>(A.n));
        std::iota(perm.begin(), perm.end(), 0);
        SplitMix64 rp(stream_seed(static_cast<uint64_t>(perm_seed), 5));
        for (int i = A.n - 1; i > 0; --i) {
            const int j = static_cast<int>(rp.next() % static_cast<uint64_t>(i + 1));
            std::swap(perm[static_cast<size_t>(i)], perm[static_cast<size_t>(j)]);
        }
        CsrBuild B;
        B.n = A.n;
        permute_symmetric(A.n, A.row_ptr.data(), A.col_idx.data(), A.values.data(), perm.data(),
                          B.row_ptr, B.col_idx, B.values);
        A = std::move(B);
    }
    if (rcm) {
        std::vector<int> perm(static_cast<size_t>(A.n));
        rcm_order(A.n, A.row_ptr.data(), A.col_idx.data(), perm.data());
        CsrBuild B;
        B.n = A.n;
        permute_symmetric(A.n, A.row_ptr.data(), A.col_idx.data(), A.values.data(), perm.data(),
                          B.row_ptr, B.col_idx, B.values);
        A = std::move(B);
    }
    *n = A.n;
    *nnz = A.row_ptr[static_cast<size_t>(A.n)];
    (void)row_ptr; (void)col_idx; (void)values; (void)b; (void)x_true; (void)x_seed;
}

}  // namespace
}  // namespace xplus

using namespace xplus;

namespace {
// The two-phase protocol (size query, then fill) would assemble the system twice; the
// last assembled system is kept per thread and reused when the same parameters return.
struct GenKey {
    int dim, g, rcm;
    double sigma, jitter;
    uint64_t seed, x_seed;
    int64_t perm_seed;
    bool operator==(const GenKey& o) const {
        return dim == o.dim && g == o.g && rcm == o.rcm && sigma == o.sigma && jitter == o.jitter &&
               seed == o.seed && x_seed == o.x_seed && perm_seed == o.perm_seed;
    }
};
thread_local GenKey g_key{-1, 0, 0, 0, 0, 0, 0, 0};
thread_local CsrBuild g_cached;

int generate(const GenKey& key, int* n, int* nnz, int* row_ptr, int* col_idx, double* values,
             double* b, double* x_true) {
    return guarded([&] {
        require(n && nnz, XPLUS_ERR_ARG, "null argument");
        require(!row_ptr || (col_idx && values), XPLUS_ERR_ARG,
                "row_ptr, col_idx and values go together");
        require(key.jitter >= 0.0 && key.jitter < 0.5 && key.sigma >= 0.0, XPLUS_ERR_ARG,
                "fem: bad jitter/sigma");
        if (!(key == g_key)) {
            g_key.dim = -1;
            CsrBuild A = key.dim == 2 ? fem2d(key.g, key.sigma, key.jitter, key.seed)
                                      : fem3d(key.g, key.sigma, key.jitter, key.seed);
            int nn = 0, nz = 0;
            finish(A, key.perm_seed, key.rcm, key.x_seed, &nn, &nz, nullptr, nullptr, nullptr,
                   nullptr, nullptr);
            g_cached = std::move(A);
            g_key = key;
        }
        CsrBuild& A = g_cached;
        *n = A.n;
        *nnz = A.row_ptr[static_cast<size_t>(A.n)];
        if (!row_ptr) return;
        std::memcpy(row_ptr, A.row_ptr.data(), A.row_ptr.size() * sizeof(int));
        std::memcpy(col_idx, A.col_idx.data(), A.col_idx.size() * sizeof(int));
        std::memcpy(values, A.values.data(), A.values.size() * sizeof(double));
        SplitMix64 rx(stream_seed(key.x_seed, 4));
        std::vector<double> xt(static_cast<size_t>(A.n));
        for (auto& v : xt) v = 2.0 * rx.uniform() - 1.0;
        if (x_true) std::memcpy(x_true, xt.data(), xt.size() * sizeof(double));
        if (b)
            for (int row = 0; row < A.n; ++row) {
                double acc = 0.0;
                for (int k = A.row_ptr[static_cast<size_t>(row)];
                     k < A.row_ptr[static_cast<size_t>(row) + 1]; ++k)
                    acc += A.values[static_cast<size_t>(k)] *
                           xt[static_cast<size_t>(A.col_idx[static_cast<size_t>(k)])];
                b[row] = acc;
            }
        // release the cache once the caller has its copy
        g_cached = CsrBuild();
        g_key.dim = -1;
    });
}
}  // namespace

extern "C" {

int xplus_gen_fem2d(int g, double sigma, double jitter, uint64_t seed, int64_t perm_seed, int rcm,
                    uint64_t x_seed, int* n, int* nnz, int* row_ptr, int* col_idx, double* values,
                    double* b, double* x_true) {
    return generate(GenKey{2, g, rcm, sigma, jitter, seed, x_seed, perm_seed}, n, nnz, row_ptr,
                    col_idx, values, b, x_true);
}

int xplus_gen_fem3d(int g, double sigma, double jitter, uint64_t seed, int64_t perm_seed, int rcm,
                    uint64_t x_seed, int* n, int* nnz, int* row_ptr, int* col_idx, double* values,
                    double* b, double* x_true) {
    return generate(GenKey{3, g, rcm, sigma, jitter, seed, x_seed, perm_seed}, n, nnz, row_ptr,
                    col_idx, values, b, x_true);
}

}  // extern "C"
