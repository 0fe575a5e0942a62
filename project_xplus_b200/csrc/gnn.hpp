// gnn.hpp -- internal interface of the learned-preconditioner network (gnn.cu): parameter
// layout, graph arrays, workspace and the forward / loss-backward / Adam launches.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace xplus {
namespace gnn {

constexpr int kHidden = 32;
constexpr int kLayers = 3;

// Offsets of every parameter block in the flat parameter vector (floats).
struct ParamOffsets {
    int W0, b0;
    int Wa[kLayers], ba[kLayers], Wl[kLayers], Wu[kLayers];
    int P, bp, Q, c, c2, w, bw, wd, bwd;
    int total;
};
ParamOffsets param_offsets();

// Graph arrays of one system in its own row order (host side).
struct HostGraph {
    int n = 0, n_adj = 0, n_low = 0, n_glow = 0;
    std::vector<int> adj_ptr, adj_col;   // off-diagonal neighbours, ascending columns
    std::vector<float> adj_e;            // a_ij / sqrt(a_ii a_jj)
    std::vector<int> low_ptr, low_col, low_row;  // strictly lower edges by row (k index)
    std::vector<float> low_e;
    std::vector<float> low_f;                    // sum_{m < i, m != j} e_jm e_mi per lower edge
    std::vector<int> up_ptr, up_k, up_row;       // lower edges grouped by column
    std::vector<int> a_ptr, a_col;               // A (all entries, FP32) for the probe loss
    std::vector<float> a_val;
    std::vector<float> x, isq;                   // node inputs [n][2], 1/sqrt(a_ii)
    std::vector<int> pos_low, pos_diag;          // G entry -> position among A's entries with col <= row
    void build(int n, const int* row_ptr, const int* col_idx, const double* values);
};

// Device allocations owned by one object, freed together.
struct Arena {
    std::vector<void*> ptrs;
    void* raw(size_t bytes);
    template <typename T>
    T* get(size_t count) { return static_cast<T*>(raw(count * sizeof(T))); }
    void release();
};

struct DevGraph {
    int n = 0, n_adj = 0, n_low = 0, n_glow = 0;
    int *adj_ptr = nullptr, *adj_col = nullptr, *low_ptr = nullptr, *low_col = nullptr, *low_row = nullptr;
    int *up_ptr = nullptr, *up_k = nullptr, *up_row = nullptr, *a_ptr = nullptr, *a_col = nullptr;
    int *pos_low = nullptr, *pos_diag = nullptr;
    float *adj_e = nullptr, *low_e = nullptr, *low_f = nullptr, *a_val = nullptr, *x = nullptr, *isq = nullptr;
    void upload(const HostGraph& g, Arena& ar, cudaStream_t st);
    // The arrays inference needs (adjacency, lower edges with e and f, node inputs, 1/sqrt(a_ii),
    // g_low positions), built on the GPU from a device CSR; the host CSR only supplies the host
    // builder's error message when the diagonal is not positive or repeated.
    void build_on_device(int n, const int* d_rp, const int* d_ci, const double* d_v, const int* row_ptr,
                         const int* col_idx, const double* values, Arena& ar, cudaStream_t st);
};

// Activations and temporaries, sized for the largest system.
constexpr int kLossProbe = 0;    // sum ||G A G^T v - v||^2 / (K n) over K probes
constexpr int kLossKaporin = 1;  // (1/n) sum_i [log (G A G^T)_ii - 2 log Ghat_ii]

struct Work {
    int K = 0;
    int loss_kind = kLossProbe;
    float* h[kLayers + 1] = {};
    float* s[kLayers] = {};
    float *a = nullptr, *hl = nullptr, *hu = nullptr, *ph = nullptr, *qh = nullptr;
    float *gval = nullptr, *gdiag = nullptr;           // G values (lower edges, diagonal)
    float *zpre = nullptr, *go = nullptr, *gd = nullptr, *td = nullptr;  // Ghat lower, Ghat_ii, log Ghat_ii
    int* bad = nullptr;
    float *v = nullptr, *w1 = nullptr, *w2 = nullptr, *r = nullptr, *t = nullptr, *y = nullptr;
    float *dgo = nullptr, *dexp = nullptr;
    float *dh = nullptr, *dh2 = nullptr, *ds = nullptr, *dhl = nullptr, *dhu = nullptr, *dph = nullptr, *dqh = nullptr;
    float* partial = nullptr;
    double* dpartial = nullptr;
    double* loss = nullptr;
    void alloc(Arena& ar, int max_n, int max_low, int K, bool train);
};

// wr: parameters rounded to BF16 (as floats).  train keeps what the backward pass needs.
void forward(const DevGraph& g, const float* wr, Work& w, bool train, cudaStream_t st);
// G values into A's CSR order of the entries with col <= row (FP64 device array, n_glow long).
void g_to_low(const DevGraph& g, const Work& w, double* d_glow, cudaStream_t st);
// `sweeps` Gauss-Seidel sweeps over each row of the predicted Ghat (w.go, w.gval) on the row's
// quadratic form g^T A^[P_i, P_i] g at fixed Ghat_ii: every row's Kaporin term decreases.
void refine_rows(const DevGraph& g, Work& w, int sweeps, cudaStream_t st);
// Rows of the predicted G (w.gval, w.gdiag) scaled to (G A G^T)_ii = 1; waits for the stream.
void normalize_rows(const DevGraph& g, Work& w, cudaStream_t st);
// The loss w.loss_kind selects (into w.loss) and, when grad != nullptr, its gradient with
// respect to wr.  seed draws the probes of the probe loss.
void loss_backward(const DevGraph& g, const float* wr, Work& w, float* grad, unsigned long long seed, cudaStream_t st);
void backward_from_dg(const DevGraph& g, const float* wr, Work& w, float* grad, cudaStream_t st);
void adam_step(float* theta, const float* grad, float* m, float* v, int P, float lr, int step, cudaStream_t st);
void round_params(const float* master, float* wr, int P, cudaStream_t st);

}  // namespace gnn
}  // namespace xplus
