// pcg_kernels.cuh -- launch interface of the persistent Jacobi-PCG kernel and the SELL SpMV.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace xplus {

// Device-side outcome of one persistent solve (written by block 0 at exit).
struct PcgOut {
    int status;        // XPLUS_CONVERGED .. XPLUS_BREAKDOWN (XPLUS_TIMEOUT is set by the host)
    int iterations;
    int replacements;
    int stagnated;
    double rz, rr, pap, alpha;
    double true_rr;    // ||b - A x||^2 in FP64 at exit
    double reserved;   // GTG kernel: iteration at which it fell back to Jacobi (-1: never)
    double bb;         // ||b||^2 in FP64, summed by the kernel in its first residual pass
    long long t_start_ns, t_end_ns;
    long long t_phase[4];  // block 0: phase A work, barrier wait, phase B work, barrier wait (ns)
};

// Matrix + vectors + control of one persistent solve.  All vectors are in SELL order and
// n_pad long; padding rows hold zeros and stay zero.
struct PcgArgs {
    int n, n_pad, n_slices;
    const long long* slice_ptr;
    const void* col;        // int32 columns or int16 row offsets (KernelKey::idx16)
    const void* val;        // VT, slots
    float val_scale;        // stored off-diagonal values are a_ij / val_scale (1 except FP16)
    const double* val64;    // FP64 copy in the same layout (nullable)
    const void* rowsum;     // XT, n_pad: row sums s_i = sum_j a_ij (row-sum form only)
    const double* diag64;   // FP64 diagonal when the slots hold off-diagonals only
    const void* minv;       // XT, n_pad
    const double* b64;
    double* x64;            // FP64 solution accumulator (x0 on entry)
    void* rec;              // n_pad node records {z, p} of the vector type
    void* r;                // XT
    void* ap;               // XT
    // optional M^-1 = G^T G (G and its transpose in SELL form over the same ordering)
    const long long* g_slice_ptr; const int* g_col; const void* g_val;
    const long long* gt_slice_ptr; const int* gt_col; const void* gt_val;
    void* t;                // XT, n_pad: G r temporary
    void* z;                // XT, n_pad: preconditioned residual (GTG mode only)
    double* partial;        // 2 banks x 4 slots x gridDim.x
    unsigned* bar;
    int* err;
    PcgOut* out;
    double* trace;          // [trace_cap][5] alpha, beta, rz, rr, sqrt(rr) (nullable)
    int trace_cap;
    double tau_rr;          // stop when recurrence rr <= tau_rr (abs mode)
    double tau_true_rr;     // >= 0: FP64 true-residual mode, stop when ||b-Ax||^2 <= this
    double tau2_rel;        // > 0: relative true-residual mode; the kernel replaces tau_true_rr
                            // by tau2_rel * ||b||^2, ||b||^2 summed with the first residual
    int max_iters;
    int replace_every;
    double replace_drop;    // rr ratio that triggers a replacement (0: off)
    int restart_on_replace; // after a replacement beta = 0: 1 always, 2 only when drop- or convergence-triggered
    double stag_factor;     // a replacement counts as progress when ||b-Ax||^2 < stag_factor * best
    int stag_window;        // replacements without progress that stop the solve
    long long timeout_ns;
    int debug_skip_block;   // test-only fault injection: block that skips its first arrival
    // SM-resident kernel only: per-CTA shared window {first row, rows} of the search direction,
    // and how often the FP32 solution increments are folded into x64
    const int2* win;
    int flush_every;
    long long* block_clk;   // [gridDim.x][4] phase clock of every CTA (ns)
    // GTG kernel only: second residual buffer (XT, n_pad) and the iteration cap after which the
    // learned preconditioner gives way to Jacobi (0: only on stagnation)
    void* r2;
    int g_fallback_iters;
};

struct SpmvArgs {
    int n_pad, n_slices;
    const long long* slice_ptr;
    const void* col;
    const void* val;
    const void* rowsum;     // row-sum form only
    float val_scale;
};

// vt: XPLUS_F32/BF16/F64 ; xt: XPLUS_F32/F64 ; chunk 1/2/4 ; diag = row-sum form ; gtg
// preconditioner ; idx16 = int16 column offsets
struct KernelKey {
    int vt, xt, chunk, diag, gtg, idx16;
};

// Occupancy-derived cooperative grid for the persistent kernel (blocks, threads).
cudaError_t pcg_grid(const KernelKey& k, int device, int n_slices, int want_tpb, int want_bps,
                     int* grid, int* tpb);
// window: L2 access-policy window for the matrix stream (num_bytes 0 = none)
cudaError_t pcg_launch(const KernelKey& k, const PcgArgs& a, int grid, int tpb, cudaStream_t s,
                       const cudaAccessPolicyWindow& window);
// SM-resident variant (pcg_resident.cu): FP32 vectors in the row-sum form only.
bool resident_supported(const KernelKey& k);
int resident_max_slices();
// Sets the dynamic shared-memory opt-in and reports whether one CTA per SM fits.
// one_sync: the one-barrier-per-iteration kernel (records {m r, m Ap, p} x 2 generations).
cudaError_t resident_prepare(const KernelKey& k, int device, size_t smem_bytes, int tpb, bool one_sync,
                             bool* fits);
cudaError_t resident_launch(const KernelKey& k, const PcgArgs& a, int grid, int tpb, size_t smem_bytes,
                            bool one_sync, cudaStream_t s, const cudaAccessPolicyWindow& window);
// GTG-preconditioned persistent kernel (pcg_gtg.cu): FP32 vectors, row-sum form, M^-1 = G^T G
// with G and G^T in SELL form (FP32 values, int32 columns, chunk 2) over the matrix's ordering.
cudaError_t gtg_grid(const KernelKey& k, int device, int n_slices, int* grid, int* tpb);
cudaError_t gtg_launch(const KernelKey& k, const PcgArgs& a, int grid, int tpb, cudaStream_t s,
                       const cudaAccessPolicyWindow& window);
// val[q] = glow[map[q]] (0 where map[q] < 0): G values into a SELL image of G or G^T
cudaError_t gtg_fill_values(const double* d_glow, const int* d_map, float* d_val, long long slots, cudaStream_t s);
cudaError_t spmv_launch(const KernelKey& k, const SpmvArgs& a, const void* x, void* y,
                        cudaStream_t s);
// dst[i] = (T) src[perm[i]] for i < n, 0 for n <= i < n_pad   (T per xt; f64 when xt==F64)
cudaError_t gather_to_sell(int xt, const double* src, void* dst, const int* perm, int n, int n_pad,
                           cudaStream_t s);
// dst[perm[i]] = src[i]
cudaError_t scatter_from_sell(const double* src, double* dst, const int* perm, int n,
                              cudaStream_t s);

}  // namespace xplus
