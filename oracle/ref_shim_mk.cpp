// ref_shim_mk.cpp -- TEST INFRASTRUCTURE ONLY (part of the oracle).
// C entry points over the reference's golden (src/CgSolverGolden.hpp:42), its loader
// (src/CsrDataset.hpp:19) and its CPU multi-kernel solver
// (archived/host/multi_kernel_solver.hpp:100 + archived/kernels/cg_kernels.cpp),
// all compiled from the reference's own sources by oracle/Makefile.
#include "ref_shim_common.hpp"
#include "CgSolverGolden.hpp"
#include "multi_kernel_solver.hpp"

using namespace project_xplus::cgsolver;

extern "C" {

const char* ref_last_error(void) { return refshim::last_error.c_str(); }

// Golden Jacobi-PCG.  trace: [max_iters][5] alpha,beta,rz,rr,residual (nullable).
// Returns 0, or 1 when the reference threw (message in ref_last_error()).
int ref_golden(int n, const int* row_ptr, const int* col_idx, const double* val,
               const double* b, const double* x0, double tau, int max_iters, double* x,
               int* iterations, double* final_rr, int* converged, double* trace,
               double* residual_l2) {
    try {
        const CsrDataset d = refshim::make_dataset(n, row_ptr, col_idx, val, b, x0);
        SolverConfig cfg;
        cfg.tau = tau;
        cfg.max_iters = max_iters;
        const GoldenResult res = run_jacobi_pcg(d, cfg);
        std::copy(res.solution.begin(), res.solution.end(), x);
        *iterations = res.iterations;
        *final_rr = res.final_rr;
        *converged = res.converged ? 1 : 0;
        if (trace) {
            for (std::size_t i = 0; i < res.iteration_trace.size(); ++i) {
                const auto& t = res.iteration_trace[i];
                trace[5 * i + 0] = t.alpha;
                trace[5 * i + 1] = t.beta;
                trace[5 * i + 2] = t.rz;
                trace[5 * i + 3] = t.rr;
                trace[5 * i + 4] = t.residual;
            }
        }
        if (residual_l2) *residual_l2 = compute_residual_norm(d, res.solution);
        return 0;
    } catch (const std::exception& e) {
        refshim::last_error = e.what();
        return 1;
    }
}

// CsrDataset::load on a directory of the five text files; copies out the arrays.
// Call once with null outputs to get n and nnz, then again with buffers.
int ref_load(const char* dir, int* n, int* nnz, int* row_ptr, int* col_idx, double* val,
             double* b, double* x0) {
    try {
        const CsrDataset d = CsrDataset::load(dir);
        *n = d.n();
        *nnz = d.nnz();
        if (row_ptr) std::copy(d.row_ptr().begin(), d.row_ptr().end(), row_ptr);
        if (col_idx) std::copy(d.col_idx().begin(), d.col_idx().end(), col_idx);
        if (val) std::copy(d.values().begin(), d.values().end(), val);
        if (b) std::copy(d.b().begin(), d.b().end(), b);
        if (x0) std::copy(d.x0().begin(), d.x0().end(), x0);
        return 0;
    } catch (const std::exception& e) {
        refshim::last_error = e.what();
        return 1;
    }
}

// Reference jacobi diagonal (throws on missing/zero diagonal -> returns 1).
int ref_jacobi_diag(int n, const int* row_ptr, const int* col_idx, const double* val,
                    double* diag) {
    try {
        std::vector<double> zero(static_cast<std::size_t>(n), 0.0);
        const CsrDataset d = refshim::make_dataset(n, row_ptr, col_idx, val, zero.data(), zero.data());
        const auto dg = d.extract_jacobi_diag();
        std::copy(dg.begin(), dg.end(), diag);
        return 0;
    } catch (const std::exception& e) {
        refshim::last_error = e.what();
        return 1;
    }
}

// The CPU multi-kernel Jacobi-PCG.  The reference rejects n > kMaxN (1024) with an
// exception; that is reported as return code 1.  trace as in ref_golden (the [iter] line).
int ref_multi_kernel(int n, const int* row_ptr, const int* col_idx, const double* val,
                     const double* b, const double* x0, double tau, int max_iters, double* x,
                     int* iterations, double* final_rr, int* status, double* residual_l2,
                     double* trace) {
    try {
        const CsrDataset d = refshim::make_dataset(n, row_ptr, col_idx, val, b, x0);
        SolverConfig cfg;
        cfg.tau = tau;
        cfg.max_iters = max_iters;
        std::ostringstream log;
        const MultiKernelResult res = run_local_multi_kernel_solver(d, cfg, trace ? &log : nullptr);
        std::copy(res.solution.begin(), res.solution.end(), x);
        *iterations = res.iterations;
        *final_rr = res.final_rr;
        *status = static_cast<int>(res.status);
        *residual_l2 = res.residual_l2;
        if (trace) {
            std::istringstream in(log.str());
            std::string line;
            int k = 0;
            while (std::getline(in, line)) {
                if (line.rfind("[iter", 0) != 0) continue;
                double a, bb, rz, rr, res_;
                const char* s = std::strstr(line.c_str(), "alpha=");
                if (!s || std::sscanf(s, "alpha=%lf beta=%lf rz=%lf rr=%lf residual=%lf", &a, &bb,
                                      &rz, &rr, &res_) != 5) continue;
                trace[5 * k + 0] = a; trace[5 * k + 1] = bb; trace[5 * k + 2] = rz;
                trace[5 * k + 3] = rr; trace[5 * k + 4] = res_;
                ++k;
            }
        }
        return 0;
    } catch (const std::exception& e) {
        refshim::last_error = e.what();
        return 1;
    }
}

// Reference multi-kernel "kernel functions" (archived/include/cg_kernels.hpp:9-54),
// re-exported under ref_ names so tests can call them beside the GPU ones.
void ref_spmv_csr_kernel(const int* rp, const int* ci, const double* v, const double* x, double* y,
                         int n) { spmv_csr_kernel(rp, ci, v, x, y, n); }
void ref_init_pcg_kernel(const double* b, const double* ax, const double* m_inv, double* r,
                         double* z, double* p, double* metrics, int n) {
    init_pcg_kernel(b, ax, m_inv, r, z, p, metrics, n);
}
void ref_dot_kernel(const double* a, const double* b, double* out, int n) { dot_kernel(a, b, out, n); }
void ref_update_xrz_kernel(double* x, const double* p, double* r, const double* ap,
                           const double* m_inv, double* z, double* metrics, double alpha, int n) {
    update_xrz_kernel(x, p, r, ap, m_inv, z, metrics, alpha, n);
}
void ref_update_p_kernel(const double* z, double* p, double beta, int n) { update_p_kernel(z, p, beta, n); }

}  // extern "C"
