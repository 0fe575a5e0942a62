// ref_shim_cuper.cpp -- TEST INFRASTRUCTURE ONLY (part of the oracle).
// C entry points over the reference's Cuper software PCG (host/cuper_pcg_solver.hpp:311),
// its Cuper-style SpMV (:136), its 16-channel packer (host/cuper_control_matrix.hpp:130)
// and the single-launch control kernel compiled as plain C++
// (kernels/cuper_pcg_control_kernel.cpp:972), all from the reference's own sources.
#include "ref_shim_common.hpp"
#include "cuper_pcg_solver.hpp"
#include "cuper_control_matrix.hpp"

using namespace project_xplus::cgsolver;

extern "C" {
void cuper_pcg_control_kernel(const int* sp_element_list_ptr, const unsigned long* m0,
                              const unsigned long* m1, const unsigned long* m2,
                              const unsigned long* m3, const unsigned long* m4,
                              const unsigned long* m5, const unsigned long* m6,
                              const unsigned long* m7, const unsigned long* m8,
                              const unsigned long* m9, const unsigned long* m10,
                              const unsigned long* m11, const unsigned long* m12,
                              const unsigned long* m13, const unsigned long* m14,
                              const unsigned long* m15, const double* b, const double* m_inv,
                              double* x, double* r, double* z, double* p, double* ap,
                              double* metrics, int* status, double tau, int max_iters, int n,
                              int batch_count);

const char* ref_cuper_last_error(void) { return refshim::last_error.c_str(); }

// run_cuper_pcg_solver.  timing_ms: {plan_ms, spmv_ms, spmv_calls}.
int ref_cuper_pcg(int n, const int* row_ptr, const int* col_idx, const double* val,
                  const double* b, const double* x0, double tau, int max_iters, double* x,
                  int* iterations, double* final_rr, int* status, double* residual_l2,
                  double* timing_ms) {
    try {
        const CsrDataset d = refshim::make_dataset(n, row_ptr, col_idx, val, b, x0);
        SolverConfig cfg;
        cfg.tau = tau;
        cfg.max_iters = max_iters;
        const CuperPcgResult res = run_cuper_pcg_solver(d, cfg, nullptr);
        std::copy(res.solution.begin(), res.solution.end(), x);
        *iterations = res.iterations;
        *final_rr = res.final_rr;
        *status = static_cast<int>(res.status);
        *residual_l2 = res.residual_l2;
        if (timing_ms) {
            timing_ms[0] = res.timing.plan_ms;
            timing_ms[1] = res.timing.spmv_ms;
            timing_ms[2] = res.timing.spmv_calls;
        }
        return 0;
    } catch (const std::exception& e) {
        refshim::last_error = e.what();
        return 1;
    }
}

// One cuper_style_spmv call (plan built each call).
int ref_cuper_spmv(int n, const int* row_ptr, const int* col_idx, const double* val,
                   const double* x, double* y) {
    try {
        std::vector<double> zero(static_cast<std::size_t>(n), 0.0);
        const CsrDataset d = refshim::make_dataset(n, row_ptr, col_idx, val, zero.data(), zero.data());
        const auto plan = build_cuper_matrix_plan(d);
        std::vector<double> xin(x, x + n), yout;
        cuper_style_spmv(plan, xin, yout);
        std::copy(yout.begin(), yout.end(), y);
        return 0;
    } catch (const std::exception& e) {
        refshim::last_error = e.what();
        return 1;
    }
}

// Packed 16-channel control matrix.  Query sizes with words == nullptr:
// *batch_count, *matrix_len, *channel_words.  Then fill ptr[batch_count+1] and
// words[16][channel_words].
int ref_cuper_pack(int n, const int* row_ptr, const int* col_idx, const double* val,
                   int* batch_count, int* matrix_len, int* channel_words, int* ptr,
                   unsigned long long* words) {
    try {
        std::vector<double> zero(static_cast<std::size_t>(n), 0.0);
        const CsrDataset d = refshim::make_dataset(n, row_ptr, col_idx, val, zero.data(), zero.data());
        const CuperControlMatrix m = build_cuper_control_matrix(d);
        *batch_count = m.batch_count;
        *matrix_len = m.matrix_len;
        *channel_words = static_cast<int>(m.matrix_data[0].size());
        if (ptr) std::copy(m.sp_element_list_ptr.begin(), m.sp_element_list_ptr.end(), ptr);
        if (words) {
            for (int c = 0; c < 16; ++c)
                for (std::size_t k = 0; k < m.matrix_data[c].size(); ++k)
                    words[static_cast<std::size_t>(c) * m.matrix_data[c].size() + k] = m.matrix_data[c][k];
        }
        return 0;
    } catch (const std::exception& e) {
        refshim::last_error = e.what();
        return 1;
    }
}

// Whole control-kernel solve as cuper_control_local_main.cpp:115-145 does it:
// pack, m_inv, one call.  metrics[4], status[2] as the kernel writes them.
int ref_control_solve(int n, const int* row_ptr, const int* col_idx, const double* val,
                      const double* b, const double* x0, double tau, int max_iters, double* x,
                      double* metrics, int* status) {
    try {
        const CsrDataset d = refshim::make_dataset(n, row_ptr, col_idx, val, b, x0);
        const CuperControlMatrix m = build_cuper_control_matrix(d);
        std::vector<double> xv(x0, x0 + n), r(n, 0.0), z(n, 0.0), p(n, 0.0), ap(n, 0.0);
        std::vector<double> m_inv = build_jacobi_inverse(d);
        cuper_pcg_control_kernel(m.sp_element_list_ptr.data(), m.matrix_data[0].data(),
                                 m.matrix_data[1].data(), m.matrix_data[2].data(),
                                 m.matrix_data[3].data(), m.matrix_data[4].data(),
                                 m.matrix_data[5].data(), m.matrix_data[6].data(),
                                 m.matrix_data[7].data(), m.matrix_data[8].data(),
                                 m.matrix_data[9].data(), m.matrix_data[10].data(),
                                 m.matrix_data[11].data(), m.matrix_data[12].data(),
                                 m.matrix_data[13].data(), m.matrix_data[14].data(),
                                 m.matrix_data[15].data(), d.b().data(), m_inv.data(), xv.data(),
                                 r.data(), z.data(), p.data(), ap.data(), metrics, status, tau,
                                 max_iters > 0 ? max_iters : std::max(4 * n, 1000), n,
                                 m.batch_count);
        std::copy(xv.begin(), xv.end(), x);
        return 0;
    } catch (const std::exception& e) {
        refshim::last_error = e.what();
        return 1;
    }
}
}  // extern "C"
