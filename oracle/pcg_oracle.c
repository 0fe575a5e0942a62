/*
 * pcg_oracle.c -- CPU restatement of the reference's Jacobi-PCG path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm may load it.  The product library never links or calls it.
 *
 * Every function restates one reference routine in plain C, keeping the
 * reference's floating-point operation order so that results are bit-identical
 * to the reference built from source (the parity pin is
 * tests/test_oracle_pin.py, which runs both on the same inputs).
 *
 *   or_spmv_csr            src/CsrDataset.hpp:78-90        (CsrDataset::spmv)
 *   or_extract_jacobi_diag src/CsrDataset.hpp:92-116       (extract_jacobi_diag)
 *   or_golden_pcg          src/CgSolverGolden.hpp:42-124   (run_jacobi_pcg)
 *   or_residual_norm       src/CgSolverGolden.hpp:126-135  (compute_residual_norm)
 *   or_init_pcg / or_dot / or_update_xrz / or_update_p
 *                          archived/kernels/cg_kernels.cpp:73-159
 *   or_multi_kernel_pcg    archived/host/multi_kernel_solver.hpp:100-234
 *   or_cuper_style_spmv    host/cuper_pcg_solver.hpp:136-159 (+ plan :90-134)
 *   or_control_pcg         kernels/cuper_pcg_control_kernel.cpp:1069-1235
 *                          (control flow and status codes; its SpMV is the
 *                          FP32-value / FP32-vector / FP32-accumulate product
 *                          in CSR row order, see or_spmv_f32)
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_BREAKDOWN_EPS 1.0e-30 /* include/cg_common.hpp:13 kBreakdownEps */

enum { OR_CONVERGED = 0, OR_MAX_ITER = 1, OR_BREAKDOWN = 2 };

/* src/CsrDataset.hpp:78-90: y[row] = sum over the row in CSR order, FP64. */
void or_spmv_csr(int n, const int* row_ptr, const int* col_idx, const double* val,
                 const double* x, double* y) {
    for (int row = 0; row < n; ++row) {
        double acc = 0.0;
        for (int k = row_ptr[row]; k < row_ptr[row + 1]; ++k) acc += val[k] * x[col_idx[k]];
        y[row] = acc;
    }
}

/* src/CsrDataset.hpp:92-116.  Returns 0, or -(row+1) for a missing diagonal,
 * or -(n+row+1) for a zero diagonal (|d| <= DBL_MIN), matching the two throws. */
int or_extract_jacobi_diag(int n, const int* row_ptr, const int* col_idx, const double* val,
                           double* diag) {
    for (int row = 0; row < n; ++row) {
        int found = 0;
        diag[row] = 0.0;
        for (int k = row_ptr[row]; k < row_ptr[row + 1]; ++k) {
            if (col_idx[k] == row) {
                diag[row] = val[k];
                found = 1;
                break;
            }
        }
        if (!found) return -(row + 1);
        if (fabs(diag[row]) <= DBL_MIN) return -(n + row + 1);
    }
    return 0;
}

static double or_dot_seq(int n, const double* a, const double* b) {
    double acc = 0.0;
    for (int i = 0; i < n; ++i) acc += a[i] * b[i];
    return acc;
}

/* src/CgSolverGolden.hpp:42-124 (run_jacobi_pcg).
 * trace: optional [max_iters][5] = alpha, beta, rz, rr, residual per iteration.
 * Returns 0 ok, 1 breakdown (the reference throws), 2 bad tau, 3 bad diag. */
int or_golden_pcg(int n, const int* row_ptr, const int* col_idx, const double* val,
                  const double* b, const double* x0, double tau, int max_iters_in,
                  double* x, int* iterations, double* final_rr, int* converged, double* trace) {
    if (!(tau > 0.0)) return 2;
    const int max_iters = max_iters_in > 0 ? max_iters_in : (4 * n > 1000 ? 4 * n : 1000);
    double* diag = (double*)malloc(sizeof(double) * (size_t)n);
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* z = (double*)malloc(sizeof(double) * (size_t)n);
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    double* ap = (double*)malloc(sizeof(double) * (size_t)n);
    int rc = 0;
    *iterations = 0;
    if (or_extract_jacobi_diag(n, row_ptr, col_idx, val, diag) != 0) { rc = 3; goto done; }
    memcpy(x, x0, sizeof(double) * (size_t)n);
    or_spmv_csr(n, row_ptr, col_idx, val, x, ap);
    for (int i = 0; i < n; ++i) r[i] = b[i] - ap[i];
    for (int i = 0; i < n; ++i) z[i] = r[i] / diag[i]; /* apply_jacobi_inverse divides */
    memcpy(p, z, sizeof(double) * (size_t)n);
    double rz = or_dot_seq(n, r, z);
    double rr = or_dot_seq(n, r, r);
    *final_rr = rr;
    for (int it = 0; it < max_iters && rr > tau; ++it) {
        or_spmv_csr(n, row_ptr, col_idx, val, p, ap);
        const double pap = or_dot_seq(n, p, ap);
        if (fabs(pap) <= DBL_MIN) { rc = 1; goto done; }
        const double alpha = rz / pap;
        for (int i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * ap[i];
        }
        for (int i = 0; i < n; ++i) z[i] = r[i] / diag[i];
        const double rz_new = or_dot_seq(n, r, z);
        const double rr_new = or_dot_seq(n, r, r);
        const double beta = rz_new / rz;
        if (trace) {
            double* t = trace + 5 * (size_t)it;
            t[0] = alpha; t[1] = beta; t[2] = rz_new; t[3] = rr_new;
            t[4] = sqrt(rr_new > 0.0 ? rr_new : 0.0);
        }
        rz = rz_new;
        rr = rr_new;
        *iterations = it + 1;
        *final_rr = rr;
        if (rr <= tau) break;
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
done:
    *converged = (*final_rr <= tau);
    free(diag); free(r); free(z); free(p); free(ap);
    return rc;
}

/* src/CgSolverGolden.hpp:126-135: ||A x - b||_2 */
double or_residual_norm(int n, const int* row_ptr, const int* col_idx, const double* val,
                        const double* b, const double* x) {
    double* ax = (double*)malloc(sizeof(double) * (size_t)n);
    or_spmv_csr(n, row_ptr, col_idx, val, x, ax);
    for (int i = 0; i < n; ++i) ax[i] -= b[i];
    const double s = sqrt(or_dot_seq(n, ax, ax));
    free(ax);
    return s;
}

/* archived/kernels/cg_kernels.cpp:73-103 */
void or_init_pcg(int n, const double* b, const double* ax, const double* m_inv, double* r,
                 double* z, double* p, double* metrics) {
    double rz = 0.0, rr = 0.0;
    for (int i = 0; i < n; ++i) {
        const double rv = b[i] - ax[i];
        const double zv = m_inv[i] * rv;
        r[i] = rv; z[i] = zv; p[i] = zv;
        rz += rv * zv;
        rr += rv * rv;
    }
    metrics[0] = rz;
    metrics[1] = rr;
}

/* archived/kernels/cg_kernels.cpp:105-116 */
void or_dot(int n, const double* a, const double* b, double* out) { out[0] = or_dot_seq(n, a, b); }

/* archived/kernels/cg_kernels.cpp:118-147 */
void or_update_xrz(int n, double* x, const double* p, double* r, const double* ap,
                   const double* m_inv, double* z, double* metrics, double alpha) {
    double rz = 0.0, rr = 0.0;
    for (int i = 0; i < n; ++i) {
        x[i] += alpha * p[i];
        r[i] -= alpha * ap[i];
        z[i] = m_inv[i] * r[i];
        rz += r[i] * z[i];
        rr += r[i] * r[i];
    }
    metrics[0] = rz;
    metrics[1] = rr;
}

/* archived/kernels/cg_kernels.cpp:149-159 */
void or_update_p(int n, const double* z, double* p, double beta) {
    for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
}

/* host/pcg_common.hpp:42-54 build_jacobi_inverse. Returns 0 or nonzero on a bad diagonal. */
int or_jacobi_inverse(int n, const int* row_ptr, const int* col_idx, const double* val,
                      double* m_inv) {
    if (or_extract_jacobi_diag(n, row_ptr, col_idx, val, m_inv) != 0) return 1;
    for (int i = 0; i < n; ++i) {
        if (fabs(m_inv[i]) <= OR_BREAKDOWN_EPS) return 1;
        m_inv[i] = 1.0 / m_inv[i];
    }
    return 0;
}

static int or_finite(double v) { return isfinite(v); }

/* archived/host/multi_kernel_solver.hpp:100-234 (run_local_multi_kernel_solver), without
 * the n <= 1024 guard (that guard only sizes the HLS on-chip buffer).
 * trace: optional [max_iters][5] alpha, beta, rz, rr, residual (the [iter] log line).
 * out_status: 0 converged, 1 max_iter, 2 breakdown.  Returns 0, or 2 bad tau, 3 bad diag. */
int or_multi_kernel_pcg(int n, const int* row_ptr, const int* col_idx, const double* val,
                        const double* b, const double* x0, double tau, int max_iters_in,
                        double* x, int* iterations, double* final_rr, int* out_status,
                        double* residual_l2, double* trace) {
    if (!(tau > 0.0)) return 2;
    double* m_inv = (double*)malloc(sizeof(double) * (size_t)n);
    double* r = (double*)calloc((size_t)n, sizeof(double));
    double* z = (double*)calloc((size_t)n, sizeof(double));
    double* p = (double*)calloc((size_t)n, sizeof(double));
    double* y = (double*)calloc((size_t)n, sizeof(double));
    int rc = 0, breakdown = 0;
    *iterations = 0;
    if (or_jacobi_inverse(n, row_ptr, col_idx, val, m_inv) != 0) { rc = 3; goto done; }
    const int max_iters = max_iters_in > 0 ? max_iters_in : (4 * n > 1000 ? 4 * n : 1000);
    memcpy(x, x0, sizeof(double) * (size_t)n);
    double metrics[2] = {0.0, 0.0}, dot_out = 0.0;
    or_spmv_csr(n, row_ptr, col_idx, val, x, y);
    or_init_pcg(n, b, y, m_inv, r, z, p, metrics);
    double rz = metrics[0], rr = metrics[1];
    *final_rr = rr;
    for (int it = 0; it < max_iters && rr > tau; ++it) {
        or_spmv_csr(n, row_ptr, col_idx, val, p, y);
        or_dot(n, p, y, &dot_out);
        const double pap = dot_out;
        if (!or_finite(pap) || fabs(pap) <= OR_BREAKDOWN_EPS || !or_finite(rz) ||
            fabs(rz) <= OR_BREAKDOWN_EPS) { breakdown = 1; break; }
        const double alpha = rz / pap;
        if (!or_finite(alpha)) { breakdown = 1; break; }
        or_update_xrz(n, x, p, r, y, m_inv, z, metrics, alpha);
        const double rz_new = metrics[0], rr_new = metrics[1];
        if (!or_finite(rz_new) || !or_finite(rr_new)) { breakdown = 1; break; }
        const double beta = rz_new / rz;
        if (!or_finite(beta)) { breakdown = 1; break; }
        or_update_p(n, z, p, beta);
        rz = rz_new;
        rr = rr_new;
        *iterations = it + 1;
        *final_rr = rr;
        if (trace) {
            double* t = trace + 5 * (size_t)it;
            t[0] = alpha; t[1] = beta; t[2] = rz; t[3] = rr; t[4] = sqrt(rr > 0.0 ? rr : 0.0);
        }
    }
    if (residual_l2) *residual_l2 = or_residual_norm(n, row_ptr, col_idx, val, b, x);
    *out_status = breakdown ? OR_BREAKDOWN : (*final_rr <= tau ? OR_CONVERGED : OR_MAX_ITER);
done:
    free(m_inv); free(r); free(z); free(p); free(y);
    return rc;
}

/* host/cuper_pcg_solver.hpp:90-159.  The plan groups the non-zeros by 8192-wide column
 * batch, keeping CSR order inside a batch; the SpMV rounds x to an FP32 window, forms
 * the FP32 product and accumulates it into an FP64 y in that order. */
#define OR_CUPER_SLICE_WIDTH 8192
void or_cuper_style_spmv(int n, const int* row_ptr, const int* col_idx, const double* val,
                         const double* x, double* y) {
    /* y[row] only sees its own elements, so the batch-major order of the reference
     * reduces to: the row's elements stably ordered by column batch. */
    int cap = 64;
    int* order = (int*)malloc(sizeof(int) * (size_t)cap);
    for (int row = 0; row < n; ++row) {
        const int len = row_ptr[row + 1] - row_ptr[row];
        if (len > cap) { cap = len; order = (int*)realloc(order, sizeof(int) * (size_t)cap); }
        for (int j = 0; j < len; ++j) {
            const int k = row_ptr[row] + j;
            const int bk = col_idx[k] / OR_CUPER_SLICE_WIDTH;
            int pos = j;
            while (pos > 0 && col_idx[order[pos - 1]] / OR_CUPER_SLICE_WIDTH > bk) {
                order[pos] = order[pos - 1];
                --pos;
            }
            order[pos] = k;
        }
        double acc = 0.0;
        for (int j = 0; j < len; ++j) {
            const int k = order[j];
            const float prod = (float)val[k] * (float)x[col_idx[k]];
            acc += (double)prod;
        }
        y[row] = acc;
    }
    free(order);
}

/* FP32 SpMV in CSR row order: FP32 value x FP32 vector, FP32 accumulation, widened to
 * FP64 on output.  This is the arithmetic of the control kernel's packed SpMV
 * (kernels/cuper_pcg_control_kernel.cpp:240-258 decode_product, :334-345 FP32 lane
 * accumulators), with the accumulation taken in CSR order. */
void or_spmv_f32(int n, const int* row_ptr, const int* col_idx, const double* val,
                 const double* x, double* y) {
    for (int row = 0; row < n; ++row) {
        float acc = 0.0f;
        for (int k = row_ptr[row]; k < row_ptr[row + 1]; ++k)
            acc += (float)val[k] * (float)x[col_idx[k]];
        y[row] = (double)acc;
    }
}

/* kernels/cuper_pcg_control_kernel.cpp:1069-1235 (cuper_pcg_control_kernel control flow):
 * parameter check, A*x0 with fused init, then the loop with its breakdown/convergence
 * tests, metrics = {rz, rr, pAp, alpha}, status = {code, iterations}.
 * spmv_mode: 0 = FP64 CSR SpMV, 1 = FP32 SpMV (or_spmv_f32). */
void or_control_pcg(int n, const int* row_ptr, const int* col_idx, const double* val,
                    const double* b, const double* m_inv, double* x, double* r, double* z,
                    double* p, double* ap, double* metrics, int* status, double tau,
                    int max_iters, int spmv_mode, double* trace) {
    double rz = 0.0, rr = 0.0, pap = 0.0, alpha = 0.0, beta = 0.0;
    int iterations = 0, code = OR_MAX_ITER;
    if (n <= 0 || max_iters < 0 || tau <= 0.0 || tau != tau) {
        status[0] = OR_BREAKDOWN; status[1] = 0;
        metrics[0] = metrics[1] = metrics[2] = metrics[3] = 0.0;
        return;
    }
    void (*spmv)(int, const int*, const int*, const double*, const double*, double*) =
        spmv_mode ? or_spmv_f32 : or_spmv_csr;
    spmv(n, row_ptr, col_idx, val, x, ap);
    for (int i = 0; i < n; ++i) {
        const double rv = b[i] - ap[i];
        const double zv = m_inv[i] * rv;
        r[i] = rv; z[i] = zv; p[i] = zv;
        rz += rv * zv;
        rr += rv * rv;
    }
    for (int it = 0; it < max_iters; ++it) {
        if (rr <= tau) { code = OR_CONVERGED; break; }
        if (rz != rz || rr != rr || fabs(rz) <= OR_BREAKDOWN_EPS) { code = OR_BREAKDOWN; break; }
        spmv(n, row_ptr, col_idx, val, p, ap);
        pap = or_dot_seq(n, p, ap);
        if (pap != pap || fabs(pap) <= OR_BREAKDOWN_EPS) { code = OR_BREAKDOWN; break; }
        const double rz_old = rz;
        alpha = rz / pap;
        if (alpha != alpha) { code = OR_BREAKDOWN; break; }
        double rz_new = 0.0, rr_new = 0.0;
        for (int i = 0; i < n; ++i) {
            const double xv = x[i] + alpha * p[i];
            const double rv = r[i] - alpha * ap[i];
            const double zv = m_inv[i] * rv;
            x[i] = xv; r[i] = rv; z[i] = zv;
            rz_new += rv * zv;
            rr_new += rv * rv;
        }
        rz = rz_new;
        rr = rr_new;
        iterations = it + 1;
        if (trace) {
            double* t = trace + 5 * (size_t)it;
            t[0] = alpha; t[1] = (fabs(rz_old) > OR_BREAKDOWN_EPS) ? rz / rz_old : 0.0;
            t[2] = rz; t[3] = rr; t[4] = sqrt(rr > 0.0 ? rr : 0.0);
        }
        if (rz != rz || rr != rr) { code = OR_BREAKDOWN; break; }
        if (rr <= tau) { code = OR_CONVERGED; break; }
        if (fabs(rz_old) <= OR_BREAKDOWN_EPS) { code = OR_BREAKDOWN; break; }
        beta = rz / rz_old;
        if (beta != beta) { code = OR_BREAKDOWN; break; }
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    if (code == OR_MAX_ITER && rr <= tau) code = OR_CONVERGED;
    metrics[0] = rz; metrics[1] = rr; metrics[2] = pap; metrics[3] = alpha;
    status[0] = code; status[1] = iterations;
}

/* Jacobi-PCG in the precision of the product's plain kernel: matrix values and the
 * vectors x, r, p, Ap rounded to FP32 after every update, dot products accumulated in
 * FP64, convergence on rr <= tau exactly as the control kernel does.  The operation order
 * follows or_control_pcg; this is the reference algorithm evaluated at FP32 storage
 * precision, used to bound what FP32 storage alone does to the iterates. */
void or_control_pcg_f32(int n, const int* row_ptr, const int* col_idx, const double* val,
                        const double* b, double tau, int max_iters, double* x_out,
                        int* status, double* trace) {
    float* x = (float*)calloc((size_t)n, sizeof(float));
    float* r = (float*)malloc(sizeof(float) * (size_t)n);
    float* p = (float*)malloc(sizeof(float) * (size_t)n);
    float* ap = (float*)malloc(sizeof(float) * (size_t)n);
    float* minv = (float*)malloc(sizeof(float) * (size_t)n);
    for (int row = 0; row < n; ++row) {
        float d = 0.0f;
        for (int k = row_ptr[row]; k < row_ptr[row + 1]; ++k)
            if (col_idx[k] == row) d = (float)val[k];
        minv[row] = 1.0f / d;
    }
    double rz = 0.0, rr = 0.0;
    for (int i = 0; i < n; ++i) {
        r[i] = (float)b[i];
        const float zv = minv[i] * r[i];
        p[i] = zv;
        rz += (double)r[i] * (double)zv;
        rr += (double)r[i] * (double)r[i];
    }
    int code = OR_MAX_ITER, iterations = 0;
    for (int it = 0; it < max_iters; ++it) {
        if (rr <= tau) { code = OR_CONVERGED; break; }
        double pap = 0.0;
        for (int row = 0; row < n; ++row) {
            float acc = 0.0f;
            for (int k = row_ptr[row]; k < row_ptr[row + 1]; ++k)
                acc += (float)val[k] * p[col_idx[k]];
            ap[row] = acc;
            pap += (double)p[row] * (double)acc;
        }
        if (pap != pap || fabs(pap) <= OR_BREAKDOWN_EPS) { code = OR_BREAKDOWN; break; }
        const double alpha = rz / pap;
        const float af = (float)alpha;
        double rz_new = 0.0, rr_new = 0.0;
        for (int i = 0; i < n; ++i) {
            x[i] = x[i] + af * p[i];
            r[i] = r[i] - af * ap[i];
            const float zv = minv[i] * r[i];
            rz_new += (double)r[i] * (double)zv;
            rr_new += (double)r[i] * (double)r[i];
        }
        const double beta = rz_new / rz;
        iterations = it + 1;
        if (trace) {
            double* t = trace + 5 * (size_t)it;
            t[0] = alpha; t[1] = beta; t[2] = rz_new; t[3] = rr_new;
            t[4] = sqrt(rr_new > 0.0 ? rr_new : 0.0);
        }
        rz = rz_new;
        rr = rr_new;
        if (rr <= tau) { code = OR_CONVERGED; break; }
        const float bf = (float)beta;
        for (int i = 0; i < n; ++i) p[i] = minv[i] * r[i] + bf * p[i];
    }
    for (int i = 0; i < n; ++i) x_out[i] = (double)x[i];
    status[0] = code;
    status[1] = iterations;
    free(x); free(r); free(p); free(ap); free(minv);
}
