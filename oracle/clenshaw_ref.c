/*
 * ORACLE -- test infrastructure only.  CPU restatement of the reference's block
 * Clenshaw filter, used by the parity tests and by the benchmark's CPU-baseline leg.
 * Nothing in the product links or calls this file.
 *
 * Follows chebyshev_subspace_iteration.jl:554-591 (identical to polfed.jl:464-501):
 *
 *   B_{K+1} = B_{K+2} = 0
 *   B_k = c_k Q + alpha * A B_{k+1} + beta * B_{k+1} - B_{k+2},   k = K..1
 *   Y   = c_0 Q + invd * A B_1 - c*invd * B_1 - B_2
 *
 * with c = (smin+smax)/2, invd = 2/(smax-smin), alpha = 2*invd, beta = -2*c*invd
 * (chebyshev_subspace_iteration.jl:562-565).
 *
 * Blocks are column-major n x b (Julia's Matrix{Float64}).  The sparse product
 * reproduces Julia SparseArrays' generic CSC x dense kernel (the `mul!(AX,A,B1)` call at
 * chebyshev_subspace_iteration.jl:574): for each output column, zero it, then for
 * each matrix column `col` scatter nzval[j]*B[col] into AX[rowval[j]].  For a
 * symmetric matrix that adds the terms of each output row in ascending column order.
 * Build with -ffp-contract=off so that every a*b+c rounds twice, as Julia's plain
 * `+=`/`*` do.  Columns are independent, so they are spread over OpenMP threads
 * (the reference's Threads.@threads over block columns, chebyshev_subspace_iteration.jl:192).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* AX[:,k] = A * X[:,k] for the columns k in [k0, k1); CSC arrays 0-based. */
static void csc_spmm_cols(int64_t n, const int64_t *colptr, const int64_t *rowval,
                          const double *nzval, const double *X, double *AX,
                          int64_t k0, int64_t k1) {
    for (int64_t k = k0; k < k1; ++k) {
        const double *x = X + k * n;
        double *y = AX + k * n;
        memset(y, 0, (size_t)n * sizeof(double));
        for (int64_t col = 0; col < n; ++col) {
            const double xj = x[col];
            for (int64_t j = colptr[col]; j < colptr[col + 1]; ++j)
                y[rowval[j]] += nzval[j] * xj;
        }
    }
}

/* Y = A X (all b columns). */
int oracle_spmm(int64_t n, int64_t b, const int64_t *colptr, const int64_t *rowval,
                const double *nzval, const double *X, double *Y, int nthreads) {
    if (n < 0 || b < 0) return 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static, 1)
#endif
    for (int64_t k = 0; k < b; ++k)
        csc_spmm_cols(n, colptr, rowval, nzval, X, Y, k, k + 1);
    return 0;
}

/* Y = p(A_hat) Q by the block Clenshaw recurrence; coeffs has K+1 entries. */
int oracle_apply_poly_block(int64_t n, int64_t b, const int64_t *colptr,
                            const int64_t *rowval, const double *nzval, const double *Q,
                            double *Y, const double *coeffs, int64_t K, double smin,
                            double smax, int nthreads) {
    if (n < 0 || b < 0 || K < 0) return 1;
    const double c = 0.5 * (smin + smax);
    const double invd = 2.0 / (smax - smin);
    const double alpha = 2.0 * invd;
    const double beta = -2.0 * c * invd;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static, 1)
#endif
    for (int64_t j = 0; j < b; ++j) {
        /* one column carries its own three recurrence vectors and AX */
        double *buf = (double *)malloc((size_t)n * 4 * sizeof(double));
        double *B1 = buf, *B2 = buf + n, *TMP = buf + 2 * n, *AX = buf + 3 * n;
        const double *q = Q + j * n;
        memset(B1, 0, (size_t)n * sizeof(double));
        memset(B2, 0, (size_t)n * sizeof(double));
        for (int64_t k = K + 1; k >= 2; --k) {  /* Julia's k=(K+1):-1:2, coeffs[k] is c_{k-1} */
            csc_spmm_cols(n, colptr, rowval, nzval, B1, AX, 0, 1);
            const double ck = coeffs[k - 1];
            for (int64_t i = 0; i < n; ++i)
                TMP[i] = ck * q[i] + alpha * AX[i] + beta * B1[i] - B2[i];
            double *t = B2; B2 = B1; B1 = TMP; TMP = t;   /* B1,B2,TMP = TMP,B1,B2 */
        }
        csc_spmm_cols(n, colptr, rowval, nzval, B1, AX, 0, 1);
        const double c0 = coeffs[0];
        double *y = Y + j * n;
        for (int64_t i = 0; i < n; ++i)
            y[i] = c0 * q[i] + invd * AX[i] - c * invd * B1[i] - B2[i];
        free(buf);
    }
    return 0;
}
