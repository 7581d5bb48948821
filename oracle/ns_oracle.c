/*
 * Test infrastructure only (the oracle).  Plain-C restatement of the
 * reference's fixed-pivot refactor and solves; see ns_oracle.h.  Built with
 * -ffp-contract=off so every multiply and subtract rounds separately, as in
 * the reference's x86-64 build.
 */
#include "ns_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { ORC_OK = 0, ORC_INVALID = 1, ORC_NOMEM = 8, ORC_SINGULAR = 102, ORC_REORDER = 103 };

/* Column starts (0-based element index) and pivot element of each column. */
static int col_index(int n, int n_elem, const int* elem_row, const int* elem_col,
                     int* col_ptr, int* diag) {
    for (int j = 0; j <= n; ++j) col_ptr[j] = 0;
    for (int e = 0; e < n_elem; ++e) {
        if (elem_col[e] < 1 || elem_col[e] > n || elem_row[e] < 1 || elem_row[e] > n)
            return ORC_INVALID;
        if (e > 0 && elem_col[e] < elem_col[e - 1]) return ORC_INVALID;
        col_ptr[elem_col[e]]++;
    }
    for (int j = 0; j < n; ++j) col_ptr[j + 1] += col_ptr[j];
    for (int j = 0; j < n; ++j) {
        diag[j] = -1;
        for (int e = col_ptr[j]; e < col_ptr[j + 1]; ++e)
            if (elem_row[e] == j + 1) diag[j] = e;
        if (diag[j] < 0) return ORC_INVALID;
    }
    return ORC_OK;
}

/* factor.cpp:980-1052, direct (dense scatter) variant; factor.cpp:929-947
 * for the threshold re-validation. */
int nso_refactor(int n, int nnz, int n_elem, const int* elem_row, const int* elem_col,
                 const int* slot_to_elem, const double* a, double diag_gmin,
                 int check_pivots, double* lu, int* fail_step) {
    int rc = ORC_OK;
    int* col_ptr = malloc(sizeof(int) * (n + 1));
    int* diag = malloc(sizeof(int) * n);
    double* dense = malloc(sizeof(double) * (n + 1));
    if (fail_step) *fail_step = -1;
    if (!col_ptr || !diag || !dense) { rc = ORC_NOMEM; goto out; }
    if ((rc = col_index(n, n_elem, elem_row, elem_col, col_ptr, diag)) != ORC_OK) goto out;

    for (int e = 0; e < n_elem; ++e) lu[e] = 0.0;
    for (int k = 0; k < nnz; ++k) lu[slot_to_elem[k]] = a[k];
    if (diag_gmin != 0.0)
        for (int j = n - 1; j >= 0; --j) lu[diag[j]] += diag_gmin;

    for (int j = 0; j < n; ++j) {
        for (int e = col_ptr[j]; e < col_ptr[j + 1]; ++e) dense[elem_row[e]] = lu[e];
        for (int e = col_ptr[j]; e < diag[j]; ++e) {
            const int r = elem_row[e] - 1;             /* pivot step of this U entry */
            const double u = dense[r + 1] * lu[diag[r]];
            lu[e] = u;
            for (int f = diag[r] + 1; f < col_ptr[r + 1]; ++f)
                dense[elem_row[f]] -= u * lu[f];
        }
        for (int e = diag[j] + 1; e < col_ptr[j + 1]; ++e) lu[e] = dense[elem_row[e]];
        const double piv = dense[j + 1];
        if (check_pivots) {
            double largest = 0.0;
            for (int e = diag[j] + 1; e < col_ptr[j + 1]; ++e)
                if (fabs(lu[e]) > largest) largest = fabs(lu[e]);
            if (!(largest * 1e-3 < fabs(piv))) {
                if (fail_step) *fail_step = j;
                rc = ORC_REORDER;
                goto out;
            }
        } else if (piv == 0.0) {
            if (fail_step) *fail_step = j;
            rc = ORC_SINGULAR;
            goto out;
        }
        lu[diag[j]] = 1.0 / piv;
    }
out:
    free(col_ptr);
    free(diag);
    free(dense);
    return rc;
}

/* Row lists of the strictly upper part, columns ascending. */
static int upper_rows(int n, int n_elem, const int* elem_row, const int* elem_col,
                      int** urow_ptr, int** urow_elem) {
    int* ptr = calloc((size_t)n + 1, sizeof(int));
    int* el = malloc(sizeof(int) * (size_t)(n_elem ? n_elem : 1));
    int* fill = malloc(sizeof(int) * (size_t)n);
    if (!ptr || !el || !fill) { free(ptr); free(el); free(fill); return ORC_NOMEM; }
    for (int e = 0; e < n_elem; ++e)
        if (elem_row[e] < elem_col[e]) ptr[elem_row[e]]++;
    for (int i = 0; i < n; ++i) ptr[i + 1] += ptr[i];
    for (int i = 0; i < n; ++i) fill[i] = ptr[i];
    for (int e = 0; e < n_elem; ++e)
        if (elem_row[e] < elem_col[e]) el[fill[elem_row[e] - 1]++] = e;
    free(fill);
    *urow_ptr = ptr;
    *urow_elem = el;
    return ORC_OK;
}

int nso_solve(int n, int n_elem, const int* elem_row, const int* elem_col,
              const int* int_to_ext_row, const int* int_to_ext_col, const double* lu,
              double* x) {
    int rc;
    int* col_ptr = malloc(sizeof(int) * (n + 1));
    int* diag = malloc(sizeof(int) * n);
    double* inter = malloc(sizeof(double) * (n + 1));
    int *urow_ptr = NULL, *urow_elem = NULL;
    if (!col_ptr || !diag || !inter) { rc = ORC_NOMEM; goto out; }
    if ((rc = col_index(n, n_elem, elem_row, elem_col, col_ptr, diag)) != ORC_OK) goto out;
    if ((rc = upper_rows(n, n_elem, elem_row, elem_col, &urow_ptr, &urow_elem)) != ORC_OK) goto out;

    for (int i = n; i > 0; --i) inter[i] = x[int_to_ext_row[i - 1] - 1];
    for (int i = 1; i <= n; ++i) {      /* forward: L columns, reciprocal pivot */
        double t = inter[i];
        if (t != 0.0) {
            t *= lu[diag[i - 1]];
            inter[i] = t;
            for (int e = diag[i - 1] + 1; e < col_ptr[i]; ++e) inter[elem_row[e]] -= t * lu[e];
        }
    }
    for (int i = n; i > 0; --i) {       /* backward: U rows, unit diagonal */
        double t = inter[i];
        for (int k = urow_ptr[i - 1]; k < urow_ptr[i]; ++k) {
            const int e = urow_elem[k];
            t -= lu[e] * inter[elem_col[e]];
        }
        inter[i] = t;
    }
    for (int i = n; i > 0; --i) x[int_to_ext_col[i - 1] - 1] = inter[i];
out:
    free(col_ptr);
    free(diag);
    free(inter);
    free(urow_ptr);
    free(urow_elem);
    return rc;
}

int nso_solve_transposed(int n, int n_elem, const int* elem_row, const int* elem_col,
                         const int* int_to_ext_row, const int* int_to_ext_col,
                         const double* lu, double* x) {
    int rc;
    int* col_ptr = malloc(sizeof(int) * (n + 1));
    int* diag = malloc(sizeof(int) * n);
    double* inter = malloc(sizeof(double) * (n + 1));
    int *urow_ptr = NULL, *urow_elem = NULL;
    if (!col_ptr || !diag || !inter) { rc = ORC_NOMEM; goto out; }
    if ((rc = col_index(n, n_elem, elem_row, elem_col, col_ptr, diag)) != ORC_OK) goto out;
    if ((rc = upper_rows(n, n_elem, elem_row, elem_col, &urow_ptr, &urow_elem)) != ORC_OK) goto out;

    for (int i = n; i > 0; --i) inter[i] = x[int_to_ext_col[i - 1] - 1];
    for (int i = 1; i <= n; ++i) {      /* forward: U rows scatter */
        const double t = inter[i];
        if (t != 0.0)
            for (int k = urow_ptr[i - 1]; k < urow_ptr[i]; ++k) {
                const int e = urow_elem[k];
                inter[elem_col[e]] -= t * lu[e];
            }
    }
    for (int i = n; i > 0; --i) {       /* backward: L columns gather, reciprocal pivot */
        double t = inter[i];
        for (int e = diag[i - 1] + 1; e < col_ptr[i]; ++e) t -= lu[e] * inter[elem_row[e]];
        inter[i] = t * lu[diag[i - 1]];
    }
    for (int i = n; i > 0; --i) x[int_to_ext_row[i - 1] - 1] = inter[i];
out:
    free(col_ptr);
    free(diag);
    free(inter);
    free(urow_ptr);
    free(urow_elem);
    return rc;
}

/* ---- AMD-LU ------------------------------------------------------------- */

int nso_amd_replay(int n, const int* a_colptr, const int* a_rowidx, const int* q,
                   const int* pinv, const int* Lp, const int* Li, const int* Up, const int* Ui,
                   const double* a, double diag_gmin, double* Lx, double* Ux, int* fail_step) {
    /* Dense accumulator over pivot steps, cleared entry by entry as the
     * reference's replay does. */
    double* x = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    int rc = 0;
    if (!x) return 8;
    if (fail_step) *fail_step = -1;
    for (int k = 0; k < n && rc == 0; ++k) {
        const int col = q[k];
        for (int p = a_colptr[col]; p < a_colptr[col + 1]; ++p) x[pinv[a_rowidx[p]]] = a[p];
        if (diag_gmin != 0.0) x[pinv[col]] += diag_gmin;
        double colmax = 0.0;
        for (int up = Up[k]; up < Up[k + 1] - 1; ++up) {
            const int j = Ui[up];
            const double u = x[j];
            x[j] = 0.0;
            Ux[up] = u;
            if (fabs(u) > colmax) colmax = fabs(u);
            for (int p = Lp[j] + 1; p < Lp[j + 1]; ++p) x[Li[p]] -= Lx[p] * u;
        }
        const double ukk = x[k];
        x[k] = 0.0;
        const double aukk = fabs(ukk);
        if (aukk > colmax) colmax = aukk;
        if (ukk == 0.0 || (colmax > 0.0 && aukk < 1e-3 * colmax)) {
            rc = 103;
            if (fail_step) *fail_step = k;
            break;
        }
        Ux[Up[k + 1] - 1] = ukk;
        for (int p = Lp[k] + 1; p < Lp[k + 1]; ++p) {
            Lx[p] = x[Li[p]] / ukk;
            x[Li[p]] = 0.0;
        }
    }
    free(x);
    return rc;
}

int nso_amd_solve(int n, const int* q, const int* pinv, const int* Lp, const int* Li,
                  const double* Lx, const int* Up, const int* Ui, const double* Ux, double* x) {
    double* y = (double*)malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
    if (!y) return 8;
    for (int i = 0; i < n; ++i) y[pinv[i]] = x[i];
    for (int j = 0; j < n; ++j) {
        const double yj = y[j];
        for (int p = Lp[j] + 1; p < Lp[j + 1]; ++p) y[Li[p]] -= Lx[p] * yj;
    }
    for (int j = n - 1; j >= 0; --j) {
        y[j] /= Ux[Up[j + 1] - 1];
        const double yj = y[j];
        for (int p = Up[j]; p < Up[j + 1] - 1; ++p) y[Ui[p]] -= Ux[p] * yj;
    }
    for (int k = 0; k < n; ++k) x[q[k]] = y[k];
    free(y);
    return 0;
}
