// nsgpu::GpuSolver -- a header-only C++ class with the method set and error
// conventions of the reference's ISolver (src/core/solver_iface.hpp:16-41) and
// NeoSolver (src/core/neo_solver.cpp:184-297), on top of the C ABI in
// nsgpu.h.  One instance per object: this is the plain, one-instance-per-launch
// GPU path; batches of instances use nsg_batch_* / nsg_dc_batch_* directly.
// The engine is NeoSolver's Markowitz ordering by default; NSG_SOLVER_AMDLU
// or NSG_SOLVER_AUTO_AMDLU give AmdLuSolver / make_solver's AutoFallbackSolver
// (src/core/amd_lu_solver.cpp, make_solver.cpp:71-145) -- pick it with
// nsg_solver_select(num_vars, is_linear) as make_solver does.
//
//   symbolic(n, col_ptr, row_idx)   NeoSolver::symbolic (pattern in CSC)
//   numeric(values, diag_gmin)      NeoSolver::numeric: first call orders on the
//                                   host (Sparse-1.3 Markowitz, bit-identical
//                                   pivots); later calls re-validate the pivots
//                                   on the GPU and re-order on the host only if
//                                   one fails.  Returns true when singular.
//   refactorize(values, diag_gmin)  NeoSolver::refactorize (spFactor) on the GPU.
//                                   Returns true when singular.
//   solve(rhs)                      NeoSolver::solve (spSolve), in place.
//   solve_transposed(rhs)           spSolveTransposed, in place.
//   numeric_complex(ax)             NeoSolver::numeric_complex: complex
//                                   Markowitz ordering on the host (ax = 2*nnz
//                                   doubles, (re, im) per CSC slot), factor on
//                                   the GPU.
//   refactorize_complex(ax)         factor_complex with those pivots on the GPU.
//                                   Returns true when singular.
//   solve_complex(rhs)              solve_complex (rhs = 2*n doubles), in place.
//
// The real and the complex factorizations are independent (the reference
// keeps them in one matrix; an AC sweep never interleaves them).  A singular
// first complex matrix, which NeoSolver::numeric_complex does not report,
// leaves no factorization here: solve_complex then throws.
//   set_equilibrate(on)             NeoSolver's row/column equilibration
//                                   (neo_solver.cpp:57-102, 148-226): numeric()
//                                   and refactorize() factor D_r A D_c (radix-2
//                                   scale factors from the values, diag_gmin
//                                   scaled onto each diagonal), solve() scales
//                                   b by D_r and the result by D_c.  Like the
//                                   reference, only the Markowitz engine honors
//                                   it (AmdLuSolver and the auto-fallback
//                                   wrapper ignore the toggle).
//
// Misuse throws std::logic_error, a size mismatch std::invalid_argument, a
// CUDA or allocation failure std::runtime_error -- as NeoSolver does.
#pragma once
#include "nsgpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace nsgpu {

class GpuSolver {
public:
    explicit GpuSolver(int engine = NSG_SOLVER_MARKOWITZ) : engine_(engine) {}
    GpuSolver(const GpuSolver&) = delete;
    GpuSolver& operator=(const GpuSolver&) = delete;
    ~GpuSolver() { release(); }

    // ISolver::name: the engine the factorization runs (an auto engine
    // reports the one it settled on after its first numeric()).
    const char* name() const {
        const int k = topo_ ? nsg_topology_solver(topo_) : engine_;
        return k == NSG_SOLVER_MARKOWITZ ? "gpu-markowitz" : "gpu-amdlu";
    }

    void symbolic(int n, const std::vector<int>& col_ptr, const std::vector<int>& row_idx) {
        if (n <= 0 || static_cast<int>(col_ptr.size()) != n + 1 ||
            col_ptr.back() != static_cast<int>(row_idx.size()))
            throw std::invalid_argument("GpuSolver::symbolic: malformed pattern");
        release();
        n_ = n;
        col_ptr_ = col_ptr;
        row_idx_ = row_idx;
        col_of_.resize(row_idx.size());
        for (int j = 0; j < n; ++j)
            for (int k = col_ptr[j]; k < col_ptr[j + 1]; ++k) col_of_[k] = j;
        symbolized_ = true;
        numeric_called_ = false;
        factored_ = false;
    }

    void set_equilibrate(bool on) { equilibrate_ = on && engine_ == NSG_SOLVER_MARKOWITZ; }

    bool numeric(const std::vector<double>& values_in, double diag_gmin = 0.0) {
        require_symbolic("numeric");
        check_values(values_in);
        const std::vector<double>& values = equilibrate_ ? scaled(values_in, diag_gmin) : values_in;
        if (equilibrate_) diag_gmin = 0.0;  // already on the scaled diagonal
        numeric_called_ = true;
        if (!topo_) {
            nsg_topology* t = nullptr;
            const int rc = nsg_topology_order_solver(n_, nnz(), col_ptr_.data(), row_idx_.data(),
                                                     values.data(), diag_gmin, engine_, &t);
            if (rc == NSG_SINGULAR) return true;
            check(rc, "numeric");
            topo_ = t;
            rebuild_batch();
            upload(values);
            factored_ = (gpu_refactor(diag_gmin, 0) == NSG_OK);
            return !factored_;
        }
        upload(values);
        int st = gpu_refactor(diag_gmin, 1);
        if (st == NSG_REORDER) {
            int step = 0;
            const int rc = nsg_topology_numeric(topo_, values.data(), diag_gmin, &step);
            if (rc == NSG_SINGULAR) return true;
            check(rc, "numeric");
            rebuild_batch();
            st = gpu_refactor(diag_gmin, 0);
        }
        factored_ = (st == NSG_OK);
        return !factored_;
    }

    bool refactorize(const std::vector<double>& values_in, double diag_gmin = 0.0) {
        require_symbolic("refactorize");
        if (!numeric_called_)
            throw std::logic_error("GpuSolver::refactorize: numeric() not called");
        if (!topo_) return true;  // the first numeric() found the matrix singular
        check_values(values_in);
        const std::vector<double>& values = equilibrate_ ? scaled(values_in, diag_gmin) : values_in;
        if (equilibrate_) diag_gmin = 0.0;
        upload(values);
        int st = gpu_refactor(diag_gmin, 0);
        if (st == NSG_REORDER) {
            // AMD-LU: the replay's growth test failed and factor_ would pick
            // other pivots -- AmdLuSolver::refactorize falls back to a full
            // factor_ (amd_lu_solver.cpp:280-301), done here on the host.
            int step = 0;
            const int rc = nsg_topology_numeric(topo_, values.data(), diag_gmin, &step);
            if (rc == NSG_SINGULAR) {
                factored_ = false;
                return true;
            }
            check(rc, "refactorize");
            rebuild_batch();
            st = gpu_refactor(diag_gmin, 0);
        }
        factored_ = (st == NSG_OK);
        return !factored_;
    }

    void solve(std::vector<double>& rhs) {
        if (!equilibrate_) {
            sweep(rhs, false);
            return;
        }
        // (D_r A D_c) y = D_r b, then x = D_c y
        if (static_cast<int>(rhs.size()) != n_)
            throw std::invalid_argument("GpuSolver::solve: rhs size mismatch");
        for (int i = 0; i < n_; ++i) rhs[i] = dr_[i] * rhs[i];
        sweep(rhs, false);
        for (int i = 0; i < n_; ++i) rhs[i] = dc_[i] * rhs[i];
    }
    void solve_transposed(std::vector<double>& rhs) {
        if (equilibrate_)
            throw std::logic_error("GpuSolver::solve_transposed: not defined with equilibration");
        sweep(rhs, true);
    }

    void numeric_complex(const std::vector<double>& ax) {
        require_symbolic("numeric_complex");
        check_complex_values(ax);
        release_complex();
        complex_called_ = true;
        nsg_topology* t = nullptr;
        const int rc = nsg_topology_order_complex(n_, nnz(), col_ptr_.data(), row_idx_.data(),
                                                  ax.data(), &t);
        if (rc == NSG_SINGULAR) return;
        check(rc, "numeric_complex");
        ctopo_ = t;
        check(nsg_batch_create(1, &ctopo_, &cbatch_), "batch");
        long long lu_off[2] = {0, 0};
        check(nsg_batch_layout(cbatch_, nullptr, nullptr, lu_off), "layout");
        cuda(cudaMalloc(reinterpret_cast<void**>(&d_cax_), sizeof(double) * 2 * nnz()), "alloc");
        cuda(cudaMalloc(reinterpret_cast<void**>(&d_clu_), sizeof(double) * 2 * lu_off[1]),
             "alloc");
        cuda(cudaMalloc(reinterpret_cast<void**>(&d_cx_), sizeof(double) * 2 * n_), "alloc");
        cuda(cudaMalloc(reinterpret_cast<void**>(&d_cstatus_), sizeof(int)), "alloc");
        complex_factored_ = (gpu_refactor_complex(ax) == NSG_OK);
    }

    bool refactorize_complex(const std::vector<double>& ax) {
        require_symbolic("refactorize_complex");
        if (!complex_called_)
            throw std::logic_error("GpuSolver::refactorize_complex: numeric_complex() not called");
        check_complex_values(ax);
        if (!cbatch_) return true;  // the first complex matrix was singular
        complex_factored_ = (gpu_refactor_complex(ax) == NSG_OK);
        return !complex_factored_;
    }

    void solve_complex(std::vector<double>& rhs) {
        require_symbolic("solve_complex");
        if (!complex_called_)
            throw std::logic_error("GpuSolver::solve_complex: numeric_complex() not called");
        if (static_cast<int>(rhs.size()) != 2 * n_)
            throw std::invalid_argument("GpuSolver::solve_complex: rhs size must be 2*n");
        if (!complex_factored_)
            throw std::runtime_error("GpuSolver::solve_complex: no valid factorization (singular)");
        cuda(cudaMemcpy(d_cx_, rhs.data(), sizeof(double) * 2 * n_, cudaMemcpyHostToDevice),
             "rhs");
        check(nsg_batch_solve_complex(cbatch_, d_clu_, d_cx_, nullptr), "solve_complex");
        cuda(cudaMemcpy(rhs.data(), d_cx_, sizeof(double) * 2 * n_, cudaMemcpyDeviceToHost),
             "result");
    }

private:
    int engine_ = NSG_SOLVER_MARKOWITZ;
    int n_ = 0;
    bool equilibrate_ = false;
    std::vector<int> col_of_;           // column of each CSC slot
    std::vector<double> dr_, dc_, scaled_;  // scale factors and D_r A D_c
    bool symbolized_ = false;
    bool numeric_called_ = false;  // NeoSolver's factored_ flag
    bool factored_ = false;        // the last factorization succeeded
    std::vector<int> col_ptr_, row_idx_;
    nsg_topology* topo_ = nullptr;
    nsg_batch* batch_ = nullptr;
    double* d_values_ = nullptr;
    double* d_x_ = nullptr;
    int* d_status_ = nullptr;
    // complex (AC) factorization
    bool complex_called_ = false;    // NeoSolver's factored_complex_ flag
    bool complex_factored_ = false;  // the last complex factorization succeeded
    nsg_topology* ctopo_ = nullptr;
    nsg_batch* cbatch_ = nullptr;
    double* d_cax_ = nullptr;
    double* d_clu_ = nullptr;
    double* d_cx_ = nullptr;
    int* d_cstatus_ = nullptr;

    int nnz() const { return static_cast<int>(row_idx_.size()); }

    static void check(int rc, const char* what) {
        if (rc != NSG_OK)
            throw std::runtime_error(std::string("GpuSolver::") + what + ": " + nsg_last_error());
    }
    static void cuda(cudaError_t e, const char* what) {
        if (e != cudaSuccess)
            throw std::runtime_error(std::string("GpuSolver::") + what + ": " +
                                     cudaGetErrorString(e));
    }
    void require_symbolic(const char* what) const {
        if (!symbolized_)
            throw std::logic_error(std::string("GpuSolver::") + what + ": symbolic() not called");
    }
    void check_values(const std::vector<double>& v) const {
        if (static_cast<int>(v.size()) != nnz())
            throw std::invalid_argument("GpuSolver: values size mismatch");
    }
    // The nearest power of two to v in log2 (the boundary is v = 2^k *
    // sqrt(2)/2 below 2^k): scaling by it only moves exponents.  1 for
    // zero, negative or non-finite v.
    static double nearest_pow2(double v) {
        if (!(v > 0.0) || !std::isfinite(v)) return 1.0;
        int e = 0;
        const double m = std::frexp(v, &e);  // v = m * 2^e, m in [0.5, 1)
        return std::ldexp(1.0, m < 0.70710678118654752440 ? e - 1 : e);
    }
    // D_r A D_c with diag_gmin * D_r[i] * D_c[i] added to each diagonal slot:
    // row infinity norms, column norms of the row-scaled matrix, then one
    // refining row pass on the fully scaled one, each rounded to powers of two.
    const std::vector<double>& scaled(const std::vector<double>& a, double diag_gmin) {
        const int nz = nnz();
        dr_.assign(n_, 1.0);
        dc_.assign(n_, 1.0);
        std::vector<double> mx(n_, 0.0);
        for (int k = 0; k < nz; ++k) {
            const double v = std::abs(a[k]);
            if (v > mx[row_idx_[k]]) mx[row_idx_[k]] = v;
        }
        for (int i = 0; i < n_; ++i) dr_[i] = nearest_pow2(mx[i] > 0.0 ? 1.0 / mx[i] : 1.0);
        std::fill(mx.begin(), mx.end(), 0.0);
        for (int k = 0; k < nz; ++k) {
            const double v = std::abs(dr_[row_idx_[k]] * a[k]);
            if (v > mx[col_of_[k]]) mx[col_of_[k]] = v;
        }
        for (int j = 0; j < n_; ++j) dc_[j] = nearest_pow2(mx[j] > 0.0 ? 1.0 / mx[j] : 1.0);
        std::fill(mx.begin(), mx.end(), 0.0);
        for (int k = 0; k < nz; ++k) {
            const double v = std::abs(dr_[row_idx_[k]] * a[k] * dc_[col_of_[k]]);
            if (v > mx[row_idx_[k]]) mx[row_idx_[k]] = v;
        }
        for (int i = 0; i < n_; ++i)
            if (mx[i] > 0.0) dr_[i] *= nearest_pow2(1.0 / mx[i]);
        scaled_.resize(nz);
        for (int k = 0; k < nz; ++k) scaled_[k] = dr_[row_idx_[k]] * a[k] * dc_[col_of_[k]];
        if (diag_gmin != 0.0)
            for (int k = 0; k < nz; ++k)
                if (row_idx_[k] == col_of_[k])
                    scaled_[k] += dr_[row_idx_[k]] * dc_[row_idx_[k]] * diag_gmin;
        return scaled_;
    }
    void check_complex_values(const std::vector<double>& ax) const {
        if (static_cast<int>(ax.size()) != 2 * nnz())
            throw std::invalid_argument("GpuSolver: complex values size must be 2*nnz");
    }
    int gpu_refactor_complex(const std::vector<double>& ax) {
        cuda(cudaMemcpy(d_cax_, ax.data(), sizeof(double) * 2 * nnz(), cudaMemcpyHostToDevice),
             "upload");
        check(nsg_batch_refactor_complex(cbatch_, d_cax_, d_clu_, d_cstatus_, nullptr),
              "refactor_complex");
        int st = 0;
        cuda(cudaMemcpy(&st, d_cstatus_, sizeof(int), cudaMemcpyDeviceToHost), "status");
        if (st == 104) throw std::runtime_error("GpuSolver: complex refactor wait timed out");
        return st;
    }
    void release_complex() {
        if (cbatch_) nsg_batch_free(cbatch_);
        if (ctopo_) nsg_topology_free(ctopo_);
        if (d_cax_) cudaFree(d_cax_);
        if (d_clu_) cudaFree(d_clu_);
        if (d_cx_) cudaFree(d_cx_);
        if (d_cstatus_) cudaFree(d_cstatus_);
        cbatch_ = nullptr;
        ctopo_ = nullptr;
        d_cax_ = d_clu_ = d_cx_ = nullptr;
        d_cstatus_ = nullptr;
        complex_factored_ = false;
    }
    void rebuild_batch() {
        if (batch_) nsg_batch_free(batch_);
        batch_ = nullptr;
        check(nsg_batch_create(1, &topo_, &batch_), "batch");
        if (!d_values_) {
            cuda(cudaMalloc(reinterpret_cast<void**>(&d_values_), sizeof(double) * nnz()), "alloc");
            cuda(cudaMalloc(reinterpret_cast<void**>(&d_x_), sizeof(double) * n_), "alloc");
            cuda(cudaMalloc(reinterpret_cast<void**>(&d_status_), sizeof(int)), "alloc");
        }
    }
    void upload(const std::vector<double>& values) {
        cuda(cudaMemcpy(d_values_, values.data(), sizeof(double) * nnz(), cudaMemcpyHostToDevice),
             "upload");
    }
    int gpu_refactor(double diag_gmin, int check_pivots) {
        check(nsg_batch_refactor(batch_, d_values_, diag_gmin, check_pivots, d_status_, nullptr,
                                 nullptr), "refactor");
        int st = 0;
        cuda(cudaMemcpy(&st, d_status_, sizeof(int), cudaMemcpyDeviceToHost), "status");
        if (st == 104) throw std::runtime_error("GpuSolver: refactor wait timed out");
        return st;
    }
    void sweep(std::vector<double>& rhs, bool transposed) {
        require_symbolic(transposed ? "solve_transposed" : "solve");
        if (!numeric_called_)
            throw std::logic_error("GpuSolver::solve: numeric() not called");
        if (!factored_)
            throw std::runtime_error("GpuSolver::solve: no valid factorization (singular)");
        if (static_cast<int>(rhs.size()) != n_)
            throw std::invalid_argument("GpuSolver::solve: rhs size mismatch");
        cuda(cudaMemcpy(d_x_, rhs.data(), sizeof(double) * n_, cudaMemcpyHostToDevice), "rhs");
        check(transposed ? nsg_batch_solve_transposed(batch_, d_x_, nullptr)
                         : nsg_batch_solve(batch_, d_x_, nullptr), "solve");
        cuda(cudaMemcpy(rhs.data(), d_x_, sizeof(double) * n_, cudaMemcpyDeviceToHost), "result");
    }
    void release() {
        release_complex();
        complex_called_ = false;
        if (batch_) nsg_batch_free(batch_);
        if (topo_) nsg_topology_free(topo_);
        if (d_values_) cudaFree(d_values_);
        if (d_x_) cudaFree(d_x_);
        if (d_status_) cudaFree(d_status_);
        batch_ = nullptr;
        topo_ = nullptr;
        d_values_ = d_x_ = nullptr;
        d_status_ = nullptr;
    }
};

}  // namespace nsgpu
