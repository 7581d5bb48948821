// Test infrastructure only: the reference's own analyses running on this
// repository's GPU solver through the reference's solver seam.
//
// GpuNeoSolver below is the ISolver adapter a maintainer adds to the
// reference (src/core/solver_iface.hpp:16-41) to put libnsgpu under its
// Newton loop.  This file is linked (oracle/Makefile, target `seam`) with the
// reference's own objects into oracle/_ref/libnsseam.so, with make_solver's
// definition renamed in its object file to reference_make_solver, so that
// the make_solver below is the one solve_dc (src/core/dc.cpp:80),
// solve_transient (src/core/transient.cpp:713-727) and every other caller
// reach: with the GPU seam switched on it returns a GpuNeoSolver on the
// engine the reference would pick (nsg_solver_select = make_solver's
// policy); switched off, the reference's own solver.  The tests then compare
// the reference's analyses on both engines.
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <utility>
#include <vector>

#include "core/matrix.hpp"
#include "core/neo_solver.hpp"
#include "core/solver_iface.hpp"
#include "nsgpu_solver.hpp"

namespace neospice {

// make_solver of src/core/make_solver.cpp:156-178, renamed at link time.
std::unique_ptr<ISolver> reference_make_solver(int num_vars, bool is_linear);

namespace {

long long g_gpu_solvers = 0;  // GpuNeoSolver objects created
bool g_gpu_seam = false;

class GpuNeoSolver : public ISolver {
public:
    explicit GpuNeoSolver(int engine) : gpu_(engine) { ++g_gpu_solvers; }

    void symbolic(const SparsityPattern& pattern) override {
        CSCData csc = pattern.to_csc();
        gpu_.symbolic(pattern.size(), csc.col_ptr, csc.row_idx);
        nnz_ = pattern.nnz();
    }
    bool numeric(const SparsityPattern&, const NumericMatrix& mat, double diag_gmin) override {
        return gpu_.numeric(values(mat), diag_gmin);  // true = singular, as NeoSolver
    }
    bool refactorize(const NumericMatrix& mat, double diag_gmin) override {
        return gpu_.refactorize(values(mat), diag_gmin);
    }
    void solve(std::vector<double>& rhs) override { gpu_.solve(rhs); }
    // Row/column equilibration (solve_dc's last aid, dc.cpp:355-387): the
    // scaled matrix is factored on the GPU; only the Markowitz engine honors
    // it, as only NeoSolver does in the reference.
    void set_equilibrate(bool on) override { gpu_.set_equilibrate(on); }
    // Complex (AC): Markowitz ordering on the host, factor and sweeps on the
    // GPU (the reference's AC uses NeoSolver whatever the circuit).
    void numeric_complex(const SparsityPattern&, const std::vector<double>& ax) override {
        gpu_.numeric_complex(ax);
    }
    bool refactorize_complex(const std::vector<double>& ax) override {
        return gpu_.refactorize_complex(ax);
    }
    void solve_complex(std::vector<double>& rhs) override { gpu_.solve_complex(rhs); }
    const char* name() const override { return gpu_.name(); }

private:
    std::vector<double> values(const NumericMatrix& m) const {
        return std::vector<double>(m.data(), m.data() + nnz_);
    }
    nsgpu::GpuSolver gpu_;
    int nnz_ = 0;
};

}  // namespace

std::unique_ptr<ISolver> make_solver(int num_vars, bool is_linear) {
    if (g_gpu_seam)
        return std::make_unique<GpuNeoSolver>(nsg_solver_select(num_vars, is_linear ? 1 : 0));
    return reference_make_solver(num_vars, is_linear);
}

}  // namespace neospice

extern "C" {

// Route every make_solver of the reference through GpuNeoSolver (on != 0)
// or back to its own solvers.
void nsseam_use_gpu(int on) { neospice::g_gpu_seam = on != 0; }

// GpuNeoSolver objects created so far (proof that the seam was used).
long long nsseam_gpu_solvers(void) { return neospice::g_gpu_solvers; }

// numeric() on values[0] and refactorize() on values[1..npoints-1], each
// followed by solve() of rhs, through whatever ISolver make_solver returns,
// with equilibration on (equilibrate != 0) as solve_dc's last aid switches
// it on; out receives n doubles per point, singular[f] each call's verdict.
// Returns 0, or -1 when the solver threw.
int nsseam_solve_sequence(int n, int nnz, const int* col_ptr, const int* row_idx,
                          const double* values, const double* rhs, int npoints, double diag_gmin,
                          int equilibrate, int is_linear, double* out, int* singular) {
    try {
        std::vector<std::pair<int32_t, int32_t>> entries;
        entries.reserve(nnz);
        for (int j = 0; j < n; ++j)
            for (int k = col_ptr[j]; k < col_ptr[j + 1]; ++k) entries.emplace_back(row_idx[k], j);
        neospice::SparsityPattern pattern(n, std::move(entries));
        auto solver = neospice::make_solver(n, is_linear != 0);
        solver->symbolic(pattern);
        solver->set_equilibrate(equilibrate != 0);
        neospice::NumericMatrix mat(pattern);
        std::vector<double> z(n);
        for (int f = 0; f < npoints; ++f) {
            std::memcpy(mat.data(), values + static_cast<size_t>(nnz) * f, sizeof(double) * nnz);
            singular[f] = (f == 0 ? solver->numeric(pattern, mat, diag_gmin)
                                  : solver->refactorize(mat, diag_gmin)) ? 1 : 0;
            z.assign(rhs, rhs + n);
            if (!singular[f]) solver->solve(z);
            std::memcpy(out + static_cast<size_t>(n) * f, z.data(), sizeof(double) * n);
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// An AC sweep through whatever ISolver make_solver returns, with the
// per-frequency steps of solve_ac (src/core/ac.cpp:196-216): ax = G + j*omega*C
// in interleaved CSC order, numeric_complex at the first point and
// refactorize_complex after, solve_complex of the excitation.  out receives
// 2*n doubles per point; singular[f] the refactor's verdict (0 at f = 0).
// Returns 0, or -1 when the solver threw.
int nsseam_ac_sweep(int n, int nnz, const int* col_ptr, const int* row_idx, const double* g,
                    const double* c, const double* rhs, int npoints, const double* omega,
                    double* out, int* singular) {
    try {
        std::vector<std::pair<int32_t, int32_t>> entries;
        entries.reserve(nnz);
        for (int j = 0; j < n; ++j)
            for (int k = col_ptr[j]; k < col_ptr[j + 1]; ++k) entries.emplace_back(row_idx[k], j);
        neospice::SparsityPattern pattern(n, std::move(entries));
        auto solver = neospice::make_solver(n, false);
        solver->symbolic(pattern);
        std::vector<double> ax(2 * static_cast<size_t>(nnz));
        std::vector<double> z(2 * static_cast<size_t>(n));
        for (int f = 0; f < npoints; ++f) {
            for (int k = 0; k < nnz; ++k) {
                ax[2 * k] = g[k];
                ax[2 * k + 1] = omega[f] * c[k];
            }
            singular[f] = 0;
            if (f == 0) solver->numeric_complex(pattern, ax);
            else singular[f] = solver->refactorize_complex(ax) ? 1 : 0;
            z.assign(rhs, rhs + 2 * static_cast<size_t>(n));
            solver->solve_complex(z);
            std::memcpy(out + 2 * static_cast<size_t>(n) * f, z.data(), sizeof(double) * z.size());
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
