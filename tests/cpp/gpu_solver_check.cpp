// Drives nsgpu::GpuSolver the way newton_solve drives an ISolver, on the
// known-answer systems of the reference's solver tests
// (tests/unit/test_neo_solver.cpp:15-99) and a banded system; prints one line
// per check and exits non-zero on any failure.
#include "nsgpu_solver.hpp"

#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

static int failures = 0;

static void expect(bool ok, const char* what) {
    std::printf("%s %s\n", ok ? "ok  " : "FAIL", what);
    if (!ok) ++failures;
}

static void dense_pattern(int n, std::vector<int>& cp, std::vector<int>& ri) {
    cp.assign(n + 1, 0);
    ri.clear();
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) ri.push_back(i);
        cp[j + 1] = static_cast<int>(ri.size());
    }
}

int main() {
    std::vector<int> cp, ri;
    {   // [2 1; 1 3] x = [5; 7] -> [1.6; 1.8]; then refactor [4 2; 1 5] x = [14; 17] -> [2; 3]
        dense_pattern(2, cp, ri);
        nsgpu::GpuSolver s;
        s.symbolic(2, cp, ri);
        expect(!s.numeric({2.0, 1.0, 1.0, 3.0}), "2x2 numeric");
        std::vector<double> b = {5.0, 7.0};
        s.solve(b);
        expect(std::fabs(b[0] - 1.6) < 1e-10 && std::fabs(b[1] - 1.8) < 1e-10, "2x2 solve");
        expect(!s.refactorize({4.0, 1.0, 2.0, 5.0}), "2x2 refactorize");
        b = {14.0, 17.0};
        s.solve(b);
        expect(std::fabs(b[0] - 2.0) < 1e-10 && std::fabs(b[1] - 3.0) < 1e-10, "2x2 refactor solve");
        // A^T x = b with A = [4 2; 1 5]: [4 1; 2 5] x = [6; 12] -> [1; 2]
        b = {6.0, 12.0};
        s.solve_transposed(b);
        expect(std::fabs(b[0] - 1.0) < 1e-10 && std::fabs(b[1] - 2.0) < 1e-10, "2x2 transposed");
        // later numeric() re-validates on the GPU
        expect(!s.numeric({2.0, 1.0, 1.0, 3.0}), "2x2 second numeric");
        b = {5.0, 7.0};
        s.solve(b);
        expect(std::fabs(b[0] - 1.6) < 1e-10, "2x2 solve after re-validation");
    }
    {   // diag 10, off-diagonal 1, x_true = 1..5
        dense_pattern(5, cp, ri);
        std::vector<double> v;
        for (int j = 0; j < 5; ++j)
            for (int i = 0; i < 5; ++i) v.push_back(i == j ? 10.0 : 1.0);
        nsgpu::GpuSolver s;
        s.symbolic(5, cp, ri);
        expect(!s.numeric(v), "5x5 numeric");
        std::vector<double> b(5, 0.0);
        for (int i = 0; i < 5; ++i)
            for (int j = 0; j < 5; ++j) b[i] += (i == j ? 10.0 : 1.0) * (j + 1);
        s.solve(b);
        double err = 0;
        for (int i = 0; i < 5; ++i) err = std::fmax(err, std::fabs(b[i] - (i + 1)));
        expect(err < 1e-10, "5x5 solve");
    }
    {   // misuse and singular conventions
        nsgpu::GpuSolver s;
        bool threw = false;
        std::vector<double> b = {1.0};
        try { s.solve(b); } catch (const std::logic_error&) { threw = true; }
        expect(threw, "solve before symbolic throws logic_error");
        dense_pattern(2, cp, ri);
        s.symbolic(2, cp, ri);
        threw = false;
        try { s.refactorize({1.0, 0.0, 0.0, 1.0}); } catch (const std::logic_error&) { threw = true; }
        expect(threw, "refactorize before numeric throws logic_error");
        expect(!s.numeric({1.0, 0.0, 0.0, 1.0}), "identity numeric");
        threw = false;
        b = {1.0};
        try { s.solve(b); } catch (const std::invalid_argument&) { threw = true; }
        expect(threw, "rhs size mismatch throws invalid_argument");
        expect(s.refactorize({0.0, 0.0, 0.0, 1.0}), "zero pivot refactorize reports singular");
    }
    {   // AMD-LU engine: the reference's AmdLuSolver unit cases
        // (tests/unit/test_amd_lu.cpp): a row pivot on a zero diagonal, and a
        // refactorize whose reused pivot fails the growth test.
        cp = {0, 1, 3};
        ri = {1, 0, 1};  // [0 1; 1 1]
        nsgpu::GpuSolver s(NSG_SOLVER_AMDLU);
        s.symbolic(2, cp, ri);
        expect(!s.numeric({1.0, 1.0, 1.0}), "amdlu 2x2 zero-diagonal numeric");
        std::vector<double> b = {1.0, 2.0};
        s.solve(b);
        expect(std::fabs(b[0] - 1.0) < 1e-12 && std::fabs(b[1] - 1.0) < 1e-12, "amdlu 2x2 solve");
        expect(std::string(s.name()) == "gpu-amdlu", "amdlu name");
        dense_pattern(3, cp, ri);
        const double a0[3][3] = {{10, 1, 2}, {1, 12, 3}, {2, 1, 15}};
        const double a1[3][3] = {{1e-12, 1, 2}, {1, 12, 3}, {2, 1, 15}};
        std::vector<double> v0, v1;
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                v0.push_back(a0[i][j]);
                v1.push_back(a1[i][j]);
            }
        nsgpu::GpuSolver t(NSG_SOLVER_AMDLU);
        t.symbolic(3, cp, ri);
        expect(!t.numeric(v0), "amdlu 3x3 numeric");
        expect(!t.refactorize(v1), "amdlu 3x3 refactorize with growth fallback");
        const double xt[3] = {2.0, -1.0, 0.5};
        b.assign(3, 0.0);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) b[i] += a1[i][j] * xt[j];
        t.solve(b);
        double err = 0;
        for (int i = 0; i < 3; ++i) err = std::fmax(err, std::fabs(b[i] - xt[i]));
        expect(err < 1e-7, "amdlu 3x3 solve after fallback");
        // structurally singular: the auto engine falls back to Markowitz,
        // which reports singular as well
        cp = {0, 2, 2};
        ri = {0, 1};
        nsgpu::GpuSolver u(NSG_SOLVER_AUTO_AMDLU);
        u.symbolic(2, cp, ri);
        expect(u.numeric({1.0, 1.0}), "auto engine structurally singular numeric");
        expect(nsg_solver_select(300, 1) == NSG_SOLVER_AUTO_AMDLU &&
                   nsg_solver_select(300, 0) == NSG_SOLVER_MARKOWITZ &&
                   nsg_solver_select(255, 1) == NSG_SOLVER_MARKOWITZ,
               "make_solver policy");
    }
    std::printf("%d failure(s)\n", failures);
    return failures == 0 ? 0 : 1;
}
