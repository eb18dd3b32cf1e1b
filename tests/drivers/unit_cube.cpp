// Unit-cube driver written against the reference's C++ surface
// (psp::Discretization, psp::DistUniformGrid, psp::DistHelmholtz), in the
// style of the reference's tests/UnitCube.cpp: a converging-lens velocity,
// Gaussian point sources, timed Initialize and Solve.
//
//   unit_cube [n] [omega] [precision 0|1] [m] [relTol] [diagnostics]
//
// diagnostics: bit 0 solves with viewIterates (iterates-<it> volumes in the
// working directory), bit 1 prints the first-cycle Ritz values as the
// reference's PRINT_RITZ_VALUES build does.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "psp/psp.hpp"

int main(int argc, char** argv) {
    using namespace psp;
    typedef Complex<double> C;
    const int n = argc > 1 ? std::atoi(argv[1]) : 30;
    const double omega = argc > 2 ? std::atof(argv[2]) : 15.0;
    const Precision prec = (argc > 3 && std::atoi(argv[3]) == 1) ? MIXED : FP64;
    const int m = argc > 4 ? std::atoi(argv[4]) : 20;
    const double relTol = argc > 5 ? std::atof(argv[5]) : 1e-5;
    const int diagnostics = argc > 6 ? std::atoi(argv[6]) : 0;
    try {
        Discretization<double> disc(omega, n, n, n, 1., 1., 1., PML, PML, PML, PML, PML, 5, 1.5);
        DistHelmholtz<double> helmholtz(disc);

        DistUniformGrid<double> velocity(n, n, n);
        double* v = velocity.Buffer();
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) {
                    const double X = x / (n + 1.0), Y = y / (n + 1.0), Z = z / (n + 1.0);
                    const double r2 = (X - 0.5) * (X - 0.5) + (Y - 0.5) * (Y - 0.5) + (Z - 0.5) * (Z - 0.5);
                    v[x + y * n + z * n * n] = 0.95 - 0.4 * std::exp(-32. * r2);  // converging lens
                }
        const auto t0 = std::chrono::steady_clock::now();
        helmholtz.Initialize(velocity, CLIQUE_LDL_SELINV_1D, prec);
        const double tInit = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

        const int k = 2;
        DistUniformGrid<C> B(n, n, n, 0, k);
        C* b = B.Buffer();
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) {
                    const double X = x / (n + 1.0), Y = y / (n + 1.0), Z = z / (n + 1.0);
                    const double a0 = (X - .5) * (X - .5) + (Y - .5) * (Y - .5) + (Z - .1) * (Z - .1);
                    const double a1 = (X - .25) * (X - .25) + (Y - .25) * (Y - .25) + (Z - .1) * (Z - .1);
                    const int i = B.LocalIndex(x, y, z);
                    b[i + 0] = -n * std::exp(-10. * n * a0);
                    b[i + 1] = -n * std::exp(-10. * n * a1);
                }
        if (diagnostics & 2) helmholtz.SetRitzValues(2);
        const auto t1 = std::chrono::steady_clock::now();
        const psp_cu_stats st = helmholtz.Solve(B, m, relTol, (diagnostics & 1) != 0);
        const double tSolve = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
        double norm = 0;
        for (int i = 0; i < n * n * n * k; ++i) norm += std::norm(b[i]);
        std::printf("n=%d init %.3f s solve %.3f s iterations %d converged %d resid %.3e |x| %.6e\n", n, tInit,
                    tSolve, st.iterations, st.converged, st.final_max_rel_resid, std::sqrt(norm));
        helmholtz.Finalize();
        return st.converged ? 0 : 2;
    } catch (std::exception& e) {
        std::fprintf(stderr, "exception: %s\n", e.what());
        return 1;
    }
}
