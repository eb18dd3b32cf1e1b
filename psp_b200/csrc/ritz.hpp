// Ritz values of the GMRES Hessenberg matrix (the PRINT_RITZ_VALUES
// diagnostic of PSP include/psp/dist_helmholtz/solve.hpp:589-608).
#pragma once
#include <complex>
#include <vector>

namespace psp_b200 {

// Eigenvalues of the n x n complex upper Hessenberg matrix H (column-major,
// leading dimension ldh; entries below the first subdiagonal are ignored):
// the counterpart of Elemental's lapack::HessenbergEig (LAPACK zhseqr,
// eigenvalues only) called at solve.hpp:597-598.  Throws std::logic_error
// for bad sizes and std::runtime_error when the QR iteration does not
// converge.
std::vector<std::complex<double>> HessenbergEigenvalues(int n, const std::complex<double>* H, int ldh);

}  // namespace psp_b200
