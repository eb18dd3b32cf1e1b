#include "ritz.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>

namespace psp_b200 {

namespace {

typedef std::complex<double> Cd;

// [c s; -conj(s) c] [f; g] = [r; 0] with c real and non-negative.
void Rotation(Cd f, Cd g, double& c, Cd& s) {
    const double af = std::abs(f), ag = std::abs(g);
    if (ag == 0) { c = 1; s = 0; return; }
    if (af == 0) { c = 0; s = std::conj(g) / ag; return; }
    const double nrm = std::hypot(af, ag);
    c = af / nrm;
    s = (f / af) * std::conj(g) / nrm;
}

}  // namespace

// Explicitly shifted QR iteration on the unreduced trailing window [l, hi]
// of the Hessenberg matrix, scaled by a power of two to unit size (Golub &
// Van Loan, Matrix Computations, 4th ed., 7.5): H - mu I = QR by Givens
// rotations, H := RQ + mu I.  The shift is the
// eigenvalue of the trailing 2x2 block closer to its last diagonal entry
// (Wilkinson), replaced by an ad hoc shift after 10 and 20 sweeps without a
// deflation.  A subdiagonal entry deflates when it is below the unit
// roundoff times its two diagonal neighbours; only the window is updated,
// since the eigenvalues alone are wanted.
std::vector<Cd> HessenbergEigenvalues(int n, const Cd* H, int ldh) {
    if (n < 0) throw std::logic_error("Hessenberg order must be non-negative");
    if (n > 0 && (!H || ldh < n)) throw std::logic_error("Hessenberg matrix needs ldh >= n");
    std::vector<Cd> A((size_t)n * n, Cd(0));
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= std::min(j + 1, n - 1); ++i) A[(size_t)j * n + i] = H[(size_t)j * ldh + i];
    auto a = [&](int i, int j) -> Cd& { return A[(size_t)j * n + i]; };
    double amax = 0;
    for (const Cd& v : A) {
        if (!std::isfinite(v.real()) || !std::isfinite(v.imag()))
            throw std::runtime_error("Hessenberg matrix has a non-finite entry");
        amax = std::max({amax, std::abs(v.real()), std::abs(v.imag())});
    }
    // Work on H / 2^e with the largest entry near 1 (exact: a power of two),
    // so that the shifts' products neither overflow nor underflow.
    const int e = amax > 0 ? std::ilogb(amax) : 0;
    if (e != 0)
        for (Cd& v : A) v = Cd(std::ldexp(v.real(), -e), std::ldexp(v.imag(), -e));

    std::vector<Cd> w(n);
    std::vector<double> cs(n);
    std::vector<Cd> sn(n);
    const double eps = std::numeric_limits<double>::epsilon();
    const double tiny = std::numeric_limits<double>::min() * (n / eps);
    const int maxSweeps = 30 * std::max(10, n);
    int hi = n - 1, stall = 0;
    while (hi >= 0) {
        int l = hi;
        for (; l > 0; --l) {
            const double sub = std::abs(a(l, l - 1));
            double ref = std::abs(a(l - 1, l - 1)) + std::abs(a(l, l));
            if (ref == 0)
                for (int i = l - 1; i <= hi; ++i) ref += std::abs(a(i, i));
            if (sub <= tiny || sub <= eps * ref) {
                a(l, l - 1) = 0;
                break;
            }
        }
        if (l == hi) {
            w[hi] = a(hi, hi);
            --hi;
            stall = 0;
            continue;
        }
        if (++stall > maxSweeps) throw std::runtime_error("Hessenberg QR iteration did not converge");
        Cd mu;
        if (stall % 10 == 0) {
            mu = a(hi, hi) + 0.75 * std::abs(a(hi, hi - 1));
        } else {
            const Cd p = a(hi - 1, hi - 1), q = a(hi - 1, hi), r = a(hi, hi - 1), s = a(hi, hi);
            // eigenvalues s + t +- d, t = (p - s)/2, d^2 = t^2 + q r; the one
            // nearer s is -q r / (t +- d) with the larger denominator.
            const Cd t = 0.5 * (p - s), d = std::sqrt(t * t + q * r);
            const Cd big = (std::real(std::conj(t) * d) >= 0) ? t + d : t - d;
            mu = (std::abs(big) == 0) ? s : s - q * r / big;
        }
        for (int i = l; i <= hi; ++i) a(i, i) -= mu;
        for (int k = l; k < hi; ++k) {
            Rotation(a(k, k), a(k + 1, k), cs[k], sn[k]);
            const double c = cs[k];
            const Cd s = sn[k];
            for (int j = k; j <= hi; ++j) {
                const Cd x = a(k, j), y = a(k + 1, j);
                a(k, j) = c * x + s * y;
                a(k + 1, j) = -std::conj(s) * x + c * y;
            }
            a(k + 1, k) = 0;
        }
        for (int k = l; k < hi; ++k) {
            const double c = cs[k];
            const Cd s = sn[k];
            for (int i = l; i <= k + 1; ++i) {
                const Cd x = a(i, k), y = a(i, k + 1);
                a(i, k) = x * c + y * std::conj(s);
                a(i, k + 1) = -x * s + y * c;
            }
        }
        for (int i = l; i <= hi; ++i) a(i, i) += mu;
    }
    if (e != 0)
        for (Cd& v : w) v = Cd(std::ldexp(v.real(), e), std::ldexp(v.imag(), e));
    return w;
}

}  // namespace psp_b200
