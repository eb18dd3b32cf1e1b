// psp::Discretization / psp::DistUniformGrid / psp::DistHelmholtz for one
// B200, header-only over the C ABI of libpsp_b200.so (include/psp_b200.h).
//
// Mirrors the reference's C++ surface (include/psp/discretization.hpp,
// dist_uniform_grid.hpp, dist_helmholtz.hpp) so that a driver written against
// it keeps compiling: the MPI communicator argument becomes a CUDA device
// index, every grid is owned by the single process (px = py = pz = 1), and the
// reference's std::logic_error / std::runtime_error conventions are kept.
#pragma once

#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../psp_b200.h"

namespace psp {

template <typename R>
using Complex = std::complex<R>;

enum Boundary { PML = PSP_CU_PML, DIRICHLET = PSP_CU_DIRICHLET };
enum PanelScheme { CLIQUE_LDL_1D = PSP_CU_LDL_1D, CLIQUE_LDL_SELINV_1D = PSP_CU_LDL_SELINV_1D };
enum Precision { FP64 = PSP_CU_FP64, MIXED = PSP_CU_MIXED };
enum GridDataOrder { XYZ, XZY, YXZ, YZX, ZXY, ZYX };
enum PlaneType { XY, XZ, YZ };  // dist_uniform_grid.hpp:24-28

namespace detail {
inline void Check(int code) {
    if (code == PSP_CU_OK) return;
    const std::string msg = psp_cu_last_error();
    if (code == PSP_CU_LOGIC_ERROR) throw std::logic_error(msg);
    throw std::runtime_error(msg);
}
}  // namespace detail

// Initialize/Finalize of the reference (src/global.cpp:23-51) had MPI and
// Clique to bring up; here there is nothing global to set up.
inline void Initialize(int&, char**&) {}
inline void Finalize() {}

// Discretization<R> (discretization.hpp:36-110); widths are those of the
// PML-padded box.
template <typename Real>
struct Discretization {
    Real omega;
    int nx, ny, nz;
    Real wx, wy, wz;
    Boundary frontBC, rightBC, backBC, leftBC, topBC;
    int bx, by, bz;
    Real sigmax, sigmay, sigmaz;

    Discretization(Real frequency, int xSize, int ySize, int zSize, Real xWidth, Real yWidth, Real zWidth)
        : Discretization(frequency, xSize, ySize, zSize, xWidth, yWidth, zWidth, PML, PML, PML, PML, PML) {}
    Discretization(Real frequency, int xSize, int ySize, int zSize, Real xWidth, Real yWidth, Real zWidth,
                   Boundary front, Boundary right, Boundary back, Boundary left, Boundary top)
        : Discretization(frequency, xSize, ySize, zSize, xWidth, yWidth, zWidth, front, right, back, left, top, 5,
                         5, 5) {}
    Discretization(Real frequency, int xSize, int ySize, int zSize, Real xWidth, Real yWidth, Real zWidth,
                   Boundary front, Boundary right, Boundary back, Boundary left, Boundary top, int xPML, int yPML,
                   int zPML)
        : omega(frequency), nx(xSize), ny(ySize), nz(zSize), wx(xWidth), wy(yWidth), wz(zWidth),
          frontBC(front), rightBC(right), backBC(back), leftBC(left), topBC(top), bx(xPML), by(yPML), bz(zPML) {
        const Real maxDim = std::max(wx, std::max(wy, wz));
        sigmax = sigmay = sigmaz = Real(1.2) * maxDim;
    }
    Discretization(Real frequency, int xSize, int ySize, int zSize, Real xWidth, Real yWidth, Real zWidth,
                   Boundary front, Boundary right, Boundary back, Boundary left, Boundary top, int pmlSize,
                   double sigma)
        : omega(frequency), nx(xSize), ny(ySize), nz(zSize), wx(xWidth), wy(yWidth), wz(zWidth),
          frontBC(front), rightBC(right), backBC(back), leftBC(left), topBC(top), bx(pmlSize), by(pmlSize),
          bz(pmlSize), sigmax(sigma), sigmay(sigma), sigmaz(sigma) {}

    psp_cu_disc ToC() const {
        psp_cu_disc d;
        d.omega = omega;
        d.nx = nx; d.ny = ny; d.nz = nz;
        d.wx = wx; d.wy = wy; d.wz = wz;
        d.frontBC = frontBC; d.rightBC = rightBC; d.backBC = backBC; d.leftBC = leftBC; d.topBC = topBC;
        d.bx = bx; d.by = by; d.bz = bz;
        d.sigmax = sigmax; d.sigmay = sigmay; d.sigmaz = sigmaz;
        return d;
    }
};

// DistUniformGrid<F> for one process (dist_uniform_grid.hpp:48-145): the
// local buffer is the whole grid, x fastest, numScalars entries per point.
template <typename F>
class DistUniformGrid {
public:
    // The buffer is always held in natural (XYZ) order; `order` is the layout
    // of the files SequentialLoad reads (dist_uniform_grid.hpp:349-482).
    DistUniformGrid(int nx, int ny, int nz, int /*device*/ = 0, int numScalars = 1, GridDataOrder order = XYZ)
        : nx_(nx), ny_(ny), nz_(nz), numScalars_(numScalars), order_(order),
          data_((size_t)nx * ny * nz * numScalars) {}

    // SequentialLoad (dist_uniform_grid.hpp:349-482): the file, stored in the
    // grid's order, reordered on the GPU into this buffer.
    void SequentialLoad(const std::string& filename) {
        detail::Check(psp_cu_grid_load(filename.c_str(), nx_, ny_, nz_, numScalars_, kComplex, order_,
                                       reinterpret_cast<double*>(data_.data())));
    }
    // InterpolateTo (dist_uniform_grid.hpp:484-714), computed on the GPU.
    void InterpolateTo(int nx, int ny, int nz) {
        if (nx == nx_ && ny == ny_ && nz == nz_) return;
        std::vector<F> out((size_t)nx * ny * nz * numScalars_);
        detail::Check(psp_cu_grid_interpolate(reinterpret_cast<const double*>(data_.data()), nx_, ny_, nz_,
                                              numScalars_, kComplex, reinterpret_cast<double*>(out.data()), nx,
                                              ny, nz));
        data_.swap(out);
        nx_ = nx;
        ny_ = ny;
        nz_ = nz;
    }
    // WritePlane / WriteVolume (dist_uniform_grid.hpp:716-2200): ASCII VTK.
    void WritePlane(PlaneType planeType, int whichPlane, const std::string& basename) const {
        detail::Check(psp_cu_grid_write_plane(reinterpret_cast<const double*>(data_.data()), nx_, ny_, nz_,
                                              numScalars_, kComplex, planeType, whichPlane, basename.c_str()));
    }
    void WriteVolume(const std::string& basename) const {
        detail::Check(psp_cu_grid_write_volume(reinterpret_cast<const double*>(data_.data()), nx_, ny_, nz_,
                                               numScalars_, kComplex, basename.c_str()));
    }
    int XSize() const { return nx_; }
    int YSize() const { return ny_; }
    int ZSize() const { return nz_; }
    int NumScalars() const { return numScalars_; }
    int XShift() const { return 0; }
    int YShift() const { return 0; }
    int ZShift() const { return 0; }
    int XStride() const { return 1; }
    int YStride() const { return 1; }
    int ZStride() const { return 1; }
    int XLocalSize() const { return nx_; }
    int YLocalSize() const { return ny_; }
    int ZLocalSize() const { return nz_; }
    int OwningProcess(int, int, int) const { return 0; }
    int NaturalIndex(int x, int y, int z) const { return x + y * nx_ + z * nx_ * ny_; }
    int LocalIndex(int x, int y, int z) const { return NaturalIndex(x, y, z) * numScalars_; }
    F* Buffer() { return data_.data(); }
    const F* LockedBuffer() const { return data_.data(); }
    GridDataOrder Order() const { return order_; }

private:
    static constexpr int kComplex = sizeof(F) == 2 * sizeof(double) ? 1 : 0;
    int nx_, ny_, nz_, numScalars_;
    GridDataOrder order_;
    std::vector<F> data_;
};

// DistHelmholtz<double> (dist_helmholtz.hpp:21-287) on one GPU.
template <typename R>
class DistHelmholtz {
    static_assert(sizeof(R) == sizeof(double), "the solver takes double-precision inputs");

public:
    typedef Complex<R> C;

    DistHelmholtz(const Discretization<R>& disc, int device = 0, R damping = 7.0, int numPlanesPerPanel = 4,
                  int cutoff = 12)
        : disc_(disc) {
        const psp_cu_disc d = disc.ToC();
        detail::Check(psp_cu_create(&d, damping, numPlanesPerPanel, cutoff, device, &h_));
    }
    ~DistHelmholtz() { psp_cu_destroy(h_); }
    DistHelmholtz(const DistHelmholtz&) = delete;
    DistHelmholtz& operator=(const DistHelmholtz&) = delete;

    void Initialize(const DistUniformGrid<R>& velocity, PanelScheme panelScheme = CLIQUE_LDL_SELINV_1D,
                    Precision precision = FP64) {
        if (velocity.XSize() != disc_.nx || velocity.YSize() != disc_.ny || velocity.ZSize() != disc_.nz)
            throw std::logic_error("Velocity grid is incorrect");
        if (velocity.NumScalars() != 1) throw std::logic_error("Velocity grid should have one entry per point");
        detail::Check(psp_cu_initialize(h_, velocity.LockedBuffer(), panelScheme, precision));
    }

    // Solves in place: the numScalars right-hand sides of B become solutions.
    // viewIterates writes the iterate of every inner step that does not
    // converge as iterates-<it> with WriteVolume (solve.hpp:579-585).
    psp_cu_stats Solve(DistUniformGrid<C>& B, int m = 20, R relTol = 1e-4, bool viewIterates = false) const {
        psp_cu_stats st;
        if (viewIterates) detail::Check(psp_cu_set_view_iterates(h_, "iterates"));
        const int e = psp_cu_solve(h_, reinterpret_cast<double*>(B.Buffer()), B.NumScalars(), m, relTol, &st);
        if (viewIterates) psp_cu_set_view_iterates(h_, nullptr);
        detail::Check(e);
        return st;
    }

    // The reference's PRINT_RITZ_VALUES build option as a run-time switch
    // (0 off, 1 record, 2 record and print), and the recorded Ritz values of
    // the first restart cycle of the last Solve: right-hand side r's at
    // [r * count + s], count = the cycle's inner steps.
    void SetRitzValues(int mode) { detail::Check(psp_cu_set_ritz_values(h_, mode)); }
    std::vector<C> RitzValues(int* count = nullptr) const {
        int c = 0, k = 0;
        detail::Check(psp_cu_get_ritz_values(h_, &c, &k, nullptr));
        std::vector<C> out((size_t)c * k);
        if (!out.empty()) detail::Check(psp_cu_get_ritz_values(h_, &c, &k, reinterpret_cast<double*>(out.data())));
        if (count) *count = c;
        return out;
    }
    psp_cu_stats SolveWithGMRES(DistUniformGrid<C>& B, int m = 20, R relTol = 1e-4) const {
        return Solve(B, m, relTol);
    }

    void Finalize() { detail::Check(psp_cu_finalize(h_)); }
    psp_cu_handle* handle() const { return h_; }

private:
    Discretization<R> disc_;
    psp_cu_handle* h_ = nullptr;
};

}  // namespace psp
