// ORACLE — test infrastructure only (the checker, never the product).
//
// C entry points around the reference's own psp::DistUniformGrid
// (include/psp/dist_uniform_grid.hpp, compiled unchanged from the reference
// tree with its psp.hpp, against the one-process stand-in for Clique and
// Elemental in clique.hpp), so tests can check
// the numpy restatement in oracle/grid_io.py and the product's grid kernels
// against the reference code itself:
//   SequentialLoad  dist_uniform_grid.hpp:349-482
//   InterpolateTo   dist_uniform_grid.hpp:484-714
//   WritePlane      dist_uniform_grid.hpp:716-1640 (real and complex helpers)
//   WriteVolume     dist_uniform_grid.hpp:1795-2200
// Grids cross this boundary in the one-process buffer layout: natural order
// (x fastest), numScalars entries interleaved per point; complex entries as
// (re, im) double pairs.  Every function returns 0, or 1 with the
// exception's text in ref_grid_error().
#include "clique.hpp"
#include "psp.hpp"

#include <algorithm>
#include <complex>
#include <string>

namespace {

std::string g_error;

template <typename F>
int Guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

template <typename T>
void Fill(psp::DistUniformGrid<T>& g, const T* in) {
    const size_t n = (size_t)g.XLocalSize() * g.YLocalSize() * g.ZLocalSize() * g.NumScalars();
    std::copy(in, in + n, g.Buffer());
}

template <typename T>
void Drain(const psp::DistUniformGrid<T>& g, T* out) {
    const size_t n = (size_t)g.XLocalSize() * g.YLocalSize() * g.ZLocalSize() * g.NumScalars();
    std::copy(g.LockedBuffer(), g.LockedBuffer() + n, out);
}

// The grid in natural order, whatever its storage order: entry (x, y, z) is
// read at the grid's own LocalIndex (dist_uniform_grid.hpp:302-343).
template <typename T>
void DrainNatural(const psp::DistUniformGrid<T>& g, T* out) {
    const int nx = g.XSize(), ny = g.YSize(), nz = g.ZSize(), ns = g.NumScalars();
    const T* b = g.LockedBuffer();
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const int li = g.LocalIndex(x, y, z);
                for (int s = 0; s < ns; ++s) out[((size_t)(z * ny + y) * nx + x) * ns + s] = b[li + s];
            }
}

}  // namespace

extern "C" {

const char* ref_grid_error() { return g_error.c_str(); }

// SequentialLoad of an nx x ny x nz grid of ns scalars stored in GridDataOrder
// `order` (the grid keeps that order in memory); written out in natural order.
int ref_grid_load(const char* path, int nx, int ny, int nz, int ns, int order, int isComplex, double* out) {
    return Guard([&] {
        if (isComplex) {
            psp::DistUniformGrid<std::complex<double>> g(nx, ny, nz, 0, ns, (psp::GridDataOrder)order);
            g.SequentialLoad(path);
            DrainNatural(g, reinterpret_cast<std::complex<double>*>(out));
        } else {
            psp::DistUniformGrid<double> g(nx, ny, nz, 0, ns, (psp::GridDataOrder)order);
            g.SequentialLoad(path);
            DrainNatural(g, out);
        }
    });
}

// InterpolateTo(nx1, ny1, nz1) of a natural-order grid.
int ref_grid_interpolate(const double* in, int nx, int ny, int nz, int ns, int isComplex, int nx1, int ny1, int nz1,
                         double* out) {
    return Guard([&] {
        if (isComplex) {
            psp::DistUniformGrid<std::complex<double>> g(nx, ny, nz, 0, ns);
            Fill(g, reinterpret_cast<const std::complex<double>*>(in));
            g.InterpolateTo(nx1, ny1, nz1);
            Drain(g, reinterpret_cast<std::complex<double>*>(out));
        } else {
            psp::DistUniformGrid<double> g(nx, ny, nz, 0, ns);
            Fill(g, in);
            g.InterpolateTo(nx1, ny1, nz1);
            Drain(g, out);
        }
    });
}

// WritePlane(planeType, which, basename): planeType 0 XY, 1 XZ, 2 YZ.
int ref_grid_write_plane(const double* in, int nx, int ny, int nz, int ns, int isComplex, int planeType, int which,
                         const char* basename) {
    return Guard([&] {
        if (isComplex) {
            psp::DistUniformGrid<std::complex<double>> g(nx, ny, nz, 0, ns);
            Fill(g, reinterpret_cast<const std::complex<double>*>(in));
            g.WritePlane((psp::PlaneType)planeType, which, basename);
        } else {
            psp::DistUniformGrid<double> g(nx, ny, nz, 0, ns);
            Fill(g, in);
            g.WritePlane((psp::PlaneType)planeType, which, basename);
        }
    });
}

int ref_grid_write_volume(const double* in, int nx, int ny, int nz, int ns, int isComplex, const char* basename) {
    return Guard([&] {
        if (isComplex) {
            psp::DistUniformGrid<std::complex<double>> g(nx, ny, nz, 0, ns);
            Fill(g, reinterpret_cast<const std::complex<double>*>(in));
            g.WriteVolume(basename);
        } else {
            psp::DistUniformGrid<double> g(nx, ny, nz, 0, ns);
            Fill(g, in);
            g.WriteVolume(basename);
        }
    });
}

}  // extern "C"
