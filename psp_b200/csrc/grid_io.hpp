// Grid ingest and output of psp::DistUniformGrid on one process
// (PSP include/psp/dist_uniform_grid.hpp): the velocity model enters the
// solver from a binary file, optionally resampled, and fields leave as VTK
// ImageData files.
//
// A grid is nx x ny x nz points with `scalars` values per point (complex
// values are two doubles), in natural order (x fastest, then y, then z)
// unless stated otherwise.
#pragma once
#include <string>

namespace psp_b200 {

// GridDataOrder (dist_uniform_grid.hpp:15-22): the file layout's axes from
// fastest to slowest.
enum GridOrder { kXYZ = 0, kXZY, kYXZ, kYZX, kZXY, kZYX };
// PlaneType (dist_uniform_grid.hpp:24-28).
enum GridPlane { kPlaneXY = 0, kPlaneXZ, kPlaneYZ };

// SequentialLoad (dist_uniform_grid.hpp:349-482): reads the file (stored in
// `order`, `doubles` doubles per point) and writes the grid in natural order
// to d_out (device, current device), reordering on the device.
void GridLoad(const std::string& filename, int nx, int ny, int nz, int doubles, int order, double* d_out);

// InterpolateTo (dist_uniform_grid.hpp:484-714): trilinear resampling of
// d_in (device, old sizes) to d_out (device, new sizes), `doubles` doubles per
// point, each component interpolated independently (as the reference does
// for real and complex scalars alike).  Equal sizes copy.
void GridInterpolate(const double* d_in, int nxOld, int nyOld, int nzOld, int doubles, double* d_out, int nx,
                     int ny, int nz);

// WritePlane (dist_uniform_grid.hpp:716-1631) and WriteVolume (1788-2200)
// from host data in natural order: one ASCII .vti file per scalar (complex:
// a _real and an _imag file), numbers formatted as the reference's streams
// format them.  WriteVolume writes the one-process layout: a .pvti
// description per scalar whose single piece is basename_k/0.vti.
void GridWritePlane(const double* data, int nx, int ny, int nz, int scalars, bool isComplex, int plane, int which,
                    const std::string& basename);
void GridWriteVolume(const double* data, int nx, int ny, int nz, int scalars, bool isComplex,
                     const std::string& basename);

}  // namespace psp_b200
