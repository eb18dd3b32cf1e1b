// Grid ingest (device kernels) and VTK output (host) of psp::DistUniformGrid
// on one process; see grid_io.hpp.
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <vector>

#include "common.cuh"
#include "grid_io.hpp"

namespace psp_b200 {

namespace {

constexpr int kIoThreads = 256;

// Offset (in points) of natural point (x, y, z) in a file stored in `order`
// (the index expressions of SequentialLoad, dist_uniform_grid.hpp:360-478).
__device__ __forceinline__ int64_t FileIndex(int order, int64_t x, int64_t y, int64_t z, int64_t nx, int64_t ny,
                                             int64_t nz) {
    switch (order) {
        case kXZY: return x + z * nx + y * nx * nz;
        case kYXZ: return y + x * ny + z * nx * ny;
        case kYZX: return y + z * ny + x * ny * nz;
        case kZXY: return z + x * nz + y * nz * nx;
        case kZYX: return z + y * nz + x * nz * ny;
        default: return x + y * nx + z * nx * ny;
    }
}

// dst[natural point p][w] := src[file point of p][w], one 8-byte word per
// thread; the natural side is written coalesced.
__global__ void __launch_bounds__(kIoThreads) grid_reorder_kernel(const double* __restrict__ src,
                                                                  double* __restrict__ dst, int nx, int ny, int nz,
                                                                  int words, int order) {
    const int64_t total = (int64_t)nx * ny * nz * words;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = e / words, w = e % words;
        const int64_t x = p % nx, y = (p / nx) % ny, z = p / ((int64_t)nx * ny);
        dst[e] = src[FileIndex(order, x, y, z, nx, ny, nz) * words + w];
    }
}

// Old-grid neighbours of new index i along one axis: lower, upper (clamped
// at the last point) and the weight of the upper one, with the reference's
// IEEE operations (InterpolateTo, dist_uniform_grid.hpp:508-532, 640-654);
// ratio = (n-1)/(nOld-1) comes from the host.
struct AxisTaps {
    int lo, hi;
    double t;
};
__device__ __forceinline__ AxisTaps Taps(int i, double ratio, int nOld) {
    const double old = __ddiv_rn((double)i, ratio);
    const double f = floor(old);
    AxisTaps a;
    a.lo = min(max((int)f, 0), nOld - 1);  // rounding never leaves the old grid
    a.hi = a.lo != nOld - 1 ? a.lo + 1 : a.lo;
    a.t = __dsub_rn(old, f);
    return a;
}

// (1 - t) a + t b, each operation rounded on its own (no contraction), as
// the reference's expression evaluates.
__device__ __forceinline__ double Lerp(double a, double b, double t) {
    return __dadd_rn(__dmul_rn(__dsub_rn(1.0, t), a), __dmul_rn(t, b));
}

// kRowsPerBlock rows (y from blockIdx.y * kRowsPerBlock, z = blockIdx.z) of
// the new grid per block; threads over x and the point's components.  z
// first, then y, then x (the reference's order, dist_uniform_grid.hpp:690-709).
constexpr int kRowsPerBlock = 8;
__global__ void __launch_bounds__(kIoThreads) grid_interpolate_kernel(const double* __restrict__ src,
                                                                      double* __restrict__ dst, int nxOld, int nyOld,
                                                                      int nzOld, int nx, int ny, int words,
                                                                      double xRatio, double yRatio, double zRatio) {
    const int z = blockIdx.z;
    const AxisTaps Z = Taps(z, zRatio, nzOld);
    const int64_t pl = (int64_t)nxOld * nyOld;
    const int rowLen = nx * words;
    const int y0 = blockIdx.y * kRowsPerBlock, y1 = min(y0 + kRowsPerBlock, ny);
    for (int y = y0; y < y1; ++y) {
        const AxisTaps Y = Taps(y, yRatio, nyOld);
        const double* r00 = src + ((int64_t)Y.lo * nxOld + (int64_t)Z.lo * pl) * words;  // (y lower, z lower)
        const double* r01 = src + ((int64_t)Y.lo * nxOld + (int64_t)Z.hi * pl) * words;
        const double* r10 = src + ((int64_t)Y.hi * nxOld + (int64_t)Z.lo * pl) * words;
        const double* r11 = src + ((int64_t)Y.hi * nxOld + (int64_t)Z.hi * pl) * words;
        double* out = dst + ((int64_t)y * nx + (int64_t)z * nx * ny) * words;
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < rowLen; e += gridDim.x * blockDim.x) {
            const int x = e / words, w = e % words;
            const AxisTaps X = Taps(x, xRatio, nxOld);
            const int a = X.lo * words + w, b = X.hi * words + w;
            const double v00 = Lerp(r00[a], r01[a], Z.t);  // x lower, y lower
            const double v01 = Lerp(r10[a], r11[a], Z.t);  // x lower, y upper
            const double v10 = Lerp(r00[b], r01[b], Z.t);  // x upper, y lower
            const double v11 = Lerp(r10[b], r11[b], Z.t);
            const double v0 = Lerp(v00, v01, Y.t);
            const double v1 = Lerp(v10, v11, Y.t);
            out[e] = Lerp(v0, v1, X.t);
        }
    }
}

int IoGrid(int64_t total) {
    const int64_t b = (total + kIoThreads - 1) / kIoThreads;
    return (int)std::min<int64_t>(b, 148 * 16);
}

bool OnDevice(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // not a pointer CUDA knows: host memory
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// A device buffer of n doubles freed on scope exit.
struct DeviceDoubles {
    double* p = nullptr;
    explicit DeviceDoubles(size_t n) { CUDA_CHECK(cudaMalloc(&p, n * sizeof(double))); }
    ~DeviceDoubles() { cudaFree(p); }
};

void CheckSizes(int nx, int ny, int nz, int doubles) {
    if (nx < 1 || ny < 1 || nz < 1 || doubles < 1) throw PspError(kLogicError, "grid sizes must be positive");
}

// Default stream formatting of a value, with |value| < 1e-300 written as 0
// (the reference's writers).
void PutValue(std::ostream& os, double v) {
    if (std::fabs(v) < 1.0e-300) v = 0;
    os << v << " ";
}

std::string Header(const std::string& wholeExtent, const std::string& origin, double h,
                   const std::string& pieceExtent) {
    std::ostringstream os;
    os << "<?xml version=\"1.0\"?>\n"
       << "<VTKFile type=\"ImageData\" version=\"0.1\">\n"
       << " <ImageData WholeExtent=\"" << wholeExtent << "\" "
       << "Origin=\"" << origin << "\" "
       << "Spacing=\"" << h << " " << h << " " << h << "\">\n"
       << "  <Piece Extent=\"" << pieceExtent << "\">\n"
       << "    <CellData Scalars=\"cell_scalars\">\n"
       << "     <DataArray type=\"Float64\" Name=\"cell_scalars\" "
       << "format=\"ascii\">\n";
    return os.str();
}

const char* kTrailer =
    "    </DataArray>\n"
    "   </CellData>\n"
    "  </Piece>\n"
    " </ImageData>\n"
    "</VTKFile>";

std::ofstream OpenOut(const std::string& name) {
    std::ofstream f(name.c_str(), std::ios::out);
    if (!f.is_open()) throw PspError(kLogicError, "Could not open " + name);
    return f;
}

void EnsureDir(const std::string& dir) {
    if (mkdir(dir.c_str(), 0755) != 0 && errno != EEXIST)
        throw PspError(kLogicError, "Could not create directory " + dir);
}

}  // namespace

void GridLoad(const std::string& filename, int nx, int ny, int nz, int doubles, int order, double* out) {
    CheckSizes(nx, ny, nz, doubles);
    if (order < kXYZ || order > kZYX) throw PspError(kLogicError, "invalid grid data order");
    if (!out) throw PspError(kLogicError, "null output grid");
    const size_t count = (size_t)nx * ny * nz * doubles;
    if (!OnDevice(out)) {  // host output: through a device buffer
        DeviceDoubles d(count);
        GridLoad(filename, nx, ny, nz, doubles, order, d.p);
        CUDA_CHECK(cudaMemcpy(out, d.p, count * sizeof(double), cudaMemcpyDeviceToHost));
        return;
    }
    double* d_out = out;
    std::vector<double> host(count);
    FILE* f = std::fopen(filename.c_str(), "rb");
    if (!f) throw PspError(kLogicError, "Could not open " + filename);
    const size_t got = std::fread(host.data(), sizeof(double), count, f);
    std::fclose(f);
    if (got != count) throw PspError(kLogicError, filename + " holds fewer values than the grid");
    if (order == kXYZ) {
        CUDA_CHECK(cudaMemcpy(d_out, host.data(), count * sizeof(double), cudaMemcpyHostToDevice));
        return;
    }
    double* d_src = nullptr;
    CUDA_CHECK(cudaMalloc(&d_src, count * sizeof(double)));
    cudaError_t e = cudaMemcpy(d_src, host.data(), count * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        grid_reorder_kernel<<<IoGrid((int64_t)count), kIoThreads>>>(d_src, d_out, nx, ny, nz, doubles, order);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    cudaFree(d_src);
    CUDA_CHECK(e);
}

void GridInterpolate(const double* d_in, int nxOld, int nyOld, int nzOld, int doubles, double* d_out, int nx,
                     int ny, int nz) {
    CheckSizes(nxOld, nyOld, nzOld, doubles);
    CheckSizes(nx, ny, nz, doubles);
    if (!d_in || !d_out) throw PspError(kLogicError, "null grid");
    const size_t count = (size_t)nx * ny * nz * doubles;
    if (!OnDevice(d_in) || !OnDevice(d_out)) {  // host grids: through device buffers
        const size_t countOld = (size_t)nxOld * nyOld * nzOld * doubles;
        DeviceDoubles in(countOld), outBuf(count);
        CUDA_CHECK(cudaMemcpy(in.p, d_in, countOld * sizeof(double), cudaMemcpyDefault));
        GridInterpolate(in.p, nxOld, nyOld, nzOld, doubles, outBuf.p, nx, ny, nz);
        CUDA_CHECK(cudaMemcpy(d_out, outBuf.p, count * sizeof(double), cudaMemcpyDefault));
        return;
    }
    if (nx == nxOld && ny == nyOld && nz == nzOld) {
        CUDA_CHECK(cudaMemcpy(d_out, d_in, count * sizeof(double), cudaMemcpyDeviceToDevice));
        return;
    }
    if (nxOld < 2 || nyOld < 2 || nzOld < 2)
        throw PspError(kLogicError, "interpolation needs at least two points along each axis");
    if (nz > 65535) throw PspError(kLogicError, "grid too large for interpolation");
    const double xRatio = (1. * (nx - 1)) / (nxOld - 1);
    const double yRatio = (1. * (ny - 1)) / (nyOld - 1);
    const double zRatio = (1. * (nz - 1)) / (nzOld - 1);
    const int rowLen = nx * doubles;
    const dim3 grid((unsigned)std::min((rowLen + kIoThreads - 1) / kIoThreads, 64),
                    (unsigned)((ny + kRowsPerBlock - 1) / kRowsPerBlock), (unsigned)nz);
    grid_interpolate_kernel<<<grid, kIoThreads>>>(d_in, d_out, nxOld, nyOld, nzOld, nx, ny, doubles, xRatio, yRatio,
                                                   zRatio);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaDeviceSynchronize());
}

void GridWritePlane(const double* data, int nx, int ny, int nz, int scalars, bool isComplex, int plane, int which,
                    const std::string& basename) {
    CheckSizes(nx, ny, nz, scalars);
    if (!data) throw PspError(kLogicError, "null grid");
    const int perPoint = scalars * (isComplex ? 2 : 1);
    // plane axes (a fastest, b) and the natural point of (a, b)
    int na, nb, bound;
    std::string whole, origin;
    const int maxPoints = plane == kPlaneXY ? std::max(nx, ny) : plane == kPlaneXZ ? std::max(nx, nz) : std::max(ny, nz);
    const double h = 1. / (maxPoints + 1.0);
    std::ostringstream o;
    if (plane == kPlaneXY) {
        na = nx; nb = ny; bound = nz;
        o << "0 0 " << h * which;
    } else if (plane == kPlaneXZ) {
        na = nx; nb = nz; bound = ny;
        o << "0 " << h * which << " 0";
    } else if (plane == kPlaneYZ) {
        na = ny; nb = nz; bound = nx;
        o << h * which << " 0 0";
    } else {
        throw PspError(kLogicError, "invalid plane type");
    }
    if (which < 0 || which >= bound) throw PspError(kLogicError, "Invalid plane");
    std::ostringstream ext;
    if (plane == kPlaneXY) ext << "0 " << nx << " 0 " << ny << " 0 1";
    else if (plane == kPlaneXZ) ext << "0 " << nx << " 0 1 0 " << nz;
    else ext << "0 1 0 " << ny << " 0 " << nz;
    const std::string head = Header(ext.str(), o.str(), h, ext.str());
    auto point = [&](int a, int b) -> int64_t {
        if (plane == kPlaneXY) return (int64_t)a + (int64_t)b * nx + (int64_t)which * nx * ny;
        if (plane == kPlaneXZ) return (int64_t)a + (int64_t)which * nx + (int64_t)b * nx * ny;
        return (int64_t)which + (int64_t)a * nx + (int64_t)b * nx * ny;
    };
    for (int k = 0; k < scalars; ++k) {
        for (int part = 0; part < (isComplex ? 2 : 1); ++part) {
            std::ostringstream name;
            name << basename << "_" << k << (isComplex ? (part ? "_imag" : "_real") : "") << ".vti";
            std::ofstream file = OpenOut(name.str());
            file << head;
            for (int b = 0; b < nb; ++b) {
                for (int a = 0; a < na; ++a)
                    PutValue(file, data[point(a, b) * perPoint + (isComplex ? 2 * k + part : k)]);
                file << "\n";
            }
            file << kTrailer << std::endl;
        }
    }
}

void GridWriteVolume(const double* data, int nx, int ny, int nz, int scalars, bool isComplex,
                     const std::string& basename) {
    CheckSizes(nx, ny, nz, scalars);
    if (!data) throw PspError(kLogicError, "null grid");
    const int perPoint = scalars * (isComplex ? 2 : 1);
    const double h = 1.0 / (std::max(std::max(nx, ny), nz) + 1.0);
    std::ostringstream ext;
    ext << "0 " << nx << " 0 " << ny << " 0 " << nz;
    const std::string head = Header(ext.str(), "0 0 0", h, ext.str());
    for (int k = 0; k < scalars; ++k) {
        for (int part = 0; part < (isComplex ? 2 : 1); ++part) {
            std::ostringstream stem;
            stem << basename << "_" << k << (isComplex ? (part ? "_imag" : "_real") : "");
            // the parallel description of the one piece
            {
                std::ofstream p = OpenOut(stem.str() + ".pvti");
                p << "<?xml version=\"1.0\"?>\n"
                  << "<VTKFile type=\"PImageData\" version=\"0.1\">\n"
                  << " <PImageData WholeExtent=\"" << ext.str() << "\" "
                  << "Origin=\"0 0 0\" "
                  << "Spacing=\"" << h << " " << h << " " << h << "\" "
                  << "GhostLevel=\"0\">\n"
                  << "  <PCellData Scalars=\"cell_scalars\">\n"
                  << "    <PDataArray type=\"Float64\" Name=\"cell_scalars\"/>\n"
                  << "  </PCellData>\n"
                  << "  <Piece Extent=\"" << ext.str() << "\" "
                  << "Source=\"" << stem.str() << "/0.vti\"/>\n"
                  << " </PImageData>\n"
                  << "</VTKFile>" << std::endl;
            }
            EnsureDir(stem.str());
            std::ofstream file = OpenOut(stem.str() + "/0.vti");
            file << head;
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y) {
                    for (int x = 0; x < nx; ++x) {
                        const int64_t pt = (int64_t)x + (int64_t)y * nx + (int64_t)z * nx * ny;
                        PutValue(file, data[pt * perPoint + (isComplex ? 2 * k + part : k)]);
                    }
                    file << "\n";
                }
            file << kTrailer << std::endl;
        }
    }
}

}  // namespace psp_b200
