"""ORACLE — test infrastructure only (the checker, never the product).

numpy restatement of psp::DistUniformGrid's ingest and output on one process
(PSP include/psp/dist_uniform_grid.hpp), used by tests/test_grid_io.py to
check the device kernels and the C-ABI writers:

* ``file_index`` / ``sequential_load`` / ``to_file_order`` follow the index
  expressions of SequentialLoad (dist_uniform_grid.hpp:349-482);
* ``interpolate_to`` follows InterpolateTo (484-714): old coordinate
  n / ratio with ratio = (n-1)/(nOld-1), upper neighbour clamped at the last
  point, (1-t) a + t b along z, then y, then x, each operation rounded on its
  own (numpy evaluates elementwise operations separately);
* ``plane_text`` / ``volume_texts`` restate the ASCII VTK files of
  WritePlane (716-1631) and WriteVolume (1788-2200) with the values
  formatted as C++ streams do by default (printf %g, 6 significant digits)
  and |value| < 1e-300 written as 0.

Grids are numpy arrays of shape (nz, ny, nx, numScalars) in natural order.
"""
import numpy as np

XYZ, XZY, YXZ, YZX, ZXY, ZYX = range(6)
XY, XZ, YZ = range(3)


def file_index(order, x, y, z, nx, ny, nz):
    """Point offset of natural point (x, y, z) in a file stored in `order`
    (dist_uniform_grid.hpp:360-478)."""
    if order == XYZ:
        return x + y * nx + z * nx * ny
    if order == XZY:
        return x + z * nx + y * nx * nz
    if order == YXZ:
        return y + x * ny + z * nx * ny
    if order == YZX:
        return y + z * ny + x * ny * nz
    if order == ZXY:
        return z + x * nz + y * nz * nx
    if order == ZYX:
        return z + y * nz + x * nz * ny
    raise ValueError(order)


def _natural_file_index(order, nx, ny, nz):
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return file_index(order, x, y, z, nx, ny, nz).reshape(-1)


def sequential_load(flat, nx, ny, nz, numScalars, order):
    """Natural-order grid from the values of a file stored in `order`."""
    a = np.asarray(flat).reshape(-1, numScalars)
    return a[_natural_file_index(order, nx, ny, nz)].reshape(nz, ny, nx, numScalars)


def to_file_order(grid, order):
    """The file layout in `order` of a natural-order grid (inverse of
    sequential_load)."""
    nz, ny, nx, ns = grid.shape
    out = np.empty((nx * ny * nz, ns), dtype=grid.dtype)
    out[_natural_file_index(order, nx, ny, nz)] = grid.reshape(-1, ns)
    return out.reshape(-1)


def _bracket(n, nOld):
    ratio = (1.0 * (n - 1)) / (nOld - 1)
    old = np.arange(n, dtype=np.float64) / ratio
    f = np.floor(old)
    lo = f.astype(np.int64)
    hi = np.where(lo != nOld - 1, lo + 1, lo)
    return lo, hi, old - f


def interpolate_to(grid, nx, ny, nz):
    """Trilinear resampling of a natural-order grid to nx x ny x nz."""
    nzO, nyO, nxO, ns = grid.shape
    if (nx, ny, nz) == (nxO, nyO, nzO):
        return grid.copy()
    xl, xu, tx = _bracket(nx, nxO)
    yl, yu, ty = _bracket(ny, nyO)
    zl, zu, tz = _bracket(nz, nzO)
    Z = lambda a: a[:, None, None, None]
    Y = lambda a: a[None, :, None, None]
    X = lambda a: a[None, None, :, None]

    def at(xi, yi, zi):
        return grid[Z(zi), Y(yi), X(xi), np.arange(ns)[None, None, None, :]]

    def lerp(a, b, t):
        return (1.0 - t) * a + t * b

    v00 = lerp(at(xl, yl, zl), at(xl, yl, zu), Z(tz))
    v01 = lerp(at(xl, yu, zl), at(xl, yu, zu), Z(tz))
    v10 = lerp(at(xu, yl, zl), at(xu, yl, zu), Z(tz))
    v11 = lerp(at(xu, yu, zl), at(xu, yu, zu), Z(tz))
    v0 = lerp(v00, v01, Y(ty))
    v1 = lerp(v10, v11, Y(ty))
    return lerp(v0, v1, X(tx))


def _fmt(v):
    v = float(v)
    if abs(v) < 1.0e-300:
        v = 0.0
    return "%g" % v


def _header(whole, origin, h, piece):
    return ('<?xml version="1.0"?>\n'
            '<VTKFile type="ImageData" version="0.1">\n'
            ' <ImageData WholeExtent="%s" Origin="%s" Spacing="%s %s %s">\n'
            '  <Piece Extent="%s">\n'
            '    <CellData Scalars="cell_scalars">\n'
            '     <DataArray type="Float64" Name="cell_scalars" format="ascii">\n'
            % (whole, origin, _fmt(h), _fmt(h), _fmt(h), piece))


_TRAILER = "    </DataArray>\n   </CellData>\n  </Piece>\n </ImageData>\n</VTKFile>\n"


def _parts(grid):
    """(suffix, real array) per file of one scalar: real grids one, complex
    grids _real and _imag."""
    if np.iscomplexobj(grid):
        return [("_real", grid.real), ("_imag", grid.imag)]
    return [("", grid)]


def plane_text(grid, plane, which):
    """{file suffix: text} of WritePlane for a natural-order grid; suffixes
    are '_<k>' plus '_real'/'_imag' for complex grids."""
    nz, ny, nx, ns = grid.shape
    if plane == XY:
        h = 1.0 / (max(nx, ny) + 1.0)
        ext, origin = "0 %d 0 %d 0 1" % (nx, ny), "0 0 %s" % _fmt(h * which)
        sl = lambda a: a[which, :, :]          # rows over y, x fastest
    elif plane == XZ:
        h = 1.0 / (max(nx, nz) + 1.0)
        ext, origin = "0 %d 0 1 0 %d" % (nx, nz), "0 %s 0" % _fmt(h * which)
        sl = lambda a: a[:, which, :]          # rows over z, x fastest
    else:
        h = 1.0 / (max(ny, nz) + 1.0)
        ext, origin = "0 1 0 %d 0 %d" % (ny, nz), "%s 0 0" % _fmt(h * which)
        sl = lambda a: a[:, :, which]          # rows over z, y fastest
    out = {}
    for k in range(ns):
        for suffix, part in _parts(grid[..., k]):
            rows = sl(part)
            body = "".join("".join(_fmt(v) + " " for v in row) + "\n" for row in rows)
            out["_%d%s" % (k, suffix)] = _header(ext, origin, h, ext) + body + _TRAILER
    return out


def volume_texts(grid, basename):
    """{file name relative to basename's directory: text} of WriteVolume on
    one process: '<base>_<k>[_real|_imag].pvti' and the piece
    '<base>_<k>[_real|_imag]/0.vti'."""
    nz, ny, nx, ns = grid.shape
    h = 1.0 / (max(nx, ny, nz) + 1.0)
    ext = "0 %d 0 %d 0 %d" % (nx, ny, nz)
    out = {}
    for k in range(ns):
        for suffix, part in _parts(grid[..., k]):
            stem = "%s_%d%s" % (basename, k, suffix)
            out[stem + ".pvti"] = (
                '<?xml version="1.0"?>\n'
                '<VTKFile type="PImageData" version="0.1">\n'
                ' <PImageData WholeExtent="%s" Origin="0 0 0" Spacing="%s %s %s" GhostLevel="0">\n'
                '  <PCellData Scalars="cell_scalars">\n'
                '    <PDataArray type="Float64" Name="cell_scalars"/>\n'
                '  </PCellData>\n'
                '  <Piece Extent="%s" Source="%s/0.vti"/>\n'
                ' </PImageData>\n'
                '</VTKFile>\n' % (ext, _fmt(h), _fmt(h), _fmt(h), ext, stem))
            body = "".join("".join(_fmt(v) + " " for v in part[z, y, :]) + "\n"
                           for z in range(nz) for y in range(ny))
            out[stem + "/0.vti"] = _header(ext, "0 0 0", h, ext) + body + _TRAILER
    return out
