"""Independent numpy/scipy restatement of PSP's discrete operators.

Test infrastructure only: used to pin the oracle's panel factorizations and
sweep against sparse direct solves.  Everything is in natural ordering
(x fastest, then y, then z) with the sweep coordinate v = nz-1-z.

* PML stretches: initialize_finalize.hpp:415-525 (s1Inv, s2Inv, s3Inv,
  s3InvArtificial).
* Global row: FormGlobalRow, initialize_finalize.hpp:527-587.
* Panel subproblem: FormLowerColumnOfNode, initialize_finalize.hpp:589-806
  (artificial PML below the panel, omega -> omega + i*damping, Dirichlet
  truncation at the subproblem's first and last plane).
"""
import numpy as np
import scipy.sparse as sp

PML = 0


def stretch(i, n, b, sigma, h, omega, low_pml, high_pml, low_edge=0):
    eta = b * h
    if low_pml and i < low_edge + b - 1:
        delta = (low_edge + b - 1) - i
    elif high_pml and i > n - b:
        delta = i - (n - b)
    else:
        return 1.0 + 0.0j
    return 1.0 + 1j * (sigma / eta) * (delta / b) ** 2 * (2 * np.pi / omega)


def _tables(d):
    hx, hy, hz = d.wx / (d.nx + 1), d.wy / (d.ny + 1), d.wz / (d.nz + 1)
    s1 = lambda x: stretch(x, d.nx, d.bx, d.sigmax, hx, d.omega, d.frontBC == PML, d.backBC == PML)
    s2 = lambda y: stretch(y, d.ny, d.by, d.sigmay, hy, d.omega, d.leftBC == PML, d.rightBC == PML)
    return hx, hy, hz, s1, s2


def _assemble(d, vel, v_lo, v_hi, s3, omega_c):
    """Rows for planes v in [v_lo, v_hi) with Dirichlet truncation outside."""
    hx, hy, hz, s1, s2 = _tables(d)
    nx, ny, nz = d.nx, d.ny, d.nz
    nv = v_hi - v_lo
    n = nx * ny * nv
    rows, cols, vals = [], [], []
    idx = lambda x, y, vl: x + y * nx + vl * nx * ny
    for vl in range(nv):
        v = v_lo + vl
        z = nz - 1 - v
        s3L, s3M, s3R = s3(v - 1), s3(v), s3(v + 1)
        for y in range(ny):
            s2L, s2M, s2R = s2(y - 1), s2(y), s2(y + 1)
            for x in range(nx):
                s1L, s1M, s1R = s1(x - 1), s1(x), s1(x + 1)
                xTop, yTop, zTop = s2M * s3M, s1M * s3M, s1M * s2M
                xL = (xTop / s1L + xTop / s1M) / (2 * hx * hx)
                xR = (xTop / s1R + xTop / s1M) / (2 * hx * hx)
                yL = (yTop / s2L + yTop / s2M) / (2 * hy * hy)
                yR = (yTop / s2R + yTop / s2M) / (2 * hy * hy)
                vL = (zTop / s3L + zTop / s3M) / (2 * hz * hz)
                vR = (zTop / s3R + zTop / s3M) / (2 * hz * hz)
                alpha = vel[z, y, x]
                c = xL + xR + yL + yR + vL + vR - (omega_c / alpha) ** 2 * s1M * s2M * s3M
                i = idx(x, y, vl)
                rows.append(i); cols.append(i); vals.append(c)
                for ok, j, t in ((x > 0, idx(x - 1, y, vl), xL), (x + 1 < nx, idx(x + 1, y, vl), xR),
                                 (y > 0, idx(x, y - 1, vl), yL), (y + 1 < ny, idx(x, y + 1, vl), yR),
                                 (vl > 0, idx(x, y, vl - 1), vL), (vl + 1 < nv, idx(x, y, vl + 1), vR)):
                    if ok:
                        rows.append(i); cols.append(j); vals.append(-t)
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def global_matrix(d, vel):
    """Global operator in natural z-major ordering (planes stored by z)."""
    hz = d.wz / (d.nz + 1)
    s3 = lambda v: stretch(v, d.nz, d.bz, d.sigmaz, hz, d.omega, True, d.topBC == PML)
    A_v = _assemble(d, vel, 0, d.nz, s3, d.omega)   # ordered by v
    # reorder v-major -> z-major (z = nz-1-v)
    nxy = d.nx * d.ny
    perm = np.concatenate([np.arange(nxy) + (d.nz - 1 - z) * nxy for z in range(d.nz)])
    return A_v[perm][:, perm].tocsr()


def panel_matrix(d, vel, v_offset, v_size, damping):
    """Padded panel subproblem on planes [v_offset, v_offset + v_size), v-major."""
    hz = d.wz / (d.nz + 1)
    s3 = lambda v: stretch(v, d.nz, d.bz, d.sigmaz, hz, d.omega, True, d.topBC == PML, low_edge=v_offset)
    return _assemble(d, vel, v_offset, v_offset + v_size, s3, d.omega + 1j * damping)


def apply_panel_inverse(d, vel, B, low_v, depth, padding, damping):
    """T_p B as SolvePanel computes it (solve.hpp:736-882): the panel's planes
    of B go through the inverse of the padded subproblem, padding planes enter
    as zero; every other plane of B is returned unchanged."""
    nxy = d.nx * d.ny
    k = B.shape[-1]
    v_off, v_size = low_v - padding, depth + padding
    A = panel_matrix(d, vel, v_off, v_size, damping).tocsc()
    Bv = B.reshape(d.nz, nxy, k)[::-1]          # index by v
    rhs = np.zeros((v_size * nxy, k), dtype=np.complex128)
    rhs[padding * nxy:] = Bv[low_v:low_v + depth].reshape(-1, k)
    import scipy.sparse.linalg as spla
    lu = spla.splu(A)
    X = np.stack([lu.solve(rhs[:, r]) for r in range(k)], -1)
    out = Bv.copy()
    out[low_v:low_v + depth] = X[padding * nxy:].reshape(depth, nxy, k)
    return out[::-1].reshape(B.shape)


def velocity_derivative_diag(d, vel):
    """dA_ii/dvel_i in natural z-major order: the derivative of FormGlobalRow's
    centre term -(omega/vel)^2 s1 s2 s3 (initialize_finalize.hpp:567-568),
    i.e. 2 omega^2 / vel^3 * s1 s2 s3.  ``vel`` has shape (nz, ny, nx)."""
    hx, hy, hz, s1, s2 = _tables(d)
    s3 = lambda v: stretch(v, d.nz, d.bz, d.sigmaz, hz, d.omega, True, d.topBC == PML)
    t1 = np.array([s1(x) for x in range(d.nx)])
    t2 = np.array([s2(y) for y in range(d.ny)])
    t3 = np.array([s3(d.nz - 1 - z) for z in range(d.nz)])
    s = t3[:, None, None] * t2[None, :, None] * t1[None, None, :]
    return (2 * d.omega ** 2 / np.asarray(vel) ** 3 * s).reshape(-1)


def adjoint_gradient(d, vel, f, receivers, data):
    """Misfit J = 1/2 sum |u[receivers] - data|^2 with u = A(vel)^{-1} f by a
    sparse direct solve, and its velocity gradient by the adjoint-state
    method (A is complex symmetric, so the adjoint solve reuses A)."""
    import scipy.sparse.linalg as spla
    lu = spla.splu(global_matrix(d, vel).tocsc())
    u = lu.solve(np.ascontiguousarray(f))
    r = u[receivers] - data
    J = 0.5 * float(np.sum(np.abs(r) ** 2))
    G = np.zeros_like(u)
    G[receivers] = r
    z = lu.solve(np.conj(G))
    g = -np.real(velocity_derivative_diag(d, vel) * np.sum(z * u, axis=1))
    return J, g, u
