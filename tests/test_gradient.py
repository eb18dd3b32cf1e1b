"""Velocity gradients by the adjoint-state method (the differentiation layer;
the reference has no adjoint).

CPU: the adjoint formula against central finite differences of the misfit,
both from sparse direct solves of the independent numpy operator.  GPU: the
device gradient kernel against the same formula, and the autograd path
(forward solve, adjoint solve with the forward factors, gradient kernel)
against the direct-solve adjoint gradient.
"""
import numpy as np
import pytest

import helmholtz_np as hn
from psp_b200 import workloads as W


def _misfit_case():
    w = W.small_case()
    d = w.disc
    vel = np.asarray(w.velocity).reshape(d.nz, d.ny, d.nx)
    rng = np.random.Generator(np.random.PCG64(2024))
    N = d.nx * d.ny * d.nz
    receivers = np.sort(rng.choice(N, size=200, replace=False))
    # observed data from a 3 % perturbed model
    pert = vel * (1 + 0.03 * np.sin(np.linspace(0, 6, vel.size)).reshape(vel.shape))
    import scipy.sparse.linalg as spla
    f = np.ascontiguousarray(np.asarray(w.rhs).reshape(N, -1))
    u_obs = spla.splu(hn.global_matrix(d, pert).tocsc()).solve(f)
    return w, d, vel, f, receivers, u_obs[receivers]


def test_adjoint_formula_matches_finite_differences():
    w, d, vel, f, receivers, data = _misfit_case()
    J0, g, _ = hn.adjoint_gradient(d, vel, f, receivers, data)
    assert J0 > 0
    rng = np.random.Generator(np.random.PCG64(5))
    voxels = rng.choice(vel.size, size=6, replace=False)
    for i in voxels:
        h = 1e-4 * vel.reshape(-1)[i]
        vp, vm = vel.copy().reshape(-1), vel.copy().reshape(-1)
        vp[i] += h
        vm[i] -= h
        Jp = hn.adjoint_gradient(d, vp.reshape(vel.shape), f, receivers, data)[0]
        Jm = hn.adjoint_gradient(d, vm.reshape(vel.shape), f, receivers, data)[0]
        fd = (Jp - Jm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(g[i]), 1e-3 * np.abs(g).max()), (i, fd, g[i])


@pytest.mark.gpu
def test_gradient_kernel_matches_formula(product_lib):
    import torch
    import psp_b200 as P
    w = W.small_case()
    d = w.disc
    H = P.DistHelmholtz(d)
    H.Initialize(w.velocity, precision=P.FP64)
    rng = np.random.Generator(np.random.PCG64(11))
    N, k = d.nx * d.ny * d.nz, 3
    U = rng.standard_normal((N, k)) + 1j * rng.standard_normal((N, k))
    Z = rng.standard_normal((N, k)) + 1j * rng.standard_normal((N, k))
    g = H.gradient_device(torch.from_numpy(U).cuda(), torch.from_numpy(Z).cuda()).cpu().numpy()
    vel = np.asarray(w.velocity).reshape(d.nz, d.ny, d.nx)
    ref = -np.real(hn.velocity_derivative_diag(d, vel) * np.sum(Z * U, axis=1))
    assert np.linalg.norm(g - ref) <= 1e-12 * np.linalg.norm(ref)
    g2 = H.gradient_device(torch.from_numpy(U).cuda(), torch.from_numpy(Z).cuda(),
                           grad=torch.from_numpy(ref.copy()).cuda(), accumulate=True).cpu().numpy()
    assert np.linalg.norm(g2 - 2 * ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(0, 1e-7), (1, 2e-3)])
def test_autograd_gradient_matches_direct_adjoint(product_lib, precision, tol):
    import torch
    import psp_b200 as P
    from psp_b200.autograd import misfit_and_gradient, helmholtz_solve
    w, d, vel, f_np, receivers, data = _misfit_case()
    J_ref, g_ref, u_ref = hn.adjoint_gradient(d, vel, f_np, receivers, data)
    H = P.DistHelmholtz(d)
    v = torch.from_numpy(vel.reshape(-1).copy()).cuda()
    f = torch.from_numpy(f_np).cuda()
    J, g = misfit_and_gradient(H, v, f, torch.from_numpy(receivers).cuda(), torch.from_numpy(data).cuda(),
                               m=60, rel_tol=1e-11 if precision == 0 else 1e-8, precision=precision)
    assert abs(float(J) - J_ref) <= tol * J_ref
    assert np.linalg.norm(g.cpu().numpy() - g_ref) <= tol * np.linalg.norm(g_ref)
    # the source gradient: dL/dconj(f) = conj(z), z = A^{-1} conj(dL/dconj(u))
    vv = v.clone()
    ff = f.clone().requires_grad_(True)
    u = helmholtz_solve(H, vv, ff, m=60, rel_tol=1e-11, precision=P.FP64)
    (u.real.sum() + 2 * u.imag.sum()).backward()
    import scipy.sparse.linalg as spla
    lu = spla.splu(hn.global_matrix(d, vel).tocsc())
    G = np.ones_like(u_ref) * (1 + 2j)  # dL/dconj(u) for L = sum(re u) + 2 sum(im u)
    ref = np.conj(lu.solve(np.conj(G)))
    assert np.linalg.norm(ff.grad.cpu().numpy() - ref) <= 1e-7 * np.linalg.norm(ref)


@pytest.mark.gpu
def test_autograd_gradient_matches_finite_differences_layered(product_lib):
    """The differentiation workload's generator at test size (layered,
    faulted velocity; sources and receivers on the surface plane; data from
    a 3 %-perturbed model): the FP64 autograd gradient (forward solve,
    adjoint solve with the forward factors, device gradient kernel) matches
    central finite differences of the misfit (step 1e-4 of the velocity) at
    8 seeded voxels to 1e-4 relative; the mixed-precision gradient is
    reported against the same differences."""
    import torch
    import psp_b200 as P
    from psp_b200.autograd import misfit_and_gradient
    w = W.CONFIGS["layered_faults_24"]()
    d = w.disc
    N, k = d.nx * d.ny * d.nz, w.k
    H = P.DistHelmholtz(d)
    f = torch.from_numpy(np.ascontiguousarray(w.rhs.reshape(N, k))).cuda()
    recv = torch.from_numpy(w.meta["receivers"]).cuda()
    H.Initialize(torch.from_numpy(w.meta["observed_model"].reshape(-1)).cuda(), precision=P.FP64)
    u_obs = f.clone()
    H.Solve(u_obs, 60, 1e-12)
    data = u_obs[recv].clone()
    vel = torch.from_numpy(np.ascontiguousarray(w.velocity.reshape(-1))).cuda()
    tol_solve = 1e-12
    J, g = misfit_and_gradient(H, vel, f, recv, data, m=60, rel_tol=tol_solve, precision=P.FP64)
    g = g.cpu().numpy()
    assert float(J) > 0

    def misfit(v):
        u = f.clone()
        H.Initialize(v, precision=P.FP64)
        H.Solve(u, 60, tol_solve)
        r = u[recv.long()] - data
        return float(0.5 * (r.real.square() + r.imag.square()).sum())

    # interior voxels below the source plane, where the model is sensed
    rng = np.random.Generator(np.random.PCG64(8))
    z0 = w.pml + 1
    cand = np.arange(N).reshape(d.nz, d.ny, d.nx)[z0:d.nz - w.pml, w.pml:d.ny - w.pml, w.pml:d.nx - w.pml].reshape(-1)
    voxels = rng.choice(cand, size=8, replace=False)
    gmax = np.abs(g).max()
    fd = []
    for i in voxels:
        h = 1e-4 * float(vel[i])
        vp, vm = vel.clone(), vel.clone()
        vp[i] += h
        vm[i] -= h
        fd.append((misfit(vp) - misfit(vm)) / (2 * h))
    fd = np.array(fd)
    for i, v in zip(voxels, fd):
        assert abs(v - g[i]) <= 1e-4 * max(abs(g[i]), 1e-2 * gmax), (i, v, g[i])
    _, gm = misfit_and_gradient(H, vel, f, recv, data, m=60, rel_tol=1e-8, precision=P.MIXED)
    gm = gm.cpu().numpy()
    err_mixed = np.max(np.abs(gm[voxels] - fd) / np.maximum(np.abs(fd), 1e-2 * gmax))
    print("mixed-precision gradient vs finite differences: max relative error %.2e" % err_mixed)
    assert err_mixed < 1e-3


@pytest.mark.gpu
def test_gradient_with_recomputed_panels_matches_resident(product_lib, monkeypatch):
    """When the factors do not fit (forced here by capping the resident
    panels) the adjoint solve recomputes panels as the forward solve does:
    the gradient equals the one from resident factors."""
    import torch
    import psp_b200 as P
    from psp_b200.autograd import misfit_and_gradient
    w, d, vel, f_np, receivers, data = _misfit_case()
    v = torch.from_numpy(vel.reshape(-1).copy()).cuda()
    f = torch.from_numpy(f_np).cuda()
    recv, dat = torch.from_numpy(receivers).cuda(), torch.from_numpy(data).cuda()
    grads = []
    for cap in (None, "1"):
        if cap is None:
            monkeypatch.delenv("PSP_B200_RESIDENT_PANELS", raising=False)
        else:
            monkeypatch.setenv("PSP_B200_RESIDENT_PANELS", cap)
        H = P.DistHelmholtz(d)
        J, g = misfit_and_gradient(H, v, f, recv, dat, m=60, rel_tol=1e-11, precision=P.FP64)
        info = H.memory_info()
        assert (info["resident_panels"] == 1) == (cap is not None)
        assert (info["refactorizations"] > 0) == (cap is not None)
        grads.append(g.cpu().numpy())
    assert np.linalg.norm(grads[1] - grads[0]) <= 1e-10 * np.linalg.norm(grads[0])
