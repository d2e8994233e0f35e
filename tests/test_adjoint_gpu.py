"""Discrete adjoint on the GPU: Brinkman-forced forward parity and gradients
against central finite differences of FP64 forward runs.

The objective is J = sum over bulk cells of |u|^2 at step T with
u = sum c f / (rho + alpha/2); the parameters are the per-cell porosity alpha,
tau and the lid speed.  Tolerances are stated per test.  The per-cell bar is
1e-4 relative for FP64 and FP32S storage (FP32 deviations f - rho0 w); FP32
storage of f itself carries a trajectory error of ~1e-5 that leaves cells with
small gradients above 1e-4, so it is held to 1e-3.
"""
import numpy as np
import pytest

import freelb_b200 as F
from conftest import rel_maxnorm
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def brinkman_cavity(ni, tau, ulid, alpha, storage):
    lat = F.cavity(ni, tau=tau, ulid=ulid, storage=storage, model="brinkman")
    lat.upload_field("alpha", np.asarray(alpha, dtype=lat.real))
    return lat


@pytest.mark.parametrize("storage,tol", [("fp64", 1e-12), ("fp32", 1e-5), ("fp32s", 1e-6)])
def test_brinkman_forward_matches_oracle(gpu_ok, storage, tol):
    """FP32S is held against the FP64 oracle: it stores deviations, so its
    trajectory follows FP64, not the FP32 rounding of f."""
    ni, tau, steps = 14, 0.56, 60
    a = O.porosity(ni, 3)
    dt = np.float32 if storage == "fp32" else np.float64
    lat = brinkman_cavity(ni, tau, 0.1, a, storage)
    lat.step(steps)
    ref = O.cavity(ni, model="brinkman", tau=tau, ulid=0.1, dtype=dt, alpha=a)
    ref.step(steps)
    assert rel_maxnorm(lat.download_pops(), ref.pops) < tol
    assert abs(lat.objective_u2() - ref.objective_u2()) / ref.objective_u2() < 10 * tol


def fd_objective(ni, tau, ulid, alpha, steps, storage="fp64"):
    lat = brinkman_cavity(ni, tau, ulid, alpha, storage)
    lat.step(steps)
    j = lat.objective_u2()
    lat.close()
    return j


@pytest.mark.parametrize("storage,tol", [("fp64", 1e-6), ("fp32s", 1e-4), ("fp32", 1e-3)])
def test_adjoint_gradients_match_central_differences(gpu_ok, storage, tol):
    """dJ/dalpha on seeded cells, dJ/dtau and dJ/du_lid against FP64 central
    differences (h = 1e-4).  Checkpoints every 25 steps over 70 steps exercise
    uneven recompute segments."""
    ni, tau, ulid, steps, every = 12, 0.56, 0.1, 70, 25
    n = ni + 2
    a = O.porosity(ni, 11)
    lat = brinkman_cavity(ni, tau, ulid, a, storage)
    J = lat.adjoint_forward(steps, every)
    g_alpha, g_tau, g_ulid = lat.adjoint_backward()
    J64 = fd_objective(ni, tau, ulid, a, steps)
    assert abs(J - J64) / J64 < {"fp64": 1e-12, "fp32s": 1e-6, "fp32": 1e-4}[storage]
    h = 1e-4
    flags = F.cavity_flags(ni)
    fluid = np.flatnonzero(flags == 2)
    cells = np.random.default_rng(5).choice(fluid, size=6, replace=False)
    for c in cells:
        ap, am = a.copy(), a.copy()
        ap[c] += h
        am[c] -= h
        fd = (fd_objective(ni, tau, ulid, ap, steps) - fd_objective(ni, tau, ulid, am, steps)) / (2 * h)
        assert abs(g_alpha[c] - fd) <= tol * abs(fd) + 1e-9, (c, g_alpha[c], fd)
    # tau and u_lid: central differences at h and h/2, Richardson-extrapolated
    # (the O(h^2) term of a plain h = 1e-4 difference in tau is ~1e-6 relative)
    def richardson(fn):
        d1 = (fn(h) - fn(-h)) / (2 * h)
        d2 = (fn(h / 2) - fn(-h / 2)) / h
        return (4 * d2 - d1) / 3, d1

    fd_tau, fd_tau_h = richardson(lambda d: fd_objective(ni, tau + d, ulid, a, steps))
    assert abs(g_tau - fd_tau) <= tol * abs(fd_tau), (g_tau, fd_tau)
    assert abs(g_tau - fd_tau_h) <= 1e-4 * abs(fd_tau_h)   # the plain h = 1e-4 bar
    fd_u, fd_u_h = richardson(lambda d: fd_objective(ni, tau, ulid + d, a, steps))
    assert abs(g_ulid - fd_u) <= tol * abs(fd_u), (g_ulid, fd_u)
    assert abs(g_ulid - fd_u_h) <= 1e-4 * abs(fd_u_h)
    # the lattice keeps the forward end state
    ref = O.cavity(ni, model="brinkman", tau=tau, ulid=ulid,
                   dtype=np.float32 if storage == "fp32" else np.float64, alpha=a)
    ref.step(steps)
    assert rel_maxnorm(lat.download_pops(), ref.pops) < {"fp64": 1e-12, "fp32s": 1e-6,
                                                         "fp32": 1e-5}[storage]
    # non-bulk cells carry no porosity gradient
    assert np.all(g_alpha.reshape(n, n, n)[0] == 0)


def test_adjoint_plain_bgk_tau_and_lid(gpu_ok):
    """Without a porosity field the adjoint still gives dJ/dtau and dJ/du_lid."""
    ni, tau, ulid, steps = 10, 0.6, 0.08, 40
    lat = F.cavity(ni, tau=tau, ulid=ulid, storage="fp64")
    lat.adjoint_forward(steps, 16)
    g_alpha, g_tau, g_ulid = lat.adjoint_backward(alpha_grad=False)
    assert g_alpha is None

    def J(t, u):
        m = F.cavity(ni, tau=t, ulid=u, storage="fp64")
        m.step(steps)
        return m.objective_u2()

    h = 1e-4
    d1 = (J(tau + h, ulid) - J(tau - h, ulid)) / (2 * h)
    d2 = (J(tau + h / 2, ulid) - J(tau - h / 2, ulid)) / h
    fd_tau = (4 * d2 - d1) / 3
    fd_u = (J(tau, ulid + h) - J(tau, ulid - h)) / (2 * h)
    assert abs(g_tau - fd_tau) <= 1e-6 * abs(fd_tau), (g_tau, fd_tau)
    assert abs(g_ulid - fd_u) <= 1e-6 * abs(fd_u), (g_ulid, fd_u)


@pytest.mark.parametrize("storage,tol", [("fp64", 1e-6), ("fp32s", 1e-4), ("fp32", 2e-3)])
def test_adjoint_mrt_tau_and_lid(gpu_ok, storage, tol):
    """MRT (Gram-Schmidt D3Q19 basis, shear rates 1/tau, others 1.2): the
    transposed collision Jacobian gives dJ/dtau and dJ/du_lid matching FP64
    central differences of the MRT forward."""
    ni, tau, ulid, steps = 10, 0.58, 0.08, 40
    lat = F.cavity(ni, tau=tau, ulid=ulid, storage=storage, model="mrt")
    J = lat.adjoint_forward(steps, 16)
    g_alpha, g_tau, g_ulid = lat.adjoint_backward(alpha_grad=False)

    def Jf(t, u):
        m = F.cavity(ni, tau=t, ulid=u, storage="fp64", model="mrt")
        m.step(steps)
        return m.objective_u2()

    assert abs(J - Jf(tau, ulid)) / J < {"fp64": 1e-12, "fp32s": 1e-6, "fp32": 1e-4}[storage]
    h = 1e-4
    d1 = (Jf(tau + h, ulid) - Jf(tau - h, ulid)) / (2 * h)
    d2 = (Jf(tau + h / 2, ulid) - Jf(tau - h / 2, ulid)) / h
    fd_tau = (4 * d2 - d1) / 3
    fd_u = (Jf(tau, ulid + h) - Jf(tau, ulid - h)) / (2 * h)
    assert abs(g_tau - fd_tau) <= tol * abs(fd_tau), (g_tau, fd_tau)
    assert abs(g_ulid - fd_u) <= tol * abs(fd_u), (g_ulid, fd_u)


def test_adjoint_rejects_unsupported(gpu_ok):
    lat = F.cavity(8, storage="fp16s")
    with pytest.raises(F.FlbError):
        lat.adjoint_forward(4, 2)
    lat2 = F.cavity(8, storage="fp64")
    with pytest.raises(F.FlbError):
        lat2.adjoint_backward()


@pytest.mark.skipif(O.ref_binary(np.float64) is None, reason="reference harness not built")
def test_adjoint_matches_reference_solver_finite_differences(gpu_ok):
    """dJ/dalpha and dJ/dtau of the FP64 device adjoint against central
    differences of the reference CPU solver itself (the harness's
    Brinkman-forced BGK built from the reference's ForcePop / SecondOrder /
    BGKForce), with J evaluated on the reference's own populations."""
    ni, tau, ulid, steps, h = 6, 0.6, 0.1, 25, 1e-4
    a = O.porosity(ni, 2)
    lat = brinkman_cavity(ni, tau, ulid, a, "fp64")
    lat.adjoint_forward(steps, 10)
    g_alpha, g_tau, _ = lat.adjoint_backward()

    def j_ref(al, t=tau):
        r = O.run_reference("brinkman", ni, t, ulid, steps, 0, dtype=np.float64, alpha=al,
                            threads=1)
        m = O.cavity(ni, model="brinkman", tau=t, dtype=np.float64, alpha=al)
        m.pops[:] = r["pops"]
        return m.objective_u2()

    fluid = np.flatnonzero(F.cavity_flags(ni) == 2)
    for c in (int(fluid[5]), int(fluid[len(fluid) // 2])):
        ap, am = a.copy(), a.copy()
        ap[c] += h
        am[c] -= h
        fd = (j_ref(ap) - j_ref(am)) / (2 * h)
        assert abs(g_alpha[c] - fd) <= 1e-6 * abs(fd), (c, g_alpha[c], fd)
    # tau: h and h/2 differences, Richardson-extrapolated
    d1 = (j_ref(a, tau + h) - j_ref(a, tau - h)) / (2 * h)
    d2 = (j_ref(a, tau + h / 2) - j_ref(a, tau - h / 2)) / h
    fd_tau = (4 * d2 - d1) / 3
    assert abs(g_tau - fd_tau) <= 1e-6 * abs(fd_tau), (g_tau, fd_tau)


@pytest.mark.parametrize("storage", ["fp64", "fp32s", "fp32"])
def test_objective_and_conservation_sums_are_deterministic(gpu_ok, storage):
    """J and the mass / momentum sums are FP64 reductions in a fixed order: the
    same state gives the same bits on every call (a finite difference of J at
    h = 1e-4 needs J to 1e-15 relative, below the jitter of atomic sums)."""
    lat = brinkman_cavity(40, 0.56, 0.1, O.porosity(40, 4), storage)
    lat.step(30)
    js = {lat.objective_u2() for _ in range(5)}
    assert len(js) == 1, js
    sums = [lat.conservation(key=2) for _ in range(5)]
    assert all(np.array_equal(s, sums[0]) for s in sums)
