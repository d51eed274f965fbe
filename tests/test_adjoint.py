"""Gradients of a final-state misfit through the engine's adjoint kernels
(sph_adjoint_forward / sph_adjoint_backward and the torch.autograd.Function
in sph_playground_b200/adjoint.py), on the 2D periodic shear flow of the
adjoint workload at a small size.  Checked against central finite
differences of the same forward map (eps = 1e-6) along random directions of
v0, u0, r0, single velocity components, and for alpha and beta; FP32-comp
gradients against the FP64 gradient.  Tolerances are stated per check."""
import numpy as np
import pytest

from sph_playground_b200 import abi, consts, ic

pytestmark = pytest.mark.gpu

V = [consts.es["vx"] - 1, consts.es["vy"] - 1, consts.es["vz"] - 1]
R = [0, 1, 2]
U = consts.es["u"] - 1
NSTEPS, EVERY, DT = 7, 3, 4e-3


def _setup(n=12):
    st, store = ic.shear2d(n=n)
    ic.set_state(st, "adden", consts.eif["yes"])
    ic.set_state(st, "artts", consts.eif["yes"])
    return st, store


def _run(lib, st, store, alpha=1.0, beta=2.0, prec=abi.PREC_FP64):
    e = abi.Engine(st, store, "m6", precision=prec, lib=lib)
    e.set_param(abi.P_AV_ALPHA, alpha)
    e.set_param(abi.P_AV_BETA, beta)
    e.set_param(abi.P_FIXED_DT, DT)
    e.adjoint_forward(NSTEPS, EVERY)
    return e


def _loss(vT, target):
    return float(np.sum((vT - target) ** 2))


def _target(store):
    rng = np.random.default_rng(11)
    t = store[:, V] * 1.2
    t[:, :2] += rng.normal(0, 1e-3, (store.shape[0], 2))
    t[:, 2] = 0.0
    return t


def _grads(lib, st, store, target, prec=abi.PREC_FP64):
    e = _run(lib, st, store, prec=prec)
    try:
        vT = e.get_store()[:, V]
        g = e.adjoint_backward(dl_dv=2.0 * (vT - target))
        return _loss(vT, target), g
    finally:
        e.close()


def _fd(lib, st, store, target, perturb, eps=1e-6):
    vals = []
    for sgn in (1.0, -1.0):
        s2, st2, kw2 = perturb(sgn * eps)
        e = _run(lib, st2, s2, **kw2)
        try:
            vals.append(_loss(e.get_store()[:, V], target))
        finally:
            e.close()
    return (vals[0] - vals[1]) / (2 * eps)


def _direction(n, cols, seed):
    d = np.random.default_rng(seed).normal(size=(n, len(cols)))
    if len(cols) == 3:
        d[:, 2] = 0.0  # 2D
    return d


def test_gradient_v0_matches_fd(engine_lib, cuda_ok):
    # With alpha = 0 the viscosity term is C1 in v (beta dn^2), so a random
    # direction through every particle is a clean finite-difference check.
    st, store = _setup()
    target = _target(store)
    e = _run(engine_lib, st, store, alpha=0.0)
    try:
        vT = e.get_store()[:, V]
        g = e.adjoint_backward(dl_dv=2.0 * (vT - target))
    finally:
        e.close()
    d = _direction(store.shape[0], V, 1)

    def pert(eps):
        s2 = store.copy()
        s2[:, V] += eps * d
        return s2, st, {"alpha": 0.0}
    fd = _fd(engine_lib, st, store, target, pert)
    ad = float(np.sum(g["g_v0"] * d))
    assert abs(ad - fd) <= 1e-6 * abs(fd) + 1e-10, (ad, fd)


def test_gradient_v0_single_particles_with_alpha(engine_lib, cuda_ok):
    # The alpha term switches on at v_ab . r_ab = 0 (dn = min(s, 0),
    # circuit2.f90:294-336), a kink in v; a random direction through all
    # particles crosses it for a few pairs within eps, so the alpha case is
    # checked one particle's velocity at a time.
    st, store = _setup()
    target = _target(store)
    _, g = _grads(engine_lib, st, store, target)
    for i in (0, 5, 37, 100):
        for comp in (0, 1):
            def pert(eps):
                s2 = store.copy()
                s2[i, V[comp]] += eps
                return s2, st, {}
            fd = _fd(engine_lib, st, store, target, pert)
            ad = float(g["g_v0"][i, comp])
            assert abs(ad - fd) <= 1e-6 * abs(fd) + 1e-10, (i, comp, ad, fd)


def test_gradient_u0_and_r0_match_fd(engine_lib, cuda_ok):
    st, store = _setup()
    target = _target(store)
    _, g = _grads(engine_lib, st, store, target)
    du = np.random.default_rng(2).normal(size=store.shape[0]) * store[:, U]

    def pert_u(eps):
        s2 = store.copy()
        s2[:, U] += eps * du
        return s2, st, {}
    fd_u = _fd(engine_lib, st, store, target, pert_u)
    ad_u = float(np.sum(g["g_u0"] * du))
    assert abs(ad_u - fd_u) <= 1e-5 * abs(fd_u) + 1e-10, (ad_u, fd_u)
    dx = _direction(store.shape[0], R, 3) * 1e-2  # positions: a small fraction of dx

    def pert_r(eps):
        s2 = store.copy()
        s2[:, R] += eps * dx
        return s2, st, {}
    fd_r = _fd(engine_lib, st, store, target, pert_r)
    ad_r = float(np.sum(g["g_r0"] * dx))
    assert abs(ad_r - fd_r) <= 1e-5 * abs(fd_r) + 1e-10, (ad_r, fd_r)


@pytest.mark.parametrize("which", [0, 1])
def test_gradient_viscosity_params_match_fd(engine_lib, cuda_ok, which):
    st, store = _setup()
    target = _target(store)
    _, g = _grads(engine_lib, st, store, target)

    def pert(eps):
        kw = {"alpha": 1.0 + (eps if which == 0 else 0.0), "beta": 2.0 + (eps if which == 1 else 0.0)}
        return store, st, kw
    fd = _fd(engine_lib, st, store, target, pert)
    ad = float(g["g_par"][which])
    assert abs(ad - fd) <= 1e-5 * abs(fd) + 1e-10, (which, ad, fd)


def test_fp32_gradient_near_fp64(engine_lib, cuda_ok):
    st, store = _setup()
    target = _target(store)
    _, g64 = _grads(engine_lib, st, store, target, abi.PREC_FP64)
    _, g32 = _grads(engine_lib, st, store, target, abi.PREC_FP32_COMP)
    rel = np.linalg.norm(g32["g_v0"] - g64["g_v0"]) / np.linalg.norm(g64["g_v0"])
    assert rel <= 1e-4, rel


def test_torch_function(engine_lib, cuda_ok):
    import torch
    from sph_playground_b200.adjoint import Rollout, RolloutSetup
    st, store = _setup()
    target = _target(store)
    setup = RolloutSetup(st, store, NSTEPS, EVERY, DT, lib=engine_lib)
    v0 = torch.tensor(store[:, V], dtype=torch.float64, requires_grad=True)
    alpha = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    beta = torch.tensor(2.0, dtype=torch.float64, requires_grad=True)
    vT = Rollout.apply(v0, alpha, beta, setup)
    loss = ((vT - torch.as_tensor(target)) ** 2).sum()
    loss.backward()
    _, g = _grads(engine_lib, st, store, target)
    assert np.allclose(v0.grad.numpy(), g["g_v0"], rtol=1e-12, atol=1e-14)
    assert alpha.grad.item() == pytest.approx(g["g_par"][0], rel=1e-12)
    assert beta.grad.item() == pytest.approx(g["g_par"][1], rel=1e-12)


def test_adjoint_rejects_other_equations(engine_lib, cuda_ok):
    st, store = ic.diffusion2d(12, tfinish=1e-3)
    with abi.Engine(st, store, "m6", lib=engine_lib) as e:
        e.set_param(abi.P_FIXED_DT, 1e-4)
        with pytest.raises(abi.SphError) as ex:
            e.adjoint_forward(2, 1)
        assert ex.value.status == "SPH_ERR_UNSUPPORTED"


# ---- the diffusion adjoint: dL/dT0 and dL/d difcond ---------------------------------------
T_COL = consts.es["t"] - 1
D_STEPS, D_EVERY, D_DT = 10, 4, 2e-4


def _diff_setup(ddw, full):
    st, store = ic.diffusion2d(16, ddw=ddw, full_tensor=full)
    ic.set_state(st, "eqonsts", 0.0)  # leapfrog on T (the differentiated integrator)
    return st, store


def _diff_run(lib, st, store, full, prec=abi.PREC_FP64):
    e = abi.Engine(st, store, "m6", precision=prec, lib=lib)
    e.set_param(abi.P_FULL_TENSOR, 1.0 if full else 0.0)
    e.set_param(abi.P_FIXED_DT, D_DT)
    e.adjoint_forward(D_STEPS, D_EVERY)
    return e


def _diff_loss(T, target):
    return float(np.sum((T - target) ** 2))


@pytest.mark.parametrize("ddw,full", [("fab", False), ("fw", False), ("n2w", False),
                                      ("fab", True)])
def test_diffusion_gradients_match_fd(engine_lib, cuda_ok, ddw, full):
    """dL/dT0 along a random direction and dL/d difcond against central
    differences (the map is linear in T0 and in difcond, so the differences
    are exact up to rounding): relative 1e-6."""
    st, store = _diff_setup(ddw, full)
    target = 0.9 * store[:, T_COL]
    e = _diff_run(engine_lib, st, store, full)
    T = e.get_store()[:, T_COL]
    gT0, gdc = e.adjoint_backward_diffusion(2.0 * (T - target))
    e.close()
    rng = np.random.default_rng(7)
    d = rng.normal(size=store.shape[0])
    eps = 1e-6

    def loss_at(T0=None, dc=None):
        s2, st2 = store.copy(), st.copy()
        if T0 is not None:
            s2[:, T_COL] = T0
        if dc is not None:
            ic.set_state(st2, "dcondconst", dc)
        e2 = _diff_run(engine_lib, st2, s2, full)
        try:
            return _diff_loss(e2.get_store()[:, T_COL], target)
        finally:
            e2.close()
    fd_T = (loss_at(T0=store[:, T_COL] + eps * d) - loss_at(T0=store[:, T_COL] - eps * d)) / (2 * eps)
    assert float(gT0 @ d) == pytest.approx(fd_T, rel=1e-6)
    dc0 = ic.get_state(st, "dcondconst")
    fd_dc = (loss_at(dc=dc0 + eps) - loss_at(dc=dc0 - eps)) / (2 * eps)
    assert gdc == pytest.approx(fd_dc, rel=1e-6)


def test_diffusion_gradient_fp32_near_fp64(engine_lib, cuda_ok):
    st, store = _diff_setup("fab", False)
    target = 0.9 * store[:, T_COL]
    out = []
    for prec in (abi.PREC_FP64, abi.PREC_FP32_COMP):
        e = _diff_run(engine_lib, st, store, False, prec)
        T = e.get_store()[:, T_COL]
        out.append(e.adjoint_backward_diffusion(2.0 * (T - target)))
        e.close()
    (g64, d64), (g32, d32) = out
    assert np.linalg.norm(g32 - g64) <= 1e-4 * np.linalg.norm(g64)
    assert d32 == pytest.approx(d64, rel=1e-4)


def test_diffusion_adjoint_rejects_sts(engine_lib, cuda_ok):
    st, store = ic.diffusion2d(16, ddw="fab")  # fixed-stage STS integrator
    e = abi.Engine(st, store, "m6", lib=engine_lib)
    e.set_param(abi.P_FIXED_DT, D_DT)
    with pytest.raises(abi.SphError) as ex:
        e.adjoint_forward(2, 1)
    assert ex.value.status == "SPH_ERR_UNSUPPORTED"
    e.close()


def test_diffusion_torch_function(engine_lib, cuda_ok):
    import torch
    from sph_playground_b200.adjoint import DiffusionRollout, RolloutSetup
    st, store = _diff_setup("fab", False)
    target = 0.9 * store[:, T_COL]
    setup = RolloutSetup(st, store, D_STEPS, D_EVERY, D_DT, lib=engine_lib)
    T0 = torch.tensor(store[:, T_COL], dtype=torch.float64, requires_grad=True)
    dc = torch.tensor(ic.get_state(st, "dcondconst"), dtype=torch.float64, requires_grad=True)
    TT = DiffusionRollout.apply(T0, dc, setup)
    ((TT - torch.as_tensor(target)) ** 2).sum().backward()
    e = _diff_run(engine_lib, st, store, False)
    T = e.get_store()[:, T_COL]
    gT0, gdc = e.adjoint_backward_diffusion(2.0 * (T - target))
    e.close()
    assert np.allclose(T0.grad.numpy(), gT0, rtol=1e-12, atol=1e-14)
    assert dc.grad.item() == pytest.approx(gdc, rel=1e-12)


def test_adjoint_workload_fd_spot_check(engine_lib, cuda_ok):
    """The adjoint workload itself at its FP64 check size: shear flow on a
    64^2 periodic lattice, M6, alpha = 1, beta = 2, 200 fixed-dt leapfrog
    steps (dt 5e-4) with a checkpoint every 20 steps and recomputation in
    between; the target is the final velocity field of the same run started
    with shear amplitude 0.12 instead of 0.1.  Central differences
    (eps = 1e-6) of the loss against the
    adjoint for alpha and for single initial velocity components; the
    tolerance, 1e-4 relative, allows for the few pairs whose v_ab . r_ab
    crosses the viscosity's switch within eps over 200 steps."""
    n, nsteps, every, dt, eps = 64, 200, 20, 5e-4, 1e-6
    st, store = ic.shear2d(n=n)

    def run(s, alpha=1.0):
        e = abi.Engine(st, s, "m6", lib=engine_lib)
        e.set_param(abi.P_AV_ALPHA, alpha)
        e.set_param(abi.P_FIXED_DT, dt)
        e.adjoint_forward(nsteps, every)
        return e

    e = run(ic.shear2d(n=n, amp=0.12)[1])
    try:
        target = e.get_store()[:, V]
    finally:
        e.close()
    e = run(store)
    try:
        vT = e.get_store()[:, V]
        g = e.adjoint_backward(dl_dv=2.0 * (vT - target))
    finally:
        e.close()

    def loss(s, alpha=1.0):
        e = run(s, alpha)
        try:
            return _loss(e.get_store()[:, V], target)
        finally:
            e.close()
    fd = (loss(store, 1.0 + eps) - loss(store, 1.0 - eps)) / (2 * eps)
    ad = float(g["g_par"][0])
    assert abs(ad - fd) <= 1e-4 * abs(fd), ("alpha", ad, fd)
    for i in (0, 1234, 3001):
        sp, sm = store.copy(), store.copy()
        sp[i, V[0]] += eps
        sm[i, V[0]] -= eps
        fd = (loss(sp) - loss(sm)) / (2 * eps)
        ad = float(g["g_v0"][i, 0])
        assert abs(ad - fd) <= 1e-4 * abs(fd) + 1e-9, (i, ad, fd)
