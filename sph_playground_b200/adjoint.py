"""Differentiable rollouts: a torch.autograd.Function over the engine's
fixed-dt hydro steps (sph_adjoint_forward / sph_adjoint_backward).

The forward runs `nsteps` leapfrog steps of the engine from a given
particle table with the initial velocities and the artificial-viscosity
parameters (alpha, beta) as inputs, and returns the final velocities; the
backward runs the engine's hand-written adjoint kernels, replaying the run
from copies of the particle table taken every `every` steps.  PyTorch is only
the front end: the numbers come from the CUDA engine.

    setup = RolloutSetup(state, store, nsteps=200, every=20, dt=1e-4)
    vT = Rollout.apply(v0, alpha, beta, setup)
    loss = ((vT - v_target) ** 2).sum()
    loss.backward()            # v0.grad, alpha.grad, beta.grad

For a diffusion run (fixed positions, leapfrog on T) the same setup drives
DiffusionRollout: T(T) from the initial temperatures and the conductivity
(state slot dcondconst), gradients by sph_adjoint_backward_diffusion.

    TT = DiffusionRollout.apply(T0, difcond, setup)
"""
from dataclasses import dataclass, field

import numpy as np
import torch

from . import abi, consts

_V = [consts.es["vx"] - 1, consts.es["vy"] - 1, consts.es["vz"] - 1]


@dataclass
class RolloutSetup:
    """Initial particle table (velocities replaced by the v0 input), run
    length, checkpoint spacing and step size."""
    state: np.ndarray
    store: np.ndarray
    nsteps: int
    every: int
    dt: float
    kernel: str = "m6"
    precision: int = abi.PREC_FP64
    params: dict = field(default_factory=dict)
    lib: object = None
    engines: list = field(default_factory=list)  # open engines of pending backwards


def _engine(setup, v0, alpha, beta):
    store = np.array(setup.store, dtype=np.float64, copy=True)
    store[:, _V] = np.asarray(v0, dtype=np.float64).reshape(-1, 3)
    e = abi.Engine(setup.state, store, setup.kernel, precision=setup.precision, lib=setup.lib)
    for k, v in setup.params.items():
        e.set_param(k, v)
    e.set_param(abi.P_AV_ALPHA, float(alpha))
    e.set_param(abi.P_AV_BETA, float(beta))
    e.set_param(abi.P_FIXED_DT, float(setup.dt))
    return e


def final_velocities(setup, v0, alpha, beta):
    """The forward map alone (no graph): v(T) as a numpy array."""
    e = _engine(setup, v0, alpha, beta)
    try:
        e.adjoint_forward(setup.nsteps, setup.every)
        return e.get_store()[:, _V]
    finally:
        e.close()


class Rollout(torch.autograd.Function):
    """v(T) = rollout(v0, alpha, beta); gradients by the engine's adjoint."""

    @staticmethod
    def forward(ctx, v0, alpha, beta, setup):
        e = _engine(setup, v0.detach().cpu().numpy(), alpha.item(), beta.item())
        try:
            e.adjoint_forward(setup.nsteps, setup.every)
            vT = e.get_store()[:, _V]
        except Exception:
            e.close()
            raise
        ctx.engine = e
        ctx.dev, ctx.dtype = v0.device, v0.dtype
        return torch.as_tensor(vT, dtype=v0.dtype, device=v0.device)

    @staticmethod
    def backward(ctx, g_vT):
        e = ctx.engine
        try:
            res = e.adjoint_backward(dl_dv=g_vT.detach().cpu().numpy())
        finally:
            e.close()
            ctx.engine = None
        t = lambda a: torch.as_tensor(a, dtype=ctx.dtype, device=ctx.dev)  # noqa: E731
        return t(res["g_v0"]), t(res["g_par"][0]), t(res["g_par"][1]), None


_T = consts.es["t"] - 1


def _diffusion_engine(setup, T0, difcond):
    store = np.array(setup.store, dtype=np.float64, copy=True)
    store[:, _T] = np.asarray(T0, dtype=np.float64).reshape(-1)
    state = np.array(setup.state, dtype=np.float64, copy=True)
    state[consts.ec["dcondconst"] - 1] = float(difcond)
    e = abi.Engine(state, store, setup.kernel, precision=setup.precision, lib=setup.lib)
    for k, v in setup.params.items():
        e.set_param(k, v)
    e.set_param(abi.P_FIXED_DT, float(setup.dt))
    return e


class DiffusionRollout(torch.autograd.Function):
    """T(T) = rollout(T0, difcond) of a diffusion run; gradients by the
    engine's adjoint of the diffusion term."""

    @staticmethod
    def forward(ctx, T0, difcond, setup):
        e = _diffusion_engine(setup, T0.detach().cpu().numpy(), difcond.item())
        try:
            e.adjoint_forward(setup.nsteps, setup.every)
            TT = e.get_store()[: e.n_real, _T]
        except Exception:
            e.close()
            raise
        ctx.engine = e
        ctx.dev, ctx.dtype = T0.device, T0.dtype
        return torch.as_tensor(TT, dtype=T0.dtype, device=T0.device)

    @staticmethod
    def backward(ctx, g_TT):
        e = ctx.engine
        try:
            g_T0, g_dc = e.adjoint_backward_diffusion(g_TT.detach().cpu().numpy())
        finally:
            e.close()
            ctx.engine = None
        t = lambda a: torch.as_tensor(a, dtype=ctx.dtype, device=ctx.dev)  # noqa: E731
        return t(g_T0), t(g_dc), None
