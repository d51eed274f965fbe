"""sph_density_noalloc: the density entry point for callers that cannot
allocate device memory (code running inside another application's fixed
device-memory budget, or that must avoid the device synchronisation of
cudaMalloc/cudaFree).  It keeps its cell list in a fixed static device array
instead of allocating, so it is checked here against the allocating engine:
the same particles through sph_create + sph_density (direct summation,
adden = no, no periodic images) give rho within the FP64 parity tolerance,
1e-12 relative, on two calls in a row (the second call reuses the array the
first one left behind).

Cases: 1, 2 and 3 dimensions (y and z passed as NULL below 3) with the M4,
M6 and Gauss kernels; a particle count at the array's limit; a set whose
smallest h would need a cell grid far larger than the array holds, so the
cell edge is widened until it fits; and a smoothing length of 1e-12 in the
unit box, where the cells per axis approach 1e9 and their product would
overflow 64 bits if it were not checked one axis at a time.

This file is collected last, so a run that stops at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from sph_playground_b200 import abi, consts, ic

pytestmark = pytest.mark.gpu

COL = {k: v - 1 for k, v in consts.es.items()}
MAX_N = 262144  # SPH_NOALLOC_MAX_PARTICLES


def _bind(lib):
    f = lib.sph_density_noalloc
    P = ctypes.c_void_p
    f.argtypes = [P, P, P, P, P, ctypes.c_int64, ctypes.c_int, ctypes.c_int, P, P]
    f.restype = ctypes.c_int
    return f


def _particles(n, dim, seed=21):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 3))
    pos[:, :dim] = rng.uniform(0.0, 1.0, (n, dim))
    dx = (1.0 / n) ** (1.0 / dim)
    h = 1.2 * dx * rng.uniform(0.9, 1.1, n)
    m = np.full(n, 1.0 / n) * rng.uniform(0.8, 1.2, n)
    return pos, h, m


def _engine_density(lib, pos, h, m, dim, kernel):
    n = pos.shape[0]
    st = ic.make_state(dim, equations="hydro", adden="no", process="borderless", hfac=1.2)
    for k, v in (("realpn", n), ("fixedpn", 0), ("gamma", 5.0 / 3.0), ("dcondconst", 1.0),
                 ("time", 0.0), ("dtprint", 1.0)):
        ic.set_state(st, k, v)
    store = np.zeros((n, 32))
    store[:, 0:3] = pos
    store[:, COL["h"]] = h
    store[:, COL["m"]] = m
    store[:, COL["den"]] = 1.0
    store[:, COL["om"]] = 1.0
    store[:, COL["u"]] = 1.0
    store[:, COL["type"]] = consts.ept["real"]
    with abi.Engine(st, store, kernel, lib=lib) as e:
        e.density()
        return e.get_store()[:, COL["den"]]


def _check_two_calls(lib, pos, h, m, dim, kernel):
    import torch
    ref = _engine_density(lib, pos, h, m, dim, kernel)
    dev = torch.device("cuda:0")
    cols = [torch.tensor(np.ascontiguousarray(pos[:, k]), device=dev) for k in range(dim)]
    ptr = [c.data_ptr() for c in cols] + [None] * (3 - dim)
    th = torch.tensor(h, device=dev)
    tm = torch.tensor(m, device=dev)
    f = _bind(lib)
    for call in range(2):
        rho = torch.full((pos.shape[0],), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = f(ptr[0], ptr[1], ptr[2], tm.data_ptr(), th.data_ptr(), pos.shape[0], dim,
               consts.KERNELS[kernel], rho.data_ptr(), None)
        assert rc == 0, lib.sph_last_error()
        got = rho.cpu().numpy()
        err = float(np.max(np.abs(got - ref) / np.abs(ref)))
        assert err <= 1e-12, (call, err)


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("kernel", ["m4", "m6", "gauss"])
def test_density_noalloc_matches_engine(engine_lib, cuda_ok, dim, kernel):
    # the Gauss kernel reaches 10 h: fewer particles keep its rows short
    n = 1500 if kernel == "gauss" else 6000
    pos, h, m = _particles(n, dim)
    _check_two_calls(engine_lib, pos, h, m, dim, kernel)


def test_density_noalloc_at_the_limit(engine_lib, cuda_ok):
    pos, h, m = _particles(MAX_N, 3, seed=22)
    _check_two_calls(engine_lib, pos, h, m, 3, "m6")


@pytest.mark.parametrize("h_small", [1e-4, 1e-12])
def test_density_noalloc_widens_the_grid(engine_lib, cuda_ok, h_small):
    # one particle's h sets a cell edge of krad * h_small: the grid is
    # widened until it fits the array (and, at 1e-12, until each axis is
    # below 1e9 cells and their product below the cap)
    pos, h, m = _particles(4000, 3, seed=23)
    h[17] = h_small
    _check_two_calls(engine_lib, pos, h, m, 3, "m6")


def test_density_noalloc_rejects_oversize(engine_lib, cuda_ok):
    f = _bind(engine_lib)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = f(dummy, dummy, dummy, dummy, dummy, MAX_N + 1, 3, 1, dummy, None)
    assert rc == 1  # SPH_ERR_ARG
    assert b"262144" in engine_lib.sph_last_error()
