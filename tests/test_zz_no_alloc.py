"""sph_density_noalloc: the density entry point for callers that cannot
allocate device memory (code running inside another application's fixed
device-memory budget, or that must avoid the device synchronisation of
cudaMalloc/cudaFree).  It keeps its cell list in a fixed static device array
instead of allocating, so it is checked here against the allocating engine:
the same particles through sph_create + sph_density (direct summation,
adden = no, no periodic images) give rho within the FP64 parity tolerance,
1e-12 relative, on two calls in a row (the second call reuses the array the
first one left behind).

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


def _particles(n=6000, seed=21):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, 1.0, (n, 3))
    dx = (1.0 / n) ** (1.0 / 3.0)
    h = 1.2 * dx * rng.uniform(0.9, 1.1, n)
    m = np.full(n, 1.0 / n) * rng.uniform(0.8, 1.2, n)
    return pos, h, m


def _engine_density(lib, pos, h, m):
    n = pos.shape[0]
    st = ic.make_state(3, equations="hydro", adden="no", process="borderless", hfac=1.2)
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
    with abi.Engine(st, store, "m6", lib=lib) as e:
        e.density()
        return e.get_store()[:, COL["den"]]


def test_density_noalloc_matches_engine(engine_lib, cuda_ok):
    import torch
    pos, h, m = _particles()
    ref = _engine_density(engine_lib, pos, h, m)
    dev = torch.device("cuda:0")
    x, y, z = (torch.tensor(np.ascontiguousarray(pos[:, k]), device=dev) for k in range(3))
    th = torch.tensor(h, device=dev)
    tm = torch.tensor(m, device=dev)
    f = _bind(engine_lib)
    for call in range(2):
        rho = torch.full((pos.shape[0],), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = f(x.data_ptr(), y.data_ptr(), z.data_ptr(), tm.data_ptr(), th.data_ptr(),
               pos.shape[0], 3, consts.KERNELS["m6"], rho.data_ptr(), None)
        assert rc == 0, engine_lib.sph_last_error()
        got = rho.cpu().numpy()
        err = float(np.max(np.abs(got - ref) / np.abs(ref)))
        assert err <= 1e-12, (call, err)


def test_density_noalloc_rejects_oversize(engine_lib, cuda_ok):
    f = _bind(engine_lib)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = f(dummy, dummy, dummy, dummy, dummy, MAX_N + 1, 3, 1, dummy, None)
    assert rc == 1  # SPH_ERR_ARG
    assert b"262144" in engine_lib.sph_last_error()
