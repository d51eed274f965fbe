"""Device-resident steps replayed as CUDA graphs (SPH_P_GRAPH): the same
kernels as the host-driven step with every size and decision taken on the
device, so the results must equal the host-driven step's bit for bit (the
host step with a fresh search every iterate, SPH_P_SKIN = 0, as the graph
takes: skin lists give the same sets in another order); a step that cannot
be planned on the device (here: Newton sweeps beyond the device-resident
limit) is redone on the host path, with the same result."""
import numpy as np
import pytest

from sph_playground_b200 import abi, consts, ic

pytestmark = pytest.mark.gpu

FP64, FP32 = abi.PREC_FP64, abi.PREC_FP32_COMP


def _run(lib, st, store, prec, steps, graph, kernel="m6", params=None):
    with abi.Engine(st, store, kernel, precision=prec, lib=lib) as e:
        e.set_param(abi.P_SKIN, 0.0)
        for k, v in (params or {}).items():
            e.set_param(k, v)
        e.set_param(abi.P_GRAPH, 1.0 if graph else 0.0)
        e.step(steps)
        return e.get_store(), e.get_state(), e.counters()


CASES = {
    "sedov3d": lambda: ic.sedov3d(n=12, tfinish=1.0),
    "sod_shock12": lambda: ic.sod2d(tfinish=0.2),
    "diffusion_sts_fab": lambda: ic.diffusion2d(16, ddw="fab", sts_stages=4, tfinish=1.0),
    "diffusion_sts_2nw": lambda: ic.diffusion2d(16, ddw="2nw_ds", sts_stages=4, tfinish=1.0),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("prec", [FP64, FP32])
def test_graph_steps_equal_host_steps(engine_lib, cuda_ok, case, prec):
    st, store = CASES[case]()
    steps = 10  # past a row re-ordering (every 8 steps), which re-captures the graph
    s0, t0, c0 = _run(engine_lib, st, store, prec, steps, graph=False)
    s1, t1, c1 = _run(engine_lib, st, store, prec, steps, graph=True)
    assert c1["steps"] == c0["steps"] == steps
    assert c1["graph_steps"] + c1["graph_redos"] >= steps - 1  # the first step starts the run
    assert c1["graph_steps"] >= steps - 2
    assert np.array_equal(t0, t1)
    assert np.array_equal(s0, s1)


def test_graph_redo_on_the_host_path(engine_lib, cuda_ok):
    # a Newton tolerance no sweep count meets: every device-resident step
    # reports it and is redone on the host path (up to the sweep cap)
    st, store = ic.diffusion2d(16, ddw="2nw_ds", sts_stages=4, tfinish=1.0)
    params = {abi.P_NEWTON_TOL: 1e-300, abi.P_NEWTON_MAXITER: 9}
    s0, t0, _ = _run(engine_lib, st, store, FP64, 3, graph=False, params=params)
    s1, t1, c1 = _run(engine_lib, st, store, FP64, 3, graph=True, params=params)
    assert c1["graph_redos"] >= 2
    assert np.array_equal(t0, t1)
    assert np.array_equal(s0, s1)


def test_graph_falls_back_where_not_eligible(engine_lib, cuda_ok):
    # the radiation exchange runs on the host path only
    st, store = ic.hyrad1d(64, kernel="m6", exchange_only=True)
    s0, t0, _ = _run(engine_lib, st, store, FP64, 2, graph=False)
    s1, t1, c1 = _run(engine_lib, st, store, FP64, 2, graph=True)
    assert c1["graph_steps"] == 0
    assert np.array_equal(s0, s1)


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_graph_reorder_every_two_steps(engine_lib, cuda_ok, prec):
    # the table alternates between two buffers: each buffer's capture is
    # replayed again after the next reordering
    st, store = ic.sedov3d(n=12, tfinish=1.0)
    params = {abi.P_REORDER_EVERY: 2}
    s0, t0, _ = _run(engine_lib, st, store, prec, 12, graph=False, params=params)
    s1, t1, c1 = _run(engine_lib, st, store, prec, 12, graph=True, params=params)
    assert c1["graph_steps"] >= 10
    assert np.array_equal(t0, t1)
    assert np.array_equal(s0, s1)


def test_graph_parameter_change_mid_run(engine_lib, cuda_ok):
    # a parameter set between steps must reach the next replayed step
    st, store = ic.diffusion2d(16, ddw="fab", sts_stages=4, tfinish=1.0)
    out = []
    for graph in (False, True):
        with abi.Engine(st, store, "m6", precision=FP64, lib=engine_lib) as e:
            e.set_param(abi.P_SKIN, 0.0)  # (as the graph's steps: a fresh search)
            e.set_param(abi.P_GRAPH, 1.0 if graph else 0.0)
            e.step(4)
            e.set_param(abi.P_NEWTON_TOL, 1e-6)
            e.step(4)
            out.append((e.get_store(), e.get_state(), e.counters()))
    assert out[1][2]["graph_steps"] >= 6
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][0], out[1][0])
