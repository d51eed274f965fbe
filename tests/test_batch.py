"""Batches of instances (sph_batch_*): several runs stepped together give
what each run gives alone.  The CPU tests drive the oracle's batch (the
reference's sequential sweep); the GPU tests drive the engine's concurrent
batch, against single engine runs (bit-exact: every instance runs the same
kernels on its own stream) and against the oracle (parity tolerance)."""
import numpy as np
import pytest

from sph_playground_b200 import abi, consts, ic

from parity import rel_field

T_END = 2e-3
SWEEP = [(12, "fab"), (16, "n2w"), (20, "2nw_ds")]  # (lattice per axis, ddw method)


def _instances():
    return [ic.diffusion2d(n, ddw=ddw, tfinish=T_END, sts_stages=4) for n, ddw in SWEEP]


def _alone(lib, prec=abi.PREC_FP64):
    # a fresh search every iterate, as the batch's device loop takes (skin
    # lists give the same sets in another order, so not the same bits)
    out = []
    for st, store in _instances():
        with abi.Engine(st, store, "m6", precision=prec, lib=lib) as e:
            e.set_param(abi.P_SKIN, 0.0)
            e.run_to(T_END)
            out.append((e.get_store(), e.get_state()))
    return out


def _batched(lib, prec=abi.PREC_FP64, steps=None):
    engines = [abi.Engine(st, store, "m6", precision=prec, lib=lib) for st, store in _instances()]
    for e in engines:
        e.set_param(abi.P_SKIN, 0.0)
    try:
        with abi.Batch(engines) as b:
            if steps is None:
                b.run_to(T_END)
            else:
                b.step(steps)
            assert b.status() == [0] * len(engines)
        return [(e.get_store(), e.get_state()) for e in engines]
    finally:
        for e in engines:
            e.close()


def test_batch_oracle_matches_single_runs(oracle_lib):
    alone, batched = _alone(oracle_lib), _batched(oracle_lib)
    for (s1, t1), (s2, t2) in zip(alone, batched):
        assert np.array_equal(s1, s2)
        assert np.array_equal(t1, t2)
        assert t1[consts.ec["time"] - 1] == pytest.approx(T_END)


def test_batch_reports_failing_instance(oracle_lib):
    insts = _instances()
    st, store = insts[1]
    store = store.copy()
    store[3, consts.es["den"] - 1] = -1.0  # preruncheck: density <= 0
    engines = [abi.Engine(*insts[0], "m6", lib=oracle_lib), abi.Engine(st, store, "m6", lib=oracle_lib)]
    try:
        with abi.Batch(engines) as b:
            with pytest.raises(abi.SphError) as ex:
                b.run_to(T_END)
            assert "instance 1" in str(ex.value)
            assert b.status()[0] == 0 and b.status()[1] != 0
    finally:
        for e in engines:
            e.close()


def test_batch_rejects_repeated_handle(oracle_lib):
    e = abi.Engine(*_instances()[0], "m6", lib=oracle_lib)
    try:
        with pytest.raises(abi.SphError):
            abi.Batch([e, e])
    finally:
        e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_batch_engine_matches_single_runs(engine_lib, cuda_ok, prec):
    alone, batched = _alone(engine_lib, prec), _batched(engine_lib, prec)
    for (s1, t1), (s2, t2) in zip(alone, batched):
        assert np.array_equal(s1, s2)
        assert np.array_equal(t1, t2)


@pytest.mark.gpu
def test_batch_engine_matches_oracle(engine_lib, oracle_lib, cuda_ok):
    ref, got = _alone(oracle_lib), _batched(engine_lib)
    col = consts.es["t"] - 1
    for (s_ref, _), (s_got, _) in zip(ref, got):
        assert rel_field(s_got[:, col], s_ref[:, col]) <= 1e-11


@pytest.mark.gpu
def test_batch_engine_step_count(engine_lib, cuda_ok):
    batched = _batched(engine_lib, steps=2)
    for _, st in batched:
        assert st[consts.ec["time"] - 1] > 0.0


# ---- the engine's device loop (one CUDA graph per launch over all instances) ----

SWEEP_FULL = [(n, ddw) for ddw in ("fab", "n2w", "2nw_ds")
              for n in (32, 48, 64, 96, 128, 192, 256)]


def _engines(lib, sets, prec, params=None):
    # a fresh search every iterate, as the device loop's steps take (skin
    # lists give the same sets in another order, so not the same bits)
    out = []
    for st, store in sets:
        e = abi.Engine(st, store, "m6", precision=prec, lib=lib)
        e.set_param(abi.P_SKIN, 0.0)
        for k, v in (params or {}).items():
            e.set_param(k, v)
        out.append(e)
    return out


def _alone_and_batched(lib, sets, prec, run, params=None):
    alone = []
    for e in _engines(lib, sets, prec, params):
        run(e)
        alone.append((e.get_store(), e.get_state(), e.counters()))
        e.close()
    eng = _engines(lib, sets, prec, params)
    try:
        with abi.Batch(eng) as b:
            run(b)
            assert b.status() == [0] * len(eng)
        batched = [(e.get_store(), e.get_state(), e.counters()) for e in eng]
    finally:
        for e in eng:
            e.close()
    return alone, batched


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_batch_device_loop_full_sweep(engine_lib, cuda_ok, prec):
    """The 21 uneven instances of the convergence sweep (7 lattices x 3
    second-derivative methods, fixed-stage STS to t = 0.01) stepped by the
    batch's device loop equal the instances run alone on the host path, bit
    for bit, and the loop took their steps."""
    sets = [ic.diffusion2d(n, ddw=ddw, tfinish=0.01) for n, ddw in SWEEP_FULL]
    alone, batched = _alone_and_batched(engine_lib, sets, prec, lambda x: x.run_to(0.01))
    for (s1, t1, _), (s2, t2, c2) in zip(alone, batched):
        assert np.array_equal(t1, t2)
        assert np.array_equal(s1, s2)
        assert c2["graph_steps"] >= c2["steps"] - 1 and c2["graph_steps"] > 0, c2


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_batch_device_loop_reorders_rows(engine_lib, cuda_ok, prec):
    """Hydro instances of different sizes re-ordering their rows every 2
    steps inside the device loop (in place, gated on the device) equal the
    host path, which re-orders by swapping tables."""
    sets = [ic.sedov3d(n=10, tfinish=1.0), ic.sedov3d(n=13, tfinish=1.0),
            ic.sod2d(tfinish=1.0)]
    alone, batched = _alone_and_batched(engine_lib, sets, prec, lambda x: x.step(9),
                                        params={abi.P_REORDER_EVERY: 2})
    for (s1, t1, c1), (s2, t2, c2) in zip(alone, batched):
        assert c1["steps"] == c2["steps"] == 9
        assert c2["graph_steps"] >= 8, c2
        assert np.array_equal(t1, t2)
        assert np.array_equal(s1, s2)


@pytest.mark.gpu
def test_batch_device_loop_redoes_on_the_host(engine_lib, cuda_ok):
    """A Newton tolerance no sweep count meets makes every device-resident
    step report it; the loop stops, that instance's step is redone on the
    host path from the saved table and clock, and the result equals the
    host path's."""
    params = {abi.P_NEWTON_TOL: 1e-300, abi.P_NEWTON_MAXITER: 9}
    sets = [ic.diffusion2d(16, ddw="2nw_ds", sts_stages=4, tfinish=1.0),
            ic.diffusion2d(20, ddw="fab", sts_stages=4, tfinish=1.0)]
    alone, batched = _alone_and_batched(engine_lib, sets, abi.PREC_FP64, lambda x: x.step(3),
                                        params=params)
    assert batched[0][2]["graph_redos"] >= 2
    for (s1, t1, _), (s2, t2, _) in zip(alone, batched):
        assert np.array_equal(t1, t2)
        assert np.array_equal(s1, s2)


@pytest.mark.gpu
def test_batch_device_loop_reports_failing_instance(engine_lib, cuda_ok):
    insts = _instances()
    st, store = insts[1]
    store = store.copy()
    store[3, consts.es["den"] - 1] = -1.0  # preruncheck: density <= 0
    engines = [abi.Engine(*insts[0], "m6", lib=engine_lib),
               abi.Engine(st, store, "m6", lib=engine_lib)]
    try:
        with abi.Batch(engines) as b:
            with pytest.raises(abi.SphError) as ex:
                b.run_to(T_END)
            assert "instance 1" in str(ex.value)
            assert b.status()[0] == 0 and b.status()[1] != 0
        t0 = engines[0].get_state()[consts.ec["time"] - 1]
        assert t0 == pytest.approx(T_END)
    finally:
        for e in engines:
            e.close()
