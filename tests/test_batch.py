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
    out = []
    for st, store in _instances():
        with abi.Engine(st, store, "m6", precision=prec, lib=lib) as e:
            e.run_to(T_END)
            out.append((e.get_store(), e.get_state()))
    return out


def _batched(lib, prec=abi.PREC_FP64, steps=None):
    engines = [abi.Engine(st, store, "m6", precision=prec, lib=lib) for st, store in _instances()]
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
