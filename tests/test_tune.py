"""The autotuner's search and cache logic (sph_playground_b200/tune.py) with
an injected timing function (the device timings themselves need a GPU)."""
import numpy as np

from sph_playground_b200 import abi, ic, tune


def _fake_timer(calls):
    def t(state, store, kernel, precision, params, steps, warmup, lib):
        calls.append(dict(params))
        # a bowl with its minimum at lanes_search 16, lanes_pair 4, cell 0.33
        return (1.0 + abs(params["P_LANES_SEARCH"] - 16) + abs(params["P_LANES_PAIR"] - 4)
                + 10 * abs(params["P_CELL_FACTOR"] - 0.33))
    return t


def test_autotune_finds_the_minimum_and_caches(tmp_path):
    st, store = ic.sedov3d(n=8)
    calls = []
    cache = str(tmp_path / "tune.json")
    r = tune.autotune(st, store, "m6", abi.PREC_FP32_COMP, cache=cache, timer=_fake_timer(calls))
    assert (r["P_LANES_SEARCH"], r["P_LANES_PAIR"], r["P_CELL_FACTOR"]) == (16, 4, 0.33)
    assert r["ms_per_step"] == 1.0
    n = len(calls)
    assert n <= 1 + sum(len(v) for v in tune.SPACE.values())
    r2 = tune.autotune(st, store, "m6", abi.PREC_FP32_COMP, cache=cache, timer=_fake_timer(calls))
    assert r2 == r and len(calls) == n  # served from the cache


def test_cache_key_separates_workloads():
    st3, s3 = ic.sedov3d(n=8)
    st2, s2 = ic.diffusion2d(16)
    k = {tune.key(st3, "m6", 0, s3.shape[0]), tune.key(st3, "m6", 1, s3.shape[0]),
         tune.key(st3, "m4", 0, s3.shape[0]), tune.key(st2, "m6", 0, s2.shape[0]),
         tune.key(st3, "m6", 0, 8 * s3.shape[0])}
    assert len(k) == 5


def test_time_steps_runs_on_the_oracle(oracle_lib):
    st, store = ic.sedov3d(n=6)
    t = tune.time_steps(st, store, "m6", abi.PREC_FP64, {"P_CELL_FACTOR": 0.4}, steps=1,
                        warmup=1, lib=oracle_lib)
    assert np.isfinite(t) and t >= 0.0
