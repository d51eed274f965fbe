"""Autotuner for the engine's launch shapes.

The tunable shapes of the CUDA engine are the lanes per centre of the
neighbour search (SPH_P_LANES_SEARCH: the group of centres that shares one
candidate stream), the lanes per centre of the pair passes circuit1 /
circuit2 (SPH_P_LANES_PAIR) and the cell edge of the search grid in units of
krad * h_min (SPH_P_CELL_FACTOR).  The best values depend on the dimension,
the kernel, the precision and the particle count, so `autotune` times a few
leapfrog steps per candidate (device time from the engine's CUDA events),
descending one coordinate at a time from the defaults, and keeps the result
in a JSON cache keyed by (dim, kernel, precision, equations, log2 N).

    params = autotune(state, store, "m6", abi.PREC_FP32_COMP)
    e = abi.Engine(state, store, "m6", precision=abi.PREC_FP32_COMP)
    apply(e, params)
"""
import json
import math
import os

from . import abi, consts

SPACE = {
    "P_LANES_SEARCH": [4, 8, 16],
    "P_LANES_PAIR": [4, 8, 16],
    "P_CELL_FACTOR": [0.33, 0.4, 0.5],
}
DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "sph_playground_b200", "tune.json")


def key(state, kernel, precision, n_rows):
    """Cache key of a workload: dimension, kernel, precision, equations and
    the particle count rounded to a power of two."""
    dim = int(state[consts.ec["dim"] - 1])
    eqs = int(state[consts.ec["eqs"] - 1])
    return f"d{dim}-{kernel}-p{int(precision)}-e{eqs}-n{int(round(math.log2(max(n_rows, 1))))}"


def apply(engine, params):
    for name, v in params.items():
        engine.set_param(getattr(abi, name), float(v))


def time_steps(state, store, kernel, precision, params, steps=3, warmup=2, lib=None):
    """Device ms per step of `steps` leapfrog steps after `warmup` ones, each
    with a fresh neighbour search (no skin lists: the search's shapes are
    what is tuned, and skin-list iterates rarely search)."""
    e = abi.Engine(state, store, kernel, precision=precision, lib=lib)
    try:
        e.set_param(abi.P_SKIN, 0.0)
        apply(e, params)
        e.set_param("tfinish", 1e30)
        e.step(warmup)
        e.reset_counters()
        e.set_param(abi.P_TIMING, 2)
        e.step(steps)
        return e.timers()["step"] / steps
    finally:
        e.close()


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(path, data):
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only loses the cache


def autotune(state, store, kernel="m6", precision=abi.PREC_FP64, lib=None, cache=DEFAULT_CACHE,
             steps=3, warmup=2, space=None, timer=time_steps, refresh=False):
    """Best launch shapes for this workload (cached).  Returns a dict of
    abi.P_* names to values and, under "ms_per_step", the time it measured."""
    space = space or SPACE
    k = key(state, kernel, precision, store.shape[0])
    data = _load(cache) if cache else {}
    if not refresh and k in data:
        return data[k]
    best = {name: (8 if "LANES" in name else 0.4) for name in space}
    best = {name: (v if v in space[name] else space[name][len(space[name]) // 2])
            for name, v in best.items()}
    t_best = timer(state, store, kernel, precision, best, steps, warmup, lib)
    tried = {tuple(sorted(best.items())): t_best}
    for name, values in space.items():
        for v in values:
            cand = dict(best)
            cand[name] = v
            sig = tuple(sorted(cand.items()))
            if sig in tried:
                continue
            t = timer(state, store, kernel, precision, cand, steps, warmup, lib)
            tried[sig] = t
            if t < t_best:
                best, t_best = cand, t
    result = dict(best)
    result["ms_per_step"] = t_best
    if cache:
        data[k] = result
        _save(cache, data)
    return result
