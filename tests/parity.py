"""Helpers that run the oracle and the engine on the same input and compare."""
import numpy as np

from sph_playground_b200 import abi, consts, ic

COL = {k: v - 1 for k, v in consts.es.items()}


def run_pass(lib, state, store, kernel="m6", prec=abi.PREC_FP64, what="iterate",
             params=None, steps=0):
    e = abi.Engine(state, store, kernel, precision=prec, lib=lib)
    try:
        for k, v in (params or {}).items():
            e.set_param(k, v)
        if what == "iterate":
            e.iterate()
        elif what == "density":
            e.density()
        elif what == "steps":
            e.step(steps)
        out = e.get_store()
        nb = e.get_neighbours() if what in ("iterate", "density") else None
        cnt = e.counters()
        st = e.get_state()
    finally:
        e.close()
    return out, nb, cnt, st


def rel_particle(a, b):
    """max_i |a_i - b_i| / |b_i| (fields that never vanish: rho, h, Omega)."""
    return float(np.max(np.abs(a - b) / np.abs(b)))


def rel_field(a, b):
    """max_i |a_i - b_i| / max_i |b_i| (signed fields: a, du, dh, dT, dB)."""
    scale = float(np.max(np.abs(b)))
    if scale == 0.0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b))) / scale


def neighbour_sets_equal(nb_a, nb_b):
    oa, pa = nb_a
    ob, pb = nb_b
    return np.array_equal(oa, ob) and np.array_equal(pa, pb)
