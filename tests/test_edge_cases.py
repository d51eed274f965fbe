"""Edge cases of the search and density pass against the oracle: coincident
particles (distance 0 between distinct rows, decided by the FP64 predicate
in the guard-band pass), a box so small that a particle sees several images
of itself and of its neighbours, and a neighbour-list overflow (a particle
set clustered after the capacities were sized for the spread one) that the
engine must detect and redo with larger rows."""
import numpy as np
import pytest

from sph_playground_b200 import abi, ic
from tests.parity import COL, neighbour_sets_equal, rel_particle, run_pass

pytestmark = pytest.mark.gpu

FP64, FP32 = abi.PREC_FP64, abi.PREC_FP32_COMP
TOL = {FP64: 1e-12, FP32: 1e-6}


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_coincident_particles(oracle_lib, engine_lib, cuda_ok, prec):
    st, store = ic.density3d(n=10, seed=3)
    # rows 1, 2 and 3 placed exactly on row 0 (and row 50 on row 51)
    store[1:4, COL["rx"]:COL["rz"] + 1] = store[0, COL["rx"]:COL["rz"] + 1]
    store[50, COL["rx"]:COL["rz"] + 1] = store[51, COL["rx"]:COL["rz"] + 1]
    ref, nb_ref, _, _ = run_pass(oracle_lib, st, store, "m6", FP64, "density")
    got, nb_got, _, _ = run_pass(engine_lib, st, store, "m6", prec, "density")
    assert neighbour_sets_equal(nb_got, nb_ref)
    for f in ("den", "h", "om"):
        assert rel_particle(got[:, COL[f]], ref[:, COL[f]]) <= TOL[prec], f


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_tiny_periodic_box(oracle_lib, engine_lib, cuda_ok, prec):
    """4^3 particles with a support radius of 3.6 spacings: the strips are
    the whole box, so every particle meets images of itself."""
    st, store = ic.density3d(n=4, seed=5)
    ref, nb_ref, _, _ = run_pass(oracle_lib, st, store, "m6", FP64, "density")
    got, nb_got, _, _ = run_pass(engine_lib, st, store, "m6", prec, "density")
    assert neighbour_sets_equal(nb_got, nb_ref)
    for f in ("den", "h", "om"):
        assert rel_particle(got[:, COL[f]], ref[:, COL[f]]) <= TOL[prec], f


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_list_overflow_is_redone(oracle_lib, engine_lib, cuda_ok, prec):
    """The row capacities follow the previous search's counts; after the
    particles are squeezed into an eighth of the box (8x the neighbours at
    the same h) the rows overflow and the search must be redone."""
    st, store = ic.density3d(n=12, seed=4)
    squeezed = store.copy()
    squeezed[:, COL["rx"]:COL["rz"] + 1] *= 0.5
    ref, nb_ref, _, _ = run_pass(oracle_lib, st, squeezed, "m6", FP64, "density")
    with abi.Engine(st, store, "m6", precision=prec, lib=engine_lib) as e:
        e.density()
        before = e.get_neighbours()[0][-1]
        e.set_store(squeezed)
        e.reset_counters()
        e.density()
        got, nb_got, cnt = e.get_store(), e.get_neighbours(), e.counters()
    assert nb_got[0][-1] > 3 * before
    assert cnt["searches"] >= 2  # the overflowing search was redone
    assert neighbour_sets_equal(nb_got, nb_ref)
    for f in ("den", "h", "om"):
        assert rel_particle(got[:, COL[f]], ref[:, COL[f]]) <= TOL[prec], f


def test_fixedreal_copies_run_like_the_oracle(oracle_lib, engine_lib, cuda_ok, tmp_path):
    """The runner/006.1 set-up (borderless 1D colliding flows with periodic
    fixedreal copies of the border strips: integrated rows that are not
    centres) run to t = 0.02 on both engines, FP64."""
    from tests.test_driver import _runner_006_sequence
    c = _runner_006_sequence(tmp_path)
    out = []
    for lib in (oracle_lib, engine_lib):
        with abi.Engine(c.state, c.store, "m6", lib=lib) as e:
            e.run_to(0.02)
            out.append((e.get_store(), e.get_state()))
    (s0, t0), (s1, t1) = out
    assert t0[45] == t1[45]  # same time reached
    for f in ("den", "u", "h"):
        assert rel_particle(s1[:, COL[f]], s0[:, COL[f]]) <= 1e-9, f
    np.testing.assert_allclose(s1[:, 0], s0[:, 0], rtol=0, atol=1e-11)


@pytest.mark.parametrize("h_small", [1e-4, 1e-12])
@pytest.mark.parametrize("prec", [FP64, FP32])
def test_tiny_smoothing_length_grid(oracle_lib, engine_lib, cuda_ok, prec, h_small):
    """One particle with a tiny h in the unit box sets a cell edge that would
    need up to ~1e9 cells per axis: the cell count is checked one axis at a
    time (their product would overflow 64 bits) and the grid is widened to
    fit, with the neighbour sets and densities of the oracle."""
    rng = np.random.default_rng(32)
    n = 3000
    st = ic.make_state(3, equations="hydro", adden="no", process="borderless", hfac=1.2)
    for k, v in (("realpn", n), ("fixedpn", 0), ("gamma", 5.0 / 3.0), ("dcondconst", 1.0),
                 ("time", 0.0), ("dtprint", 1.0)):
        ic.set_state(st, k, v)
    store = np.zeros((n, 32))
    store[:, 0:3] = rng.uniform(0.0, 1.0, (n, 3))
    h = 1.2 * (1.0 / n) ** (1 / 3) * rng.uniform(0.9, 1.1, n)
    h[7] = h_small
    store[:, COL["h"]] = h
    store[:, COL["m"]] = 1.0 / n
    store[:, COL["den"]] = 1.0
    store[:, COL["om"]] = 1.0
    store[:, COL["u"]] = 1.0
    store[:, COL["type"]] = 1.0
    ref, nb_ref, _, _ = run_pass(oracle_lib, st, store, "m6", FP64, "density")
    got, nb_got, _, _ = run_pass(engine_lib, st, store, "m6", prec, "density")
    assert neighbour_sets_equal(nb_got, nb_ref)
    assert rel_particle(got[:, COL["den"]], ref[:, COL["den"]]) <= TOL[prec]


@pytest.mark.parametrize("case", ["coincident", "tiny_box", "overflow"])
def test_staged_search_edge_cases(oracle_lib, engine_lib, cuda_ok, case):
    """The edge cases above with the bulk-copy staged search."""
    if case == "coincident":
        st, store = ic.density3d(n=10, seed=3)
        store[1:4, COL["rx"]:COL["rz"] + 1] = store[0, COL["rx"]:COL["rz"] + 1]
    elif case == "tiny_box":
        st, store = ic.density3d(n=4, seed=5)
    else:
        st, store = ic.density3d(n=12, seed=4)
        store[:, COL["rx"]:COL["rz"] + 1] *= 0.5
    ref, nb_ref, _, _ = run_pass(oracle_lib, st, store, "m6", FP64, "density")
    got, nb_got, _, _ = run_pass(engine_lib, st, store, "m6", FP64, "density",
                                 params={abi.P_SEARCH_STAGED: 1})
    assert neighbour_sets_equal(nb_got, nb_ref)
    assert rel_particle(got[:, COL["den"]], ref[:, COL["den"]]) <= TOL[FP64]
