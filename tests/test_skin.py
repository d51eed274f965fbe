"""Skin lists (SPH_P_SKIN): neighbour lists kept between iterates with a
radius of (1 + s) krad h; every iterate each centre keeps its row (nothing
near it moved), refilters its skin list with the FP64 predicate, or (near
a fast particle) is searched afresh.  The sets must be those of a fresh
search on the same state, step after step, through iterates served from
the lists and through rebuilds.

The check runs each step in parts (timestep, predict, density, forces,
correct): after the predictor the table goes to a fresh oracle handle,
whose density pass searches the same positions and h; its neighbour-set
digests must equal the engine's.  The fields of whole runs must match the
runs without skin lists to the summation-order level (FP64) or within the
FP32 path's tolerances of the FP64 oracle."""
import numpy as np
import pytest

from sph_playground_b200 import abi, consts, ic
from parity import COL, rel_field, rel_particle

FP64, FP32 = abi.PREC_FP64, abi.PREC_FP32_COMP


def _split_run(engine_lib, oracle_lib, st, store, prec, nsteps, skin=0.1, kernel="m6",
               params=None, between=None):
    """nsteps leapfrog steps in parts; after every predictor the engine's
    neighbour sets are compared with a fresh oracle search on the same
    table.  Returns the engine's counters and final store."""
    e = abi.Engine(st, store, kernel, precision=prec, lib=engine_lib)
    try:
        e.set_param(abi.P_SKIN, skin)
        for k, v in (params or {}).items():
            e.set_param(k, v)
        e.density()
        e.forces()
        for step in range(nsteps):
            if between is not None:
                between(e, step)
            dt = e.timestep()
            e.predict(dt)
            mid, mst = e.get_store(), e.get_state()
            e.density()
            got = e.get_neighbour_digest()
            with abi.Engine(mst, mid, kernel, precision=FP64, lib=oracle_lib) as o:
                o.density()
                ref = o.get_neighbour_digest()
            assert np.array_equal(got[0], ref[0]), f"step {step}: neighbour counts differ"
            assert np.array_equal(got[1], ref[1]), f"step {step}: neighbour sets differ"
            e.forces()
            e.correct(dt)
        return e.counters(), e.get_store()
    finally:
        e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [FP64, FP32])
def test_skin_sedov_sets_match_oracle(engine_lib, oracle_lib, cuda_ok, prec):
    """Sedov blast: the blast particles move (fast records, dirty centres
    searched afresh with a widened cell range), the rest are at rest (at
    48^3 the blast is a small part of the box, as in the 128^3 workload)."""
    st, store = ic.sedov3d(n=48)
    cnt, _ = _split_run(engine_lib, oracle_lib, st, store, prec, nsteps=24)
    info = {k: cnt[k] for k in ("skin_builds", "skin_reuses", "skin_dirty", "skin_kept",
                                "searches")}
    assert cnt["skin_builds"] >= 1, info
    assert cnt["skin_reuses"] >= 6, info
    assert cnt["skin_dirty"] > 0, info  # some centres were searched afresh,
    assert cnt["skin_kept"] > 0, info  # some rows kept,
    n = st[abi.consts.ec["realpn"] - 1]  # and some filtered
    assert cnt["skin_kept"] + cnt["skin_dirty"] < cnt["skin_reuses"] * n, info


@pytest.mark.gpu
def test_skin_sedov_rebuilds(engine_lib, oracle_lib, cuda_ok):
    """A thin skin (s = 0.02) runs out within a few steps: lists rebuilt
    mid-run, sets still the fresh search's."""
    st, store = ic.sedov3d(n=16)
    cnt, _ = _split_run(engine_lib, oracle_lib, st, store, FP64, nsteps=16, skin=0.02)
    info = {k: cnt[k] for k in ("skin_builds", "skin_reuses", "skin_dirty")}
    assert cnt["skin_builds"] >= 2, info
    assert cnt["skin_reuses"] >= 1, info


@pytest.mark.gpu
def test_skin_shear_flow_across_boundaries(engine_lib, oracle_lib, cuda_ok):
    """2D shear flow in a periodic box: particles cross the image strips and
    the box faces (image sets change, rows wrap)."""
    st, store = ic.shear2d(n=24, amp=0.3)
    cnt, _ = _split_run(engine_lib, oracle_lib, st, store, FP64, nsteps=12)
    assert cnt["skin_builds"] >= 1


@pytest.mark.gpu
def test_skin_sod_tube(engine_lib, oracle_lib, cuda_ok):
    """Sod tube (y periodic, hfac 1: lattice pairs at exactly the radius)."""
    st, store = ic.sod2d()
    cnt, _ = _split_run(engine_lib, oracle_lib, st, store, FP64, nsteps=8)
    assert cnt["skin_reuses"] + cnt["skin_builds"] >= 8


@pytest.mark.gpu
def test_skin_moved_by_the_caller(engine_lib, oracle_lib, cuda_ok):
    """Positions and h written by the caller between steps (sph_set_columns)
    are measured like the integrator's moves."""
    st, store = ic.sedov3d(n=12)
    dx = 1.0 / 12
    rng = np.random.default_rng(3)

    def nudge(e, step):
        if step % 3 == 1:
            x = e.get_columns(["rx", "ry", "rz", "h"])
            x[:3] += rng.uniform(-0.05 * dx, 0.05 * dx, size=x[:3].shape)
            x[3] *= 1.0 + rng.uniform(0.0, 0.02, size=x[3].shape)
            e.set_columns(["rx", "ry", "rz", "h"], x)

    cnt, _ = _split_run(engine_lib, oracle_lib, st, store, FP64, nsteps=9, between=nudge)
    assert cnt["skin_reuses"] >= 1, {k: cnt[k] for k in ("skin_builds", "skin_reuses")}


@pytest.mark.gpu
def test_skin_fields_match_fresh_search(engine_lib, oracle_lib, cuda_ok):
    """Whole runs through sph_step: FP64 with skin lists equals FP64 without
    them up to summation order; FP32-comp with skin lists stays within the
    FP32 tolerances of the FP64 oracle."""
    st, store = ic.sedov3d(n=48, npics=1)  # (no output-time clipping: see test_domain)
    out = {}
    for name, lib, prec, skin in (("ref", oracle_lib, FP64, 0.0), ("fresh", engine_lib, FP64, 0.0),
                                  ("skin64", engine_lib, FP64, 0.1),
                                  ("skin32", engine_lib, FP32, 0.1)):
        with abi.Engine(st, store, "m6", precision=prec, lib=lib) as e:
            e.set_param(abi.P_SKIN, skin)
            e.step(15)
            out[name] = (e.get_store(), e.get_state(), e.counters())
    assert out["skin64"][2]["skin_reuses"] >= 8, out["skin64"][2]
    s_f, s_s = out["fresh"][0], out["skin64"][0]
    t_f, t_s = (out[k][1][consts.ec["time"] - 1] for k in ("fresh", "skin64"))
    assert abs(t_s - t_f) <= 1e-12 * t_f  # (dt from fields summed in another order)
    for f in ("den", "h", "om"):
        assert rel_particle(s_s[:, COL[f]], s_f[:, COL[f]]) < 1e-12, f
    for f in ("rx", "ry", "rz", "vx", "vy", "vz", "u"):
        assert rel_field(s_s[:, COL[f]], s_f[:, COL[f]]) < 1e-12, f
    ref, s32 = out["ref"][0], out["skin32"][0]
    assert rel_particle(s32[:, COL["den"]], ref[:, COL["den"]]) < 1e-6
    for f in ("vx", "vy", "vz", "u"):
        assert rel_field(s32[:, COL[f]], ref[:, COL[f]]) < 1e-5, f


@pytest.mark.gpu
def test_skin_parameter_change_rebuilds(engine_lib, oracle_lib, cuda_ok):
    """Density passes over a table that does not move are served from the
    lists; a parameter that can change the sets (the cell factor) ends them,
    one that cannot (the timing switch) keeps them."""
    st, store = ic.density3d(n=16, seed=2)
    with abi.Engine(st, store, "m6", precision=FP64, lib=engine_lib) as e:
        e.set_param(abi.P_SKIN, 0.1)
        for _ in range(5):  # (lists that serve fewer iterates start a pause of plain searches)
            e.density()
        c = e.counters()
        assert (c["skin_builds"], c["skin_reuses"]) == (1, 4)
        e.set_param(abi.P_TIMING, 1)
        e.density()
        assert e.counters()["skin_builds"] == 1
        e.set_param(abi.P_CELL_FACTOR, 0.45)
        mid, mst = e.get_store(), e.get_state()  # (each pass moves h)
        e.density()
        assert e.counters()["skin_builds"] == 2
        got = e.get_neighbour_digest()
    with abi.Engine(mst, mid, "m6", precision=FP64, lib=oracle_lib) as o:
        o.density()
        ref = o.get_neighbour_digest()
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


@pytest.mark.gpu
def test_skin_lists_survive_a_table_upload(engine_lib, oracle_lib, cuda_ok):
    """sph_set_store puts the rows back in caller order: the lists are
    renamed and serve the next pass, whose sets equal a fresh search's on the
    uploaded table (moved positions and h measured like any move); a changed
    particle type ends them."""
    st, store = ic.density3d(n=16, seed=2)
    dx = 1.0 / 16
    rng = np.random.default_rng(5)
    with abi.Engine(st, store, "m6", precision=FP64, lib=engine_lib) as e:
        e.set_param(abi.P_SKIN, 0.1)
        for _ in range(5):
            e.density()
        b0 = e.counters()["skin_builds"]
        table = e.get_store()
        table[:, 0:3] += rng.uniform(-0.02 * dx, 0.02 * dx, size=(table.shape[0], 3))
        table[:, COL["h"]] *= 1.0 + rng.uniform(0.0, 0.01, size=table.shape[0])
        e.set_store(table)
        mst = e.get_state()
        e.density()
        assert e.counters()["skin_builds"] == b0  # served from the renamed lists
        got = e.get_neighbour_digest()
        with abi.Engine(mst, table, "m6", precision=FP64, lib=oracle_lib) as o:
            o.density()
            ref = o.get_neighbour_digest()
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
        table = e.get_store()
        table[3, COL["type"]] = consts.ept["fixed"]
        e.set_store(table)
        e.density()
        assert e.counters()["skin_builds"] == b0 + 1  # a changed type ends them


# ---- skin lists of the device-resident step (the batch's device loop, SPH_P_GRAPH) ----

def _device_runs(lib, sets, prec, skin, run):
    eng = [abi.Engine(st, store, "m6", precision=prec, lib=lib) for st, store in sets]
    try:
        for e in eng:
            e.set_param(abi.P_SKIN, skin)
        run(eng)
        return [(e.get_store(), e.get_state(), e.counters(), e.get_neighbour_digest())
                for e in eng]
    finally:
        for e in eng:
            e.close()


def _ways(c):
    return {k: c[k] for k in ("steps", "iterates", "searches", "skin_builds", "skin_reuses",
                              "graph_steps", "graph_redos")}


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [FP64, FP32])
def test_device_loop_skin_lists(engine_lib, oracle_lib, cuda_ok, prec):
    """The batch's device loop at the default skin: the lattices at rest are
    served from the lists nearly every iterate (a search after each row
    reorder), the sets after the run equal a fresh oracle search on the
    final table (FP64), and the fields equal the loop's without lists to the
    summation order (FP64) or within the FP32 tolerances."""
    tf = 2e-3
    sets = [ic.diffusion2d(n, ddw=ddw, tfinish=tf, sts_stages=4)
            for n, ddw in ((12, "fab"), (16, "n2w"), (20, "2nw_ds"))]

    def batch(eng):
        with abi.Batch(eng) as b:
            b.run_to(tf)
            assert b.status() == [0] * len(eng)

    fresh = _device_runs(engine_lib, sets, prec, 0.0, batch)
    skin = _device_runs(engine_lib, sets, prec, 0.1, batch)
    for (s0, t0, c0, _), (s1, t1, c1, dg) in zip(fresh, skin):
        info = _ways(c1)
        assert c1["graph_steps"] > 0 and c1["skin_builds"] >= 1, info
        assert 2 * c1["skin_reuses"] >= c1["iterates"], info
        assert c1["searches"] + c1["skin_reuses"] == c1["iterates"], info
        assert c0["steps"] == c1["steps"]
        tol = (1e-12, 1e-12) if prec == FP64 else (1e-6, 1e-5)
        assert abs(t1[consts.ec["time"] - 1] - t0[consts.ec["time"] - 1]) <= 1e-12
        for f in ("den", "h"):
            assert rel_particle(s1[:, COL[f]], s0[:, COL[f]]) < tol[0], f
        assert rel_field(s1[:, COL["t"]], s0[:, COL["t"]]) < tol[1]
        if prec == FP64:
            with abi.Engine(t1, s1, "m6", precision=FP64, lib=oracle_lib) as o:
                o.density()
                ref = o.get_neighbour_digest()
            assert np.array_equal(dg[0], ref[0]) and np.array_equal(dg[1], ref[1])


@pytest.mark.gpu
def test_graph_steps_skin_lists_hydro(engine_lib, cuda_ok):
    """Device-resident steps (SPH_P_GRAPH) of the Sedov blast with skin
    lists: served while the records move little, searched afresh (plainly in
    a pause after short-lived lists) once the blast moves them; the fields
    equal the steps without lists to the summation order."""
    st, store = ic.sedov3d(n=24, npics=1)

    def steps(eng):
        for e in eng:
            e.set_param(abi.P_GRAPH, 1.0)
            e.step(12)

    (s0, t0, c0, _), = _device_runs(engine_lib, [(st, store)], FP64, 0.0, steps)
    (s1, t1, c1, _), = _device_runs(engine_lib, [(st, store)], FP64, 0.1, steps)
    info = _ways(c1)
    assert c1["graph_steps"] >= 10 and c1["skin_builds"] >= 1, info
    assert c1["searches"] + c1["skin_reuses"] == c1["iterates"], info
    assert abs(t1[consts.ec["time"] - 1] - t0[consts.ec["time"] - 1]) <= 1e-12 * t0[consts.ec["time"] - 1]
    for f in ("den", "h", "om"):
        assert rel_particle(s1[:, COL[f]], s0[:, COL[f]]) < 1e-12, f
    for f in ("rx", "ry", "rz", "vx", "vy", "vz", "u"):
        assert rel_field(s1[:, COL[f]], s0[:, COL[f]]) < 1e-12, f


@pytest.mark.gpu
def test_skin_lists_end_on_a_long_move(engine_lib, oracle_lib, cuda_ok):
    """A record moved by the caller farther than a search radius ends the
    lists (the device-side checks of the iterate); the next pass searches
    afresh and its sets equal the oracle's."""
    st, store = ic.density3d(n=16, seed=2)
    with abi.Engine(st, store, "m6", precision=FP64, lib=engine_lib) as e:
        e.set_param(abi.P_SKIN, 0.1)
        for _ in range(5):
            e.density()
        b0 = e.counters()["skin_builds"]
        x = e.get_columns(["rx"])
        x[0, 7] = (x[0, 7] + 0.31) % 1.0  # (the unit box: about five spacings)
        e.set_columns(["rx"], x)
        mst = e.get_state()
        table = e.get_store()
        e.density()
        assert e.counters()["skin_builds"] == b0 + 1
        got = e.get_neighbour_digest()
    with abi.Engine(mst, table, "m6", precision=FP64, lib=oracle_lib) as o:
        o.density()
        ref = o.get_neighbour_digest()
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
