"""The engine's own initial conditions (IC/place.f90, IC/IC.f90 setupV2,
BC.f90 createFixedBorders) restated in sph_playground_b200/icsetup.py, and
the runner workflow they feed (CleanRun -> ContinueRun -> result.info) on
the oracle (CPU) and on the CUDA engine against it (GPU)."""
import os

import numpy as np
import pytest
from scipy.spatial import cKDTree

from sph_playground_b200 import abi, consts, core, ic, icsetup

COL = {k: v - 1 for k, v in consts.es.items()}


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_uniform_place_matches_place_uniform(dim):
    s1 = ic.make_state(dim, resolution=12)
    s2 = s1.copy()
    a, b = ic.place_uniform(s1, "m6"), icsetup.place(s2, "m6")
    assert np.array_equal(a, b) and np.array_equal(s1, s2)


def test_closepacked_rows_are_dx_apart():
    st = ic.make_state(2, resolution=16, placement="closepacked")
    s = icsetup.place(st, "m6")
    d, _ = cKDTree(s[:, :3]).query(s[:, :3], k=2)
    np.testing.assert_allclose(d[:, 1], 1.0 / 16, rtol=1e-12)
    assert int(ic.get_state(st, "realpn")) == s.shape[0]


def test_random_place_stays_in_box_and_is_seeded():
    a = icsetup.place(ic.make_state(2, resolution=16, placement="random"), "m6", seed=3)
    b = icsetup.place(ic.make_state(2, resolution=16, placement="random"), "m6", seed=3)
    assert np.array_equal(a, b)
    assert a[:, 0].min() >= 0 and a[:, 0].max() <= 1 and a[:, 1].min() >= 0 and a[:, 1].max() <= 1


def test_fixed_borders_are_mirror_images():
    """Every fixed row of the hydroshock set-up (walls at x = -0.5, 0.5) is
    the mirror of a real row within bordersize of that wall, and every such
    real row has exactly one image."""
    st = ic.make_state(2, ics="hydroshock", resolution=64, hfac=1.2)
    s = icsetup.setup_v2(st, "m6")
    rpn, fpn = int(ic.get_state(st, "realpn")), int(ic.get_state(st, "fixedpn"))
    assert s.shape[0] == rpn + fpn and fpn > 0
    real, fixed = s[:rpn], s[rpn:]
    assert np.all(real[:, COL["type"]] == consts.ept["real"])
    assert np.all(fixed[:, COL["type"]] == consts.ept["fixed"])
    bs = ic.get_state(st, "bordsize")
    x = real[:, 0]
    left, right = x < -0.5 + bs, x > 0.5 - bs
    want = np.concatenate([np.c_[-1.0 - x[left], real[left, 1]],
                           np.c_[1.0 - x[right], real[right, 1]]])
    np.testing.assert_array_equal(fixed[:, :2], want)
    # fields follow the side of the image: x <= 0 is the dense state
    dense = fixed[:, 0] <= 0
    assert np.all(fixed[dense, COL["den"]] == 1.0) and np.all(fixed[~dense, COL["den"]] == 0.125)


def test_corner_images_in_every_strip():
    """createFixedBorders(all) in 2D: an x image lying in a y strip is
    mirrored again across y (the corners)."""
    st = ic.make_state(2, ics="fld_gauss", resolution=64, hfac=1.2)
    s = icsetup.setup_v2(st, "m6")
    rpn = int(ic.get_state(st, "realpn"))
    fixed = s[rpn:, :2]
    real = s[:rpn, :2]
    corner = (np.abs(fixed[:, 0]) > 10.0) & (np.abs(fixed[:, 1]) > 1.0)
    assert corner.any()
    # a corner image mirrors a real row across both walls
    src = np.c_[np.sign(fixed[corner, 0]) * 20.0 - fixed[corner, 0],
                np.sign(fixed[corner, 1]) * 2.0 - fixed[corner, 1]]
    tree = cKDTree(real)
    d, _ = tree.query(src)
    assert d.max() < 1e-12


@pytest.mark.parametrize("ics", ["shock12", "pulse", "ring", "soundwave", "hydroshock",
                                 "alfvenwave", "otvortex", "boilingtank", "fld_gauss"])
def test_setup_fields_are_valid(ics):
    """Every set-up passes the engine's pre-run checks (positive density,
    sound speed, h, pressure where the problem has one, energy)."""
    dim = 2
    st = ic.make_state(dim, ics=ics, resolution=64 if ics == "fld_gauss" else 32)
    s = icsetup.setup_v2(st, "m6", seed=1)
    assert s.shape[0] == int(ic.get_state(st, "realpn") + ic.get_state(st, "fixedpn"))
    for f in ("den", "c", "h", "u", "m"):
        assert np.all(s[:, COL[f]] > 0), f
    assert ic.get_state(st, "gamma") > 1


def test_setup_errors_like_the_reference():
    with pytest.raises(ValueError):
        icsetup.setup_v2(ic.make_state(2, ics="sin3", resolution=32), "m6")
    with pytest.raises(ValueError):  # IC.f90:575-577: 2 nb >= resolution
        icsetup.setup_v2(ic.make_state(2, ics="shock12", resolution=6), "m6")


def _hydroshock_context(tmp_path, res=64):
    c = core.Context(pwd=str(tmp_path))
    s = c.setup
    s.kernel, s.dim, s.equations, s.hfac, s.tfinish = "m6", 2, "hydro", 1.2, 0.0
    s.resolution, s.nsnapshots, s.ics, s.process = res, 1, "hydroshock", "borderless"
    s.adden, s.artts, s.au = "yes", "yes", 1.0
    c.CleanRun()
    c.ReadDumpHDF(os.path.join(str(tmp_path), "output", "dump_full.h5"))
    c.setup.tfinish, c.setup.dtprint, c.setup.time = 0.05, 0.05, 0.0
    c.Apply()
    return c


def test_runner_workflow_hydroshock_on_oracle(oracle_lib, tmp_path):
    """006.1_hydro_shock.py's sequence: CleanRun with ics = hydroshock (walls
    of fixed particles), ContinueRun to t = 0.05, result.info written."""
    c = _hydroshock_context(tmp_path)
    c.ContinueRun(lib=oracle_lib)
    assert abs(c.GetState("time") - 0.05) < 1e-12
    line = open(os.path.join(str(tmp_path), "result.info")).read().split()
    assert len(line) == 5 and 0.0 < float(line[2]) < 0.2


@pytest.mark.gpu
def test_gpu_hydroshock_with_fixed_walls_matches_oracle(engine_lib, oracle_lib, cuda_ok, tmp_path):
    """The same fixed-wall run on the CUDA engine (FP64) and the oracle."""
    c = _hydroshock_context(tmp_path)
    st, store = c.state.copy(), c.store.copy()
    out = []
    for lib in (oracle_lib, engine_lib):
        with abi.Engine(st, store, "m6", lib=lib) as e:
            e.run_to(0.05)
            out.append((e.get_store(), e.get_state(), e.errcalc()[1]))
    (s0, t0, l0), (s1, t1, l1) = out
    assert t0[consts.ec["time"] - 1] == t1[consts.ec["time"] - 1]
    np.testing.assert_allclose(s1[:, COL["den"]], s0[:, COL["den"]], rtol=1e-9)
    np.testing.assert_allclose(s1[:, :3], s0[:, :3], rtol=0, atol=1e-11)
    assert l1 == pytest.approx(l0, rel=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("ics", ["mti", "mtilowres"])
def test_gpu_mti_setup_density_pass_matches_oracle(engine_lib, oracle_lib, cuda_ok, ics):
    """The set-up's closing density pass on the CUDA engine (FP64) and on the
    oracle: the same lattice, the same den / h / om."""
    out = []
    for lib in (oracle_lib, engine_lib):
        st = ic.make_state(2, ics=ics, resolution=32, process="backcompatibility")
        out.append(icsetup.setup_v2(st, "m6", lib=lib))
    s0, s1 = out
    np.testing.assert_array_equal(s1[:, :3], s0[:, :3])
    for f in ("den", "h", "om"):
        np.testing.assert_allclose(s1[:, COL[f]], s0[:, COL[f]], rtol=1e-9, err_msg=f)


def test_mti_setups_on_the_oracle(oracle_lib):
    """mti: the stretch map gives the lattice the Hopkins (2017) profile
    rho ~ (3 - y)^4 (the density the closing pass finds follows its slope);
    mtilowres: no walls, so the closing pass (periodic along x only) finds
    the density falling off at the y edges.  Both end with the real / fixed
    row counts of the lattice."""
    st = ic.make_state(2, ics="mti", resolution=32, process="backcompatibility")
    s = icsetup.setup_v2(st, "m6", lib=oracle_lib)
    rpn, fpn = int(ic.get_state(st, "realpn")), int(ic.get_state(st, "fixedpn"))
    assert fpn > 0 and s.shape[0] == rpn + fpn
    r = s[:rpn]
    y, d = r[:, 1], r[:, COL["den"]]
    mid = (y > 0.02) & (y < 0.08)
    prof = (3 - y[mid]) ** 4
    slope = np.polyfit(y[mid], d[mid], 1)[0]
    want = np.polyfit(y[mid], prof / prof.mean() * d[mid].mean(), 1)[0]
    assert slope == pytest.approx(want, rel=0.05)
    assert np.all(r[:, COL["bx"]] == 1e-11) and np.any(r[:, COL["vy"]] != 0)
    st2 = ic.make_state(2, ics="mtilowres", resolution=32, process="backcompatibility")
    s2 = icsetup.setup_v2(st2, "m6", lib=oracle_lib)
    assert int(ic.get_state(st2, "fixedpn")) == 0
    y2, d2 = s2[:, 1], s2[:, COL["den"]]
    assert d2[np.abs(y2) > 1.9].mean() < 0.9 * d2[np.abs(y2) < 1.0].mean()


def test_context_cleanrun_mti_on_oracle(oracle_lib, tmp_path):
    """Context.CleanRun with ics = mti writes the set-up, density pass
    included, to output/dump_full.h5, which reads back unchanged."""
    c = core.Context(pwd=str(tmp_path))
    s = c.setup
    s.kernel, s.dim, s.equations, s.hfac, s.tfinish = "m6", 2, "hydro", 1.2, 0.0
    s.resolution, s.nsnapshots, s.ics, s.process = 32, 1, "mti", "backcompatibility"
    c.CleanRun(lib=oracle_lib)
    direct = icsetup.setup_v2(c.state.copy(), "m6", lib=oracle_lib)
    c.ReadDumpHDF(os.path.join(str(tmp_path), "output", "dump_full.h5"))
    assert c.store.shape == direct.shape
    assert int(c.GetState("fixedpn")) > 0
    np.testing.assert_array_equal(c.store[:, COL["den"]], direct[:, COL["den"]])


def test_stretch_map_inverts_the_mass_function():
    """A particle at c lands where the profile's mass from cmin equals
    rho0 (c - cmin), the mass being the reference's trapezoid on 1024 steps
    with the first left end taken as 0: M(x) = x + x^3 - rho(0) x / 2048
    up to the O(dx^2) trapezoid error."""
    store = np.zeros((50, consts.ES_TOTAL))
    store[:, 1] = np.linspace(0.01, 0.99, 50)
    rho = lambda y: 1.0 + 3.0 * y * y  # noqa: E731
    icsetup.stretch_map(store, 0.0, 1.0, rho, axis=1)
    y = store[:, 1]
    m = lambda x: x + x ** 3 - x / 2048.0  # noqa: E731
    np.testing.assert_allclose(m(y), m(1.0) * np.linspace(0.01, 0.99, 50), rtol=2e-6)

