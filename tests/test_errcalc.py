"""The closing error evaluation (main.f90:374-402, errcalc.f90): err per
real particle for the run's initial-condition type and L1 = sum err / realpn.

CPU: the oracle against a numpy restatement of each calculator, its exact
Sod density against the published star states of Toro's test 1, and the
driver's result.info line.  GPU: the CUDA calculators against the oracle on
the same states, and after a run whose rows were reordered on the device."""
import math
import os

import numpy as np
import pytest
from scipy.special import erf

from sph_playground_b200 import abi, consts, core, ic
from tests.test_oracle import sod_exact

COL = {k: v - 1 for k, v in consts.es.items()}
KINDS = ["shock12", "shock12_aniso", "ring", "pulse", "pulse_aniso", "sin3", "soundwave",
         "hydroshock", "alfvenwave", "mti", "none"]


def _case(kind, t=0.2, seed=7):
    """A Sod-geometry particle set (x in [-1, 1]) with random fields, the
    state's initial-condition type set to `kind`, time t."""
    st, store = ic.sod2d(tfinish=0.2)
    rng = np.random.default_rng(seed)
    n = store.shape[0]
    store[:, COL["t"]] = rng.uniform(0.5, 2.5, n)
    store[:, COL["den"]] = rng.uniform(0.1, 1.2, n)
    store[:, COL["bx"]] = np.where(rng.uniform(size=n) < 0.5, 1.0, 0.3)
    store[:, COL["by"]] = rng.normal(size=n)
    store[:, COL["rz"]] = rng.uniform(-0.05, 0.05, n)
    base = kind.replace("_aniso", "")
    ic.set_state(st, "ics", consts.ICS[base])
    ic.set_state(st, "disotropic", 0.0 if kind.endswith("_aniso") else 1.0)
    ic.set_state(st, "dcondconst", 0.7)
    ic.set_state(st, "time", t)
    return st, store


def _expected(kind, st, store):
    """numpy restatement of the calculators (errcalc.f90)."""
    n = int(ic.get_state(st, "realpn"))
    s = store[:n]
    x, y, z = s[:, 0], s[:, 1], s[:, 2]
    t = ic.get_state(st, "time")
    dim = int(ic.get_state(st, "dim"))
    diso = int(ic.get_state(st, "disotropic"))
    base = kind.replace("_aniso", "")
    if base == "shock12":
        tt = np.where((diso == 1) | (s[:, COL["bx"]] == 1.0), t, 1e-15)
        exact = 1.5 + 0.5 * erf(x / np.sqrt(4 * tt))
        return np.abs(exact - s[:, COL["t"]])
    if base == "ring":
        rho, phi = np.sqrt(x * x + y * y), np.arctan2(y, x)
        exact = np.exp(-0.5 * ((rho - 0.3) ** 2 / 0.05 ** 2 + phi ** 2 / (0.25 + 2 * t / rho / rho)))
        return np.abs(exact - s[:, COL["t"]])
    if base == "pulse":
        eps, d = 0.1, ic.get_state(st, "dcondconst")
        ekt = eps ** 2 + 2 * d * t
        pifac = (2 * math.pi) ** (-dim / 2)
        if diso == 1:
            exact = pifac / ekt ** (dim / 2) * np.exp(-0.5 * (x * x + y * y + z * z) / ekt)
        else:
            exact = pifac / eps ** (dim - 1) / math.sqrt(ekt) * np.exp(
                -0.5 * (x * x / ekt + (y * y + z * z) / eps ** 2))
        return np.abs(exact - s[:, COL["t"]])
    if base == "soundwave":
        return np.abs(1 + 0.005 * np.sin(math.pi * (x - t)) - s[:, COL["den"]])
    if base == "hydroshock":
        return np.abs(s[:, COL["den"]] - sod_exact(x, t, gamma=1.4))
    if base == "alfvenwave":
        x1 = (x + 2 * y + 2 * z) / 3
        b2 = (s[:, COL["by"]] - 2 * s[:, COL["bx"]]) / math.sqrt(5)
        return np.abs(0.1 * np.sin(2 * math.pi * (x1 - t)) - b2)
    return np.zeros(n)  # sin3 (filled only when the type is 1), mti, none


@pytest.mark.parametrize("kind", KINDS)
def test_oracle_errcalc_against_restatement(oracle_lib, kind):
    st, store = _case(kind)
    with abi.Engine(st, store, "m6", lib=oracle_lib) as e:
        err, l1 = e.errcalc()
    want = _expected(kind, st, store)
    np.testing.assert_allclose(err, want, rtol=1e-12, atol=1e-14)
    assert l1 == pytest.approx(want.sum() / want.shape[0], rel=1e-12, abs=1e-15)


def test_oracle_sod_star_states_kat(oracle_lib):
    """Toro, Riemann Solvers, table 4.3, test 1 (gamma 1.4, (1, 0, 1) |
    (0.125, 0, 0.1)): rho*_L = 0.42632, rho*_R = 0.26557 (5 digits); at
    t = 0.2 the points x = 0.1 and 0.3 lie in the two star regions, -0.5
    and 0.4 in the undisturbed states.  With den = 0, err is the exact
    density itself."""
    st, store = _case("hydroshock")
    n = store.shape[0]
    xs = np.array([-0.5, 0.1, 0.3, 0.4])
    store[:, COL["den"]] = 0.0
    store[:4, COL["rx"]] = xs
    with abi.Engine(st, store, "m6", lib=oracle_lib) as e:
        err, _ = e.errcalc()
    np.testing.assert_allclose(err[:4], [1.0, 0.42632, 0.26557, 0.125], rtol=2e-5)
    assert n > 4


def test_oracle_errcalc_unsupported_types(oracle_lib):
    st, store = _case("none")
    ic.set_state(st, "ics", consts.ett["fld_gauss"])
    with abi.Engine(st, store, "m6", lib=oracle_lib) as e:
        with pytest.raises(abi.SphError) as ex:
            e.errcalc()
    assert ex.value.status == "SPH_ERR_UNSUPPORTED"


def test_driver_writes_result_line(oracle_lib, tmp_path):
    """ContinueRun ends like main.f90:425-428: (resolution, realpn, L1, 0,
    hfac) appended to result.info."""
    st, store = ic.sod2d(tfinish=0.002)
    ic.set_state(st, "ics", consts.ett["hydroshock"])
    ic.set_state(st, "dtprint", 0.002)
    c = core.Context(pwd=str(tmp_path))
    os.makedirs(os.path.join(str(tmp_path), "output"), exist_ok=True)
    c.state, c.store = st.copy(), store.copy()
    c.setup.kernel = "m6"
    c.ContinueRun(lib=oracle_lib)
    line = open(os.path.join(str(tmp_path), "result.info")).read().split()
    assert len(line) == 5
    vals = [float(v) for v in line]
    assert vals[1] == ic.get_state(st, "realpn")
    assert vals[3] == 0.0 and vals[4] == ic.get_state(st, "hfac")
    with abi.Engine(c.state, c.store, "m6", lib=oracle_lib) as e:
        _, l1 = e.errcalc()
    assert vals[2] == pytest.approx(l1, rel=1e-15)
    assert 0.0 < vals[2] < 0.05


# ---- GPU: the CUDA calculators against the oracle ----------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_gpu_errcalc_matches_oracle(engine_lib, oracle_lib, cuda_ok, kind):
    st, store = _case(kind)
    with abi.Engine(st, store, "m6", lib=oracle_lib) as e:
        err0, l10 = e.errcalc()
    with abi.Engine(st, store, "m6", lib=engine_lib) as e:
        err1, l11 = e.errcalc()
    np.testing.assert_allclose(err1, err0, rtol=1e-12, atol=1e-14)
    assert l11 == pytest.approx(l10, rel=1e-12, abs=1e-15)


@pytest.mark.gpu
def test_gpu_errcalc_after_reordered_run(engine_lib, oracle_lib, cuda_ok):
    """A Sod run whose rows the device reorders every 2 steps: err comes
    back in the original row order, equal to the oracle's after the same
    steps (the states agree to ~1e-12)."""
    st, store = ic.sod2d(tfinish=0.2)
    ic.set_state(st, "ics", consts.ett["hydroshock"])
    out = []
    for lib in (oracle_lib, engine_lib):
        with abi.Engine(st, store, "m6", lib=lib) as e:
            e.set_param(abi.P_REORDER_EVERY, 2)
            e.step(6)
            out.append(e.errcalc())
    np.testing.assert_allclose(out[1][0], out[0][0], rtol=1e-8, atol=1e-10)
    assert out[1][1] == pytest.approx(out[0][1], rel=1e-9)
