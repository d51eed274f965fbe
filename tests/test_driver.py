"""The fortdriver-compatible Context (sph_playground_b200/core.py) on CPU:
the call sequence of the reference runners (CleanRun, ReadDumpHDF,
CalcUniformMass, ModifyParticlesProperties, Apply, ContinueRun), driven
through the oracle library so it runs without a GPU."""
import os

import numpy as np

from sph_playground_b200 import core


def test_context_runner_sequence(oracle_lib, tmp_path):
    c = core.Context(pwd=str(tmp_path))
    s = c.setup
    s.kernel, s.dim, s.equations, s.hfac, s.tfinish = "m6", 2, "hydro", 1.2, 0.0
    s.resolution, s.nsnapshots = 16, 2
    s.xmin, s.xmax, s.ymin, s.ymax = 0.0, 1.0, 0.0, 1.0
    s.adden, s.artts, s.process = "yes", "yes", "fullyperiodic"
    c.CleanRun()
    c.ReadDumpHDF(os.path.join(str(tmp_path), "output", "dump_full.h5"))
    assert c.store.shape == (256, 32) and int(c.setup.realpn) == 256
    m = c.CalcUniformMass(1.0)
    assert m == 1.0 / 256
    c.ModifyParticlesProperties(
        properties=["m", "den", "h", "p", "u", "c", "om"],
        value=[lambda x: m, lambda x: 1.0, lambda x: 1.2 / 16, lambda x: 1.0,
               lambda x: 1.5, lambda x: 1.29, lambda x: 1.0])
    c.setup.tfinish, c.setup.dtprint, c.setup.gamma = 0.02, 0.01, 5.0 / 3.0
    c.setup.dcondconst, c.setup.time = 1.0, 0.0
    c.Apply()
    c.ContinueRun(lib=oracle_lib)
    assert abs(c.GetState("time") - 0.02) < 1e-12
    outs = sorted(os.listdir(os.path.join(str(tmp_path), "output")))
    assert any(o.startswith("dump_00001") for o in outs)
    assert any(o.startswith("dump_00002") for o in outs)
    assert np.all(np.isfinite(c.store))


def test_enum_tables_in_context():
    c = core.Context()
    assert c.esd["2nw_ds"] == 403 and c.epc["fullyperiodic"] == 601
    assert c.ecRev[46] == "time" and c.esRev[31] == "type"


def _runner_006_sequence(tmp_path, resolution=128, tfinish=0.02):
    """The call sequence of runner/006.1_hydro_shock.py (1D colliding flows,
    borderless, manual equations with hydro only, periodic fixedreal copies
    of the border strips), shortened: resolution 128, a short ContinueRun."""
    c = core.Context(pwd=str(tmp_path))
    s = c.setup
    s.xmin, s.xmax, s.dim, s.placement, s.tfinish = -1, 1, 1.0, "uniform", 0.0
    s.kernel, s.hfac, s.nsnapshots, s.coordsys, s.silent = "m6", 1.0, 10.0, "cartesian", "no"
    s.usedumps, s.adden, s.artts, s.au, s.resolution = "yes", "no", "yes", 1.0, resolution
    c.CleanRun()
    c.BackupDump("output/dump_full.h5")
    c.ReadDumpHDF(os.path.join(str(tmp_path), "output", "dump_full.h5"))
    s = c.setup
    s.tfinish, s.dtprint, s.process, s.time = tfinish, tfinish / 2, c.epc["borderless"], 0.0
    s.disotropic, s.eqs, s.eqonhydro = 1.0, c.eeq["manual"], c.eif["yes"]
    s.ddw, s.eqondiff, s.eqonfluxlim = c.esd["fab"], c.eif["no"], c.eif["no"]
    s.eqonradexch, s.eqonsts, s.ststype = c.eif["no"], c.eif["no"], c.ests["auto"]
    rho, csound, kappa, gamma, prs = 1.0, 1.0, 1.0, 5.0 / 3.0, 1.0
    mass = c.CalcUniformMass(rho)
    h = s.hfac * s.spacing
    s.dcondconst, s.molecularmass, s.gamma = kappa, 2.0, gamma
    u = prs / rho / (gamma - 1.0)
    k = lambda v: (lambda x: v)  # noqa: E731
    c.ModifyParticlesProperties(
        properties=["kappa", "t", "c", "m", "den", "h", "p", "u", "om"],
        value=[k(kappa), k(0), k(csound), k(mass), k(rho), k(h), k(prs), k(u), k(1.0)])
    c.AddParticles(dim="x", type="fixedreal", method="periodic")
    c.ModifyParticlesProperties(properties=["vx"],
                                value=[lambda rx: csound if rx <= 0.0 else -csound],
                                valuearg=["rx"])
    c.Apply()
    return c


def test_runner_006_sequence_on_the_oracle(oracle_lib, tmp_path):
    c = _runner_006_sequence(tmp_path)
    n_fixed = int(c.setup.fixedpn)
    assert n_fixed > 0 and c.store.shape[0] == int(c.setup.realpn) + n_fixed
    c.ContinueRun(lib=oracle_lib)
    assert abs(c.GetState("time") - 0.02) < 1e-12
    assert np.all(np.isfinite(c.store))
    # the colliding flows heat the middle
    x = c.store[: int(c.setup.realpn), 0]
    u = c.store[: int(c.setup.realpn), c.es["u"] - 1]
    assert u[np.abs(x) < 0.05].max() > u[np.abs(x) > 0.5].max()
