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
