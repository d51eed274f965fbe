"""The dump file written and read without libhdf5 (sph_playground_b200/h5dump.py).

The reader is checked on a file the HDF5 library wrote (a MATLAB v7.3 file
that ships with scipy's test data, whose dataset holds pi/4 * (0..8)); the
writer through the reader and through a walk of its structures against the
format's rules (signatures, node sizes inside the file, end-of-file
address)."""
import os
import struct

import numpy as np
import pytest
import scipy

from sph_playground_b200 import consts, core, h5dump, ic

SAMPLE = os.path.join(os.path.dirname(scipy.__file__), "io", "matlab", "tests", "data",
                      "testhdf5_7.4_GLNX86.mat")


@pytest.mark.skipif(not os.path.exists(SAMPLE), reason="scipy test data not installed")
def test_reader_on_a_library_written_file():
    d = h5dump.read(SAMPLE)
    assert np.array_equal(d["testdouble"].ravel(), np.pi / 4 * np.arange(9, dtype=float))


def test_write_read_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    st, store = rng.normal(size=49), rng.normal(size=(777, 32))
    p = str(tmp_path / "dump_full.h5")
    h5dump.write(p, {"state": st, "store": store})
    d = h5dump.read(p)
    assert np.array_equal(d["state"], st) and np.array_equal(d["store"], store)


def test_written_structures(tmp_path):
    p = str(tmp_path / "d.h5")
    h5dump.write(p, {"state": np.zeros(49), "store": np.ones((10, 32))})
    b = open(p, "rb").read()
    assert b[:8] == b"\x89HDF\r\n\x1a\n" and b[8] == 0
    eof = struct.unpack_from("<Q", b, 40)[0]
    assert eof == len(b)
    root_oh, cache, btree, heap = struct.unpack_from("<8xQI4xQQ", b, 56)
    assert cache == 1 and b[btree:btree + 4] == b"TREE" and b[heap:heap + 4] == b"HEAP"
    # the group B-tree node with its full 2K children fits in the file
    assert btree + 24 + 33 * 8 + 32 * 8 <= len(b)
    snod = struct.unpack_from("<Q", b, btree + 32)[0]
    assert b[snod:snod + 4] == b"SNOD" and struct.unpack_from("<H", b, snod + 6)[0] == 2
    # each dataset: chunked layout (class 2) with unlimited maximum dimensions
    for k in range(2):
        ohdr = struct.unpack_from("<Q", b, snod + 8 + 40 * k + 8)[0]
        ver, _, nmsg, _, size = struct.unpack_from("<BBHII", b, ohdr)
        at, seen = ohdr + 16, {}
        for _ in range(nmsg):
            mt, ms = struct.unpack_from("<HH", b, at)
            seen[mt] = at + 8
            at += 8 + ms
        assert at == ohdr + 16 + size and set(seen) == {1, 3, 5, 8}
        rank = b[seen[1] + 1]
        maxd = struct.unpack_from("<%dQ" % rank, b, seen[1] + 8 + 8 * rank)
        assert all(m == 0xFFFFFFFFFFFFFFFF for m in maxd)
        assert b[seen[8]] == 3 and b[seen[8] + 1] == 2
        bt = struct.unpack_from("<Q", b, seen[8] + 3)[0]
        assert b[bt:bt + 4] == b"TREE" and b[bt + 4] == 1


def test_context_dumps_are_hdf5(tmp_path):
    """CleanRun writes output/dump_full.h5 as an HDF5 file that reads back."""
    c = core.Context(pwd=str(tmp_path))
    s = c.setup
    s.kernel, s.dim, s.equations, s.hfac, s.tfinish = "m6", 2, "hydro", 1.2, 0.0
    s.resolution, s.nsnapshots = 16, 1
    s.xmin, s.xmax, s.ymin, s.ymax = 0.0, 1.0, 0.0, 1.0
    s.adden, s.artts, s.process = "yes", "yes", "fullyperiodic"
    c.CleanRun()
    p = os.path.join(str(tmp_path), "output", "dump_full.h5")
    assert open(p, "rb").read(8) == b"\x89HDF\r\n\x1a\n"
    st, store = core.read_dump(p)
    assert store.shape == (256, consts.ES_TOTAL) and st.shape == (consts.EC_TOTAL,)
    assert ic.get_state(st, "realpn") == 256
