"""Sedov 3D at the larger of its lattices, 160^3 = 4,096,000 particles, on
the CUDA engine: properties that do not depend on the size, checked at full
size where the oracle would take too long.

* The first search runs with the set-up's uniform h on a periodic lattice,
  so every particle has the same neighbours: the lattice points within
  krad * hfac = 3.6 spacings, 178 of them (no lattice distance lies within
  0.3 % of the radius, so rounding cannot move one across it).
* The pair forces are antisymmetric, so FP64 sum_i m_i a_i vanishes to
  rounding against sum_i m_i |a_i|.
* The FP32-comp path stays within the FP64 path's tolerances: density 1e-6
  per particle, accelerations 1e-5 of the field maximum."""
import itertools

import numpy as np
import pytest

from sph_playground_b200 import abi, ic
from tests.parity import COL, rel_field

FP64, FP32 = abi.PREC_FP64, abi.PREC_FP32_COMP
N_SIDE = 160


def _lattice_neighbours(radius):
    r = int(radius) + 1
    return sum(1 for i, j, k in itertools.product(range(-r, r + 1), repeat=3)
               if i * i + j * j + k * k <= radius * radius) - 1


@pytest.mark.gpu
def test_sedov3d_160_full_size(engine_lib, cuda_ok):
    st, store = ic.sedov3d(n=N_SIDE)
    n = N_SIDE ** 3
    out = {}
    for prec in (FP64, FP32):
        with abi.Engine(st, store, "m6", precision=prec, lib=engine_lib) as e:
            e.reset_counters()
            e.iterate()
            out[prec] = (e.get_store(), e.counters())
    k = _lattice_neighbours(3.6)
    assert k == 178
    for prec in (FP64, FP32):
        c = out[prec][1]
        assert c["searches"] == 1 and c["neib_max"] == k, (prec, c)
        assert c["neib_pairs"] == n * k, (prec, c)

    s64, s32 = out[FP64][0], out[FP32][0]
    m = s64[:, COL["m"]]
    a = s64[:, [COL["ax"], COL["ay"], COL["az"]]]
    net = np.abs((m[:, None] * a).sum(axis=0))
    scale = (m[:, None] * np.abs(a)).sum(axis=0)
    assert np.all(net <= 1e-10 * scale), (net, scale)

    den_rel = np.max(np.abs(s32[:, COL["den"]] / s64[:, COL["den"]] - 1.0))
    assert den_rel <= 1e-6, den_rel
    for f in ("ax", "ay", "az"):
        err = rel_field(s32[:, COL[f]], s64[:, COL[f]])
        assert err <= 1e-5, (f, err)
