"""The runners' unit helper (sph_playground_b200/units.py): the constants the
radiation runners use and the unit systems of Scale (c = 1, G = 1)."""
import math

import pytest

from sph_playground_b200.units import PhysicalConstants, Unit


def test_constants_used_by_the_runners():
    pc = PhysicalConstants()
    # runner/004.2_fluxlimdif_shock.py:84-92 use these
    assert pc.STEBOLTZ == 5.67051e-5 and pc.C == 2.997924e10 and pc.RG == 8.314e7
    assert pc.CGSMU0 == pytest.approx(4 * math.pi, rel=1e-9)
    assert pc.KB_ON_MH == pytest.approx(pc.KBOLTZ / pc.PROTON_MASS_CGS, rel=1e-15)


@pytest.mark.parametrize("kw", [dict(idist=1.5e13), dict(imass=2e33), dict(itime=3.0), {}])
def test_scale_with_c_equal_one(kw):
    pc = PhysicalConstants()
    u = pc.Scale(ic=1, **kw)
    assert u.dist / u.time == pytest.approx(pc.C, rel=1e-12)            # c = 1
    assert pc.GG * u.mass / u.dist == pytest.approx(pc.C ** 2, rel=1e-12)  # G M / L = c^2


@pytest.mark.parametrize("kw", [dict(idist=1.5e13, imass=2e33), dict(idist=2.0, itime=3.0),
                                dict(imass=5.0, itime=7.0), dict(itime=2.0), {}])
def test_scale_with_g_equal_one(kw):
    pc = PhysicalConstants()
    u = pc.Scale(ig=1, **kw)
    if "itime" in kw and "imass" not in kw:
        # the reference's mass from length and time: dist^2 / (G time^2)
        assert pc.GG * u.mass * u.time ** 2 / u.dist ** 2 == pytest.approx(1.0, rel=1e-12)
    else:
        assert pc.GG * u.mass * u.time ** 2 / u.dist ** 3 == pytest.approx(1.0, rel=1e-12)
    for k, attr in (("idist", "dist"), ("imass", "mass"), ("itime", "time")):
        if k in kw:
            assert getattr(u, attr) == kw[k]


def test_derived_units():
    u = Unit(2.0, 3.0, 5.0)
    assert u.velocity == 2.0 / 5.0 and u.density == 3.0 / 8.0
    assert u.pressure == 3.0 / (2.0 * 25.0) and u.energ == 3.0 * (2.0 / 5.0) ** 2
    assert u.charge == pytest.approx(math.sqrt(6.0 / (4 * math.pi)), rel=1e-9)
