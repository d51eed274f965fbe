"""The engine's own initial conditions: placement and per-type set-up.

When `./execute` starts a run (main.f90:133-139) it either places particles
(``place``, IC/place.f90:22-91: uniform, random or close-packed lattices) or,
for a named initial-condition type, runs ``setupV2`` (IC/IC.f90:48-560),
which places the lattice of that problem, mirrors border strips into fixed
particles where the problem has walls (``createFixedBorders``,
BC.f90:196-309, 477-640) and sets every field.  This module restates those
steps on the host with numpy; the driver's ``Context.CleanRun`` calls them.

Rows come out in the reference's order: the lattice rows (x outermost, then
y, then z), then the fixed rows in the order createFixedBorders appends
them.  The random lattice draws its offsets from numpy's seeded generator
(the reference uses the compiler's unseeded ``random_number``).
"""
import math

import numpy as np

from . import consts
from .ic import col, get_state, set_state

ept, ett, ebc = consts.ept, consts.ett, consts.ebc


def _nulls(dim):
    return (0, 0) if dim == 1 else ((1, 0) if dim == 2 else (1, 1))


def _store(pos):
    st = np.zeros((pos.shape[0], consts.ES_TOTAL))
    st[:, col("rx"):col("rz") + 1] = pos
    st[:, col("type")] = ept["real"]
    return st


def _set_borders(state, box, dbsz, pd):
    """setBorders (state.f90:397-408)."""
    for k, v in zip(("xmin", "xmax", "ymin", "ymax", "zmin", "zmax"), box):
        set_state(state, k, v)
    set_state(state, "bordsize", dbsz)
    set_state(state, "padding", pd)


def uniform_v4(state, box, dbsz, dxmin, dxmax=None, padding=0.0):
    """uniformV4 (IC/placeUniform.f90:14-84): a lattice of spacing dxmin for
    x cells i < 0 and dxmax for i >= 0, offset by `padding` cells."""
    dim = int(get_state(state, "dim"))
    n2, n3 = _nulls(dim)
    xmin, xmax, ymin, ymax, zmin, zmax = box
    dmx = dxmin if dxmax is None or dxmax <= 0 else dxmax
    pdg = padding
    blocks, sp = [], dmx
    for i in range(int(xmin / dxmin), int(xmax / dmx) - int(2 * pdg) + 1):
        sp = dxmin if i < 0 else dmx
        jj = np.arange(int(ymin / sp), int(ymax / sp) - int(2 * pdg) * n2 + 1)
        kk = np.arange(int(zmin / sp), int(zmax / sp) - int(2 * pdg) * n3 + 1)
        J, K = np.meshgrid(jj, kk, indexing="ij")
        p = np.empty((J.size, 3))
        p[:, 0] = (pdg + i) * sp
        p[:, 1] = (n2 * pdg + J.ravel()) * sp
        p[:, 2] = (n3 * pdg + K.ravel()) * sp
        blocks.append(p)
    store = _store(np.concatenate(blocks) if blocks else np.zeros((0, 3)))
    set_state(state, "realpn", store.shape[0])
    set_state(state, "fixedpn", 0)
    _set_borders(state, box, dbsz, pdg * sp)
    return store


def random_place(state, box, dbsz, dxmin, dxmax=None, padding=0.0, displacement=0.0,
                 seed=None):
    """random (IC/placeRandom.f90:14-126): the uniform lattice with every
    point moved by displacement * (u - 1/2) cells per axis, u uniform in
    [0, 1); points that leave the box are dropped."""
    dim = int(get_state(state, "dim"))
    n2, n3 = _nulls(dim)
    xmin, xmax, ymin, ymax, zmin, zmax = box
    dmx = dxmin if dxmax is None else dxmax
    pdg, drd = padding, displacement
    rng = np.random.default_rng(seed)
    blocks, sp = [], dmx
    for i in range(int(xmin / dxmin), int(xmax / dmx) - int(2 * pdg) + 1):
        sp = dxmin if i <= 0 else dmx
        jj = np.arange(int(ymin / sp), int(ymax / sp) - int(2 * pdg) * n2 + 1)
        kk = np.arange(int(zmin / sp), int(zmax / sp) - int(2 * pdg) * n3 + 1)
        J, K = np.meshgrid(jj, kk, indexing="ij")
        u = rng.random((J.size, 3))
        p = np.empty((J.size, 3))
        p[:, 0] = (pdg + i + drd * (u[:, 0] - 0.5)) * sp
        p[:, 1] = n2 * (pdg + J.ravel() + drd * (u[:, 1] - 0.5)) * sp
        p[:, 2] = n3 * (pdg + K.ravel() + drd * (u[:, 2] - 0.5)) * sp
        keep = ~((p[:, 0] < xmin) | (p[:, 0] > xmax) | (p[:, 1] < ymin) | (p[:, 1] > ymax)
                 | (p[:, 2] < zmin) | (p[:, 2] > zmax))
        blocks.append(p[keep])
    store = _store(np.concatenate(blocks) if blocks else np.zeros((0, 3)))
    set_state(state, "realpn", store.shape[0])
    set_state(state, "fixedpn", 0)
    _set_borders(state, box, dbsz, pdg * sp)
    return store


def closepacked(state, box, dbsz, dx, padding=(0.0, 0.0, 0.0)):
    """closepacked (IC/placeClose.f90:14-127): hexagonal rows of spacing dx,
    row pitch sqrt(3/4) dx, alternate rows shifted by dx/2; z layers of the
    same pitch alternate between the two row sets.  The y (and z) extent is
    widened by one row on both sides when that fits the box better."""
    dim = int(get_state(state, "dim"))
    n2, n3 = _nulls(dim)
    xmin, xmax, ymin, ymax, zmin, zmax = box
    pdg = padding
    spdx = dx
    ix1, ix2 = int(xmin / spdx), int(xmax / spdx)
    sph = math.sqrt(3.0 / 4.0 * spdx * spdx)
    spdx2, sph3 = spdx / 2.0, sph / 3.0

    def widen(lo, hi, new_lo, new_hi):
        i1, i2 = int(lo / sph), int(hi / sph)
        if i1 - i2 != 0:
            emin = abs((hi - lo) - (i2 - i1) * sph) / abs(hi - lo)
            emax = abs((hi - lo) - (i2 - i1 + 2) * sph) / abs(hi - lo)
            if emax < emin:
                i1, i2 = i1 - 1, i2 + 1
                new_lo, new_hi = i1 * sph, i2 * sph
        return i1, i2, new_lo, new_hi

    iy1, iy2, nymin, nymax = widen(ymin, ymax, sph * int(ymin / sph), sph * int(ymax / sph))
    iz1, iz2, nzmin, nzmax = widen(zmin, zmax, zmin, zmax)
    ii = np.arange(ix1, ix2 - int(2 * pdg[0]) + 1)
    jj = np.arange(iy1, iy2 - int(2 * pdg[1]) * n2 + 1)
    kk = np.arange(iz1, iz2 - int(2 * pdg[2]) * n3 + 1)
    I, J, K = (a.ravel() for a in np.meshgrid(ii, jj, kk, indexing="ij"))  # k fastest
    jm = (J - iy1) % 2
    even = (K - iz1) % 2 == 0
    keep = np.where(even, ~((I == ix2) & (jm != 0)), ~((I == ix1) & (jm == 0)))
    x = np.where(even, pdg[0] * spdx + spdx * I + jm * spdx2, spdx * I - spdx2 + jm * spdx2)
    y = np.where(even, n2 * pdg[1] * sph + sph * J, sph * J + sph3)
    z = np.where(even, n3 * pdg[2] * sph + sph * K, sph * K)
    pts = np.stack([x, y, z], axis=1)[keep]
    store = _store(pts)
    set_state(state, "realpn", store.shape[0])
    set_state(state, "fixedpn", 0)
    _set_borders(state, (xmin, xmax, nymin, nymax, nzmin, nzmax), dbsz, pdg[1] * sph)
    return store


def _inside_border(state, store, dim):
    """findInsideBorderParticles (BC.f90:196-309): per side, the real /
    fixed / fixedreal rows inside the border strip (closer to the wall than
    bordersize) and inside the padded box, in row order."""
    bs, pd = get_state(state, "bordsize"), get_state(state, "padding")
    lo = np.array([get_state(state, k) for k in ("xmin", "ymin", "zmin")])
    hi = np.array([get_state(state, k) for k in ("xmax", "ymax", "zmax")])
    bmin, bmax = lo + bs, hi - bs
    pmin, pmax = lo.copy(), hi.copy()
    if pd == 0:
        pmin, pmax = lo + pd / 10, hi - pd / 10
    t = store[:, col("type")].astype(int)
    ok = (t == ept["real"]) | (t == ept["fixed"]) | (t == ept["fixedreal"])
    r = store[:, col("rx"):col("rz") + 1]
    out = {}
    for a, name in enumerate("xyz"[:dim]):
        low = ok & (r[:, a] < bmin[a])
        out[name + "1"] = list(np.nonzero(low & (r[:, a] > pmin[a]))[0])
        out[name + "2"] = list(np.nonzero(ok & ~low & (r[:, a] > bmax[a]) & (r[:, a] < pmax[a]))[0])
    return out, lo, hi, bmin, bmax


def create_fixed_borders(state, store, side):
    """createFixedBorders (BC.f90:477-640): every row in a selected side's
    border strip gets a mirror image across that wall as a new fixed row
    (positions only; the set-up fills the fields).  Images made for x that
    fall in a y (z) strip join that strip's list, and images made for y join
    the z lists, so corners are mirrored again, as in the reference."""
    dim = int(get_state(state, "dim"))
    ib, lo, hi, bmin, bmax = _inside_border(state, store, dim)
    k0 = store.shape[0]
    blocks = []  # positions of the new rows, in creation order
    nnew = 0
    rx = col("rx")

    def mirror(pi_rows, axis, wall, later):
        # one side at a time, in list order: the images of the rows in this
        # side's strip, and their indices appended to the later strips'
        # lists in creation order
        nonlocal nnew
        if not len(pi_rows):
            return
        allpos = np.concatenate([store[:, rx:rx + 3]] + blocks) if blocks else store[:, rx:rx + 3]
        p = allpos[np.asarray(pi_rows, dtype=np.int64)].copy()
        p[:, axis] = wall + (wall - p[:, axis])
        k = k0 + nnew + np.arange(p.shape[0])
        for a in later:
            ib["xyz"[a] + "1"].extend(k[p[:, a] < bmin[a]].tolist())
            ib["xyz"[a] + "2"].extend(k[~(p[:, a] < bmin[a]) & (p[:, a] > bmax[a])].tolist())
        blocks.append(p)
        nnew += p.shape[0]

    if side in (ebc["all"], ebc["x"]):
        later = [a for a in (1, 2) if a < dim]
        mirror(ib["x1"], 0, lo[0], later)
        mirror(ib["x2"], 0, hi[0], later)
    if dim > 1:
        later = [2] if dim == 3 else []
        if side in (ebc["all"], ebc["y"], ebc["y1"]):
            mirror(ib["y1"], 1, lo[1], later)
        if side in (ebc["all"], ebc["y"], ebc["y2"]):
            mirror(ib["y2"], 1, hi[1], later)
        if dim == 3 and side in (ebc["all"], ebc["z"]):
            mirror(ib["z1"], 2, lo[2], [])
            mirror(ib["z2"], 2, hi[2], [])
    out = store
    if blocks:
        new = np.zeros((nnew, consts.ES_TOTAL))
        new[:, rx:rx + 3] = np.concatenate(blocks)
        new[:, col("type")] = ept["fixed"]
        out = np.concatenate([store, new], axis=0)
    set_state(state, "fixedpn", get_state(state, "fixedpn") + nnew)
    return out


def place(state, kernel="m6", seed=None):
    """place (IC/place.f90:22-91): the lattice of ec_placement over the box,
    spacing from resolution (or resolution from spacing)."""
    dim = int(get_state(state, "dim"))
    hfac = get_state(state, "hfac")
    n2, n3 = _nulls(dim)
    xmin, xmax = get_state(state, "xmin"), get_state(state, "xmax")
    ymin, ymax = get_state(state, "ymin") * n2, get_state(state, "ymax") * n2
    zmin, zmax = get_state(state, "zmin") * n3, get_state(state, "zmax") * n3
    res, spacing = get_state(state, "resolution"), get_state(state, "spacing")
    nb = int(consts.KRAD[kernel] * hfac) + 1
    if int(res) <= 0 and spacing <= 0:
        raise ValueError("Both resolution and spacing were not specified")
    if int(res) <= 0:
        res = int((xmax - xmin) / spacing)
    spacing = (xmax - xmin) / res
    dbsz = nb * spacing
    set_state(state, "resolution", res)
    set_state(state, "spacing", spacing)
    box = (xmin, xmax, ymin, ymax, zmin, zmax)
    pl = int(get_state(state, "placement"))
    if pl == consts.epl["random"]:
        return random_place(state, box, dbsz, spacing, displacement=0.8, seed=seed)
    if pl == consts.epl["closepacked"]:
        return closepacked(state, box, dbsz, spacing, padding=(0.0, 0.5, 0.5))
    return uniform_v4(state, box, dbsz, spacing, padding=0.5)


def setup_v2(state, kernel="m6", cv=1.0, seed=None, lib=None):
    """setupV2 (IC/IC.f90:48-560) for the initial-condition type in the
    state: lattice, fixed walls, fields.  The mti types end with a density
    pass over every row (IC.f90:597-606), run by the engine library `lib`
    (the CUDA engine by default).  sin3 stops in the reference ("Not set
    yet") and raises ValueError here."""
    dim = int(get_state(state, "dim"))
    n2, n3 = _nulls(dim)
    hfac = get_state(state, "hfac")
    ivt = int(get_state(state, "ics"))
    cs = int(get_state(state, "coordsys"))
    resol = int(get_state(state, "resolution"))
    pspc1 = get_state(state, "spacing")
    kr = consts.KRAD[kernel]
    nb = int(kr * hfac) + 1
    pi = math.pi
    # IC.f90:83-85, then per type
    set_state(state, "muzero", 1.0)
    set_state(state, "disotropic", 1.0)
    set_state(state, "dcondconst", 1.0)

    def res_from(b1, b2):
        r = resol if resol != 0 else int((b2 - b1) / pspc1)
        return r, (b2 - b1) / r

    rho2 = prs2 = eA = theta = phi = 0.0
    fixed_side = None
    if ivt == ett["sin3"]:
        raise ValueError("sin3: Not set yet (IC.f90:103)")
    elif ivt == ett["mti"]:  # IC.f90:160-177
        set_state(state, "dcondconst", 0.01)
        rho1, gamma = 1.0, 5.0 / 3.0
        b1, b2 = 0.0, 1.0 / 10.0
        resol, pspc1 = res_from(b1, b2)
        pspc2 = pspc1
        box = (b1, b2, 0.0, n2 * 1.0 / 10.0, 0.0, n3 * 1.0 / 10.0)
        bsz = nb * pspc2
        store = uniform_v4(state, box, bsz, pspc1, padding=0.5)
        store = create_fixed_borders(state, store, ebc["y"])
        # the Hopkins (2017) profile rho(y) = 2 (3 - y)^(1 - g h), g = -1, h = 3
        stretch_map(store, box[2] - bsz, box[3] + bsz, lambda y: 2.0 * (3.0 - y) ** 4, axis=1)
    elif ivt == ett["mtilowres"]:  # IC.f90:178-205
        set_state(state, "dcondconst", 0.1)
        rho1, gamma = 1.0, 5.0 / 3.0
        b1, b2 = -1.0, 1.0
        resol, pspc1 = res_from(b1, b2)
        pspc2 = pspc1
        box = (b1, b2, -2.0, 2.0, 0.0, n3 * 1.0)
        store = uniform_v4(state, box, nb * pspc2, pspc1, padding=0.5)
    elif ivt == ett["shock12"]:
        rho1, prs1, gamma = 1.0, 1.0, 5.0 / 3.0
        b1, b2 = -1.0, 1.0
        resol, pspc1 = res_from(b1, b2)
        pspc2 = pspc1
        box = (b1, b2, -pspc1 * nb * 2 * n2, pspc1 * nb * 2 * n2,
               -pspc1 * nb * 2 * n3, pspc1 * nb * 2 * n3)
        store = uniform_v4(state, box, nb * pspc1, pspc1, padding=0.5)
    elif ivt in (ett["pulse"], ett["ring"]):
        set_state(state, "disotropic", 0.0)
        rho1, prs1, gamma = 1.0, 1.0, 5.0 / 3.0
        b1, b2 = -1.0, 1.0
        resol, pspc1 = res_from(b1, b2)
        pspc2 = pspc1
        box = (b1, b2, -n2 * 1.0, n2 * 1.0, -n3 * 1.0, n3 * 1.0)
        store = random_place(state, box, nb * pspc2, pspc1, displacement=0.8, seed=seed)
    elif ivt == ett["soundwave"]:
        rho1, gamma, eA, prs1 = 1.0, 5.0 / 3.0, 0.1, 1.0
        b1, b2 = -1.0, 1.0
        resol, pspc1 = res_from(b1, b2)
        pspc2 = pspc1
        box = (b1, b2, -pspc1 * nb * 2 * n2, pspc1 * nb * 2 * n2,
               -pspc1 * nb * 2 * n3, pspc1 * nb * 2 * n3)
        store = uniform_v4(state, box, nb * pspc2, pspc1, padding=0.5)
    elif ivt == ett["hydroshock"]:
        gamma, prs1, rho1 = 5.0 / 3.0, 1.0, 1.0
        prs2, rho2 = prs1 / 10.0, rho1 / 8.0
        b1, b2 = -0.5, 0.5
        if resol == 0:
            resol = abs(int(b1 / pspc1))
        pspc1 = abs(b1 / resol)
        pspc2 = pspc1 * (8.0 if dim == 1 else 4.0)
        box = (b1, b2, -n2 * pspc2 * nb * 2, n2 * pspc2 * nb * 2,
               -n3 * pspc2 * nb * 2, n3 * pspc2 * nb * 2)
        store = uniform_v4(state, box, nb * pspc2, pspc1, dxmax=pspc2, padding=0.5)
        fixed_side = ebc["x"]
    elif ivt == ett["alfvenwave"]:
        set_state(state, "disotropic", 0.0)
        theta = phi = pi / 2.0
        rho1, gamma, eA, prs1 = 1.0, 5.0 / 3.0, 0.1, 0.1
        b1, b2 = 0.0, 1.0
        resol, pspc1 = res_from(b1, b2)
        pspc2 = pspc1
        nb = int(kr * hfac * 2)
        y2 = 1.0 / math.sin(theta) if dim > 1 else 0.0
        z2 = 1.0 if dim == 3 else 0.0
        box = (b1, b2, 0.0, y2, 0.0, z2)
        store = uniform_v4(state, box, nb * pspc2, pspc1, dxmax=pspc2, padding=0.5)
    elif ivt == ett["OTvortex"]:
        set_state(state, "disotropic", 0.0)
        prs1, rho1, gamma = 0.133, 0.221, 5.0 / 3.0
        b1, b2 = 0.0, 1.0
        resol, pspc1 = res_from(b1, b2)
        pspc2 = pspc1
        nb = int(kr * hfac * 2)
        box = (b1, b2, 0.0, 1.0 * n2, -pspc1 * nb * n3, pspc1 * nb * n3)
        store = uniform_v4(state, box, nb * pspc2, pspc1, padding=0.5)
    elif ivt == ett["boilingtank"]:
        rho1, gamma, prs1 = 1.0, 5.0 / 3.0, 0.0
        b1, b2 = -0.5, 0.5
        resol, pspc1 = res_from(b1, b2)
        pspc2 = pspc1
        box = (b1, b2, 0.0, n2 * 1.0, 0.0, n3 * 1.0)
        store = uniform_v4(state, box, nb * pspc2, pspc1, padding=0.5)
        fixed_side = ebc["y"]
    elif ivt == ett["fld_gauss"]:  # IC/setups/place_fld_gauss.f90
        rho1, prs1, gamma = 1.0, 1.0, 2.0
        b1, b2 = -10.0, 10.0
        resol, pspc1 = res_from(b1, b2)
        pspc2 = pspc1
        box = (b1, b2, -n2 * 1.0, n2 * 1.0, -n3 * 1.0, n3 * 1.0)
        store = uniform_v4(state, box, nb * pspc2, pspc1)
        fixed_side = ebc["all"]
    else:
        raise ValueError("Problem was not set: %d" % ivt)
    if fixed_side is not None:
        store = create_fixed_borders(state, store, fixed_side)
    if 2 * nb >= resol:
        raise ValueError("There is not enough resolution to cover artificial particles: %d" % resol)
    set_state(state, "gamma", gamma)
    rpn = int(get_state(state, "realpn"))
    xmn, xmx = box[0], box[1]
    lx, ly, lz = box[1] - box[0], box[3] - box[2], box[5] - box[4]
    ly = 1.0 if ly == 0.0 else ly
    lz = 1.0 if lz == 0.0 else lz
    s = store
    x, y, z = s[:, col("rx")], s[:, col("ry")], s[:, col("rz")]
    n = s.shape[0]
    s[:, col("c")] = cv
    s[:, col("om")] = 1.0
    sp = np.where(x < 0, pspc1, pspc2)
    C = lambda name: col(name)  # noqa: E731
    if ivt == ett["shock12"]:  # IC.f90:401-421
        s[:, C("h")] = hfac * sp
        s[:, C("m")] = lx * ly * lz * rho1 / rpn
        s[:, C("den")] = rho1
        s[:, C("p")] = prs1
        s[:, C("bx")], s[:, C("by")], s[:, C("bz")] = 1.0, 0.0, 0.0
        s[:, C("t")] = np.where(x < 0.0, 1.0, 2.0)
        s[:, C("u")] = prs1 / (gamma - 1) / rho1
    elif ivt == ett["pulse"]:  # :422-437
        s[:, C("h")] = hfac * sp
        s[:, C("m")] = (box[1] - box[0]) * (box[3] - box[2]) * rho1 / rpn
        s[:, C("den")] = rho1
        s[:, C("p")] = prs1
        s[:, C("bx")], s[:, C("by")], s[:, C("bz")] = 1.0, 0.0, 0.0
        s[:, C("kappa")] = 1.0
        s[:, C("u")] = prs1 / (gamma - 1) / rho1
    elif ivt == ett["ring"]:  # :438-471
        s[:, C("h")] = hfac * sp
        s[:, C("m")] = sp ** dim * rho1
        s[:, C("den")] = rho1
        s[:, C("p")] = prs1
        rr, ph = np.sqrt(x * x + y * y), np.arctan2(y, x)
        bx, by = np.zeros(n), np.ones(n)
        if cs == 1:  # the unit phi vector rotated into cartesian axes
            bx, by = np.cos(ph) * 0.0 - np.sin(ph) * 1.0, np.sin(ph) * 0.0 + np.cos(ph) * 1.0
        s[:, C("bx")], s[:, C("by")], s[:, C("bz")] = bx, by, 0.0
        s[:, C("t")] = np.exp(-0.5 * ((rr - 0.3) ** 2 / (0.05 * 0.05) + ph * ph / (0.5 * 0.5)))
        s[:, C("u")] = s[:, C("t")]
    elif ivt == ett["soundwave"]:  # :472-478
        s[:, C("h")] = hfac * sp
        s[:, C("den")] = rho1 * (1.0 + eA * np.sin(pi * x))
        s[:, C("m")] = sp ** dim * s[:, C("den")]
        s[:, C("vx")] = eA * np.sin(pi * x)
        s[:, C("p")] = prs1
        s[:, C("u")] = prs1 / (gamma - 1) / rho1
    elif ivt == ett["hydroshock"]:  # :479-492
        left = x <= 0.0
        s[:, C("h")] = np.where(left, hfac * pspc1, hfac * pspc2)
        s[:, C("den")] = np.where(left, rho1, rho2)
        s[:, C("p")] = np.where(left, prs1, prs2)
        s[:, C("m")] = np.where(left, pspc1 ** dim * rho1, pspc2 ** dim * rho2)
        s[:, C("u")] = np.where(left, prs1 / (gamma - 1) / rho1, prs2 / (gamma - 1) / rho2)
    elif ivt == ett["alfvenwave"]:  # :493-505
        s[:, C("h")] = hfac * sp
        s[:, C("m")] = sp ** dim * rho1
        s[:, C("den")] = rho1
        s[:, C("p")] = prs1
        s[:, C("u")] = prs1 / (gamma - 1) / rho1
        cca = np.array([math.cos(theta) * math.cos(phi), math.cos(theta) * math.sin(phi),
                        math.sin(theta)])
        dp = x * cca[0] + y * cca[1] + z * cca[2]
        s[:, C("vx")] = eA * 0.0
        s[:, C("vy")] = eA * np.sin(2 * pi * dp)
        s[:, C("vz")] = eA * np.cos(2 * pi * dp)
        s[:, C("bx")] = 1.0 + s[:, C("vx")]
        s[:, C("by")] = 0.0 + s[:, C("vy")]
        s[:, C("bz")] = 0.0 + s[:, C("vz")]
    elif ivt == ett["OTvortex"]:  # :538-557
        s[:, C("h")] = hfac * sp
        s[:, C("m")] = sp ** dim * rho1
        s[:, C("den")] = rho1
        s[:, C("p")] = prs1
        s[:, C("u")] = prs1 / (gamma - 1) / rho1
        s[:, C("vx")] = -np.sin(2 * pi * y)
        s[:, C("vy")] = np.sin(2 * pi * x)
        s[:, C("vz")] = 0.01
        s[:, C("bx")] = -1.0 / math.sqrt(4 * pi) * np.sin(2 * pi * y)
        s[:, C("by")] = 1.0 / math.sqrt(4 * pi) * np.sin(4 * pi * x)
        s[:, C("bz")] = 0.0
        if dim == 1:
            s[:, C("vy")] = s[:, C("vz")] = s[:, C("by")] = s[:, C("bz")] = 0.0
        elif dim == 2:
            s[:, C("vz")] = s[:, C("bz")] = 0.0
    elif ivt == ett["boilingtank"]:  # :558-575
        s[:, C("h")] = hfac * sp
        s[:, C("m")] = sp ** dim * rho1
        s[:, C("den")] = rho1
        s[:, C("u")] = 1.0
        s[:, C("t")] = 1.0
        hot = ((s[:, C("type")] == ept["fixed"]) & (y < box[2]) & (x > -0.075) & (x < 0.075))
        s[hot, C("t")] = 10.0
        s[hot, C("u")] = 10.0
        s[:, C("p")] = (gamma - 1.0) * s[:, C("den")] * s[:, C("u")]
        s[:, C("bx")] = s[:, C("by")] = 1.0
        s[:, C("vx")] = s[:, C("vy")] = s[:, C("vz")] = 0.0
    elif ivt == ett["fld_gauss"]:  # IC/setups/init_fld_gauss.f90
        s[:, C("h")] = hfac * sp
        s[:, C("m")] = sp ** dim * rho1
        s[:, C("den")] = rho1
        s[:, C("p")] = prs1
        s[:, C("t")] = 1.0 / ((2.0 * pi * (1.0 / 3.0) ** 2) ** (-dim / 2.0)) * np.exp(
            -0.5 * (x * x + y * y + z * z) / (1.0 / 3.0) ** 2)
        s[:, C("u")] = prs1 / (gamma - 1.0) / rho1
        s[:, C("kappa")] = 0.1
    elif ivt in (ett["mti"], ett["mtilowres"]):  # IC.f90:507-537
        s[:, C("h")] = hfac * sp
        s[:, C("m")] = sp ** dim * rho1
        s[:, C("den")] = rho1
        yy = y if ivt == ett["mti"] else np.abs(y)
        s[:, C("u")] = (3.0 / 2.0) * (1.0 - yy / 3.0)
        s[:, C("t")] = s[:, C("u")]
        s[:, C("p")] = (gamma - 1.0) * s[:, C("den")] * s[:, C("u")]
        s[:, C("vx")] = s[:, C("vy")] = s[:, C("vz")] = 0.0
        s[:, C("bx")] = s[:, C("by")] = s[:, C("bz")] = 0.0
        if ivt == ett["mti"]:
            r2 = x * x + y * y + z * z
            kick = (r2 > 0) & (s[:, C("type")] == ept["real"])
            s[kick, C("vy")] = 1e-2 * np.sqrt(gamma * s[kick, C("p")] / s[kick, C("den")]) * \
                np.sin(4.0 * pi * x[kick] / (box[1] - box[0]))
        s[:, C("bx")] = 1e-11
        s = _mti_density_pass(state, s, kernel, lib)
    del xmn, xmx
    return s


def stretch_map(store, cmin, cmax, rhofunc, axis=1, ngrid=1024, tol=1e-9, maxits=100,
                maxits_nr=30):
    """Stretch mapping of a uniform arrangement onto the density profile
    rhofunc along one axis (Price 2004, the cartesian form used by
    set_density_profile, utils/stretchmap.f90): a particle at c moves to c'
    with M(c') = rho0 (c - cmin), M(c) the mass of the profile between cmin
    and c and rho0 = M(cmax) / (cmax - cmin).  M is the trapezoid rule on
    ngrid steps with the first step's left end taken as 0, as the
    reference integrates; the root is found by Newton steps held within
    0.8-1.2 of the previous iterate, falling back to bisection, until
    |M(c') - rho0 (c - cmin)| <= tol M(cmax).  Moves positions in place."""

    def mass(x):  # x: array of end points
        dx = (x - cmin) / ngrid
        xi = cmin + dx[:, None] * np.arange(1, ngrid + 1)[None, :]
        d = rhofunc(xi) * dx[:, None]
        return d.sum(axis=1) - 0.5 * d[:, -1]

    totmass = float(mass(np.array([cmax]))[0])
    rhozero = totmass / (cmax - cmin)
    c = store[:, col("rx") + axis]
    for lo in range(0, c.shape[0], 4096):
        idx = np.arange(lo, min(lo + 4096, c.shape[0]))
        xold = c[idx]
        act = xold > cmin
        f0 = rhozero * (xold - cmin)
        xi = xold.copy()
        func = np.where(act, mass(np.where(act, xi, cmax)) - f0, 0.0)
        blo, bhi = np.full_like(xi, cmin), np.full_like(xi, cmax)
        bis = np.zeros(xi.shape, dtype=bool)
        its = np.zeros(xi.shape, dtype=int)
        run = act & (np.abs(func / totmass) > tol)
        while run.any():
            r = np.nonzero(run)[0]
            xprev = xi[r]
            its[r] += 1
            fr = mass(xprev) - f0[r]
            dfr = rhofunc(xprev)
            nb_ = bis[r]
            # bisection where it has taken over
            bl, bh = blo[r], bhi[r]
            bh = np.where(nb_ & (fr > 0), xprev, bh)
            bl = np.where(nb_ & ~(fr > 0), xprev, bl)
            xb = 0.5 * (bl + bh)
            # Newton elsewhere, its step held within 0.8-1.2 of the previous
            xn = xprev - fr / dfr
            ax, ap = np.abs(xn), np.abs(xprev)
            xn = np.where(ax < 0.8 * ap, 0.8 * xprev, np.where(ax > 1.2 * ap, 1.2 * xprev, xn))
            fail = ~nb_ & ((xn > cmax) | (xn < cmin) | (its[r] > maxits_nr))
            newbis = nb_ | fail
            xnew = np.where(nb_, xb, np.where(fail, 0.5 * (bl + bh), xn))
            xi[r], blo[r], bhi[r], bis[r] = xnew, bl, bh, newbis
            func[r] = fr
            run = act & (np.abs(func / totmass) > tol) & (its < maxits)
        if np.any(act & (its >= maxits)):
            raise ValueError("set_density_profile: Stretch mapping not converged")
        c[idx] = np.where(act, xi, xold)
    store[:, col("rx") + axis] = c


def _mti_density_pass(state, store, kernel, lib):
    """IC.f90:597-606: every row counted as real for one density pass with
    periodic images along x (the mti types' boundary), then the numbers of
    real and fixed rows restored."""
    from . import abi
    rpn, fpn = int(get_state(state, "realpn")), int(get_state(state, "fixedpn"))
    st = state.copy()
    set_state(st, "realpn", rpn + fpn)
    set_state(st, "fixedpn", 0)
    # the process whose boundary for these types is periodic along x alone
    # (iterator.f90:99-110), as the set-up's createPeriodicBorder(ebc_x)
    set_state(st, "process", consts.epc["backcompatibility"])
    with abi.Engine(st, store, kernel, lib=lib if lib is not None else abi.load()) as e:
        e.density()
        return e.get_store()
