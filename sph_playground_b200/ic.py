"""Host-side initial conditions and state vectors.

Initial conditions are not part of the GPU hot path: the reference builds
them on the host (``place``, playground/src/IC/place.f90:22-91) and the
experiment runners then edit fields in the dump
(playground/runner/006.1_hydro_shock.py:70-116).  This module restates
``fillargs`` defaults (args.f90:29-176), ``place`` + ``uniformV4``
(IC/placeUniform.f90:14-84) in numpy, and builds the synthetic particle sets
of the benchmark configurations with seeded generators.
"""
import math

import numpy as np

from . import consts

ec, es, ept = consts.ec, consts.es, consts.ept


def col(name):
    """0-based store column of a field name."""
    return es[name] - 1


def blank_state():
    """clearState(): every slot -1 (state.f90:43-45)."""
    return np.full(consts.EC_TOTAL, -1.0)


def set_state(state, key, value):
    state[ec[key] - 1] = value


def get_state(state, key):
    return state[ec[key] - 1]


def make_state(dim, equations="hydro", ddw="fab", hfac=1.2, tfinish=1.0,
               npics=0, adden="yes", artts="yes", au=0.0, disotropic="yes",
               coordsys="cartesian", process="fullyperiodic", ics="none",
               usedumps="yes", silent="yes", xmin=0.0, xmax=1.0, ymin=0.0,
               ymax=1.0, zmin=0.0, zmax=1.0, placement="uniform",
               resolution=0, spacing=0.0):
    """The state vector that `./execute --key value ...` sets before place()
    runs (args.f90:29-176, state.f90 setters)."""
    s = blank_state()
    if resolution:
        set_state(s, "resolution", resolution)
    set_state(s, "xmin", xmin); set_state(s, "xmax", xmax)
    set_state(s, "ymin", ymin); set_state(s, "ymax", ymax)
    set_state(s, "zmin", zmin); set_state(s, "zmax", zmax)
    set_state(s, "placement", consts.PLACEMENT[placement])
    set_state(s, "ics", consts.ICS[ics])
    if npics:
        set_state(s, "npics", npics)
    if tfinish != 0.0:
        set_state(s, "tfinish", tfinish)
    set_state(s, "coordsys", {"cartesian": 1, "cylindric": 2}[coordsys])
    set_state(s, "artts", consts.eif[artts])
    set_state(s, "eqs", consts.EQUATIONS[equations] if equations in consts.EQUATIONS
              else consts.eeq[equations])
    set_state(s, "ddw", consts.DDW[ddw] if ddw in consts.DDW else consts.esd[ddw])
    set_state(s, "hfac", hfac)
    set_state(s, "silent", 1 if silent == "yes" else 0)
    if spacing:
        set_state(s, "spacing", spacing)
    set_state(s, "adden", consts.eif[adden])
    set_state(s, "usedumps", 1 if usedumps == "yes" else 0)
    set_state(s, "dim", dim)
    set_state(s, "process", consts.PROCESS[process])
    set_state(s, "au", au)
    set_state(s, "disotropic", consts.eif[disotropic])
    set_state(s, "lastprint", 0)
    return s


def place_uniform(state, kernel="m6", dxmin=None, dxmax=None):
    """place() with uniform placement (IC/place.f90:22-91 and
    IC/placeUniform.f90:14-84).  Returns the (N, 32) store with positions and
    type set; updates resolution, spacing, borders, particle counts in
    `state`.  `dxmin`/`dxmax` give the two-spacing layout (x<0 / x>=0) that
    uniformV4 supports."""
    dim = int(get_state(state, "dim"))
    hfac = get_state(state, "hfac")
    xmin, xmax = get_state(state, "xmin"), get_state(state, "xmax")
    ymin, ymax = get_state(state, "ymin"), get_state(state, "ymax")
    zmin, zmax = get_state(state, "zmin"), get_state(state, "zmax")
    resolution = get_state(state, "resolution")
    spacing = get_state(state, "spacing")
    kr = consts.KRAD[kernel]
    null2 = 0 if dim == 1 else 1
    null3 = 1 if dim == 3 else 0
    nb = int(kr * hfac) + 1
    if int(resolution) <= 0 and spacing <= 0:
        raise ValueError("Both resolution and spacing were not specified")
    if int(resolution) <= 0:
        resolution = int((xmax - xmin) / spacing)
    spacing = (xmax - xmin) / resolution
    bordersize = nb * spacing
    set_state(state, "resolution", resolution)
    set_state(state, "spacing", spacing)
    ymin, ymax = ymin * null2, ymax * null2
    zmin, zmax = zmin * null3, zmax * null3
    d_min = spacing if dxmin is None else dxmin
    d_max = d_min if dxmax is None or dxmax <= 0 else dxmax
    pdg = 0.5
    rows = []
    ix1, ix2 = int(xmin / d_min), int(xmax / d_max)
    sp = d_max
    for i in range(ix1, ix2 - int(2 * pdg) + 1):
        sp = d_min if i < 0 else d_max
        iy1, iy2 = int(ymin / sp), int(ymax / sp)
        iz1, iz2 = int(zmin / sp), int(zmax / sp)
        jj = np.arange(iy1, iy2 - int(2 * pdg) * null2 + 1)
        kk = np.arange(iz1, iz2 - int(2 * pdg) * null3 + 1)
        J, K = np.meshgrid(jj, kk, indexing="ij")
        blk = np.zeros((J.size, consts.ES_TOTAL))
        blk[:, col("rx")] = (pdg + i) * sp
        blk[:, col("ry")] = (null2 * pdg + J.ravel()) * sp
        blk[:, col("rz")] = (null3 * pdg + K.ravel()) * sp
        blk[:, col("type")] = ept["real"]
        rows.append(blk)
    store = np.concatenate(rows, axis=0)
    set_state(state, "realpn", store.shape[0])
    set_state(state, "fixedpn", 0)
    set_state(state, "bordsize", bordersize)
    set_state(state, "padding", pdg * sp)
    for k, v in (("xmin", xmin), ("xmax", xmax), ("ymin", ymin),
                 ("ymax", ymax), ("zmin", zmin), ("zmax", zmax)):
        set_state(state, k, v)
    return store


def m6_w(r, h, dim):
    """M6 kernel W(r, h) (kernel/base_m6.f90:36-55, kernel.f90:178-187)."""
    norm = {1: 1.0 / 120.0, 2: 7.0 / (478.0 * math.pi),
            3: 1.0 / (120.0 * math.pi)}[dim]
    q = np.asarray(r) / h
    t3 = np.clip(3.0 - q, 0, None)
    t2 = np.clip(2.0 - q, 0, None)
    t1 = np.clip(1.0 - q, 0, None)
    return norm * (t3 ** 5 - 6 * t2 ** 5 + 15 * t1 ** 5) / h ** dim


def periodic_lattice(n, dim, seed=None, amp=0.0, box=1.0):
    """n^dim lattice at (i+1/2)*dx in [0, box)^dim with an optional seeded
    uniform(-amp, amp)*dx offset per axis, wrapped back into the box."""
    dx = box / n
    ax = (np.arange(n) + 0.5) * dx
    grids = np.meshgrid(*([ax] * dim), indexing="ij")
    pos = np.zeros((n ** dim, 3))
    for k in range(dim):
        pos[:, k] = grids[k].ravel()
    if amp:
        rng = np.random.default_rng(seed)
        pos[:, :dim] += rng.uniform(-amp, amp, size=(n ** dim, dim)) * dx
        pos[:, :dim] = np.mod(pos[:, :dim], box)
    return pos, dx


def _periodic_state(dim, n, hfac, kernel, equations, **kw):
    s = make_state(dim, equations=equations, hfac=hfac, resolution=n, **kw)
    spacing = 1.0 / n
    kr = consts.KRAD[kernel]
    set_state(s, "spacing", spacing)
    set_state(s, "bordsize", (int(kr * hfac) + 1) * spacing)
    set_state(s, "padding", 0.5 * spacing)
    set_state(s, "xmin", 0.0); set_state(s, "xmax", 1.0)
    set_state(s, "ymin", 0.0); set_state(s, "ymax", 1.0 if dim > 1 else 0.0)
    set_state(s, "zmin", 0.0); set_state(s, "zmax", 1.0 if dim > 2 else 0.0)
    set_state(s, "fixedpn", 0)
    set_state(s, "dcondconst", 1.0)  # preruncheck.f90:32 wants it > 0 when isotropic
    return s


def density3d(n=128, seed=2, amp=0.1, hfac=1.2, kernel="m6"):
    """Density + Newton h-iteration workload: n^3 periodic lattice perturbed
    by uniform(-amp, amp)*dx per axis, equal masses, rho0 = 1, h0 = hfac*dx."""
    pos, dx = periodic_lattice(n, 3, seed=seed, amp=amp)
    N = pos.shape[0]
    st = _periodic_state(3, n, hfac, kernel, "hydro", tfinish=1.0)
    set_state(st, "realpn", N)
    set_state(st, "gamma", 5.0 / 3.0)
    set_state(st, "dtprint", 1.0)
    set_state(st, "time", 0.0)
    store = np.zeros((N, consts.ES_TOTAL))
    store[:, 0:3] = pos
    store[:, col("m")] = 1.0 / N
    store[:, col("den")] = 1.0
    store[:, col("h")] = hfac * dx
    store[:, col("om")] = 1.0
    store[:, col("u")] = 1.0
    store[:, col("p")] = 1.0
    store[:, col("c")] = 1.0
    store[:, col("type")] = ept["real"]
    return st, store


def sedov3d(n=128, E=1.0, p0=1e-5, gamma=5.0 / 3.0, hfac=1.2,
            kernel="m6", tfinish=0.05, npics=10):
    """Sedov blast in the unit periodic box: n^3 lattice, rho = 1, background
    P = p0, energy E deposited kernel-weighted (M6, h0 = hfac*dx) on the
    particles within 2*h0 of the centre."""
    pos, dx = periodic_lattice(n, 3)
    N = pos.shape[0]
    st = _periodic_state(3, n, hfac, kernel, "hydro", tfinish=tfinish,
                         npics=npics)
    set_state(st, "realpn", N)
    set_state(st, "gamma", gamma)
    set_state(st, "dtprint", tfinish / npics)
    set_state(st, "time", 0.0)
    set_state(st, "au", 1.0)
    m = 1.0 / N
    h0 = hfac * dx
    u0 = p0 / ((gamma - 1.0) * 1.0)
    u = np.full(N, u0)
    r = np.linalg.norm(pos - 0.5, axis=1)
    sel = r < 2.0 * h0
    w = m6_w(r[sel], h0, 3)
    u[sel] += E * w / (m * w.sum())
    store = np.zeros((N, consts.ES_TOTAL))
    store[:, 0:3] = pos
    store[:, col("m")] = m
    store[:, col("den")] = 1.0
    store[:, col("h")] = h0
    store[:, col("om")] = 1.0
    store[:, col("u")] = u
    store[:, col("p")] = (gamma - 1.0) * u
    store[:, col("c")] = np.sqrt(gamma * (gamma - 1.0) * u)
    store[:, col("type")] = ept["real"]
    return st, store


def sod2d(hfac=1.0, gamma=5.0 / 3.0, tfinish=0.2, npics=10, kernel="m6",
          adden="yes"):
    """2D Sod-type tube: x in [-1, 1] free, y periodic with width 0.125.
    Left spacing 1/256 (rho 1, P 1), right 1/128 (rho 0.125, P 0.1), v = 0,
    m = rho * sp^2 on each side.  Ghosts in y only, the reference's shock12
    geometry (IC/IC.f90:102-114, iterator.f90:79-87)."""
    st = make_state(2, equations="hydro", hfac=hfac, tfinish=tfinish,
                    npics=npics, adden=adden, artts="yes", au=1.0,
                    process="backcompatibility", ics="shock12",
                    xmin=-1.0, xmax=1.0, ymin=-0.0625, ymax=0.0625,
                    zmin=0.0, zmax=0.0, spacing=1.0 / 128)
    store = place_uniform(st, kernel, dxmin=1.0 / 256, dxmax=1.0 / 128)
    N = store.shape[0]
    x = store[:, col("rx")]
    left = x < 0
    sp = np.where(left, 1.0 / 256, 1.0 / 128)
    rho = np.where(left, 1.0, 0.125)
    P = np.where(left, 1.0, 0.1)
    u = P / ((gamma - 1.0) * rho)
    store[:, col("m")] = rho * sp ** 2
    store[:, col("den")] = rho
    store[:, col("p")] = P
    store[:, col("u")] = u
    store[:, col("c")] = np.sqrt(gamma * P / rho)
    store[:, col("h")] = hfac * sp
    store[:, col("om")] = 1.0
    set_state(st, "gamma", gamma)
    set_state(st, "dtprint", tfinish / npics)
    set_state(st, "time", 0.0)
    set_state(st, "realpn", N)
    set_state(st, "dcondconst", 1.0)
    return st, store


def diffusion2d(n, ddw="fab", seed=None, amp=0.05, hfac=1.2, kernel="m6",
                tfinish=0.01, sts_stages=8, bangle_deg=30.0, k_par=1.0,
                full_tensor=False, npics=1):
    """Anisotropic diffusion instance: n^2 periodic lattice perturbed by
    uniform(-amp, amp)*dx (seed n by default), T0 = sin(2 pi x) sin(2 pi y)
    (or the b b^T eigen-mode for the full tensor), B = b on every particle,
    difcond = k_par, disotropic = no, diffusion only, fixed-s STS."""
    seed = n if seed is None else seed
    pos, dx = periodic_lattice(n, 2, seed=seed, amp=amp)
    N = pos.shape[0]
    st = _periodic_state(2, n, hfac, kernel, "manual", ddw=ddw,
                         tfinish=tfinish, npics=npics, disotropic="no",
                         artts="no")
    set_state(st, "realpn", N)
    set_state(st, "gamma", 5.0 / 3.0)
    set_state(st, "dcondconst", k_par)
    set_state(st, "eqonhydro", 0.0)
    set_state(st, "eqondiff", 1.0)
    set_state(st, "eqonfluxlim", 0.0)
    set_state(st, "eqonradexch", 0.0)
    set_state(st, "eqonsts", 1.0)
    set_state(st, "ststype", consts.ests["fixeds"])
    set_state(st, "stsfixeds", sts_stages)
    set_state(st, "dtprint", tfinish / npics)
    set_state(st, "time", 0.0)
    set_state(st, "muzero", 1.0)
    b = (math.cos(math.radians(bangle_deg)), math.sin(math.radians(bangle_deg)))
    x, y = pos[:, 0], pos[:, 1]
    if full_tensor:
        T0 = 0.5 * (np.cos(2 * np.pi * (x - y)) - np.cos(2 * np.pi * (x + y)))
    else:
        T0 = np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y)
    gamma = 5.0 / 3.0
    u = 1.0 / (gamma * (gamma - 1.0))  # EOS gives c = 1 (dt_diff uses min c)
    store = np.zeros((N, consts.ES_TOTAL))
    store[:, 0:3] = pos
    store[:, col("m")] = 1.0 / N
    store[:, col("den")] = 1.0
    store[:, col("h")] = hfac * dx
    store[:, col("om")] = 1.0
    store[:, col("u")] = u
    store[:, col("p")] = (gamma - 1.0) * u
    store[:, col("c")] = 1.0
    store[:, col("kappa")] = 1.0
    store[:, col("t")] = T0
    store[:, col("bx")] = b[0]
    store[:, col("by")] = b[1]
    store[:, col("type")] = ept["real"]
    return st, store


def diffusion_exact(pos, t, bangle_deg=30.0, k_par=1.0, full_tensor=False):
    """Analytic T(t) of diffusion2d: diagonal K = k_par diag(bx^2, by^2)
    decays sin*sin as exp(-4 pi^2 k_par (bx^2 + by^2) t); the full k_par b b^T
    splits the initial mode into cos 2pi(x-y) and cos 2pi(x+y) with rates
    4 pi^2 k_par (bx -/+ by)^2."""
    b = (math.cos(math.radians(bangle_deg)), math.sin(math.radians(bangle_deg)))
    x, y = pos[:, 0], pos[:, 1]
    if full_tensor:
        a1 = math.exp(-4 * math.pi ** 2 * k_par * (b[0] - b[1]) ** 2 * t)
        a2 = math.exp(-4 * math.pi ** 2 * k_par * (b[0] + b[1]) ** 2 * t)
        return 0.5 * (np.cos(2 * np.pi * (x - y)) * a1 - np.cos(2 * np.pi * (x + y)) * a2)
    a = math.exp(-4 * math.pi ** 2 * k_par * (b[0] ** 2 + b[1] ** 2) * t)
    return np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * a


def shear2d(n=256, amp=0.1, seed=4, noise_seed=5, noise=1e-3, rho=1.0,
            P=2.5, gamma=5.0 / 3.0, hfac=1.2, kernel="m6", tfinish=1.0):
    """Adjoint workload: n^2 periodic lattice perturbed by uniform(-0.1,0.1)*dx
    (seed 4), rho = 1, P = 2.5, vx = amp*sin(2 pi y) + N(0, noise) (seed 5)."""
    pos, dx = periodic_lattice(n, 2, seed=seed, amp=0.1)
    N = pos.shape[0]
    st = _periodic_state(2, n, hfac, kernel, "hydro", tfinish=tfinish)
    set_state(st, "realpn", N)
    set_state(st, "gamma", gamma)
    set_state(st, "dtprint", tfinish)
    set_state(st, "time", 0.0)
    set_state(st, "au", 0.0)
    u = P / ((gamma - 1.0) * rho)
    rng = np.random.default_rng(noise_seed)
    store = np.zeros((N, consts.ES_TOTAL))
    store[:, 0:3] = pos
    store[:, col("vx")] = amp * np.sin(2 * np.pi * pos[:, 1]) + rng.normal(0.0, noise, N)
    store[:, col("m")] = rho / N
    store[:, col("den")] = rho
    store[:, col("h")] = hfac * dx
    store[:, col("om")] = 1.0
    store[:, col("u")] = u
    store[:, col("p")] = P
    store[:, col("c")] = math.sqrt(gamma * P / rho)
    store[:, col("type")] = ept["real"]
    return st, store


def hyrad1d(resolution=128, kernel="gauss", T_gas=1500.0, T_rad=2000.0, rho=1e-10,
            kappa=4e-3, mu=2.0, gamma=5.0 / 3.0, csound=3.2e5, ststype="auto",
            exchange_only=False):
    """Radiating shock tube (runner/004.3_fluxlimdif_shock.py): 1D uniform
    particles on x in [-1e15, 1e15], periodic (the runner closes the tube
    with periodic fixed particles instead), rho = 1e-10, gas at T_gas,
    radiation energy xi = 4 sigma T_rad^4 / (c rho), flows of +-csound
    towards x = 0; hydro + flux-limited diffusion (fab, isotropic) +
    radiation exchange, STS.  With `exchange_only` the gas is at rest and
    only the exchange acts (hydro, diffusion and STS off)."""
    RG, STEBOLTZ, C = 8.314e7, 5.67051e-5, 2.997924e10  # const.f90:6-8
    st = make_state(1, "manual", ddw="fab", hfac=1.0, tfinish=1e9, adden="yes",
                    artts="yes", au=1.0, disotropic="yes", process="fullyperiodic",
                    xmin=-1e15, xmax=1e15, resolution=resolution)
    store = place_uniform(st, kernel)
    N = store.shape[0]
    sp = get_state(st, "spacing")
    set_state(st, "gamma", gamma)
    set_state(st, "molecularmass", mu)
    set_state(st, "dcondconst", kappa)
    set_state(st, "time", 0.0)
    set_state(st, "dtprint", 1e9)
    set_state(st, "eqonhydro", 0.0 if exchange_only else consts.eif["yes"])
    set_state(st, "eqondiff", 0.0 if exchange_only else consts.eif["yes"])
    set_state(st, "eqonfluxlim", 0.0 if exchange_only else consts.eif["yes"])
    set_state(st, "eqonradexch", consts.eif["yes"])
    set_state(st, "eqonsts", 0.0 if exchange_only else consts.eif["yes"])
    set_state(st, "ststype", consts.ests[ststype])
    set_state(st, "muzero", 1.0)
    ksi = 4.0 * STEBOLTZ * T_rad ** 4 / C / rho
    u = T_gas * RG / (gamma - 1.0) / mu
    store[:, col("m")] = rho * sp  # CalcUniformMass in 1D
    store[:, col("den")] = rho
    store[:, col("h")] = get_state(st, "hfac") * sp
    store[:, col("om")] = 1.0
    store[:, col("u")] = u
    store[:, col("p")] = u * rho * (gamma - 1.0)
    store[:, col("c")] = csound
    store[:, col("kappa")] = kappa
    store[:, col("t")] = ksi
    if not exchange_only:
        x = store[:, col("rx")]
        store[:, col("vx")] = np.where(x <= 0.0, csound, -csound)
    return st, store

