"""Enumerations of the reference engine, as the Python driver sees them.

The reference driver parses ``src/const.f90`` at run time
(playground/runner/fortdriver/core.py:235-319) into dictionaries keyed by the
name without its prefix (``ec_time`` -> ``ec['time']``).  The values are an
interface: state slots, store columns and the enum codes written into the
state vector must be the same numbers the Fortran engine used, so they are
kept identical here (playground/src/const.f90:14-193).  ``tests/golden/``
holds the table as parsed from the reference file and a test checks these
dictionaries against it.
"""

# state vector slots, 1-based (const.f90:14-66)
ec = {
    "dim": 1, "eqs": 2, "ddw": 3, "ics": 4, "adden": 5, "artts": 6,
    "coordsys": 7, "disotropic": 8, "dcondconst": 9, "muzero": 10,
    "tfinish": 11, "npics": 12, "hfac": 13, "silent": 14, "resolution": 15,
    "spacing": 16, "xmin": 17, "xmax": 18, "ymin": 19, "ymax": 20,
    "zmin": 21, "zmax": 22, "bordsize": 23, "padding": 24, "realpn": 25,
    "fixedpn": 26, "gamma": 27, "lastprint": 28, "usedumps": 29,
    "dtprint": 30, "process": 31, "au": 32, "placement": 33,
    "eqonhydro": 34, "eqondiff": 35, "eqonfluxlim": 36, "eqonradexch": 37,
    "eqonsts": 38, "udist": 39, "umass": 40, "utime": 41, "uvelocity": 42,
    "udensity": 43, "upressure": 44, "uacceller": 45, "time": 46,
    "molecularmass": 47, "ststype": 48, "stsfixeds": 49,
}
EC_TOTAL = 49

# particle table columns, 1-based (const.f90:69-101); "total" is skipped as
# core.py:245 does.
es = {
    "rx": 1, "ry": 2, "rz": 3, "vx": 4, "vy": 5, "vz": 6, "ax": 7, "ay": 8,
    "az": 9, "m": 10, "den": 11, "h": 12, "dh": 13, "p": 14, "u": 15,
    "du": 16, "t": 17, "kappa": 18, "dtdx": 19, "dtdy": 20, "dtdz": 21,
    "ddt": 22, "bx": 23, "by": 24, "bz": 25, "dbx": 26, "dby": 27,
    "dbz": 28, "c": 29, "om": 30, "type": 31, "vfld": 32,
}
ES_TOTAL = 32

ept = {"empty": 0, "real": 1, "fixed": 2, "fixedreal": 21,
       "fixedmirror": 22, "periodic": 3}
ett = {"sin3": 100, "mti": 101, "shock12": 102, "pulse": 103, "ring": 104,
       "soundwave": 105, "hydroshock": 106, "alfvenwave": 107,
       "OTvortex": 108, "boilingtank": 109, "mtilowres": 110,
       "fld_gauss": 111}
ebc = {"all": 200, "x": 201, "y": 202, "z": 203, "x1": 204, "y1": 205,
       "z1": 206, "x2": 207, "y2": 208, "z2": 209}
eeq = {"hydro": 300, "diffusion": 301, "magnetohydro": 302,
       "magnetohydrodiffusion": 303, "hydrodiffusion": 304, "kd2": 305,
       "hyrad": 306, "manual": 307}
esd = {"fab": 400, "n2w": 401, "fw": 402, "2nw_ds": 403, "2nw_sd": 404}
edi = {}
eqs = {"hydro": 1, "magneto": 2, "diff": 3, "fld": 4, "radexch": 5,
       "sts": 6, "total": 6}
epc = {"backcompatibility": 600, "fullyperiodic": 601, "borderless": 602}
eif = {"yes": 1.0, "no": 0.0}
ests = {"auto": 0.0, "fixeds": 1.0}
epl = {"uniform": 700, "random": 701, "closepacked": 702}


def reverse(d):
    """Value -> name map, like the ``*Rev`` dictionaries of core.py:199-233."""
    return {v: k for k, v in d.items()}


ecRev = reverse(ec)
esRev = reverse(es)

# command-line strings accepted by the reference's string -> enum setters
# (state.f90:91-112, :151-168, :174-213, :479-491, :497-512)
EQUATIONS = {"hydro": eeq["hydro"], "magnetohydro": eeq["magnetohydro"],
             "diffusion": eeq["diffusion"],
             "mhd": eeq["magnetohydrodiffusion"],
             "hydi": eeq["hydrodiffusion"], "kd2": eeq["kd2"],
             "hyrad": eeq["hyrad"]}
DDW = {"n2w": esd["n2w"], "fab": esd["fab"], "2nw-+": esd["2nw_ds"],
       "2nw+-": esd["2nw_sd"], "fw": esd["fw"]}
PROCESS = {"borderless": epc["borderless"],
           "fullyperiodic": epc["fullyperiodic"],
           "backcompatibility": epc["backcompatibility"]}
ICS = {"sin3": ett["sin3"], "mti": ett["mti"], "mtilowres": ett["mtilowres"],
       "shock12": ett["shock12"], "pulse": ett["pulse"], "ring": ett["ring"],
       "soundwave": ett["soundwave"], "hydroshock": ett["hydroshock"],
       "alfvenwave": ett["alfvenwave"], "otvortex": ett["OTvortex"],
       "boilingtank": ett["boilingtank"], "fld_gauss": ett["fld_gauss"],
       "none": -1}
PLACEMENT = dict(epl)

# kernel names of `make kernel=<k>` (playground/Makefile:14) -> C-ABI id
KERNELS = {"m4": 0, "m6": 1, "gauss": 2}
# support radius krad of each kernel (base_m4.f90:18, base_m6.f90:17,
# base_gauss.f90:19)
KRAD = {"m4": 2.0, "m6": 3.0, "gauss": 10.0}


# ---- const.f90 parsing (core.py:235-319) ------------------------------------------
CONST_PREFIXES = ["ec_", "es_", "ept_", "ett_", "ebc_", "eeq_", "esd_", "edi_", "eqs_",
                  "epc_", "eif_", "ests_"]


def parse_const_f90(path):
    """The reference driver's rule for reading src/const.f90: split each line
    into whitespace tokens and keep `name = value,&` triples; ec_/es_ entries
    only with the trailing ",&", es_total skipped.  Returns one dictionary
    per prefix, keyed by the name without the prefix."""
    out = {p[:-1]: {} for p in CONST_PREFIXES}
    with open(path) as f:
        for line in f:
            tok = line.split()
            if len(tok) != 3:
                continue
            name, val = tok[0], tok[2]
            for p in CONST_PREFIXES:
                if not name.startswith(p):
                    continue
                key = name[len(p):]
                if val.endswith(",&"):
                    val = val[:-2]
                elif p in ("ec_", "es_"):
                    continue
                if p == "es_" and key == "total":
                    continue
                out[p[:-1]][key] = float(val) if p in ("eif_", "ests_") else int(val)
    return out
