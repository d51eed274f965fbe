"""fortdriver-compatible driver: ``Setup`` and ``Context``.

Mirrors the reference's Python driver (playground/runner/fortdriver/core.py)
method for method, so experiment runners keep working, but runs the step in
process on the GPU engine instead of spawning ``./execute``:

* ``ReadConstFile`` fills the enum dictionaries (core.py:235-319) from the
  same const.f90 rules, or from the embedded tables when no file is given;
* ``SimpleRun`` / ``CleanRun`` do what ``./execute --key value`` does with
  tfinish = 0 (args.f90:29-176 + place, IC/place.f90:22-91): build the state
  vector and the particle table, and write the dump;
* ``ReadDumpHDF`` / ``Apply`` / ``ModifyParticlesProperties`` /
  ``AddParticles`` / ``CalcUniformMass`` edit the arrays as the reference
  does (core.py:321-470);
* ``ContinueRun`` (core.py:152-156) restores the dump into the engine and
  runs the time loop to tfinish, writing a dump at every output time
  (main.f90:241-373, printer.f90:19-38, dumper.f90:14-42).

Dumps are HDF5 files with the reference's two chunked, resizable datasets
(``state`` (49,) and ``store`` (N, 32), dumper.f90:26-34): through h5py when
it is importable, otherwise through this package's own HDF5 writer and
reader (sph_playground_b200/h5dump.py).
"""
import copy
import datetime
import os
import shutil

import numpy as np

from . import abi, consts, h5dump, ic, icsetup

try:  # optional: the reference's dump format
    import h5py  # noqa: F401
    HAVE_H5PY = True
except Exception:  # pragma: no cover - depends on the image
    HAVE_H5PY = False


class Setup:
    """Run settings; attribute names are the CLI keys / state names."""
    stderrfile = "__stderr.info"
    stdoutfile = "__stdout.info"
    logfile = "__runslog.info"
    kernel = "m4"

    def toArgs(self):
        args = []
        for k in self.__dict__.keys():
            args.append("--" + k)
            args.append(str(self.__dict__[k]))
        return args


def write_dump(path, state, store):
    """dumper.f90:14-42: write state and the real+fixed rows of store."""
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".new"
    if HAVE_H5PY:
        import h5py
        with h5py.File(tmp, "w") as f:
            f.create_dataset("state", data=state, maxshape=(None,), chunks=(state.shape[0],))
            f.create_dataset("store", data=store, maxshape=(None, consts.ES_TOTAL),
                             chunks=store.shape)
    else:
        h5dump.write(tmp, {"state": np.asarray(state, dtype=np.float64),
                           "store": np.asarray(store, dtype=np.float64)})
    os.replace(tmp, path)  # atomic rename, dumper.f90:36
    return path


def read_dump(path):
    if HAVE_H5PY:
        import h5py
        with h5py.File(path, "r") as f:
            return np.array(f["state"]), np.array(f["store"])
    d = h5dump.read(path)
    return np.array(d["state"]), np.array(d["store"])


class Context:
    """The reference's Context (core.py:46-470) over the in-process engine."""

    def __init__(self, constf90=None, pwd=None, precision=abi.PREC_FP64):
        self.pwd = pwd or os.getcwd()
        self.env = os.environ.copy()
        self.setup = Setup()
        self.store = None
        self.result = None  # the last run's result.info line (resolution, realpn, L1, chi, hfac)
        self.state = None
        self.precision = precision
        self.constf90 = constf90
        self.ReadConstFile()
        for key in self.ec.keys():
            self.setup.__dict__[key] = 0.0

    # ---- logs (core.py:60-132) -------------------------------------------
    def _log(self, name, s):
        fn = getattr(self.setup, name)
        if fn != "none":
            with open(os.path.join(self.pwd, fn), "a+") as f:
                f.write(s + "\n")

    def __tolog__(self, s):
        self._log("logfile", s)

    def CleanSTDLogs(self):
        for n in ("stdoutfile", "stderrfile"):
            fn = getattr(self.setup, n)
            if fn != "none":
                open(os.path.join(self.pwd, fn), "w").close()

    def CleanAllLogs(self):
        self.CleanSTDLogs()
        if self.setup.logfile != "none":
            open(os.path.join(self.pwd, self.setup.logfile), "w").close()

    def SetThreadsOMP(self, i):
        if i != 1:
            self.env["OMP_NUM_THREADS"] = str(i)

    def GetDateTimeString(self):
        d = datetime.datetime.today()
        return f"{d.year}-{d.month}-{d.day}-{d.hour}-{d.minute}-{d.second}"

    # ---- build / run ---------------------------------------------------------
    def SimpleMake(self, debug=False):
        """`make kernel=<k>` in the reference; here: build the library once
        (the kernel is chosen at run time)."""
        if not os.path.exists(abi.LIB_PATH):
            import subprocess
            subprocess.run(["make", "-C", os.path.join(os.path.dirname(abi.__file__), "csrc")],
                           check=True, capture_output=True)
        self.__tolog__("CMD [make kernel=" + str(self.setup.kernel) + "] EXECUTED")

    def _out(self, name):
        return os.path.join(self.pwd, "output", name)

    def SimpleRun(self, lib=None):
        """./execute --key value ... with tfinish = 0: fillargs + place + dump."""
        s = self.setup.__dict__
        get = lambda k, d=None: s.get(k, d)
        eqs = get("equations", "hydro")
        state = ic.make_state(
            int(get("dim", 1)), equations=eqs if isinstance(eqs, str) and eqs else "hydro",
            ddw=get("ddw", "fab") if isinstance(get("ddw"), str) else "fab",
            hfac=float(get("hfac", 1.2)), tfinish=float(get("tfinish", 1.0)),
            npics=int(float(get("nsnapshots", 0) or 0)),
            adden=get("adden", "yes") or "yes", artts=get("artts", "yes") or "yes",
            au=float(get("au", 0.0) or 0.0), disotropic=get("disotropic", "yes")
            if isinstance(get("disotropic"), str) else "yes",
            process=get("process", "fullyperiodic") if isinstance(get("process"), str)
            else "fullyperiodic",
            xmin=float(get("xmin", 0.0)), xmax=float(get("xmax", 1.0)),
            ymin=float(get("ymin", 0.0)), ymax=float(get("ymax", 1.0)),
            zmin=float(get("zmin", 0.0)), zmax=float(get("zmax", 1.0)),
            placement=get("placement", "uniform") or "uniform",
            ics=get("ics", "none") if isinstance(get("ics"), str) and get("ics") else "none",
            resolution=int(float(get("resolution", 0) or 0)),
            spacing=float(get("spacing", 0.0) or 0.0))
        kernel = str(self.setup.kernel)
        # main.f90:133-139: place() without an initial-condition type,
        # setupV2 with one
        if int(ic.get_state(state, "ics")) == consts.ICS["none"]:
            store = icsetup.place(state, kernel)
        else:
            store = icsetup.setup_v2(state, kernel, cv=1.0, lib=lib)
        tf = ic.get_state(state, "tfinish")
        npics = max(int(ic.get_state(state, "npics")), 1)
        ic.set_state(state, "dtprint", tf / npics if tf > 0 else 1.0)
        ic.set_state(state, "time", 0.0)
        self.state, self.store = state, store
        write_dump(self._out("dump_full.h5"), state, store)
        self.__tolog__("CMD [./execute " + " ".join(self.setup.toArgs()) + "] EXECUTED")

    def CleanRun(self, lib=None):
        """(lib: the engine library for the mti set-ups' density pass; the
        CUDA engine when not given)"""
        out = os.path.join(self.pwd, "output")
        if os.path.isdir(out):
            shutil.rmtree(out)
        os.makedirs(out, exist_ok=True)
        self.SimpleRun(lib)

    def CleanFinalDumps(self):
        for n in ("finaldump", "fulldump"):
            p = self._out(n)
            if os.path.exists(p):
                os.remove(p)

    def MakeAndRun(self, debug=False):
        self.SimpleMake(debug)
        self.CleanRun()

    def ContinueRun(self, lib=None):
        """Restore the dump into the engine and run to tfinish, dumping at
        every output time (main.f90:241-373)."""
        if self.state is None:
            self.ReadDumpHDF(self._out("dump_full.h5"))
        state = np.ascontiguousarray(self.state, dtype=np.float64)
        store = np.ascontiguousarray(self.store, dtype=np.float64)
        tfinish = ic.get_state(state, "tfinish")
        dtout = ic.get_state(state, "dtprint")
        with abi.Engine(state, store, str(self.setup.kernel), precision=self.precision,
                        lib=lib) as e:
            t = ic.get_state(state, "time")
            nxt = t + dtout if dtout > 0 else tfinish
            while True:
                target = min(nxt, tfinish)
                e.run_to(target)
                st = e.get_state()
                st[consts.ec["lastprint"] - 1] += 1
                e.set_param("lastprint", st[consts.ec["lastprint"] - 1])
                self.state, self.store = st, e.get_store()
                write_dump(self._out("dump_full.h5"), self.state, self.store)
                shutil.copyfile(self._out("dump_full.h5"),
                                self._out("dump_%05d.h5" % int(st[consts.ec["lastprint"] - 1])))
                t = st[consts.ec["time"] - 1]
                if t >= tfinish - 1e-15 * max(1.0, abs(tfinish)) or dtout <= 0:
                    break
                nxt = t + dtout
            if tfinish > 0:
                self._write_result(e)
        self.__tolog__("CMD [./execute] EXECUTED")

    def _write_result(self, e):
        """The closing error evaluation of main.f90:374-435: err per real
        particle for the run's initial condition type (sph_errcalc, on the
        device), the line (resolution, realpn, L1, chi = 0, hfac) appended
        to result.info in the working directory, and the L1 line of the
        engine's output in the stdout log.  Where the reference stops with an
        error instead (a type without an error calculator, main.f90:396-397)
        the message goes to the stderr log and no line is written."""
        try:
            _, l1 = e.errcalc()
        except abi.SphError as ex:
            self._log("stderrfile", str(ex))
            return
        st = e.get_state()
        row = [st[consts.ec["resolution"] - 1], st[consts.ec["realpn"] - 1], l1, 0.0,
               st[consts.ec["hfac"] - 1]]
        with open(os.path.join(self.pwd, "result.info"), "a") as f:
            f.write(" " + "  ".join("%.17G" % v for v in row) + "\n")
        self._log("stdoutfile", " # #   L1-error: %20.10f" % l1)
        self.result = row

    def PrintCell(self, file, row, column):
        with open(file.split()[0]) as f:
            lines = f.readlines()
        return lines[min(row, len(lines)) - 1].split()[column - 1]

    # ---- enums (core.py:235-319) -----------------------------------------------
    def ReadConstFile(self):
        for name in ("ec", "es", "ept", "ett", "ebc", "eeq", "esd", "edi", "eqs", "epc",
                     "eif", "ests"):
            setattr(self, name, dict(getattr(consts, name)))
        if self.constf90 and os.path.exists(self.constf90):
            parsed = consts.parse_const_f90(self.constf90)
            for k, v in parsed.items():
                setattr(self, k, v)
        for name in ("ec", "es", "ept", "ett", "ebc", "eeq", "esd", "edi", "eqs", "epc",
                     "eif", "ests"):
            setattr(self, name + "Rev", {v: k for k, v in getattr(self, name).items()})

    # ---- dump editing (core.py:321-470) -------------------------------------------
    def ReadDumpHDF(self, filename):
        self.state, self.store = read_dump(filename)
        self.dumpfile = filename
        for i in range(1, len(self.state) + 1):
            self.setup.__dict__[self.ecRev[i]] = self.state[i - 1]

    def PrintSetup(self):
        for i in self.ecRev:
            e = self.ecRev[i]
            if e in self.setup.__dict__:
                print("\t |", "{0:^15}".format(e), "|", "{0:^40}".format(str(self.setup.__dict__[e])), "|")

    def PrintState(self):
        for i in self.ecRev:
            print("\t |", "{0:^15}".format(self.ecRev[i]), "|", "{0:^40}".format(self.state[i - 1]), "|")

    def idx(self, prop, i):
        return (i, self.es[prop] - 1)

    def ParticlesWithWrongPositions(self):
        s = self.setup
        out = []
        for i in range(int(s.realpn)):
            x, y, z = self.store[i, 0:3]
            if not (s.xmin <= x <= s.xmax and s.ymin <= y <= s.ymax and s.zmin <= z <= s.zmax):
                out.append(i)
        return out

    def PrintPropertyKeys(self):
        print("Properties: " + str(self.es.keys()))

    def GetState(self, key):
        return self.state[self.ec[key] - 1]

    def SetState(self, key, val):
        self.state[self.ec[key] - 1] = val

    def BackupOutput(self, name):
        shutil.copytree(os.path.join(self.pwd, "output"), os.path.join(self.pwd, name),
                        dirs_exist_ok=True)

    def BackupDump(self, file):
        p = os.path.join(self.pwd, file)
        if os.path.exists(p):
            shutil.copyfile(p, p + ".bck")

    def AddParticles(self, dim, type, method):
        """Periodic copies of the rows within the border strip of axis `dim`
        (core.py:383-416)."""
        iprop = self.es["r" + dim] - 1
        itype = self.es["type"] - 1
        bs = self.setup.bordsize
        lo = self.setup.__dict__[dim + "min"]
        hi = self.setup.__dict__[dim + "max"]
        dr = (hi - lo) / self.setup.resolution
        bmin, bmax = lo + bs, hi - bs
        new = []
        for i in range(int(self.setup.realpn)):
            oldr = self.store[i, iprop]
            newr = oldr
            if oldr < bmin:
                newr = hi + oldr - lo
            if oldr > bmax:
                newr = lo + oldr - hi
            if abs(oldr - newr) > dr * 1e-3:
                p = self.store[i].copy()
                p[itype] = self.ept[type]
                p[iprop] = newr
                new.append(p)
        if new:
            self.store = np.concatenate([self.store, np.array(new)], axis=0)
        if type in ("fixed", "fixedreal"):
            self.setup.fixedpn = len(new)

    def CalcUniformMass(self, rho):
        lx = ly = lz = 1.0
        if self.setup.dim > 0:
            lx = abs(self.setup.xmax - self.setup.xmin)
        if self.setup.dim > 1:
            ly = abs(self.setup.ymax - self.setup.ymin)
        if self.setup.dim > 2:
            lz = abs(self.setup.zmax - self.setup.zmin)
        return lx * ly * lz * rho / self.setup.realpn

    def CopyContext(self):
        c = copy.copy(self)
        c.setup = copy.deepcopy(self.setup)
        c.store = None if self.store is None else self.store.copy()
        c.state = None if self.state is None else self.state.copy()
        return c

    def ModifyParticlesProperties(self, condition=(lambda rx: True,), conditionarg=("rx",),
                                  properties=("rx",), value=(lambda rx: 1.0,),
                                  valuearg=("rx",)):
        n = int(self.setup.realpn) + int(self.setup.fixedpn)
        new = self.store.copy()
        for i in range(n):
            for j, prop in enumerate(properties):
                arg = valuearg[0] if len(valuearg) == 1 else valuearg[j]
                new[i, self.es[prop] - 1] = value[j](self.store[i, self.es[arg] - 1])
        self.store = new

    def Apply(self):
        for i in self.ecRev:
            e = self.ecRev[i]
            if e in self.setup.__dict__:
                v = self.setup.__dict__[e]
                try:
                    self.state[i - 1] = float(v)
                except (TypeError, ValueError):
                    pass
        self.state[self.ec["realpn"] - 1] = float(self.setup.realpn)
        self.state[self.ec["fixedpn"] - 1] = float(self.setup.fixedpn)
        write_dump(getattr(self, "dumpfile", self._out("dump_full.h5")), self.state, self.store)
