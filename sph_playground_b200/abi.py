"""ctypes binding of the C-ABI declared in include/sph_abi.h.

``Engine`` wraps one ``sph_handle``.  The same binding loads the CUDA engine
(``sph_playground_b200/_lib/libsph.so``) and, for tests and baselines only,
the CPU oracle library, which exports the same symbols.
"""
import ctypes
import os

import numpy as np

from . import consts

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libsph.so")

# status codes (include/sph_abi.h)
STATUS = {
    0: "SPH_OK", 1: "SPH_ERR_ARG", 2: "SPH_ERR_CUDA", 3: "SPH_ERR_Q_NAN",
    4: "SPH_ERR_Q_NEG", 5: "SPH_ERR_H_NEG", 6: "SPH_ERR_NEIB_OVERFLOW",
    7: "SPH_ERR_IC_DENSITY", 8: "SPH_ERR_IC_CSOUND", 9: "SPH_ERR_IC_H",
    10: "SPH_ERR_IC_PRESSURE", 11: "SPH_ERR_IC_ENERGY",
    12: "SPH_ERR_IC_MUZERO", 13: "SPH_ERR_IC_DIFFCOND",
    14: "SPH_ERR_UNSUPPORTED", 15: "SPH_ERR_FLD_ANISO", 16: "SPH_ERR_DDW",
    17: "SPH_ERR_PROCESS", 18: "SPH_ERR_GRID", 19: "SPH_ERR_OOM",
    20: "SPH_ERR_TIMEOUT", 21: "SPH_ERR_STATE", 22: "SPH_ERR_RAD_NEGATIVE",
}

PREC_FP64 = 0
PREC_FP32_COMP = 1

P_AV_ALPHA = 50
P_AV_BETA = 51
P_NEWTON_TOL = 52
P_NEWTON_MAXITER = 53
P_FULL_TENSOR = 54
P_NEIB_CAP_CHECK = 55
P_CELL_FACTOR = 56
P_REORDER_EVERY = 57
P_TIMING = 58
P_NEIB_CAP = 59
P_LANES_SEARCH = 60
P_LANES_PAIR = 61
P_FIXED_DT = 62
P_GRAPH = 63
P_SEARCH_STAGED = 64
P_SKIN = 65

COUNTERS = ["iterates", "steps", "neib_pairs", "c1_pairs", "c1_sweeps",
            "c2_pairs", "ghosts", "candidates", "centres",
            "c1_centre_sweeps", "launches", "neib_max", "searches",
            "exact_tests", "allocs", "graph_steps", "graph_redos",
            "skin_builds", "skin_reuses", "skin_dirty", "skin_kept",
            "skin_relayouts"]
TIMERS = ["predict", "ghosts", "sort", "neighbours", "circuit1", "circuit2",
          "correct", "timestep", "sts", "step", "pack"]

# every symbol include/sph_abi.h declares
ABI_SYMBOLS = [
    "sph_create", "sph_set_param", "sph_get_param", "sph_set_store",
    "sph_iterate", "sph_density", "sph_step", "sph_run_to", "sph_get_store",
    "sph_get_state", "sph_get_neighbours", "sph_get_neighbour_digest", "sph_get_counters",
    "sph_reset_counters", "sph_get_timers", "sph_last_error", "sph_destroy",
    "sph_batch_create", "sph_batch_step", "sph_batch_run_to", "sph_batch_status",
    "sph_batch_destroy", "sph_errcalc", "sph_timestep", "sph_predict", "sph_forces",
    "sph_correct", "sph_get_columns", "sph_set_columns",
]


class SphError(RuntimeError):
    """An engine call returned a non-zero status (a reference abort site)."""

    def __init__(self, code, message):
        self.code = code
        self.status = STATUS.get(code, str(code))
        super().__init__(f"{self.status}: {message}")


_libs = {}


def load(path=None):
    """Load (once) and type the library at `path` (default: the CUDA engine)."""
    path = os.path.abspath(path or LIB_PATH)
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is not built; run `python __graft_entry__.py build` or "
            "`make -C sph_playground_b200/csrc`")
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    P = ctypes.POINTER
    d, i64, c_int = ctypes.c_double, ctypes.c_int64, ctypes.c_int
    vp = ctypes.c_void_p
    lib.sph_create.argtypes = [P(d), P(d), i64, c_int, c_int, P(vp)]
    lib.sph_set_param.argtypes = [vp, c_int, d]
    lib.sph_get_param.argtypes = [vp, c_int, P(d)]
    lib.sph_set_store.argtypes = [vp, P(d), i64]
    lib.sph_iterate.argtypes = [vp]
    lib.sph_density.argtypes = [vp]
    lib.sph_step.argtypes = [vp, c_int]
    lib.sph_run_to.argtypes = [vp, d]
    lib.sph_get_store.argtypes = [vp, P(d), i64]
    lib.sph_get_state.argtypes = [vp, P(d)]
    lib.sph_get_neighbours.argtypes = [vp, P(i64), P(i64), i64]
    lib.sph_get_neighbour_digest.argtypes = [vp, P(ctypes.c_uint64), i64]
    lib.sph_get_counters.argtypes = [vp, P(i64), c_int]
    lib.sph_reset_counters.argtypes = [vp]
    lib.sph_get_timers.argtypes = [vp, P(d), c_int]
    lib.sph_last_error.argtypes = []
    lib.sph_last_error.restype = ctypes.c_char_p
    lib.sph_destroy.argtypes = [vp]
    lib.sph_destroy.restype = None
    lib.sph_batch_create.argtypes = [c_int, P(vp), P(vp)]
    lib.sph_batch_step.argtypes = [vp, c_int]
    lib.sph_batch_run_to.argtypes = [vp, d]
    lib.sph_batch_status.argtypes = [vp, P(c_int), c_int]
    lib.sph_batch_destroy.argtypes = [vp]
    lib.sph_batch_destroy.restype = None
    lib.sph_errcalc.argtypes = [vp, P(d), i64, P(d)]
    lib.sph_timestep.argtypes = [vp, P(d)]
    lib.sph_predict.argtypes = [vp, d]
    lib.sph_forces.argtypes = [vp]
    lib.sph_correct.argtypes = [vp, d]
    lib.sph_get_columns.argtypes = [vp, P(c_int), c_int, vp]
    lib.sph_set_columns.argtypes = [vp, P(c_int), c_int, vp]
    if hasattr(lib, "sph_adjoint_forward"):  # the CUDA engine only
        lib.sph_adjoint_forward.argtypes = [vp, c_int, c_int]
        lib.sph_adjoint_forward.restype = c_int
        lib.sph_adjoint_backward.argtypes = [vp, P(d), P(d), P(d), P(d), P(d), P(d), P(d)]
        lib.sph_adjoint_backward.restype = c_int
        lib.sph_adjoint_backward_diffusion.argtypes = [vp, P(d), P(d), P(d)]
        lib.sph_adjoint_backward_diffusion.restype = c_int
    for name in ABI_SYMBOLS:
        if name not in ("sph_last_error", "sph_destroy", "sph_batch_destroy"):
            getattr(lib, name).restype = c_int
    _libs[path] = lib
    return lib


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


class Engine:
    """One engine instance: owns a handle, takes and returns numpy arrays."""

    def __init__(self, state, store, kernel="m6", precision=PREC_FP64,
                 lib=None):
        self.lib = lib if lib is not None else load()
        state = np.ascontiguousarray(state, dtype=np.float64)
        store = np.ascontiguousarray(store, dtype=np.float64)
        if state.shape != (consts.EC_TOTAL,):
            raise ValueError("state must have 49 entries")
        if store.ndim != 2 or store.shape[1] != consts.ES_TOTAL:
            raise ValueError("store must be (N, 32)")
        kid = consts.KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
        self.n_rows = store.shape[0]
        self.n_real = int(state[consts.ec["realpn"] - 1])
        h = ctypes.c_void_p()
        self._check(self.lib.sph_create(_dptr(state), _dptr(store),
                                        self.n_rows, kid, int(precision),
                                        ctypes.byref(h)))
        self.h = h

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.sph_last_error()
            raise SphError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None):
            self.lib.sph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- parameters ---------------------------------------------------------
    def set_param(self, index, value):
        if isinstance(index, str):
            index = consts.ec[index]
        self._check(self.lib.sph_set_param(self.h, int(index), float(value)))

    def get_param(self, index):
        if isinstance(index, str):
            index = consts.ec[index]
        v = ctypes.c_double()
        self._check(self.lib.sph_get_param(self.h, int(index), ctypes.byref(v)))
        return v.value

    # ---- passes -------------------------------------------------------------
    def iterate(self):
        self._check(self.lib.sph_iterate(self.h))

    def density(self):
        self._check(self.lib.sph_density(self.h))

    def step(self, n=1):
        self._check(self.lib.sph_step(self.h, int(n)))

    def run_to(self, tfinish):
        self._check(self.lib.sph_run_to(self.h, float(tfinish)))

    # ---- data ----------------------------------------------------------------
    def set_store(self, store):
        store = np.ascontiguousarray(store, dtype=np.float64)
        self._check(self.lib.sph_set_store(self.h, _dptr(store), store.shape[0]))

    def get_store(self, out=None):
        if out is None:
            out = np.empty((self.n_rows, consts.ES_TOTAL), dtype=np.float64)
        self._check(self.lib.sph_get_store(self.h, _dptr(out), out.shape[0]))
        return out

    def get_state(self):
        out = np.empty(consts.EC_TOTAL, dtype=np.float64)
        self._check(self.lib.sph_get_state(self.h, _dptr(out)))
        return out

    # ---- adjoint (CUDA engine only) -----------------------------------------
    def adjoint_forward(self, nsteps, every):
        """nsteps fixed-dt steps (P_FIXED_DT) with a table copy every `every`
        steps, for adjoint_backward."""
        self._check(self.lib.sph_adjoint_forward(self.h, int(nsteps), int(every)))

    def adjoint_backward(self, dl_dv=None, dl_du=None, dl_dr=None):
        """Gradients at the initial state of the last adjoint_forward run from
        dL/dv, dL/du, dL/dr at its final state (caller row order): dict with
        g_r0 (n x 3), g_v0 (n x 3), g_u0 (n), g_par (d/d alpha, d/d beta)."""
        n = self.n_rows

        def inp(a, shape):
            if a is None:
                return None
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))
            return a
        iv, iu, ir = inp(dl_dv, (n, 3)), inp(dl_du, (n,)), inp(dl_dr, (n, 3))
        out = {"g_r0": np.zeros((n, 3)), "g_v0": np.zeros((n, 3)), "g_u0": np.zeros(n),
               "g_par": np.zeros(2)}
        nul = ctypes.POINTER(ctypes.c_double)()
        ptr = lambda a: _dptr(a) if a is not None else nul  # noqa: E731
        self._check(self.lib.sph_adjoint_backward(
            self.h, ptr(iv), ptr(iu), ptr(ir), _dptr(out["g_r0"]), _dptr(out["g_v0"]),
            _dptr(out["g_u0"]), _dptr(out["g_par"])))
        return out

    def errcalc(self):
        """(err per real particle in original row order, L1): the closing
        error evaluation of main.f90:374-402 for the run's initial
        condition type at the handle's time."""
        err = np.zeros(self.n_real, dtype=np.float64)
        l1 = np.zeros(1, dtype=np.float64)
        self._check(self.lib.sph_errcalc(self.h, _dptr(err), err.shape[0], _dptr(l1)))
        return err, float(l1[0])

    def adjoint_backward_diffusion(self, dl_dT):
        """(dL/dT0 per real particle, dL/d difcond) after adjoint_forward on
        a diffusion run, for dL/dT(T) per real particle (original order)."""
        g = np.zeros(self.n_real, dtype=np.float64)
        gd = np.zeros(1, dtype=np.float64)
        lt = np.ascontiguousarray(dl_dT, dtype=np.float64)
        assert lt.shape == (self.n_real,)
        self._check(self.lib.sph_adjoint_backward_diffusion(self.h, _dptr(lt), _dptr(g), _dptr(gd)))
        return g, float(gd[0])

    def get_neighbours(self):
        """(offsets[n_real+1], pairs) with pairs = (rj << 5) | image code."""
        off = np.zeros(self.n_real + 1, dtype=np.int64)
        rc = self.lib.sph_get_neighbours(self.h, _iptr(off), None, 0)
        if rc not in (0, 1):
            self._check(rc)
        pairs = np.empty(max(int(off[-1]), 1), dtype=np.int64)
        self._check(self.lib.sph_get_neighbours(self.h, _iptr(off), _iptr(pairs),
                                                pairs.shape[0]))
        return off, pairs[: int(off[-1])]

    def get_neighbour_digest(self):
        """(count, digest) per real row in original order: the neighbour
        count and the order-independent 64-bit sum of a mix of each entry of
        get_neighbours' encoding; equal digests mean equal sets (up to a
        2^-64 collision per row) without copying the pair arrays."""
        out = np.zeros((self.n_real, 2), dtype=np.uint64)
        self._check(self.lib.sph_get_neighbour_digest(
            self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), self.n_real))
        return out[:, 0].astype(np.int64), out[:, 1]

    # ---- one leapfrog step in parts (sph_timestep .. sph_correct) ----------
    def timestep(self):
        """dt over this handle's real rows (before clipping to tfinish)."""
        v = ctypes.c_double()
        self._check(self.lib.sph_timestep(self.h, ctypes.byref(v)))
        return v.value

    def predict(self, dt):
        self._check(self.lib.sph_predict(self.h, float(dt)))

    def forces(self):
        self._check(self.lib.sph_forces(self.h))

    def correct(self, dt):
        self._check(self.lib.sph_correct(self.h, float(dt)))

    @staticmethod
    def _fields(names):
        idx = [consts.es[n] if isinstance(n, str) else int(n) for n in names]
        return (ctypes.c_int * len(idx))(*idx), len(idx)

    def get_columns(self, names, out=None):
        """(len(names), n_rows) array of the named fields in caller row
        order; `out` may be a numpy array or a device pointer (int)."""
        f, nf = self._fields(names)
        if out is None:
            out = np.empty((nf, self.n_rows), dtype=np.float64)
        ptr = out if isinstance(out, int) else out.ctypes.data
        self._check(self.lib.sph_get_columns(self.h, f, nf, ctypes.c_void_p(ptr)))
        return out

    def set_columns(self, names, values):
        """Write the named fields (len(names), n_rows) in caller row order;
        `values` may be a numpy array or a device pointer (int)."""
        f, nf = self._fields(names)
        if isinstance(values, int):
            ptr = values
        else:
            values = np.ascontiguousarray(values, dtype=np.float64)
            assert values.shape == (nf, self.n_rows)
            ptr = values.ctypes.data
        self._check(self.lib.sph_set_columns(self.h, f, nf, ctypes.c_void_p(ptr)))

    def counters(self):
        out = np.zeros(len(COUNTERS), dtype=np.int64)
        self._check(self.lib.sph_get_counters(self.h, _iptr(out), len(COUNTERS)))
        return dict(zip(COUNTERS, (int(x) for x in out)))

    def reset_counters(self):
        self._check(self.lib.sph_reset_counters(self.h))

    def timers(self):
        out = np.zeros(len(TIMERS), dtype=np.float64)
        self._check(self.lib.sph_get_timers(self.h, _dptr(out), len(TIMERS)))
        return dict(zip(TIMERS, (float(x) for x in out)))


class Batch:
    """Several Engine instances stepped together (sph_batch_*): every
    instance runs its own time loop, the instances overlap on the device.
    The engines stay usable after the batch is closed."""

    def __init__(self, engines):
        self.engines = list(engines)
        if not self.engines:
            raise ValueError("empty batch")
        self.lib = self.engines[0].lib
        if any(e.lib is not self.lib for e in self.engines):
            raise ValueError("all engines of a batch must use the same library")
        arr = (ctypes.c_void_p * len(self.engines))(*[e.h.value for e in self.engines])
        b = ctypes.c_void_p()
        self._check(self.lib.sph_batch_create(len(self.engines), arr, ctypes.byref(b)))
        self.b = b

    def _check(self, rc):
        if rc != 0:
            raise SphError(rc, self.lib.sph_last_error().decode(errors="replace"))

    def step(self, nsteps=1):
        self._check(self.lib.sph_batch_step(self.b, int(nsteps)))

    def run_to(self, tfinish):
        self._check(self.lib.sph_batch_run_to(self.b, float(tfinish)))

    def status(self):
        out = (ctypes.c_int * len(self.engines))()
        self._check(self.lib.sph_batch_status(self.b, out, len(self.engines)))
        return list(out)

    def close(self):
        if getattr(self, "b", None) is not None and self.b.value:
            self.lib.sph_batch_destroy(self.b)
            self.b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
