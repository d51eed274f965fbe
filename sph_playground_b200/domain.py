"""One SPH problem on several GPUs: a particle decomposition of the leapfrog
step over torch.distributed (NCCL between GPUs, gloo on the CPU).

Every rank keeps the whole particle table on its own device.  Rank r owns a
contiguous range of the particles in Morton order of their initial
positions; in its table the owned particles are the real rows (the centres
of its neighbour search, circuit1 and circuit2) and all others are fixedreal
rows (neighbours that are integrated but are not centres,
main.f90:181-184).  The pair work of a step is therefore split N ways, while
the images, the sort and the integration of all rows are repeated on every
rank.  One step (main.f90:241-373, leapfrog):

  dt      = min over ranks of each rank's timestep over its owned rows
            (timestep.f90:40-166), clipped to tfinish and the output times
            as main.f90:273-299 does;
  predict (all rows, from the same values on every rank);
  density (owned centres: images, search, circuit1, EOS)
            -> all-gather of rho, h, Omega, P, c of the owned rows;
  forces  (owned centres: circuit2)
            -> all-gather of a, du/dt, dh/dt of the owned rows;
  correct (all rows).

Each rank thus holds the same state after every step, and every owned
centre sees the same neighbours as in a single-domain run; the results equal
the single-domain run's up to the summation order inside a neighbour list
(the rows of a rank's table are ordered differently).  Supported: the
hydro / MHD equations without STS or radiation exchange (the split step of
include/sph_abi.h)."""
import numpy as np

from . import abi, consts

# fields each exchange carries (the fields the next pass reads from the
# rows it does not compute)
AFTER_DENSITY = ("den", "h", "om", "p", "c")
AFTER_FORCES = ("ax", "ay", "az", "du", "dh", "dbx", "dby", "dbz")
# equations whose circuit1 reads its neighbours' Newton iterates (the
# temperature gradient of the diffusion / flux-limited paths) or whose step
# has more stages (STS, radiation exchange): not decomposed by this driver
_EQS_EXCLUDED = {consts.EQUATIONS[k] for k in ("diffusion", "hydi", "kd2", "hyrad")}
_EPS = np.finfo(np.float64).eps


def morton_owners(pos, dim, nranks, bits=10):
    """Owner rank of every particle: the particles sorted by the Morton key
    of their positions quantised to 2^bits cells per axis over the bounding
    box, cut into nranks contiguous ranges of (nearly) equal counts."""
    n = pos.shape[0]
    lo, hi = pos[:, :dim].min(axis=0), pos[:, :dim].max(axis=0)
    span = np.where(hi > lo, hi - lo, 1.0)
    q = np.clip(((pos[:, :dim] - lo) / span * (1 << bits)).astype(np.int64), 0, (1 << bits) - 1)
    key = np.zeros(n, dtype=np.int64)
    for b in range(bits):
        for k in range(dim):
            key |= ((q[:, k] >> b) & 1) << (b * dim + k)
    order = np.argsort(key, kind="stable")
    owner = np.empty(n, dtype=np.int64)
    for r, part in enumerate(np.array_split(order, nranks)):
        owner[part] = r
    return owner


class SplitRun:
    """The leapfrog time loop of one handle driven through the split-step
    entry points (sph_timestep .. sph_correct), with the exchange hooks a
    decomposed run fills in.  With no exchange it is one domain's run, the
    same steps sph_run_to takes."""

    def __init__(self, engine):
        self.e = engine
        st = engine.get_state()
        self.t = float(st[consts.ec["time"] - 1])
        self.dtout = float(st[consts.ec["dtprint"] - 1])
        self.ltout = 0.0
        if self.dtout > 0:
            while self.ltout < self.t:
                self.ltout += self.dtout
        self.stopped = False
        self.steps = 0

    # hooks: a decomposed run exchanges fields here
    def after_density(self):
        pass

    def after_forces(self):
        pass

    def reduce_dt(self, dt):
        return dt

    def start(self):
        """The start-up iterate before the time loop (main.f90:241)."""
        self.e.density()
        self.after_density()
        self.e.forces()
        self.after_forces()

    def step(self, tfinish):
        """One pass of the time loop; False once the loop condition fails."""
        if not (self.t < tfinish + _EPS and not self.stopped):
            return False
        dt = self.reduce_dt(self.e.timestep())
        t = self.t
        if t + dt > tfinish:
            dt = tfinish - t
            self.stopped = True
        if self.dtout > 0:
            if t >= self.ltout:
                while self.ltout <= t:
                    self.ltout += self.dtout
            if t + dt > self.ltout:
                if self.dtout < dt:
                    self.ltout = self.ltout - self.dtout + dt
                else:
                    dt = self.ltout - t
        self.e.predict(dt)
        self.e.density()
        self.after_density()
        self.e.forces()
        self.after_forces()
        self.e.correct(dt)
        self.t = t + dt
        self.steps += 1
        return True

    def run_to(self, tfinish, max_steps=None):
        while self.step(tfinish):
            if max_steps is not None and self.steps >= max_steps:
                break
        return self.t


class DecomposedRun(SplitRun):
    """One problem over the ranks of the current torch.distributed group
    (a particle decomposition: see the module docstring).  `state` and
    `store` are the whole problem, the same on every rank; `device` is the
    torch device of the exchange buffers (a CUDA device under NCCL, the CPU
    under gloo)."""

    def __init__(self, state, store, kernel="m6", precision=abi.PREC_FP64, lib=None,
                 device="cpu"):
        import torch.distributed as dist
        self.rank, self.size = dist.get_rank(), dist.get_world_size()
        self.device = device
        state = np.array(state, dtype=np.float64)
        store = np.array(store, dtype=np.float64)
        n = store.shape[0]
        if int(state[consts.ec["fixedpn"] - 1]) > 0:
            raise ValueError("a decomposed run takes real particles only")
        flag = lambda k: int(state[consts.ec[k] - 1]) == 1  # noqa: E731
        if (int(state[consts.ec["eqs"] - 1]) in _EQS_EXCLUDED or flag("eqondiff") or
                flag("eqonfluxlim") or flag("eqonsts") or flag("eqonradexch")):
            raise ValueError("a decomposed run takes the hydro / MHD leapfrog step only")
        dim = int(state[consts.ec["dim"] - 1])
        self.owner = morton_owners(store[:, 0:3], dim, self.size)
        self.owned = [np.nonzero(self.owner == r)[0] for r in range(self.size)]
        own = self.owned[self.rank]
        other = np.nonzero(self.owner != self.rank)[0]
        # local row i holds global particle order[i]: owned rows first
        self.order = np.concatenate([own, other])
        self.n_own = own.shape[0]
        local = store[self.order].copy()
        local[self.n_own:, consts.es["type"] - 1] = consts.ept["fixedreal"]
        st = state.copy()
        st[consts.ec["realpn"] - 1] = self.n_own
        st[consts.ec["fixedpn"] - 1] = n - self.n_own
        self.n = n
        super().__init__(abi.Engine(st, local, kernel, precision=precision, lib=lib))
        # position of each global particle in this rank's table
        self.local_of = np.empty(n, dtype=np.int64)
        self.local_of[self.order] = np.arange(n)
        self.max_own = max(o.shape[0] for o in self.owned)

    def _exchange(self, fields):
        """All-gather the named fields of every rank's owned rows and write
        them into this rank's non-owned rows.  On a CUDA device the columns
        go from the engine's table to a device buffer, through the
        collective and back without touching the host."""
        import torch
        import torch.distributed as dist
        nf = len(fields)
        if str(self.device) == "cpu":
            vals = self.e.get_columns(fields)  # (nf, n) in local order
            mine = torch.zeros((nf, self.max_own), dtype=torch.float64)
            mine[:, :self.n_own] = torch.from_numpy(vals[:, :self.n_own])
            parts = [torch.empty_like(mine) for _ in range(self.size)]
            dist.all_gather(parts, mine)
            for r, part in enumerate(parts):
                if r != self.rank:
                    g = self.owned[r]
                    vals[:, self.local_of[g]] = part[:, :g.shape[0]].numpy()
            self.e.set_columns(fields, vals)
            return
        if getattr(self, "_dev_idx", None) is None:
            self._dev_idx = [torch.as_tensor(self.local_of[g], device=self.device)
                             for g in self.owned]
        buf = torch.empty((nf, self.n), dtype=torch.float64, device=self.device)
        self.e.get_columns(fields, out=buf.data_ptr())  # the engine syncs its stream
        mine = torch.zeros((nf, self.max_own), dtype=torch.float64, device=self.device)
        mine[:, :self.n_own] = buf[:, :self.n_own]
        parts = [torch.empty_like(mine) for _ in range(self.size)]
        dist.all_gather(parts, mine)
        for r, part in enumerate(parts):
            if r != self.rank:
                buf[:, self._dev_idx[r]] = part[:, :self.owned[r].shape[0]]
        torch.cuda.current_stream(self.device).synchronize()
        self.e.set_columns(fields, buf.data_ptr())

    def after_density(self):
        self._exchange(AFTER_DENSITY)

    def after_forces(self):
        self._exchange(AFTER_FORCES)

    def reduce_dt(self, dt):
        import torch
        import torch.distributed as dist
        v = torch.tensor([dt], dtype=torch.float64, device=self.device)
        dist.all_reduce(v, op=dist.ReduceOp.MIN)
        return float(v.item())

    def global_store(self):
        """The whole table in the caller's original row order (every rank
        holds all rows; owned rows are returned as reals again)."""
        local = self.e.get_store()
        out = local[self.local_of].copy()
        out[:, consts.es["type"] - 1] = consts.ept["real"]
        return out

    def close(self):
        self.e.close()
