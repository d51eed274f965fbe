#!/usr/bin/env python
"""SPH step throughput on B200: particle-steps/s of the two-loop SPH step.

Workload: Sedov blast, 128^3 = 2,097,152 lattice particles in the unit
periodic box, M6 kernel, hfac 1.2, alpha = 1, beta = 2, gamma = 5/3.  One
step is the full leapfrog step of the reference's time loop: timestep
reductions, predictor, periodic images, neighbour lists, circuit1 (Newton
h-iteration + EOS), circuit2 (hydro + AV + conductivity + dh/dt) and
corrector.  The headline runs the FP32-compensated pair path; the plain FP64
path is timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (launched under torchrun) every rank runs an independent replica
of the workload on its own GPU (the reference has no domain decomposition):
`value` is the sum over ranks, timed as the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from sph_playground_b200 import abi  # noqa: E402  (ctypes only; no CUDA at import)

METRIC = "particle-steps/s, 2.1M 3D: FP32-comp vs FP64 on B200 at rho err<=1e-6"
UNIT = "particle-steps/s"
# per-pair algorithmic FLOP weights (circuit1 per pair per Newton sweep,
# circuit2 per pair for hydro + AV + conductivity + dh/dt), counted from the
# reference formulas with sqrt/div each as one FLOP
F1_C1 = 50.0
F2_C2 = 150.0
# DRAM bytes per in-support pair of the FP32-comp circuit2 launch:
# dram__bytes_read.sum + dram__bytes_write.sum = 849.04 MB + 73.09 MB over
# 157.49M pairs of an ncu capture of k_c2 on the Sedov 96^3 step (FP32-comp, 4
# lanes per centre, cell edge 0.4 krad h_min) (the
# neighbour index, 4 B, plus the gathered pair data that misses L2); the
# traffic scales with the pairs a launch processes
C2_DRAM_BYTES_PER_PAIR = (849.04e6 + 73.09e6) / 157.49e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128, help="lattice particles per axis")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the default launch shapes instead of autotuning them")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint cost / gradient check (2D shear 256^2)")
    ap.add_argument("--no-density", action="store_true",
                    help="skip the density-only pass (3D perturbed lattice 128^3, FP32 vs FP64)")
    ap.add_argument("--no-errors", action="store_true",
                    help="skip the FP32-vs-FP64 error check (profiling runs)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-n", type=int, default=64, help="lattice per axis of the CPU sample")
    ap.add_argument("--param", action="append", default=[],
                    help="engine parameter NAME=VALUE (abi.P_* name or slot), for both arms")
    return ap.parse_args()


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.path = os.path.join(os.environ.get("SPH_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                   "-lms", "20"]
            if self.uuid:
                cmd += ["-i", self.uuid]
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(cmd, stdout=self.f, stderr=subprocess.DEVNULL)
            # the timed region starts once the sampler is producing lines
            t0 = time.time()
            while time.time() - t0 < 10 and self.proc.poll() is None:
                if os.path.getsize(self.path) > 0:
                    break
                time.sleep(0.02)
            self.skip = sum(1 for _ in open(self.path))
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = [[c.strip() for c in r] for r in rows[getattr(self, "skip", 0):] if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "samples": len(rows), "reasons": reasons}


def measure_peak():
    import ctypes
    path = os.path.join(ROOT, "sph_playground_b200", "_lib", "libsph_peak.so")
    lib = ctypes.CDLL(path)
    lib.sph_peak_flops.restype = ctypes.c_double
    lib.sph_peak_flops.argtypes = [ctypes.c_int, ctypes.c_int]
    fp32 = max(lib.sph_peak_flops(0, 20) for _ in range(3))
    fp64 = max(lib.sph_peak_flops(1, 10) for _ in range(2))
    return fp32, fp64


def cpu_baseline(n):
    """The oracle (CPU FP64 OpenMP restatement) on a bounded sample: one
    leapfrog step of the same Sedov set-up at n^3 after its start-up iterate."""
    from sph_playground_b200 import ic
    lib = abi.load(os.path.join(ROOT, "oracle", "liboracle.so"))
    st, store = ic.sedov3d(n=n)
    e = abi.Engine(st, store, "m6", lib=lib)
    e.step(0)
    t0 = time.perf_counter()
    e.step(1)
    dt = time.perf_counter() - t0
    e.close()
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": store.shape[0] / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"sedov3d {n}^3 ({store.shape[0]} particles), 1 leapfrog step after the "
                      f"start-up iterate, CPU oracle (FP64, OpenMP {cores} threads)"}


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from sph_playground_b200 import ic
    lib = abi.load(os.path.join(ROOT, "oracle", "liboracle.so"))
    n = args.cpu_n
    st, store = ic.sedov3d(n=n)
    e = abi.Engine(st, store, "m6", lib=lib)
    e.step(0)
    for _ in range(args.warmup):
        e.step(1)
    t0 = time.perf_counter()
    e.step(args.steps)
    dt = time.perf_counter() - t0
    e.close()
    N = store.shape[0]
    value = N * args.steps / dt
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": f"sedov3d {n}^3 ({N} particles) sample of the 128^3 Sedov step, "
                               "M6 hfac 1.2, full leapfrog step",
                   "particles": N, "note": "reference Fortran not compiled (no gfortran/HDF5 "
                   "in the image); the CPU oracle restatement of its path is timed instead"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"sedov3d {n}^3, {args.steps} steps after {args.warmup} warm-up"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def adjoint_block(lib, n=256, n_ref=64, nsteps=200, every=20, dt=5e-4):
    """The adjoint workload: 2D periodic shear flow (n^2 particles, M6,
    alpha = 1, beta = 2), nsteps fixed-dt leapfrog steps with a checkpoint
    every `every` steps; forward and backward timed on the host around the
    synchronous C-ABI calls.  Also the FP32-comp gradient against the FP64
    gradient at n_ref^2."""
    from sph_playground_b200 import ic
    V = [abi.consts.es["vx"] - 1, abi.consts.es["vy"] - 1, abi.consts.es["vz"] - 1]

    def grads(nn, prec, steps):
        st, store = ic.shear2d(n=nn)
        target = store[:, V] * 1.2
        target[:, 2] = 0.0
        e = abi.Engine(st, store, "m6", precision=prec, lib=lib)
        e.set_param(abi.P_FIXED_DT, dt)
        t0 = time.perf_counter()
        e.adjoint_forward(steps, every)
        t1 = time.perf_counter()
        vT = e.get_store()[:, V]
        t2 = time.perf_counter()
        g = e.adjoint_backward(dl_dv=2.0 * (vT - target))
        t3 = time.perf_counter()
        e.close()
        return g, (t1 - t0) * 1e3 / steps, (t3 - t2) * 1e3 / steps

    grads(64, abi.PREC_FP64, 4)  # warm-up
    _, fwd, bwd = grads(n, abi.PREC_FP64, nsteps)
    g64, _, _ = grads(n_ref, abi.PREC_FP64, nsteps)
    g32, _, _ = grads(n_ref, abi.PREC_FP32_COMP, nsteps)
    rel = float(np.linalg.norm(g32["g_v0"] - g64["g_v0"]) / np.linalg.norm(g64["g_v0"]))
    return {"workload": f"shear2d {n}^2 ({n * n} particles), M6, alpha 1, beta 2, {nsteps} steps "
                        f"of dt {dt}, checkpoint every {every}, FP64",
            "forward_ms_per_step": fwd, "backward_ms_per_step": bwd,
            "backward_over_forward": bwd / fwd,
            "grad_v0_fp32_vs_fp64_rel": rel,
            "grad_reference": f"FP64 adjoint gradient at {n_ref}^2",
            "timing": "host clock around synchronous C-ABI calls"}


def density_block(lib, shapes, n=128, tol=1e-6, reps=5):
    """The density-only workload: one density + Newton-h pass over a 3D
    periodic n^3 lattice perturbed by uniform(-0.1, 0.1) dx (seed 2), M6,
    hfac 1.2, Newton tolerance `tol`; FP32-comp against FP64: device time of
    the pass (CUDA events of the neighbour and circuit1 phases, averaged
    over `reps` passes after one warm-up) and the per-particle relative
    error of rho and h."""
    from sph_playground_b200 import ic
    st, store = ic.density3d(n=n, seed=2)
    out, res = {}, {}
    for prec, name in ((abi.PREC_FP64, "fp64"), (abi.PREC_FP32_COMP, "fp32_comp")):
        e = abi.Engine(st, store, "m6", precision=prec, lib=lib)
        for k, v in shapes.get(prec, {}).items():  # the launch shapes of the step arms
            e.set_param(getattr(abi, k), float(v))
        e.set_param(abi.P_NEWTON_TOL, tol)
        e.density()
        res[name] = e.get_store()
        e.reset_counters()
        e.set_param(abi.P_TIMING, 1)
        for _ in range(reps):
            e.set_store(store)
            e.density()
        t = e.timers()
        e.close()
        ms = sum(t[k] for k in ("ghosts", "sort", "neighbours", "pack", "circuit1")) / reps
        out[name] = {"ms_per_pass": ms, "particle_passes_per_s": store.shape[0] / (ms * 1e-3)}
    C = {k: v - 1 for k, v in abi.consts.es.items()}
    for f in ("den", "h"):
        rel = np.abs(res["fp32_comp"][:, C[f]] - res["fp64"][:, C[f]]) / np.abs(res["fp64"][:, C[f]])
        out[("rho" if f == "den" else f) + "_rel_err"] = {"max": float(rel.max()),
                                                        "p99.9": float(np.quantile(rel, 0.999))}
    out["fp32_over_fp64_speed"] = out["fp64"]["ms_per_pass"] / out["fp32_comp"]["ms_per_pass"]
    out["workload"] = (f"density3d {n}^3 ({store.shape[0]} particles), perturbed lattice, M6 hfac 1.2, "
                       f"Newton tolerance {tol}, one density pass (images, sort, search, circuit1)")
    return out


def max_over_ranks(x, device="cuda"):
    """The largest of every rank's x (every rank calls this at the same
    point); x itself without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(ws, n_particles, steps, ms_max):
    """Whole-job particle-steps/s of ws independent replicas of n_particles
    each, `steps` steps, timed as the slowest rank's ms."""
    return ws * n_particles * steps / (ms_max * 1e-3)


def timed_steps(e, K):
    """Run K steps timed by CUDA events on the engine's stream: one pair
    around the call (the step time) and one per phase (SPH_P_TIMING = 1);
    returns (device ms of the K steps, counters of the K steps, per-phase ms
    per step)."""
    e.reset_counters()
    e.set_param(abi.P_TIMING, 1)
    e.step(K)
    t = e.timers()
    e.set_param(abi.P_TIMING, 0)
    return t["step"], e.counters(), {k: v / K for k, v in t.items()}


def main():
    args = parse()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    from sph_playground_b200 import ic

    lib = abi.load()
    st, store = ic.sedov3d(n=args.n)
    N = store.shape[0]
    peak32, peak64 = measure_peak()

    # launch shapes (lanes per centre, cell edge) picked by the autotuner on
    # this workload, per precision (sph_playground_b200/tune.py)
    tuned = {abi.PREC_FP32_COMP: {}, abi.PREC_FP64: {}}
    if not args.no_autotune:
        from sph_playground_b200 import tune
        for prec in tuned:
            r = tune.autotune(st, store, "m6", prec, lib=lib, cache=None)
            tuned[prec] = {k: v for k, v in r.items() if k.startswith("P_")}

    def engine(prec, st_=None, store_=None):
        e = abi.Engine(st if st_ is None else st_, store if store_ is None else store_, "m6",
                       precision=prec, lib=lib)
        for k, v in tuned[prec].items():
            e.set_param(getattr(abi, k), float(v))
        for kv in args.param:
            k, v = kv.split("=")
            e.set_param(int(k) if k.isdigit() else getattr(abi, k, k), float(v))
        return e

    def field_errors(st_, store_):
        """FP32-comp vs FP64: one iterate on the same state; rho and h per
        particle, a / du/dt / dh/dt per particle relative to the field's
        largest magnitude (a lattice at rest has a ~ 0 almost everywhere)."""
        e32, e64 = engine(abi.PREC_FP32_COMP, st_, store_), engine(abi.PREC_FP64, st_, store_)
        e32.iterate()
        e64.iterate()
        r32, r64 = e32.get_store(), e64.get_store()
        e32.close()
        e64.close()
        C = {k: v - 1 for k, v in abi.consts.es.items()}
        out = {}
        for name in ("den", "h"):
            rel = np.abs(r32[:, C[name]] - r64[:, C[name]]) / np.abs(r64[:, C[name]])
            out["rho" if name == "den" else name] = {"max": float(rel.max()),
                                                     "p99.9": float(np.quantile(rel, 0.999))}
        for name, cols in (("a", [C["ax"], C["ay"], C["az"]]), ("du", [C["du"]]),
                           ("dh", [C["dh"]])):
            d = np.linalg.norm(r32[:, cols] - r64[:, cols], axis=1)
            ref = np.linalg.norm(r64[:, cols], axis=1).max()
            rel = d / ref if ref > 0 else d
            out[name + "_rel_field_max"] = {"max": float(rel.max()),
                                            "p99.9": float(np.quantile(rel, 0.999))}
        return out

    # FP32 vs FP64 errors on the bench input and after the warm-up steps
    errs, rho_err = None, None
    if not args.no_errors:
        errs = {"t0": field_errors(st, store)}
        e64 = engine(abi.PREC_FP64)
        e64.set_param(abi.consts.ec["tfinish"], 1.0)
        e64.step(max(args.warmup, 1))
        mid_store, mid_st = e64.get_store(), e64.get_state()
        e64.close()
        errs[f"after_{max(args.warmup, 1)}_steps"] = field_errors(mid_st, mid_store)
        rho_err = max((v["rho"] for v in errs.values()), key=lambda x: x["max"])

    def run(prec):
        e = engine(prec)
        e.set_param(abi.consts.ec["tfinish"], 1.0)
        for _ in range(args.warmup):
            e.step(1)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        uuid = None
        try:
            uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
        except Exception:
            uuid = None
        with Clocks(uuid) as ck:
            ms, cnt, tm = timed_steps(e, args.steps)
            torch.cuda.synchronize()
        ms = max_over_ranks(ms)
        if ws > 1:
            dist.barrier()
        return e, ms, cnt, tm, ck.summary()

    e, ms, cnt, tm, clocks = run(abi.PREC_FP32_COMP)
    value = replica_throughput(ws, N, args.steps, ms)

    # roofline of the dominant pair kernel: algorithmic FLOPs / its event time
    c1_flops = cnt["c1_pairs"] * F1_C1
    c2_flops = cnt["c2_pairs"] * F2_C2
    kern = {"circuit1": (c1_flops / args.steps, tm["circuit1"]),
            "circuit2": (c2_flops / args.steps, tm["circuit2"])}
    dom = max(kern, key=lambda k: kern[k][1])
    # (no per-phase events inside a device-resident graph step)
    ach = kern[dom][0] / (kern[dom][1] * 1e-3) / 1e12 if kern[dom][1] > 0 else 0.0
    traffic = C2_DRAM_BYTES_PER_PAIR * cnt["c2_pairs"] / args.steps if dom == "circuit2" else None
    roofline = {"bound": "fp32", "kernel": dom, "achieved": ach, "peak": peak32 / 1e12,
                "unit": "TFLOP/s", "frac": ach / (peak32 / 1e12), "traffic": traffic,
                "traffic_source": "ncu DRAM bytes of the k_c2 capture on the Sedov 96^3 step "
                                  "per pair, times this launch's pairs",
                "peak_source": "live FFMA-chain probe (libsph_peak.so) on this GPU; "
                               "MEASURED_PEAKS.json holds no non-tensor FP32 figure"}

    # end to end through the C-ABI with pinned host buffers, per step:
    # H2D of the particle table, one step, D2H of the particle table
    e2e = None
    if not args.no_e2e:
        host_in = torch.empty((N, 32), dtype=torch.float64).pin_memory().numpy()
        host_out = torch.empty((N, 32), dtype=torch.float64).pin_memory().numpy()
        e.get_store(host_in)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e.set_store(host_in)
            e.step(1)
            e.get_store(host_out)
            host_in, host_out = host_out, host_in
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        el = max_over_ranks(el)
        e2e = {"value": replica_throughput(ws, N, args.e2e_steps, el * 1e3), "unit": UNIT,
               "h2d_bytes_per_step": N * 32 * 8, "d2h_bytes_per_step": N * 32 * 8,
               "steps": args.e2e_steps,
               "timing": "host clock around synchronous C-ABI calls (set_store, step, get_store)"}
    e.close()

    fp64 = None
    if not args.no_fp64:
        e6, ms6, cnt6, tm6, _ = run(abi.PREC_FP64)
        e6.close()
        fp64 = {"value": replica_throughput(ws, N, args.steps, ms6), "ms_per_step": ms6 / args.steps,
                "work_per_step": {"c1_pairs": cnt6["c1_pairs"] / args.steps,
                                  "device_allocations_in_timed_steps": cnt6["allocs"],
                                  "c1_max_sweeps": cnt6["c1_sweeps"], "neib_max": cnt6["neib_max"],
                                  "searches": cnt6["searches"] / args.steps,
                                  "candidates": cnt6["candidates"] / args.steps},
                "phases_ms_per_step": tm6,
                "peak_fp64_tflops": peak64 / 1e12}

    adj = None
    if not args.no_adjoint:
        adj = adjoint_block(lib)
    dens = None
    if not args.no_density:
        extra = dict(kv.split("=") for kv in args.param if not kv.split("=")[0].isdigit())
        dens = density_block(lib, {p: {**tuned[p], **extra} for p in tuned})

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_n)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"sedov3d {args.n}^3 ({N} particles), M6 hfac 1.2, "
                                   "FP32-comp pair sums, full leapfrog step",
                       "particles": N, "kernel": "m6", "precision": "fp32_comp",
                       "l2": "inputs larger than L2 (particle table "
                             f"{N * 32 * 8 / 1e6:.0f} MB + pair streams)",
                       "parallelism": f"replicas x{ws}",
                       "launch_shapes": {"fp32_comp": tuned[abi.PREC_FP32_COMP],
                                         "fp64": tuned[abi.PREC_FP64],
                                         "source": "autotuned on this workload" if not
                                         args.no_autotune else "defaults"}},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": cnt["launches"],
            "clocks": clocks,
            "rho_rel_err_fp32_vs_fp64": rho_err,
            "errors_fp32_vs_fp64": errs,
            "phases_ms_per_step": tm,
            "work_per_step": {"neib_pairs": cnt["neib_pairs"] / args.steps,
                              "c1_pairs": cnt["c1_pairs"] / args.steps,
                              "c2_pairs": cnt["c2_pairs"] / args.steps,
                              "c1_max_sweeps": cnt["c1_sweeps"],
                              "neib_max": cnt["neib_max"],
                              "searches": cnt["searches"] / args.steps,
                              "exact_tests": cnt["exact_tests"] / args.steps,
                              "device_allocations_in_timed_steps": cnt["allocs"],
                              "candidates": cnt["candidates"] / args.steps},
            "fp64": fp64,
            "adjoint": adj,
            "density_pass": dens,
            "speedup_fp32_vs_fp64": (value / fp64["value"]) if fp64 else None,
            "peak_fp32_tflops": peak32 / 1e12,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
