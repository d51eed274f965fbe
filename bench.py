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
# dram__bytes_read.sum + dram__bytes_write.sum = 862.28 MB + 73.97 MB over
# 157.49M pairs of an ncu capture of k_c2 on the Sedov 96^3 step (FP32-comp, 4
# lanes per centre, cell edge 0.4 krad h_min, an iterate served from skin
# lists) (the neighbour index, 4 B, plus the gathered pair data that misses
# L2); the traffic scales with the pairs a launch processes
C2_DRAM_BYTES_PER_PAIR = (862.28e6 + 73.97e6) / 157.49e6
# DRAM bytes per in-support pair of the neighbour search (k_neighbours),
# same capture workload: 198.36 MB read + 684.48 MB written over 157.49M
# pairs; the search's algorithmic bytes are the 4 B list entry per pair it
# writes plus its per-centre reads and writes (FP32 image 16 B, h 8 B, row
# offset / capacity 12 B, count 4 B)
SEARCH_DRAM_BYTES_PER_PAIR = (198.36e6 + 684.48e6) / 157.49e6
SEARCH_BYTES_PER_PAIR = 4.0
SEARCH_BYTES_PER_CENTRE = 40.0
# per-particle FLOP per step (Newton update, EOS, epilogue, leapfrog)
F_PARTICLE = 100.0


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth of this pool's B200s when
    the peaks file is present, else the stated fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (no measured peaks file)"


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
    ap.add_argument("--cpu-n", type=int, default=128,
                    help="lattice per axis of the CPU baseline and the reference arm")
    ap.add_argument("--no-oracle-errors", action="store_true",
                    help="skip the errors against the CPU oracle at the bench size")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the 21-instance diffusion batch (config 3)")
    ap.add_argument("--no-full-run", action="store_true",
                    help="skip the whole Sedov run to t = 0.05")
    ap.add_argument("--no-160", action="store_true",
                    help="skip the 160^3 Sedov throughput line (config 5b)")
    ap.add_argument("--no-decomposed", action="store_true",
                    help="with N > 1: skip the one-problem-over-N-ranks block")
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
                      f"start-up iterate, CPU oracle (FP64, OpenMP {cores} threads)",
            "same_config": True}


def field_report(got, ref):
    """rho, h per particle and a, du/dt, dh/dt relative to the field's
    largest magnitude (max and 99.9th percentile)."""
    C = {k: v - 1 for k, v in abi.consts.es.items()}
    out = {}
    for name in ("den", "h"):
        rel = np.abs(got[:, C[name]] - ref[:, C[name]]) / np.abs(ref[:, C[name]])
        out["rho" if name == "den" else name] = {"max": float(rel.max()),
                                                 "p99.9": float(np.quantile(rel, 0.999))}
    for name, cols in (("a", [C["ax"], C["ay"], C["az"]]), ("du", [C["du"]]),
                       ("dh", [C["dh"]])):
        d = np.linalg.norm(got[:, cols] - ref[:, cols], axis=1)
        scale = np.linalg.norm(ref[:, cols], axis=1).max()
        rel = d / scale if scale > 0 else d
        out[name + "_rel_field_max"] = {"max": float(rel.max()),
                                        "p99.9": float(np.quantile(rel, 0.999))}
    return out


def batch_block(lib, tfinish=0.01):
    """Config 3: the anisotropic diffusion sweep, 7 lattices (32^2 .. 256^2)
    x 3 second-derivative methods (fab, n2w, 2nw_ds) = 21 uneven instances,
    fixed-stage STS to t = 0.01, stepped together as one batch; the batch's
    host-clock time per precision and the L2 error of T against the analytic
    exponential decay for every instance."""
    from sph_playground_b200 import ic
    sizes = (32, 48, 64, 96, 128, 192, 256)
    methods = ("fab", "n2w", "2nw_ds")
    sets = [(n, ddw, ic.diffusion2d(n, ddw=ddw, tfinish=tfinish)) for ddw in methods
            for n in sizes]
    C = {k: v - 1 for k, v in abi.consts.es.items()}
    out = {"workload": "diffusion2d n^2 for n in 32..256 x ddw fab / n2w / 2nw_ds, "
                       f"k_par b b^T diagonal form, STS 8 stages, to t = {tfinish}",
           "instances": len(sets), "particles": int(sum(n * n for n, _, _ in sets))}
    for prec, name in ((abi.PREC_FP64, "fp64"), (abi.PREC_FP32_COMP, "fp32_comp")):
        # warm-up of the kernels and graphs on a short batch
        eng = [abi.Engine(st, store, "m6", precision=prec, lib=lib) for _, _, (st, store) in sets]
        with abi.Batch(eng) as b:
            b.step(2)
        for e in eng:
            e.close()
        eng = [abi.Engine(st, store, "m6", precision=prec, lib=lib) for _, _, (st, store) in sets]
        t0 = time.perf_counter()
        with abi.Batch(eng) as b:
            # the first step starts every instance (its start-up iterate on
            # the host path) and builds the device loop; the rest of the
            # run to tfinish is the loop itself
            b.step(1)
            t1 = time.perf_counter()
            b.run_to(tfinish)
            t2 = time.perf_counter()
        el = t2 - t0
        l2, steps = {}, 0
        for (n, ddw, _), e in zip(sets, eng):
            s = e.get_store()
            t = e.get_state()[abi.consts.ec["time"] - 1]
            exact = ic.diffusion_exact(s[:, 0:3], t)
            l2[f"{ddw}_{n}"] = float(np.sqrt(np.mean((s[:, C["t"]] - exact) ** 2)))
            steps += e.counters()["steps"] * n * n
            e.close()
        out[name] = {"seconds": el, "seconds_start_and_first_step": t1 - t0,
                     "seconds_device_loop": t2 - t1, "particle_steps_per_s": steps / el,
                     "l2_vs_analytic": l2}
    # the floor for any batching: the longest instance (256^2 fab) alone,
    # its steps replayed as CUDA graphs, after its own first step
    for prec, name in ((abi.PREC_FP64, "fp64"), (abi.PREC_FP32_COMP, "fp32_comp")):
        st, store = ic.diffusion2d(256, ddw="fab", tfinish=tfinish)
        with abi.Engine(st, store, "m6", precision=prec, lib=lib) as e:
            e.set_param(abi.P_GRAPH, 1.0)
            e.step(1)
            t0 = time.perf_counter()
            e.run_to(tfinish)
            out[name]["longest_instance_alone_seconds"] = time.perf_counter() - t0
    out["timing"] = ("host clock around the synchronous sph_batch_step(1) (instance start-up, "
                     "loop build) and sph_batch_run_to (the device loop) calls")
    return out


def decomposed_block(lib, st, store, steps, warmup, shapes, device):
    """One problem over all ranks (sph_playground_b200.domain.DecomposedRun:
    each rank computes the pairs of its Morton range of particles, two
    all-gathers per step): the Sedov step of this workload, FP32-comp,
    timed on the host between barriers after `warmup` steps (max over
    ranks)."""
    import torch
    import torch.distributed as dist
    from sph_playground_b200 import domain
    run = domain.DecomposedRun(st, store, "m6", precision=abi.PREC_FP32_COMP, lib=lib,
                               device=device)
    for k, v in shapes.items():
        run.e.set_param(getattr(abi, k), float(v))
    run.start()
    run.run_to(1.0, max_steps=warmup)
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    run.run_to(1.0, max_steps=warmup + steps)
    torch.cuda.synchronize()
    el = max_over_ranks(time.perf_counter() - t0)
    n_own = run.n_own
    run.close()
    N = store.shape[0]
    return {"workload": workload_name(round(N ** (1 / 3))) + ", FP32-comp, one problem over "
                        f"{dist.get_world_size()} ranks (particle decomposition)",
            "value": N * steps / el, "unit": UNIT, "ms_per_step": 1e3 * el / steps,
            "scaling": "strong", "owned_particles_rank0": n_own,
            "timing": "host clock between barriers around synchronous steps, max over ranks"}


def size160_block(engine, st, store, steps, warmup):
    """Config 5b: the Sedov step at 160^3 = 4,096,000 particles, FP32-comp
    and FP64, device time of `steps` steps after `warmup` steps."""
    out = {"workload": workload_name(160)}
    N = store.shape[0]
    for prec, name in ((abi.PREC_FP32_COMP, "fp32_comp"), (abi.PREC_FP64, "fp64")):
        e = engine(prec, st, store)
        e.set_param(abi.consts.ec["tfinish"], 1.0)
        for _ in range(warmup):
            e.step(1)
        ms, cnt, tm = timed_steps(e, steps)
        e.close()
        out[name] = {"value": N * steps / (ms * 1e-3), "ms_per_step": ms / steps,
                     "phases_ms_per_step": tm,
                     "work_per_step": {"neib_pairs": cnt["neib_pairs"] / steps,
                                       "c1_pairs": cnt["c1_pairs"] / steps,
                                       "newton_sweeps_per_particle":
                                           cnt["c1_centre_sweeps"] / (steps * N),
                                       "c1_max_sweeps": cnt["c1_sweeps"]}}
    out["speedup_fp32_vs_fp64"] = out["fp32_comp"]["value"] / out["fp64"]["value"]
    return out


def workload_name(n):
    return (f"sedov3d {n}^3 ({n ** 3} particles), M6 hfac 1.2, full leapfrog step "
            "(timestep, predictor, images, neighbour lists, circuit1, circuit2, corrector)")


def run_reference(args, ws, rank):
    """The reference arm: the CPU oracle (the C++ FP64 OpenMP restatement of
    the reference engine's path; the Fortran itself cannot be built without
    gfortran and HDF5) on the same workload as the GPU arm, all host
    threads, `warmup` untimed steps and `steps` timed steps after the
    start-up iterate."""
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
        "config": {"workload": workload_name(n), "particles": N, "same_config": n == args.n,
                   "note": "reference Fortran not compiled (no gfortran/HDF5 in the image); "
                           "the CPU oracle restatement of its path is timed instead; its "
                           "search is a uniform cell grid, not the reference's per-step "
                           "kd-tree, so it is likely faster than the Fortran would be"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"sedov3d {n}^3, {args.steps} steps after {args.warmup} warm-up"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def adjoint_block(lib, n=256, n_ref=64, nsteps=200, every=20, dt=5e-4):
    """The adjoint workload: 2D periodic shear flow (n^2 particles, M6,
    alpha = 1, beta = 2), nsteps fixed-dt leapfrog steps with a checkpoint
    every `every` steps, loss sum |v(T) - v_target|^2 with the target from
    the run with shear amplitude 0.12; forward and backward timed on the
    host around the synchronous C-ABI calls.  Also the FP32-comp gradient
    against the FP64 gradient at n_ref^2."""
    from sph_playground_b200 import ic
    V = [abi.consts.es["vx"] - 1, abi.consts.es["vy"] - 1, abi.consts.es["vz"] - 1]

    targets = {}

    def target_of(nn, steps):
        # the final velocities of the same run started with shear amplitude
        # 0.12 instead of 0.1 (FP64, shared by both precisions)
        if (nn, steps) not in targets:
            st, store = ic.shear2d(n=nn, amp=0.12)
            e = abi.Engine(st, store, "m6", precision=abi.PREC_FP64, lib=lib)
            e.set_param(abi.P_FIXED_DT, dt)
            e.adjoint_forward(steps, every)
            targets[(nn, steps)] = e.get_store()[:, V]
            e.close()
        return targets[(nn, steps)]

    def grads(nn, prec, steps):
        target = target_of(nn, steps)
        st, store = ic.shear2d(n=nn)
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

    # warm-up at the timed size: kernels loaded, and the checkpoint and
    # per-step slots' device blocks held by the library's cache afterwards
    grads(n, abi.PREC_FP64, nsteps)
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


def density_block(lib, shapes, n=128, tol=1e-6, reps=5, oracle=None):
    """The density-only workload: one density + Newton-h pass over a 3D
    periodic n^3 lattice perturbed by uniform(-0.1, 0.1) dx (seed 2), M6,
    hfac 1.2, Newton tolerance `tol`; FP32-comp against FP64: device time of
    the pass (CUDA events of the neighbour and circuit1 phases, averaged
    over `reps` passes after one warm-up), its phases, and the per-particle
    relative error of rho and h against the FP64 path and, when `oracle` is
    given, against the CPU oracle (with the neighbour sets' digests)."""
    from sph_playground_b200 import ic
    st, store = ic.density3d(n=n, seed=2)
    out, res, dig = {}, {}, {}
    for prec, name in ((abi.PREC_FP64, "fp64"), (abi.PREC_FP32_COMP, "fp32_comp")):
        e = abi.Engine(st, store, "m6", precision=prec, lib=lib)
        for k, v in shapes.get(prec, {}).items():  # the launch shapes of the step arms
            e.set_param(getattr(abi, k), float(v))
        e.set_param(abi.P_NEWTON_TOL, tol)
        # one pass from a table just uploaded: a plain search (skin lists
        # would cost their wider search and serve no later pass)
        e.set_param(abi.P_SKIN, 0.0)
        e.density()
        res[name] = e.get_store()
        dig[name] = e.get_neighbour_digest()
        e.reset_counters()
        e.set_param(abi.P_TIMING, 1)
        for _ in range(reps):
            e.set_store(store)
            e.density()
        t = e.timers()
        c = e.counters()
        e.close()
        ph = {k: t[k] / reps for k in ("ghosts", "sort", "neighbours", "pack", "circuit1")}
        ms = sum(ph.values())
        out[name] = {"ms_per_pass": ms, "particle_passes_per_s": store.shape[0] / (ms * 1e-3),
                     "phases_ms": ph,
                     "newton_sweeps_per_particle": c["c1_centre_sweeps"] / (reps * store.shape[0])}
    C = {k: v - 1 for k, v in abi.consts.es.items()}
    for f in ("den", "h"):
        rel = np.abs(res["fp32_comp"][:, C[f]] - res["fp64"][:, C[f]]) / np.abs(res["fp64"][:, C[f]])
        out[("rho" if f == "den" else f) + "_rel_err"] = {"max": float(rel.max()),
                                                        "p99.9": float(np.quantile(rel, 0.999))}
    if oracle is not None:
        with abi.Engine(st, store, "m6", lib=oracle) as o:
            o.set_param(abi.P_NEWTON_TOL, tol)
            o.density()
            ref, dref = o.get_store(), o.get_neighbour_digest()
        vs = {}
        for name in ("fp64", "fp32_comp"):
            r = {}
            for f in ("den", "h", "om"):
                rel = np.abs(res[name][:, C[f]] - ref[:, C[f]]) / np.abs(ref[:, C[f]])
                r[{"den": "rho", "h": "h", "om": "omega"}[f]] = {
                    "max": float(rel.max()), "p99.9": float(np.quantile(rel, 0.999))}
            r["neighbour_sets_equal"] = bool(np.array_equal(dig[name][0], dref[0]) and
                                             np.array_equal(dig[name][1], dref[1]))
            vs[name] = r
        out["errors_vs_oracle"] = vs
    out["fp32_over_fp64_speed"] = out["fp64"]["ms_per_pass"] / out["fp32_comp"]["ms_per_pass"]
    out["workload"] = (f"density3d {n}^3 ({store.shape[0]} particles), perturbed lattice, M6 hfac 1.2, "
                       f"Newton tolerance {tol}, one density pass (images, sort, search, circuit1)")
    return out


def full_run_block(engine, st, store, tfinish=0.05):
    """The whole Sedov run of the workload (leapfrog from t = 0 to
    tfinish): device time of every step (CUDA events around the sph_run_to
    call), particle-steps/s, and how the skin lists served it; FP32-comp with
    skin lists (the default), FP32-comp with a fresh search every iterate,
    FP64 with skin lists."""
    st = st.copy()
    st[abi.consts.ec["tfinish"] - 1] = tfinish
    out = {}
    for name, prec, skin in (("fp32_comp", abi.PREC_FP32_COMP, None),
                             ("fp32_comp_fresh_search", abi.PREC_FP32_COMP, 0.0),
                             ("fp64", abi.PREC_FP64, None)):
        e = engine(prec, st, store)
        if skin is not None:
            e.set_param(abi.P_SKIN, skin)
        e.reset_counters()
        e.set_param(abi.P_TIMING, 2)
        e.run_to(tfinish)
        t, c = e.timers(), e.counters()
        e.close()
        k = max(c["steps"], 1)
        out[name] = {"steps": c["steps"], "seconds": t["step"] * 1e-3,
                     "ms_per_step": t["step"] / k,
                     "particle_steps_per_s": store.shape[0] * c["steps"] / (t["step"] * 1e-3),
                     "skin": {"builds": c["skin_builds"], "iterates_served": c["skin_reuses"],
                              "rows_kept_per_served": c["skin_kept"] / max(c["skin_reuses"], 1),
                              "rows_searched_afresh_per_served":
                                  c["skin_dirty"] / max(c["skin_reuses"], 1)}}
    out["workload"] = (f"sedov3d {round(store.shape[0] ** (1 / 3))}^3, leapfrog from t = 0 to "
                       f"t = {tfinish} (the whole Sedov run), device time of the run_to call")
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

    oracle = None
    if rank == 0 and not args.no_oracle_errors:
        oracle = abi.load(os.path.join(ROOT, "oracle", "liboracle.so"))

    def field_errors(st_, store_):
        """One iterate on the same state: FP32-comp against FP64 on the GPU
        and, with the oracle, both GPU paths against the CPU FP64 oracle
        (rho and h per particle; a, du/dt, dh/dt relative to the field's
        largest magnitude, since a lattice at rest has a ~ 0 almost
        everywhere) with the neighbour sets' digests."""
        res, dig = {}, {}
        for prec, name in ((abi.PREC_FP32_COMP, "fp32_comp"), (abi.PREC_FP64, "fp64")):
            e = engine(prec, st_, store_)
            e.iterate()
            res[name], dig[name] = e.get_store(), e.get_neighbour_digest()
            e.close()
        out = {"fp32_vs_fp64": field_report(res["fp32_comp"], res["fp64"])}
        if oracle is not None:
            with abi.Engine(st_, store_, "m6", lib=oracle) as o:
                o.iterate()
                ref, dref = o.get_store(), o.get_neighbour_digest()
            for name in ("fp32_comp", "fp64"):
                r = field_report(res[name], ref)
                r["neighbour_sets_equal"] = bool(np.array_equal(dig[name][0], dref[0]) and
                                                 np.array_equal(dig[name][1], dref[1]))
                out[name + "_vs_oracle"] = r
        return out

    # errors on the bench input and after the warm-up steps
    errs, rho_err = None, None
    if not args.no_errors:
        errs = {"t0": field_errors(st, store)}
        e64 = engine(abi.PREC_FP64)
        e64.set_param(abi.consts.ec["tfinish"], 1.0)
        e64.step(max(args.warmup, 1))
        mid_store, mid_st = e64.get_store(), e64.get_state()
        e64.close()
        errs[f"after_{max(args.warmup, 1)}_steps"] = field_errors(mid_st, mid_store)
        key = "fp32_comp_vs_oracle" if oracle is not None else "fp32_vs_fp64"
        rho_err = max((v[key]["rho"] for v in errs.values()), key=lambda x: x["max"])

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

    # per-kernel rooflines (algorithmic work per launch / its CUDA-event time)
    # and the step-level figure; the roofline line is the kernel that takes
    # the most time per step
    K = args.steps
    hbm, hbm_src = hbm_peak()
    p32 = peak32 / 1e12
    kernels = {
        "neighbours": {"bound": "hbm", "unit": "GB/s", "peak": hbm,
                       "work": (SEARCH_BYTES_PER_PAIR * cnt["neib_pairs"] +
                                SEARCH_BYTES_PER_CENTRE * N * cnt["searches"]) / K,
                       "traffic": SEARCH_DRAM_BYTES_PER_PAIR * cnt["neib_pairs"] / K,
                       "ms": tm["neighbours"],
                       "candidate_tests_per_s": cnt["candidates"] / K / (tm["neighbours"] * 1e-3)
                       if tm["neighbours"] > 0 else None},
        "circuit1": {"bound": "fp32", "unit": "TFLOP/s", "peak": p32,
                     "work": cnt["c1_pairs"] * F1_C1 / K, "traffic": None, "ms": tm["circuit1"]},
        "circuit2": {"bound": "fp32", "unit": "TFLOP/s", "peak": p32,
                     "work": cnt["c2_pairs"] * F2_C2 / K,
                     "traffic": C2_DRAM_BYTES_PER_PAIR * cnt["c2_pairs"] / K, "ms": tm["circuit2"]},
    }
    for name, kk in kernels.items():
        scale = 1e9 if kk["unit"] == "GB/s" else 1e12
        kk["achieved"] = kk["work"] / (kk["ms"] * 1e-3) / scale if kk["ms"] > 0 else 0.0
        kk["frac"] = kk["achieved"] / kk["peak"]
    served = cnt["skin_reuses"]
    if served:
        # iterates served from skin lists write only the rows they filter or
        # search afresh (the kept rows stay): the phase is a mix of small
        # kernels with no single work figure, reported by what it did
        nbk = kernels["neighbours"]
        nbk.update({"bound": "skin lists", "achieved": None, "frac": None, "work": None,
                    "traffic": None,
                    "iterates": {"served_from_skin_lists": served,
                                 "skin_list_builds": cnt["skin_builds"],
                                 "rows_kept_per_served": cnt["skin_kept"] / served,
                                 "rows_searched_afresh_per_served": cnt["skin_dirty"] / served}})
    dom = max((k for k in kernels if kernels[k]["frac"] is not None),
              key=lambda k: kernels[k]["ms"])
    step_flops = (cnt["c1_pairs"] * F1_C1 + cnt["c2_pairs"] * F2_C2) / K + N * F_PARTICLE
    step_ach = step_flops / ((ms / K) * 1e-3) / 1e12
    roofline = {"bound": kernels[dom]["bound"], "kernel": dom,
                "achieved": kernels[dom]["achieved"], "peak": kernels[dom]["peak"],
                "unit": kernels[dom]["unit"], "frac": kernels[dom]["frac"],
                "traffic": kernels[dom]["traffic"],
                "step_frac": step_ach / p32, "step_achieved_tflops": step_ach,
                "kernels": kernels,
                "binding_unit": {"circuit2": {"unit": "L1/TEX data path", "ncu_pct_of_peak": 96.9,
                                              "fma_pipe_pct": 52.5, "issue_active_pct": 74.8,
                                              "source": "profiles/k_c2_fp32_sedov3d_96.md"}},
                "traffic_source": "ncu DRAM bytes per pair of the kernel's capture on the "
                                  "Sedov 96^3 step, times this launch's pairs",
                "peak_source": {"fp32": "live FFMA-chain probe (libsph_peak.so) on this GPU; "
                                        "MEASURED_PEAKS.json holds no non-tensor FP32 figure",
                                "hbm": hbm_src},
                "work_definition": "fp32 kernels: in-support pairs x per-pair FLOP (circuit1 "
                                   f"{F1_C1:.0f} per sweep, circuit2 {F2_C2:.0f}); search (iterates "
                                   f"with a fresh search): 4 B per pair written + "
                                   f"{SEARCH_BYTES_PER_CENTRE:.0f} B per centre; "
                                   "step: both pair passes + "
                                   f"{F_PARTICLE:.0f} FLOP per particle"}

    # end to end through the C-ABI with pinned host buffers, per step:
    # H2D of the particle table, one step, D2H of the particle table
    e2e = None
    if not args.no_e2e:
        host_in = torch.empty((N, 32), dtype=torch.float64).pin_memory().numpy()
        host_out = torch.empty((N, 32), dtype=torch.float64).pin_memory().numpy()
        e.get_store(host_in)
        # one untimed round trip (the first touch of the pinned buffers)
        e.set_store(host_in)
        e.step(1)
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
        dens = density_block(lib, {p: {**tuned[p], **extra} for p in tuned}, oracle=oracle)
    batch = None
    if not args.no_batch:
        batch = batch_block(lib)
    decomposed = None
    if ws > 1 and not args.no_decomposed:
        # every rank runs the same steps, so an error is raised on all of them
        # at the same point; it is recorded instead of ending the replicas'
        # line
        try:
            decomposed = decomposed_block(lib, st, store, args.steps, args.warmup,
                                          tuned[abi.PREC_FP32_COMP], f"cuda:{local}")
        except Exception as exc:  # noqa: BLE001
            decomposed = {"error": f"{type(exc).__name__}: {exc}"}
    full = None
    if not args.no_full_run and ws == 1:
        full = full_run_block(engine, st, store)
    big = None
    if not args.no_160 and args.n == 128:
        st160, store160 = ic.sedov3d(n=160)
        big = size160_block(engine, st160, store160, args.steps, args.warmup)
        del st160, store160

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_n)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": workload_name(args.n) + ", FP32-comp pair sums",
                       "particles": N, "kernel": "m6", "precision": "fp32_comp",
                       "l2": "inputs larger than L2 (particle table "
                             f"{N * 32 * 8 / 1e6:.0f} MB + pair streams)",
                       "parallelism": f"replicas x{ws}",
                       "neighbour_lists": "skin lists (SPH_P_SKIN = 0.1): radius 1.1 krad h, "
                                          "rows kept, refiltered with the FP64 predicate or "
                                          "searched afresh every iterate; sets equal a fresh "
                                          "search's",
                       "launch_shapes": {"fp32_comp": tuned[abi.PREC_FP32_COMP],
                                         "fp64": tuned[abi.PREC_FP64],
                                         "source": "autotuned on this workload" if not
                                         args.no_autotune else "defaults"}},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": cnt["launches"],
            "clocks": clocks,
            "rho_rel_err_fp32": rho_err,
            "rho_rel_err_fp32_reference": "the CPU FP64 oracle" if oracle is not None
                                          else "the FP64 GPU path",
            "errors": errs,
            "phases_ms_per_step": tm,
            "work_per_step": {"neib_pairs": cnt["neib_pairs"] / args.steps,
                              "c1_pairs": cnt["c1_pairs"] / args.steps,
                              "c2_pairs": cnt["c2_pairs"] / args.steps,
                              "c1_max_sweeps": cnt["c1_sweeps"],
                              "newton_sweeps_per_particle":
                                  cnt["c1_centre_sweeps"] / (args.steps * N),
                              "neib_max": cnt["neib_max"],
                              "searches": cnt["searches"] / args.steps,
                              "exact_tests": cnt["exact_tests"] / args.steps,
                              "device_allocations_in_timed_steps": cnt["allocs"],
                              "candidates": cnt["candidates"] / args.steps},
            "fp64": fp64,
            "adjoint": adj,
            "density_pass": dens,
            "diffusion_batch": batch,
            "decomposed": decomposed,
            "sedov3d_160": big,
            "sedov3d_full_run": full,
            "speedup_fp32_vs_fp64": (value / fp64["value"]) if fp64 else None,
            "peak_fp32_tflops": peak32 / 1e12,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
