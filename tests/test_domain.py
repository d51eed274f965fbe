"""The split step (sph_timestep, sph_predict, sph_density, sph_forces,
sph_correct, sph_get_columns / sph_set_columns) and the particle
decomposition over torch.distributed built on it
(sph_playground_b200/domain.py).

On the CPU: the oracle driven through the split step equals its own time
loop bit for bit; two gloo ranks, each holding the whole table with its
Morton half as centres, equal the single-domain oracle run.  On the GPU: the
same with the CUDA engine (the two ranks share one GPU and exchange through
gloo on the host, so no kernel waits on another rank)."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from sph_playground_b200 import abi, consts, domain, ic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COL = {k: v - 1 for k, v in consts.es.items()}
T_END = 0.03


def _sedov():
    # one output time (the end): the output-time clipping of the time loop
    # (main.f90:273-299) flips between a clipped step and a full one on
    # rounding-level differences of t and dt, and FP32 runs that sum in
    # another order would then take different steps
    return ic.sedov3d(n=10, tfinish=T_END, npics=1)


def _alone(lib_path, prec, st, store, t_end, params=None):
    lib = abi.load(lib_path)
    with abi.Engine(st, store, "m6", precision=prec, lib=lib) as e:
        for k, v in (params or {}).items():
            e.set_param(k, v)
        e.run_to(t_end)
        return e.get_store(), e.get_state(), e.counters()["steps"]


def _rel(a, b):
    scale = np.max(np.abs(b), axis=0)
    scale[scale == 0] = 1.0
    return float(np.max(np.abs(a - b) / scale))


def test_morton_owners_split_evenly():
    st, store = _sedov()
    own = domain.morton_owners(store[:, 0:3], 3, 3)
    counts = np.bincount(own, minlength=3)
    assert counts.max() - counts.min() <= 1
    # each rank's particles form a compact block: its bounding box is a
    # fraction of the box
    for r in range(3):
        p = store[own == r, 0:3]
        assert np.prod(p.max(0) - p.min(0)) < 0.75


def test_split_run_equals_time_loop_oracle(oracle_lib):
    st, store = _sedov()
    ref, ref_st, steps = _alone(os.path.join(ROOT, "oracle", "liboracle.so"), abi.PREC_FP64,
                                st, store, T_END)
    with abi.Engine(st, store, "m6", lib=oracle_lib) as e:
        run = domain.SplitRun(e)
        run.start()
        run.run_to(T_END)
        got, got_st = e.get_store(), e.get_state()
    assert run.steps == steps and steps >= 3
    assert np.array_equal(got_st, ref_st)
    assert np.array_equal(got, ref)


def _rank(rank, world, port, lib_path, prec, device, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    if device != "cpu":
        torch.cuda.set_device(0)
    lib = abi.load(lib_path)
    st, store = _sedov()
    run = domain.DecomposedRun(st, store, "m6", precision=prec, lib=lib, device="cpu")
    run.start()
    run.run_to(T_END)
    out[rank] = (run.global_store(), run.steps, run.t)
    run.close()
    dist.barrier()
    dist.destroy_process_group()


def _decomposed(lib_path, prec, device="cpu", world=2):
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = 29500 + (os.getpid() * 7 + world) % 2000
    mp.start_processes(_rank, args=(world, port, lib_path, prec, device, out), nprocs=world,
                       start_method="spawn", join=True)
    return [out[r] for r in range(world)]


def test_decomposed_oracle_equals_single_domain():
    path = os.path.join(ROOT, "oracle", "liboracle.so")
    st, store = _sedov()
    ref, ref_st, steps = _alone(path, abi.PREC_FP64, st, store, T_END)
    res = _decomposed(path, abi.PREC_FP64)
    print("decomposed oracle vs single domain:", [_rel(r[0], ref) for r in res], "steps", steps)
    for got, nsteps, t in res:
        assert nsteps == steps
        assert t == pytest.approx(ref_st[consts.ec["time"] - 1], abs=1e-15)
        assert _rel(got, ref) <= 1e-10
    # every rank ends with the same table
    assert np.array_equal(res[0][0], res[1][0])


@pytest.mark.gpu
def test_split_run_equals_time_loop_engine(engine_lib, cuda_ok):
    st, store = _sedov()
    params = {abi.P_REORDER_EVERY: 0}
    ref, ref_st, steps = _alone(os.path.join(ROOT, "sph_playground_b200", "_lib", "libsph.so"),
                                abi.PREC_FP64, st, store, T_END, params)
    with abi.Engine(st, store, "m6", lib=engine_lib) as e:
        for k, v in params.items():
            e.set_param(k, v)
        run = domain.SplitRun(e)
        run.start()
        run.run_to(T_END)
        got = e.get_store()
    assert run.steps == steps
    assert _rel(got, ref) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_decomposed_engine_equals_single_domain(engine_lib, cuda_ok, prec):
    path = os.path.join(ROOT, "sph_playground_b200", "_lib", "libsph.so")
    st, store = _sedov()
    ref, ref_st, steps = _alone(path, prec, st, store, T_END)
    res = _decomposed(path, prec, device="cuda")
    print("decomposed engine vs single domain:", [_rel(r[0], ref) for r in res], "steps", steps)
    tol = 1e-10 if prec == abi.PREC_FP64 else 1e-5
    for got, nsteps, _ in res:
        assert nsteps == steps
        assert _rel(got, ref) <= tol


@pytest.mark.gpu
def test_decomposed_device_exchange_single_rank(engine_lib, cuda_ok):
    """The exchange through device buffers (the NCCL path): one rank of an
    NCCL group owns every particle, so the columns go from the engine's
    table to a CUDA tensor, through the collective and back unchanged; the
    run equals the split run on the same engine to rounding."""
    import torch
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ["MASTER_PORT"] = str(29500 + (os.getpid() * 13) % 2000)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        torch.cuda.set_device(0)
        st, store = _sedov()
        run = domain.DecomposedRun(st, store, "m6", precision=abi.PREC_FP64, lib=engine_lib,
                                   device="cuda:0")
        run.start()
        run.run_to(T_END)
        got = run.global_store()
        nsteps = run.steps
        run.close()
    finally:
        dist.destroy_process_group()
    with abi.Engine(st, store, "m6", lib=engine_lib) as e:
        ref_run = domain.SplitRun(e)
        ref_run.start()
        ref_run.run_to(T_END)
        ref = e.get_store()
    assert nsteps == ref_run.steps
    # the rank's table holds the rows in Morton order, so the sums inside a
    # neighbour list run in another order
    assert _rel(got, ref) <= 1e-12
