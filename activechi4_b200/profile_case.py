"""Small, self-contained cases for profiling one stage of the timestep.

Used as the command under Nsight Compute; prints nothing but a summary line.

  python -m activechi4_b200.profile_case --stage force --n 100000 --reps 3
  python -m activechi4_b200.profile_case --stage step --n 100000 --reps 64

  python -m activechi4_b200.profile_case --stage step --replicas 256 --reps 64

Stages: force (pair forces only, the force kernel's work), rebuild (cell
build + neighbour lists at the current positions), step (whole timesteps,
launched kernel by kernel so each launch is listed separately), latency (no
profiler: one system at T = 0.45 from a lattice, NHC, 200 steps, then the
step time of the production graphs over 640 steps and the kick/drift, force
and rebuild stages alone, CUDA events; prints one JSON line).  The state is
a seeded lattice disordered by `--melt` steps at T=2.0.  With `--replicas R`
the engine holds the batched workload instead: R FP32 replicas with N uniform
in [500, 4000] and parameters from the batched sets (`batch.replica_set`,
seed 11), melted `--melt` steps at T=2.0 and `--melt` at their own T, launch
shape threads-per-particle 4 / block 128 / group and box TPP 2.
"""
import argparse
import ctypes

import numpy as np

from activechi4_b200 import Engine, default_params
from activechi4_b200.init import lattice_state


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--stage", default="force", choices=["force", "rebuild", "step", "latency"])
    ap.add_argument("--n", type=int, default=100000)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--melt", type=int, default=256)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--tpp", type=int, default=0)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--list-mode", type=int, default=0)
    ap.add_argument("--group-tpp", type=int, default=0)
    ap.add_argument("--replicas", type=int, default=0)
    ap.add_argument("--tpp-force", type=int, default=0, help="latency: threads per particle of the force kernels")
    a = ap.parse_args()
    if a.stage == "latency":
        latency(a)
        return
    if a.replicas:
        from activechi4_b200.batch import make_engine, replica_set
        reps = replica_set(count=a.replicas, seed=11, precision=1)
        e = make_engine(reps)
        for r in range(len(reps)):
            e.set_temperature(r, 2.0)
        e.step(a.melt)
        for r, (p, _) in enumerate(reps):
            e.set_temperature(r, p.T)
        e.step(a.melt)
        e.set_launch(a.tpp or 4, a.block or 128)
        e.set_group_tpp(a.group_tpp or 2)
    else:
        e = Engine(default_params(a.n, T=2.0, precision=a.precision, list_mode=a.list_mode))
        if a.tpp:
            e.set_launch(a.tpp, a.block or 128)
        if a.group_tpp:
            e.set_group_tpp(a.group_tpp)
        e.set_state(0, lattice_state(a.n, 2.0, seed=3))
        e.set_nhc(0, np.zeros(3), np.array([0.1, 0.0, -0.1]))
        e.step(a.melt)
        e.set_temperature(0, 0.45)
    e.sync()
    # profiler range (ncu --profile-from-start off): the stage alone, without
    # the set-up launches
    cu = ctypes.CDLL("libcuda.so.1")
    cu.cuProfilerStart()
    if a.stage == "force":
        ms = e.time_stage(1, a.reps)
    elif a.stage == "rebuild":
        ms = e.time_stage(2, a.reps)
    else:
        e.step_eager(a.reps)
        e.sync()
        ms = float("nan")
    cu.cuProfilerStop()
    th = e.thermo(0)
    if a.replicas:
        th["rebuilds"] = sum(e.thermo(r)["rebuilds"] for r in range(e.nsys))
    print(f"stage={a.stage} n={a.n} replicas={a.replicas} reps={a.reps} ms/launch={ms:.4f} rebuilds={th['rebuilds']} "
          f"overflow={th['overflow']} launch={e.get_launch()}")


def latency(a):
    """Step latency of one small system alone (the served workload's runs)."""
    import json
    e = Engine(default_params(a.n, T=0.45, f0=1.0, precision=a.precision, list_mode=a.list_mode,
                              rebuild_factor=4.0))
    if a.tpp_force:
        e.set_group_tpp(a.tpp_force)
    if a.tpp:
        e.set_launch(a.tpp, a.block or 128)
    e.set_state(0, lattice_state(a.n, 0.45, seed=5))
    e.set_nhc(0, np.zeros(3), np.array([0.1, 0.0, 0.0]))
    e.step(200)
    e.sync()
    ms, nl = e.bench_steps(640, 0)
    out = {"n": a.n, "precision": a.precision, "step_us": 1e3 * ms / 640, "launches_per_step": nl / 640,
           "force_us": 1e3 * e.time_stage(1, 50), "rebuild_us": 1e3 * e.time_stage(2, 10),
           "kick_drift_us": 1e3 * e.time_stage(0, 50), "rebuilds": e.thermo(0)["rebuilds"],
           "launch": e.get_launch()}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
