"""Small, self-contained cases for profiling one stage of the timestep.

Used as the command under Nsight Compute; prints nothing but a summary line.

  python -m activechi4_b200.profile_case --stage force --n 100000 --reps 3
  python -m activechi4_b200.profile_case --stage step --n 100000 --reps 64

Stages: force (pair forces only, the force kernel's work), rebuild (cell
build + neighbour lists at the current positions), step (whole timesteps,
launched kernel by kernel so each launch is listed separately).  The state is
a seeded lattice disordered by `--melt` steps at T=2.0.
"""
import argparse

import numpy as np

from activechi4_b200 import Engine, default_params
from activechi4_b200.init import lattice_state


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--stage", default="force", choices=["force", "rebuild", "step"])
    ap.add_argument("--n", type=int, default=100000)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--melt", type=int, default=256)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--tpp", type=int, default=0)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--list-mode", type=int, default=0)
    ap.add_argument("--group-tpp", type=int, default=0)
    a = ap.parse_args()
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
    if a.stage == "force":
        ms = e.time_stage(1, a.reps)
    elif a.stage == "rebuild":
        ms = e.time_stage(2, a.reps)
    else:
        e.step_eager(a.reps)
        e.sync()
        ms = float("nan")
    th = e.thermo(0)
    print(f"stage={a.stage} n={a.n} reps={a.reps} ms/launch={ms:.4f} rebuilds={th['rebuilds']} "
          f"overflow={th['overflow']} launch={e.get_launch()}")


if __name__ == "__main__":
    main()
