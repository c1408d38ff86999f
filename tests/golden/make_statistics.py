"""Generate tests/golden/stats_n1000.npz: the reference program's statistics
at N = 1000 (T = 0.45, f0 = 1.0, tau_p = 200 steps, dt = 0.005), for the
statistical parity test of the GPU path (tests/test_gpu_statistics.py).

Protocol, per seed s (one process per seed: the reference sets up its arrays
once per process):
  1. the reference's own initializeSystem for srand(SRAND0 + s), jobno s
     (random grid, active set, coldstart and breakxal ramps at T;
     MDcode/initialise.c:203-227);
  2. Nose-Hoover chain eta = 0, p_eta = P_ETA[s] (drawn here, handed to both
     sides); fixDrift;
  3. EQUIL steps of the run() loop body from loop index 0 (ShuffleActDirec
     every TAU_per steps before the step, fixDrift after every 100000th;
     MDcode/main.c:244-265);
  4. RUN more steps of the same loop (index EQUIL ..), with the unfolded
     coordinates taken after every step the log-time schedule needs (run
     length RUN, 200 origins, factor 1.4: prepareSavingArray,
     MDcode/main.c:62-119), analysed by the restatement of the reference's
     Analysis program (oracle/observables.py, pinned to it by
     tests/test_observables_vs_reference_analysis.py): per time bin the sums
     of Q (a = 0.3), Q^2, MSD, its 4th moments and Fs at |q| = 7.25.
The NVE energy drift of the reference from the golden N = 1000 state (f0 = 0,
NVE_STEPS leap-frog steps) is stored beside them.

Runs the reference compiled from its sources (oracle/_ref/libref_md_n1000.so);
about 3 CPU-minutes per seed, seeds in parallel on the host's cores.

Usage:  python tests/golden/make_statistics.py [--seeds 16] [--procs 8]
"""
from __future__ import annotations

import argparse
import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

N = 1000
T = 0.45
F0 = 1.0
EQUIL = 20000
RUN = 100000
ORIGINS = 200
FACTOR = 1.4
LIVE = 128
A = 0.3
Q = 7.25
SRAND0 = 9000
NVE_STEPS = 20000
NVE_EVERY = 1000


def p_eta_for(seed):
    """Initial thermostat momenta of seed s (InitialiseNoseHoover draws
    p_eta ~ sqrt(T Q_j) N(0,1), MDcode/time_evolve.c:476-493)."""
    from activechi4_b200.init import box_length  # noqa: F401
    tau = 0.2
    q = np.array([(3.0 * N - 3.0) * T * tau * tau, T * tau * tau, T * tau * tau])
    return np.sqrt(T * q) * np.random.default_rng(seed).standard_normal(3)


def one_seed(s):
    from activechi4_b200.engine import qvectors
    from activechi4_b200.init import box_length
    from oracle import Reference
    from oracle.observables import analyse, log_pairs
    r = Reference(N)
    with tempfile.TemporaryDirectory() as d:
        r.initialize_system(T, F0, s, SRAND0 + s, d)
    r.set_nhc(np.zeros(3), p_eta_for(s))
    r.fix_drift()
    r.run(EQUIL, start=0, shuffle=True, drift=True)
    L = box_length(N)
    qv = qvectors(L, Q)
    _, pairs = log_pairs(RUN, ORIGINS, FACTOR, 0, LIVE)
    need = sorted({t for p in pairs for t in p[:2]})
    frames, done = {}, 0
    for t in need:  # frame t: the state after loop index EQUIL + t
        r.run(t + 1 - done, start=EQUIL + done, shuffle=True, drift=True)
        done = t + 1
        frames[t] = r.get_state()[1].copy()
    offs, sums = analyse(frames, L, RUN, ORIGINS, FACTOR, 0, A, qv, LIVE)
    return s, offs, sums


def nve_drift():
    """Total energy per particle of the reference every NVE_EVERY NVE steps
    from the golden N = 1000 state with f0 = 0."""
    from activechi4_b200.init import State
    from oracle import Reference
    g = dict(np.load(os.path.join(HERE, "ka_n1000.npz")))
    st = State(float(g["L"]), g["x"], g["xu"], g["p"], g["type"], g["act_tag"], g["k"])
    r = Reference(N)
    r.setup(st, 0.45, 0.0)
    e = []
    for k in range(NVE_STEPS // NVE_EVERY + 1):
        if k:
            r.run_nve(NVE_EVERY)
        sc = r.scalars()
        x, xu, p, F = r.get_state()
        e.append((sc["pe"] + 0.5 * float((p * p).sum())) / N)
    return np.array(e)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=16)
    ap.add_argument("--procs", type=int, default=min(8, os.cpu_count() or 1))
    args = ap.parse_args()
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.procs, maxtasksperchild=1) as pool:
        res = sorted(pool.map(one_seed, range(args.seeds), chunksize=1))
        energy = pool.apply(nve_drift)
    offs = res[0][1]
    sums = np.stack([r[2] for r in res])
    out = os.path.join(HERE, "stats_n1000.npz")
    np.savez_compressed(out, offsets=offs, sums=sums, seeds=np.arange(args.seeds), n=N, T=T, f0=F0,
                        equil=EQUIL, run=RUN, origins=ORIGINS, factor=FACTOR, live=LIVE, a=A, q=Q,
                        srand0=SRAND0, nve_energy=energy, nve_every=NVE_EVERY)
    print("wrote", out, sums.shape)


if __name__ == "__main__":
    main()
