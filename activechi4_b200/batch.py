"""Many independent replicas in one engine (one launch per kernel per step).

`replica_set` draws the replica parameters of the batched workload: N uniform
in [n_min, n_max] with an 80:20 composition at density 1.2, T from
{0.45, 0.5, 0.6}, f0 from {0, 0.5, 1, 2}, tau_p from {0.1, 1, 10} time units
(20, 200, 2000 steps of 0.005), seeded.  `combine_chi4` adds the observable
sums of replicas with equal (T, f0, tau_p), so Q and chi4 are averaged over
origins and replicas together.
"""
from __future__ import annotations

from collections import defaultdict

import numpy as np

from .engine import Engine, default_params, observables_from_sums
from .init import lattice_state

T_SET = (0.45, 0.5, 0.6)
F0_SET = (0.0, 0.5, 1.0, 2.0)
TAU_SET = (20, 200, 2000)


def replica_set(count=256, n_min=500, n_max=4000, seed=0, precision=1, skin=0.35):
    rng = np.random.default_rng(seed)
    out = []
    for r in range(count):
        n = int(rng.integers(n_min, n_max + 1))
        T = float(rng.choice(T_SET))
        f0 = float(rng.choice(F0_SET))
        tau = int(rng.choice(TAU_SET))
        p = default_params(n, T=T, f0=f0, tau_p_steps=tau, precision=precision, seed=1000 + r,
                           list_mode=1, rebuild_factor=4.0, skin=skin)
        out.append((p, lattice_state(n, T, seed=seed * 100000 + r)))
    return out


def make_engine(replicas, device=0):
    e = Engine([p for p, _ in replicas], device=device)
    rng = np.random.default_rng(7)
    for r, (p, st) in enumerate(replicas):
        e.set_state(r, st)
        q = e.thermo(r)["q"]
        e.set_nhc(r, np.zeros(3), np.sqrt(p.T * q) * rng.standard_normal(3))
    return e


def combine_chi4(e: Engine, replicas, dt=0.005):
    groups = defaultdict(list)
    for r, (p, _) in enumerate(replicas):
        groups[(p.T, p.f0, p.tau_p_steps)].append(r)
    out = {}
    for key, members in groups.items():
        off, s = e.obs_sums(members[0])
        tot = np.zeros_like(s)
        for r in members:
            tot += e.obs_sums(r)[1]
        out[key] = observables_from_sums(off, tot, dt)
    return out
