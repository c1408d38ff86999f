"""Synthetic initial configurations for the active Kob-Andersen mixture.

Host-side set-up, run once per system (not part of the timestep).  It follows
the reference's initialisation:

* ``lattice_state`` — particles on a random permutation of the points of an
  n^3 grid (n = smallest integer with n^3 >= N) in reduced units, 20% of them
  type B, momenta uniform in [-0.5, 0.5) with the mean removed, rescaled to
  temperature T (MDcode/initialise.c:34-101 GetFccGrid, :140-151
  adjustInitialTemp).  The reference's drift fix has a typo (``py = pz/N`` at
  MDcode/initialise.c:88) that leaves a net momentum; this generator removes
  the mean of every component.
* ``select_active`` — a random set of Nact = (int)(0.1 N) particles drawn from
  all N (not only type A), with direction components +1 for the first Nact/2
  and -1 for the rest, per component, so the net active force is zero when
  Nact is even (MDcode/active.c:4-43).

The random streams are numpy's, seeded; the reference seeds from time() so
its streams cannot be reproduced anyway.
"""
from __future__ import annotations

import dataclasses

import numpy as np

DENSITY = 1.2
ACTIVE_DENSITY = 0.1


def box_length(n: int, density: float = DENSITY) -> float:
    """L = pow(N/DENSITY, 0.33333333) as in MDcode/main.c:465."""
    return float(np.power(float(n) / density, 0.33333333))


def n_active(n: int, active_density: float = ACTIVE_DENSITY) -> int:
    """Nact = (int)((double)N * ACTIVE_DENSITY) (MDcode/global.h:55)."""
    return int(float(n) * active_density)


@dataclasses.dataclass
class State:
    """One system in the reference's units.

    x, xu: [N,3] reduced coordinates (wrapped to [0,1), and unfolded);
    p: [N,3] momenta (unit mass); type: [N] 0=A 1=B; act_tag: [N] -1 or the
    index into the direction arrays; k: [3, Nact] direction components."""

    L: float
    x: np.ndarray
    xu: np.ndarray
    p: np.ndarray
    type: np.ndarray
    act_tag: np.ndarray
    k: np.ndarray

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    @property
    def nact(self) -> int:
        return int(self.k.shape[1])

    def copy(self) -> "State":
        return State(self.L, self.x.copy(), self.xu.copy(), self.p.copy(), self.type.copy(),
                     self.act_tag.copy(), self.k.copy())


def select_active(n: int, rng: np.random.Generator, nact: int | None = None):
    nact = n_active(n) if nact is None else nact
    idx = rng.permutation(n)[:nact]
    act_tag = np.full(n, -1, dtype=np.int32)
    act_tag[idx] = np.arange(nact, dtype=np.int32)
    k = np.where(np.arange(nact) < nact // 2, 1, -1).astype(np.int32)
    return act_tag, np.stack([k, k.copy(), k.copy()])


def lattice_state(n: int, T: float, seed: int, density: float = DENSITY,
                  nact: int | None = None) -> State:
    rng = np.random.default_rng(seed)
    L = box_length(n, density)
    m = 1
    while m * m * m < n:
        m += 1
    g = np.arange(m * m * m)
    pts = np.stack([g % m, (g // m) % m, g // (m * m)], axis=1).astype(np.float64) / m
    x = pts[rng.permutation(m * m * m)[:n]]
    typ = np.zeros(n, dtype=np.int32)
    typ[rng.permutation(n)[: n - int(0.8 * n)]] = 1
    p = rng.random((n, 3)) - 0.5
    p -= p.mean(axis=0)
    ke = 0.5 * float((p * p).sum())
    p *= np.sqrt(T / (2.0 * ke / (3.0 * n - 3.0)))
    act_tag, k = select_active(n, rng, nact)
    return State(L, x.copy(), x.copy(), p, typ, act_tag, k)


def shuffle_directions(k: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """A uniformly random permutation of each direction component (keeps the
    +1/-1 counts, so a zero net active force stays zero)."""
    return np.stack([rng.permutation(row) for row in k]).astype(np.int32)
