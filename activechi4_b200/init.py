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

``reference_draws`` and ``initialize_systems`` instead reproduce the
reference program's own initialisation (initializeSystem,
MDcode/initialise.c:203-227) for a given srand() seed: the host makes the
reference's rand() draws (C library rand(), as the reference does) for the
grid sites, types, momenta and active set, and the device places the grid
(acg_set_lattice), runs the coldstart and breakxal ramps (acg_start_ramp) and
the final rescale, with the direction stream seeded as initializeGsl seeds
it.
"""
from __future__ import annotations

import ctypes
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


# ---------------------------------------------------------------------------
# the reference program's own initialisation, for a given srand() seed
RAND_MAX = 2147483647  # glibc


def _libc():
    lib = ctypes.CDLL(None)
    lib.srand.argtypes = [ctypes.c_uint]
    lib.rand.restype = ctypes.c_int
    return lib


def _pick(r: int, n: int) -> int:
    """floor((float)rand() / (float)RAND_MAX * N) in single precision
    (MDcode/initialise.c:50, :63; MDcode/active.c:17)."""
    f = np.float32(np.float32(r) / np.float32(RAND_MAX)) * np.float32(n)
    return int(np.floor(np.float64(np.float32(f))))


@dataclasses.dataclass
class ReferenceDraws:
    """The reference's random initial choices: grid site of every particle,
    types, momenta (with the reference's drift fix, typo included), active
    tags and directions, and the MT19937 seed initializeGsl derives."""

    site: np.ndarray
    type: np.ndarray
    p: np.ndarray
    act_tag: np.ndarray
    k: np.ndarray
    gsl_seed: int


def reference_draws(n: int, srand_seed: int, jobno: int = 0, clock: int = 1700000000,
                    nact: int | None = None) -> ReferenceDraws:
    """rand() draws of initializeSystem for srand(srand_seed), in the
    reference's order: initializeGsl's seed (time(NULL) + jobno + rand() +
    node, MDcode/initialise.c:5-11; `clock` stands for time(NULL)), GetFccGrid's
    site picks, type picks and momenta (:34-90), and
    selectRandomActiveParticles' permutation (MDcode/active.c:4-43)."""
    lib = _libc()
    lib.srand(ctypes.c_uint(srand_seed & 0xffffffff).value)
    rand = lib.rand
    gsl_seed = (clock + jobno + rand() + 0) & 0xffffffffffffffff
    free = np.ones(n, dtype=bool)
    site = np.empty(n, dtype=np.int32)
    k = 0
    while k < n:
        i = _pick(rand(), n)
        if i < n and free[i]:  # i == n reads past the reference's array: never taken here
            site[k] = i
            free[i] = False
            k += 1
    typ = np.zeros(n, dtype=np.int32)
    nb = n - int(0.80 * float(n))
    k = 0
    while k < nb:
        i = _pick(rand(), n)
        if i < n and typ[i] == 0:
            typ[i] = 1
            k += 1
    p = np.empty((n, 3))
    for i in range(n):
        for c in range(3):
            p[i, c] = float(rand()) / float(RAND_MAX) - 0.5
    # the reference's drift fix (MDcode/initialise.c:84-93): px by its mean,
    # py by the mean of pz, pz by the SUM of pz
    sx, sy, sz = 0.0, 0.0, 0.0
    for i in range(n):
        sx += p[i, 0]
        sy += p[i, 1]
        sz += p[i, 2]
    mx = sx / float(n)
    my = sz / float(n)
    p[:, 0] -= mx
    p[:, 1] -= my
    p[:, 2] -= sz
    nact = n_active(n) if nact is None else nact
    idx = np.arange(n, dtype=np.int64)
    for i in range(n):
        j = _pick(rand(), n)
        if j < n:
            idx[i], idx[j] = idx[j], idx[i]
    act_tag = np.full(n, -1, dtype=np.int32)
    act_tag[idx[:nact]] = np.arange(nact, dtype=np.int32)
    kk = np.where(np.arange(nact) < nact // 2, 1, -1).astype(np.int32)
    return ReferenceDraws(site, typ, p, act_tag, np.stack([kk, kk.copy(), kk.copy()]), int(gsl_seed))


def initialize_systems(engine, draws: dict, T, rate: float = 0.1) -> dict:
    """initializeSystem on the device for the systems in `draws` ({system:
    ReferenceDraws}) at temperatures T ({system: T} or one value): grid
    placement, the coldstart ramp to T, the breakxal ramp from 1.5 T to T and
    the final rescale to T (MDcode/initialise.c:203-227).  Systems whose ramps
    differ in length pad them at their end temperature, so the engine's
    other systems must be ramping too.  Returns the ramp lengths."""
    Ts = {s: (T[s] if isinstance(T, dict) else float(T)) for s in draws}
    for s, d in draws.items():
        engine.set_lattice(s, d.site, d.type, d.p, d.act_tag)
        if engine.nact(s):
            engine.set_directions(s, d.k)
        engine.seed_shuffle(s, d.gsl_seed)
    lengths = {}
    for name, lo, hi in (("coldstart", 0.5, 1.0), ("breakxal", 1.5, 1.0)):
        ks = {s: engine.start_ramp(s, lo * Ts[s], hi * Ts[s], rate) for s in draws}
        kmax = max(ks.values())
        for s in draws:
            if ks[s] < kmax:
                engine.extend_ramp(s, kmax)
        engine.step(kmax)
        lengths[name] = ks
    for s in draws:
        engine.adjust_temperature(s, Ts[s])
    return lengths
