"""Python mirror of the C ABI: an Engine holds one or many systems on a GPU.

The names follow the reference's routines (MDcode/subroutine.h): ``rebuild``
is update_cell_list, ``compute_forces`` is calculate_forces, ``step`` is the
run() loop body (ShuffleActDirec when due + AdvanceTimeNVTNoseHoover),
``shuffle`` is ShuffleActDirec, ``set_nhc`` is the chain set-up of
InitialiseNoseHoover.  Arrays are numpy, in the caller's particle order and the
reference's units.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _abi
from ._abi import acg_params, acg_thermo, check


def default_params(n: int, **kw) -> acg_params:
    p = acg_params()
    check(_abi.lib().acg_params_default(C.byref(p), int(n)))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(f"acg_params has no field {k}")
        setattr(p, k, v)
    return p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f64(a, shape):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))


def _i32(a, shape):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(shape))


def measure_fp64_peak(device: int = 0) -> float:
    """FP64 FMA throughput of the device in TFLOP/s."""
    t = C.c_double()
    check(_abi.lib().acg_measure_fp64_peak(int(device), C.byref(t)))
    return t.value


def release_retired():
    """Destroy the CUDA graphs of closed engines (waits for the device)."""
    check(_abi.lib().acg_release_retired())


def observables_from_sums(offset, sums, dt=0.005) -> dict:
    """Per-bin averages from summed (Q, Q^2, msd, msd_d4, msd_r4, Fs, count);
    sums of several replicas with equal parameters may be added first (chi4
    across replicas).  chi4 = <Q^2> - <Q>^2, not multiplied by N
    (Analysis/overlap.c:118)."""
    s = np.asarray(sums, dtype=np.float64)
    cnt = s[:, 6]
    m = cnt > 0
    c = cnt[m]
    Q = s[m, 0] / c
    return {"t": np.asarray(offset)[m] * dt, "offset": np.asarray(offset)[m], "count": c.astype(np.int64),
            "Q": Q, "chi4": s[m, 1] / c - Q * Q, "msd": s[m, 2] / c, "msd_d4": s[m, 3] / c,
            "msd_r4": s[m, 4] / c, "Fs": s[m, 5] / c}


def qvectors(L: float, q: float, count: int = 48, tol: float = 0.1):
    """Integer vectors n with |2 pi n / L| within tol of q (up to `count`,
    nearest first, sign-symmetric pairs kept together)."""
    nmax = int(np.ceil((q + tol) * L / (2 * np.pi))) + 1
    r_lo = max(q - tol, 0.0) * L / (2 * np.pi)
    r_hi = (q + tol) * L / (2 * np.pi)
    # only the columns (nx, ny) that reach the shell, and the nz range there
    g = np.arange(-nmax, nmax + 1)
    nx, ny = (a.ravel() for a in np.meshgrid(g, g, indexing="ij"))
    rho2 = (nx * nx + ny * ny).astype(np.float64)
    keep = rho2 <= r_hi * r_hi + 1.0
    nx, ny, rho2 = nx[keep], ny[keep], rho2[keep]
    zmax = np.floor(np.sqrt(np.maximum(r_hi * r_hi - rho2, 0.0)) + 1.0).astype(np.int64)
    zmin = np.maximum(np.ceil(np.sqrt(np.maximum(r_lo * r_lo - rho2, 0.0))) - 1.0, 0.0).astype(np.int64)
    rows = []
    for sgn in (1, -1):
        lo = zmin if sgn > 0 else np.maximum(zmin, 1)  # z = 0 once
        cnt = np.maximum(zmax - lo + 1, 0)
        base = np.repeat(lo, cnt)
        off = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        rows.append(np.stack([np.repeat(nx, cnt), np.repeat(ny, cnt), sgn * (base + off)], axis=1))
    n = np.concatenate(rows)
    qq = 2 * np.pi * np.sqrt((n * n).sum(axis=1)) / L
    sel = np.abs(qq - q) <= tol
    n, qq = n[sel], qq[sel]
    order = np.lexsort((n[:, 2], n[:, 1], n[:, 0], np.abs(qq - q)))
    return n[order][:count].astype(np.int32)


def footprint(params: Sequence[acg_params]) -> int:
    arr = (acg_params * len(params))(*params)
    out = C.c_size_t(0)
    check(_abi.lib().acg_footprint(arr, len(params), C.byref(out)))
    return int(out.value)


class Engine:
    """A batch of independent systems resident on one GPU."""

    def __init__(self, params: acg_params | Sequence[acg_params], device: int = 0):
        if isinstance(params, acg_params):
            params = [params]
        self.params = list(params)
        self._lib = _abi.lib()
        arr = (acg_params * len(self.params))(*self.params)
        h = C.c_void_p()
        check(self._lib.acg_create(arr, len(self.params), int(device), C.byref(h)))
        self.h = h
        self._meta = {}
        self.sizes = []
        for r in range(len(self.params)):
            n, na = C.c_int(), C.c_int()
            check(self._lib.acg_system_size(self.h, r, C.byref(n), C.byref(na)))
            self.sizes.append((n.value, na.value))

    def close(self):
        if getattr(self, "h", None):
            self._lib.acg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def nsys(self) -> int:
        return len(self.params)

    def n(self, sys: int = 0) -> int:
        return self.sizes[sys][0]

    def nact(self, sys: int = 0) -> int:
        return self.sizes[sys][1]

    # -- state -----------------------------------------------------------
    def set_state(self, sys: int, state, set_directions: bool = True):
        n = self.n(sys)
        x = _f64(state.x, (n, 3))
        xu = _f64(state.xu, (n, 3))
        p = _f64(state.p, (n, 3))
        t = _i32(state.type, (n,))
        a = _i32(state.act_tag, (n,))
        check(self._lib.acg_set_state(self.h, sys, _ptr(x), _ptr(xu), _ptr(p), _ptr(t), _ptr(a)))
        self._meta[sys] = (float(state.L), t.copy(), a.copy())
        if set_directions and self.nact(sys):
            self.set_directions(sys, state.k)

    def get_state(self, sys: int = 0):
        n = self.n(sys)
        x, xu, p, F = (np.empty((n, 3)) for _ in range(4))
        check(self._lib.acg_get_state(self.h, sys, _ptr(x), _ptr(xu), _ptr(p), _ptr(F)))
        return x, xu, p, F

    def state_meta(self, sys: int = 0) -> dict:
        """Box length, types and active tags of the last set_state (constant
        during a run: the device keeps particles in id order at the ABI)."""
        if sys not in self._meta:
            raise KeyError(f"system {sys} has no state loaded")
        L, t, a = self._meta[sys]
        return {"L": L, "type": t, "act_tag": a}

    def set_directions(self, sys: int, k):
        na = self.nact(sys)
        kk = _i32(k, (3 * na,))
        check(self._lib.acg_set_directions(self.h, sys, _ptr(kk)))

    def get_directions(self, sys: int = 0):
        na = self.nact(sys)
        k = np.zeros(3 * max(na, 1), dtype=np.int32)
        check(self._lib.acg_get_directions(self.h, sys, _ptr(k)))
        return k[: 3 * na].reshape(3, na)

    def shuffle(self, sys: int = 0):
        """ShuffleActDirec now (MDcode/active.c:45-85)."""
        check(self._lib.acg_shuffle_directions(self.h, sys))

    def seed_shuffle(self, sys: int, seed: int):
        """Reseed the system's MT19937 direction stream (gsl_rng_set)."""
        check(self._lib.acg_seed_shuffle(self.h, sys, C.c_uint64(int(seed))))

    def fix_drift(self, sys: int = 0):
        """fixDrift now (MDcode/initialise.c:104-138)."""
        check(self._lib.acg_fix_drift(self.h, sys))

    def adjust_temperature(self, sys: int, T: float) -> float:
        """adjustInitialTemp (MDcode/initialise.c:141-151); returns inst_T after."""
        t = C.c_double()
        check(self._lib.acg_adjust_temperature(self.h, sys, float(T), C.byref(t)))
        return t.value

    def start_ramp(self, sys: int, T_start: float, T_end: float, rate: float) -> int:
        """Arm a coldstart / breakxal ramp (MDcode/initialise.c:166-201); returns
        its step count (the ramp runs in the next that many steps)."""
        k = C.c_int64()
        check(self._lib.acg_start_ramp(self.h, sys, float(T_start), float(T_end), float(rate), C.byref(k)))
        return int(k.value)

    def extend_ramp(self, sys: int, total_steps: int):
        """Pad an armed ramp to total_steps (the extra steps hold its end T)."""
        check(self._lib.acg_extend_ramp(self.h, sys, int(total_steps)))

    def set_lattice(self, sys: int, site, type_, p, act_tag):
        """GetFccGrid placement on the device from the caller's grid sites."""
        n = self.n(sys)
        si = _i32(site, (n,))
        t = _i32(type_, (n,))
        pp = _f64(p, (n, 3))
        a = _i32(act_tag, (n,))
        check(self._lib.acg_set_lattice(self.h, sys, _ptr(si), _ptr(t), _ptr(pp), _ptr(a)))

    def set_nhc(self, sys: int, eta, p_eta):
        e = _f64(eta, (3,))
        pe = _f64(p_eta, (3,))
        check(self._lib.acg_set_nhc(self.h, sys, _ptr(e), _ptr(pe)))

    def set_barostat(self, sys: int, eta_baro, p_eta_baro, p_eps: float):
        """Barostat chain and p_eps of a Nose-Hoover NPT system (thermostat 5)."""
        e = _f64(eta_baro, (3,))
        pe = _f64(p_eta_baro, (3,))
        check(self._lib.acg_set_barostat(self.h, sys, _ptr(e), _ptr(pe), float(p_eps)))

    def set_temperature(self, sys: int, T: float):
        check(self._lib.acg_set_temperature(self.h, sys, float(T)))

    # -- stepping --------------------------------------------------------
    def rebuild(self):
        check(self._lib.acg_rebuild(self.h))

    def compute_forces(self):
        check(self._lib.acg_compute_forces(self.h))

    def step(self, nsteps: int):
        check(self._lib.acg_step(self.h, int(nsteps)))

    def step_eager(self, nsteps: int):
        check(self._lib.acg_step_eager(self.h, int(nsteps)))

    def sync(self):
        check(self._lib.acg_sync(self.h))

    def poll(self) -> bool:
        """True when all queued work has finished (does not block)."""
        d = C.c_int()
        check(self._lib.acg_poll(self.h, C.byref(d)))
        return bool(d.value)

    def thermo(self, sys: int = 0) -> dict:
        t = acg_thermo()
        rc = self._lib.acg_get_thermo(self.h, sys, C.byref(t))
        out = {f: getattr(t, f) for f, _ in acg_thermo._fields_}
        for f in ("eta", "p_eta", "q", "eta_baro", "p_eta_baro"):
            out[f] = np.array(list(out[f]))
        check(rc)
        return out

    def cells(self, sys: int = 0):
        dims = np.zeros(3, dtype=np.int32)
        nc = C.c_int()
        check(self._lib.acg_get_cells(self.h, sys, _ptr(dims), C.byref(nc), None, None))
        counts = np.zeros(nc.value, dtype=np.int32)
        members = np.zeros(self.n(sys), dtype=np.int32)
        check(self._lib.acg_get_cells(self.h, sys, _ptr(dims), C.byref(nc), _ptr(counts), _ptr(members)))
        return dims, counts, members

    # -- in-place observables -------------------------------------------
    def obs_configure(self, sys: int, run_length: int, num_origins: int = 200, factor: float = 1.4,
                      max_interval: int = 0, a: float = 0.3, qvec=None, max_live_origins: int = 64):
        q = np.ascontiguousarray(np.zeros((0, 3)) if qvec is None else qvec, dtype=np.int32).reshape(-1, 3)
        cfg = _abi.acg_obs_config(int(run_length), int(num_origins), float(factor), int(max_interval),
                                  float(a), int(q.shape[0]), q.ctypes.data_as(C.c_void_p) if q.size else None,
                                  int(max_live_origins))
        check(self._lib.acg_obs_configure(self.h, sys, C.byref(cfg)))

    def obs_sums(self, sys: int = 0):
        nb = C.c_int()
        check(self._lib.acg_obs_sums(self.h, sys, C.byref(nb), None, None))
        off = np.zeros(nb.value, dtype=np.int64)
        sums = np.zeros((nb.value, 7))
        check(self._lib.acg_obs_sums(self.h, sys, C.byref(nb), _ptr(off), _ptr(sums)))
        return off, sums

    def observables(self, sys: int = 0, dt: float = 0.005) -> dict:
        """Q(t), chi4(t), MSD and moments, Fs(q,t) per time bin with data."""
        off, s = self.obs_sums(sys)
        return observables_from_sums(off, s, dt)

    # -- tuning / timing -------------------------------------------------
    def set_launch(self, tpp: int, block: int):
        check(self._lib.acg_set_launch(self.h, int(tpp), int(block)))

    def set_group_tpp(self, gtpp: int):
        check(self._lib.acg_set_group_tpp(self.h, int(gtpp)))

    def set_box_cells(self, cells: int):
        """Cells per block of the whole-box kernels (1..8)."""
        check(self._lib.acg_set_box_cells(self.h, int(cells)))

    def get_box_cells(self) -> int:
        c = C.c_int()
        check(self._lib.acg_get_box_cells(self.h, C.byref(c)))
        return c.value

    def get_launch(self):
        t, b = C.c_int(), C.c_int()
        check(self._lib.acg_get_launch(self.h, C.byref(t), C.byref(b)))
        return t.value, b.value

    def time_stage(self, stage: int, reps: int = 20) -> float:
        ms = C.c_double()
        check(self._lib.acg_time_stage(self.h, int(stage), int(reps), C.byref(ms)))
        return ms.value

    def bench_steps(self, nsteps: int, flush_bytes: int = 256 << 20):
        """(device ms summed over the timed launches of exactly nsteps steps,
        kernel launches inside them)"""
        ms = C.c_double()
        nl = C.c_int64()
        check(self._lib.acg_bench_steps(self.h, int(nsteps), int(flush_bytes), C.byref(ms), C.byref(nl)))
        return ms.value, nl.value

    def prepare(self):
        """Prime and build the step graphs now (may wait for queued device
        work; safe to call from another thread)."""
        check(self._lib.acg_prepare(self.h))

    def set_priority(self, level: int):
        """Stream priority among engines on the device (0 = default, higher
        first)."""
        check(self._lib.acg_set_priority(self.h, int(level)))

    @property
    def stream(self) -> int:
        return int(self._lib.acg_stream(self.h) or 0)
