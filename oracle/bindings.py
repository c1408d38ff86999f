"""ctypes bindings for the oracle libraries.  TEST INFRASTRUCTURE ONLY.

``Oracle`` wraps the project's restatement (acg_oracle.c); ``Reference`` wraps
the reference engine compiled from its own sources (ref_harness.c + MDcode).
Both take and return the reference's units: reduced coordinates in [0,1),
momenta, forces in absolute units.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def oracle_lib_path() -> str:
    return os.path.join(HERE, "_build", "libacg_oracle.so")


def ref_lib_path(n: int, kind: str = "ref") -> str:
    return os.path.join(HERE, "_ref", f"lib{kind}_md_n{n}.so")


def reference_available(n: int, kind: str = "ref") -> bool:
    return os.path.exists(ref_lib_path(n, kind))


def build_oracle() -> str:
    """Compile the restatement (gcc only, no reference sources needed)."""
    path = oracle_lib_path()
    src = [os.path.join(HERE, f) for f in ("acg_oracle.c", "acg_oracle.h")]
    if not os.path.exists(path) or any(os.path.getmtime(s) > os.path.getmtime(path) for s in src):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        subprocess.check_call(["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-o", path,
                               os.path.join(HERE, "acg_oracle.c"), "-lm"])
    return path


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if shape is None else a.reshape(shape)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


_olib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        lib = C.CDLL(build_oracle())
        v = C.c_void_p
        lib.ora_create.restype = v
        lib.ora_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                   C.c_double, C.c_int]
        lib.ora_destroy.argtypes = [v]
        lib.ora_set_state.argtypes = [v, _dp, _dp, _dp, _ip, _ip]
        lib.ora_get_state.argtypes = [v, _dp, _dp, _dp, _dp]
        lib.ora_set_k.argtypes = [v, _ip]
        lib.ora_get_k.argtypes = [v, _ip]
        lib.ora_set_nhc.argtypes = [v, _dp, _dp]
        lib.ora_get_nhc.argtypes = [v, _dp]
        lib.ora_set_thermostat.argtypes = [v, C.c_double]
        lib.ora_seed_rng.argtypes = [v, C.c_ulong]
        lib.ora_shuffle.argtypes = [v]
        lib.ora_rebuild.argtypes = [v]
        lib.ora_forces.argtypes = [v, _dp, _dp]
        lib.ora_run.restype = C.c_int
        lib.ora_run.argtypes = [v, C.c_long, C.c_int, C.c_int, C.c_int]
        lib.ora_fix_drift.argtypes = [v]
        lib.ora_adjust_temp.restype = C.c_double
        lib.ora_adjust_temp.argtypes = [v, C.c_double]
        lib.ora_ramp.restype = C.c_long
        lib.ora_ramp.argtypes = [v, C.c_double, C.c_double, C.c_double]
        lib.ora_run_nve.restype = C.c_int
        lib.ora_run_nve.argtypes = [v, C.c_int]
        lib.ora_get_scalars.argtypes = [v, _dp]
        lib.ora_get_cells.restype = C.c_int
        lib.ora_get_cells.argtypes = [v, _ip, C.c_void_p, C.c_void_p]
        lib.ora_get_neighbors.restype = C.c_long
        lib.ora_get_neighbors.argtypes = [v, C.c_void_p, C.c_void_p]
        lib.ora_cell_geometry.argtypes = [C.c_double, _ip, _dp]
        lib.ora_log_schedule.restype = C.c_int
        lib.ora_log_schedule.argtypes = [C.c_ulonglong, C.c_int, C.c_double, _up, C.c_int]
        _olib = lib
    return _olib


class _Common:
    """Shared readers; subclasses provide self._call(name, *args)."""

    n: int
    nact: int

    def get_state(self):
        x, xu, p, F = (np.zeros((self.n, 3)) for _ in range(4))
        self._call("get_state", x, xu, p, F)
        return x, xu, p, F

    def get_k(self):
        k = np.zeros(3 * max(self.nact, 1), dtype=np.int32)
        self._call("get_k", k)
        return k[: 3 * self.nact].reshape(3, self.nact)

    def get_nhc(self):
        o = np.zeros(9)
        self._call("get_nhc", o)
        return o[0:3].copy(), o[3:6].copy(), o[6:9].copy()

    def forces(self):
        F = np.zeros((self.n, 3))
        o = np.zeros(3)
        self._call("forces", F, o)
        return F, o[0], o[1], o[2]

    def scalars(self):
        o = np.zeros(6)
        self._call("get_scalars", o)
        return dict(pe=o[0], ke=o[1], virial=o[2], vir_act=o[3], inst_T=o[4], maxD=o[5])

    def cells(self):
        dims = np.zeros(3, dtype=np.int32)
        nc = self._call("get_cells", dims, None, None)
        counts = np.zeros(nc, dtype=np.int32)
        members = np.zeros(self.n, dtype=np.int32)
        self._call("get_cells", dims, counts.ctypes.data_as(C.c_void_p),
                   members.ctypes.data_as(C.c_void_p))
        return dims, counts, members

    def neighbors(self):
        """Half list as (counts[N], pairs[M,2])."""
        m = self._call("get_neighbors", None, None)
        counts = np.zeros(self.n, dtype=np.int32)
        pairs = np.zeros((max(m, 1), 2), dtype=np.int32)
        self._call("get_neighbors", counts.ctypes.data_as(C.c_void_p),
                   pairs.ctypes.data_as(C.c_void_p))
        return counts, pairs[:m]


class Oracle(_Common):
    """The project's C restatement of the reference timestep (one system)."""

    def __init__(self, n, nact, L, T, f0, tau_p_steps=200, rebuild_factor=3.0, list_mode=0):
        self.lib = _oracle_lib()
        self.n, self.nact = int(n), int(nact)
        self.h = self.lib.ora_create(self.n, self.nact, float(L), float(T), float(f0),
                                     int(tau_p_steps), float(rebuild_factor), int(list_mode))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ora_destroy(self.h)
            self.h = None

    def _call(self, name, *args):
        return getattr(self.lib, "ora_" + name)(self.h, *args)

    @classmethod
    def from_state(cls, st, T, f0, tau_p_steps=200, rebuild_factor=3.0, list_mode=0, eta=None,
                   p_eta=None):
        o = cls(st.n, st.nact, st.L, T, f0, tau_p_steps, rebuild_factor, list_mode)
        o.set_state(st)
        o.set_nhc(np.zeros(3) if eta is None else eta, np.zeros(3) if p_eta is None else p_eta)
        o.rebuild()
        o.forces()
        return o

    def set_state(self, st):
        self._call("set_state", _f64(st.x), _f64(st.xu), _f64(st.p), _i32(st.type), _i32(st.act_tag))
        self.set_k(st.k)

    def set_k(self, k):
        self._call("set_k", _i32(np.asarray(k).reshape(-1)) if self.nact else np.zeros(1, np.int32))

    def set_nhc(self, eta, p_eta):
        self._call("set_nhc", _f64(eta), _f64(p_eta))

    def set_thermostat(self, T):
        self._call("set_thermostat", float(T))

    def seed_rng(self, seed):
        self._call("seed_rng", int(seed))

    def shuffle(self):
        self._call("shuffle")

    def rebuild(self):
        self._call("rebuild")

    def run(self, nsteps, start=0, shuffle=False, drift=False):
        return self._call("run", int(start), int(nsteps), int(bool(shuffle)), int(bool(drift)))

    def run_nve(self, nsteps):
        return self._call("run_nve", int(nsteps))

    def fix_drift(self):
        self._call("fix_drift")

    def adjust_temp(self, T):
        return self._call("adjust_temp", float(T))

    def ramp(self, T_start, T_end, rate=0.1):
        return self._call("ramp", float(T_start), float(T_end), float(rate))

    @staticmethod
    def cell_geometry(L):
        lib = _oracle_lib()
        nc = np.zeros(3, dtype=np.int32)
        inv = np.zeros(3)
        lib.ora_cell_geometry(float(L), nc, inv)
        return nc, inv

    @staticmethod
    def log_schedule(run_length, num_origins=200, factor=1.4):
        lib = _oracle_lib()
        cap = num_origins * 80 + 64
        out = np.zeros(cap, dtype=np.uint64)
        m = lib.ora_log_schedule(int(run_length), int(num_origins), float(factor), out, cap)
        return out[:m].copy()


_rlibs: dict[tuple, C.CDLL] = {}


class Reference(_Common):
    """The reference engine compiled from its own sources (N fixed per library).

    kind "ref": the reference's own timestep files; kind "dropin": the same
    program with cell_list+forces.c and time_evolve.c replaced by the drop-in
    files of activechi4_b200/legacy (the timestep runs on the GPU).
    The reference keeps its state in process globals, so there is exactly one
    system per particle count and kind per process."""

    def __init__(self, n, kind="ref"):
        self.n = int(n)
        self.kind = kind
        key = (self.n, kind)
        if key not in _rlibs:
            path = ref_lib_path(self.n, kind)
            if not os.path.exists(path):
                raise FileNotFoundError(f"reference oracle for N={n} not built: {path}")
            lib = C.CDLL(path)
            lib.ref_setup.argtypes = [C.c_double, C.c_double, C.c_double, _dp, _dp, _dp, _ip, _ip, _ip]
            lib.ref_get_state.argtypes = [_dp, _dp, _dp, _dp]
            lib.ref_set_k.argtypes = [_ip]
            lib.ref_get_k.argtypes = [_ip]
            lib.ref_set_nhc.argtypes = [_dp, _dp]
            lib.ref_get_nhc.argtypes = [_dp]
            lib.ref_seed_rng.argtypes = [C.c_ulong]
            lib.ref_forces.argtypes = [_dp, _dp]
            lib.ref_run.restype = C.c_int
            lib.ref_run.argtypes = [C.c_long, C.c_int, C.c_int, C.c_int]
            lib.ref_run_berendsen.restype = C.c_int
            lib.ref_run_berendsen.argtypes = [C.c_int]
            lib.ref_run_gauss.restype = C.c_int
            lib.ref_run_gauss.argtypes = [C.c_int]
            lib.ref_run_npt.restype = C.c_int
            lib.ref_run_npt.argtypes = [C.c_int, C.c_double]
            lib.ref_get_box.argtypes = [_dp]
            lib.ref_set_npt.argtypes = [_dp, _dp, _dp, _dp, C.c_double]
            lib.ref_run_nhc_npt.restype = C.c_int
            lib.ref_run_nhc_npt.argtypes = [C.c_int, C.c_double]
            lib.ref_get_npt.argtypes = [_dp]
            lib.ref_run_brown.restype = C.c_int
            lib.ref_run_brown.argtypes = [C.c_int, _dp]
            lib.ref_adjust_temp.restype = C.c_double
            lib.ref_adjust_temp.argtypes = [C.c_double]
            lib.ref_coldstart.argtypes = [C.c_double, C.c_double]
            lib.ref_breakxal.argtypes = [C.c_double, C.c_double]
            lib.ref_initialize_system.restype = C.c_int
            lib.ref_initialize_system.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_uint,
                                                  C.c_char_p]
            lib.ref_run_nve.restype = C.c_int
            lib.ref_run_nve.argtypes = [C.c_int]
            lib.ref_get_scalars.argtypes = [_dp]
            lib.ref_get_cells.restype = C.c_int
            lib.ref_get_cells.argtypes = [_ip, C.c_void_p, C.c_void_p]
            lib.ref_get_neighbors.restype = C.c_long
            lib.ref_get_neighbors.argtypes = [C.c_void_p, C.c_void_p]
            lib.ref_log_schedule.restype = C.c_int
            lib.ref_log_schedule.argtypes = [C.c_ulonglong, C.c_int, C.c_double, C.c_char_p, _up, C.c_int]
            lib.ref_write_restart.argtypes = [C.c_char_p, C.c_int, C.c_int]
            lib.ref_set_time.argtypes = [C.c_long]
            _rlibs[key] = lib
        self.lib = _rlibs[key]
        self.nact = self.lib.ref_nact()
        self.tau_per = self.lib.ref_tau_per()

    def _call(self, name, *args):
        return getattr(self.lib, "ref_" + name)(*args)

    def setup(self, st, T, f0, eta=None, p_eta=None):
        assert st.n == self.n and st.nact == self.nact
        self.lib.ref_setup(float(st.L), float(T), float(f0), _f64(st.x), _f64(st.xu), _f64(st.p),
                           _i32(st.type), _i32(st.act_tag), _i32(np.asarray(st.k).reshape(-1)))
        self.set_nhc(np.zeros(3) if eta is None else eta, np.zeros(3) if p_eta is None else p_eta)

    def set_k(self, k):
        self.lib.ref_set_k(_i32(np.asarray(k).reshape(-1)))

    def set_nhc(self, eta, p_eta):
        self.lib.ref_set_nhc(_f64(eta), _f64(p_eta))

    def seed_rng(self, seed):
        self.lib.ref_seed_rng(int(seed))

    def rebuild(self):
        self.lib.ref_rebuild()

    def run(self, nsteps, start=0, shuffle=False, drift=False):
        return self.lib.ref_run(int(start), int(nsteps), int(bool(shuffle)), int(bool(drift)))

    def fix_drift(self):
        self.lib.ref_fix_drift()

    def run_gauss(self, nsteps):
        """AdvanceTimeNVTGaussOSM nsteps times (the reference's own build)."""
        if self.lib.ref_run_gauss(int(nsteps)):
            raise RuntimeError("this build has no AdvanceTimeNVTGaussOSM")

    def run_npt(self, nsteps, P):
        """advance_time_NPT nsteps times at target pressure P (the reference's own build)."""
        if self.lib.ref_run_npt(int(nsteps), float(P)):
            raise RuntimeError("this build has no advance_time_NPT")

    def set_npt(self, eta, p_eta, eta_baro, p_eta_baro, p_eps):
        """Nose-Hoover NPT state (InitialiseNoseHooverNPT with the momenta given)."""
        f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(3))  # noqa: E731
        self.lib.ref_set_npt(f(eta), f(p_eta), f(eta_baro), f(p_eta_baro), float(p_eps))

    def run_nhc_npt(self, nsteps, P):
        """AdvanceTimeNPTNoseHoover nsteps times at target pressure P."""
        if self.lib.ref_run_nhc_npt(int(nsteps), float(P)):
            raise RuntimeError("this build has no AdvanceTimeNPTNoseHoover")

    def npt_state(self):
        """eps, p_eps, eta_baro, p_eta_baro, eta, p_eta of the program's globals."""
        out = np.zeros(14)
        self.lib.ref_get_npt(out)
        return {"eps": out[0], "p_eps": out[1], "eta_baro": out[2:5], "p_eta_baro": out[5:8],
                "eta": out[8:11], "p_eta": out[11:14]}

    def run_brown(self, noise):
        """advance_time_ActiveBrown_PC once per noise[step] ([steps][N][3]
        standard normals by particle) in place of the program's draws."""
        noise = np.ascontiguousarray(noise, dtype=np.float64)
        if self.lib.ref_run_brown(int(noise.shape[0]), noise.reshape(-1)):
            raise RuntimeError("this build has no advance_time_ActiveBrown_PC")

    def box(self):
        """(L, inv_L, DENSITY) of the program's globals."""
        out = np.zeros(3)
        self.lib.ref_get_box(out)
        return tuple(float(v) for v in out)

    def run_berendsen(self, nsteps):
        """advance_time_NVT_Berendsen nsteps times (the reference's own build)."""
        if self.lib.ref_run_berendsen(int(nsteps)):
            raise RuntimeError("this build has no advance_time_NVT_Berendsen")

    def step_propagators(self, nsteps):
        """NVT steps composed from U1..U4, update_cell_list and calculate_forces."""
        for _ in range(int(nsteps)):
            self.lib.ref_step_propagators()

    def adjust_temp(self, T):
        return self.lib.ref_adjust_temp(float(T))

    def coldstart(self, rate, T):
        self.lib.ref_coldstart(float(rate), float(T))

    def breakxal(self, rate, T):
        self.lib.ref_breakxal(float(rate), float(T))

    def initialize_system(self, T, f0, jobno, srand_seed, workdir, density=1.2):
        """The reference's fresh-start initialisation (lattice, active set,
        coldstart, breakxal); once per process and particle count."""
        rc = self.lib.ref_initialize_system(float(density), float(T), float(f0), int(jobno), int(srand_seed),
                                            str(workdir).encode())
        if rc:
            raise RuntimeError("the reference's arrays are already set up in this process")

    def run_nve(self, nsteps):
        return self.lib.ref_run_nve(int(nsteps))

    def log_schedule(self, run_length, num_origins, factor, workdir):
        cap = num_origins * 80 + 64
        out = np.zeros(cap, dtype=np.uint64)
        m = self.lib.ref_log_schedule(int(run_length), int(num_origins), float(factor),
                                      str(workdir).encode(), out, cap)
        return out[:m].copy()

    def write_restart(self, path, it=0, last_saved_index=0):
        self.lib.ref_write_restart(str(path).encode(), int(it), int(last_saved_index))
