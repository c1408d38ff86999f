"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference MD engine compiled from its own sources (oracle/_ref, built
by `make -C oracle ref` where the reference sources are present) and stores
its inputs and outputs as .npz files:

  ka_n1000.npz  melted KA state at T=0.45 (N=1000, 3 cells per side) and the
                reference's cell lists, forces/energy/virials, and the state
                after 50 NVT steps without and with direction shuffles, and
                after 50 NVE steps
  ka_n4000.npz  the same for N=4000 (4 cells per side), fewer outputs
  ka_n500.npz   N=500 (2 cells per side): the reference's forces, which count
                every pair twice there (MDcode/cell_list+forces.c:37-49)
  schedule.npz  prepareSavingArray schedules (MDcode/main.c:62-119)

The states are melted with the reference too: a random lattice (seeded numpy
stream) heated by 2000 NVT steps at T=2.0 with direction shuffles, then 1000
NVT steps at T=0.45.

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from activechi4_b200.init import State, lattice_state  # noqa: E402
from oracle import Reference  # noqa: E402

P_ETA0 = np.array([0.5, -0.3, 0.2])
ETA0 = np.array([0.0, 0.0, 0.0])


def melt(n, seed, hot_steps=2000, cold_steps=1000):
    st = lattice_state(n, 2.0, seed=seed)
    ref = Reference(n)
    ref.setup(st, 2.0, 1.0)
    ref.seed_rng(seed)
    ref.run(hot_steps, shuffle=True)
    x, xu, p, _ = ref.get_state()
    st = State(st.L, x, xu, p, st.type, st.act_tag, ref.get_k())
    ref.setup(st, 0.45, 1.0)
    ref.run(cold_steps, start=hot_steps, shuffle=True)
    x, xu, p, _ = ref.get_state()
    # the fixture starts from folded coordinates, like a restart (MDcode/main.c:322-326)
    return State(st.L, x, x.copy(), p, st.type, st.act_tag, ref.get_k())


def snapshot(ref, prefix, out):
    x, xu, p, F = ref.get_state()
    sc = ref.scalars()
    eta, p_eta, q = ref.get_nhc()
    out[prefix + "x"] = x
    out[prefix + "xu"] = xu
    out[prefix + "p"] = p
    out[prefix + "F"] = F
    for k in ("pe", "ke", "virial", "vir_act", "inst_T", "maxD"):
        out[prefix + k] = np.float64(sc[k])
    out[prefix + "eta"] = eta
    out[prefix + "p_eta"] = p_eta
    out[prefix + "q"] = q


def state_arrays(st, out):
    out["L"] = np.float64(st.L)
    out["x"] = st.x
    out["xu"] = st.xu
    out["p"] = st.p
    out["type"] = st.type.astype(np.int32)
    out["act_tag"] = st.act_tag.astype(np.int32)
    out["k"] = st.k.astype(np.int32)
    out["eta0"] = ETA0
    out["p_eta0"] = P_ETA0


def full_case(n, seed, outs):
    st = melt(n, seed)
    out = {}
    state_arrays(st, out)
    ref = Reference(n)
    ref.setup(st, 0.45, 1.0, ETA0, P_ETA0)
    dims, counts, members = ref.cells()
    out["cell_dims"] = dims
    out["cell_counts"] = counts
    out["cell_members"] = members
    F, pe, vir, va = ref.forces()
    out["F0"] = F
    out["pe0"], out["vir0"], out["viract0"] = np.float64(pe), np.float64(vir), np.float64(va)
    cnt, _ = ref.neighbors()
    out["half_list_pairs"] = np.int64(cnt.sum())
    if "nvt" in outs:
        ref.setup(st, 0.45, 1.0, ETA0, P_ETA0)
        out["nvt_rebuilds"] = np.int64(ref.run(50, shuffle=False))
        snapshot(ref, "nvt_", out)
    if "shuffle" in outs:
        ref.setup(st, 0.45, 1.0, ETA0, P_ETA0)
        ref.seed_rng(4242)
        out["shf_rebuilds"] = np.int64(ref.run(50, start=0, shuffle=True))
        snapshot(ref, "shf_", out)
        out["shf_k"] = ref.get_k()
    if "nve" in outs:
        ref.setup(st, 0.45, 1.0, ETA0, P_ETA0)
        out["nve_rebuilds"] = np.int64(ref.run_nve(50))
        snapshot(ref, "nve_", out)
    return out


def main():
    np.savez_compressed(os.path.join(HERE, "ka_n1000.npz"), **full_case(1000, 11, {"nvt", "shuffle", "nve"}))
    np.savez_compressed(os.path.join(HERE, "ka_n4000.npz"), **full_case(4000, 12, {"nvt"}))
    # N=500: lattice state heated briefly (the double count makes the
    # reference's own dynamics unphysical, so no long melt)
    st = lattice_state(500, 0.45, seed=13)
    ref = Reference(500)
    ref.setup(st, 0.45, 1.0)
    out = {}
    state_arrays(st, out)
    F, pe, vir, va = ref.forces()
    out["F0"] = F
    out["pe0"], out["vir0"], out["viract0"] = np.float64(pe), np.float64(vir), np.float64(va)
    np.savez_compressed(os.path.join(HERE, "ka_n500.npz"), **out)
    sched = {}
    with tempfile.TemporaryDirectory() as d:
        for run_length, origins in ((20000, 200), (200000, 200), (1000, 10)):
            sched[f"s_{run_length}_{origins}"] = Reference(1000).log_schedule(run_length, origins, 1.4, d)
    np.savez_compressed(os.path.join(HERE, "schedule.npz"), **sched)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
