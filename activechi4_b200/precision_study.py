"""FP32 pair forces against the FP64 path, on the GPU.

  python -m activechi4_b200.precision_study --n 100000 --nve-steps 1000000
  python -m activechi4_b200.precision_study --chi4 --replicas 16 --n-small 1000 --steps 100000

Prints one JSON object:

* ``force``: per-step force error of the FP32 pair math against the FP64 path
  on the same state (max |dF| / rms |F|, and the largest per-particle relative
  error among particles with |F| above the rms), plus the relative error of pe
  and virial, at several states along an NVT run.
* ``nve``: total-energy drift of an NVE run (f0 = 0: the active force is not
  conservative) in both precisions from the same melted state, as
  (E(t) - E(0)) / |E(0)| sampled every ``--nve-every`` steps, and the fitted
  drift per million steps.
* ``chi4`` (with ``--chi4``): Q(t), MSD, Fs(q=7.25, t) and chi4 of
  ``--replicas`` independent replicas per precision (same seeds in both), with
  the standard error over replicas; the chi4 peak height and position of each
  precision, and the largest difference of each curve between the precisions
  in combined standard errors.

States are the seeded lattice melted on the device at T = 2.0, then NVT at
T = 0.45 (the plain workload's state point).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from .engine import Engine, default_params, observables_from_sums, qvectors
from .init import lattice_state


def melted(n, prec, seed, f0=1.0, equil=2000, T=0.45):
    p = default_params(n, T=2.0, f0=f0, tau_p_steps=200, precision=prec, seed=seed, list_mode=1,
                       rebuild_factor=4.0, thermostat=1)
    e = Engine(p)
    st = lattice_state(n, 2.0, seed=seed)
    e.set_state(0, st)
    rng = np.random.default_rng(seed)
    q = e.thermo(0)["q"]
    e.set_nhc(0, np.zeros(3), np.sqrt(2.0 * q) * rng.standard_normal(3))
    e.step(equil)
    e.set_temperature(0, T)
    e.step(equil)
    e.sync()
    return e, st


def force_errors(n, seed, samples=5, gap=500):
    """An FP64 engine advances; at each sample its state is loaded into an FP32
    engine and both evaluate forces at the same positions."""
    e64, st = melted(n, 0, seed)
    e32 = Engine(default_params(n, T=0.45, f0=1.0, precision=1, list_mode=1, rebuild_factor=4.0))
    out = []
    for _ in range(samples):
        e64.step(gap)
        x, xu, p, _ = e64.get_state(0)
        s = type(st)(st.L, x, xu, p, st.type, st.act_tag, e64.get_directions(0))
        e64.compute_forces()
        e32.set_state(0, s)
        e32.compute_forces()
        F64 = e64.get_state(0)[3]
        F32 = e32.get_state(0)[3]
        t64, t32 = e64.thermo(0), e32.thermo(0)
        dF = np.linalg.norm(F32 - F64, axis=1)
        mag = np.linalg.norm(F64, axis=1)
        rms = float(np.sqrt((mag ** 2).mean()))
        big = mag > rms
        out.append({"max_dF_over_rmsF": float(dF.max() / rms),
                    "max_rel_dF_large_F": float((dF[big] / mag[big]).max()),
                    "pe_rel": abs(t32["pe"] - t64["pe"]) / abs(t64["pe"]),
                    "virial_rel": abs(t32["virial"] - t64["virial"]) / abs(t64["virial"])})
    e64.close()
    e32.close()
    return out


def nve_drift(n, seed, steps, every):
    res = {}
    # the same starting state for both precisions: an FP64 melt
    e, st = melted(n, 0, seed, f0=0.0)
    x, xu, p, _ = e.get_state(0)
    start = (x, xu, p, e.get_directions(0))
    e.close()
    for prec in (0, 1):
        e = Engine(default_params(n, T=0.45, f0=0.0, precision=prec, thermostat=0, shuffle=0, list_mode=1,
                                  rebuild_factor=4.0))
        e.set_state(0, type(st)(st.L, start[0], start[1], start[2], st.type, st.act_tag, start[3]))
        e.compute_forces()
        th = e.thermo(0)
        E0 = th["pe"] + th["ke"]
        ts, es = [0], [0.0]
        done = 0
        while done < steps:
            k = min(every, steps - done)
            e.step(k)
            done += k
            th = e.thermo(0)
            ts.append(done)
            es.append((th["pe"] + th["ke"] - E0) / abs(E0))
        slope = float(np.polyfit(np.array(ts, dtype=float), np.array(es), 1)[0]) * 1e6
        res["fp64" if prec == 0 else "fp32"] = {"E0": E0, "rel_drift_end": es[-1], "rel_drift_per_1e6_steps": slope,
                                                "max_abs_rel_dev": float(np.abs(es).max()), "steps": steps}
        e.close()
    return res


def chi4_study(n, replicas, steps, seed):
    out = {}
    for prec in (0, 1):
        params = [default_params(n, T=0.45, f0=1.0, tau_p_steps=200, precision=prec, seed=1000 + r, list_mode=1,
                                 rebuild_factor=4.0) for r in range(replicas)]
        e = Engine(params)
        for r in range(replicas):
            e.set_state(r, lattice_state(n, 2.0, seed=seed + r))
            e.set_temperature(r, 2.0)
            e.set_nhc(r, np.zeros(3), np.array([0.1, -0.1, 0.05]))
        e.step(2000)
        for r in range(replicas):
            e.set_temperature(r, 0.45)
        e.step(20000)
        qv = qvectors(e.state_meta(0)["L"], 7.25, 24)
        for r in range(replicas):
            e.obs_configure(r, steps, 20, 1.4, 0, 0.3, qv, 16)
        e.step(steps)
        curves = [observables_from_sums(*e.obs_sums(r)) for r in range(replicas)]
        t = curves[0]["t"]
        sq = np.sqrt(replicas)
        rec = {"t": t.tolist()}
        for key in ("chi4", "Q", "msd", "Fs"):
            a = np.array([c[key] for c in curves])
            rec[key] = a.mean(0).tolist()
            rec[key + "_se"] = (a.std(0, ddof=1) / sq).tolist()
        m = np.array(rec["chi4"])
        k = int(np.argmax(m))
        rec.update({"chi4_peak": float(m[k]), "chi4_peak_se": rec["chi4_se"][k], "t_peak": float(t[k])})
        out["fp64" if prec == 0 else "fp32"] = rec
        e.close()
    a, b = out["fp64"], out["fp32"]
    out["peak_diff_over_se"] = abs(a["chi4_peak"] - b["chi4_peak"]) / float(np.hypot(a["chi4_peak_se"],
                                                                                      b["chi4_peak_se"]))
    # largest difference of each curve between the precisions, in combined standard errors
    for key in ("Q", "msd", "Fs", "chi4"):
        d = np.abs(np.array(a[key]) - np.array(b[key]))
        e = np.hypot(np.array(a[key + "_se"]), np.array(b[key + "_se"]))
        ok = e > 0
        out[f"max_{key}_diff_over_se"] = float((d[ok] / e[ok]).max()) if ok.any() else 0.0
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=100000)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--nve-steps", type=int, default=100000)
    ap.add_argument("--nve-every", type=int, default=10000)
    ap.add_argument("--chi4", action="store_true")
    ap.add_argument("--replicas", type=int, default=16)
    ap.add_argument("--n-small", type=int, default=1000)
    ap.add_argument("--steps", type=int, default=100000)
    a = ap.parse_args()
    res = {"n": a.n, "force": force_errors(a.n, a.seed), "nve": nve_drift(a.n, a.seed, a.nve_steps, a.nve_every)}
    if a.chi4:
        res["chi4"] = chi4_study(a.n_small, a.replicas, a.steps, a.seed)
        res["chi4"]["n"] = a.n_small
    print(json.dumps(res))


if __name__ == "__main__":
    main()
