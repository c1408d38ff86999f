"""Statistical parity with the reference program at N = 1000 (T = 0.45,
f0 = 1.0, tau_p = 200 steps): the GPU path, in FP64 and with FP32 pair
forces, follows the protocol of tests/golden/make_statistics.py from the same
initial configurations (the reference's own initializeSystem draws, ramps run
on the device, same thermostat momenta, directions re-drawn on the device
from the reference's MT19937 seeds) and its in-place observables are compared
with the reference's statistics over the same seeds (tests/golden/
stats_n1000.npz).

Trajectories are chaotic, so the two sides agree only in distribution.  For
every time bin, Q(t) (a = 0.3), chi4(t) = Var_origins(Q), the MSD and
Fs(|q| = 7.25, t) averaged over seeds must agree within Z = 4 combined
standard errors of the seed means (Z allows for the ~130 correlated
comparisons); the chi4 peak height and its time bin likewise.  NVE energy
drift (f0 = 0) from the golden state: the GPU's total-energy change over the
run within twice the reference's (or 2e-4 per particle, the size of the
energy's own fluctuation at this time step), in FP64 and FP32.

Set ACG_STATS_TABLE=<path> to also write the comparison table there."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, golden_state

pytestmark = pytest.mark.gpu
Z = 4.0


@pytest.fixture(scope="module")
def ref_stats():
    path = os.path.join(GOLDEN, "stats_n1000.npz")
    if not os.path.exists(path):
        pytest.skip("stats_n1000.npz not generated")
    return dict(np.load(path))


def per_seed(sums):
    """sums [seeds, bins, 7] -> per-seed Q, chi4, msd, Fs [seeds, bins]"""
    c = sums[..., 6]
    Q = sums[..., 0] / c
    return {"Q": Q, "chi4": sums[..., 1] / c - Q * Q, "msd": sums[..., 2] / c, "Fs": sums[..., 5] / c}


def gpu_sums(ref, precision):
    if GOLDEN not in sys.path:
        sys.path.insert(0, GOLDEN)
    import make_statistics as ms
    from activechi4_b200 import Engine, default_params, qvectors
    from activechi4_b200.init import box_length, initialize_systems, reference_draws
    seeds = [int(s) for s in ref["seeds"]]
    n = int(ref["n"])
    e = Engine([default_params(n, T=ms.T, f0=ms.F0, precision=precision) for _ in seeds])
    draws = {r: reference_draws(n, ms.SRAND0 + s, jobno=s) for r, s in enumerate(seeds)}
    initialize_systems(e, draws, ms.T)
    for r, s in enumerate(seeds):
        e.set_nhc(r, np.zeros(3), ms.p_eta_for(s))
        e.fix_drift(r)
    e.step(ms.EQUIL)
    qv = qvectors(box_length(n), ms.Q)
    for r in range(len(seeds)):
        e.obs_configure(r, ms.RUN, ms.ORIGINS, ms.FACTOR, 0, ms.A, qv, ms.LIVE)
    e.step(ms.RUN)
    out = []
    for r in range(len(seeds)):
        off, s = e.obs_sums(r)
        assert np.array_equal(off, ref["offsets"])
        out.append(s)
    e.close()
    return np.stack(out)


def compare(ref, sums, label):
    a, b = per_seed(ref["sums"]), per_seed(sums)
    ns = ref["sums"].shape[0]
    rows, bad = [], []
    for key in ("Q", "chi4", "msd", "Fs"):
        ma, mb = a[key].mean(axis=0), b[key].mean(axis=0)
        sa, sb = a[key].std(axis=0, ddof=1) / np.sqrt(ns), b[key].std(axis=0, ddof=1) / np.sqrt(ns)
        tol = Z * np.sqrt(sa ** 2 + sb ** 2) + 1e-12 * np.abs(ma)
        for m in np.nonzero(np.abs(ma - mb) > tol)[0]:
            bad.append((key, int(ref["offsets"][m]), ma[m], mb[m], tol[m]))
        rows.append((key, ma, sa, mb, sb))
    # chi4 peak: height and bin
    ca, cb = a["chi4"].mean(axis=0), b["chi4"].mean(axis=0)
    ka, kb = int(np.argmax(ca)), int(np.argmax(cb))
    sa = a["chi4"][:, ka].std(ddof=1) / np.sqrt(ns)
    sb = b["chi4"][:, kb].std(ddof=1) / np.sqrt(ns)
    peak = (ca[ka], sa, cb[kb], sb, int(ref["offsets"][ka]), int(ref["offsets"][kb]))
    if abs(ca[ka] - cb[kb]) > Z * np.hypot(sa, sb):
        bad.append(("chi4 peak", int(ref["offsets"][ka]), ca[ka], cb[kb], Z * np.hypot(sa, sb)))
    return rows, peak, bad


def nve_energy(precision, every, steps):
    from activechi4_b200 import Engine, default_params
    from conftest import load_golden
    g = load_golden("ka_n1000.npz")
    st = golden_state(g)
    e = Engine(default_params(st.n, T=0.45, f0=0.0, thermostat=0, shuffle=0, drift_every=0,
                              precision=precision))
    e.set_state(0, st)
    out = []
    for k in range(steps // every + 1):
        if k:
            e.step(every)
        th = e.thermo()
        out.append((th["pe"] + th["ke"]) / st.n)
    e.close()
    return np.array(out)


def write_table(path, ref, results, nve):
    off = ref["offsets"] * 0.005
    with open(path, "w") as f:
        f.write(f"# reference vs GPU, N={int(ref['n'])}, {ref['sums'].shape[0]} seeds per side\n\n")
        for label, (rows, peak, bad) in results.items():
            f.write(f"## {label}\n\nchi4 peak: reference {peak[0]:.5f} +- {peak[1]:.5f} at step {peak[4]}, "
                    f"GPU {peak[2]:.5f} +- {peak[3]:.5f} at step {peak[5]}; bins outside {Z:g} SE: {len(bad)}\n\n")
            f.write("| t | Q ref | Q gpu | chi4 ref | chi4 gpu | MSD ref | MSD gpu | Fs ref | Fs gpu |\n")
            f.write("|---|---|---|---|---|---|---|---|---|\n")
            cols = {r[0]: r for r in rows}
            for m in range(len(off)):
                cells = [f"{off[m]:.3f}"]
                for key in ("Q", "chi4", "msd", "Fs"):
                    _, ma, sa, mb, sb = cols[key]
                    cells += [f"{ma[m]:.4g} +- {sa[m]:.1g}", f"{mb[m]:.4g} +- {sb[m]:.1g}"]
                f.write("| " + " | ".join(cells) + " |\n")
            f.write("\n")
        f.write("## NVE total energy per particle (f0 = 0, golden state)\n\n| side | E(0) | E(end) | change |\n"
                "|---|---|---|---|\n")
        for label, e in nve.items():
            f.write(f"| {label} | {e[0]:.8f} | {e[-1]:.8f} | {e[-1] - e[0]:+.3e} |\n")


def test_statistics_match_reference(cuda_lib, ref_stats):
    results = {}
    for label, prec in (("FP64", 0), ("FP32 pair forces", 1)):
        results[label] = compare(ref_stats, gpu_sums(ref_stats, prec), label)
    every = int(ref_stats["nve_every"])
    steps = every * (len(ref_stats["nve_energy"]) - 1)
    nve = {"reference": ref_stats["nve_energy"], "GPU FP64": nve_energy(0, every, steps),
           "GPU FP32": nve_energy(1, every, steps)}
    if os.environ.get("ACG_STATS_TABLE"):
        write_table(os.environ["ACG_STATS_TABLE"], ref_stats, results, nve)
    for label, (_, _, bad) in results.items():
        assert not bad, (label, bad[:5])
    dref = abs(nve["reference"][-1] - nve["reference"][0])
    for label in ("GPU FP64", "GPU FP32"):
        d = abs(nve[label][-1] - nve[label][0])
        assert d <= max(2.0 * dref, 2e-4), (label, d, dref)
