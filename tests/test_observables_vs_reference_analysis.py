"""The numpy restatement of the observables against the reference's own
analysis program (Analysis/, compiled from its sources into oracle/_ref;
skipped where it was not built), on the same trajectory written in the
reference's formats (data_coor.out at %.5lf, time_index_file.dat).  CPU only.

The analysis program takes L = (N/1.2)^(1/3) (Analysis/main.c:15), not the
MD code's pow(N/DENSITY, 0.33333333); the comparison uses the analysis' L."""
import os
import subprocess

import numpy as np
import pytest

from conftest import golden_state
from oracle import Oracle
from oracle.bindings import HERE as ORACLE_DIR
from oracle.observables import analyse

EXE = os.path.join(ORACLE_DIR, "_ref", "analysis_n1000")


def _write_run(tmp, st, run, no):
    sched = [int(s) for s in Oracle.log_schedule(run, no, 1.4)]
    o = Oracle.from_state(st, 0.45, 1.0, p_eta=np.array([0.1, -0.2, 0.3]))
    o.seed_rng(7)
    frames, lines, step = {}, [], 0
    for s in sched:
        o.run(s + 1 - step, start=step, shuffle=True)
        step = s + 1
        xu = o.get_state()[1]
        txt = [f"{a:.5f}\t{b:.5f}\t{c:.5f}\t{t}" for (a, b, c), t in zip(xu, st.type)]
        lines += txt
        frames[s] = np.array([[float(v) for v in ln.split("\t")[:3]] for ln in txt])
    sub = tmp / "0.450" / "data_001"
    sub.mkdir(parents=True)
    (sub / "data_coor.out").write_text("\n".join(lines) + "\n")
    (sub / "time_index_file.dat").write_text(f"total timesteps equals {len(sched)}\n" +
                                             "".join(f"{s}\n" for s in sched))
    (sub / "ActiveFileIndex.dat").write_text("".join(f"{i}\n" for i in np.flatnonzero(st.act_tag >= 0)))
    run_dir = tmp / "run"
    run_dir.mkdir()
    (run_dir / "para_file").write_text("DENSITY\tT\tP\tDIAMETER\tnb\ttau_alpha\n1.2\t0.45\t0.1\t0.3\t1\t2.5\n"
                                       "start_ensemble\tend_ensemble\n1\t1\n")
    return frames, sub, run_dir


def test_restatement_matches_reference_analysis(tmp_path, g1000):
    if not os.path.exists(EXE):
        pytest.skip("reference analysis program not built")
    st = golden_state(g1000)
    run, no = 2000, 20
    frames, sub, run_dir = _write_run(tmp_path, st, run, no)
    subprocess.run([EXE, "1", "0.45", "1.0"], cwd=run_dir, check=True, capture_output=True, timeout=600)
    L_an = (1000 / 1.2) ** (1.0 / 3.0)
    off, s = analyse(frames, L_an, run, no, 1.4, 0, 0.3, None, max_live=no, skip_missing=True)
    m = s[:, 6] > 0
    c = s[m, 6]
    Q = s[m, 0] / c
    chi4 = s[m, 1] / c - Q * Q
    relax = np.loadtxt(sub / "relax_a_0.30.dat")[1:]
    msd = np.loadtxt(sub / "msd.dat")[1:]
    assert np.allclose(relax[:, 0], off[m] * 0.005, rtol=1e-12)
    assert np.allclose(relax[:, 1], Q, rtol=1e-10, atol=1e-13)
    assert np.allclose(relax[:, 2], chi4, rtol=1e-8, atol=1e-13)
    assert np.allclose(msd[:, 1], s[m, 2] / c, rtol=1e-10, atol=1e-13)
    assert np.allclose(msd[:, 2], s[m, 3] / c, rtol=1e-10, atol=1e-13)
    assert np.allclose(msd[:, 3], s[m, 4] / c, rtol=1e-10, atol=1e-13)
