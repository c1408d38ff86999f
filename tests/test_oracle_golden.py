"""The oracle restatement against the golden fixtures made by the reference
itself (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from conftest import golden_state
from oracle import Oracle


def brute_force(st, f0):
    """All-pairs KA forces with the reference's pair term and minimum image
    (MDcode/cell_list+forces.c:174-218), vectorised; each pair once."""
    L = st.L
    x = st.x
    n = st.n
    sig = np.array([[1.0, 0.8], [0.8, 0.88]])
    eps = np.array([[1.0, 1.5], [1.5, 0.5]])
    C0, C2 = 0.0162665594880, -0.001949973872640
    F = np.zeros((n, 3))
    pe = vir = 0.0
    for i in range(n - 1):
        d = x[i] - x[i + 1:]
        d = np.where(d < -0.5, d + 1.0, d)
        d = np.where(d > 0.5, d - 1.0, d)
        dr2 = (d * d).sum(axis=1) * L * L
        s = sig[st.type[i], st.type[i + 1:]]
        e = eps[st.type[i], st.type[i + 1:]]
        rs2 = dr2 / (s * s)
        m = rs2 < 6.25
        s2 = 1.0 / rs2[m]
        s6 = s2 ** 3
        pe += (4.0 * e[m] * (s6 * (s6 - 1.0) + C0 + C2 * rs2[m])).sum()
        g = 8.0 * e[m] * (6.0 * s6 * (s6 - 0.5) / dr2[m] - C2 / (s[m] ** 2))
        fij = (g * L)[:, None] * d[m]
        F[i] += fij.sum(axis=0)
        np.subtract.at(F, np.arange(i + 1, n)[m], fij)
        vir += (g * dr2[m]).sum()
    va = 0.0
    for i in range(n):
        a = st.act_tag[i]
        if a >= 0:
            k = st.k[:, a].astype(float)
            F[i] += f0 * k
            va += f0 * (k @ st.xu[i])
    return F, pe, vir / 3.0, va


def oracle_for(g, T=0.45, f0=1.0):
    return Oracle.from_state(golden_state(g), T, f0, eta=g["eta0"], p_eta=g["p_eta0"])


@pytest.mark.parametrize("name", ["g1000", "g4000"])
def test_cells_bit_exact(name, request):
    g = request.getfixturevalue(name)
    dims, counts, members = oracle_for(g).cells()
    assert np.array_equal(dims, g["cell_dims"])
    assert np.array_equal(counts, g["cell_counts"])
    assert np.array_equal(members, g["cell_members"])


@pytest.mark.parametrize("name", ["g1000", "g4000"])
def test_forces_bit_exact(name, request):
    g = request.getfixturevalue(name)
    o = oracle_for(g)
    F, pe, vir, va = o.forces()
    assert np.array_equal(F, g["F0"])
    assert (pe, vir, va) == (g["pe0"], g["vir0"], g["viract0"])
    cnt, _ = o.neighbors()
    assert cnt.sum() == g["half_list_pairs"]


def _check_snapshot(o, g, pre):
    x, xu, p, F = o.get_state()
    for k, a in (("x", x), ("xu", xu), ("p", p), ("F", F)):
        assert np.array_equal(a, g[pre + k]), k
    sc = o.scalars()
    for k in ("pe", "ke", "virial", "vir_act", "inst_T", "maxD"):
        assert sc[k] == g[pre + k], k
    eta, p_eta, q = o.get_nhc()
    assert np.array_equal(eta, g[pre + "eta"]) and np.array_equal(p_eta, g[pre + "p_eta"])
    assert np.array_equal(q, g[pre + "q"])


@pytest.mark.parametrize("name", ["g1000", "g4000"])
def test_nvt_steps_bit_exact(name, request):
    g = request.getfixturevalue(name)
    o = oracle_for(g)
    assert o.run(50) == g["nvt_rebuilds"]
    _check_snapshot(o, g, "nvt_")


def test_shuffle_steps_bit_exact(g1000):
    o = oracle_for(g1000)
    o.seed_rng(4242)
    assert o.run(50, shuffle=True) == g1000["shf_rebuilds"]
    _check_snapshot(o, g1000, "shf_")
    assert np.array_equal(o.get_k(), g1000["shf_k"])


def test_nve_steps_bit_exact(g1000):
    o = oracle_for(g1000)
    assert o.run_nve(50) == g1000["nve_rebuilds"]
    x, xu, p, F = o.get_state()
    assert np.array_equal(x, g1000["nve_x"]) and np.array_equal(p, g1000["nve_p"])


def test_forces_match_brute_force(g1000):
    st = golden_state(g1000)
    F, pe, vir, va = brute_force(st, 1.0)
    Fo, peo, viro, vao = oracle_for(g1000).forces()
    rms = np.sqrt((F ** 2).sum(axis=1).mean())
    assert np.abs(Fo - F).max() / rms < 1e-12
    assert abs(peo - pe) / abs(pe) < 1e-12 and abs(viro - vir) / abs(vir) < 1e-12
    assert abs(vao - va) <= 1e-12 * max(1.0, abs(va))


def test_two_cells_per_side(g500):
    """N=500 has 2 cells per side.  The reference's neighbour-cell map then
    repeats cells and counts pairs more than once; the restatement visits each
    distinct cell once and agrees with the all-pairs sum instead."""
    st = golden_state(g500)
    F, pe, vir, va = brute_force(st, 1.0)
    Fo, peo, viro, vao = Oracle.from_state(st, 0.45, 1.0).forces()
    rms = np.sqrt((F ** 2).sum(axis=1).mean())
    assert np.abs(Fo - F).max() / rms < 1e-12
    assert abs(peo - pe) / abs(pe) < 1e-12
    # the reference's own value differs (pairs counted repeatedly)
    assert abs(g500["pe0"] - pe) / abs(pe) > 0.1


def test_log_schedule(sched):
    for key, want in sched.items():
        _, rl, no = key.split("_")
        got = Oracle.log_schedule(int(rl), int(no), 1.4)
        assert np.array_equal(got, want), key


@pytest.mark.parametrize("n,nc", [(500, 2), (1000, 3), (4000, 4), (8000, 6), (100000, 15), (256000, 20)])
def test_cell_geometry(n, nc):
    from activechi4_b200.init import box_length
    dims, inv = Oracle.cell_geometry(box_length(n))
    assert list(dims) == [nc] * 3
    L = box_length(n)
    assert inv[0] == L / (L / nc)
