"""The oracle restatement against the reference compiled from its own sources,
on fresh seeded states (skipped where oracle/_ref was not built).  CPU only."""
import numpy as np
import pytest

from activechi4_b200.init import lattice_state
from oracle import Oracle, Reference, reference_available


@pytest.mark.parametrize("n,seed", [(1000, 1), (1000, 2), (4000, 3), (8000, 4)])
def test_bit_exact_against_reference(n, seed):
    if not reference_available(n):
        pytest.skip(f"reference library for N={n} not built")
    st = lattice_state(n, 1.5, seed=seed)
    p_eta = np.array([0.3, 0.1, -0.2])
    ref = Reference(n)
    ref.setup(st, 1.5, 2.0, p_eta=p_eta)
    o = Oracle.from_state(st, 1.5, 2.0, p_eta=p_eta)
    for a, b in zip(ref.cells(), o.cells()):
        assert np.array_equal(a, b)
    Fr, *sr = ref.forces()
    Fo, *so = o.forces()
    assert np.array_equal(Fr, Fo) and sr == so
    ref.seed_rng(seed)
    o.seed_rng(seed)
    assert ref.run(30, shuffle=True) == o.run(30, shuffle=True)
    for a, b in zip(ref.get_state(), o.get_state()):
        assert np.array_equal(a, b)
    assert np.array_equal(ref.get_k(), o.get_k())


def test_schedule_against_reference(tmp_path):
    if not reference_available(1000):
        pytest.skip("reference library not built")
    ref = Reference(1000)
    for rl, no in ((5000, 50), (123457, 200), (2000000, 200)):
        assert np.array_equal(ref.log_schedule(rl, no, 1.4, tmp_path), Oracle.log_schedule(rl, no, 1.4))


@pytest.mark.parametrize("n,seed", [(1000, 5), (4000, 6)])
def test_drift_and_ramps_against_reference(n, seed):
    """fixDrift inside the run loop, adjustInitialTemp, and the coldstart /
    breakxal ramps of initialisation: bit-exact."""
    if not reference_available(n):
        pytest.skip(f"reference library for N={n} not built")
    st = lattice_state(n, 0.45, seed=seed)
    st.p[:, 2] += 0.3  # a net momentum for fixDrift to remove
    p_eta = np.array([0.1, -0.1, 0.05])
    ref = Reference(n)
    ref.setup(st, 0.45, 1.0, p_eta=p_eta)
    o = Oracle.from_state(st, 0.45, 1.0, p_eta=p_eta)
    ref.seed_rng(seed)
    o.seed_rng(seed)
    assert ref.run(5, shuffle=True, drift=True) == o.run(5, shuffle=True, drift=True)
    ref.fix_drift()
    o.fix_drift()
    assert ref.adjust_temp(0.3) == o.adjust_temp(0.3)
    ref.coldstart(0.1, 0.45)
    assert o.ramp(0.225, 0.45, 0.1) == 450
    for a, b in zip(ref.get_state(), o.get_state()):
        assert np.array_equal(a, b)
    ref.breakxal(0.1, 0.45)
    o.ramp(0.675, 0.45, 0.1)
    for a, b in zip(ref.get_state(), o.get_state()):
        assert np.array_equal(a, b)


_INIT_SCRIPT = r"""
import sys, tempfile, numpy as np
sys.path.insert(0, {root!r})
from oracle import Reference
n, T, job, seed = {n}, {T}, {job}, {seed}
r = Reference(n)
with tempfile.TemporaryDirectory() as d:
    r.initialize_system(T, 1.0, job, seed, d)
x, xu, p, F = r.get_state()
r.run(1, start=0, shuffle=True)
np.savez({out!r}, x=x, xu=xu, p=p, F=F, k=r.get_k())
"""


def reference_initialize(n, T, job, seed, out):
    """The reference's initializeSystem in a process of its own (it sets up
    the reference's arrays once per process); saves the state and the
    directions after the first run-loop shuffle."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = _INIT_SCRIPT.format(root=root, n=n, T=T, job=job, seed=seed, out=str(out))
    subprocess.run([sys.executable, "-c", code], check=True, capture_output=True, timeout=600)
    return dict(np.load(out))


def lattice_positions(site, n):
    """GetFccGrid's grid coordinates (MDcode/initialise.c:40-47)."""
    t = 1
    while t ** 3 < n:
        t += 1
    dr, t2 = 1.0 / t, t * t
    i = site.astype(np.int64)
    return np.stack([dr * ((i % t2) % t).astype(np.float64), dr * (i % t2).astype(np.float64) / float(t),
                     dr * (i / float(t2))], axis=1)


def test_reference_initialisation_draws(tmp_path):
    """The host's mirror of the reference's rand() draws plus the oracle's
    ramps give the reference program's initializeSystem bit for bit, and the
    derived MT19937 seed gives its first direction shuffle."""
    n, T, job, seed = 1000, 0.45, 3, 4242
    if not reference_available(n):
        pytest.skip("reference library not built")
    from activechi4_b200.init import State, box_length, reference_draws
    ref = reference_initialize(n, T, job, seed, tmp_path / "init.npz")
    d = reference_draws(n, seed, jobno=job)
    x = lattice_positions(d.site, n)
    st = State(box_length(n), x, x.copy(), d.p.copy(), d.type, d.act_tag, d.k)
    o = Oracle(n, st.nact, st.L, T, 1.0)
    o.set_state(st)
    o.set_nhc(np.zeros(3), np.zeros(3))
    o.rebuild()
    o.forces()
    o.ramp(0.5 * T, T, 0.1)
    o.ramp(1.5 * T, T, 0.1)
    o.adjust_temp(T)
    for name, a in zip(("x", "xu", "p", "F"), o.get_state()):
        assert np.array_equal(a, ref[name]), name
    o.seed_rng(d.gsl_seed)
    o.shuffle()
    assert np.array_equal(o.get_k(), ref["k"])
