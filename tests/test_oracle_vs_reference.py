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
