"""Host-side synthetic state generation.  CPU only."""
import numpy as np

from activechi4_b200.init import box_length, lattice_state, n_active, shuffle_directions


def test_lattice_state_properties():
    st = lattice_state(4000, 0.45, seed=5)
    assert st.x.shape == (4000, 3) and np.all((st.x >= 0) & (st.x < 1))
    assert abs(st.L - (4000 / 1.2) ** 0.33333333) < 1e-12
    assert (st.type == 1).sum() == 4000 - int(0.8 * 4000)
    assert st.nact == n_active(4000) == 400
    assert np.all(np.abs(st.k.sum(axis=1)) == 0)  # zero net active force
    assert np.allclose(st.p.sum(axis=0), 0.0, atol=1e-12)
    T = (st.p ** 2).sum() / (3 * 4000 - 3)
    assert abs(T - 0.45) < 1e-12
    tags = st.act_tag[st.act_tag >= 0]
    assert sorted(tags) == list(range(400))
    # no two particles on the same lattice point
    assert len({tuple(r) for r in np.round(st.x * 1e6).astype(int)}) == 4000


def test_shuffle_keeps_counts():
    st = lattice_state(1000, 0.45, seed=1)
    k2 = shuffle_directions(st.k, np.random.default_rng(3))
    assert np.array_equal(np.sort(k2, axis=1), np.sort(st.k, axis=1))
    assert not np.array_equal(k2, st.k)


def test_box_length_matches_reference_formula():
    assert box_length(100000) == float(np.power(100000 / 1.2, 0.33333333))
