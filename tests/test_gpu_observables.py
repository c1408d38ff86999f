"""In-place observables on the device against the numpy restatement of the
reference's analysis applied to frames read back at every scheduled step.
Tolerance: 1e-12 relative on every per-bin sum (same FP64 positions)."""
import numpy as np
import pytest

from conftest import golden_state

pytestmark = pytest.mark.gpu


def test_observables_match_oracle(cuda_lib, g1000):
    from activechi4_b200 import Engine, default_params, qvectors
    from oracle.observables import analyse, log_pairs
    st = golden_state(g1000)
    run, no, fac, mi, a, live = 600, 6, 1.4, 300, 0.3, 3
    q = qvectors(st.L, 7.25, 24)
    e = Engine(default_params(st.n, shuffle=1, tau_p_steps=50, seed=5))
    e.set_state(0, st)
    e.set_nhc(0, g1000["eta0"], g1000["p_eta0"])
    e.obs_configure(0, run, no, fac, mi, a, q, live)
    _, pairs = log_pairs(run, no, fac, mi, live)
    need = sorted({s for p in pairs for s in p[:2]})
    frames, done = {}, 0
    for s in need:  # frame s = state after loop index s, i.e. s+1 steps
        e.step(s + 1 - done)
        done = s + 1
        frames[s] = e.get_state(0)[1]
    off, sums = e.obs_sums(0)
    off_o, want = analyse(frames, st.L, run, no, fac, mi, a, q, live)
    assert np.array_equal(off, off_o)
    assert np.array_equal(sums[:, 6], want[:, 6])  # pair counts per bin
    assert np.allclose(sums, want, rtol=1e-12, atol=1e-12)
    obs = e.observables(0)
    assert obs["Q"][0] > 0.9 and np.all(obs["chi4"] >= -1e-15)


def test_observables_same_alone_and_batched(cuda_lib, g1000):
    from activechi4_b200 import Engine, default_params, lattice_state
    st1 = golden_state(g1000)
    st2 = lattice_state(2000, 0.5, seed=3)
    p1 = default_params(1000, seed=1)
    p2 = default_params(2000, T=0.5, seed=2)

    def run(engine, sysids, states):
        for r, s in zip(sysids, states):
            engine.set_state(r, s)
            engine.set_nhc(r, [0, 0, 0], [0.1, 0.2, 0.3])
            engine.obs_configure(r, 200, 4, 1.4, 100, 0.3, None, 4)
        engine.step(201)
        return [engine.obs_sums(r)[1] for r in sysids]

    alone = run(Engine(p1), [0], [st1])[0]
    both = run(Engine([p2, p1]), [0, 1], [st2, st1])[1]
    assert np.array_equal(alone, both)
