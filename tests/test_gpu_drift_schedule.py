"""Drift removals scheduled by the host between graph launches.

The step graphs hold no drift-removal node: the engine keeps a copy of each
system's step counter and ramp steps left and launches the removal kernels
between graphs after every drift_every-th step.  These tests run systems
with short cadences, ramps in front (whose steps do not count), uneven step
calls and several systems of different cadences through the graphs and
kernel by kernel, and compare bit for bit; acg_bench_steps checks the host's
counters against the device's and cuts its timed graphs the same way."""
import numpy as np
import pytest

from conftest import golden_state

pytestmark = pytest.mark.gpu


def _engines(params):
    from activechi4_b200 import Engine
    return Engine(params), Engine(params)


def test_drift_schedule_graph_equals_eager(cuda_lib, g1000):
    from activechi4_b200 import default_params
    st = golden_state(g1000)
    st.p[:, 1] += 0.05  # a net momentum for the removals to take out
    params = [default_params(st.n, T=0.45, f0=1.0, shuffle=1, tau_p_steps=20, drift_every=de, seed=3 + r)
              for r, de in enumerate((7, 11, 0))]
    a, b = _engines(params)
    for e in (a, b):
        for r in range(3):
            e.set_state(r, st)
        k = e.start_ramp(1, 0.3, 0.45, 0.5)  # ramp steps first on system 1
        assert k > 0
    for n in (5, 33, 1, 64, 17):
        a.step(n)
        b.step_eager(n)
    for r in range(3):
        for u, w in zip(a.get_state(r), b.get_state(r)):
            assert np.array_equal(u, w)
        assert a.thermo(r)["step"] == b.thermo(r)["step"]
    # the removals did their work: systems 0 and 1 keep almost no net momentum
    for r in (0, 1):
        p = a.get_state(r)[2]
        assert np.abs(p.sum(axis=0)).max() < 1e-3 * np.abs(p).sum(axis=0).max()
    assert np.abs(a.get_state(2)[2].sum(axis=0)).max() > 1.0
    # the timed path agrees with the host's counters and cuts at the same steps
    ms, nl = a.bench_steps(40, 0)
    b.step_eager(40)
    for r in range(3):
        for u, w in zip(a.get_state(r), b.get_state(r)):
            assert np.array_equal(u, w)
    assert ms > 0 and nl > 0
