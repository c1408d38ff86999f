"""Batched replicas, the run server, and the FP32 pair-force precision path."""
import numpy as np
import pytest

from conftest import force_err, golden_state, rel

pytestmark = pytest.mark.gpu


def test_batched_replicas(cuda_lib):
    from activechi4_b200.batch import combine_chi4, make_engine, replica_set
    from activechi4_b200.tune import autotune
    reps = replica_set(count=24, seed=3)
    e = make_engine(reps)
    cfg = autotune(e, reps=3)
    assert cfg["group_tpp"] in (1, 2, 4)
    for r in range(e.nsys):
        e.obs_configure(r, 400, 4, 1.4, 0, 0.3, None, 4)
    e.step(401)
    for r in range(e.nsys):
        th = e.thermo(r)
        assert np.isfinite(th["pe"]) and th["step"] == 401
    obs = combine_chi4(e, reps)
    assert obs and all(len(v["Q"]) > 0 for v in obs.values())


def test_served_results_equal_alone(cuda_lib):
    from activechi4_b200.serve import RunRequest, Server, run_serial
    reqs = [RunRequest(0, 1500, 300, 0.45, 1.0, 20, seed=1, arrival=0.0),
            RunRequest(1, 6000, 200, 0.5, 2.0, 200, seed=2, arrival=0.01),
            RunRequest(2, 800, 500, 0.6, 0.5, 2000, seed=3, arrival=0.02),
            RunRequest(3, 3000, 250, 0.45, 0.0, 200, seed=4, arrival=0.03)]
    mixed = Server(max_active=4, chunk_work=2e5).run(reqs)
    alone, _ = run_serial(reqs, precision=1)
    assert [r.rid for r in mixed] == [0, 1, 2, 3]
    for m, a in zip(mixed, alone):
        assert np.array_equal(m.observables[0], a.observables[0])
        assert np.array_equal(m.observables[1], a.observables[1])
        assert m.pe == a.pe and m.ke == a.ke
        assert m.latency > 0


def test_fp32_forces_and_nve_drift(cuda_lib, g4000):
    """FP32 pair math against the FP64 path on the same state: forces within
    1e-5 (max|dF|/rms|F|), and the total energy of 2000 NVE steps drifts by
    less than 1e-4 relative in both precisions."""
    from activechi4_b200 import Engine, default_params
    st = golden_state(g4000)
    out = {}
    for prec in (0, 1):
        e = Engine(default_params(st.n, f0=0.0, thermostat=0, shuffle=0, precision=prec, list_mode=1,
                                  rebuild_factor=4.0))
        e.set_state(0, st)
        e.compute_forces()
        F = e.get_state()[3]
        th0 = e.thermo()
        e0 = th0["pe"] + th0["ke"]
        e.step(2000)
        th = e.thermo()
        out[prec] = (F, th0["pe"], abs(th["pe"] + th["ke"] - e0) / abs(e0))
    assert force_err(out[1][0], out[0][0]) <= 1e-5
    assert rel(out[1][1], out[0][1]) <= 1e-5
    assert out[0][2] < 1e-4 and out[1][2] < 1e-4
