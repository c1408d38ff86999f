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


def test_batch_equals_alone(cuda_lib):
    """Replicas advanced inside one batch engine give bit-identical states,
    energies and observables to the same systems advanced alone (the batch
    splits whole boxes into blocks differently; the sums do not depend on it)."""
    from activechi4_b200.batch import make_engine, replica_set
    reps = replica_set(count=6, n_min=600, n_max=9000, seed=5)
    p_eta = np.array([0.1, -0.05, 0.02])
    e = make_engine(reps)
    for r in range(e.nsys):
        e.set_nhc(r, np.zeros(3), p_eta)
        e.obs_configure(r, 300, 3, 1.4, 0, 0.3, None, 4)
    # rebuilds during set-up (each load primes the lists) are not part of the run
    rb0 = [e.thermo(r)["rebuilds"] for r in range(e.nsys)]
    e.step(300)
    for r, (p, st) in enumerate(reps):
        a = make_engine([(p, st)])
        a.set_nhc(0, np.zeros(3), p_eta)
        a.obs_configure(0, 300, 3, 1.4, 0, 0.3, None, 4)
        ra0 = a.thermo(0)["rebuilds"]
        a.step(300)
        for u, w in zip(a.get_state(0), e.get_state(r)):
            assert np.array_equal(u, w)
        ta, tb = a.thermo(0), e.thermo(r)
        assert ta["pe"] == tb["pe"] and ta["ke"] == tb["ke"]
        assert ta["rebuilds"] - ra0 == tb["rebuilds"] - rb0[r]
        assert np.array_equal(a.obs_sums(0)[1], e.obs_sums(r)[1])
        a.close()
    e.close()


def test_restart_files_round_trip(cuda_lib, tmp_path):
    """A GPU run saved in the reference's restart/active files and resumed in
    a fresh engine the way initialise_restart_state does gives the same forces
    as the saved state (to the files' 14 decimals)."""
    from activechi4_b200 import Engine, default_params, formats
    from activechi4_b200.init import lattice_state
    n = 4000
    e = Engine(default_params(n, T=0.45, f0=1.0))
    e.set_state(0, lattice_state(n, 0.8, seed=9))
    e.step(200)
    formats.save_run(e, 0, tmp_path / "restart_file.dat", tmp_path / "ActiveDirection.dat",
                     tmp_path / "ActiveFileIndex.dat", iteration=200)
    st, it, _ = formats.load_restart_state(tmp_path / "restart_file.dat", tmp_path / "ActiveFileIndex.dat",
                                           tmp_path / "ActiveDirection.dat", n)
    assert it == 200
    e.compute_forces()
    F0 = e.get_state(0)[3]
    b = Engine(default_params(n, T=0.45, f0=1.0, L=st.L))
    b.set_state(0, st)
    b.compute_forces()
    F1 = b.get_state(0)[3]
    assert force_err(F1, F0) < 1e-9
    assert np.array_equal(b.get_directions(0), e.get_directions(0))


def test_large_batch_finite_and_equal_alone(cuda_lib):
    """The batched workload's 256 replicas (whole boxes split several cells
    per block, two-cell boxes one cell per block) stay finite, and replicas of
    each box kind match the same system run alone."""
    from activechi4_b200.batch import make_engine, replica_set
    from activechi4_b200.init import box_length
    reps = replica_set(count=256, seed=11, precision=1)
    p_eta = np.array([0.1, -0.05, 0.02])
    e = make_engine(reps)
    for r in range(e.nsys):
        e.set_nhc(r, np.zeros(3), p_eta)
    e.step(96)
    for r in range(e.nsys):
        th = e.thermo(r)
        assert np.isfinite(th["ke"]) and 0.0 < th["inst_T"] < 10.0, (r, th["inst_T"])
    nc = [int(int(box_length(p.n)) / 2.85) for p, _ in reps]
    picks = [nc.index(k) for k in (2, 3, 4) if k in nc]
    for r in picks:
        a = make_engine([reps[r]])
        a.set_nhc(0, np.zeros(3), p_eta)
        a.step(96)
        for u, w in zip(a.get_state(0), e.get_state(r)):
            assert np.array_equal(u, w)
        a.close()
    e.close()
