"""The device's direction shuffle, drift removal and initialisation ramps
against the oracle (which is pinned bit-exact to the reference program by
tests/test_oracle_vs_reference.py).

Tolerances: directions bit-exact (same MT19937 stream, same swap order);
trajectories within 1e-9 after 100 steps (chaotic growth of rounding
differences); one drift removal within 1e-14 of the momentum scale (the two
sides sum the momenta in different orders); ramps of ~450 NVE steps within
1e-8, the whole initialisation (~900 steps) within 1e-8 in positions and
1e-7 in momenta."""
import numpy as np
import pytest

from conftest import force_err, golden_state

pytestmark = pytest.mark.gpu


def engine_for(st, **kw):
    from activechi4_b200 import Engine, default_params
    p = default_params(st.n, T=kw.pop("T", 0.45), f0=kw.pop("f0", 1.0), **kw)
    e = Engine(p)
    e.set_state(0, st)
    return e


def oracle_for(st, T=0.45, f0=1.0, tau_p=200, p_eta=None):
    from oracle import Oracle
    return Oracle.from_state(st, T, f0, tau_p_steps=tau_p, p_eta=p_eta)


def test_device_shuffle_is_the_reference_sequence(cuda_lib, g1000):
    st = golden_state(g1000)
    e = engine_for(st, shuffle=1, tau_p_steps=20, seed=2024, drift_every=0)
    o = oracle_for(st, tau_p=20)
    o.seed_rng(2024)
    # steps 0 | 1-20 | 21-40 | 41-60 | 61-79: shuffles at 0, 20, 40, 60, none after
    for block, shuffles in ((1, 1), (20, 1), (20, 1), (20, 1), (19, 0)):
        e.step(block)
        for _ in range(shuffles):
            o.shuffle()
        assert np.array_equal(e.get_directions(), o.get_k())
    e.shuffle(0)  # acg_shuffle_directions: the same stream, outside the step
    o.shuffle()
    assert np.array_equal(e.get_directions(), o.get_k())


def test_device_shuffle_global_memory_path(cuda_lib):
    """More active particles than fit the shared-memory staging (32768)."""
    from activechi4_b200 import lattice_state
    from oracle import Oracle
    n = 340000
    st = lattice_state(n, 0.45, seed=9)
    assert st.nact > 32768
    e = engine_for(st, shuffle=1, seed=77, drift_every=0)
    e.shuffle(0)
    o = Oracle(n, st.nact, st.L, 0.45, 1.0)
    o.set_k(st.k)
    o.seed_rng(77)
    o.shuffle()
    assert np.array_equal(e.get_directions(), o.get_k())


def test_trajectory_with_device_shuffles(cuda_lib, g1000):
    """100 NVT steps with the directions re-drawn on the device every 20
    steps: the oracle with the same seed follows the same trajectory."""
    st = golden_state(g1000)
    e = engine_for(st, shuffle=1, tau_p_steps=20, seed=31, drift_every=0)
    e.set_nhc(0, g1000["eta0"], g1000["p_eta0"])
    o = oracle_for(st, tau_p=20, p_eta=g1000["p_eta0"])
    o.seed_rng(31)
    e.step(100)
    o.run(100, shuffle=True)
    x, xu, p, F = e.get_state()
    xo, xuo, po, Fo = o.get_state()
    assert np.abs(xu - xuo).max() < 1e-9
    assert np.abs(p - po).max() / np.sqrt((po ** 2).sum(axis=1).mean()) < 1e-9
    assert force_err(F, Fo) < 1e-9
    assert np.array_equal(e.get_directions(), o.get_k())


def test_fix_drift(cuda_lib, g1000):
    st = golden_state(g1000)
    st.p[:, 0] += 0.2
    st.p[:, 2] -= 0.1
    e = engine_for(st, shuffle=0, drift_every=0)
    e.set_nhc(0, g1000["eta0"], g1000["p_eta0"])
    o = oracle_for(st, p_eta=g1000["p_eta0"])
    e.fix_drift(0)
    o.fix_drift()
    p = e.get_state()[2]
    po = o.get_state()[2]
    assert np.abs(p - po).max() < 1e-14 * np.abs(po).max() * 10
    assert np.abs(p.sum(axis=0)).max() < 1e-10


def test_drift_removal_inside_the_step(cuda_lib, g1000):
    """drift_every = 1: fixDrift after every step, as the reference's run()
    loop does after every 100000th (the oracle's run from start 0 removes it
    after its step 0)."""
    st = golden_state(g1000)
    st.p[:, 1] += 0.05
    e = engine_for(st, shuffle=0, drift_every=1)
    e.set_nhc(0, g1000["eta0"], g1000["p_eta0"])
    o = oracle_for(st, p_eta=g1000["p_eta0"])
    for _ in range(5):
        e.step(1)
        o.run(1, start=0, drift=True)
    x, xu, p, F = e.get_state()
    xo, xuo, po, Fo = o.get_state()
    assert np.abs(xu - xuo).max() < 1e-9
    assert np.abs(p - po).max() / np.sqrt((po ** 2).sum(axis=1).mean()) < 1e-9
    th = e.thermo()
    assert abs(th["ke"] - o.scalars()["ke"]) < 1e-9 * abs(th["ke"])
    assert e.thermo()["step"] == 5


@pytest.mark.parametrize("T_start,T_end", [(0.22495, 0.4499), (0.67485, 0.4499)])
def test_ramp_matches_oracle(cuda_lib, g1000, T_start, T_end):
    """A coldstart-like heating and a breakxal-like cooling ramp: the same
    number of NVE leap-frog steps with the same per-step rescale (the end
    temperature 0.4499 keeps the last step's comparison T < T_end away from a
    tie, where the two sides' last-bit differences could change the count)."""
    st = golden_state(g1000)
    e = engine_for(st, shuffle=1, seed=5)
    o = oracle_for(st)
    k = e.start_ramp(0, T_start, T_end, 0.1)
    ko = o.ramp(T_start, T_end, 0.1)
    assert k == ko and k > 400
    d0 = e.get_directions()
    e.step(k)
    th = e.thermo()
    assert th["step"] == 0  # ramp steps do not advance the run's step counter
    assert np.array_equal(e.get_directions(), d0)  # nor shuffle
    x, xu, p, F = e.get_state()
    xo, xuo, po, Fo = o.get_state()
    assert np.abs(xu - xuo).max() < 1e-8
    assert np.abs(p - po).max() / np.sqrt((po ** 2).sum(axis=1).mean()) < 1e-8
    assert abs(e.adjust_temperature(0, T_end) - o.adjust_temp(T_end)) < 1e-12


def test_reference_initialisation_on_device(cuda_lib):
    """initializeSystem of the reference program for one srand() seed: the
    host's rand() draws, the device's grid placement, coldstart and breakxal
    ramps and final rescale, against the oracle (bit-exact to the reference
    program for these draws); then the first run-loop shuffle on the device
    equals the reference's."""
    from activechi4_b200 import Engine, default_params
    from activechi4_b200.init import State, box_length, initialize_systems, reference_draws
    from oracle import Oracle
    from test_oracle_vs_reference import lattice_positions
    n, T, seed = 1000, 0.4499, 4242
    d = reference_draws(n, seed, jobno=3)
    e = Engine(default_params(n, T=T, f0=1.0))
    lengths = initialize_systems(e, {0: d}, T)
    x = lattice_positions(d.site, n)
    st = State(box_length(n), x, x.copy(), d.p.copy(), d.type, d.act_tag, d.k)
    o = Oracle(n, st.nact, st.L, T, 1.0)
    o.set_state(st)
    o.set_nhc(np.zeros(3), np.zeros(3))
    o.rebuild()
    o.forces()
    assert lengths["coldstart"][0] == o.ramp(0.5 * T, T, 0.1)
    assert lengths["breakxal"][0] == o.ramp(1.5 * T, T, 0.1)
    o.adjust_temp(T)
    xg, xug, pg, Fg = e.get_state()
    xo, xuo, po, Fo = o.get_state()
    # ~900 steps: rounding differences grow chaotically (measured 1.2e-8 in
    # the momenta), so 1e-7 here against 1e-8 for the single ramps
    assert np.abs(xug - xuo).max() < 1e-8
    assert np.abs(pg - po).max() / np.sqrt((po ** 2).sum(axis=1).mean()) < 1e-7
    e.set_nhc(0, np.zeros(3), np.zeros(3))
    e.step(1)
    o.seed_rng(d.gsl_seed)
    o.shuffle()
    assert np.array_equal(e.get_directions(), o.get_k())


def test_berendsen_nvt_matches_reference(cuda_lib, g1000):
    """thermostat = 2: the reference's advance_time_NVT_Berendsen (NVE step,
    then the momenta scaled towards T) for 50 steps, against the reference
    program itself."""
    from oracle import Reference, reference_available
    if not reference_available(1000):
        pytest.skip("reference library not built")
    st = golden_state(g1000)
    ref = Reference(1000)
    ref.setup(st, 0.45, 1.0)
    ref.run_berendsen(50)
    e = engine_for(st, shuffle=0, drift_every=0, thermostat=2)
    e.step(50)
    x, xu, p, F = e.get_state()
    xr, xur, pr, Fr = ref.get_state()
    assert np.abs(xu - xur).max() < 1e-9
    assert np.abs(p - pr).max() / np.sqrt((pr ** 2).sum(axis=1).mean()) < 1e-9
    th, sr = e.thermo(), ref.scalars()
    assert abs(th["ke"] - sr["ke"]) < 1e-9 * sr["ke"] and abs(th["pe"] - sr["pe"]) < 1e-9 * abs(sr["pe"])


def test_gaussian_isokinetic_matches_reference(cuda_lib, g1000):
    """thermostat = 3: the reference's AdvanceTimeNVTGaussOSM (each half kick
    p = f1 (p + f2 F), the factors from sum p.F, sum F^2 and sum p^2) for 50
    steps, against the reference program itself; the kinetic energy stays at
    its starting value."""
    from oracle import Reference, reference_available
    if not reference_available(1000):
        pytest.skip("reference library not built")
    st = golden_state(g1000)
    ref = Reference(1000)
    ref.setup(st, 0.45, 1.0)
    ref.run_gauss(50)
    e = engine_for(st, shuffle=0, drift_every=0, thermostat=3)
    ke0 = e.thermo()["ke"]
    e.step(20)
    e.step(30)
    x, xu, p, F = e.get_state()
    xr, xur, pr, Fr = ref.get_state()
    assert np.abs(xu - xur).max() < 1e-9
    assert np.abs(p - pr).max() / np.sqrt((pr ** 2).sum(axis=1).mean()) < 1e-9
    th, sr = e.thermo(), ref.scalars()
    assert abs(th["ke"] - sr["ke"]) < 1e-9 * sr["ke"] and abs(th["pe"] - sr["pe"]) < 1e-9 * abs(sr["pe"])
    assert abs(th["ke"] - ke0) < 1e-9 * ke0
    assert abs(0.5 * (p ** 2).sum() - ke0) < 1e-9 * ke0


def test_gaussian_isokinetic_drift_and_graph_match_eager(cuda_lib, g1000):
    """The Gaussian isokinetic step in the CUDA graph (with a drift removal
    every 7 steps, which re-derives the next first half from the corrected
    momenta) equals the same steps launched kernel by kernel, bit for bit; a
    ramp is refused on such a system."""
    from activechi4_b200._abi import AcgError
    st = golden_state(g1000)
    a = engine_for(st, shuffle=0, drift_every=7, thermostat=3)
    b = engine_for(st, shuffle=0, drift_every=7, thermostat=3)
    a.step(40)
    b.step_eager(40)
    for u, w in zip(a.get_state(), b.get_state()):
        assert np.array_equal(u, w)
    p = a.get_state()[2]
    assert np.abs(p.sum(axis=0)).max() < 1e-9 * np.abs(p).sum()
    with pytest.raises(AcgError):
        a.start_ramp(0, 0.2, 0.45, 0.1)


def _npt_target(ref, st):
    """A target pressure 0.3 above the starting state's (so the box shrinks)."""
    L0, _, rho0 = ref.box()
    inst = (st.p ** 2).sum() / (3.0 * st.n - 3.0)
    return rho0 * inst + ref.scalars()["virial"] / L0 ** 3 + 0.3


def test_berendsen_npt_matches_reference(cuda_lib, g1000):
    """thermostat = 4: the reference's advance_time_NPT (box rescaled by the
    Berendsen barostat and forces recomputed before each Berendsen NVT step)
    for 50 steps, against the reference program itself: positions, momenta,
    energies and the box length."""
    from oracle import Reference, reference_available
    if not reference_available(1000):
        pytest.skip("reference library not built")
    st = golden_state(g1000)
    ref = Reference(1000)
    ref.setup(st, 0.45, 1.0)
    P = _npt_target(ref, st)
    ref.run_npt(50, P)
    e = engine_for(st, shuffle=0, drift_every=0, thermostat=4, P=P, L=st.L)
    e.step(50)
    x, xu, p, F = e.get_state()
    xr, xur, pr, Fr = ref.get_state()
    Lr = ref.box()[0]
    th, sr = e.thermo(), ref.scalars()
    assert abs(th["L"] - Lr) < 1e-12 * Lr and th["L"] < st.L * (1 - 1e-4)
    assert np.abs(xu - xur).max() < 1e-9
    assert np.abs(p - pr).max() / np.sqrt((pr ** 2).sum(axis=1).mean()) < 1e-9
    assert abs(th["ke"] - sr["ke"]) < 1e-9 * sr["ke"] and abs(th["pe"] - sr["pe"]) < 1e-9 * abs(sr["pe"])


def test_berendsen_npt_graph_eager_and_reconfiguration(cuda_lib, g1000):
    """The constant-pressure step in the CUDA graph equals the kernel-by-kernel
    launches bit for bit, also across a change of the launch shape (which
    uploads the descriptors again and must keep the device's box length)."""
    st = golden_state(g1000)
    a = engine_for(st, shuffle=0, drift_every=0, thermostat=4, P=5.3, L=st.L)
    b = engine_for(st, shuffle=0, drift_every=0, thermostat=4, P=5.3, L=st.L)
    a.step(30)
    b.step_eager(30)
    cells = a.get_box_cells()
    a.set_box_cells(1 if cells != 1 else 2)
    b.set_box_cells(1 if cells != 1 else 2)
    a.step(20)
    b.step_eager(20)
    for u, w in zip(a.get_state(), b.get_state()):
        assert np.array_equal(u, w)
    assert a.thermo()["L"] == b.thermo()["L"] < st.L


def test_nose_hoover_npt_matches_reference(cuda_lib, g1000):
    """thermostat = 5: the reference's AdvanceTimeNPTNoseHoover (particle and
    barostat chains, p_eps, L = L0 exp(eps), U1..U4PropagatorNPT) for 50
    steps from the same chain and barostat state, against the reference
    program itself: positions, momenta, energies, box, eps, p_eps and both
    chains."""
    from oracle import Reference, reference_available
    if not reference_available(1000):
        pytest.skip("reference library not built")
    st = golden_state(g1000)
    p_eta, p_eta_b, p_eps, P = g1000["p_eta0"], np.array([0.1, -0.05, 0.02]), 20.0, 5.3
    ref = Reference(1000)
    ref.setup(st, 0.45, 1.0)
    ref.set_npt(np.zeros(3), p_eta, np.zeros(3), p_eta_b, p_eps)
    ref.run_nhc_npt(50, P)
    e = engine_for(st, shuffle=0, drift_every=0, thermostat=5, P=P, L=st.L)
    e.set_nhc(0, np.zeros(3), p_eta)
    e.set_barostat(0, np.zeros(3), p_eta_b, p_eps)
    e.step(25)
    e.step(25)
    x, xu, p, F = e.get_state()
    xr, xur, pr, Fr = ref.get_state()
    th, sr, nr = e.thermo(), ref.scalars(), ref.npt_state()
    Lr = ref.box()[0]
    assert abs(th["L"] - Lr) < 1e-12 * Lr and th["L"] < st.L * (1 - 1e-4)
    assert abs(th["eps"] - nr["eps"]) < 1e-12 and abs(th["p_eps"] - nr["p_eps"]) < 1e-9 * abs(nr["p_eps"])
    assert np.allclose(th["p_eta_baro"], nr["p_eta_baro"], rtol=1e-9, atol=1e-12)
    assert np.allclose(th["p_eta"], nr["p_eta"], rtol=1e-9, atol=1e-12)
    assert np.abs(xu - xur).max() < 1e-9
    assert np.abs(p - pr).max() / np.sqrt((pr ** 2).sum(axis=1).mean()) < 1e-9
    assert abs(th["ke"] - sr["ke"]) < 1e-9 * sr["ke"] and abs(th["pe"] - sr["pe"]) < 1e-9 * abs(sr["pe"])


def test_active_brownian_matches_reference(cuda_lib, g1000):
    """thermostat = 6: the reference's advance_time_ActiveBrown_PC
    (predictor-corrector with random forces minus their mean) for 30 steps,
    against the reference program itself fed the engine's random stream
    (restated on the host in tests/brown_noise.py) in place of its GSL draws."""
    from brown_noise import normals
    from oracle import Reference, reference_available
    if not reference_available(1000):
        pytest.skip("reference library not built")
    st = golden_state(g1000)
    seed, nsteps = 2024, 30
    ref = Reference(1000)
    ref.setup(st, 0.45, 1.0)
    ref.run_brown(np.stack([normals(seed, s, st.n) for s in range(nsteps)]))
    e = engine_for(st, shuffle=0, drift_every=0, thermostat=6, seed=seed, rebuild_factor=2.5)
    e.step(10)
    e.step(nsteps - 10)
    x, xu, p, F = e.get_state()
    xr, xur, pr, Fr = ref.get_state()
    assert np.abs(xu - xur).max() < 1e-9
    assert np.abs(p - pr).max() / np.sqrt((pr ** 2).sum(axis=1).mean()) < 1e-9
    th, sr = e.thermo(), ref.scalars()
    assert abs(th["pe"] - sr["pe"]) < 1e-9 * abs(sr["pe"])
    assert np.abs(xu - st.xu).max() * st.L > 0.05  # the particles moved


def test_active_brownian_graph_equals_eager(cuda_lib, g1000):
    """The Brownian step in the CUDA graph equals the kernel-by-kernel
    launches bit for bit (same random stream by particle and step)."""
    st = golden_state(g1000)
    a = engine_for(st, shuffle=1, drift_every=11, thermostat=6, seed=5)
    b = engine_for(st, shuffle=1, drift_every=11, thermostat=6, seed=5)
    a.step(40)
    b.step_eager(40)
    for u, w in zip(a.get_state(), b.get_state()):
        assert np.array_equal(u, w)
