"""CUDA timestep against the reference's golden outputs and the oracle.

Tolerances (stated per test): cell assignment and in-cell order bit-exact;
FP64 forces max|dF|/rms|F| <= 1e-12, energy and virials 1e-12 relative right
after a list rebuild; trajectories after 50 steps within 1e-9 (chaotic growth
of rounding differences); FP32 pair forces max|dF|/rms|F| <= 1e-5."""
import numpy as np
import pytest

from conftest import force_err, golden_state, rel

pytestmark = pytest.mark.gpu


def engine_for(g, nsys=1, **kw):
    from activechi4_b200 import Engine, default_params
    st = golden_state(g)
    kw.setdefault("shuffle", 0)
    p = default_params(st.n, T=0.45, f0=1.0, **kw)
    e = Engine([p] * nsys)
    for r in range(nsys):
        e.set_state(r, st)
        e.set_nhc(r, g["eta0"], g["p_eta0"])
    return e


@pytest.mark.parametrize("name", ["g1000", "g4000"])
def test_cells_bit_exact(cuda_lib, name, request):
    g = request.getfixturevalue(name)
    e = engine_for(g)
    dims, counts, members = e.cells()
    assert np.array_equal(dims, g["cell_dims"])
    assert np.array_equal(counts, g["cell_counts"])
    assert np.array_equal(members, g["cell_members"])


@pytest.mark.parametrize("name", ["g1000", "g4000"])
@pytest.mark.parametrize("list_mode", [0, 1])
def test_forces_fp64(cuda_lib, name, list_mode, request):
    g = request.getfixturevalue(name)
    e = engine_for(g, list_mode=list_mode)
    e.compute_forces()
    F = e.get_state()[3]
    th = e.thermo()
    assert force_err(F, g["F0"]) <= 1e-12
    assert rel(th["pe"], g["pe0"]) <= 1e-12
    assert rel(th["virial"], g["vir0"]) <= 1e-12
    assert abs(th["vir_act"] - g["viract0"]) <= 1e-12 * max(1.0, abs(g["viract0"]))


def test_forces_neighbour_overflow_fallback(cuda_lib, g1000):
    """A row capacity of 32 sends every particle to the cell-list path."""
    e = engine_for(g1000, nb_capacity=32)
    e.compute_forces()
    assert force_err(e.get_state()[3], g1000["F0"]) <= 1e-12
    assert e.thermo()["overflow"] == 1000


def _check_traj(e, g, pre, tol=1e-9):
    x, xu, p, F = e.get_state()
    assert np.abs(xu - g[pre + "xu"]).max() < tol
    dx = np.abs(x - g[pre + "x"])
    assert np.minimum(dx, 1.0 - dx).max() < tol  # wrapped coordinates
    prms = np.sqrt((g[pre + "p"] ** 2).sum(axis=1).mean())
    assert np.abs(p - g[pre + "p"]).max() / prms < tol
    assert force_err(F, g[pre + "F"]) < tol
    th = e.thermo()
    assert rel(th["pe"], g[pre + "pe"]) < tol
    assert rel(th["ke"], g[pre + "ke"]) < tol
    assert rel(th["virial"], g[pre + "virial"]) < tol
    assert np.allclose(th["p_eta"], g[pre + "p_eta"], rtol=tol, atol=tol)
    assert np.allclose(th["eta"], g[pre + "eta"], rtol=tol, atol=tol)


@pytest.mark.parametrize("name", ["g1000", "g4000"])
def test_nvt_50_steps(cuda_lib, name, request):
    g = request.getfixturevalue(name)
    e = engine_for(g)
    e.step(50)
    _check_traj(e, g, "nvt_")
    assert e.thermo()["step"] == 50
    assert e.thermo()["rebuilds"] == 1 + g["nvt_rebuilds"]  # + the set-up build


def test_shuffled_directions_50_steps(cuda_lib, g1000):
    """The reference shuffles at step 0 with its own RNG; the same directions
    handed to the device reproduce its trajectory."""
    e = engine_for(g1000)
    e.compute_forces()  # initial forces with the pre-shuffle directions, as the reference
    e.set_directions(0, g1000["shf_k"])
    e.step(50)
    _check_traj(e, g1000, "shf_")


def test_nve_50_steps(cuda_lib, g1000):
    e = engine_for(g1000, thermostat=0)
    e.step(50)
    x, xu, p, F = e.get_state()
    assert np.abs(xu - g1000["nve_xu"]).max() < 1e-9
    prms = np.sqrt((g1000["nve_p"] ** 2).sum(axis=1).mean())
    assert np.abs(p - g1000["nve_p"]).max() / prms < 1e-9


def test_graph_and_eager_identical(cuda_lib, g1000):
    a = engine_for(g1000, shuffle=1, tau_p_steps=20)
    b = engine_for(g1000, shuffle=1, tau_p_steps=20)
    a.step(70)
    b.step_eager(70)
    for u, w in zip(a.get_state(), b.get_state()):
        assert np.array_equal(u, w)
    assert np.array_equal(a.get_directions(), b.get_directions())


def test_oracle_random_states(cuda_lib):
    from activechi4_b200 import Engine, default_params, lattice_state
    from oracle import Oracle
    for n, seed in ((1000, 21), (8000, 22), (27000, 23)):
        st = lattice_state(n, 1.0, seed=seed)
        o = Oracle.from_state(st, 1.0, 2.0, p_eta=np.array([0.1, 0.2, 0.3]))
        o.run(40)  # melt the lattice a little on the CPU
        x, xu, p, _ = o.get_state()
        st.x, st.xu, st.p = x, xu, p
        Fo, pe, vir, va = Oracle.from_state(st, 1.0, 2.0).forces()
        e = Engine(default_params(n, T=1.0, f0=2.0, shuffle=0))
        e.set_state(0, st)
        e.compute_forces()
        assert force_err(e.get_state()[3], Fo) <= 1e-12
        th = e.thermo()
        assert rel(th["pe"], pe) <= 1e-12 and rel(th["virial"], vir) <= 1e-12
        e.close()


def test_fp32_pair_forces(cuda_lib, g4000):
    e = engine_for(g4000, precision=1)
    e.compute_forces()
    err = force_err(e.get_state()[3], g4000["F0"])
    assert err <= 1e-5, err
    th = e.thermo()
    assert rel(th["pe"], g4000["pe0"]) <= 1e-5


def test_fp32_pair_forces_all_paths(cuda_lib):
    """FP32 pair forces against the C restatement (FP64) on each force path:
    N = 8000 and 16000 take the per-particle kernels (6 and 7 cells per side,
    N <= 20000), N = 27000 the cell groups split over several blocks; both list
    cuts; max|dF|/rms|F| and pe within 1e-5."""
    from activechi4_b200 import Engine, default_params, lattice_state
    from oracle import Oracle
    for n, seed, lm in ((8000, 31, 0), (16000, 32, 1), (27000, 33, 1)):
        st = lattice_state(n, 1.0, seed=seed)
        o = Oracle.from_state(st, 1.0, 2.0, p_eta=np.array([0.1, 0.2, 0.3]))
        o.run(40)
        x, xu, p, _ = o.get_state()
        st.x, st.xu, st.p = x, xu, p
        Fo, pe, vir, va = Oracle.from_state(st, 1.0, 2.0).forces()
        e = Engine(default_params(n, T=1.0, f0=2.0, shuffle=0, precision=1, list_mode=lm))
        e.set_state(0, st)
        e.compute_forces()
        assert force_err(e.get_state()[3], Fo) <= 1e-5, n
        th = e.thermo()
        assert rel(th["pe"], pe) <= 1e-5 and rel(th["virial"], vir) <= 1e-5
        e.close()


def test_list_by_cells_staging_overflow(cuda_lib):
    """A per-particle system (N = 8000, 6 cells per side) squeezed into x <
    0.45: cells in the dense slab have more neighbour candidates than the list
    build by cells stages (~2000 against ~1630), so their particles take the
    force kernel's cell scan (rows of 512 entries, so that the row capacity is
    not what overflows).  Against the C restatement: FP64 forces <= 1e-12,
    pe and virial <= 1e-11 (here sums of ~1e6 pair terms up to ~1e5 each, the
    overlapping particles of the squeezed slab, summed in another order), FP32
    pair forces, pe and virial <= 1e-5."""
    from activechi4_b200 import Engine, default_params, lattice_state
    from oracle import Oracle
    n = 8000
    st = lattice_state(n, 1.0, seed=41)
    st.x[:, 0] *= 0.45
    st.xu = st.x.copy()
    Fo, pe, vir, _ = Oracle.from_state(st, 1.0, 2.0).forces()
    for prec, tol, tol_sum in ((0, 1e-12, 1e-11), (1, 1e-5, 1e-5)):
        e = Engine(default_params(n, T=1.0, f0=2.0, shuffle=0, nb_capacity=512, precision=prec))
        e.set_state(0, st)
        e.compute_forces()
        th = e.thermo()
        assert th["overflow"] > 0
        err = force_err(e.get_state()[3], Fo)
        assert err <= tol, (prec, err)
        assert rel(th["pe"], pe) <= tol_sum and rel(th["virial"], vir) <= tol_sum, prec
        e.close()


def test_batched_bricks_past_32(cuda_lib):
    """Twelve whole-box replicas (N = 1800 at rho = 0.8: 4 cells and 9 list
    sub-cells per side, bricks of 2 x 2 x 2 sub-cells with ~20 particles
    expected; 21600 particles in all, so the engine lists by bricks) with x
    squeezed into [0, 0.6) in the odd replicas: ~30 bricks of each of those
    hold more than 32 particles, and their particles past 32 are listed one
    warp each.  Against the C restatement for every replica: FP64 forces <=
    1e-12, pe and virial <= 1e-11; FP32 pair forces, pe and virial <= 1e-5."""
    from activechi4_b200 import Engine, default_params, lattice_state
    from oracle import Oracle
    n, rho, nrep = 1800, 0.8, 12
    sts = []
    for k in range(nrep):
        st = lattice_state(n, 1.0, seed=200 + k, density=rho)
        if k % 2:
            st.x[:, 0] *= 0.6
            st.xu = st.x.copy()
        sts.append(st)
    ref = [Oracle.from_state(st, 1.0, 2.0).forces() for st in sts]
    for prec, tol, tol_sum in ((0, 1e-12, 1e-11), (1, 1e-5, 1e-5)):
        p = default_params(n, T=1.0, f0=2.0, shuffle=0, precision=prec, density=rho)
        e = Engine([p] * nrep)
        for k, st in enumerate(sts):
            e.set_state(k, st)
        e.compute_forces()
        for k in range(nrep):
            Fo, pe, vir, _ = ref[k]
            err = force_err(e.get_state(k)[3], Fo)
            assert err <= tol, (prec, k, err)
            th = e.thermo(k)
            assert rel(th["pe"], pe) <= tol_sum and rel(th["virial"], vir) <= tol_sum, (prec, k)
        e.close()


def test_batch_members_identical_to_alone(cuda_lib, g1000, g4000):
    from activechi4_b200 import Engine, default_params, lattice_state
    st3 = lattice_state(2000, 0.6, seed=9)
    cases = [(golden_state(g1000), dict(T=0.45, f0=1.0, tau_p_steps=20, seed=1)),
             (golden_state(g4000), dict(T=0.5, f0=2.0, tau_p_steps=200, seed=2)),
             (st3, dict(T=0.6, f0=0.5, tau_p_steps=2000, seed=3))]
    params = [default_params(s.n, **kw) for s, kw in cases]
    alone = []
    for (s, _), p in zip(cases, params):
        e = Engine(p)
        e.set_state(0, s)
        e.set_nhc(0, [0, 0, 0], [0.2, 0.1, -0.1])
        e.step(100)
        alone.append((e.get_state(), e.get_directions(), e.thermo()))
    b = Engine(params)
    for r, (s, _) in enumerate(cases):
        b.set_state(r, s)
        b.set_nhc(r, [0, 0, 0], [0.2, 0.1, -0.1])
    b.step(100)
    for r in range(3):
        st, k, th = alone[r]
        for u, w in zip(st, b.get_state(r)):
            assert np.array_equal(u, w)
        assert np.array_equal(k, b.get_directions(r))
        tb = b.thermo(r)
        assert th["pe"] == tb["pe"] and th["heff"] == tb["heff"]


def test_device_shuffle_keeps_counts(cuda_lib, g4000):
    e = engine_for(g4000, shuffle=1, tau_p_steps=10, seed=77)
    k0 = e.get_directions()
    e.step(1)
    k1 = e.get_directions()
    assert not np.array_equal(k0, k1)
    assert np.array_equal(k1.sum(axis=1), k0.sum(axis=1))
    assert np.all(np.abs(k1) == 1)
    # each component is permuted independently
    assert not np.array_equal(k1[0], k1[1])
    e.step(9)
    assert np.array_equal(e.get_directions(), k1)  # no shuffle before step 10
    e.step(1)
    assert not np.array_equal(e.get_directions(), k1)


def test_nonfinite_state_is_reported(cuda_lib, g1000):
    from activechi4_b200._abi import AcgError
    st = golden_state(g1000)
    st.x[1] = st.x[0]  # two particles on top of each other
    st.xu[1] = st.xu[0]
    from activechi4_b200 import Engine, default_params
    e = Engine(default_params(1000, shuffle=0))
    e.set_state(0, st)
    e.step(2)
    with pytest.raises(AcgError) as ei:
        e.thermo()
    assert ei.value.code == -4


def test_reused_step_graph_matches_eager(cuda_lib, g1000):
    """A closed engine leaves its device-loop step graph for reuse by the next
    engine of the same shape (updated in place, not instantiated anew); the
    reusing engine must step exactly like the eager launches."""
    a = engine_for(g1000, shuffle=1, tau_p_steps=20)
    a.step(70)
    a.close()
    b = engine_for(g1000, shuffle=1, tau_p_steps=20)
    c = engine_for(g1000, shuffle=1, tau_p_steps=20)
    b.step(70)
    c.step_eager(70)
    for u, w in zip(b.get_state(), c.get_state()):
        assert np.array_equal(u, w)
    assert b.thermo()["rebuilds"] == c.thermo()["rebuilds"]


@pytest.mark.parametrize("n,rho", [(300, 1.2), (600, 1.2), (1500, 1.2), (2500, 1.2), (3400, 1.2), (380, 0.9),
                                   (1800, 0.8)])
def test_whole_box_list_paths(cuda_lib, n, rho):
    """Whole-box systems of every list geometry against the oracle: 2 cells per
    side with fewer than 5 list sub-cells (minimum-image pass, n=300), 5
    sub-cells per side where a brick's neighbourhood is wider than the box
    (n=600; at rho=0.9, n=380, on all three axes), 3 and 4 cells per side with
    7 to 9 sub-cells, bricks of depth 1 (rho=1.2) and 2 (rho=0.8, n=1800).
    FP64 forces, pe and virial <= 1e-12 (both list cuts); FP32 pair forces
    <= 1e-5."""
    from activechi4_b200 import Engine, default_params, lattice_state
    from oracle import Oracle
    st = lattice_state(n, 1.0, seed=100 + n, density=rho)
    o = Oracle.from_state(st, 1.0, 2.0, p_eta=np.array([0.1, 0.2, 0.3]))
    o.run(40)  # melt the lattice a little on the CPU
    x, xu, p, _ = o.get_state()
    st.x, st.xu, st.p = x, xu, p
    for list_mode in (0, 1):
        Fo, pe, vir, _ = Oracle.from_state(st, 1.0, 2.0, list_mode=list_mode).forces()
        for prec, tol in ((0, 1e-12), (1, 1e-5)):
            e = Engine(default_params(n, T=1.0, f0=2.0, shuffle=0, list_mode=list_mode, precision=prec,
                                      density=rho))
            e.set_state(0, st)
            e.compute_forces()
            assert e.thermo()["overflow"] == 0
            err = force_err(e.get_state()[3], Fo)
            assert err <= tol, (n, list_mode, prec, err)
            th = e.thermo()
            assert rel(th["pe"], pe) <= tol and rel(th["virial"], vir) <= tol, (n, list_mode, prec)
            e.close()
