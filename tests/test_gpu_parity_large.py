"""The headline configuration (N = 100 000, 15 cells per side: the cell-group
list and force kernels) against the reference program compiled from its own
sources, and N = 256 000 (20 cells per side, the largest served size)
against the oracle.

Tolerances: cells and in-cell order bit-exact; FP64 forces max|dF|/rms|F| <=
1e-12 and pe / virial / active virial <= 1e-12 relative right after a
rebuild; 50 NVT steps (the direction shuffle at step 0 drawn on the device
from the same MT19937 seed, the drift removal after step 0) within 1e-9;
FP32 pair forces <= 1e-5."""
import numpy as np
import pytest

from conftest import force_err, rel

pytestmark = pytest.mark.gpu


def melted(n, seed):
    """A lattice start melted on the device (300 steps at T = 2, 200 at 0.45):
    only an input configuration, handed to both sides."""
    from activechi4_b200 import Engine, default_params, lattice_state
    st = lattice_state(n, 2.0, seed=seed)
    e = Engine(default_params(n, T=2.0, f0=1.0, shuffle=2, seed=seed))
    e.set_state(0, st)
    e.set_nhc(0, np.zeros(3), np.array([0.2, -0.1, 0.05]))
    e.step(300)
    e.set_temperature(0, 0.45)
    e.step(200)
    x, xu, p, _ = e.get_state()
    st.x, st.xu, st.p = x, xu, p
    st.k = e.get_directions()
    e.close()
    return st


@pytest.fixture(scope="module")
def s100k(cuda_lib):
    return melted(100000, 11)


@pytest.fixture(scope="module")
def ref100k(s100k):
    from oracle import Reference, reference_available
    if not reference_available(100000):
        pytest.skip("reference library for N=100000 not built")
    return Reference(100000)


P_ETA = np.array([0.05, -0.02, 0.01])


def gpu(st, **kw):
    from activechi4_b200 import Engine, default_params
    kw.setdefault("shuffle", 0)
    e = Engine(default_params(st.n, T=0.45, f0=1.0, **kw))
    e.set_state(0, st)
    e.set_nhc(0, np.zeros(3), P_ETA)
    return e


def test_cells_forces_n100k(s100k, ref100k):
    ref100k.setup(s100k, 0.45, 1.0, p_eta=P_ETA)
    e = gpu(s100k)
    dims, counts, members = e.cells()
    rd, rc, rm = ref100k.cells()
    assert dims.tolist() == [15, 15, 15]
    assert np.array_equal(dims, rd) and np.array_equal(counts, rc) and np.array_equal(members, rm)
    Fr, pe, vir, va = ref100k.forces()
    e.compute_forces()
    th = e.thermo()
    assert force_err(e.get_state()[3], Fr) <= 1e-12
    assert rel(th["pe"], pe) <= 1e-12 and rel(th["virial"], vir) <= 1e-12
    assert abs(th["vir_act"] - va) <= 1e-12 * max(1.0, abs(va))
    assert th["overflow"] == 0
    e.close()
    e = gpu(s100k, precision=1)
    e.compute_forces()
    assert force_err(e.get_state()[3], Fr) <= 1e-5
    e.close()


def test_nvt_50_steps_n100k(s100k, ref100k):
    """The run loop's first 50 steps: shuffle at step 0 (device MT19937 with
    the reference's seed), NHC NVT, the drift removal after step 0."""
    ref100k.setup(s100k, 0.45, 1.0, p_eta=P_ETA)
    ref100k.seed_rng(606)
    nref = ref100k.run(50, start=0, shuffle=True, drift=True)
    e = gpu(s100k, shuffle=1, seed=606)
    e.step(50)
    th = e.thermo()
    assert th["step"] == 50
    assert th["rebuilds"] == 1 + nref
    assert np.array_equal(e.get_directions(), ref100k.get_k())
    x, xu, p, F = e.get_state()
    xr, xur, pr, Fr = ref100k.get_state()
    assert np.abs(xu - xur).max() < 1e-9
    dx = np.abs(x - xr)
    assert np.minimum(dx, 1.0 - dx).max() < 1e-9
    assert np.abs(p - pr).max() / np.sqrt((pr ** 2).sum(axis=1).mean()) < 1e-9
    assert force_err(F, Fr) < 1e-9
    sr = ref100k.scalars()
    assert rel(th["pe"], sr["pe"]) < 1e-9 and rel(th["ke"], sr["ke"]) < 1e-9
    eta, p_eta, _ = ref100k.get_nhc()
    assert np.allclose(th["p_eta"], p_eta, rtol=1e-9, atol=1e-9)
    assert np.allclose(th["eta"], eta, rtol=1e-9, atol=1e-9)
    e.close()


def test_forces_n256k_against_oracle(cuda_lib):
    from oracle import Oracle
    st = melted(256000, 12)
    o = Oracle.from_state(st, 0.45, 1.0)
    Fo, pe, vir, va = o.forces()
    e = gpu(st)
    dims, counts, members = e.cells()
    od, oc, om = o.cells()
    assert dims.tolist() == [20, 20, 20]
    assert np.array_equal(dims, od) and np.array_equal(counts, oc) and np.array_equal(members, om)
    e.compute_forces()
    th = e.thermo()
    assert force_err(e.get_state()[3], Fo) <= 1e-12
    assert rel(th["pe"], pe) <= 1e-12 and rel(th["virial"], vir) <= 1e-12
    e.close()
    e = gpu(st, precision=1)
    e.compute_forces()
    assert force_err(e.get_state()[3], Fo) <= 1e-5
    e.close()
