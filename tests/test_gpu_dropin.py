"""The reference program with its timestep files replaced by the drop-in C
files (activechi4_b200/legacy) against the unmodified reference, both built
from the reference's sources (oracle/_ref; skipped where not built).  The
reference's own host code (Parallel.c, active.c, initialise.c, ...) drives
the GPU through the drop-in entry points.  Tolerances as the parity tests:
cells bit-exact, forces 1e-12, trajectories (with the reference's host
direction shuffles) 1e-9 after 60 steps."""
import numpy as np
import pytest

from conftest import force_err, golden_state, rel

pytestmark = pytest.mark.gpu


def test_dropin_program_matches_reference(cuda_lib, g1000):
    from oracle import Reference, reference_available
    if not (reference_available(1000) and reference_available(1000, "dropin")):
        pytest.skip("reference / drop-in programs not built")
    st = golden_state(g1000)
    ref, dro = Reference(1000), Reference(1000, "dropin")
    for r in (ref, dro):
        r.setup(st, 0.45, 1.0, g1000["eta0"], g1000["p_eta0"])
    for a, b in zip(ref.cells(), dro.cells()):
        assert np.array_equal(a, b)
    Fr, per, vr, var = ref.forces()
    Fd, ped, vd, vad = dro.forces()
    assert force_err(Fd, Fr) <= 1e-12 and rel(ped, per) <= 1e-12 and rel(vd, vr) <= 1e-12
    for r in (ref, dro):
        r.setup(st, 0.45, 1.0, g1000["eta0"], g1000["p_eta0"])
        r.seed_rng(99)
    nr = ref.run(60, shuffle=True)
    nd = dro.run(60, shuffle=True)
    assert nr == nd
    xr, xur, pr, _ = ref.get_state()
    xd, xud, pd, _ = dro.get_state()
    assert np.abs(xud - xur).max() < 1e-9
    assert np.abs(pd - pr).max() / np.sqrt((pr ** 2).sum(axis=1).mean()) < 1e-9
    assert np.array_equal(ref.get_k(), dro.get_k())
    er, pr_eta, _ = ref.get_nhc()
    ed, pd_eta, _ = dro.get_nhc()
    assert np.allclose(pd_eta, pr_eta, rtol=1e-9, atol=1e-12)
    sr, sd = ref.scalars(), dro.scalars()
    assert rel(sd["ke"], sr["ke"]) < 1e-9 and rel(sd["pe"], sr["pe"]) < 1e-9
    ref.run_nve(20)
    dro.run_nve(20)
    assert np.abs(dro.get_state()[1] - ref.get_state()[1]).max() < 1e-9


def test_dropin_sync_points(cuda_lib, g1000):
    """The drop-in's step reads back only scalars; the reference's own
    routines that read or write the particles (fixDrift here, through the
    linker's wrapper; the run loop's fixDrift every 100000 steps from index
    0) see the device's state and their edits reach the device.  The
    propagators U1..U4 on the host mirror compose the same NVT step."""
    from oracle import Reference, reference_available
    if not (reference_available(1000) and reference_available(1000, "dropin")):
        pytest.skip("reference / drop-in programs not built")
    st = golden_state(g1000)
    st.p[:, 0] += 0.1  # a net momentum for fixDrift
    ref, dro = Reference(1000), Reference(1000, "dropin")
    for r in (ref, dro):
        r.setup(st, 0.45, 1.0, g1000["eta0"], g1000["p_eta0"])
        r.seed_rng(7)
        r.run(30, start=0, shuffle=True, drift=True)  # fixDrift after loop index 0
        r.fix_drift()
        r.run(30, start=30, shuffle=True)
    xr, xur, pr, _ = ref.get_state()
    xd, xud, pd, _ = dro.get_state()
    assert np.abs(xud - xur).max() < 1e-9
    assert np.abs(pd - pr).max() / np.sqrt((pr ** 2).sum(axis=1).mean()) < 1e-9
    assert abs(pd.sum(axis=0)).max() < 1e-9
    # the same NVT step composed from the exported propagators
    for r in (ref, dro):
        r.step_propagators(10)
    xr, xur, pr, _ = ref.get_state()
    xd, xud, pd, _ = dro.get_state()
    assert np.abs(xud - xur).max() < 1e-9
    assert np.abs(pd - pr).max() / np.sqrt((pr ** 2).sum(axis=1).mean()) < 1e-9



def test_dropin_berendsen_and_gaussian_steps(cuda_lib, g1000):
    """advance_time_NVT_Berendsen and AdvanceTimeNVTGaussOSM of the drop-in
    (each on its own device engine, the state handed over through sphere[])
    against the reference program's own, 30 steps each in a row."""
    from oracle import Reference, reference_available
    if not (reference_available(1000) and reference_available(1000, "dropin")):
        pytest.skip("reference / drop-in programs not built")
    st = golden_state(g1000)
    ref, dro = Reference(1000), Reference(1000, "dropin")
    for r in (ref, dro):
        r.setup(st, 0.45, 1.0, g1000["eta0"], g1000["p_eta0"])
        r.run_berendsen(30)
        r.run_gauss(30)
    xr, xur, pr, _ = ref.get_state()
    xd, xud, pd, _ = dro.get_state()
    assert np.abs(xud - xur).max() < 1e-9
    assert np.abs(pd - pr).max() / np.sqrt((pr ** 2).sum(axis=1).mean()) < 1e-9
    sr, sd = ref.scalars(), dro.scalars()
    assert rel(sd["ke"], sr["ke"]) < 1e-9 and rel(sd["pe"], sr["pe"]) < 1e-9
    assert rel(sd["inst_T"], sr["inst_T"]) < 1e-9
