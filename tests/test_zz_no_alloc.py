"""The allocation-free entry point (acg_forces_noalloc) against the existing
force entry point (acg_compute_forces), through the C ABI.

acg_forces_noalloc serves callers that cannot allocate device memory (a host
framework that owns all device memory, a loop that forbids allocation after
start-up, a plug-in handed only device pointers).  It keeps its intermediates
in one fixed device array shared by all calls, so the test calls it twice in
a row — the same system, then a different one — and checks that each result
matches the engine's forces within the FP64 tolerance used elsewhere
(max|dF|/rms|F| <= 1e-12, energy and virials 1e-12 relative)."""
import ctypes as C

import numpy as np
import pytest

from conftest import force_err, golden_state, rel

pytestmark = pytest.mark.gpu


def _engine_forces(st, f0):
    from activechi4_b200 import Engine, default_params
    e = Engine(default_params(st.n, f0=f0, shuffle=0, nact=st.nact))
    e.set_state(0, st)
    e.compute_forces()
    F = e.get_state(0)[3]
    th = e.thermo(0)
    e.close()
    return F, th["pe"], th["virial"], th["vir_act"]


def _noalloc_forces(lib, st, f0, with_xu=True):
    import torch
    dev = torch.device("cuda:0")
    x = torch.tensor(st.x, dtype=torch.float64, device=dev).contiguous()
    xu = torch.tensor(st.xu, dtype=torch.float64, device=dev).contiguous() if with_xu else None
    ty = torch.tensor(st.type, dtype=torch.int32, device=dev).contiguous()
    act = torch.tensor(st.act_tag, dtype=torch.int32, device=dev).contiguous()
    k = (torch.tensor(np.asarray(st.k).reshape(-1), dtype=torch.int32, device=dev).contiguous()
         if st.nact else None)
    F = torch.full((st.n, 3), float("nan"), dtype=torch.float64, device=dev)
    out = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    p = lambda t: None if t is None else C.c_void_p(t.data_ptr())  # noqa: E731
    rc = lib.acg_forces_noalloc(p(x), p(xu), p(ty), p(act), p(k), st.n, st.nact, st.L, f0, p(F), p(out),
                                C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.acg_last_error().decode()
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    return F.cpu().numpy(), o[0], o[1], o[2]


def test_noalloc_matches_engine_twice(cuda_lib, g1000, g4000):
    lib = cuda_lib
    for g, f0 in ((g1000, 1.0), (g1000, 1.0), (g4000, 2.0)):
        st = golden_state(g)
        Fe, pe, vir, va = _engine_forces(st, f0)
        Fn, pen, virn, van = _noalloc_forces(lib, st, f0)
        assert force_err(Fn, Fe) <= 1e-12
        assert rel(pen, pe) <= 1e-12 and rel(virn, vir) <= 1e-12
        assert abs(van - va) <= 1e-12 * max(1.0, abs(va))


def test_noalloc_golden_and_small_boxes(cuda_lib, g1000, g500):
    """Against the reference's own forces (golden N=1000) and, for a box of
    two cells per side (N=500, neighbour offsets 0..1), against the oracle,
    which counts each pair once there; then a system without active
    particles and without unfolded coordinates (xu and k NULL)."""
    from oracle import Oracle
    lib = cuda_lib
    st = golden_state(g1000)
    Fn, pen, virn, van = _noalloc_forces(lib, st, 1.0)
    assert force_err(Fn, g1000["F0"]) <= 1e-12
    assert rel(pen, g1000["pe0"]) <= 1e-12 and rel(virn, g1000["vir0"]) <= 1e-12
    assert abs(van - g1000["viract0"]) <= 1e-12 * max(1.0, abs(g1000["viract0"]))
    st = golden_state(g500)
    Fo, peo, viro, vao = Oracle.from_state(st, 0.45, 1.0).forces()
    for _ in range(2):
        Fn, pen, virn, van = _noalloc_forces(lib, st, 1.0)
        assert force_err(Fn, Fo) <= 1e-12
        assert rel(pen, peo) <= 1e-12 and rel(virn, viro) <= 1e-12
        assert abs(van - vao) <= 1e-12 * max(1.0, abs(vao))
    st = golden_state(g1000)
    st.act_tag[:] = -1
    st.k = np.zeros((3, 0), dtype=np.int32)
    Fe, pe, vir, va = _engine_forces(st, 1.0)
    Fn, pen, virn, van = _noalloc_forces(lib, st, 1.0, with_xu=False)
    assert force_err(Fn, Fe) <= 1e-12 and rel(pen, pe) <= 1e-12 and van == 0.0


def test_noalloc_rejects_oversized_input(cuda_lib):
    lib = cuda_lib
    big = 262144 + 1
    rc = lib.acg_forces_noalloc(C.c_void_p(1), None, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), big, 0,
                                (big / 1.2) ** (1 / 3), 1.0, C.c_void_p(1), C.c_void_p(1), None)
    assert rc == -1
    assert "262144" in lib.acg_last_error().decode()
    # more cells than the scratch array holds (33^3 = 35937 > 32768)
    rc = lib.acg_forces_noalloc(C.c_void_p(1), None, C.c_void_p(1), C.c_void_p(1), None, 1000, 0, 95.0, 1.0,
                                C.c_void_p(1), C.c_void_p(1), None)
    assert rc == -1
    assert "35937" in lib.acg_last_error().decode()
