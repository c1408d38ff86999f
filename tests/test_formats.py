"""Restart, active-file and trajectory formats (activechi4_b200.formats)
against the reference's own writer and by round trips.  CPU only."""
import numpy as np
import pytest

from activechi4_b200 import formats
from activechi4_b200.init import lattice_state
from oracle import Reference, reference_available


def test_restart_bytes_match_reference_writer(tmp_path):
    n = 1000
    if not reference_available(n):
        pytest.skip("reference library not built")
    st = lattice_state(n, 0.8, seed=21)
    ref = Reference(n)
    ref.setup(st, 0.8, 1.0, p_eta=np.array([0.2, -0.1, 0.05]))
    ref.run(40)                       # unfolded coordinates leave [0, 1)
    ref.write_restart(tmp_path / "ref.dat", 20000, 7)
    x, xu, p, F = ref.get_state()
    formats.write_restart(tmp_path / "ours.dat", st.L, xu, p, st.type, 20000, 7)
    a = (tmp_path / "ref.dat").read_bytes()
    b = (tmp_path / "ours.dat").read_bytes()
    assert a == b


def test_restart_round_trip(tmp_path):
    st = lattice_state(500, 0.45, seed=3)
    xu = st.xu + np.random.default_rng(0).integers(-3, 4, size=st.xu.shape)
    formats.write_restart(tmp_path / "r.dat", st.L, xu, st.p, st.type, 5, 2)
    L, it, last, xu2, p2, t2 = formats.read_restart(tmp_path / "r.dat", st.n)
    assert (it, last) == (5, 2)
    assert abs(L - st.L) <= 1e-14 and np.abs(xu2 - xu).max() <= 1e-14 and np.abs(p2 - st.p).max() <= 1e-14
    assert np.array_equal(t2, st.type)
    # writing what was read reproduces the file (the text is a fixed point)
    formats.write_restart(tmp_path / "r2.dat", L, xu2, p2, t2, it, last)
    assert (tmp_path / "r.dat").read_bytes() == (tmp_path / "r2.dat").read_bytes()
    with pytest.raises(ValueError):
        formats.read_restart(tmp_path / "r.dat", st.n + 1)


def _applypbc_scalar(v):
    while v >= 1.0:
        v -= 1.0
    while v < 0.0:
        v += 1.0
    return v


def test_wrap_matches_applypbc():
    rng = np.random.default_rng(4)
    v = np.concatenate([rng.uniform(-6, 7, 2000), [-1e-17, -0.0, 1.0, 2.0, -3.0, 0.9999999999999999, -5e-324]])
    w = formats.wrap_repeated(v)
    assert np.array_equal(w, np.array([_applypbc_scalar(float(t)) for t in v]))
    assert (w >= 0).all() and (w <= 1).all()
    assert w[-7] == 1.0 and w[-1] == 1.0   # the reference keeps x = 1.0 for tiny negatives


def test_active_files_round_trip(tmp_path):
    st = lattice_state(1000, 0.45, seed=5)
    idx = formats.active_index_from_tag(st.act_tag)
    assert np.array_equal(formats.act_tag_from_index(st.n, idx), st.act_tag)
    formats.write_active_index(tmp_path / "ActiveFileIndex.dat", idx)
    formats.write_active_direction(tmp_path / "ActiveDirection.dat", st.k)
    assert np.array_equal(formats.read_active_index(tmp_path / "ActiveFileIndex.dat", len(idx)), idx)
    k2 = formats.read_active_direction(tmp_path / "ActiveDirection.dat", len(idx))
    assert np.array_equal(k2, np.asarray(st.k).reshape(3, -1))
    first = (tmp_path / "ActiveDirection.dat").read_text().splitlines()[0]
    kk = np.asarray(st.k).reshape(3, -1)
    assert first == "%d\t%d\t%d" % (kk[0, 0], kk[1, 0], kk[2, 0])


def test_load_restart_state(tmp_path):
    st = lattice_state(1000, 0.45, seed=6)
    xu = st.xu + np.random.default_rng(1).integers(-2, 3, size=st.xu.shape)
    formats.write_restart(tmp_path / "restart_file.dat", st.L, xu, st.p, st.type, 100000, 3)
    formats.write_active_index(tmp_path / "ActiveFileIndex.dat", formats.active_index_from_tag(st.act_tag))
    formats.write_active_direction(tmp_path / "ActiveDirection.dat", st.k)
    s2, it, last = formats.load_restart_state(tmp_path / "restart_file.dat", tmp_path / "ActiveFileIndex.dat",
                                              tmp_path / "ActiveDirection.dat", st.n)
    assert (it, last) == (100000, 3)
    assert np.array_equal(s2.x, s2.xu) and (s2.x >= 0).all() and (s2.x <= 1).all()
    assert np.abs(s2.x - st.x).max() < 1e-13
    assert np.array_equal(s2.act_tag, st.act_tag) and np.array_equal(s2.k, np.asarray(st.k).reshape(3, -1))
    (tmp_path / "bad.dat").write_text("0\n5\n5\n")
    with pytest.raises(ValueError):
        formats.load_restart_state(tmp_path / "restart_file.dat", tmp_path / "bad.dat",
                                   tmp_path / "ActiveDirection.dat", st.n)


def test_frames_and_time_index(tmp_path):
    st = lattice_state(100, 0.45, seed=7)
    formats.append_frame(tmp_path / "data_coor.out", st.xu, st.type)
    formats.append_frame(tmp_path / "data_coor.out", st.xu + 1.0, st.type)
    lines = (tmp_path / "data_coor.out").read_text().splitlines()
    assert len(lines) == 200
    assert lines[0] == "%.5f\t%.5f\t%.5f\t%d" % (st.xu[0, 0], st.xu[0, 1], st.xu[0, 2], st.type[0])
    steps = np.array([0, 1, 2, 3, 5, 7, 10, 14, 1000, 1001])
    formats.write_time_index(tmp_path / "time_index_file.dat", steps)
    assert (tmp_path / "time_index_file.dat").read_text().startswith("total timesteps equals 10\n")
    assert np.array_equal(formats.read_time_index(tmp_path / "time_index_file.dat"), steps)
