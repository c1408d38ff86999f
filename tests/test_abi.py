"""The C ABI library loads and exports everything include/activechi4.h
declares; host-side parameter logic works without a GPU.  CPU only."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def lib():
    from activechi4_b200 import build
    build.build()
    from activechi4_b200 import _abi
    return _abi.lib()


def header_functions():
    src = open(os.path.join(ROOT, "include", "activechi4.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(acg_[a-z_0-9]+)\s*\(", src)))


def test_header_matches_bindings():
    from activechi4_b200 import _abi
    assert header_functions() == sorted(_abi.exported_symbols())


def test_library_exports_every_symbol(lib):
    from activechi4_b200 import _abi
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (acg_\w+)", out))
    missing = set(header_functions()) - exported
    assert not missing, missing


def test_params_default(lib):
    from activechi4_b200 import default_params
    p = default_params(1000)
    assert (p.n, p.nact, p.tau_p_steps, p.dt, p.skin, p.rebuild_factor) == (1000, -1, 200, 0.005, 0.35, 3.0)
    assert p.thermostat == 1 and p.precision == 0


def test_footprint_and_validation(lib):
    from activechi4_b200 import default_params, footprint
    from activechi4_b200._abi import AcgError
    f1 = footprint([default_params(1000)])
    f2 = footprint([default_params(100000)])
    f3 = footprint([default_params(1000)] * 4)
    assert 0 < f1 < f2 and f3 > 3 * f1
    with pytest.raises(AcgError) as ei:
        footprint([default_params(100)])  # box below 2 cells per side
    assert ei.value.code == -1 and "box too small" in str(ei.value)
    p = default_params(1000, precision=1)
    with pytest.raises(AcgError):
        footprint([default_params(1000), p])  # mixed precision in one engine


def test_create_without_gpu_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from activechi4_b200 import Engine, default_params
    from activechi4_b200._abi import AcgError
    with pytest.raises(AcgError) as ei:
        Engine(default_params(1000))
    assert ei.value.code == -2


def test_dropin_files_define_the_reference_entry_points():
    """The drop-in C files define the timestep entry points of
    MDcode/subroutine.h that other reference files call."""
    import glob
    src = "".join(open(f).read() for f in glob.glob(os.path.join(ROOT, "activechi4_b200", "legacy", "*.c")))
    for name in ("update_cell_list", "calculate_forces", "getcell_I", "maps", "len_check",
                 "AdvanceTimeNVTNoseHoover", "advance_time_NVEFrog", "InitialiseNoseHoover",
                 "applypbc1", "applypbc"):
        assert re.search(r"\b" + name + r"\s*\([^;{]*\)\s*\{", src), name
