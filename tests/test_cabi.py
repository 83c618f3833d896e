"""The C-ABI library: it builds for sm_100a, loads, and exports every entry
point include/vring_b200.h declares.  No compute call runs here."""
import ctypes
import os
import subprocess

import pytest


def test_library_exports_every_declared_symbol():
    import vring_b200 as V
    from vring_b200 import build
    build.build()
    assert os.path.exists(V.LIB_PATH)
    out = subprocess.run(["nm", "-D", "--defined-only", V.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    declared = V.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    L = V.lib()
    for s in declared:
        assert hasattr(L, s)


def test_library_targets_sm100a():
    import vring_b200 as V
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", V.LIB_PATH],
                         capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import vring_b200 as V
    with pytest.raises(V.VrError) as e:
        V.Run(8, 16, 16, 4.0, 12.0, 1e-3, 100.0)
    assert e.value.code in (10, 3)


def test_descriptor_validation_codes():
    import vring_b200 as V
    from vring_b200.api import Desc
    L = V.lib()
    h = ctypes.c_void_p()
    bad = Desc(99, 8, 16, 16, 4.0, 12.0, 1e-3, 100.0, 1.0, 0.0, 0, 0, 0, 0, 0)
    assert L.vr_create(ctypes.byref(bad), ctypes.byref(h)) == 1      # VR_ERR_DESC: abi
    bad = Desc(1, 2, 16, 16, 4.0, 12.0, 1e-3, 100.0, 1.0, 0.0, 0, 0, 0, 0, 0)
    assert L.vr_create(ctypes.byref(bad), ctypes.byref(h)) == 1      # ntheta < 3
    bad = Desc(1, 8, 16, 16, -4.0, 12.0, 1e-3, 100.0, 1.0, 0.0, 0, 0, 0, 0, 0)
    assert L.vr_create(ctypes.byref(bad), ctypes.byref(h)) == 1      # rmax <= 0
    bad = Desc(1, 300, 16, 16, 4.0, 12.0, 1e-3, 100.0, 1.0, 0.0, 1, 0, 0, 0, 0)
    assert L.vr_create(ctypes.byref(bad), ctypes.byref(h)) == 1      # VR_MIXED: ntheta > 257
    bad = Desc(1, 8, 16, 16, 4.0, 12.0, 1e-3, 100.0, 1.0, 0.0, 2, 0, 0, 0, 0)
    assert L.vr_create(ctypes.byref(bad), ctypes.byref(h)) == 1      # unknown precision
    assert L.vr_create(None, ctypes.byref(h)) == 8                   # VR_ERR_ARG


def test_analysis_line_uses_gfortran_e16_8():
    """analysis.dat is written with (I5,20(E16.8)) (run.F90:383); the library's
    formatter follows gfortran's Ew.d layout: 0.d1..d8, exponent letter and a
    two-digit exponent (three digits and no letter beyond 99)."""
    from vring_b200.api import format_e16_8 as f
    assert f(1.0) == "  0.10000000E+01"
    assert f(-3.141592653589793) == " -0.31415927E+01"
    assert f(123456789.0) == "  0.12345679E+09"
    assert f(2.5e-5) == "  0.25000000E-04"
    assert f(0.0) == "  0.00000000E+00"
    assert f(1e-101) == "  0.10000000-100"
    assert f(float("nan")) == "             NaN"
    assert all(len(f(x)) == 16 for x in (1.0, -1e300, 7e-7, 0.999999999))
