"""The C ABI library loads without a GPU and exports every function that
include/trk.h declares; error reporting works without a device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(trk_[a-z_0-9]+)\s*\(", text)))


def test_exports_match_header():
    import elegant_b200
    lib = elegant_b200.load_library()
    missing = [n for n in declared("trk.h") if not hasattr(lib, n)]
    assert not missing, missing


def test_no_device_context_error():
    import elegant_b200
    lib = elegant_b200.load_library()
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    ctx = ctypes.c_void_p()
    rc = lib.trk_context_create(ctypes.byref(ctx), 0)
    assert rc == -5  # TRK_ERR_CUDA
    assert b"CUDA" in lib.trk_last_error() or b"device" in lib.trk_last_error()


def test_parameter_tables():
    import elegant_b200
    lib = elegant_b200.load_library()
    kq = lib.trk_type_code(b"KQUAD")
    assert kq == 3
    assert lib.trk_param_index(kq, b"N_SLICES") >= 0
    i = lib.trk_param_index(kq, b"N_SLICES")
    assert lib.trk_param_default(kq, i) == 1.0
    cs = lib.trk_type_code(b"CSBEND")
    assert lib.trk_param_index(cs, b"N_KICKS") == lib.trk_param_index(cs, b"N_SLICES")
    assert lib.trk_param_default(cs, lib.trk_param_index(cs, b"FINT")) == 0.5
    assert lib.trk_param_index(kq, b"NOPE") == -3


def test_lattice_parse_and_errors():
    import elegant_b200
    lib = elegant_b200.load_library()
    lat = ctypes.c_void_p()
    assert lib.trk_lattice_create(ctypes.byref(lat)) == 0
    text = b"""
! a FODO cell
QF: KQUAD, L=0.3, K1=1.2, N_KICKS=8
D: DRIF, L=1.0
B: CSBEND, L=1.0, ANGLE=0.0785398163, &
   N_KICKS=16
QD: QF, K1=-1.2
CELL: LINE=(QF, D, B, D, QD, D, B, D)
RING: LINE=(2*CELL, -CELL)
"""
    assert lib.trk_lattice_parse(lat, text, b"RING") == 0, lib.trk_last_error()
    assert lib.trk_lattice_length(lat) == 24
    v = ctypes.c_double()
    assert lib.trk_lattice_get(lat, 4, b"K1", ctypes.byref(v)) == 0 and v.value == -1.2
    # reversed third cell: last element of CELL first
    assert lib.trk_lattice_type(lat, 16) == 1  # D
    assert abs(lib.trk_lattice_total_length(lat) - 3 * 6.6) < 1e-12
    assert lib.trk_lattice_parse(lat, b"X: SBEN, L=1", b"X") == -2
    assert lib.trk_lattice_set(lat, 0, b"K7", 1.0) == -3
    lib.trk_lattice_destroy(lat)
