"""The C-ABI library: loads, exports every declared symbol, and the host-side API contract
(CPU only: no compute calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

from pm3_rs import _lib, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "pm3gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(pm3gpu_\w+)\s*\(", text, re.M)))


def test_library_exists_and_loads():
    assert os.path.exists(_lib.LIB_PATH), "build with python pm3-rs_b200/build.py"
    _lib.load()


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(_lib.EXPORTS) == names


def test_default_options_mirror_pm3options():  # scf.rs:259-287
    lib = _lib.load()
    o = _lib.Options()
    lib.pm3gpu_default_options(ctypes.byref(o))
    assert (o.max_scf, o.e_tol, o.p_tol, o.use_diis, o.accelerator, o.adiis_switch) == (200, 1e-8, 1e-7, 1, 2, 0.1)
    assert (o.reference, o.guess, o.stability, o.scf_memory_mb) == (0, 0, 1, 512)


def test_supported_elements_and_basis_size():
    lib = _lib.load()
    for zz in (1, 3, 4, 5, 6, 7, 8, 9, 11, 12, 13, 14, 15, 16, 17):
        assert lib.pm3gpu_supported_element(zz) == 1
    for zz in (0, 2, 10, 18, 35, 53, 64):
        assert lib.pm3gpu_supported_element(zz) == 0
    z = np.array([8, 1, 1, 6], dtype=np.int32)
    nao = ctypes.c_int()
    assert lib.pm3gpu_result_sizes(4, z.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(nao)) == 10
    bad = np.array([8, 35], dtype=np.int32)
    assert lib.pm3gpu_result_sizes(2, bad.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(nao)) == -1


def test_struct_layouts_match_header():
    assert ctypes.sizeof(_lib.Options) == 8 + 4 + 4 + 8 + 8 + 4 + 4 + 8 + 4 * 4 + 8 + 8 + 4 + 4 + 4 + 4
    assert _lib.Options.scf_memory_mb.offset == 80 and _lib.Options.variant.offset == 84
    assert _lib.Options.mmok.offset == 88
    # pm3gpu_result: 4 ints, 4 doubles, 3+1 doubles, 2 doubles, 2 ints, 4 ints, 1 double, 1 double
    assert ctypes.sizeof(_lib.Result) == 16 + 32 + 32 + 16 + 8 + 16 + 16


def test_unsupported_method_and_field_raise_before_any_gpu_work():
    with pytest.raises(ValueError):
        native.single_point([8, 1, 1], np.zeros((3, 3)), method="am1")
    with pytest.raises(ValueError):
        native.single_point([8, 1, 1], np.zeros((3, 3)), field=[0.0, 0.0, 0.01])
    with pytest.raises(ValueError):
        native.single_point([8, 1, 1], np.zeros((3, 3)), reference="rohf")
    with pytest.raises(ValueError):
        native.single_point([8, 1, 1], np.zeros((2, 3)))


def test_tuning_file_is_checked_without_a_device(tmp_path):
    """pm3gpu_load_tuning with no context only parses the file (host code, no CUDA call)."""
    lib = _lib.load()
    good = tmp_path / "tuning.json"
    good.write_text('{\n  "device": "B200",\n  "sms": 148,\n  "batch": [\n'
                    '    {"nmax_le": 256, "ctas_per_sm": 1, "ms_1cta": 900.0, "ms_2cta": 950.0}\n  ],\n'
                    '  "large": [\n    {"n_le": 512, "coop": 1, "ms_coop": 1.0, "ms_multi": 2.0}\n  ]\n}\n')
    assert lib.pm3gpu_load_tuning(None, str(good).encode()) == _lib.OK
    bad = tmp_path / "bad.json"
    bad.write_text('{"large": [{"n_le": 512, "coop": 2}]}')
    assert lib.pm3gpu_load_tuning(None, str(bad).encode()) == _lib.INVALID_INPUT
    empty = tmp_path / "empty.json"
    empty.write_text('{"batch": [], "large": []}')
    assert lib.pm3gpu_load_tuning(None, str(empty).encode()) == _lib.INVALID_INPUT
    assert lib.pm3gpu_load_tuning(None, str(tmp_path / "missing.json").encode()) == _lib.INVALID_INPUT
    assert lib.pm3gpu_tuning_choice(None, 0, 100) == -1


def test_entry_points_without_coefficients_raise_loudly():
    """orbitals / molden need MO coefficients, which the library does not export: a ValueError
    that says so, before any GPU work."""
    for fn in (native.orbitals, native.molden):
        with pytest.raises(ValueError, match="MO coefficients"):
            fn([8, 1, 1], np.zeros((3, 3)))
