"""The C ABI library without a GPU: it loads, exports what the header
declares, and rejects invalid arguments before touching the device."""
import ctypes
import os
import re

import numpy as np
import pytest

from tomocam_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tomocam_b200.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tc_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_functions():
    names = header_functions()
    assert "tc_mbir_solve" in names and "tc_radon" in names and len(names) >= 18


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    for name in header_functions():
        assert hasattr(lib, name), f"{name} declared in the header but not exported"


def test_ctypes_prototypes_cover_header():
    assert set(header_functions()) == set(_lib.PROTOTYPES)


def test_exported_symbols_are_c_linkage():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r" T (tc_[a-z0-9_]+)$", out, flags=re.M))
    assert set(header_functions()) <= exported


def test_version_and_defaults_without_gpu():
    lib = _lib.lib()
    assert lib.tc_version().decode().startswith("tomocam-b200")
    o = _lib.MbirOpts()
    lib.tc_mbir_opts_default(ctypes.byref(o))
    assert o.num_iters == 100 and abs(o.p - 1.2) < 1e-7 and o.use_graph == 1
    assert abs(o.sigma - 100.0) < 1e-5 and o.prior_weight == 1.0


def test_argument_errors_without_gpu():
    lib = _lib.lib()
    assert lib.tc_plan_create(None, None) == _lib.TC_ERR_ARG
    assert b"NULL" in lib.tc_last_error_string()
    h = ctypes.c_void_p()
    ang = np.zeros(4, np.float32)
    g = _lib.Geom(2, 4, ang.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 0.0, 0, 0)
    assert lib.tc_plan_create(ctypes.byref(g), ctypes.byref(h)) == _lib.TC_ERR_SHAPE
    g = _lib.Geom(16, 4, None, 0.0, 0, 0)
    assert lib.tc_plan_create(ctypes.byref(g), ctypes.byref(h)) == _lib.TC_ERR_ARG
    g = _lib.Geom(16, 4, ang.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 0.0, 0, 16)
    assert lib.tc_plan_create(ctypes.byref(g), ctypes.byref(h)) == _lib.TC_ERR_ARG
    bad = np.array([0.0, np.inf, 0.0, 0.0], np.float32)
    g = _lib.Geom(16, 4, bad.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 0.0, 0, 0)
    assert lib.tc_plan_create(ctypes.byref(g), ctypes.byref(h)) == _lib.TC_ERR_NAN
    assert lib.tc_radon(None, None, None, 1, None) == _lib.TC_ERR_ARG
    assert lib.tc_fft_c2c(None, None, 1, 8, 0, None) == _lib.TC_ERR_ARG
    assert lib.tc_fft_c2c(None, None, 0, 8, -1, None) == _lib.TC_OK
    assert lib.tc_qggmrf_grad(None, None, 0, 4, 4, 1.0, 1.2, 1.0, None) == _lib.TC_OK
    assert lib.tc_mbir_solve(None, None, 0.0, None, 1, None, None, None) == _lib.TC_ERR_ARG
    assert lib.tc_plan_destroy(None) == _lib.TC_OK


def test_errors_raise_typed_exception():
    with pytest.raises(_lib.TomocamError) as e:
        _lib.call("tc_plan_create", None, None)
    assert e.value.code == _lib.TC_ERR_ARG


def test_python_api_validation_without_gpu():
    import tomocam_b200 as tomocam
    from tomocam_b200 import modeling
    s = np.zeros((1, 4, 8), np.float32)
    a = np.zeros(4, np.float32)
    with pytest.raises(ValueError):
        tomocam.MBIR(s, a, 4.0, 1, smoothness=0.0)
    with pytest.raises(ValueError):
        modeling.update_total_variation(s, s, smoothness=-1.0)
    with pytest.raises(ValueError):
        tomocam.radon(np.zeros((2, 2)), np.zeros(2))


def test_reference_import_name():
    """`import tomocam` gives the reference package's names (tomocam/__init__.py:4-7)."""
    import tomocam
    import tomocam.gradients
    import tomocam.modeling
    import tomocam.recon
    import tomocam.transform
    from tomocam import cTomocam
    import tomocam_b200
    assert tomocam.MBIR is tomocam_b200.modeling.MBIR
    assert tomocam.radon is tomocam_b200.transform.radon
    assert tomocam.radon_adj is tomocam_b200.transform.radon_adj
    assert tomocam.recon.MBIR is tomocam_b200.modeling.MBIR
    assert callable(tomocam.modeling.calc_gradients) and callable(tomocam.modeling.update_total_variation)
    assert callable(tomocam.gradients.gradients)
    for name in ("radon", "backproject", "mbir", "set_num_of_gpus", "radon_adj", "gradients",
                 "total_variation"):
        assert hasattr(cTomocam, name), name


def test_ingest_argument_errors_without_gpu():
    lib = _lib.lib()
    h = np.zeros((3, 4, 5), np.float32)
    hp = h.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    assert lib.tc_sino_ingest_psd(None, 3, 4, 5, 0, 4, None) == _lib.TC_ERR_ARG
    assert lib.tc_sino_ingest_psd(hp, 3, 4, 5, 0, 4, None) == _lib.TC_ERR_ARG
    assert lib.tc_sino_ingest_psd(hp, 0, 4, 5, 0, 4, 1) == _lib.TC_ERR_SHAPE
    assert lib.tc_sino_ingest_psd(hp, 3, 4, 5, 2, 3, 1) == _lib.TC_ERR_SHAPE
    assert lib.tc_sino_ingest_psd(hp, 3, 4, 5, -1, 1, 1) == _lib.TC_ERR_SHAPE
    assert lib.tc_sino_ingest_psd(hp, 3, 4, 5, 4, 0, None) == _lib.TC_OK


def test_ingest_python_validation_without_gpu():
    from tomocam_b200.ingest import sinogram_from_psd
    a = np.zeros((3, 4, 5), np.float32)
    with pytest.raises(ValueError):
        sinogram_from_psd(a[0])
    with pytest.raises(ValueError):
        sinogram_from_psd(a, 3, 2)
    with pytest.raises(ValueError):
        sinogram_from_psd(a, -1)
