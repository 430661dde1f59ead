"""The C-ABI library loads and exports every symbol include/sbletkf.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

from sbpom_letkf_v2_b200 import _abi
from sbpom_letkf_v2_b200.params import CParams, LETKFParams

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "sbletkf.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sbletkf_[a-z_0-9]+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(_abi.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.sbletkf_abi_version() == 1


def test_params_struct_layout():
    # 20 int32 then 18 doubles, no padding holes
    assert ctypes.sizeof(CParams) == 20 * 4 + 18 * 8
    assert CParams.cov_infl_mul.offset == 80


def test_invalid_params_rejected_before_device_use():
    lib = _abi.load()
    bad = LETKFParams(nmem=1).to_c()
    ws = ctypes.c_void_p()
    assert lib.sbletkf_workspace_create(ctypes.byref(bad), 10, 10, 0, ctypes.byref(ws)) == _abi.ERR_ARG
    p = LETKFParams(nmem=8)
    c = p.to_c()
    c.iswitch_da = 7
    assert lib.sbletkf_workspace_create(ctypes.byref(c), 10, 10, 0, ctypes.byref(ws)) == _abi.ERR_ARG
    assert lib.sbletkf_analysis(None, ctypes.byref(p.to_c()), None, None, None, None, None, 0, None, None, None,
                                None) == _abi.ERR_ARG


def test_params_validation_messages():
    with pytest.raises(ValueError, match="iswitch_da"):
        LETKFParams(iswitch_da=4).validate()
    with pytest.raises(ValueError, match="RM"):
        LETKFParams(rm=5).validate()
    p = LETKFParams(sigma_obs=200e3)
    assert abs(p.dist_zero - 2 * (10 / 3) ** 0.5 * 200e3) < 1e-6
    q = p.replace(sigma_obs=100e3)
    assert abs(q.dist_zero - 2 * (10 / 3) ** 0.5 * 100e3) < 1e-6
