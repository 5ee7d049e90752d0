"""The C ABI library loads on a machine without a GPU, exports every symbol
the header declares, and the ctypes mirror matches the C structs."""
import ctypes as C
import os
import re

import pytest

import mdff_b200
from mdff_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "mdff_engine.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mdff_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = mdff_b200.lib()
    names = header_functions()
    assert len(names) >= 12
    for name in names:
        assert hasattr(L, name), name


def test_struct_sizes_match():
    L = mdff_b200.lib()
    L.mdff_struct_size.restype = C.c_int
    assert L.mdff_struct_size(0) == C.sizeof(abi.Params)
    assert L.mdff_struct_size(1) == C.sizeof(abi.Energies)
    assert L.mdff_struct_size(2) == C.sizeof(abi.Thermo)
    assert L.mdff_struct_size(3) == C.sizeof(abi.ParamGrad)
    assert L.mdff_struct_size(4) == C.sizeof(abi.OptResult)
    assert L.mdff_struct_size(5) == C.sizeof(abi.EfgDistParams)
    assert L.mdff_struct_size(6) == C.sizeof(abi.FrameHeader)
    assert L.mdff_struct_size(7) == C.sizeof(abi.RmcParams)
    assert L.mdff_struct_size(8) == C.sizeof(abi.RmcResult)
    assert L.mdff_struct_size(9) == C.sizeof(abi.RmcEfgParams)


def test_defaults_match_library():
    a = abi.default_params()
    b = mdff_b200.params_default()
    assert bytes(a) == bytes(b)


def test_create_rejects_bad_parameters_without_gpu():
    p = abi.default_params()
    p.ntype = 0
    with pytest.raises(mdff_b200.EngineError) as e:
        mdff_b200.Engine(p, [1], [[0, 0, 0]], [[10, 0, 0], [0, 10, 0], [0, 0, 10]])
    assert e.value.code == abi.E_ARG


def test_error_codes_match_header():
    src = open(os.path.join(ROOT, "include", "mdff_engine.h")).read()
    for name in ("OK", "E_ARG", "E_CUDA", "E_NOCONV", "E_LISTOVF", "E_NONFINITE", "E_STATE", "E_UNSUPPORTED", "E_NOMEM"):
        m = re.search(r"#define MDFF_%s\s+(-?\d+)" % name, src)
        assert int(m.group(1)) == getattr(abi, name), name


def test_batch_rejects_unsupported_models_without_gpu():
    from mdff_b200 import systems
    confs = systems.mgo_batch(nconf=2, nmin=120, nmax=140, seed=1)
    p = systems.mgo_params(6.0, 0.5, 6)
    p.lnmlj = 1
    with pytest.raises(mdff_b200.EngineError) as e:
        mdff_b200.Batch(p, confs)
    assert e.value.code == abi.E_UNSUPPORTED
    p = systems.mgo_params(6.0, 0.5, 6)
    p.ntype = 3
    with pytest.raises(mdff_b200.EngineError) as e:
        mdff_b200.Batch(p, confs)
    assert e.value.code == abi.E_UNSUPPORTED
