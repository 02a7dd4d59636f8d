"""The C-ABI library: loads, exports every symbol include/parahpop.h
declares, and fails loudly (status 1 + message) without a CUDA device."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from parahpop_b200 import api

HEADER = Path(__file__).resolve().parents[1] / "include" / "parahpop.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(phop_\w+|paraHPOP_\w+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("paraHPOP_run", "paraHPOP_setLogLevel", "phop_create", "phop_propagate", "phop_destroy",
                 "phop_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = api.library()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_null_context_calls_fail_cleanly():
    lib = api.library()
    z = np.zeros(6)
    D = api._dp
    assert lib.phop_propagate(None, 1, D(z), D(z), D(z), D(z), D(z), D(z), D(z), None, None, D(z), D(z)) == 1
    assert lib.phop_propagate_device(None, 1, None, 0.0, D(z), D(z), D(z), D(z), D(z), 1.0, 1.0, D(z)) == 1
    assert lib.phop_set_option(None, b"lanes", 4.0) == 1
    assert lib.phop_last_stats(None, None) == 1
    out = C.c_void_p()
    assert lib.phop_server_create(None, 16, 20.0, C.byref(out)) == 1
    rid = C.c_int64()
    assert lib.phop_server_submit(None, 1, D(z), D(z), D(z), D(z), D(z), D(z), D(z), None, None, C.byref(rid)) == 1
    assert lib.phop_server_step(None, None) == 1
    assert lib.phop_server_take(None, 1, D(z), D(z), D(z), D(z)) == 1
    assert lib.phop_server_get_stats(None, None) == 1
    f = lib.phop_propagate_device_noalloc
    f.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double,
                  C.POINTER(C.c_double)]
    assert f(None, 1, None, None, None, 0.0, 1.0, 1.0, None) == 1


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device failure path")
def test_create_without_device_fails_loudly(golden):
    case = golden("full_600s")
    with pytest.raises(api.PhopError, match="No usable CUDA device"):
        api.Propagator(case.config_path)


def test_create_reports_config_errors(tmp_path):
    bad = tmp_path / "c.json"
    bad.write_text('{"run": {"duration_seconds": 60}, "execution": {"integration": '
                   '{"initialStepSize": 60, "maxNumSteps": 10}}, "model": {}, "extra": 1}')
    with pytest.raises(api.PhopError, match="Unsupported configuration option: extra"):
        api.Propagator(bad)
