"""CPU tests of the C ABI boundary: the library loads and exports every symbol
declared in include/*.h; calls that touch no device behave without a GPU."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names.update(re.findall(r"FLB_API\s+[\w\s\*]+?\b(flb_\w+)\s*\(", src))
    return sorted(names)


def test_header_declares_symbols():
    names = declared_symbols()
    assert "flb_create" in names and "flb_step" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    from freelb_b200 import _capi
    lib = _capi.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_python_signatures_cover_header():
    from freelb_b200 import _capi
    missing = [n for n in declared_symbols() if n not in _capi.SIGNATURES]
    assert not missing, missing


def test_version_and_default_desc_without_gpu():
    import freelb_b200
    from freelb_b200 import _capi
    abi, arch = freelb_b200.version()
    assert abi == 1 and arch == 100
    d = freelb_b200.make_desc(12, 12, 12, 0.53)
    assert abs(d.omega - 1 / 0.53) < 1e-15
    assert list(d.task_keys[:3]) == [2, 4, 8]
    assert list(d.task_ops[:3]) == [_capi.OP_BULK, _capi.OP_BOUNCEBACK, _capi.OP_MOVINGWALL]


@pytest.mark.parametrize("field,value", [("nx", 2), ("omega", 2.5), ("ntasks", 9),
                                         ("storage", 7), ("model", 5)])
def test_create_rejects_bad_descriptors(field, value):
    """Validation happens before any device call, so it is testable without a GPU."""
    import freelb_b200
    from freelb_b200 import _capi
    d = freelb_b200.make_desc(12, 12, 12, 0.53)
    setattr(d, field, value)
    h = ctypes.c_void_p()
    rc = _capi.load().flb_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == -1
    assert h.value is None
    assert _capi.load().flb_last_error()


def test_null_arguments_are_errors_not_crashes():
    from freelb_b200 import _capi
    lib = _capi.load()
    assert lib.flb_step(None, 1, None) == -1
    assert lib.flb_destroy(None) == 0
    assert lib.flb_create(None, None) == -1
