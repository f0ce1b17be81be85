"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, the ctypes mirrors match the C struct layouts, and the entry
points fail closed (no CPU fallback) when no device is present."""

import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "b200fe.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(b200fe_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_exported_list(libmod):
    assert declared_functions() == sorted(libmod.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol(libmod):
    lib = libmod.load()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_struct_layouts_match_header(libmod, tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include "b200fe.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(void){printf("%zu %zu %zu %zu\\n", sizeof(b200fe_options),'
                   ' sizeof(b200fe_result), offsetof(b200fe_result, abs_residual),'
                   ' offsetof(b200fe_result, kernel_launches));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert int(out[0]) == ctypes.sizeof(libmod.Options)
    assert int(out[1]) == ctypes.sizeof(libmod.Result)
    assert int(out[2]) == libmod.Result.abs_residual.offset
    assert int(out[3]) == libmod.Result.kernel_launches.offset


def test_default_options(libmod):
    o = libmod.default_options()
    assert o.tol == 1e-8 and o.precision == libmod.PREC_MIXED and o.certify == 1
    assert o.tolerance_mode == 1 and o.max_iter > 0


def _has_gpu(libmod):
    return bool(libmod.load().b200fe_device_available())


def test_fail_closed_without_device(libmod, pkg):
    if _has_gpu(libmod):
        pytest.skip("a CUDA device is present")
    with pytest.raises(pkg.AbsorberError) as e:
        pkg.Absorber(0)
    assert e.value.status == libmod.UNAVAILABLE
    # the raw entry point reports unavailability and leaves its inputs untouched
    y = np.arange(6, dtype=np.float64)
    y0 = y.copy()
    with pytest.raises(pkg.AbsorberError):
        pkg.demean_raw(y, None, [np.array([0, 0, 1, 1, 2, 2], np.int32)], [3])
    assert np.array_equal(y, y0)


def test_null_arguments_rejected(libmod):
    lib = libmod.load()
    o = libmod.default_options()
    r = libmod.Result()
    # null context: invalid argument, never a crash
    rc = lib.b200fe_absorb(None, None, None, 10, 0, 1, None, None, None, ctypes.byref(o),
                           None, None, ctypes.byref(r))
    assert rc == libmod.INVALID_ARG
    rc = lib.b200fe_fe_recovery_max_delta(None, None, 10, 1, None, None, None, None, None)
    assert rc == libmod.INVALID_ARG
