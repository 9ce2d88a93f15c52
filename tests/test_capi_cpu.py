"""CPU: the C-ABI library loads, exports every symbol include/ope.h declares,
and refuses to compute without a device (no CPU fallback).  One GPU test:
the library runs as sm_100a code on the device."""
import os

import numpy as np
import pytest

from conftest import HAS_GPU, ROOT


def test_header_symbols_are_exported(ope):
    from ope_b200 import _lib

    declared = _lib.declared_symbols(os.path.join(ROOT, "include", "ope.h"))
    assert len(declared) >= 15
    L = _lib.load()
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing


def test_python_signatures_cover_header(ope):
    from ope_b200 import _lib

    declared = set(_lib.declared_symbols(os.path.join(ROOT, "include", "ope.h")))
    assert declared <= set(_lib._SIGS), declared - set(_lib._SIGS)


def test_record_layouts_match_header():
    from ope_b200.api import RESULT_DTYPE
    from ope_b200.workloads import CONTRACT_DTYPE

    assert CONTRACT_DTYPE.itemsize == 56 and RESULT_DTYPE.itemsize == 64
    assert list(CONTRACT_DTYPE.names) == ["spot", "strike", "expiry", "rate", "div_yield", "vol", "opt_type", "pad"]


def test_tune_structs_match_header(tmp_path):
    """ope_launch_shape / ope_tune_entry: the ctypes mirrors have the header's
    sizes and field offsets (compiled with the host C compiler)."""
    import ctypes
    import subprocess

    from ope_b200 import _lib

    fields = {"ope_launch_shape": ["warps_per_block", "deepest_first", "occupancy", "per_unit", "reserved"],
              "ope_tune_entry": ["max_contracts", "shape", "ms_default", "ms_tuned"]}
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "ope.h"', "int main(void) {"]
    for st, fs in fields.items():
        src.append(f'printf("%zu\\n", sizeof({st}));')
        src += [f'printf("%zu\\n", offsetof({st}, {f}));' for f in fs]
    src.append("return 0; }")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = []
    for mirror, fs in ((_lib.LaunchShape, fields["ope_launch_shape"]), (_lib.TuneEntry, fields["ope_tune_entry"])):
        want.append(ctypes.sizeof(mirror))
        want += [getattr(mirror, f).offset for f in fs]
    assert got == want


@pytest.mark.gpu
def test_library_runs_on_sm100a(ope):
    """The library carries sm_100a code only: on the device it reports compute
    capability 10.0 and its pricing kernel launches and prices."""
    sms, major, minor = ope.device_info()
    assert (major, minor) == (10, 0) and sms > 0
    launches = ope.kernel_launch_count()
    assert ope.heston_price(100.0, 100.0, 1.0, 0.03, 0.0, [0.04, 2.0, 0.04, 0.3, -0.7]) > 0.0
    assert ope.kernel_launch_count() == launches + 1


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_no_device_fails_loudly(ope):
    with pytest.raises(ope.OpeError) as e:
        ope.heston_price(100.0, 100.0, 1.0, 0.03, 0.0, [0.04, 2.0, 0.04, 0.3, -0.7])
    assert e.value.status == 4  # OPE_ERR_NO_DEVICE


def test_empty_batch_needs_no_device(ope):
    assert ope.batch_heston(np.zeros(0, ope.api.CONTRACT_DTYPE), [0.04, 2.0, 0.04, 0.3, -0.7]).size == 0


def test_api_rejects_wrong_param_shapes(ope):
    with pytest.raises(ValueError):
        ope.batch_bates(np.zeros(1, ope.api.CONTRACT_DTYPE), [0.04, 2.0, 0.04, 0.3, -0.7])
    with pytest.raises(ValueError):
        ope.price_surfaces(ope.MODEL_HESTON, np.zeros(2, ope.api.CONTRACT_DTYPE), [0, 1, 2],
                           [[0.04, 2.0, 0.04, 0.3, -0.7]])


def test_workspace_limit_needs_no_device(ope):
    ope.set_workspace_limit(1 << 20)
    ope.set_workspace_limit(0)
    assert ope.workspace_bytes() == 0
