"""The C ABI: the library loads, exports every entry point include/xplus_b200.h declares,
and fails loudly (no CPU fallback) when no GPU is present."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from project_xplus_b200 import _lib

HEADER = Path(__file__).resolve().parent.parent / "include" / "xplus_b200.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s+\**([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                       text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) > 20
    for name in names:
        assert hasattr(_lib.lib, name), name
    # and the binding covers them all
    assert set(names) <= set(_lib.EXPORTED)


def test_exports_nothing_else():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert exported == set(declared_functions())


def test_library_is_built_for_sm100a():
    import subprocess
    out = subprocess.run(["cuobjdump", "--list-elf", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_no_gpu_fails_loudly():
    import project_xplus_b200 as xp
    if xp.device_count() > 0:
        pytest.skip("a GPU is present")
    from project_xplus_b200 import generators as g
    d, _ = g.fem2d(4)
    with pytest.raises(xp.XplusError) as e:
        xp.PcgSolver.from_dataset(d)
    assert e.value.code == _lib.XPLUS_ERR_CUDA
    assert "no CUDA device" in str(e.value)


def test_opts_default_and_version():
    o = _lib.default_opts()
    assert o.slice_height == 32 and o.sigma == 256 and o.keep_fp64 == 1
    assert b"sm_100a" in _lib.lib.xplus_version()


def test_argument_errors():
    import project_xplus_b200 as xp
    with pytest.raises(xp.XplusError) as e:
        xp.CsrDataset.load("/nonexistent-dir-xyz")
    assert e.value.code == _lib.XPLUS_ERR_IO
    h = C.c_void_p()
    rc = _lib.lib.xplus_pcg_create(None, None, None, 4, None, C.byref(h))
    assert rc == _lib.XPLUS_ERR_ARG


def test_batch_entry_points_reject_a_null_handle():
    """The batched solver's setters and queries check the handle before any CUDA call."""
    for rc in (_lib.lib.xplus_batch_set_resident(None, 1),
               _lib.lib.xplus_batch_set_stage_matrix(None, 1),
               _lib.lib.xplus_batch_staged_info(None, None, None, None),
               _lib.lib.xplus_batch_resident_info(None, None, None, None),
               _lib.lib.xplus_batch_split_info(None, None, None, None, None)):
        assert rc == _lib.XPLUS_ERR_ARG
