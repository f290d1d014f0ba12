"""The C ABI library: it loads, exports every symbol include/nkr_b200.h
declares, reports its name, and refuses to compute without a GPU (no CPU
fallback)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def _declared():
    txt = open(os.path.join(ROOT, "include", "nkr_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(nkr_b200_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    import nkr_b200 as nk
    names = _declared()
    assert len(names) > 20
    lib = nk.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_backend_name():
    import nkr_b200 as nk
    assert nk.backend_name() == "b200"


def test_library_built_for_sm100a():
    import nkr_b200 as nk
    # the sm_100a cubin is embedded in the library (names only, no code inspection)
    data = open(nk.LIB_PATH, "rb").read()
    assert b"sm_100a" in data


def test_no_cpu_fallback_without_gpu():
    import nkr_b200 as nk
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(nk.B200Error) as e:
        nk.Context(0)
    assert e.value.status in (nk.ENODEV, nk.ECUDA)


def test_invalid_generator_arguments():
    import nkr_b200 as nk
    with pytest.raises(nk.B200Error):
        nk.generate("nonexistent", 4)
    with pytest.raises(nk.B200Error):
        nk.generate("sql-aggregate", 3)  # not a power of two
    with pytest.raises(nk.B200Error):
        nk.generate("fibonacci", 1)
