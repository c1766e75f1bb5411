"""The C-ABI library loads and exports every symbol include/psdm_rtm.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "psdm_rtm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(psdm_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_expected(engine_lib):
    from psdm_b200 import _lib
    assert sorted(_lib.EXPORTS) == header_functions()


def test_library_exports_every_header_symbol(engine_lib):
    for name in header_functions():
        assert hasattr(engine_lib, name), name


def test_no_gpu_fails_loudly(engine_lib):
    """Without a usable GPU, engine creation must fail (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from psdm_b200._lib import PsdmError
    from psdm_b200.rtm import Engine
    with pytest.raises(PsdmError) as ei:
        Engine(0)
    assert ei.value.code == -2
