"""The C-ABI library loads and exports every symbol include/pastix_gpu.h
declares (no GPU needed); the entry points reject bad arguments without a
device (the product path has no CPU fallback)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "pastix_gpu.h")).read()
    return sorted(set(re.findall(r"PASTIX_GPU_API\s+\w+\s+(pastix_gpu_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    d = _declared()
    assert "pastix_gpu_numfact" in d and "pastix_gpu_solve" in d and len(d) >= 15


def test_library_exports_every_declared_symbol():
    from pastix_b200 import gpu
    L = gpu.load()
    for name in _declared():
        assert hasattr(L, name), name


def test_python_binding_lists_exports():
    from pastix_b200 import gpu
    for name in gpu.EXPORTS:
        assert name in _declared()


def test_init_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from pastix_b200 import gpu
    with pytest.raises(gpu.PastixGpuError):
        gpu.Solver()
