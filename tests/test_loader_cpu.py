"""CPU: the bindings refuse to run without the native library (there is no
CPU fallback), and a context cannot be created without a CUDA device."""
import pytest

import fastgrid_b200 as fg


def test_missing_library_raises(monkeypatch):
    monkeypatch.setattr(fg, "_lib", None)
    monkeypatch.setattr(fg, "LIB_PATH", "/nonexistent/libfastgrid_b200.so")
    with pytest.raises(fg.AgError, match="no CPU fallback"):
        fg.lib()


def test_context_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(fg.AgError, match="no CUDA device"):
        fg.Context(0)
