"""Which stream the Python drop-ins launch on when the caller names none (CPU,
with a fake cupy module and a fake initialised torch): cupy arrays take cupy's
current stream even in a process where torch is initialised, so a reference
driver capturing a CUDA graph on a cupy stream (lbm_mine2.py:75-81) captures
these launches; torch tensors take torch's current stream."""
import ctypes as C
import sys
import types

import pytest

import lbm_b200 as L

CUPY_STREAM, TORCH_STREAM = 0x1111, 0x2222


class _FakeCupyArray:
    def __init__(self, ptr):
        self.data = types.SimpleNamespace(ptr=ptr)


class _FakeTorchTensor:
    def data_ptr(self):
        return 0x5000


@pytest.fixture
def both_libraries(monkeypatch):
    fake = types.ModuleType("cupy")
    fake.cuda = types.SimpleNamespace(get_current_stream=lambda: types.SimpleNamespace(ptr=CUPY_STREAM))
    monkeypatch.setitem(sys.modules, "cupy", fake)
    import torch

    monkeypatch.setattr(torch.cuda, "is_available", lambda: True)
    monkeypatch.setattr(torch.cuda, "is_initialized", lambda: True)
    monkeypatch.setattr(torch.cuda, "current_stream", lambda: types.SimpleNamespace(cuda_stream=TORCH_STREAM))


def test_cupy_arrays_use_cupys_stream(both_libraries):
    assert L._stream(None, _FakeCupyArray(0x4000)).value == CUPY_STREAM
    assert L._stream(None, None, _FakeCupyArray(0x4000)).value == CUPY_STREAM


def test_torch_tensors_use_torchs_stream(both_libraries):
    assert L._stream(None, _FakeTorchTensor()).value == TORCH_STREAM


def test_no_arrays_prefers_initialised_torch(both_libraries):
    assert L._stream(None).value == TORCH_STREAM


def test_explicit_stream_wins(both_libraries):
    assert L._stream(0x3333, _FakeCupyArray(0x4000)).value == 0x3333
    assert L._stream(types.SimpleNamespace(ptr=0x4444), _FakeTorchTensor()).value == 0x4444


def test_dropin_wrapper_passes_the_cupy_stream(both_libraries, monkeypatch):
    seen = {}

    def fake_call(name, *args):
        seen[name] = args
        return 0

    monkeypatch.setattr(L, "call", fake_call)
    arrs = [_FakeCupyArray(0x4000 + 0x100 * i) for i in range(6)]
    L.core4_step(*arrs, 64, 32, 1.8, 0.1)
    assert seen["lbm_core4_step"][-1].value == CUPY_STREAM
    L.smemaa_step(*arrs, 64, 32, 1.7, 0.1, T=4)
    assert seen["lbm_smemaa_step"][-1].value == CUPY_STREAM
    L.blocked_step(arrs[0], arrs[1], arrs[2], 64, 32, 1.7, 0.1, T=6)
    assert seen["lbm_blocked_step"][-1].value == CUPY_STREAM
    assert isinstance(seen["lbm_blocked_step"][-1], C.c_void_p)
