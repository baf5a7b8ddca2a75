"""Argument checking of the C ABI, on the CPU: every call below is refused
before the library touches the GPU, with LBM_ERR_ARG (invalid argument) or
LBM_ERR_UNSUPPORTED (a valid request this build does not implement).  The
pointers are dummy non-NULL addresses that are never dereferenced."""
import ctypes as C

import pytest

from lbm_b200 import _lib
from lbm_b200 import solver as SV

ERR_ARG, ERR_UNSUPPORTED = 1001, 1002
P = C.c_void_p(4096)  # a dummy device address, never dereferenced on these paths
P2 = C.c_void_p(8192)


@pytest.fixture(scope="module")
def lib():
    return _lib.lib()


def test_reference_dropins_refuse_bad_arguments(lib):
    nul = C.c_void_p(0)
    # lbm_core4_step: NULL buffers, aliasing source and destination, tiny domains, rates
    assert lib.lbm_core4_step(nul, P, P2, P, P, P, 64, 32, 1.8, 0.1, 1.8, None) == ERR_ARG
    assert lib.lbm_core4_step(P, P, P, P, P, P, 64, 32, 1.8, 0.1, 1.8, None) == ERR_ARG
    assert lib.lbm_core4_step(P, P, P2, P, P, P, 2, 32, 1.8, 0.1, 1.8, None) == ERR_ARG
    assert lib.lbm_core4_step(P, P, P2, P, P, P, 64, 32, 0.0, 0.1, 1.8, None) == ERR_ARG
    # lbm_core4_run: T outside 1..8, negative step count
    res = C.c_int(0)
    for T in (0, 9):
        assert lib.lbm_core4_run(P, P, P2, P, P, P, 64, 32, 1.8, 0.1, 4, T, None, C.byref(res)) == ERR_ARG
    assert lib.lbm_core4_run(P, P, P2, P, P, P, 64, 32, 1.8, 0.1, -1, 2, None, C.byref(res)) == ERR_ARG
    # the AA drop-ins: even T in 2..8 only (the reference's static_assert, lbm_core_smemaa.cu:17)
    for T in (1, 3, 10):
        assert lib.lbm_smemaa_step(P, P, P2, P, P, P, 64, 32, 1.7, 0.1, T, None) == ERR_UNSUPPORTED
        assert lib.lbm_blocked_step(P, P, P2, 64, 32, 1.0, 0.1, T, None) == ERR_UNSUPPORTED
    assert lib.lbm_smemaa_step(P, P, P, P, P, P, 64, 32, 1.7, 0.1, 4, None) == ERR_ARG
    assert lib.lbm_blocked_step(nul, P, P2, 64, 32, 1.0, 0.1, 6, None) == ERR_ARG
    # the colour map needs a 4-byte aligned image
    assert lib.lbm_visualize(P, P, P, C.c_void_p(4097), P, 64, 32, 50.0, None) == ERR_ARG
    assert lib.lbm_macro(nul, P, P, P, P, 64, 32, 0.1, None) == ERR_ARG


def _create(**kw):
    W = kw.pop("W", 64)
    p = SV.default_params(W, 32, **kw)
    h = C.c_void_p(0)
    return _lib.lib().lbm_create(C.byref(p), C.byref(h)), h


@pytest.mark.parametrize("kw,status", [
    (dict(W=2), ERR_ARG),
    (dict(s_nu=2.0), ERR_ARG),
    (dict(s_nu=0.0), ERR_ARG),
    (dict(storage=7), ERR_ARG),
    (dict(storage=4), ERR_ARG),
    (dict(storage=SV.STORE_F64, closure=SV.CLOSURE_MLP, ref_clamps=0, mlp=4096), ERR_UNSUPPORTED),
    (dict(collision=5), ERR_ARG),
    (dict(bc_left=SV.BC_PERIODIC), ERR_ARG),  # periodic on one side only
    (dict(bc_right=SV.BC_ZOUHE), ERR_ARG),  # no inlet on the right
    (dict(closure=SV.CLOSURE_MLP, ref_clamps=0), ERR_ARG),  # the network's weights are missing
    (dict(closure=SV.CLOSURE_MLP, ref_clamps=0, mlp=4097), ERR_ARG),  # unaligned weights
    (dict(closure=SV.CLOSURE_NONE, ref_clamps=0, u_lid=0.1, storage=SV.STORE_F16DEV), ERR_UNSUPPORTED),
    (dict(closure=9), ERR_UNSUPPORTED),
])
def test_create_refuses_bad_parameters(kw, status):
    rc, h = _create(**kw)
    assert rc == status
    assert not h.value


def test_solver_calls_refuse_bad_arguments(lib):
    nul = C.c_void_p(0)
    res = C.c_int(0)
    assert lib.lbm_run(nul, P, P2, P, 4, 2, None, None, None, None, C.byref(res)) == ERR_ARG
    assert lib.lbm_run_inplace(nul, P, P, 4, None, None, None, None) == ERR_ARG
    assert lib.lbm_diag_fp64(nul, P, P, P, None) == ERR_ARG
    assert lib.lbm_forces_fp64(nul, P, P, P, None) == ERR_ARG
    assert lib.lbm_destroy(nul) == ERR_ARG
    assert lib.lbm_convert_state(64, 32, P, 9, P2, 0, None) == ERR_ARG
    assert lib.lbm_periodic_halo_x(P, 64, 32, 0, 0, None) == ERR_ARG  # no halo
    assert lib.lbm_periodic_halo_x(P, 10, 32, 4, 0, None) == ERR_ARG  # narrower than three halos
    assert lib.lbm_periodic_halo_x(P, 64, 32, 2, 5, None) == ERR_ARG  # unknown storage
    # the learned-closure training calls
    assert lib.lbm_mlp_forward(nul, P, P, 10, None) == ERR_ARG
    assert lib.lbm_mlp_grad(P, P, P, nul, 0, P, P, P, C.c_size_t(1 << 20), None) == ERR_ARG
    assert lib.lbm_mlp_grad(P, P, P, nul, 100, P, P, P, C.c_size_t(4), None) == ERR_ARG  # workspace too small
    assert lib.lbm_mlp_pack(P, P, 1.0, C.c_void_p(4100), None) == ERR_ARG  # unaligned destination
    assert lib.lbm_mlp_pack(P, P, 0.0, P, None) == ERR_ARG
    # the activation-aware training and packing calls: unknown activation
    assert lib.lbm_mlp_forward_act(P, 2, P, P, 10, None) == ERR_ARG
    assert lib.lbm_mlp_grad_act(P, -1, P, P, nul, 10, P, P, P, C.c_size_t(1 << 20), None) == ERR_ARG
    assert lib.lbm_mlp_pack_act(P, 7, P, 1.0, P, None) == ERR_ARG
    # column-restricted launches: no handle, aliasing buffers, odd / empty / out-of-range columns
    assert lib.lbm_run_columns(nul, P, P2, P, 2, 0, 64, None) == ERR_ARG
    assert lib.lbm_run_columns(nul, P, P, P, 2, 0, 64, None) == ERR_ARG
    # halo pack / unpack: no side, columns beyond the width, unknown storage, no buffer
    assert lib.lbm_halo_pack(P, 64, 32, 0, -1, -1, 4, P2, None) == ERR_ARG
    assert lib.lbm_halo_pack(P, 64, 32, 0, 62, -1, 4, P2, None) == ERR_ARG
    assert lib.lbm_halo_pack(P, 64, 32, 9, 0, 60, 4, P2, None) == ERR_ARG
    assert lib.lbm_halo_unpack(P, 64, 32, 0, 0, 60, 4, nul, None) == ERR_ARG
    assert lib.lbm_halo_unpack(P, 64, 32, 0, 0, 60, 0, P2, None) == ERR_ARG
    # batch tile configuration without a batch
    rows = (C.c_int * 3)(16, 16, 16)
    t = C.c_int(0)
    assert lib.lbm_batch_get_tiles(nul, C.byref(t), rows) == ERR_ARG
    assert lib.lbm_batch_set_tiles(nul, 2, rows) == ERR_ARG
    # the wait self-test: limit outside 1 .. 2^31, arrive not 0 / 1
    assert lib.lbm_selftest_wait_timeout(0, 0, None, None) == ERR_ARG
    assert lib.lbm_selftest_wait_timeout((1 << 31) + 1, 0, None, None) == ERR_ARG
    assert lib.lbm_selftest_wait_timeout(1000, 2, None, None) == ERR_ARG


def test_batch_create_refuses_unsupported_physics(lib):
    from lbm_b200.batch import Domain

    arr = (Domain * 1)()
    arr[0].W, arr[0].H = 64, 32
    h = C.c_void_p(0)
    p = SV.default_params(1, 1, closure=SV.CLOSURE_NONE, ref_clamps=0)
    assert lib.lbm_batch_create(C.byref(p), arr, 1, C.byref(h)) == ERR_UNSUPPORTED
    p = SV.default_params(1, 1)
    assert lib.lbm_batch_create(C.byref(p), arr, 0, C.byref(h)) == ERR_ARG
    assert lib.lbm_batch_create(None, arr, 1, C.byref(h)) == ERR_ARG
