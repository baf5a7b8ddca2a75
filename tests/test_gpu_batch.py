"""GPU tests of the batched persistent launch (lbm_batch_*): every domain of a
batch of uneven sizes must evolve exactly as when run on its own, against the
single-domain solver and the general-solver oracle."""
import numpy as np
import pytest
import torch

import oracle as O
from helpers import REL_TOL, dev, host, rel_l2
from lbm_b200 import init as I
from lbm_b200 import solver as SV
from lbm_b200.batch import Batch

pytestmark = pytest.mark.gpu

SIZES = [(70, 48), (130, 66), (256, 96), (100, 100), (64, 200), (300, 64)]
PHYS = dict(cs_smag=0.1, s_nu=1.9)


def _domains(storage=SV.STORE_F32, pitch16=False):
    tdt = {SV.STORE_F32: torch.float32, SV.STORE_F16DEV: torch.float16}[storage]
    doms, hosts = [], []
    for i, (W, H) in enumerate(SIZES):
        m = I.random_discs_mask(W, H, 1 + i % 4, 3.0, 6.0, 100 + i)
        f0 = I.perturbed_state(W, H, 200 + i, amp=0.02)
        u_in = 0.02 + 0.01 * i
        pitch = ((W + 15) // 16) * 16 if pitch16 else W
        fa = torch.zeros((9, H, pitch), dtype=tdt, device="cuda")
        mk = torch.zeros((H, pitch), dtype=torch.uint8, device="cuda")
        mk[:, :W] = dev(m)
        src = dev(f0)
        if storage == SV.STORE_F32:
            fa[:, :, :W] = src
        else:
            tmp = torch.empty((9, H, W), dtype=tdt, device="cuda")
            SV.convert_state(src, SV.STORE_F32, tmp, storage)
            fa[:, :, :W] = tmp
        fb = fa.clone()
        doms.append(dict(W=W, H=H, pitch=pitch if pitch16 else 0, mask_pitch=pitch if pitch16 else 0,
                         f_a=fa, f_b=fb, mask=mk, u_in=u_in))
        hosts.append((m, f0, u_in))
    return doms, hosts


@pytest.mark.parametrize("pitch16", [False, True])
@pytest.mark.parametrize("T", [1, 2, 4, 8])
def test_batch_matches_oracle(T, pitch16):
    doms, hosts = _domains(pitch16=pitch16)
    B = Batch(doms, storage=SV.STORE_F32, **PHYS)
    n = 2 * T + 1
    which = B.run(n, T)
    for d, (m, f0, u_in) in zip(doms, hosts):
        W = d["W"]
        out = host((d["f_b"] if which else d["f_a"])[:, :, :W].contiguous())
        G = O.General(W, d["H"], collision="mrt", closure="smag", cs=0.1, s_nu=1.9, u_in=u_in)
        ref, _ = G.run(m, f0, n)
        assert rel_l2(out, ref) < REL_TOL


@pytest.mark.parametrize("storage", [SV.STORE_F32, SV.STORE_F16DEV])
def test_batch_equals_separate_launches_and_graph_replay(storage):
    doms1, _ = _domains(storage, pitch16=True)
    doms2, _ = _domains(storage, pitch16=True)
    B1 = Batch(doms1, storage=storage, **PHYS)
    B2 = Batch(doms2, storage=storage, **PHYS)
    w1 = B1.run(16, 4)  # two graph-replayed launch pairs
    w2 = B2.run_separate(16, 4)
    assert w1 == w2
    for d1, d2 in zip(doms1, doms2):
        a = host((d1["f_b"] if w1 else d1["f_a"]).float())
        b = host((d2["f_b"] if w2 else d2["f_a"]).float())
        if storage != SV.STORE_F32:  # compare populations, not the stored deviations
            a = a + I.WEIGHTS[:, None, None].astype(np.float32)
            b = b + I.WEIGHTS[:, None, None].astype(np.float32)
        # same arithmetic, separately compiled kernels: a few ulps of the storage
        # format (an FP16 deviation ulp is ~5e-6 of a population)
        assert rel_l2(a, b) < (1e-6 if storage == SV.STORE_F32 else REL_TOL)


def test_autotune_then_run():
    doms, hosts = _domains(pitch16=True)
    B = Batch(doms, storage=SV.STORE_F32, **PHYS)
    T, chunk = B.autotune()
    assert T in (1, 2, 4, 8) and chunk >= 2 * T
    which = B.run(8, 0)
    assert which in (0, 1)
    for d in doms:
        assert torch.isfinite((d["f_b"] if which else d["f_a"])).all()


CLASS_SIZES = [(70, 48), (256, 96), (512, 320), (1024, 640)]  # size classes 0, 0, 1, 2


def _class_domains(aligned, seed):
    doms = []
    for i, (W, H) in enumerate(CLASS_SIZES):
        m = I.random_discs_mask(W, H, 2, 3.0, 8.0, seed + i)
        pitch = ((W + 15) // 16) * 16 if aligned else W
        fa = torch.zeros((9, H, pitch), device="cuda")
        fa[:, :, :W] = dev(I.perturbed_state(W, H, seed + 50 + i, amp=0.02))
        mk = torch.zeros((H, pitch), dtype=torch.uint8, device="cuda")
        mk[:, :W] = dev(m)
        doms.append(dict(W=W, H=H, pitch=pitch if aligned else 0, mask_pitch=pitch if aligned else 0, f_a=fa,
                         f_b=fa.clone(), mask=mk, u_in=0.03 + 0.01 * i))
    return doms


@pytest.mark.parametrize("aligned,T,cfgs", [
    (True, 2, ([16, 16, 16], [8, 24, 32], [32, 8, 16])),       # register wavefront items
    (False, 4, ([64, 64, 64], [16, 32, 128], [128, 16, 64])),  # shared-memory wavefront items
])
def test_per_class_tile_rows_give_the_same_states(aligned, T, cfgs):
    """The rows per work item of each size class only change how the domains are
    cut into items: the register-wavefront engine gives the same states bit for
    bit; the shared-memory engine's cells near an item boundary can round
    differently (a few ulps)."""
    outs = []
    for rows in cfgs:
        doms = _class_domains(aligned, 300)
        B = Batch(doms, storage=SV.STORE_F32, **PHYS)
        B.set_tiles(T, rows)
        assert B.tiles() == (T, list(rows))
        which = B.run(6 * T, 0)
        outs.append([host((d["f_b"] if which else d["f_a"])[:, :, :d["W"]].contiguous()) for d in doms])
        B.close()
    for other in outs[1:]:
        for a, b in zip(outs[0], other):
            if aligned:
                assert np.array_equal(a, b)
            else:
                assert rel_l2(a, b) < 1e-6


def test_autotune_per_class_rows_and_validation():
    doms = _class_domains(True, 400)
    B = Batch(doms, storage=SV.STORE_F32, **PHYS)
    T, chunk = B.autotune()
    T2, rows = B.tiles()
    assert T2 == T and len(rows) == 3 and rows[2] == chunk
    assert all(8 <= r and r >= 2 * T for r in rows)
    with pytest.raises(Exception):
        B.set_tiles(2, [4, 16, 16])  # below the smallest item height
    with pytest.raises(Exception):
        B.set_tiles(3, [16, 16, 16])  # depth not built for batches
    which = B.run(2 * T, 0)
    for d in doms:
        assert torch.isfinite(d["f_b"] if which else d["f_a"]).all()
