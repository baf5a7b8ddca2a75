"""Checkpoint / resume format (lbm_b200.checkpoint): raw SoA planes + JSON header."""
import json

import numpy as np
import pytest
import torch

from lbm_b200 import checkpoint as CK
from lbm_b200 import solver as SV


@pytest.mark.parametrize("storage,dt", [(0, torch.float32), (1, torch.float16), (2, torch.bfloat16),
                                        (3, torch.float64)])
def test_round_trip_bitwise(tmp_path, storage, dt):
    W, H = 37, 11
    g = torch.Generator().manual_seed(storage)
    f = (torch.rand((9, H, W), generator=g) * 0.1).to(dt)
    m = (torch.rand((H, W), generator=g) > 0.8).to(torch.uint8)
    p = SV.default_params(W, H, storage=storage, s_nu=1.7, cs_smag=0.13)
    path = str(tmp_path / "ck")
    hdr = CK.save(path, f, m, storage=storage, step=1234, params=p, extra={"note": "test"})
    assert hdr["step"] == 1234
    f2, m2, h2 = CK.load(path, device="cpu")
    assert f2.dtype == dt and torch.equal(f2.view(torch.uint8), f.view(torch.uint8)) if storage else torch.equal(f2, f)
    assert torch.equal(m2, m)
    assert h2["extra"] == {"note": "test"}
    q = CK.params_from_header(h2)
    assert (q.W, q.H, q.storage) == (W, H, storage) and abs(q.cs_smag - 0.13) < 1e-7 and abs(q.s_nu - 1.7) < 1e-6
    # the binary file is the device layout f[q*W*H + y*W + x], little-endian
    raw = np.fromfile(path + ".f", dtype={0: "<f4", 3: "<f8"}.get(storage, "<u2"))
    assert raw.size == 9 * W * H
    # no device pointer in the header, and no weights file without the closure
    assert "mlp" not in h2["params"] and "mlp" not in h2["sha256"]
    assert CK.load_mlp(path, device="cpu") is None


def test_learned_closure_run_saves_its_weights_not_a_pointer(tmp_path):
    W, H = 16, 8
    f = torch.rand((9, H, W))
    m = torch.zeros((H, W), dtype=torch.uint8)
    p = SV.default_params(W, H, closure=SV.CLOSURE_MLP, ref_clamps=0, mlp=0xDEAD0000)
    path = str(tmp_path / "ck")
    with pytest.raises(ValueError, match="packed weights"):
        CK.save(path, f, m, params=p)
    with pytest.raises(ValueError, match="4096"):
        CK.save(path, f, m, params=p, mlp_packed=torch.zeros(100, dtype=torch.uint8))
    packed = torch.randint(0, 256, (CK.MLP_PACKED_BYTES,), dtype=torch.uint8)
    hdr = CK.save(path, f, m, params=p, mlp_packed=packed)
    assert "mlp" not in hdr["params"] and "mlp" in hdr["sha256"]
    assert "mlp" not in json.load(open(path + ".json"))["params"]
    got = CK.load_mlp(path, device="cpu")
    assert torch.equal(got, packed)
    _, _, h2 = CK.load(path, device="cpu")
    with pytest.raises(ValueError, match="load_mlp"):
        CK.params_from_header(h2)
    q = CK.params_from_header(h2, mlp=got)
    assert q.closure == SV.CLOSURE_MLP and q.mlp == got.data_ptr()
    with open(path + ".mlp", "r+b") as fh:
        fh.write(b"\x00\x01")
    with pytest.raises(ValueError, match="checksum"):
        CK.load_mlp(path, device="cpu")


def test_corruption_and_format_checks(tmp_path):
    W, H = 8, 4
    f = torch.zeros((9, H, W))
    m = torch.zeros((H, W), dtype=torch.uint8)
    path = str(tmp_path / "ck")
    CK.save(path, f, m)
    with open(path + ".f", "r+b") as fh:
        fh.seek(5)
        fh.write(b"\x01")
    with pytest.raises(ValueError, match="checksum"):
        CK.load(path, device="cpu")
    CK.load(path, device="cpu", verify=False)
    hdr = json.load(open(path + ".json"))
    hdr["version"] = 99
    json.dump(hdr, open(path + ".json", "w"))
    with pytest.raises(ValueError, match="header"):
        CK.load(path, device="cpu")
    with pytest.raises(ValueError, match="dtype"):
        CK.save(path, f.half(), m, storage=0)
