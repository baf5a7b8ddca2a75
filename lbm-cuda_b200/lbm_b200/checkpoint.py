"""Checkpoint / resume: the population state as raw SoA planes plus a JSON header.

Layout on disk, for a checkpoint named `<path>`:
  <path>.json   header: format, version, W, H, storage (0 FP32, 1 FP16 of f - w,
                2 BF16 of f - w), element type, byte order, step, the solver
                parameters and whatever the caller adds under "extra", and the
                SHA-256 of both binary files;
  <path>.f      9 planes of H x W elements, q-major then row-major (the device
                layout f[q*W*H + y*W + x]), little-endian;
  <path>.mask   H x W bytes (the mask the state was advanced with).
A state saved from one storage format reloads into the same format; the
header's parameters rebuild the solver (`params_from_header`).
"""
from __future__ import annotations

import hashlib
import json
import os

FORMAT = "lbm-b200-checkpoint"
VERSION = 1
_DTYPES = {0: ("float32", 4), 1: ("float16", 2), 2: ("bfloat16", 2)}


def _sha(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as fh:
        for block in iter(lambda: fh.read(1 << 22), b""):
            h.update(block)
    return h.hexdigest()


def _params_dict(params) -> dict:
    if params is None:
        return {}
    return {name: getattr(params, name) for name, _ in params._fields_}


def save(path: str, f, mask, storage: int = 0, step: int = 0, params=None, extra: dict | None = None) -> dict:
    """Writes the state f (torch tensor (9, H, W), any device) and its mask."""
    import torch

    _, H, W = f.shape
    name, esize = _DTYPES[int(storage)]
    expect = {0: torch.float32, 1: torch.float16, 2: torch.bfloat16}[int(storage)]
    if f.dtype != expect:
        raise ValueError(f"state dtype {f.dtype} does not match storage {storage} ({expect})")
    fc = f.detach().contiguous().cpu()
    raw = fc.view(torch.int16).numpy() if esize == 2 else fc.numpy()
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    with open(path + ".f", "wb") as fh:
        fh.write(raw.astype(raw.dtype.newbyteorder("<"), copy=False).tobytes())
    with open(path + ".mask", "wb") as fh:
        fh.write(mask.detach().contiguous().cpu().numpy().astype("uint8").tobytes())
    hdr = {"format": FORMAT, "version": VERSION, "W": int(W), "H": int(H), "planes": 9, "storage": int(storage),
           "element": name, "byteorder": "little", "layout": "f[q*W*H + y*W + x]", "step": int(step),
           "params": _params_dict(params), "extra": extra or {},
           "sha256": {"f": _sha(path + ".f"), "mask": _sha(path + ".mask")}}
    tmp = path + ".json.tmp"
    with open(tmp, "w") as fh:
        json.dump(hdr, fh, indent=1)
    os.replace(tmp, path + ".json")  # the header appears only once the data is complete
    return hdr


def load(path: str, device="cuda", verify: bool = True):
    """Returns (f, mask, header); f and mask are torch tensors on `device`."""
    import numpy as np
    import torch

    with open(path + ".json") as fh:
        hdr = json.load(fh)
    if hdr.get("format") != FORMAT or hdr.get("version") != VERSION:
        raise ValueError(f"{path}.json is not a version-{VERSION} {FORMAT} header")
    if verify:
        for key, ext in (("f", ".f"), ("mask", ".mask")):
            if _sha(path + ext) != hdr["sha256"][key]:
                raise ValueError(f"{path}{ext} does not match the checksum in its header")
    W, H, storage = hdr["W"], hdr["H"], hdr["storage"]
    name, esize = _DTYPES[storage]
    n = 9 * W * H
    buf = np.fromfile(path + ".f", dtype="<f4" if esize == 4 else "<i2")
    if buf.size != n:
        raise ValueError(f"{path}.f holds {buf.size} elements, the header says {n}")
    t = torch.from_numpy(buf.astype(buf.dtype.newbyteorder("="), copy=False).copy())
    if esize == 2:
        t = t.view({1: torch.float16, 2: torch.bfloat16}[storage])
    f = t.view(9, H, W).to(device)
    m = np.fromfile(path + ".mask", dtype=np.uint8)
    if m.size != W * H:
        raise ValueError(f"{path}.mask holds {m.size} bytes, the header says {W * H}")
    mask = torch.from_numpy(m.copy()).view(H, W).to(device)
    return f, mask, hdr


def params_from_header(hdr):
    """lbm_params of the saved run (solver.Params)."""
    from .solver import default_params

    p = dict(hdr.get("params") or {})
    W, H = p.pop("W", hdr["W"]), p.pop("H", hdr["H"])
    return default_params(W, H, **p)
