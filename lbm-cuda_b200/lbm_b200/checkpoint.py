"""Checkpoint / resume: the population state as raw SoA planes plus a JSON header.

Layout on disk, for a checkpoint named `<path>`:
  <path>.json   header: format, version, W, H, storage (0 FP32, 1 FP16 of f - w,
                2 BF16 of f - w, 3 FP64), element type, byte order, step, the
                solver parameters (every lbm_params field except the `mlp`
                device pointer, which means nothing in another process) and
                whatever the caller adds under "extra", and the SHA-256 of each
                binary file;
  <path>.f      9 planes of H x W elements, q-major then row-major (the device
                layout f[q*W*H + y*W + x]), little-endian;
  <path>.mask   H x W bytes (the mask the state was advanced with);
  <path>.mlp    only for a run with the learned closure: the packed BF16
                inference block (LBM_MLP_PACKED_BYTES bytes from lbm_mlp_pack).
A state saved from one storage format reloads into the same format; the
header's parameters rebuild the solver (`params_from_header`), and a
learned-closure run gets its weights back from `<path>.mlp` (`load_mlp`).
"""
from __future__ import annotations

import hashlib
import json
import os

FORMAT = "lbm-b200-checkpoint"
VERSION = 1
MLP_PACKED_BYTES = 4096  # LBM_MLP_PACKED_BYTES
CLOSURE_MLPS = (2, 3)    # LBM_CLOSURE_MLP, LBM_CLOSURE_MLP_SILU
_DTYPES = {0: ("float32", 4), 1: ("float16", 2), 2: ("bfloat16", 2), 3: ("float64", 8)}
_NP = {4: "<f4", 2: "<i2", 8: "<f8"}


def _sha(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as fh:
        for block in iter(lambda: fh.read(1 << 22), b""):
            h.update(block)
    return h.hexdigest()


def _params_dict(params) -> dict:
    if params is None:
        return {}
    return {name: getattr(params, name) for name, _ in params._fields_ if name != "mlp"}


def _torch_dtype(storage: int):
    import torch

    return {0: torch.float32, 1: torch.float16, 2: torch.bfloat16, 3: torch.float64}[int(storage)]


def save(path: str, f, mask, storage: int = 0, step: int = 0, params=None, extra: dict | None = None,
         mlp_packed=None) -> dict:
    """Writes the state f (torch tensor (9, H, W), any device) and its mask.

    A run with the learned closure (LBM_CLOSURE_MLP or _MLP_SILU) must pass
    its packed inference block as `mlp_packed` (the uint8 tensor of
    LBM_MLP_PACKED_BYTES that params.mlp points to, e.g. ``Mlp.packed()``); it is
    written to `<path>.mlp`, since the pointer itself cannot be resumed."""
    import torch

    _, H, W = f.shape
    name, esize = _DTYPES[int(storage)]
    expect = _torch_dtype(storage)
    if f.dtype != expect:
        raise ValueError(f"state dtype {f.dtype} does not match storage {storage} ({expect})")
    uses_mlp = params is not None and int(getattr(params, "closure", 0)) in CLOSURE_MLPS
    if uses_mlp and mlp_packed is None:
        raise ValueError("a learned-closure run needs its packed weights: pass mlp_packed=<the lbm_mlp_pack block>")
    if mlp_packed is not None and mlp_packed.numel() * mlp_packed.element_size() != MLP_PACKED_BYTES:
        raise ValueError(f"mlp_packed must hold {MLP_PACKED_BYTES} bytes")
    fc = f.detach().contiguous().cpu()
    raw = fc.view(torch.int16).numpy() if esize == 2 else fc.numpy()
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    with open(path + ".f", "wb") as fh:
        fh.write(raw.astype(raw.dtype.newbyteorder("<"), copy=False).tobytes())
    with open(path + ".mask", "wb") as fh:
        fh.write(mask.detach().contiguous().cpu().numpy().astype("uint8").tobytes())
    sha = {"f": _sha(path + ".f"), "mask": _sha(path + ".mask")}
    if mlp_packed is not None:
        with open(path + ".mlp", "wb") as fh:
            fh.write(mlp_packed.detach().contiguous().view(torch.uint8).cpu().numpy().tobytes())
        sha["mlp"] = _sha(path + ".mlp")
    hdr = {"format": FORMAT, "version": VERSION, "W": int(W), "H": int(H), "planes": 9, "storage": int(storage),
           "element": name, "byteorder": "little", "layout": "f[q*W*H + y*W + x]", "step": int(step),
           "params": _params_dict(params), "extra": extra or {}, "sha256": sha}
    tmp = path + ".json.tmp"
    with open(tmp, "w") as fh:
        json.dump(hdr, fh, indent=1)
    os.replace(tmp, path + ".json")  # the header appears only once the data is complete
    return hdr


def _header(path: str) -> dict:
    with open(path + ".json") as fh:
        hdr = json.load(fh)
    if hdr.get("format") != FORMAT or hdr.get("version") != VERSION:
        raise ValueError(f"{path}.json is not a version-{VERSION} {FORMAT} header")
    return hdr


def load(path: str, device="cuda", verify: bool = True):
    """Returns (f, mask, header); f and mask are torch tensors on `device`."""
    import numpy as np
    import torch

    hdr = _header(path)
    if verify:
        for key, ext in (("f", ".f"), ("mask", ".mask")):
            if _sha(path + ext) != hdr["sha256"][key]:
                raise ValueError(f"{path}{ext} does not match the checksum in its header")
    W, H, storage = hdr["W"], hdr["H"], hdr["storage"]
    name, esize = _DTYPES[storage]
    n = 9 * W * H
    buf = np.fromfile(path + ".f", dtype=_NP[esize])
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


def load_mlp(path: str, device="cuda", verify: bool = True):
    """The packed learned-closure block saved with a checkpoint (a uint8 tensor of
    LBM_MLP_PACKED_BYTES on `device`, 16-byte aligned as lbm_create requires), or
    None when the run had no learned closure."""
    import numpy as np
    import torch

    hdr = _header(path)
    want = hdr["sha256"].get("mlp")
    if want is None:
        return None
    if verify and _sha(path + ".mlp") != want:
        raise ValueError(f"{path}.mlp does not match the checksum in its header")
    raw = np.fromfile(path + ".mlp", dtype=np.uint8)
    if raw.size != MLP_PACKED_BYTES:
        raise ValueError(f"{path}.mlp holds {raw.size} bytes, expected {MLP_PACKED_BYTES}")
    return torch.from_numpy(raw.copy()).to(device)


def params_from_header(hdr, mlp=None):
    """lbm_params of the saved run (solver.Params).  For a learned-closure run,
    `mlp` is the packed block on the device (``load_mlp(path)``); the caller keeps
    that tensor alive while the solver uses it."""
    from .solver import default_params

    p = dict(hdr.get("params") or {})
    p.pop("mlp", None)  # headers never carry a usable pointer
    W, H = p.pop("W", hdr["W"]), p.pop("H", hdr["H"])
    if int(p.get("closure", 0)) in CLOSURE_MLPS:
        if mlp is None:
            raise ValueError("the saved run uses the learned closure: pass mlp=load_mlp(path)")
        p["mlp"] = mlp.data_ptr()
    return default_params(W, H, **p)
