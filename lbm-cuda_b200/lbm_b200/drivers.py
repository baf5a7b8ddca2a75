"""Headless versions of the reference's three driver scripts.

Each reference driver (lbm_mine2.py, lbm_smemaa_main.py,
lbm_smemaa_endfused_main.py) builds the same initial state, loads a solid mask,
captures ONE CUDA graph of two kernel launches (f_now -> f_out -> f_now) on a
non-blocking stream, and then loops over display frames: `iters_per_frame`
graph replays, the macro kernel (end-fused driver only), the vorticity colour
map into an OpenGL pixel buffer, and an FPS / MLUPS print every few frames.

Here the same loop runs without a window: the kernels are this library's
drop-ins reached through :class:`lbm_b200.RefCompatModule` (the one-line swap a
driver makes), the graph is a ``torch.cuda.CUDAGraph`` captured on a side
stream, and the colour map goes into an RGBA8 device buffer that can be read
back or written as a PNG.  MLUPS is counted the reference's way: every cell,
W * H * iters_per_frame * (steps per graph) * fps (lbm_mine2.py:106,
lbm_smemaa_main.py:202, lbm_smemaa_endfused_main.py:112), with the frame time
taken on the host clock around synchronised frames as the drivers do, and also
on the device with CUDA events.

    python -m lbm_b200.drivers --kind smemaa --frames 30 --png frame.png

`circle.bmp`, the drivers' mask image, is not part of the reference tree; the
default mask is a procedural cylinder in the channel (an image with the
drivers' rule, green == 0 -> solid, can be given instead).
"""
from __future__ import annotations

import struct
import time
import zlib
from dataclasses import dataclass

import numpy as np

from . import init as I


@dataclass(frozen=True)
class DriverConfig:
    """Constants of one reference driver."""

    kind: str  # RefCompatModule family
    T: int  # physical steps per kernel launch
    tau_inv: float
    u_in: float
    iters_per_frame: int  # graph replays per displayed frame
    stats_frames: int  # frames between two FPS / MLUPS prints
    macro_per_frame: bool  # macro_kernel before the colour map (the end-fused kernel writes no u, v, rho)
    sync_before_vis: bool  # the driver synchronises its stream before drawing
    tau_inv_bnd: float | None = None  # third rate argument of the core4 kernel


DRIVERS = {
    # lbm_mine2.py:74-81 (graph), :90-98 (frame loop), :102-106 (statistics, MLUPS)
    "core4": DriverConfig("core4", 1, 1.8, 0.10, 25, 10, False, False, 1.8),
    # lbm_smemaa_main.py:95 (T), :107-108 (rates), :137-144 (graph), :165 (iters), :195-204 (statistics)
    "smemaa": DriverConfig("smemaa", 4, 1.7, 0.10, 50, 10, False, True),
    # lbm_smemaa_endfused_main.py:61 (T), :67-68 (rates), :75-80 (graph), :89 (iters), :108-113 (statistics);
    # that driver compiles lbm_core_smemaa_policy.cu, "endfused" and "policy" differ only in the name
    "endfused": DriverConfig("endfused", 6, 1.0, 0.10, 20, 30, True, True),
}
DRIVERS["policy"] = DriverConfig("policy", 6, 1.0, 0.10, 20, 30, True, True)

VORT_SCALE = 50.0  # colour-map scale every driver passes (lbm_mine2.py:95)


def reference_initial_state(W: int, H: int) -> np.ndarray:
    """The drivers' populations: equilibrium of rho = 1, u_y = 0 and
    u_x = 0.1 (G(150, 150) - G(300, 150)), sigma 10 (lbm_mine2.py:15-36)."""
    ux = I.gaussian_pair_ux(W, H)
    return I.equilibrium(np.ones((H, W)), ux, np.zeros((H, W)), dtype=np.float32)


def default_mask(W: int, H: int) -> np.ndarray:
    """Channel (solid top and bottom rows, open ends) with a cylinder of diameter
    H / 8 at (W / 4, H / 2), 0 / 1 bytes like the drivers' bool mask."""
    return I.cylinder_mask(W, H, W / 4.0, H / 2.0, H / 8.0, value=I.SOLID)


def mlups_reference(W: int, H: int, iters_per_frame: int, steps_per_graph: int, fps: float) -> float:
    """The drivers' MLUPS: every cell, iters_per_frame graphs of steps_per_graph steps per frame."""
    return W * H * iters_per_frame * steps_per_graph * fps / 1e6


def write_png(path: str, rgba: np.ndarray) -> None:
    """RGBA8 image (H, W, 4) as an 8-bit truecolour-with-alpha PNG, row 0 at the
    bottom as the drivers' pixel buffer is drawn (OpenGL's origin)."""
    rgba = np.ascontiguousarray(np.asarray(rgba, dtype=np.uint8)[::-1])
    h, w = rgba.shape[:2]
    raw = b"".join(b"\x00" + rgba[y].tobytes() for y in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as fh:
        fh.write(b"\x89PNG\r\n\x1a\n")
        fh.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)))
        fh.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        fh.write(chunk(b"IEND", b""))


def read_png(path: str) -> np.ndarray:
    """Inverse of :func:`write_png` (8-bit RGBA, filter type 0 rows only)."""
    data = open(path, "rb").read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG file")
    pos, idat, w, h = 8, b"", 0, 0
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            if depth != 8 or ctype != 6:
                raise ValueError("only 8-bit RGBA PNGs are read")
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), dtype=np.uint8).reshape(h, 1 + 4 * w)
    if np.any(raw[:, 0] != 0):
        raise ValueError("filtered PNG rows are not supported")
    return raw[:, 1:].reshape(h, w, 4)[::-1].copy()


class HeadlessDriver:
    """One reference driver's frame loop on this library, without a window.

    ``kind``: "core4" (lbm_mine2.py), "smemaa" (lbm_smemaa_main.py), "endfused"
    or "policy" (lbm_smemaa_endfused_main.py with either T = 6 source).  ``mask``
    (H, W) bytes or ``image`` (a mask image, green == 0 -> solid) replace the
    default cylinder; ``iters_per_frame`` overrides the driver's constant.
    """

    def __init__(self, kind: str = "core4", W: int = 2048, H: int = 512, mask=None, image: str | None = None,
                 iters_per_frame: int | None = None, f0=None, use_graph: bool = True):
        import torch

        from . import RefCompatModule

        if kind not in DRIVERS:
            raise ValueError(f"unknown driver {kind!r}; one of {sorted(DRIVERS)}")
        self.cfg = DRIVERS[kind]
        self.W, self.H = int(W), int(H)
        self.iters_per_frame = int(iters_per_frame or self.cfg.iters_per_frame)
        self.steps_per_graph = 2 * self.cfg.T
        if mask is None:
            mask = I.mask_from_image(image, W, H) if image else default_mask(W, H)
        dev = "cuda"
        self.mask = torch.as_tensor(np.asarray(mask, dtype=np.uint8)).to(dev).contiguous()
        f0 = reference_initial_state(W, H) if f0 is None else np.asarray(f0, dtype=np.float32)
        self.f_now = torch.from_numpy(np.ascontiguousarray(f0)).to(dev)
        # f_out starts as a copy of f_now.  The T = 4 / 6 drivers allocate it
        # uninitialised (cp.empty_like, lbm_smemaa_main.py:44,
        # lbm_smemaa_endfused_main.py:33) and the AA kernels never write some of
        # its slots (solid cells, the outlet corners), which then keep whatever
        # the allocation held; a copy makes every run reproducible (lbm_mine2.py:36
        # copies too).
        self.f_out = self.f_now.clone()
        # the drivers pass their initial u, v, rho arrays as the kernels' macro outputs
        self.ux = torch.zeros((H, W), dtype=torch.float32, device=dev)
        self.uy = torch.zeros_like(self.ux)
        self.rho = torch.ones_like(self.ux)
        self.image = torch.zeros((H, W, 4), dtype=torch.uint8, device=dev)
        self.module = RefCompatModule(self.cfg.kind)
        self._lbm = self.module.get_function("fused_lbmkernel")
        self._vis = self.module.get_function("visualizekernel")
        self._macro = self.module.get_function("macro_kernel") if self.cfg.macro_per_frame else None
        self.stream = torch.cuda.Stream()  # the drivers' non-blocking stream
        self.graph = None
        self.frames_done = 0
        if use_graph:
            self._capture()

    # ---- the kernels, with the drivers' argument tuples ----
    def _args(self, src, dst):
        c, W, H = self.cfg, np.int32(self.W), np.int32(self.H)
        if c.kind == "core4":
            return (self.mask, src, dst, self.ux, self.uy, self.rho, W, H, np.float32(c.tau_inv),
                    np.float32(c.u_in), np.float32(c.tau_inv_bnd))
        if c.kind == "smemaa":
            return (self.mask, src, dst, self.ux, self.uy, self.rho, W, H, np.float32(c.tau_inv), np.float32(c.u_in))
        return (self.mask, src, dst, W, H, np.float32(c.tau_inv), np.float32(c.u_in))

    def _pair(self, a, b):
        """The graph's body: a -> b -> a (2 launches, 2 T steps)."""
        grid, block = (1, 1), (1, 1)  # ignored by the shim; the library picks its own launch shape
        self._lbm(grid, block, self._args(a, b))
        self._lbm(grid, block, self._args(b, a))

    def _capture(self):
        import torch

        # first calls set up per-device state (tensor-map entry point, side
        # streams); make them outside the capture, on scratch copies
        a, b = self.f_now.clone(), self.f_now.clone()
        with torch.cuda.stream(self.stream):
            self._pair(a, b)
        self.stream.synchronize()
        del a, b
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream):
            self._pair(self.f_now, self.f_out)
        self.graph = g

    def step_graph(self):
        """One replay of the captured pair (or the same two launches eagerly)."""
        import torch

        with torch.cuda.stream(self.stream):
            if self.graph is not None:
                self.graph.replay()
            else:
                self._pair(self.f_now, self.f_out)

    def frame(self):
        """iters_per_frame replays, then (end-fused) macro, then the colour map."""
        import torch

        for _ in range(self.iters_per_frame):
            self.step_graph()
        if self.cfg.sync_before_vis:
            self.stream.synchronize()
        c, W, H = self.cfg, np.int32(self.W), np.int32(self.H)
        with torch.cuda.stream(self.stream):
            if self._macro is not None:
                self._macro((1, 1), (1, 1), (self.f_now, self.ux, self.uy, self.rho, self.mask, W, H,
                                             np.float32(c.u_in)))
            self._vis((1, 1), (1, 1), (self.ux, self.uy, self.rho, self.image, self.mask, W, H,
                                       np.float32(VORT_SCALE)))
        self.frames_done += 1

    def run(self, frames: int, print_every: int | None = None, out=None) -> dict:
        """Runs `frames` frames; returns FPS and MLUPS (host clock, as the drivers
        measure, and CUDA-event device time) with the drivers' accounting."""
        import torch

        every = print_every or self.cfg.stats_frames
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(self.stream)
        t0 = last = time.time()
        count = 0
        for i in range(frames):
            self.frame()
            count += 1
            if out is not None and count >= every:
                torch.cuda.synchronize()
                now = time.time()
                fps = count / (now - last)
                mlups = mlups_reference(self.W, self.H, self.iters_per_frame, self.steps_per_graph, fps)
                out.write(f"\r[LBM Simulation] FPS: {fps:.1f} | MLUPS: {mlups:.2f}")
                last, count = now, 0
        e1.record(self.stream)
        torch.cuda.synchronize()
        wall = time.time() - t0
        dev_ms = e0.elapsed_time(e1)
        fps = frames / wall
        return {
            "frames": frames,
            "fps": fps,
            "mlups": mlups_reference(self.W, self.H, self.iters_per_frame, self.steps_per_graph, fps),
            "mlups_device": mlups_reference(self.W, self.H, self.iters_per_frame, self.steps_per_graph,
                                            frames / (dev_ms * 1e-3)),
            "physical_steps": frames * self.iters_per_frame * self.steps_per_graph,
        }

    def image_host(self) -> np.ndarray:
        import torch

        torch.cuda.synchronize()
        return self.image.cpu().numpy()

    def save_png(self, path: str) -> None:
        write_png(path, self.image_host())


def main(argv=None):
    import argparse
    import json
    import sys

    ap = argparse.ArgumentParser(description="headless reference driver on lbm_b200")
    ap.add_argument("--kind", choices=sorted(DRIVERS), default="core4")
    ap.add_argument("--W", type=int, default=2048)
    ap.add_argument("--H", type=int, default=512)
    ap.add_argument("--frames", type=int, default=60)
    ap.add_argument("--iters-per-frame", type=int, default=None)
    ap.add_argument("--image", default=None, help="mask image (green == 0 -> solid)")
    ap.add_argument("--png", default=None, help="write the last frame here")
    args = ap.parse_args(argv)
    d = HeadlessDriver(args.kind, args.W, args.H, image=args.image, iters_per_frame=args.iters_per_frame)
    res = d.run(args.frames, out=sys.stdout)
    print()
    if args.png:
        d.save_png(args.png)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
