"""GPU pieces of the overlapped x-slab exchange, on one GPU:

* lbm_run_columns: launches restricted to column ranges that tile the domain
  give the full launch bit for bit, and leave every other column untouched;
* lbm_halo_pack / lbm_halo_unpack against torch slicing;
* the whole overlapped schedule of SlabSolver (edge columns, pack, send /
  receive, interior on a second stream, unpack) with two ranks emulated by two
  host threads on the same GPU: the messages travel through a host-side
  rendezvous that synchronises each thread's stream and copies the buffers
  (no kernel waits on another); the gathered state equals one solver on the
  whole domain bit for bit."""
import threading
import types

import numpy as np
import pytest
import torch

from helpers import dev
from lbm_b200 import init as I
from lbm_b200 import solver as SV
from lbm_b200.slab import SlabSolver

pytestmark = pytest.mark.gpu

CHANNEL = dict(cs_smag=0.1, u_in=0.05, s_nu=1.0 / (3 * 6.4e-4 + 0.5))


@pytest.mark.parametrize("storage", [SV.STORE_F32, SV.STORE_F16DEV])
@pytest.mark.parametrize("T", [2, 4])
def test_columns_tile_the_full_launch(storage, T):
    W, H = 1024, 256
    S = SV.Solver(W, H, storage=storage, **CHANNEL)
    m = dev(I.cylinder_mask(W, H, 256, 128, 48, value=I.OBSTACLE))
    f = S.new_state()
    SV.convert_state(dev(I.perturbed_state(W, H, 3, amp=0.02)), SV.STORE_F32, f, storage)
    full = f.clone()
    S.run_columns(f, full, m, T, 0, W)  # the whole width as one range
    ref = f.clone()
    assert S.run(f, ref, m, T, T) == 1
    assert torch.equal(full.view(torch.int16) if storage else full, ref.view(torch.int16) if storage else ref)
    tiled = f.clone()
    for x0, x1 in ((0, 384), (384, 390), (390, 1000), (1000, 1024)):
        S.run_columns(f, tiled, m, T, x0, x1)
    assert torch.equal(tiled.view(torch.int16) if storage else tiled, ref.view(torch.int16) if storage else ref)
    # columns outside the range keep their contents (as do solid cells inside it:
    # the mask's top and bottom rows and the cylinder are never written)
    part = torch.full_like(f, 7.0)
    S.run_columns(f, part, m, T, 200, 520)
    fl = (m[:, 200:520] == 0).expand(9, H, 320)
    assert torch.equal(part[:, :, 200:520].float()[fl], ref[:, :, 200:520].float()[fl])
    assert bool((part[:, :, 200:520][~fl] == 7.0).all())
    assert bool((part[:, :, :200] == 7.0).all()) and bool((part[:, :, 520:] == 7.0).all())
    S.close()


def test_columns_refuse_odd_bounds_and_periodic_x():
    W, H = 512, 64
    S = SV.Solver(W, H, **CHANNEL)
    f = S.new_state()
    g = f.clone()
    m = torch.zeros((H, W), dtype=torch.uint8, device="cuda")
    with pytest.raises(Exception):
        S.run_columns(f, g, m, 2, 1, 100)
    P = SV.Solver(W, H, bc_left=SV.BC_PERIODIC, bc_right=SV.BC_PERIODIC, **CHANNEL)
    with pytest.raises(Exception):
        P.run_columns(f, g, m, 2, 0, 100)


@pytest.mark.parametrize("storage,dt", [(SV.STORE_F32, torch.float32), (SV.STORE_F16DEV, torch.float16),
                                        (SV.STORE_F64, torch.float64)])
def test_halo_pack_unpack(storage, dt):
    W, H, h = 100, 37, 5
    f = torch.randn((9, H, W), device="cuda").to(dt)
    buf = torch.zeros((2, 9, H, h), dtype=dt, device="cuda")
    SV.halo_pack(f, storage, 10, 80, h, buf)
    assert torch.equal(buf[0], f[:, :, 10:15]) and torch.equal(buf[1], f[:, :, 80:85])
    buf2 = torch.full((2, 9, H, h), 3.0, dtype=dt, device="cuda")
    SV.halo_pack(f, storage, -1, 0, h, buf2)  # one side only
    assert bool((buf2[0] == 3.0).all()) and torch.equal(buf2[1], f[:, :, 0:5])
    g = torch.zeros_like(f)
    SV.halo_unpack(g, storage, 0, W - h, h, buf)
    assert torch.equal(g[:, :, :h], buf[0]) and torch.equal(g[:, :, W - h:], buf[1])
    assert bool((g[:, :, h:W - h] == 0).all())


class _Rendezvous:
    def __init__(self, n):
        self.bar = threading.Barrier(n, timeout=60)
        self.posts = {}


class _ThreadComm:
    """torch.distributed's point-to-point calls for ranks that are threads of one
    process: a batch of sends and receives meets the partner's batch at a host
    barrier, after each thread's stream has finished the sent buffers."""

    isend, irecv = "isend", "irecv"

    def __init__(self, rv, rank, world):
        self.rv, self.rank, self.world = rv, rank, world

    class P2POp:
        def __init__(self, op, tensor, peer, group=None):
            self.op, self.tensor, self.peer = op, tensor, peer

    def get_world_size(self, group=None):
        return self.world

    def get_rank(self, group=None):
        return self.rank

    def get_global_rank(self, group, r):
        return r

    def batch_isend_irecv(self, ops):
        torch.cuda.current_stream().synchronize()
        self.rv.posts[self.rank] = [(o.peer, o.tensor) for o in ops if o.op == "isend"]
        self.rv.bar.wait()
        recvs = [(o.peer, o.tensor) for o in ops if o.op == "irecv"]
        for peer in sorted(set(p for p, _ in recvs)):
            mine = [t for p, t in recvs if p == peer]
            theirs = [t for dst, t in self.rv.posts[peer] if dst == self.rank]
            for a, b in zip(mine, theirs):
                a.copy_(b)
        torch.cuda.current_stream().synchronize()
        self.rv.bar.wait()  # both copied before either reuses its send buffer
        return [types.SimpleNamespace(wait=lambda: None)]


@pytest.mark.parametrize("storage", [SV.STORE_F32, SV.STORE_F16DEV])
def test_overlapped_slabs_equal_whole_domain(storage):
    W, H, T, halo, n = 1008, 256, 2, 8, 24  # local widths 512 = 504 + 8: multiples of 16
    m = I.cylinder_mask(W, H, 300, 128, 48, value=I.OBSTACLE)
    f0 = I.perturbed_state(W, H, 5, amp=0.02)
    kw = dict(CHANNEL, storage=storage)
    whole = SV.Solver(W, H, **kw)
    a = whole.new_state()
    SV.convert_state(dev(f0), SV.STORE_F32, a, storage)
    b = a.clone()
    ref = (b if whole.run(a, b, dev(m), n, T) else a).clone()
    torch.cuda.synchronize()

    rv = _Rendezvous(2)
    solvers, errors = [None, None], []

    def rank_main(r):
        try:
            S = SlabSolver(W, H, torch.from_numpy(m), T=T, halo=halo, comm=_ThreadComm(rv, r, 2), **kw)
            assert S.overlap
            g0 = torch.empty((9, H, W), dtype=S.dtype, device="cuda")
            SV.convert_state(dev(f0), SV.STORE_F32, g0, storage)
            S.set_state(g0)
            S.run(n)
            torch.cuda.current_stream().synchronize()
            solvers[r] = S
        except Exception as e:  # reported below
            errors.append(e)
            rv.bar.abort()

    threads = [threading.Thread(target=rank_main, args=(r,)) for r in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    got = torch.cat([solvers[0].owned(), solvers[1].owned()], dim=2)
    if storage != SV.STORE_F32:
        got, ref = got.view(torch.int16), ref.view(torch.int16)
    assert torch.equal(got, ref)
