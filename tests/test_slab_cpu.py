"""x-slab decomposition (lbm_b200.slab) on CPU: gloo ranks in spawned processes,
each advancing its slab with the oracle; the gathered state must equal the
oracle's run of the whole domain bit for bit (same per-cell arithmetic), and the
global FP64 mass/momentum must equal the whole-domain sums."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle as O
from lbm_b200 import init as I
from lbm_b200 import solver as SV

NAMES = {SV.BC_WALL: "wall", SV.BC_PERIODIC: "periodic", SV.BC_ZOUHE: "zouhe", SV.BC_ZOUHE_RAMP: "zouhe_ramp",
         SV.BC_OUTFLOW: "outflow"}

CASES = {
    "channel": dict(bc_left=SV.BC_ZOUHE_RAMP, bc_right=SV.BC_OUTFLOW, bc_y=SV.BC_WALL, s_nu=1.8, cs_smag=0.1,
                    u_in=0.05, ref_clamps=1, collision=SV.COLL_MRT, closure=SV.CLOSURE_SMAG),
    "periodic": dict(bc_left=SV.BC_PERIODIC, bc_right=SV.BC_PERIODIC, bc_y=SV.BC_PERIODIC, s_nu=1.5, ref_clamps=0,
                     collision=SV.COLL_BGK, closure=SV.CLOSURE_NONE),
}


def oracle_kwargs(p):
    return dict(collision="mrt" if p["collision"] == SV.COLL_MRT else "bgk",
                closure="smag" if p["closure"] == SV.CLOSURE_SMAG else "none", s_nu=p["s_nu"],
                cs=p.get("cs_smag", 0.2), bc_left=NAMES[p["bc_left"]], bc_right=NAMES[p["bc_right"]],
                bc_y=NAMES[p["bc_y"]], u_in=p.get("u_in", 0.1), ref_clamps=bool(p["ref_clamps"]))


def oracle_stepper(width, H, local):
    G = O.General(width, H, **oracle_kwargs(local))

    def step(fa, fb, m, n, t):
        a, b, mm = fa.numpy(), fb.numpy(), m.numpy()
        for _ in range(n):
            G.step(mm, a, b)
            a, b = b, a
        return n % 2

    return step


class OracleColumnsStepper:
    """The oracle stepper with a column-restricted launch (enables the overlapped
    exchange): t steps from f_a computed into scratch copies, then only columns
    [x0, x1) copied into f_b (f_a unchanged).  `log` records the calls."""

    def __init__(self, width, H, local, log=None):
        self.G = O.General(width, H, **oracle_kwargs(local))
        self.log = log

    def __call__(self, fa, fb, m, n, t):
        if self.log is not None:
            self.log.append(("full",))
        a, b, mm = fa.numpy(), fb.numpy(), m.numpy()
        for _ in range(n):
            self.G.step(mm, a, b)
            a, b = b, a
        return n % 2

    def columns(self, fa, fb, m, t, x0, x1):
        if self.log is not None:
            self.log.append(("cols", x0, x1))
        a, b, mm = fa.numpy().copy(), fb.numpy().copy(), m.numpy()
        for _ in range(t):
            self.G.step(mm, a, b)
            a, b = b, a
        fb.numpy()[:, :, x0:x1] = a[:, :, x0:x1]


def inputs(name, W, H):
    if name == "channel":
        m = I.random_discs_mask(W, H, 2, 2.0, 4.0, 7)
    else:
        m = np.zeros((H, W), np.uint8)
        m[H // 3:H // 3 + 3, W // 2:W // 2 + 4] = 1
    return m, I.perturbed_state(W, H, 11, amp=0.02)


def _rank_main(rank, world, port, name, W, H, T, n, q, overlap=False):
    import torch.distributed as dist

    from lbm_b200.slab import SlabSolver

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m, f0 = inputs(name, W, H)
        step = OracleColumnsStepper if overlap else oracle_stepper
        S = SlabSolver(W, H, torch.from_numpy(m), T=T, stepper=step, device="cpu", overlap=overlap, **CASES[name])
        assert S.overlap == overlap
        S.set_state(torch.from_numpy(f0))
        S.run(n)
        d = S.diag()
        g = S.gather()
        if rank == 0:
            q.put((g.numpy(), d.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("overlap", [False, True], ids=["plain", "overlapped"])
@pytest.mark.parametrize("name,world", [("channel", 2), ("channel", 3), ("periodic", 2), ("periodic", 3)])
def test_slabs_equal_whole_domain(name, world, overlap):
    W, H, T, n = 48, 20, 2, 7
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, name, W, H, T, n, q, overlap))
             for r in range(world)]
    for p in procs:
        p.start()
    got, d = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    m, f0 = inputs(name, W, H)
    ref, _ = O.General(W, H, **oracle_kwargs(CASES[name])).run(m, f0, n)
    assert np.array_equal(got, ref)
    fl = m == 0
    cx = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], np.float64)[:, None, None]
    cy = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], np.float64)[:, None, None]
    r64 = ref.astype(np.float64)
    want = [(r64 * fl).sum(), (r64 * cx * fl).sum(), (r64 * cy * fl).sum()]
    assert np.allclose(d, want, rtol=1e-12, atol=1e-9)


def test_single_rank_periodic_self_exchange():
    """One rank with periodic x: both halos come from the rank's own opposite edge."""
    from lbm_b200.slab import SlabSolver

    W, H, T, n = 32, 12, 2, 6
    m, f0 = inputs("periodic", W, H)
    S = SlabSolver(W, H, torch.from_numpy(m), T=T, stepper=oracle_stepper, device="cpu", **CASES["periodic"])
    assert S.lay.width == W + 2 * T
    S.set_state(torch.from_numpy(f0))
    S.run(n)
    ref, _ = O.General(W, H, **oracle_kwargs(CASES["periodic"])).run(m, f0, n)
    assert np.array_equal(S.gather().numpy(), ref)


def test_layout_split_and_halo_rules():
    from lbm_b200.slab import split_columns

    lays = split_columns(100, 3, 4, False)
    assert [(l.x0, l.x1) for l in lays] == [(0, 33), (33, 66), (66, 100)]
    assert (lays[0].left, lays[0].right, lays[2].left, lays[2].right) == (0, 4, 4, 0)
    assert lays[1].global_columns()[0] == 29
    per = split_columns(100, 3, 4, True)
    assert per[0].global_columns()[:4] == [96, 97, 98, 99]
    with pytest.raises(ValueError):
        split_columns(10, 4, 4, False)


def _ckpt_main(rank, world, port, W, H, T, n, path, mode, q):
    import torch.distributed as dist

    from lbm_b200.slab import SlabSolver

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m, f0 = inputs("channel", W, H)
        S = SlabSolver(W, H, torch.from_numpy(m), T=T, stepper=oracle_stepper, device="cpu", **CASES["channel"])
        if mode == "save":
            S.set_state(torch.from_numpy(f0))
            S.run(n)
            S.save(path, torch.from_numpy(m))
        else:
            S.load(path)
            S.run(n)
            g = S.gather()
            if rank == 0:
                q.put((g.numpy(), S.steps_done))
    finally:
        dist.destroy_process_group()


def test_checkpoint_written_by_two_ranks_resumes_on_three(tmp_path):
    W, H, T = 48, 20, 2
    path = str(tmp_path / "slabs")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    for world, mode in ((2, "save"), (3, "load")):
        port = _free_port()
        procs = [ctx.Process(target=_ckpt_main, args=(r, world, port, W, H, T, 5, path, mode, q))
                 for r in range(world)]
        for p in procs:
            p.start()
        if mode == "load":
            got, steps = q.get(timeout=240)
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
    m, f0 = inputs("channel", W, H)
    ref, _ = O.General(W, H, **oracle_kwargs(CASES["channel"])).run(m, f0, 10)
    assert steps == 10
    assert np.array_equal(got, ref)


def _order_main(rank, world, port, W, H, T, q):
    import torch.distributed as dist

    from lbm_b200.slab import SlabSolver

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        log = []
        real = dist.batch_isend_irecv

        class _Logged:
            def __init__(self, w):
                self.w = w

            def wait(self):
                log.append(("wait",))
                return self.w.wait()

        def logged(ops):
            log.append(("send", len(ops)))
            return [_Logged(w) for w in real(ops)]

        dist.batch_isend_irecv = logged
        m, f0 = inputs("channel", W, H)
        S = SlabSolver(W, H, torch.from_numpy(m), T=T, device="cpu", overlap=True,
                       stepper=lambda w, h, loc: OracleColumnsStepper(w, h, loc, log), **CASES["channel"])
        S.set_state(torch.from_numpy(f0))
        S.run(2 * T)
        q.put((rank, S.lay.left, S.lay.x1 - S.lay.x0, log))
    finally:
        dist.destroy_process_group()


def test_overlapped_schedule_order():
    """Three ranks, two launches: each launch computes the edge columns the
    neighbours need, then posts the sends and receives, then computes the
    interior while they are in flight, and only then waits; no full-domain step
    runs.  The middle rank has two edges, the end ranks one."""
    W, H, T, world = 48, 20, 2, 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_order_main, args=(r, world, port, W, H, T, q)) for r in range(world)]
    for p in procs:
        p.start()
    logs = {}
    for _ in range(world):
        rank, left, n, log = q.get(timeout=240)
        logs[rank] = (left, n, log)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, (left, n, log) in logs.items():
        h = T
        edges = []
        if rank > 0:
            edges.append(("cols", left, left + h))
        if rank < world - 1:
            edges.append(("cols", left + n - h, left + n))
        i0 = left + (h if rank > 0 else 0)
        i1 = left + n - (h if rank < world - 1 else 0)
        n_ops = 2 * len(edges)
        waits = [("wait",)] * n_ops
        one = edges + [("send", n_ops), ("cols", i0, i1)] + waits
        assert log == one + one, (rank, log)
