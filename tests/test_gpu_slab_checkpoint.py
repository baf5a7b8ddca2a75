"""GPU: the slab layer on one rank through the CUDA path, and checkpoint / resume
of the general solver (a resumed run must continue exactly)."""
import numpy as np
import pytest
import torch

import oracle as O
from helpers import REL_TOL, dev, host, rel_l2
from lbm_b200 import checkpoint as CK
from lbm_b200 import init as I
from lbm_b200 import solver as SV
from lbm_b200.slab import SlabSolver

pytestmark = pytest.mark.gpu

CHANNEL = dict(bc_left=SV.BC_ZOUHE_RAMP, bc_right=SV.BC_OUTFLOW, bc_y=SV.BC_WALL, s_nu=1.8, cs_smag=0.1, u_in=0.05,
               ref_clamps=1)
PERIODIC = dict(bc_left=SV.BC_PERIODIC, bc_right=SV.BC_PERIODIC, bc_y=SV.BC_PERIODIC, s_nu=1.5, ref_clamps=0,
                collision=SV.COLL_BGK, closure=SV.CLOSURE_NONE)


def test_single_rank_slab_is_the_plain_solver():
    W, H, n = 256, 96, 12
    m = I.random_discs_mask(W, H, 3, 3.0, 6.0, 4)
    f0 = I.perturbed_state(W, H, 5, amp=0.02)
    S = SlabSolver(W, H, torch.from_numpy(m), T=2, **CHANNEL)
    S.set_state(torch.from_numpy(f0))
    S.run(n)
    P = SV.Solver(W, H, **CHANNEL)
    a, b = dev(f0), dev(f0)
    which = P.run(a, b, dev(m), n, 2)
    assert torch.equal(S.gather(), b if which else a)
    d = S.diag()
    assert torch.allclose(d, P.diag(b if which else a, dev(m)), rtol=1e-12, atol=1e-9)


def test_single_rank_periodic_slab_matches_oracle():
    W, H, n = 128, 64, 8
    m = np.zeros((H, W), np.uint8)
    m[20:26, 40:46] = 1
    f0 = I.perturbed_state(W, H, 6, amp=0.02)
    S = SlabSolver(W, H, torch.from_numpy(m), T=4, **PERIODIC)
    S.set_state(torch.from_numpy(f0))
    S.run(n)
    G = O.General(W, H, collision="bgk", closure="none", s_nu=1.5, bc_left="periodic", bc_right="periodic",
                  bc_y="periodic", ref_clamps=False)
    ref, _ = G.run(m, f0, n)
    assert rel_l2(host(S.gather()), ref) < REL_TOL


@pytest.mark.parametrize("storage", [SV.STORE_F32, SV.STORE_F16DEV])
def test_checkpoint_resume_continues_exactly(tmp_path, storage):
    W, H = 192, 80
    m = dev(I.random_discs_mask(W, H, 2, 3.0, 5.0, 8))
    S = SV.Solver(W, H, storage=storage, **CHANNEL)
    a = S.new_state()
    SV.convert_state(dev(I.perturbed_state(W, H, 9, amp=0.02)), SV.STORE_F32, a, storage)
    b = a.clone()
    which = S.run(a, b, m, 10, 2)
    cur = b if which else a
    path = str(tmp_path / "run")
    CK.save(path, cur, m, storage=storage, step=10, params=S.params)
    nxt = a if which else b
    w2 = S.run(cur, nxt, m, 10, 2)
    straight = (nxt if w2 else cur).clone()
    f, mk, hdr = CK.load(path)
    S2 = SV.Solver(W, H, params=CK.params_from_header(hdr))
    g = f.clone()
    w3 = S2.run(f, g, mk, 10, 2)
    assert hdr["step"] == 10
    assert torch.equal((g if w3 else f), straight)


def test_checkpoint_resume_of_a_learned_closure_run(tmp_path):
    """The packed network travels with the checkpoint: a resumed learned-closure
    run (new process state: weights reloaded from <path>.mlp into a new device
    buffer) continues bit for bit."""
    import numpy as np

    from lbm_b200 import closure as CL

    W, H = 192, 80
    rng = np.random.default_rng(3)
    net = CL.Mlp(params=CL.init_params(3) + (0.05 * rng.standard_normal(CL.NPARAM)).astype(np.float32),
                 in_scale=np.full(5, 300.0, np.float32), out_scale=0.002)
    kw = dict(CHANNEL, ref_clamps=0, closure=SV.CLOSURE_MLP, storage=SV.STORE_F16DEV)
    m = dev(I.random_discs_mask(W, H, 2, 3.0, 5.0, 8))
    S = SV.Solver(W, H, mlp=net.packed().data_ptr(), **kw)
    a = S.new_state()
    SV.convert_state(dev(I.perturbed_state(W, H, 9, amp=0.02)), SV.STORE_F32, a, SV.STORE_F16DEV)
    b = a.clone()
    which = S.run(a, b, m, 10, 2)
    cur, nxt = (b, a) if which else (a, b)
    path = str(tmp_path / "mlp_run")
    CK.save(path, cur, m, storage=SV.STORE_F16DEV, step=10, params=S.params, mlp_packed=net.packed())
    w2 = S.run(cur, nxt, m, 10, 2)
    straight = (nxt if w2 else cur).clone()
    f, mk, hdr = CK.load(path)
    packed = CK.load_mlp(path)
    assert packed.data_ptr() != net.packed().data_ptr()
    S2 = SV.Solver(W, H, params=CK.params_from_header(hdr, mlp=packed))
    g = f.clone()
    w3 = S2.run(f, g, mk, 10, 2)
    assert torch.equal((g if w3 else f), straight)


@pytest.mark.parametrize("params", [PERIODIC, CHANNEL], ids=["periodic", "channel"])
def test_graph_replayed_slab_run_equals_per_launch_run(params):
    """A single-rank slab run replays pairs of (launch, halo copy) from CUDA
    graphs; calls shorter than two launches take the per-launch loop.  Both must
    give the same state bit for bit."""
    W, H = 240, 96
    m = np.zeros((H, W), np.uint8) if params is PERIODIC else I.random_discs_mask(W, H, 3, 3.0, 6.0, 8)
    f0 = I.perturbed_state(W, H, 9, amp=0.02)
    A = SlabSolver(W, H, torch.from_numpy(m), T=2, **params)
    A.set_state(torch.from_numpy(f0))
    A.run(40)  # graph replays (10 pairs)
    B = SlabSolver(W, H, torch.from_numpy(m), T=2, **params)
    B.set_state(torch.from_numpy(f0))
    for _ in range(20):
        B.run(2)  # one launch per call: the per-launch path
    assert A.steps_done == B.steps_done == 40
    assert torch.equal(A.gather(), B.gather())
    A.run(7)  # 1 pair by graph + 1 launch of 2 + 1 launch of 1
    for n in (2, 2, 2, 1):
        B.run(n)
    assert torch.equal(A.gather(), B.gather())
