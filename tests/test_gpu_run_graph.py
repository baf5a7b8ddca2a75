"""lbm_run's CUDA-graph replay of ping-pong launch pairs is bit-identical to
plain launches.  The plain sequence is made by calling lbm_run one launch at a
time (a single launch never uses the graph); the graph path by one call with
many pairs, then again with the cached graph, then with another key (buffers
swapped, another depth) that forces a new capture."""
import numpy as np
import pytest
import torch

from helpers import dev, host
from lbm_b200 import init as I
from lbm_b200 import solver as SV

pytestmark = pytest.mark.gpu

CASES = {
    "cavity_256": dict(W=256, H=256, kw=dict(collision=SV.COLL_MRT, closure=SV.CLOSURE_NONE, bc_left=SV.BC_WALL,
                                             bc_right=SV.BC_WALL, u_lid=0.1, ref_clamps=0, s_nu=1.7)),
    "channel_discs": dict(W=300, H=130, kw=dict(cs_smag=0.1, u_in=0.05, s_nu=1.9)),
}


def _mask(name, W, H):
    if name.startswith("cavity"):
        return I.cavity_mask(W, H)
    return I.random_discs_mask(W, H, 3, 3.0, 6.0, 5)


def _plain(S, a, b, m, n, T, mac):
    """n steps as single-launch lbm_run calls (each call: one launch, no graph)."""
    src, dst, done = a, b, 0
    while done < n:
        t = min(T, n - done)
        last = done + t == n
        w = S.run(src, dst, m, t, t, *(mac if last else (None, None, None)))
        assert w == 1
        src, dst = dst, src
        done += t
    return src  # the buffer holding the final state


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("n,T", [(40, 2), (43, 2), (57, 4), (16, 1)])
def test_graph_replay_matches_plain_launches(name, n, T):
    c = CASES[name]
    W, H = c["W"], c["H"]
    m = dev(_mask(name, W, H))
    f0 = I.perturbed_state(W, H, 3, amp=0.02)
    S = SV.Solver(W, H, **c["kw"])
    mac_p = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    mac_g = [torch.zeros((H, W), device="cuda") for _ in range(3)]
    a, b = dev(f0), dev(f0)
    ref = host(_plain(S, a, b, m, n, T, mac_p))
    ga, gb = dev(f0), dev(f0)
    G = SV.Solver(W, H, **c["kw"])
    which = G.run(ga, gb, m, n, T, *mac_g)
    got = host(gb if which else ga)
    assert np.array_equal(got, ref)
    for x, y in zip(mac_g, mac_p):
        assert torch.equal(x, y)
    # the same key again, continuing from the result: the cached graph replays from the first pair on
    ref2 = host(_plain(S, dev(ref), dev(ref), m, n, T, mac_p))
    ga.copy_(dev(ref))
    gb.copy_(dev(ref))
    which2 = G.run(ga, gb, m, n, T, *mac_g)
    assert np.array_equal(host(gb if which2 else ga), ref2)
    for x, y in zip(mac_g, mac_p):
        assert torch.equal(x, y)
    # another key (new buffers): a new capture
    sa, sb = dev(f0), dev(f0)
    which3 = G.run(sa, sb, m, n, T)
    assert np.array_equal(host(sb if which3 else sa), ref)
    G.close()
    S.close()


def test_graph_is_skipped_inside_a_caller_capture():
    """A caller that captures lbm_run into its own graph gets the plain
    launches recorded there; replaying that graph gives the same state."""
    W, H = 256, 256
    c = CASES["cavity_256"]
    m = dev(_mask("cavity_256", W, H))
    f0 = I.perturbed_state(W, H, 4, amp=0.02)
    S = SV.Solver(W, H, **c["kw"])
    a, b = dev(f0), dev(f0)
    ref = host(_plain(S, a, b, m, 24, 2, (None, None, None)))
    ga, gb = dev(f0), dev(f0)
    st = torch.cuda.Stream()
    G = SV.Solver(W, H, **c["kw"])
    G.run(ga, gb, m, 4, 2, stream=st)  # the per-device setup calls run outside the capture
    ga.copy_(dev(f0))
    gb.copy_(dev(f0))
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=st):
        which = G.run(ga, gb, m, 24, 2, stream=st)
    graph.replay()
    torch.cuda.synchronize()
    assert np.array_equal(host(gb if which else ga), ref)
    del graph
    G.close()
    S.close()


def test_alternating_buffer_order_keeps_both_graphs():
    """A caller that swaps (f_a, f_b) after each call of an odd launch count
    alternates between two cached graphs; the state matches plain launches."""
    c = CASES["channel_discs"]
    W, H = c["W"], c["H"]
    m = dev(_mask("channel_discs", W, H))
    f0 = I.perturbed_state(W, H, 6, amp=0.02)
    S = SV.Solver(W, H, **c["kw"])
    G = SV.Solver(W, H, **c["kw"])
    x, y = dev(f0), dev(f0)
    p, q = dev(f0), dev(f0)
    for _ in range(5):
        w = G.run(x, y, m, 42, 2)  # 21 launches: the result is in the second buffer
        assert w == 1
        x, y = y, x
        r = _plain(S, p, q, m, 42, 2, (None, None, None))
        p, q = (r, p) if r is q else (r, q)
        assert np.array_equal(host(x), host(p))
    G.close()
    S.close()


def test_graph_reset_then_new_buffers():
    """lbm_run_graph_reset drops the cached graphs: after it, new state buffers
    (here freed and reallocated, so they may reuse the old addresses) run
    correctly; the state equals plain launches."""
    c = CASES["channel_discs"]
    W, H = c["W"], c["H"]
    m = dev(_mask("channel_discs", W, H))
    f0 = I.perturbed_state(W, H, 7, amp=0.02)
    S = SV.Solver(W, H, **c["kw"])
    G = SV.Solver(W, H, **c["kw"])
    x, y = dev(f0), dev(f0)
    G.run(x, y, m, 40, 2)  # captures a graph for (x, y, m, 2)
    G.reset_graphs()
    G.reset_graphs()  # idempotent
    del x, y
    torch.cuda.synchronize()
    x, y = dev(f0), dev(f0)
    w = G.run(x, y, m, 40, 2)
    p, q = dev(f0), dev(f0)
    r = _plain(S, p, q, m, 40, 2, (None, None, None))
    assert np.array_equal(host(y if w else x), host(r))
    G.close()
    S.close()
