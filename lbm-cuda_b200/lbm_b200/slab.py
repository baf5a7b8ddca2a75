"""x-slab decomposition of one W x H domain over the ranks of a process group.

Rank r owns the columns [x0, x1) of an even split of W.  Its local domain adds
`halo` columns on each side that has a neighbour (every side when x is
periodic); the physical boundary conditions apply only at the domain's true
ends (the Zou-He inlet on the first rank, the outlet on the last).  A launch of
T <= halo steps runs on the local domain with walls at the halo edges: the wrong
values those walls produce travel one column per step, so after T steps they
are confined to the halo.  Then neighbouring ranks exchange their outermost
owned columns (one send/recv pair per side, torch.distributed: NCCL between
GPUs, gloo on CPU) and the halos are current again.

With more than one rank the exchange overlaps the launch (`overlap`, on by
default where the steps can be restricted to a column range): each launch
first computes the owned edge columns that the neighbours need (h columns per
side with a neighbour), packs them into one contiguous buffer (one kernel),
and starts the send/receive pairs; the interior columns compute meanwhile (on a
second CUDA stream on the GPU); the received columns are then unpacked into
the halos (one kernel).  The result equals the plain schedule bit for bit:
every column is computed by the same kernel from the same inputs.

Global mass and momentum are the FP64 sums over the owned columns of every rank
(one all-reduce of three doubles).  `gather` / `scatter` move the global state
to and from rank 0 (checkpoints, output).
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass
class SlabLayout:
    W: int
    H: int
    world: int
    rank: int
    halo: int
    periodic_x: bool

    @property
    def x0(self) -> int:
        return self.W * self.rank // self.world

    @property
    def x1(self) -> int:
        return self.W * (self.rank + 1) // self.world

    @property
    def left(self) -> int:  # halo columns on the left
        return self.halo if (self.periodic_x or self.rank > 0) else 0

    @property
    def right(self) -> int:
        return self.halo if (self.periodic_x or self.rank < self.world - 1) else 0

    @property
    def width(self) -> int:  # local width including halos
        return self.x1 - self.x0 + self.left + self.right

    def global_columns(self):
        """Global column of every local column (wrapped when x is periodic)."""
        cols = range(self.x0 - self.left, self.x1 + self.right)
        return [c % self.W for c in cols] if self.periodic_x else list(cols)


def split_columns(W: int, world: int, halo: int, periodic_x: bool):
    """Layouts of all ranks; every owned slab must be at least `halo` wide."""
    lays = [SlabLayout(W, 0, world, r, halo, periodic_x) for r in range(world)]
    for lay in lays:
        if lay.x1 - lay.x0 < halo:
            raise ValueError(f"slab of rank {lay.rank} is narrower than the halo ({lay.x1 - lay.x0} < {halo})")
    return lays


class SlabSolver:
    """Runs the general solver on this rank's slab.

    `stepper`, when given, is a factory make(width, H, local_params) returning
    step(f_a, f_b, mask, n_steps, T) -> 1 if the result is in f_b, else 0, which
    advances a local state (torch tensors (9, H, width) and (H, width)); a step
    with a `columns(f_a, f_b, mask, T, x0, x1)` attribute (one launch writing
    only columns [x0, x1) of f_b) enables the overlapped exchange.  By default
    the steps run on the GPU through `solver.Solver` built for the local width
    with the local boundary conditions (lbm_run, lbm_run_columns).  `params` are the global
    lbm_params overrides (bc_left, bc_right, bc_y, physics); `group` a
    torch.distributed process group (None: the default group, or a single rank
    when torch.distributed is not set up); `comm` another object with the
    torch.distributed calls used here (get_rank, get_world_size, P2POp, isend,
    irecv, batch_isend_irecv, all_reduce, send, recv, broadcast, barrier,
    get_global_rank), for a transport of the caller's own.  The GPU kernels want
    local widths (owned columns plus halos) that are multiples of 16 columns
    (TMA rows); choose `halo` accordingly.
    """

    def __init__(self, W: int, H: int, mask, T: int = 2, halo: int | None = None, group=None, stepper=None,
                 device=None, overlap: bool = True, comm=None, **params):
        import torch

        from . import solver as SV

        self.dist = comm
        self.group = group
        if comm is None:
            try:
                import torch.distributed as dist

                if dist.is_available() and dist.is_initialized():
                    self.dist = dist
            except ImportError:
                pass
        self.world = self.dist.get_world_size(group) if self.dist else 1
        self.rank = self.dist.get_rank(group) if self.dist else 0
        self.T = int(T)
        self.halo = int(halo) if halo is not None else self.T
        if self.halo < self.T:
            raise ValueError("the halo must be at least T columns wide")
        self.W, self.H = int(W), int(H)
        bc_left = params.get("bc_left", SV.default_params(W, H).bc_left)
        bc_right = params.get("bc_right", SV.default_params(W, H).bc_right)
        self.periodic_x = bc_left == SV.BC_PERIODIC
        self.lay = split_columns(self.W, self.world, self.halo, self.periodic_x)[self.rank]
        self.lay.H = self.H
        lay = self.lay
        self.device = device if device is not None else ("cuda" if stepper is None else "cpu")
        self.global_params = dict(params)
        local = dict(params)
        local["bc_left"] = bc_left if (lay.left == 0) else SV.BC_WALL
        local["bc_right"] = bc_right if (lay.right == 0) else SV.BC_WALL
        self.local_params = local
        cols = torch.tensor(lay.global_columns(), dtype=torch.long)
        self.mask = mask[:, cols].contiguous().to(self.device)
        self._columns = None  # one launch restricted to a column range, or None
        if stepper is None:
            self._solver = SV.Solver(lay.width, self.H, **local)
            self.dtype = self._solver.dtype

            def stepper(f_a, f_b, m, n, t):
                return self._solver.run(f_a, f_b, m, n, t)

            def columns(f_a, f_b, m, t, x0, x1):
                self._solver.run_columns(f_a, f_b, m, t, x0, x1)

            self.storage = self._solver.params.storage
            self._columns = columns
        else:
            self._solver = None
            self.dtype = torch.float32
            self.storage = SV.STORE_F32
            stepper = stepper(lay.width, self.H, local)
            self._columns = getattr(stepper, "columns", None)
        self.stepper = stepper
        self.overlap = bool(overlap) and self._columns is not None and self.world > 1
        self._bufs = None
        self._side = None
        self.f = None
        self.g = None
        self.steps_done = 0

    # ---- state ----
    def set_state(self, f_global):
        """Takes this rank's columns (halos included) of a global state (9, H, W)."""
        import torch

        cols = torch.tensor(self.lay.global_columns(), dtype=torch.long)
        self.f = f_global[:, :, cols].to(device=self.device, dtype=self.dtype).contiguous()
        self.g = self.f.clone()

    def set_local_state(self, f_local):
        """Takes this rank's local state (9, H, width), halos included, as it is
        (the halos become current after the first launch's exchange)."""
        if tuple(f_local.shape) != (9, self.H, self.lay.width):
            raise ValueError(f"local state must be (9, {self.H}, {self.lay.width})")
        self.f = f_local.to(device=self.device, dtype=self.dtype).contiguous()
        self.g = self.f.clone()

    def owned(self):
        """View of the owned columns of the local state."""
        lay = self.lay
        return self.f[:, :, lay.left:lay.left + (lay.x1 - lay.x0)]

    # ---- halo exchange ----
    def _neighbours(self):
        left = self.rank - 1 if self.rank > 0 else (self.world - 1 if self.periodic_x else None)
        right = self.rank + 1 if self.rank < self.world - 1 else (0 if self.periodic_x else None)
        return left, right

    def exchange(self):
        """Refresh both halos from the neighbours' owned edge columns."""
        self._exchange(self.f)

    def _exchange(self, f):
        lay, h = self.lay, self.halo
        n = lay.x1 - lay.x0
        left, right = self._neighbours()
        if self.world == 1 and left is not None and f.is_cuda and lay.left == lay.right == h:
            # periodic single rank on the GPU: both halos in one launch
            from . import _ptr, _stream
            from ._lib import call

            call("lbm_periodic_halo_x", _ptr(f), int(f.shape[2]), self.H, h, int(self.storage), _stream(None))
            return
        send_l = f[:, :, lay.left:lay.left + h].contiguous() if left is not None else None
        send_r = f[:, :, lay.left + n - h:lay.left + n].contiguous() if right is not None else None
        recv_l = f.new_empty((9, self.H, h)) if left is not None else None
        recv_r = f.new_empty((9, self.H, h)) if right is not None else None
        if self.world == 1:
            # periodic single rank: each halo is the owned edge at the other end
            if left is not None:
                recv_l.copy_(send_r)
                recv_r.copy_(send_l)
        else:
            dist = self.dist
            ops = []
            # a rank pair exchanges in both directions; when left == right (two
            # ranks, periodic) the two messages are told apart by their order
            if left is not None:
                ops.append(dist.P2POp(dist.isend, send_l, self._peer(left), self.group))
                ops.append(dist.P2POp(dist.irecv, recv_l, self._peer(left), self.group))
            if right is not None:
                ops.append(dist.P2POp(dist.isend, send_r, self._peer(right), self.group))
                ops.append(dist.P2POp(dist.irecv, recv_r, self._peer(right), self.group))
            if left is not None and left == right:
                # periodic with two ranks: both messages go to the same peer; pair
                # the first send with the peer's first receive (its right halo)
                ops = [dist.P2POp(dist.isend, send_l, self._peer(left), self.group),
                       dist.P2POp(dist.isend, send_r, self._peer(left), self.group),
                       dist.P2POp(dist.irecv, recv_r, self._peer(left), self.group),
                       dist.P2POp(dist.irecv, recv_l, self._peer(left), self.group)]
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if left is not None:
            f[:, :, :lay.left] = recv_l[:, :, h - lay.left:]
        if right is not None:
            f[:, :, lay.left + n:] = recv_r[:, :, :lay.right]

    def _edges(self):
        """Column ranges of one overlapped launch: (left edge, right edge, interior);
        an edge is None on a side without a neighbour (its columns are interior)."""
        lay, h = self.lay, self.halo
        n = lay.x1 - lay.x0
        left, right = self._neighbours()
        el = (lay.left, lay.left + h) if left is not None else None
        er = (lay.left + n - h, lay.left + n) if right is not None else None
        i0 = lay.left + (h if el else 0)
        i1 = lay.left + n - (h if er else 0)
        return el, er, (i0, i1)

    def _overlap_ok(self, t):
        if not self.overlap:
            return False
        el, er, (i0, i1) = self._edges()
        if i1 <= i0:
            return False
        if self._solver is not None:
            # the GPU kernel that restricts its output wants even column bounds
            bounds = [i0, i1] + list(el or ()) + list(er or ())
            if any(b % 2 for b in bounds):
                return False
        return True

    def _launch_overlapped(self, t):
        """One launch of t steps f -> g with the halo exchange overlapped (see the
        module docstring); returns False (nothing done) when the column-restricted
        launch is not available for this configuration."""
        import torch

        from . import solver as SV

        lay, h = self.lay, self.halo
        n = lay.x1 - lay.x0
        left, right = self._neighbours()
        el, er, (i0, i1) = self._edges()
        f, g = self.f, self.g
        gpu = self._solver is not None
        if self._bufs is None:
            self._bufs = (f.new_empty((2, 9, self.H, h)), f.new_empty((2, 9, self.H, h)))
        send, recv = self._bufs
        if gpu:
            cur = torch.cuda.current_stream()
            if self._side is None:
                self._side = torch.cuda.Stream()
            start = torch.cuda.Event()
            start.record(cur)
        try:
            for e in (el, er):
                if e is not None:
                    self._columns(f, g, self.mask, t, e[0], e[1])
        except Exception as exc:  # the restricted launch does not apply: plain schedule from now on
            from ._lib import LbmError

            if isinstance(exc, LbmError) and exc.status == 1002:
                self.overlap = False
                return False
            raise
        if gpu:
            SV.halo_pack(g, self.storage, el[0] if el else -1, er[0] if er else -1, h, send)
            self._side.wait_event(start)
            with torch.cuda.stream(self._side):
                self._columns(f, g, self.mask, t, i0, i1)
        else:
            if el:
                send[0].copy_(g[:, :, el[0]:el[1]])
            if er:
                send[1].copy_(g[:, :, er[0]:er[1]])
        dist = self.dist
        ops = []
        if left is not None and left == right:
            # two ranks, periodic: both messages go to the same peer; the first send
            # pairs with the peer's first receive (its right halo)
            ops = [dist.P2POp(dist.isend, send[0], self._peer(left), self.group),
                   dist.P2POp(dist.isend, send[1], self._peer(left), self.group),
                   dist.P2POp(dist.irecv, recv[1], self._peer(left), self.group),
                   dist.P2POp(dist.irecv, recv[0], self._peer(left), self.group)]
        else:
            if left is not None:
                ops.append(dist.P2POp(dist.isend, send[0], self._peer(left), self.group))
                ops.append(dist.P2POp(dist.irecv, recv[0], self._peer(left), self.group))
            if right is not None:
                ops.append(dist.P2POp(dist.isend, send[1], self._peer(right), self.group))
                ops.append(dist.P2POp(dist.irecv, recv[1], self._peer(right), self.group))
        works = dist.batch_isend_irecv(ops)
        if not gpu:
            self._columns(f, g, self.mask, t, i0, i1)  # the interior while the messages travel
        for w in works:
            w.wait()  # on the GPU: the current stream waits for the transfers
        if gpu:
            SV.halo_unpack(g, self.storage, 0 if left is not None else -1, lay.left + n if right is not None else -1,
                           h, recv)
            cur.wait_stream(self._side)
        else:
            if left is not None:
                g[:, :, :lay.left] = recv[0][:, :, h - lay.left:]
            if right is not None:
                g[:, :, lay.left + n:] = recv[1][:, :, :lay.right]
        return True

    def _graph_pairs(self, pairs: int):
        """`pairs` x (launch f -> g, halo copy on g, launch g -> f, halo copy on f)."""
        import torch

        # one cached pair per buffer order: a call of an odd number of launches
        # swaps f and g, so consecutive calls alternate between two keys
        key = (self.f.data_ptr(), self.g.data_ptr(), self.mask.data_ptr(), self.T)
        cache = self.__dict__.setdefault("_graph_cache", {})
        if key not in cache:
            if len(cache) >= 2:
                cache.clear()
            T = self.T
            # first calls set up per-device state outside the capture (scratch copies)
            a, b = self.f.clone(), self.g.clone()
            self.stepper(a, b, self.mask, T, T)
            self._exchange(b)
            torch.cuda.synchronize()
            del a, b
            graphs = []
            for src, dst in ((self.f, self.g), (self.g, self.f)):
                gr = torch.cuda.CUDAGraph()
                with torch.cuda.graph(gr):
                    self.stepper(src, dst, self.mask, T, T)
                    self._exchange(dst)
                graphs.append(gr)
            cache[key] = graphs
        graphs = cache[key]
        for _ in range(pairs):
            graphs[0].replay()
            graphs[1].replay()

    def _peer(self, r):
        if self.group is None or self.dist is None:
            return r
        return self.dist.get_global_rank(self.group, r)

    # ---- time stepping ----
    def run(self, n_steps: int):
        """n_steps steps, T per launch, one halo exchange after each launch.  On a
        single rank on the GPU, whole pairs of launches replay from CUDA graphs
        (launch, halo copy; twice, one per ping-pong parity): the launch-bound
        loop of small domains then costs no host time per launch."""
        done = 0
        if (self.world == 1 and self._solver is not None and str(self.device).startswith("cuda")
                and n_steps >= 2 * self.T):
            pairs = n_steps // (2 * self.T)
            self._graph_pairs(pairs)
            done = pairs * 2 * self.T
        while done < n_steps:
            t = min(self.T, n_steps - done)
            if self._overlap_ok(t) and self._launch_overlapped(t):
                self.f, self.g = self.g, self.f
            else:
                which = self.stepper(self.f, self.g, self.mask, t, t)
                if which:
                    self.f, self.g = self.g, self.f
                self.exchange()
            done += t
        self.steps_done += n_steps

    # ---- global diagnostics and state movement ----
    def diag(self):
        """Global [mass, momentum_x, momentum_y] (FP64) over every rank's owned columns."""
        import torch

        from . import _lib
        from . import solver as SV

        lay = self.lay
        n = lay.x1 - lay.x0
        own = self.owned().contiguous()
        m = self.mask[:, lay.left:lay.left + n].contiguous()
        if self.device == "cpu" or not str(self.device).startswith("cuda"):
            f = own.double()
            fl = (m == 0).double()
            cx = torch.tensor([0, 1, 0, -1, 0, 1, -1, -1, 1], dtype=torch.float64).view(9, 1, 1)
            cy = torch.tensor([0, 0, 1, 0, -1, 1, 1, -1, -1], dtype=torch.float64).view(9, 1, 1)
            out = torch.stack([(f * fl).sum(), (f * cx * fl).sum(), (f * cy * fl).sum()])
        else:
            out = torch.empty(3, dtype=torch.float64, device=own.device)
            _lib.call("lbm_diag_fp64_noalloc", n, self.H, int(self.storage), _ptr(own), _ptr(m), _ptr(out),
                      _stream(None))
        if self.dist is not None and self.world > 1:
            self.dist.all_reduce(out, group=self.group)
        return out

    def gather(self):
        """The global state (9, H, W) on rank 0 (None on the others)."""
        import torch

        own = self.owned().contiguous()
        if self.dist is None or self.world == 1:
            return own.clone()
        parts = [torch.empty((9, self.H, self.W * (r + 1) // self.world - self.W * r // self.world),
                             dtype=own.dtype, device=own.device) for r in range(self.world)] if self.rank == 0 else None
        if self.rank == 0:
            for r in range(1, self.world):
                self.dist.recv(parts[r], src=self._peer(r), group=self.group)
            parts[0].copy_(own)
            return torch.cat(parts, dim=2)
        self.dist.send(own, dst=self._peer(0), group=self.group)
        return None


    def scatter(self, f_global=None):
        """set_state from a global state that only rank 0 holds (resume)."""
        import torch

        if self.dist is None or self.world == 1:
            return self.set_state(f_global)
        buf = torch.empty((9, self.H, self.W), dtype=self.dtype, device=self.device)
        if self.rank == 0:
            buf.copy_(f_global.to(device=self.device, dtype=self.dtype))
        self.dist.broadcast(buf, src=self._peer(0), group=self.group)
        self.set_state(buf)

    def save(self, path: str, mask_global, extra=None):
        """Checkpoint of the global state, written by rank 0."""
        from . import checkpoint
        from . import solver as SV

        g = self.gather()
        if self.rank == 0:
            p = SV.default_params(self.W, self.H, **self.global_params)
            checkpoint.save(path, g, mask_global, storage=self.storage, step=self.steps_done, params=p,
                            extra=dict(extra or {}, ranks=self.world, T=self.T, halo=self.halo))
        if self.dist is not None and self.world > 1:
            self.dist.barrier(group=self.group)

    def load(self, path: str):
        """Resume from a checkpoint (any number of ranks wrote it): rank 0 reads, all ranks take their slab."""
        from . import checkpoint

        f = None
        step = 0
        if self.rank == 0:
            f, _, hdr = checkpoint.load(path, device=self.device)
            step = int(hdr["step"])
        self.scatter(f)
        if self.dist is not None and self.world > 1:
            import torch

            t = torch.tensor([step], dtype=torch.int64, device=self.device)
            self.dist.broadcast(t, src=self._peer(0), group=self.group)
            step = int(t.item())
        self.steps_done = step


def _ptr(t):
    from . import _ptr as p

    return p(t)


def _stream(s):
    from . import _stream as st

    return st(s)
