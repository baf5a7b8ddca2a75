"""Learned closure: training data from filtered high-resolution runs of this
solver, training on the GPU with the library's own forward / backward / Adam
kernels (lbm_mlp_*), and packing for the collision kernel (LBM_CLOSURE_MLP for a
ReLU network, LBM_CLOSURE_MLP_SILU for a SiLU one).

Model.  nu_t = out_scale * softplus(MLP(in_scale * x)), MLP 5 -> 32 -> 32 -> 1
with ReLU or SiLU on both hidden layers; the collision relaxes the stress
moments with 1 / (tau0 + 3 nu_t).
The per-cell features x (what the kernel computes from the pre-collision
populations) are the non-equilibrium stress moments n7 = Pi_xx - Pi_yy - rho
(u^2 - v^2), n8 = Pi_xy - rho u v, the energy moment ne = e - rho (3 |u|^2 - 2),
|(n7, n8)| and rho - 1.

Training data (a priori).  A high-resolution run of decaying periodic
turbulence (factor f finer, same flow in lattice units: nu_fine = f nu,
f times as many steps) is box-filtered f x f onto the coarse grid.  At every
snapshot the subgrid stress tau_ij = (u_i u_j)_bar - u_bar_i u_bar_j and the
filtered strain S_ij (spectral derivatives) give the least-squares eddy
viscosity nu* = max(0, -<tau^d : S> / (2 <S : S>)), <.> a 3 x 3 box average.
The inputs follow the Chapman-Enskog forms of the same moments in the coarse
solver: Pi^neq = -(2/3) tau_eff rho S with tau_eff = tau0 + 3 nu*, so
n7 = -(2/3) tau_eff rho (S_xx - S_yy), n8 = -(2/3) tau_eff rho S_xy, and
ne = -(2 / s_e) rho div(u).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call, lib

NI, NH = 5, 32
ACTS = {"relu": 0, "silu": 1}  # LBM_MLP_ACT_*
NPARAM = NH * NI + NH + NH * NH + NH + NH + 1
PACKED_BYTES = 4096
OW1, OB1 = 0, NH * NI
OW2 = OB1 + NH
OB2 = OW2 + NH * NH
OW3 = OB2 + NH
OB3 = OW3 + NH


def init_params(seed: int = 0) -> np.ndarray:
    """Xavier-uniform weights, zero biases (b3 so that softplus starts near 0.1)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)

    def xav(fan_in, fan_out, size):
        a = np.sqrt(6.0 / (fan_in + fan_out))
        return rng.uniform(-a, a, size).astype(np.float32)

    p[OW1:OB1] = xav(NI, NH, NH * NI)
    p[OW2:OB2] = xav(NH, NH, NH * NH)
    p[OW3:OB3] = xav(NH, 1, NH)
    p[OB3] = -2.25  # softplus(-2.25) ~ 0.1
    return p


class Mlp:
    """The closure network with FP32 master parameters on the GPU; act is the
    hidden activation ("relu" or "silu")."""

    def __init__(self, params=None, in_scale=None, out_scale: float = 1.0, seed: int = 0, act: str = "relu"):
        import torch

        if act not in ACTS:
            raise ValueError(f"unknown activation {act!r}")
        self.act = act
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        self.params = torch.from_numpy(p.copy()).cuda()
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        self.in_scale = np.ones(NI, np.float32) if in_scale is None else np.asarray(in_scale, np.float32)
        self.out_scale = float(out_scale)
        self._packed = None

    def forward(self, x):
        """softplus(MLP(x)) for x (n, 5) already scaled by in_scale (device tensors)."""
        import torch

        from . import _ptr, _stream

        y = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        call("lbm_mlp_forward_act", _ptr(self.params), ACTS[self.act], _ptr(x), _ptr(y), int(x.shape[0]),
             _stream(None))
        return y

    def loss_grad(self, x, t, w=None, workspace=None):
        import torch

        from . import _ptr, _stream

        n = int(x.shape[0])
        nbytes = int(lib().lbm_mlp_workspace_bytes(n))
        if workspace is None or workspace.numel() * 4 < nbytes:
            workspace = torch.empty((nbytes + 3) // 4, dtype=torch.float32, device=x.device)
        grad = torch.empty(NPARAM, dtype=torch.float32, device=x.device)
        loss = torch.empty(1, dtype=torch.float32, device=x.device)
        call("lbm_mlp_grad_act", _ptr(self.params), ACTS[self.act], _ptr(x), _ptr(t), _ptr(w), n, _ptr(grad),
             _ptr(loss), _ptr(workspace), C.c_size_t(nbytes), _stream(None))
        return loss, grad, workspace

    def adam(self, grad, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        from . import _ptr, _stream

        self.step += 1
        call("lbm_mlp_adam", _ptr(self.params), _ptr(grad), _ptr(self.m), _ptr(self.v), self.step, float(lr),
             float(beta1), float(beta2), float(eps), _stream(None))
        self._packed = None

    def fit(self, x_raw, nu, epochs: int = 200, batch: int = 16384, lr: float = 3e-3, seed: int = 0,
            val_frac: float = 0.1):
        """Trains on raw features (n, 5) and targets nu (n,) (numpy or torch);
        sets in_scale / out_scale from the data.  Returns (train, validation) loss
        histories (mean squared error in units of out_scale^2)."""
        import torch

        x_raw = torch.as_tensor(np.asarray(x_raw, np.float32)).cuda()
        nu = torch.as_tensor(np.asarray(nu, np.float32)).cuda()
        std = x_raw.std(dim=0).cpu().numpy()
        self.in_scale = (1.0 / np.maximum(std, 1e-12)).astype(np.float32)
        self.out_scale = float(max(nu.std().item(), 1e-12))
        xs = x_raw * torch.from_numpy(self.in_scale).cuda()
        ts = nu / self.out_scale
        g = torch.Generator(device="cpu").manual_seed(seed)
        perm = torch.randperm(xs.shape[0], generator=g).cuda()
        nval = max(1, int(val_frac * xs.shape[0]))
        xv, tv = xs[perm[:nval]].contiguous(), ts[perm[:nval]].contiguous()
        xt, tt = xs[perm[nval:]].contiguous(), ts[perm[nval:]].contiguous()
        hist_t, hist_v = [], []
        ws = None
        n = xt.shape[0]
        for ep in range(epochs):
            order = torch.randperm(n, generator=g).cuda()
            tot = 0.0
            nb = 0
            for b0 in range(0, n, batch):
                idx = order[b0:b0 + batch]
                loss, grad, ws = self.loss_grad(xt[idx].contiguous(), tt[idx].contiguous(), workspace=ws)
                self.adam(grad, lr=lr * (0.5 * (1 + np.cos(np.pi * ep / epochs))))
                tot += float(loss.item())
                nb += 1
            hist_t.append(tot / max(nb, 1))
            lv, _, ws = self.loss_grad(xv, tv, workspace=ws)
            hist_v.append(float(lv.item()))
        return hist_t, hist_v

    def predict(self, x_raw):
        """nu_t for raw features (FP32 master weights)."""
        import torch

        xs = torch.as_tensor(np.asarray(x_raw, np.float32)).cuda() * torch.from_numpy(self.in_scale).cuda()
        return self.forward(xs.contiguous()) * self.out_scale

    def packed(self):
        """Device buffer (LBM_MLP_PACKED_BYTES) for lbm_params.mlp."""
        import torch

        from . import _ptr, _stream

        if self._packed is None:
            buf = torch.zeros(PACKED_BYTES // 4, dtype=torch.float32, device="cuda")
            sc = torch.from_numpy(self.in_scale).cuda()
            call("lbm_mlp_pack_act", _ptr(self.params), ACTS[self.act], _ptr(sc), float(self.out_scale), _ptr(buf),
                 _stream(None))
            self._packed = buf
        return self._packed

    @property
    def closure(self) -> int:
        """The lbm_params closure kind that runs this network."""
        from . import solver as SV

        return SV.CLOSURE_MLP_SILU if self.act == "silu" else SV.CLOSURE_MLP

    def state(self) -> dict:
        return {"params": self.params.cpu().numpy().tolist(), "in_scale": self.in_scale.tolist(),
                "out_scale": self.out_scale, "act": self.act}

    @classmethod
    def from_state(cls, st: dict) -> "Mlp":
        return cls(params=np.array(st["params"], np.float32), in_scale=st["in_scale"], out_scale=st["out_scale"],
                   act=st.get("act", "relu"))


# ---------------------------------------------------------------------------
# training data from filtered high-resolution runs
# ---------------------------------------------------------------------------
def _deriv(a, axis):
    N = a.shape[axis]
    k = np.fft.fftfreq(N, d=1.0 / N) * 2.0 * np.pi / N
    shape = [1, 1]
    shape[axis] = N
    return np.real(np.fft.ifft(1j * k.reshape(shape) * np.fft.fft(a, axis=axis), axis=axis))


def strain(ux, uy):
    """S_xx, S_yy, S_xy of a periodic field (spectral derivatives, lattice units)."""
    dux_dx, dux_dy = _deriv(ux, 1), _deriv(ux, 0)
    duy_dx, duy_dy = _deriv(uy, 1), _deriv(uy, 0)
    return dux_dx, duy_dy, 0.5 * (dux_dy + duy_dx)


def _box3(a):
    return sum(np.roll(np.roll(a, i, 0), j, 1) for i in (-1, 0, 1) for j in (-1, 0, 1)) / 9.0


def targets_and_features(u_f, v_f, rho_f, factor: int, tau0: float, s_e: float, nu_max: float = 0.05):
    """Coarse features (n, 5) and least-squares eddy viscosities nu* (n,) from one
    fine snapshot (fields (N f) x (N f))."""
    from .spectral import box_filter

    ub, vb, rb = box_filter(u_f, factor), box_filter(v_f, factor), box_filter(rho_f, factor)
    tuu = box_filter(u_f * u_f, factor) - ub * ub
    tvv = box_filter(v_f * v_f, factor) - vb * vb
    tuv = box_filter(u_f * v_f, factor) - ub * vb
    sxx, syy, sxy = strain(ub, vb)
    tr = 0.5 * (tuu + tvv)
    num = (tuu - tr) * sxx + (tvv - tr) * syy + 2.0 * tuv * sxy  # tau^d : S
    den = sxx * sxx + syy * syy + 2.0 * sxy * sxy  # S : S
    nu = np.clip(-_box3(num) / (2.0 * np.maximum(_box3(den), 1e-20)), 0.0, nu_max)
    teff = tau0 + 3.0 * nu
    n7 = -(2.0 / 3.0) * teff * rb * (sxx - syy)
    n8 = -(2.0 / 3.0) * teff * rb * sxy
    ne = -(2.0 / s_e) * rb * (sxx + syy)
    x = np.stack([n7, n8, ne, np.hypot(n7, n8), rb - 1.0], axis=-1).reshape(-1, 5)
    return x.astype(np.float32), nu.reshape(-1).astype(np.float32)


def smagorinsky_nu(x, cs: float, tau0: float):
    """The Smagorinsky eddy viscosity of the same features (the reference's
    tau_eff = (tau0 + sqrt(tau0^2 + 18 Cs^2 Q / rho)) / 2, Q = |(n7, n8)|)."""
    x = np.asarray(x, np.float64)
    q, rho = x[:, 3], 1.0 + x[:, 4]
    teff = 0.5 * (tau0 + np.sqrt(tau0 * tau0 + 18.0 * cs * cs * q / rho))
    return (teff - tau0) / 3.0


# ---------------------------------------------------------------------------
# the decaying-turbulence judge and the a-posteriori comparison
# ---------------------------------------------------------------------------
def _run_periodic(N, f0, mask, n_steps, snap_every, T=2, on_snap=None, timing=None, **params):
    """Periodic N x N run through the slab layer (one rank, so that the register
    wavefront kernel applies); returns u, v, rho every snap_every steps (incl. 0),
    or on_snap(u, v, rho) of each when given.  `timing`, a dict, receives the
    device milliseconds of the time stepping (CUDA events around the runs)."""
    import torch

    from . import solver as SV
    from .slab import SlabSolver

    # halo >= T with N + 2 halo a multiple of 16 (TMA row pitch of the mask)
    halo = T
    while (N + 2 * halo) % 16:
        halo += 1
    S = SlabSolver(N, N, mask, T=T, halo=halo, bc_left=SV.BC_PERIODIC, bc_right=SV.BC_PERIODIC,
                   bc_y=SV.BC_PERIODIC, **params)
    S.set_state(torch.as_tensor(f0))
    snaps = []

    def macros():
        f = S.gather().double()
        if S.storage != SV.STORE_F32:
            w = torch.tensor([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, dtype=torch.float64, device=f.device)
            f = f + w[:, None, None]
        cx = torch.tensor([0, 1, 0, -1, 0, 1, -1, -1, 1], dtype=torch.float64, device=f.device)[:, None, None]
        cy = torch.tensor([0, 0, 1, 0, -1, 1, 1, -1, -1], dtype=torch.float64, device=f.device)[:, None, None]
        r = f.sum(0)
        return ((f * cx).sum(0) / r).cpu().numpy(), ((f * cy).sum(0) / r).cpu().numpy(), r.cpu().numpy()

    keep = on_snap if on_snap is not None else (lambda *a: a)
    snaps.append(keep(*macros()))
    done, ms = 0, 0.0
    while done < n_steps:
        k = min(snap_every, n_steps - done)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        S.run(k)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        done += k
        snaps.append(keep(*macros()))
    if timing is not None:
        timing["ms"] = ms
        timing["cells"] = N * N
        timing["steps"] = n_steps
    return snaps


def filtered_judge(N: int, factor: int = 4, k0: float = 4.0, u_rms: float = 0.1 * 0.5773502691896258,
                   nu: float = 5e-4, n_steps: int = 600, snap_every: int = 100, seed: int = 0, fine_cs: float = 0.0,
                   balanced: bool = False, rates=(1.1, 1.1, 1.1)):
    """Runs the factor-finer decaying turbulence (MRT, nu_fine = factor nu,
    factor n_steps steps) and returns its snapshots filtered onto N x N, the
    coarse initial state, and a-priori training data (features, nu*) per snapshot.
    balanced: start from the pressure-balanced density (spectral.balanced_density)
    on both grids instead of rho = 1.  rates: the MRT ghost-moment rates
    (s_e, s_eps, s_q) of both grids' solvers."""
    import torch

    from . import solver as SV
    from .init import equilibrium
    from .spectral import balanced_density, box_filter, random_phase_velocity

    Nf = N * factor
    ux, uy = random_phase_velocity(Nf, k0, u_rms, seed)
    rho_f = balanced_density(ux, uy) if balanced else np.ones((Nf, Nf))
    f0 = equilibrium(rho_f, ux, uy, dtype=np.float32)
    nu_f = factor * nu
    tau_f = 3.0 * nu_f + 0.5
    mask = torch.zeros((Nf, Nf), dtype=torch.uint8)
    closure = dict(closure=SV.CLOSURE_SMAG, cs_smag=fine_cs) if fine_cs > 0 else dict(closure=SV.CLOSURE_NONE)
    tau0 = 3.0 * nu + 0.5

    def reduce(u, v, r):  # filter each fine snapshot at once (a 4096^2 one is 400 MB)
        if not (np.isfinite(u).all() and np.isfinite(v).all()):
            raise FloatingPointError("the high-resolution run became unstable; raise its viscosity or Smagorinsky "
                                     "constant")
        return (box_filter(u, factor), box_filter(v, factor)), targets_and_features(u, v, r, factor, tau0=tau0,
                                                                                      s_e=rates[0])

    timing = {}
    red = _run_periodic(Nf, f0, mask, factor * n_steps, factor * snap_every, on_snap=reduce, timing=timing,
                        s_nu=1.0 / tau_f, ref_clamps=0, s_e=rates[0], s_eps=rates[1], s_q=rates[2], **closure)
    judge = [j for j, _ in red]
    data = [d for _, d in red]
    ub, vb = box_filter(ux, factor), box_filter(uy, factor)
    fc = equilibrium(box_filter(rho_f, factor), ub, vb, dtype=np.float32)
    return {"judge": judge, "data": data, "coarse_f0": fc, "tau0": tau0, "N": N, "factor": factor,
            "snap_every": snap_every, "n_steps": n_steps, "fine_timing": timing, "rates": tuple(rates)}


def velocity_error(snaps, judge):
    """Relative L2 velocity error of each snapshot against the judge."""
    out = []
    for (u, v, _), (uj, vj) in zip(snaps, judge):
        num = np.sqrt(np.sum((u - uj) ** 2 + (v - vj) ** 2))
        den = np.sqrt(np.sum(uj ** 2 + vj ** 2))
        out.append(float(num / den))
    return out


def spectrum_error(snaps, judge, rel_floor: float | None = None):
    """L2 distance of log10 energy spectra (shells 1 .. N/2) to the judge's, per
    snapshot; with rel_floor, only over the shells where the judge's energy is at
    least rel_floor times its largest shell (leaving out shells at round-off level)."""
    from .spectral import energy_spectrum

    out = []
    for (u, v, _), (uj, vj) in zip(snaps, judge):
        _, e = energy_spectrum(u, v)
        _, ej = energy_spectrum(uj, vj)
        a, b = np.log10(np.maximum(e[1:], 1e-30)), np.log10(np.maximum(ej[1:], 1e-30))
        if rel_floor is not None:
            keep = ej[1:] >= rel_floor * ej[1:].max()
            a, b = a[keep], b[keep]
        out.append(float(np.sqrt(np.mean((a - b) ** 2))))
    return out


def compare_closures(J, net, cs: float = 0.1, storage: int = 0, T: int = 2, timings=None,
                     spectrum_floor: float | None = None):
    """Coarse runs from the filtered initial state with no closure, Smagorinsky
    (Cs) and the network(s); relative L2 velocity error and log-spectrum error
    against the judge per snapshot, for each: {name: (l2, spectrum)}.  `net` is
    one Mlp (named "mlp") or a dict {name: Mlp}.  `timings`, a dict, receives
    each run's device time ({name: timing}); spectrum_floor is
    spectrum_error's rel_floor."""
    import torch

    from . import solver as SV

    N = J["N"]
    mask = torch.zeros((N, N), dtype=torch.uint8)
    se, seps, sq = J.get("rates", (1.1, 1.1, 1.1))
    base = dict(s_nu=1.0 / J["tau0"], ref_clamps=0, storage=storage, s_e=se, s_eps=seps, s_q=sq)
    nets = net if isinstance(net, dict) else {"mlp": net}
    runs = [("none", dict(closure=SV.CLOSURE_NONE)), ("smagorinsky", dict(closure=SV.CLOSURE_SMAG, cs_smag=cs))]
    runs += [(name, dict(closure=n.closure, mlp=n.packed().data_ptr())) for name, n in nets.items()]
    res = {}
    for name, extra in runs:
        f0 = J["coarse_f0"]
        if storage != SV.STORE_F32:
            f0 = f0 - np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, np.float32)[:, None, None]
            f0 = torch.from_numpy(f0).to(torch.float16 if storage == SV.STORE_F16DEV else torch.bfloat16)
        tm = {}
        snaps = _run_periodic(N, f0, mask, J["n_steps"], J["snap_every"], T=T, timing=tm, **base, **extra)
        res[name] = (velocity_error(snaps, J["judge"]), spectrum_error(snaps, J["judge"], spectrum_floor))
        if timings is not None:
            timings[name] = tm
    return res


def a_priori(J, train_snaps, test_snaps, epochs: int = 120, seed: int = 0, cs: float = 0.1, act: str = "relu"):
    """Trains a network (hidden activation act) on the a-priori data of
    train_snaps and returns it with the mean squared eddy-viscosity error on
    test_snaps of the network, of Smagorinsky (Cs) and of no closure (nu_t = 0)."""
    x = np.concatenate([J["data"][i][0] for i in train_snaps])
    y = np.concatenate([J["data"][i][1] for i in train_snaps])
    xt = np.concatenate([J["data"][i][0] for i in test_snaps])
    yt = np.concatenate([J["data"][i][1] for i in test_snaps])
    net = Mlp(seed=seed, act=act)
    net.fit(x, y, epochs=epochs, batch=8192, lr=3e-3, seed=seed)
    pm = net.predict(xt).cpu().numpy()
    ps = smagorinsky_nu(xt, cs, J["tau0"])
    return net, {"mlp": float(np.mean((pm - yt) ** 2)), "smagorinsky": float(np.mean((ps - yt) ** 2)),
                 "none": float(np.mean(yt ** 2))}
