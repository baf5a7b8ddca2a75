"""Oracle of the learned-closure MLP (test infrastructure only): numpy FP64
forward and backward of the 5 -> 32 -> 32 -> 1 network (ReLU or SiLU on both
hidden layers, softplus output) with the parameter layout of lbm-cuda_b200/csrc/mlp_train.cu, and
the loss L = (1/n) sum_i w_i (y_i - t_i)^2 whose gradient lbm_mlp_grad
returns.  No counterpart in the reference (the reference has no learned
closure); the restatement follows the mathematics of the network."""
import numpy as np

NI, NH = 5, 32
OW1, OB1 = 0, NH * NI
OW2 = OB1 + NH
OB2 = OW2 + NH * NH
OW3 = OB2 + NH
OB3 = OW3 + NH
NPARAM = OB3 + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OW1:OB1].reshape(NH, NI), p[OB1:OW2], p[OW2:OB2].reshape(NH, NH), p[OB2:OW3], p[OW3:OB3], p[OB3])


def _sig(a):
    return 1.0 / (1.0 + np.exp(-a))


def relu(a):
    return np.maximum(a, 0.0)


def relu_grad(a):
    return (a > 0.0).astype(np.float64)


def silu(a):
    return a * _sig(a)


def silu_grad(a):
    s = _sig(a)
    return s * (1.0 + a * (1.0 - s))


ACTS = {"relu": (relu, relu_grad), "silu": (silu, silu_grad)}


def forward(p, x, act="relu"):
    f, _ = ACTS[act]
    W1, b1, W2, b2, w3, b3 = unpack(p)
    x = np.asarray(x, np.float64)
    a1 = x @ W1.T + b1
    h1 = f(a1)
    a2 = h1 @ W2.T + b2
    h2 = f(a2)
    z = h2 @ w3 + b3
    y = np.where(z > 30, z, np.log1p(np.exp(np.minimum(z, 30))))
    return y, (x, a1, h1, a2, h2, z)


def loss_grad(p, x, t, w=None, act="relu"):
    _, fg = ACTS[act]
    y, (x, a1, h1, a2, h2, z) = forward(p, x, act)
    n = x.shape[0]
    w = np.ones(n) if w is None else np.asarray(w, np.float64)
    e = y - np.asarray(t, np.float64)
    loss = float(np.sum(w * e * e) / n)
    dz = 2.0 * w * e / n * _sig(z)
    W1, b1, W2, b2, w3, b3 = unpack(p)
    g = np.zeros(NPARAM)
    g[OW3:OB3] = dz @ h2
    g[OB3] = dz.sum()
    d2 = dz[:, None] * w3[None, :] * fg(a2)
    g[OW2:OB2] = (d2.T @ h1).ravel()
    g[OB2:OW3] = d2.sum(0)
    d1 = (d2 @ W2) * fg(a1)
    g[OW1:OB1] = (d1.T @ x).ravel()
    g[OB1:OW2] = d1.sum(0)
    return loss, g
