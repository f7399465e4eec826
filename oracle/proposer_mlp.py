"""FP64 restatement of the step/order proposer network (test infrastructure).

The checker for the GPU training kernels (csrc/proposer.cu): the same 3-layer
tanh MLP (11 -> 64 -> 64 -> 3) over the same flat parameter layout (W1
[64][11], b1 [64], W2 [64][64], b2 [64], W3 [3][64], b3 [3]) and the same
masked mean-squared error, loss = sum(mask (out - y)^2) / sum(mask), with its
gradient by reverse-mode differentiation in float64.
"""
import numpy as np

NF, H, NO = 11, 64, 3
SHAPES = [("W1", (H, NF)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (NO, H)), ("b3", (NO,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(w):
    w = np.asarray(w, np.float64)
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = w[o:o + n].reshape(shape)
        o += n
    return out


def forward(w, x):
    p = unpack(w)
    h1 = np.tanh(x @ p["W1"].T + p["b1"])
    h2 = np.tanh(h1 @ p["W2"].T + p["b2"])
    return h2 @ p["W3"].T + p["b3"], h1, h2


def loss_and_grad(w, x, y, mask):
    x, y, mask = (np.asarray(a, np.float64) for a in (x, y, mask))
    p = unpack(w)
    out, h1, h2 = forward(w, x)
    ws = mask.sum()
    e = out - y
    loss = float((mask * e * e).sum() / ws)
    d = 2.0 * mask * e / ws
    g = {"W3": d.T @ h2, "b3": d.sum(0)}
    dz2 = (d @ p["W3"]) * (1 - h2 * h2)
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ p["W2"]) * (1 - h1 * h1)
    g["W1"] = dz1.T @ x
    g["b1"] = dz1.sum(0)
    return loss, np.concatenate([g[name].ravel() for name, _ in SHAPES])
