"""FP64 NumPy restatement of the surrogate network's forward pass, loss and
gradient (layout of hams-mrel_b200/csrc/surrogate.h).

TEST INFRASTRUCTURE ONLY: the checker of the library's training kernels
(hams_surrogate_grad) and FP32 evaluation (hams_surrogate_eval).  The
network has no counterpart in the reference.
"""
import numpy as np

IN, OUT, WIDTH, HIDDEN = 4, 3, 128, 4
LAYERS = HIDDEN + 1


def dims(l):
    return (IN if l == 0 else WIDTH), (OUT if l == LAYERS - 1 else WIDTH)


def unpack(p):
    """[(W (out x in), b)] per layer and the output (mean, scale)."""
    p = np.asarray(p, dtype=np.float64)
    off, layers = 0, []
    for l in range(LAYERS):
        fi, fo = dims(l)
        W = p[off:off + fi * fo].reshape(fi, fo).T
        off += fi * fo
        layers.append((W, p[off:off + fo]))
        off += fo
    return layers, p[off:off + OUT], p[off + OUT:off + 2 * OUT]


def count():
    return sum(dims(l)[0] * dims(l)[1] + dims(l)[1] for l in range(LAYERS)) + 2 * OUT


def silu(z):
    return z / (1.0 + np.exp(-z))


def forward(p, feats):
    """Normalised outputs (3, n) for features (4, n), with the layer inputs."""
    layers, _, _ = unpack(p)
    h, zs, hs = np.asarray(feats, dtype=np.float64), [], []
    for l, (W, b) in enumerate(layers):
        hs.append(h)
        z = W @ h + b[:, None]
        zs.append(z)
        h = silu(z) if l < LAYERS - 1 else z
    return h, zs, hs


def loss_grad(p, feats, targ):
    """Mean squared error over all outputs and its gradient (parameter layout)."""
    y, zs, hs = forward(p, feats)
    n = y.size
    d = y - targ
    loss = float(np.sum(d * d) / n)
    dz = 2.0 * d / n
    grads = [None] * LAYERS
    for l in range(LAYERS - 1, -1, -1):
        W, _ = unpack(p)[0][l]
        grads[l] = (dz @ hs[l].T, dz.sum(axis=1))
        if l:
            dh = W.T @ dz
            s = 1.0 / (1.0 + np.exp(-zs[l - 1]))
            dz = dh * s * (1.0 + zs[l - 1] * (1.0 - s))
    g = np.zeros(count())
    off = 0
    for l in range(LAYERS):
        gW, gb = grads[l]
        fi, fo = dims(l)
        g[off:off + fi * fo] = gW.T.reshape(-1)
        off += fi * fo
        g[off:off + fo] = gb
        off += fo
    return loss, g
