"""NumPy (float64) reference of the selector network, for checking the
library's CUDA forward/backward kernels: in -> H -> H -> out, ReLU hidden
layers, parameters W1 b1 W2 b2 W3 b3 with W stored [in][out]."""
import numpy as np


def unpack(p, nin, nh, nout):
    p = np.asarray(p, np.float64)
    sizes = [nin * nh, nh, nh * nh, nh, nh * nout, nout]
    out, o = [], 0
    for s in sizes:
        out.append(p[o:o + s])
        o += s
    W1, b1, W2, b2, W3, b3 = out
    return W1.reshape(nin, nh), b1, W2.reshape(nh, nh), b2, W3.reshape(nh, nout), b3


def forward(p, x, nin, nh, nout):
    W1, b1, W2, b2, W3, b3 = unpack(p, nin, nh, nout)
    z1 = x @ W1 + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0)
    return h2 @ W3 + b3, (z1, h1, z2, h2)


def loss_and_grad(p, x, t, nin, nh, nout):
    """Masked mean squared error (NaN targets are unlabelled) and its gradient."""
    x = np.asarray(x, np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(p, nin, nh, nout)
    y, (z1, h1, z2, h2) = forward(p, x, nin, nh, nout)
    mask = np.isfinite(t)
    cnt = max(mask.sum(), 1)
    d = np.where(mask, y - np.nan_to_num(t), 0.0)
    loss = float((d * d).sum() / cnt)
    dy = 2.0 * d / cnt
    dW3 = h2.T @ dy
    db3 = dy.sum(0)
    dz2 = (dy @ W3.T) * (z2 > 0)
    dW2 = h1.T @ dz2
    db2 = dz2.sum(0)
    dz1 = (dz2 @ W2.T) * (z1 > 0)
    dW1 = x.T @ dz1
    db1 = dz1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return loss, g
