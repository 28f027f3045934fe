"""TEST INFRASTRUCTURE ONLY: FP64 NumPy restatement of the learned-guess network (forward and
backward) used to check the device kernels' outputs and gradients.

Architecture: four 3x3x3 convolutions with zero padding, channels 5 -> 32 -> 32 -> 32 -> 2, ReLU
between layers, mean-squared-error loss over both outputs. Parameter layout: per layer
W[27][Cout_pad][Cin_pad] then b[Cout_pad], Cin_pad = (16, 32, 32, 32), Cout_pad = (32, 32, 32, 8);
tap = 9 (dz+1) + 3 (dy+1) + (dx+1) addresses the neighbour (z+dz, y+dy, x+dx).
"""
import numpy as np

CIN = (16, 32, 32, 32)
COUT = (32, 32, 32, 8)


def unpack(params):
    out, off = [], 0
    for ci, co in zip(CIN, COUT):
        W = params[off:off + 27 * co * ci].reshape(27, co, ci).astype(np.float64)
        off += 27 * co * ci
        b = params[off:off + co].astype(np.float64)
        off += co
        out.append((W, b))
    return out


def _shifts(x):
    B, D, H, W, C = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    for tap in range(27):
        dz, dy, dx = tap // 9, (tap // 3) % 3, tap % 3
        yield tap, xp[:, dz:dz + D, dy:dy + H, dx:dx + W, :]


def conv(x, W, b):
    out = np.broadcast_to(b, x.shape[:4] + (W.shape[1],)).copy()
    for tap, xs in _shifts(x):
        out += xs @ W[tap].T
    return out


def forward(params, feats):
    """feats [B, D, H, W, 5] -> outputs [B, D, H, W, 2] and the cache for backward."""
    layers = unpack(params)
    x = np.zeros(feats.shape[:4] + (16,))
    x[..., :5] = feats
    cache = []
    for l, (W, b) in enumerate(layers):
        z = conv(x, W, b)
        cache.append((x, z))
        x = np.maximum(z, 0.0) if l < 3 else z
    return x[..., :2], cache


def loss_and_grads(params, feats, targets):
    y, cache = forward(params, feats)
    n = y.size
    loss = float(np.sum((y - targets) ** 2) / n)
    layers = unpack(params)
    grads = []
    dz = np.zeros(cache[-1][1].shape)
    dz[..., :2] = 2.0 * (y - targets) / n
    for l in range(3, -1, -1):
        x, z = cache[l]
        W, b = layers[l]
        dW = np.zeros_like(W)
        for tap, xs in _shifts(x):
            dW[tap] = np.einsum("bzyxo,bzyxi->oi", dz, xs)
        db = dz.sum(axis=(0, 1, 2, 3))
        grads.append((dW, db))
        if l == 0:
            break
        # input gradient: transposed convolution, then the ReLU of the layer below
        B, D, H, Wd, _ = x.shape
        dxp = np.zeros((B, D + 2, H + 2, Wd + 2, x.shape[-1]))
        for tap in range(27):
            kz, ky, kx = tap // 9, (tap // 3) % 3, tap % 3
            dxp[:, kz:kz + D, ky:ky + H, kx:kx + Wd, :] += dz @ W[tap]
        dx = dxp[:, 1:-1, 1:-1, 1:-1, :]
        dz = dx * (cache[l - 1][1] > 0)
    flat = []
    for dW, db in reversed(grads):
        flat.append(dW.ravel())
        flat.append(db)
    return loss, y, np.concatenate(flat)
