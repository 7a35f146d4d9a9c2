"""CPU restatement of the learned predictor's network (TEST INFRASTRUCTURE ONLY).

The network has no counterpart in the reference (QuickPIC starts each slice's B
passes from the previous slice's B, source/simulation_class.f03:676); this file
restates the engine's network so that its tensor-core kernels can be checked:

* 5 layers of 3x3 convolutions, stride 1, zero padding; ReLU after layers 1-4;
  layer 5 linear, 2 of its 16 output channels used;
* parameters per layer: W[9][cin][cout] (tap = 3 dy + dx for the input offset
  (dy - 1, dx - 1)), then bias[cout]; cin = 16, 32, 32, 32, 32 and
  cout = 32, 32, 32, 32, 16;
* loss = mean over pixels and the 2 outputs of (y - t)^2.

With ``bf16=True`` the arithmetic rounds where the engine's kernels round:
inputs, weights, the ReLU outputs and the output gradient to bfloat16
(round to nearest even), products summed in float64 (the tensor cores sum in
FP32).  With ``bf16=False`` everything is float64, for finite-difference checks.
"""
import numpy as np

CIN = (16, 32, 32, 32, 32)
COUT = (32, 32, 32, 32, 16)
NOUT = 2


def layer_sizes():
    return [9 * ci * co + co for ci, co in zip(CIN, COUT)]


def num_params():
    return sum(layer_sizes())


def unpack(p):
    """[(W[9][cin][cout], b[cout]) for each layer] from the flat parameters."""
    out, o = [], 0
    for ci, co in zip(CIN, COUT):
        w = np.asarray(p[o:o + 9 * ci * co], dtype=np.float64).reshape(9, ci, co)
        o += 9 * ci * co
        b = np.asarray(p[o:o + co], dtype=np.float64)
        o += co
        out.append((w, b))
    return out


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _shifts(x):
    """The 9 taps of x[n][c][h][w]: x at (y + dy - 1, x + dx - 1), zero outside."""
    n, c, h, w = x.shape
    xp = np.zeros((n, c, h + 2, w + 2), dtype=np.float64)
    xp[:, :, 1:-1, 1:-1] = x
    return [xp[:, :, dy:dy + h, dx:dx + w] for dy in range(3) for dx in range(3)]


def conv(x, w, b=None):
    out = None
    for t, xs in enumerate(_shifts(x)):
        v = np.einsum("nchw,cd->ndhw", xs, w[t], optimize=True)
        out = v if out is None else out + v
    if b is not None:
        out = out + b[None, :, None, None]
    return out


def conv_t(dy, w):
    """Gradient of conv with respect to its input: sum over taps and outputs of
    dy at (y - dy_t + 1, x - dx_t + 1) times W[t]."""
    n, co, h, ww = dy.shape
    dp = np.zeros((n, co, h + 2, ww + 2), dtype=np.float64)
    dp[:, :, 1:-1, 1:-1] = dy
    out = None
    for t in range(9):
        ty, tx = divmod(t, 3)
        ds = dp[:, :, 2 - ty:2 - ty + h, 2 - tx:2 - tx + ww]
        v = np.einsum("ndhw,cd->nchw", ds, w[t], optimize=True)
        out = v if out is None else out + v
    return out


def wgrad(x, dy):
    """dW[t][cin][cout] = sum over pixels of x at the tap's offset times dy."""
    return np.stack([np.einsum("nchw,ndhw->cd", xs, dy, optimize=True) for xs in _shifts(x)])


def forward(p, x, bf16_rounding=True):
    """(output y[n][2][h][w], the layer inputs) of the network."""
    r = bf16 if bf16_rounding else (lambda v: np.asarray(v, dtype=np.float64))
    layers = [(r(w), b) for w, b in unpack(p)]
    a = r(x)
    acts = [a]
    for l, (w, b) in enumerate(layers):
        z = conv(a, w, b)
        if l < len(layers) - 1:
            a = r(np.maximum(z, 0.0))
            acts.append(a)
        else:
            y = z[:, :NOUT]
    return y, acts, layers


def loss_grad(p, x, t, bf16_rounding=True):
    """(loss, flat gradient) of the mean squared error of the 2 outputs."""
    r = bf16 if bf16_rounding else (lambda v: np.asarray(v, dtype=np.float64))
    y, acts, layers = forward(p, x, bf16_rounding)
    n = y.size
    e = y - np.asarray(t, dtype=np.float64)
    loss = float(np.sum(e * e) / n)
    dy = np.zeros((y.shape[0], COUT[-1]) + y.shape[2:], dtype=np.float64)
    dy[:, :NOUT] = r(2.0 * e / n)
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        w, _ = layers[l]
        gw = wgrad(acts[l], dy)
        gb = dy.sum(axis=(0, 2, 3))
        grads.append((gw, gb))
        if l == 0:
            break
        dx = conv_t(dy, w)
        dy = r(np.where(acts[l] > 0.0, dx, 0.0))
    grads.reverse()
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat
