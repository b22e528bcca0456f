"""Oracle of the warm start's convolutions (test infrastructure: only the tests import it).  The 3x3x3 convolution
with stride 1 and zero padding 1 of channels-last volumes, and its two gradients, in float64 numpy, written from the
definition: y[n, z, y, x, co] = sum_{tap, ci} w[co, tap, ci] x[n, z + dz, y + dy, x + dx, ci] with
tap = 9 (dz + 1) + 3 (dy + 1) + (dx + 1) and x = 0 outside the volume.  The reference has no counterpart (the learned
warm start is not part of it), so this definition is the specification the tensor-core kernels are checked against.
"""
import numpy as np

TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def _shifted(x, dz, dy, dx):
    """x[n, z + dz, y + dy, x + dx, :] with zeros outside, for every (n, z, y, x)."""
    p = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    n, d, h, w, c = x.shape
    return p[:, 1 + dz:1 + dz + d, 1 + dy:1 + dy + h, 1 + dx:1 + dx + w, :]


def conv3d_forward(x, w, bias=None, relu=False):
    x = np.asarray(x, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    y = np.zeros(x.shape[:4] + (w.shape[0],))
    for t, (dz, dy, dx) in enumerate(TAPS):
        y += _shifted(x, dz, dy, dx) @ w[:, t, :].T
    if bias is not None:
        y += np.asarray(bias, dtype=np.float64)
    return np.maximum(y, 0.0) if relu else y


def conv3d_weight_grad(x, dy):
    """dL/dw[co, tap, ci] = sum over voxels of dy[..., co] x_shifted(tap)[..., ci]."""
    x = np.asarray(x, dtype=np.float64)
    dy = np.asarray(dy, dtype=np.float64)
    cout, cin = dy.shape[-1], x.shape[-1]
    g = np.zeros((cout, 27, cin))
    d2 = dy.reshape(-1, cout)
    for t, (dz, dy_, dx) in enumerate(TAPS):
        g[:, t, :] = d2.T @ _shifted(x, dz, dy_, dx).reshape(-1, cin)
    return g


def conv3d_input_grad(dy, w):
    """dL/dx[..., ci] = sum over taps and co of w[co, tap, ci] dy shifted by minus the tap's offset."""
    dy = np.asarray(dy, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    g = np.zeros(dy.shape[:4] + (w.shape[2],))
    for t, (dz, dy_, dx) in enumerate(TAPS):
        g += _shifted(dy, -dz, -dy_, -dx) @ w[:, t, :]
    return g
