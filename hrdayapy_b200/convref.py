"""Weight packing for the tcgen05 convolution (csrc/conv.cu).

The kernel's B operand for tap t = 9 kz + 3 ky + kx is K-major in 8-channel
core rows: Wp[t][ci // 8][co][ci % 8].  torch's conv3d weight is
w[co][ci][kz][ky][kx] (cross-correlation, zero padding 1, spatial axes
(D, H, W) = (kz, ky, kx))."""
from __future__ import annotations

import numpy as np


def pack_weights(w: np.ndarray) -> np.ndarray:
    """w (cout, cin, 3, 3, 3) -> packed (27, cin/8, cout, 8) in the same dtype."""
    cout, cin = w.shape[:2]
    assert cin % 8 == 0
    t = np.asarray(w).reshape(cout, cin, 27)            # tap = 9 kz + 3 ky + kx
    t = t.transpose(2, 1, 0)                            # (27, cin, cout)
    t = t.reshape(27, cin // 8, 8, cout).transpose(0, 1, 3, 2)
    return np.ascontiguousarray(t)


def flip_transpose(w: np.ndarray) -> np.ndarray:
    """Weights of the data-gradient convolution: dX = conv(dY, w'), with
    w'[ci][co][kz][ky][kx] = w[co][ci][2-kz][2-ky][2-kx]."""
    return np.ascontiguousarray(np.asarray(w)[:, :, ::-1, ::-1, ::-1].transpose(1, 0, 2, 3, 4))
