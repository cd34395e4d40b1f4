"""CPU check of the tcgen05 convolution's data layout: the tap / channel
indexing the kernel performs (line (dz, dy), then dx, then 16-channel K
steps over the packed weights) reproduces torch's conv3d."""
import numpy as np
import torch
import torch.nn.functional as F

from hrdayapy_b200.convref import flip_transpose, pack_weights


def emulate(x, wp, cin, cout):
    """x (D, H, W, cin); wp packed (27, cin/8, cout, 8)."""
    D, H, W, _ = x.shape
    G = cin // 8
    xp = np.zeros((D + 2, H + 2, W + 2, cin))
    xp[1:-1, 1:-1, 1:-1] = x
    y = np.zeros((D, H, W, cout))
    for s in range(9):
        dz, dy = s // 3 - 1, s % 3 - 1
        tap0 = 9 * (dz + 1) + 3 * (dy + 1)
        line = xp[1 + dz:1 + dz + D, 1 + dy:1 + dy + H]          # (D, H, W+2, cin)
        for dx in range(3):                                       # smem row shift dx*16 bytes
            A = line[:, :, dx:dx + W, :]                          # voxel w reads w + dx - 1
            for k in range(cin // 16):
                for half in range(2):
                    g = 2 * k + half
                    Bk = wp[tap0 + dx, g]                         # (cout, 8)
                    y += A[..., 8 * g:8 * g + 8] @ Bk.T
    return y


def test_emulated_kernel_matches_conv3d():
    rng = np.random.default_rng(0)
    for cin, cout in ((16, 16), (32, 48), (48, 16)):
        x = rng.normal(size=(3, 4, 5, cin))
        w = rng.normal(size=(cout, cin, 3, 3, 3))
        ref = F.conv3d(torch.tensor(x).permute(3, 0, 1, 2)[None], torch.tensor(w), padding=1)
        ref = ref[0].permute(1, 2, 3, 0).numpy()
        y = emulate(x, pack_weights(w), cin, cout)
        np.testing.assert_allclose(y, ref, rtol=1e-10, atol=1e-10)


def test_flip_transpose_is_data_gradient():
    rng = np.random.default_rng(1)
    cin, cout = 16, 32
    x = torch.tensor(rng.normal(size=(1, cin, 3, 4, 5)), requires_grad=True)
    w = torch.tensor(rng.normal(size=(cout, cin, 3, 3, 3)))
    gy = torch.tensor(rng.normal(size=(1, cout, 3, 4, 5)))
    (F.conv3d(x, w, padding=1) * gy).sum().backward()
    dx = F.conv3d(gy, torch.tensor(flip_transpose(w.numpy())), padding=1)
    np.testing.assert_allclose(dx.numpy(), x.grad.numpy(), rtol=1e-10, atol=1e-10)
