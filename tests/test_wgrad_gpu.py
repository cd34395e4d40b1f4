"""Tensor-core weight / bias gradients of a 3x3x3 convolution (hp_conv3_wgrad)
against torch autograd on the CPU (FP32 arithmetic on the same BF16-rounded
inputs), for every (cin, cout) pair the learned preconditioner uses, and
bit-identical on repeated calls (fixed-order reduction, no atomics).

Tolerance: the products are BF16 x BF16 accumulated in FP32 over thousands
of voxels; 1e-3 of the largest gradient entry."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _wgrad(x, g, cin, cout):
    import torch
    from hrdayapy_b200 import _lib
    L = _lib.lib()
    D, H, W = x.shape[:3]
    dev = torch.device("cuda")
    xd = x.to(dev).contiguous()
    gd = g.to(dev).contiguous()
    nb = int(L.hp_conv3_wgrad_workspace(D, H, W, cin, cout))
    work = torch.empty(nb // 4 + 4, dtype=torch.float32, device=dev)
    gw = torch.empty(cout * cin * 27, dtype=torch.float32, device=dev)
    gb = torch.empty(cout, dtype=torch.float32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    st = L.hp_conv3_wgrad(C.c_void_p(xd.data_ptr()), C.c_void_p(gd.data_ptr()), D, H, W, cin,
                          cout, C.c_void_p(gw.data_ptr()), C.c_void_p(gb.data_ptr()),
                          C.c_void_p(work.data_ptr()), work.numel() * 4,
                          C.c_void_p(err.data_ptr()), None)
    _lib.check(st, "hp_conv3_wgrad")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return gw.cpu().reshape(cout, cin, 27).numpy(), gb.cpu().numpy()


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32),
                                      (48, 16), (16, 1)])
def test_wgrad_vs_torch_autograd(cin, cout):
    import torch
    import torch.nn.functional as F
    D, H, W = 5, 6, 128
    gen = torch.Generator().manual_seed(cin * 1000 + cout)
    coP = max(cout, 16)
    x = torch.randn(D, H, W, cin, generator=gen).to(torch.bfloat16)
    g = torch.randn(D, H, W, coP, generator=gen).to(torch.bfloat16)
    g[..., cout:] = 0
    # reference: d/dw of sum(conv3d(x, w) * g)
    w = torch.zeros(cout, cin, 3, 3, 3, requires_grad=True)
    b = torch.zeros(cout, requires_grad=True)
    y = F.conv3d(x.float().permute(3, 0, 1, 2)[None], w, b, padding=1)[0]
    (y * g[..., :cout].float().permute(3, 0, 1, 2)).sum().backward()
    ref_w = w.grad.reshape(cout, cin, 27).numpy()
    ref_b = b.grad.numpy()
    gw, gb = _wgrad(x, g, cin, cout)
    scale = np.abs(ref_w).max()
    assert np.abs(gw - ref_w).max() <= 1e-3 * scale, (np.abs(gw - ref_w).max(), scale)
    assert np.abs(gb - ref_b).max() <= 1e-3 * np.abs(ref_b).max()
    # a second call gives the same bits
    gw2, gb2 = _wgrad(x, g, cin, cout)
    np.testing.assert_array_equal(gw, gw2)
    np.testing.assert_array_equal(gb, gb2)


def test_wgrad_two_tiles_along_w():
    """W = 256: two 128-voxel tiles per line, taps across the tile seam."""
    import torch
    import torch.nn.functional as F
    cin, cout = 32, 32
    D, H, W = 3, 4, 256
    gen = torch.Generator().manual_seed(7)
    x = torch.randn(D, H, W, cin, generator=gen).to(torch.bfloat16)
    g = torch.randn(D, H, W, cout, generator=gen).to(torch.bfloat16)
    w = torch.zeros(cout, cin, 3, 3, 3, requires_grad=True)
    y = F.conv3d(x.float().permute(3, 0, 1, 2)[None], w, padding=1)[0]
    (y * g.float().permute(3, 0, 1, 2)).sum().backward()
    ref_w = w.grad.reshape(cout, cin, 27).numpy()
    gw, _ = _wgrad(x, g, cin, cout)
    assert np.abs(gw - ref_w).max() <= 1e-3 * np.abs(ref_w).max()
