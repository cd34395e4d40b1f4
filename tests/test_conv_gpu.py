"""tcgen05 3x3x3 convolution against torch.nn.functional.conv3d on the CPU
(FP32 arithmetic on the same BF16-rounded inputs).  Tolerance: the kernel
accumulates in FP32 and rounds the output to BF16 (relative 2^-8)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(D, H, W, cin, cout, epi, seed=0):
    import torch
    import torch.nn.functional as F
    from hrdayapy_b200 import _lib
    from hrdayapy_b200.convref import pack_weights
    g = torch.Generator().manual_seed(seed)
    x = torch.randn(D, H, W, cin, generator=g).to(torch.bfloat16)
    w = (torch.randn(cout, cin, 3, 3, 3, generator=g) / np.sqrt(27 * cin)).to(torch.bfloat16)
    b = torch.randn(cout, generator=g) * 0.1
    mask = torch.randn(D, H, W, cout, generator=g).to(torch.bfloat16)
    ref = F.conv3d(x.float().permute(3, 0, 1, 2)[None], w.float(), padding=1)[0].permute(1, 2, 3, 0)
    if epi == 0:
        ref = torch.relu(ref + b)
    elif epi == 1:
        ref = ref + b
    elif epi == 2:
        ref = ref * (mask.float() > 0)
    elif epi == 3:
        ref = ref[..., :1] + b[0]
    dev = torch.device("cuda")
    xd = x.to(dev).contiguous()
    wp = torch.from_numpy(pack_weights(w.float().numpy())).to(torch.bfloat16).to(dev).contiguous()
    bd = b.to(dev).contiguous()
    md = mask.to(dev).contiguous()
    yd = (torch.empty(D, H, W, dtype=torch.float32, device=dev) if epi == 3 else
          torch.empty(D, H, W, cout, dtype=torch.bfloat16, device=dev))
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    L = _lib.lib()
    st = L.hp_conv3_forward(C.c_void_p(xd.data_ptr()), C.c_void_p(wp.data_ptr()),
                            C.c_void_p(bd.data_ptr()), C.c_void_p(yd.data_ptr()),
                            C.c_void_p(md.data_ptr()), D, H, W, cin, cout, epi,
                            C.c_void_p(err.data_ptr()), None)
    _lib.check(st, "hp_conv3_forward")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    y = yd.float().cpu()
    if epi == 3:
        y = y[..., None]
    return y, ref


# (16, 16), (16, 32), (48, 16), (32, 32) run row-blocked CTAs, (64, 32),
# (64, 64), (96, 32), (32, 96) the persistent warp-specialised kernel, the
# others one line per CTA; H = 5 leaves a partial block of output lines
@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32),
                                      (48, 16), (64, 32), (32, 96)])
def test_conv_forward(cin, cout):
    y, ref = _run(3, 5, 256, cin, cout, epi=1)
    scale = ref.abs().max().item()
    assert (y - ref).abs().max().item() <= 1e-2 * scale, ((y - ref).abs().max().item(), scale)


@pytest.mark.parametrize("epi", [0, 2, 3])
def test_conv_epilogues(epi):
    y, ref = _run(2, 3, 128, 32, 16, epi=epi, seed=1)
    scale = max(ref.abs().max().item(), 1e-6)
    assert (y - ref).abs().max().item() <= 1e-2 * scale


@pytest.mark.parametrize("epi", [0, 2])
def test_persistent_kernel_epilogues(epi):
    """The persistent kernel's epilogue warps (ReLU, ReLU-backward mask) on
    more tiles than CTAs (the tile loop and both accumulator sets)."""
    y, ref = _run(4, 9, 384, 64, 64, epi=epi, seed=2)
    scale = max(ref.abs().max().item(), 1e-6)
    assert (y - ref).abs().max().item() <= 1e-2 * scale
