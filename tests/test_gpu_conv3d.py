"""tcgen05 BF16 implicit-GEMM conv3d (forward, data gradient, weight gradient) against torch
CPU conv3d.

The reference operands are the same BF16-rounded inputs and weights promoted to float64, so
the differences come from the kernels' FP32 accumulation order and, for BF16 outputs, the
final rounding.  Bounds (max |a - b| / max |b|): FP32 forward output 1e-5, BF16 outputs
8e-3 (one BF16 rounding, 2^-8 relative), weight gradient 1e-5, bias gradient 1e-5.
Grids exercise partial x tiles (nx = 24 < 128, nx = 136 = 128 + 8), several y/z sizes and
every zero-padded face.
"""
import numpy as np
import pytest

from conftest import rel_err

PAIRS = [(16, 32), (32, 64), (64, 32), (32, 16), (16, 16), (64, 16)]
GRIDS = [(6, 5, 24), (3, 4, 136), (2, 9, 40)]


def _ref_conv(x, w, b, relu):
    import torch
    xt = x.permute(3, 0, 1, 2)[None].double()               # (1, cin, ny, nz, nx)
    y = torch.nn.functional.conv3d(xt, w.double(), b.double() if b is not None else None, padding=1)
    if relu:
        y = torch.relu(y)
    return y[0].permute(1, 2, 3, 0)


def _data(shape, cin, cout, seed):
    import torch
    g = torch.Generator().manual_seed(seed)
    ny, nz, nx = shape
    x = torch.randn((ny, nz, nx, cin), generator=g).to(torch.bfloat16)
    w = (torch.randn((27, cout, cin), generator=g) / np.sqrt(27 * cin)).float()
    b = torch.randn(cout, generator=g).float() * 0.1
    return x, w, b


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout", PAIRS)
@pytest.mark.parametrize("shape", GRIDS)
def test_forward_matches_torch(cuda, cin, cout, shape):
    import torch
    from elastic_fm_vp_vs_rho_b200 import conv3d
    x, w, b = _data(shape, cin, cout, 1)
    wb, wt = conv3d.prep_weights(w.cuda())
    assert torch.equal(wb.cpu(), w.to(torch.bfloat16))
    wq = conv3d.to_torch_weight(w.to(torch.bfloat16).float())
    for relu in (False, True):
        yb, yf = conv3d.forward(x.cuda(), wb, b.cuda(), relu=relu, out_bf16=True, out_f32=True)
        conv3d.status()
        ref = _ref_conv(x, wq, b, relu)
        assert rel_err(yf.cpu().numpy(), ref.numpy()) < 1e-5
        assert rel_err(yb.float().cpu().numpy(), ref.numpy()) < 8e-3


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout", PAIRS)
@pytest.mark.parametrize("shape", GRIDS)
def test_backward_data_matches_torch(cuda, cin, cout, shape):
    import torch
    from elastic_fm_vp_vs_rho_b200 import conv3d
    x, w, _ = _data(shape, cin, cout, 2)
    g = torch.Generator().manual_seed(5)
    dy = torch.randn(shape + (cout,), generator=g).to(torch.bfloat16)
    mask = torch.randn(shape + (cin,), generator=g).to(torch.bfloat16)
    _, wt = conv3d.prep_weights(w.cuda())
    xt = x.permute(3, 0, 1, 2)[None].double().requires_grad_(True)
    wq = conv3d.to_torch_weight(w.to(torch.bfloat16).float()).double()
    y = torch.nn.functional.conv3d(xt, wq, padding=1)
    y.backward(dy.permute(3, 0, 1, 2)[None].double())
    ref = xt.grad[0].permute(1, 2, 3, 0)
    dx = conv3d.backward_data(dy.cuda(), wt, cin)
    conv3d.status()
    assert rel_err(dx.float().cpu().numpy(), ref.numpy()) < 8e-3
    dxm = conv3d.backward_data(dy.cuda(), wt, cin, relu_mask=mask.cuda())
    refm = ref * (mask.double() > 0)
    assert rel_err(dxm.float().cpu().numpy(), refm.numpy()) < 8e-3


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout", PAIRS)
@pytest.mark.parametrize("shape", GRIDS)
def test_backward_weights_matches_torch(cuda, cin, cout, shape):
    import torch
    from elastic_fm_vp_vs_rho_b200 import conv3d
    x, w, _ = _data(shape, cin, cout, 3)
    g = torch.Generator().manual_seed(7)
    dy = torch.randn(shape + (cout,), generator=g).to(torch.bfloat16)
    xt = x.permute(3, 0, 1, 2)[None].double()
    wq = conv3d.to_torch_weight(w.float()).double().requires_grad_(True)
    bq = torch.zeros(cout, dtype=torch.float64, requires_grad=True)
    y = torch.nn.functional.conv3d(xt, wq, bq, padding=1)
    y.backward(dy.permute(3, 0, 1, 2)[None].double())
    dw, db = conv3d.backward_weights(x.cuda(), dy.cuda())
    conv3d.status()
    ref_dw = conv3d.from_torch_weight(wq.grad)
    assert rel_err(dw.cpu().numpy(), ref_dw.numpy()) < 1e-5
    assert rel_err(db.cpu().numpy(), bq.grad.numpy()) < 1e-5


def test_weight_layout_roundtrip_and_unsupported_pairs():
    """CPU: layout conversions; 64 -> 64 and odd channel counts are rejected before any
    device work."""
    import ctypes

    import torch
    from elastic_fm_vp_vs_rho_b200 import _lib, conv3d
    w = torch.randn(27, 32, 16)
    assert torch.equal(conv3d.from_torch_weight(conv3d.to_torch_weight(w)), w)
    wt = conv3d.to_torch_weight(w)
    assert torch.equal(wt[5, 3, 1, 2, 0], w[9 * 1 + 3 * 2 + 0, 5, 3])
    assert conv3d.supported(16, 64) and not conv3d.supported(64, 64) and not conv3d.supported(8, 16)
    L = _lib.load()
    d = conv3d.desc((4, 4, 8), 64, 64)
    rc = L.efm_conv3d_forward(ctypes.byref(d), None, None, None, 0, None, None, None)
    assert rc == _lib.EFM_ERR_ARG
    assert L.efm_conv3d_wgrad_workspace(ctypes.byref(d)) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout", [(32, 64), (64, 16), (16, 32), (64, 32), (32, 16)])
def test_grouped_per_slab_and_swizzled_loads_agree(cuda, cin, cout):
    """The operand staging variants give identical results: one 5-D TMA copy per input row or
    one copy per 8-channel slab (all kernels), and, for the weight gradient, full-channel
    rows in the swizzled layouts (default) or 8-channel slabs without swizzle."""
    import torch
    from elastic_fm_vp_vs_rho_b200 import _lib, conv3d
    x, w, b = _data((3, 6, 140), cin, cout, 11)
    g = torch.Generator().manual_seed(12)
    dy = torch.randn((3, 6, 140, cout), generator=g).to(torch.bfloat16).cuda()
    wb, wt = conv3d.prep_weights(w.cuda())
    L = _lib.load()
    outs = []
    for grouped, sw in ((1, 1), (1, 0), (0, 0)):
        L.efm_conv3d_set_grouped_loads(grouped)
        L.efm_conv3d_set_swizzled_loads(sw)
        try:
            _, yf = conv3d.forward(x.cuda(), wb, b.cuda(), relu=True, out_bf16=False, out_f32=True)
            dx = conv3d.backward_data(dy, wt, cin, relu_mask=x.cuda())
            dw, db = conv3d.backward_weights(x.cuda(), dy)
            conv3d.status()
        finally:
            L.efm_conv3d_set_grouped_loads(1)
            L.efm_conv3d_set_swizzled_loads(1)
        outs.append((yf.cpu(), dx.cpu(), dw.cpu(), db.cpu()))
    for k in (1, 2):
        for a, c in zip(outs[0], outs[k]):
            assert torch.equal(a, c)
