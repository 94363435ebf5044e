"""3x3x3 convolutions on the tcgen05 tensor cores (include/efm.h, efm_conv3d_*).

Thin torch-facing wrappers: volumes are channels-last BF16 CUDA tensors of shape
(ny, nz, nx, C); weights are FP32 master copies [27][cout][cin] (tap t = 9 kd + 3 kh + kw
reading (y + kd - 1, z + kh - 1, x + kw - 1)) converted to BF16 by :func:`prep_weights`.
:func:`to_torch_weight` / :func:`from_torch_weight` convert to and from the
``torch.nn.functional.conv3d`` layout [cout][cin][3][3][3] of the (1, C, ny, nz, nx) tensor.
"""
from __future__ import annotations

import ctypes

from . import _lib
from ._lib import check, stream_ptr


def _p(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def desc(shape, cin, cout):
    ny, nz, nx = shape
    return _lib.ConvDesc(nx=int(nx), ny=int(ny), nz=int(nz), cin=int(cin), cout=int(cout))


def supported(cin, cout) -> bool:
    return bool(_lib.load().efm_conv3d_supported(int(cin), int(cout)))


def to_torch_weight(w):
    """[27][cout][cin] -> [cout][cin][3][3][3]."""
    cout, cin = w.shape[1], w.shape[2]
    return w.reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2).contiguous()


def from_torch_weight(wt):
    """[cout][cin][3][3][3] -> [27][cout][cin]."""
    cout, cin = wt.shape[0], wt.shape[1]
    return wt.permute(2, 3, 4, 0, 1).reshape(27, cout, cin).contiguous()


def prep_weights(w, stream=None):
    """FP32 [27][cout][cin] CUDA tensor -> (BF16 forward weights, BF16 mirrored transpose)."""
    import torch
    _, cout, cin = w.shape
    wb = torch.empty((27, cout, cin), dtype=torch.bfloat16, device=w.device)
    wt = torch.empty((27, cin, cout), dtype=torch.bfloat16, device=w.device)
    check(_lib.load().efm_conv3d_prep_weights(cin, cout, _p(w.contiguous()), _p(wb), _p(wt),
                                              stream_ptr(stream)))
    return wb, wt


def forward(x, wb, bias=None, relu=False, out_bf16=True, out_f32=False, stream=None):
    """act(conv(x) + bias): returns (y_bf16 or None, y_f32 or None)."""
    import torch
    ny, nz, nx, cin = x.shape
    cout = wb.shape[1]
    d = desc((ny, nz, nx), cin, cout)
    yb = torch.empty((ny, nz, nx, cout), dtype=torch.bfloat16, device=x.device) if out_bf16 else None
    yf = torch.empty((ny, nz, nx, cout), dtype=torch.float32, device=x.device) if out_f32 else None
    check(_lib.load().efm_conv3d_forward(ctypes.byref(d), _p(x), _p(wb), _p(bias), int(bool(relu)),
                                         _p(yb), _p(yf), stream_ptr(stream)))
    return yb, yf


def backward_data(dy, wt, cin, relu_mask=None, stream=None):
    """conv^T(dy) (times [relu_mask > 0]) for the forward layer cin -> dy.shape[-1]."""
    import torch
    ny, nz, nx, cout = dy.shape
    d = desc((ny, nz, nx), cin, cout)
    dx = torch.empty((ny, nz, nx, cin), dtype=torch.bfloat16, device=dy.device)
    check(_lib.load().efm_conv3d_backward_data(ctypes.byref(d), _p(dy), _p(wt), _p(relu_mask),
                                               _p(dx), stream_ptr(stream)))
    return dx


class WgradWorkspace:
    """Grows on demand; one per network (the kernels of one stream share it)."""

    def __init__(self):
        self.buf = None

    def get(self, d):
        import torch
        n = int(_lib.load().efm_conv3d_wgrad_workspace(ctypes.byref(d)))
        if self.buf is None or self.buf.numel() * 4 < n:
            self.buf = torch.empty((n + 3) // 4, dtype=torch.float32, device="cuda")
        return self.buf


def backward_weights(x, dy, workspace=None, stream=None, with_bias=True):
    """(dw [27][cout][cin] fp32, db [cout] fp32 or None)."""
    import torch
    ny, nz, nx, cin = x.shape
    cout = dy.shape[-1]
    d = desc((ny, nz, nx), cin, cout)
    ws = (workspace or WgradWorkspace()).get(d)
    dw = torch.empty((27, cout, cin), dtype=torch.float32, device=x.device)
    db = torch.empty(cout, dtype=torch.float32, device=x.device) if with_bias else None
    check(_lib.load().efm_conv3d_backward_weights(ctypes.byref(d), _p(x), _p(dy), _p(dw), _p(db),
                                                  _p(ws), ws.numel() * 4, stream_ptr(stream)))
    return dw, db


def status(stream=None):
    """Raise EfmError(EFM_ERR_TIMEOUT) if a convolution kernel gave up a wait (synchronizes)."""
    check(_lib.load().efm_conv3d_status(stream_ptr(stream)))


def bench(shape=(128, 128, 256), pairs=((16, 32), (32, 64), (64, 32), (32, 16)), reps=5,
          warmup=2):
    """Device time and tensor throughput of forward / data-gradient / weight-gradient launches
    (CUDA events on the launching stream).  FLOPs per launch: 2 x 27 x cin x cout x voxels."""
    import torch
    ny, nz, nx = shape
    nvox = ny * nz * nx
    out = []
    g = torch.Generator(device="cuda").manual_seed(0)
    for cin, cout in pairs:
        x = torch.randn(shape + (cin,), device="cuda", generator=g).to(torch.bfloat16)
        dy = torch.randn(shape + (cout,), device="cuda", generator=g).to(torch.bfloat16)
        w = torch.randn((27, cout, cin), device="cuda", generator=g) * 0.05
        b = torch.zeros(cout, device="cuda")
        wb, wt = prep_weights(w)
        ws = WgradWorkspace()
        flops = 2.0 * 27 * cin * cout * nvox
        row = dict(cin=cin, cout=cout, voxels=nvox, gflop=flops / 1e9)
        cases = {
            "forward": lambda: forward(x, wb, b, relu=True),
            "backward_data": lambda: backward_data(dy, wt, cin, relu_mask=x),
            "backward_weights": lambda: backward_weights(x, dy, ws),
        }
        for name, fn in cases.items():
            for _ in range(warmup):
                fn()
            s = torch.cuda.current_stream()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(s)
            for _ in range(reps):
                fn()
            e1.record(s)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / reps
            row[name] = dict(ms=ms, tflops=flops / (ms * 1e-3) / 1e12)
        status()
        out.append(row)
    return out


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="conv3d kernel throughput")
    ap.add_argument("shape", nargs="?", default="128,128,256", help="ny,nz,nx")
    ap.add_argument("--pairs", default="16x32,32x64,64x32,32x16", help="cin x cout list")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    a = ap.parse_args()
    shp = tuple(int(v) for v in a.shape.split(","))
    prs = tuple(tuple(int(v) for v in p.split("x")) for p in a.pairs.split(","))
    for r in bench(shp, prs, reps=a.reps, warmup=a.warmup):
        print(json.dumps(r))
