"""The step's FP32 device atan2 (``vatan2``: the Abramowitz & Stegun 4.4.49 minimax polynomial for atan on
[0, 1] with the quadrant fix-up, used by the bending term in place of ``atan2f``) against the CUDA library's
``atan2f`` (torch.atan2 on the device) over a grid of (y, x): all four quadrants, both axes, the diagonals,
ratios |y/x| from 1e-30 to 1e30 and magnitudes from 1e-30 to 1e30.

Bound: |vatan2 - atan2f| <= 5e-7 rad everywhere, and <= 1e-6 |atan2f| where 1e-30 <= |atan2f| < 1e-3 (small
angles keep their relative accuracy down to where the ratio |y/x| leaves the normal FP32 range). The polynomial's own error is 4e-8; FP32 evaluation, the fast division of the
ratio (2 ulp) and the final subtraction from pi (half an ulp of pi, 1.2e-7) make up the rest. One documented
difference: x = -0.0 is taken as +0.0 (atan2f(+-0, -0) = +-pi, vatan2 gives +-0)."""

import ctypes as C

import numpy as np
import pytest
import torch

from newton_chysx_b200 import _lib

pytestmark = pytest.mark.gpu


def _vatan2(y: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
    out = torch.empty_like(y)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _lib.load().vbd_eval_atan2(y.numel(), C.c_void_p(y.data_ptr()), C.c_void_p(x.data_ptr()),
                                    C.c_void_p(out.data_ptr()), stream)  # fmt: skip
    _lib.check(rc, "vbd_eval_atan2")
    return out


def _grid():
    mags = np.concatenate([[0.0], 10.0 ** np.linspace(-30, 30, 121)])
    angles = np.linspace(-np.pi, np.pi, 4001)
    pts = [np.stack([np.sin(angles), np.cos(angles)], 1)]  # unit circle: every quadrant, axes at +-pi/2, 0, pi
    pts.append(np.array([[s * a, t * b] for a in mags for b in mags for s in (1, -1) for t in (1, -1)]))
    r = np.random.default_rng(0)
    pts.append(r.standard_normal((200000, 2)) * 10.0 ** r.uniform(-20, 20, (200000, 1)))
    yx = np.concatenate(pts).astype(np.float32)
    keep = ~((yx[:, 0] == 0) & (yx[:, 1] == 0) & np.signbit(yx[:, 1]))  # (+-0, -0): the documented difference
    return yx[keep, 0].copy(), yx[keep, 1].copy()


def test_device_atan2_matches_library_atan2f():
    yh, xh = _grid()
    y, x = torch.as_tensor(yh, device="cuda"), torch.as_tensor(xh, device="cuda")
    got = _vatan2(y, x)
    ref = torch.atan2(y, x)
    torch.cuda.synchronize()
    err = (got.double() - ref.double()).abs()
    assert torch.isfinite(got).all()
    assert err.max().item() <= 5e-7, (err.max().item(), yh[err.argmax().item()], xh[err.argmax().item()])
    small = (ref.abs() < 1e-3) & (ref.abs() >= 1e-30)
    rel = err[small] / ref[small].abs().double().clamp_min(1e-45)
    assert rel.max().item() <= 1e-6
    # exact values on the axes and at the origin
    axes = torch.tensor([[0.0, 1.0], [1.0, 0.0], [0.0, -1.0], [-1.0, 0.0], [0.0, 0.0], [-0.0, 1.0], [-0.0, -1.0]],
                        device="cuda")  # fmt: skip
    a = _vatan2(axes[:, 0].contiguous(), axes[:, 1].contiguous()).cpu().numpy()
    pi = np.float32(np.pi)
    assert a[0] == 0.0 and abs(a[1] - pi / 2) <= 1.2e-7 and abs(a[2] - pi) <= 2.4e-7
    assert abs(a[3] + pi / 2) <= 1.2e-7 and a[4] == 0.0 and a[5] == 0.0 and abs(a[6] + pi) <= 2.4e-7
    assert np.signbit(a[5])  # atan2(-0, 1) = -0
