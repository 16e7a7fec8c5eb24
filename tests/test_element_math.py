"""The product's element math (vbd_elements.cuh, compiled for the host) against the oracle.

The CUDA kernels evaluate the bending derivative in a closed vector form and accumulate symmetric
Hessians; this checks those formulas against the oracle's restatement of the reference on the
golden element cases, in FP64 (near machine precision) and FP32 (rounding level), without a GPU.
"""

import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import vbd_oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "hostcheck", "_build", "libelements_host.so")


@pytest.fixture(scope="module")
def hostlib():
    src = os.path.join(HERE, "hostcheck", "elements_host.cpp")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
        os.path.getmtime(src),
        os.path.getmtime(os.path.join(HERE, "..", "newton_chysx_b200", "csrc", "vbd_elements.cuh")),
        os.path.getmtime(os.path.join(HERE, "..", "newton_chysx_b200", "csrc", "vbd_math.cuh")),
    ):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
        subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-I/usr/local/cuda/include", "-o", LIB, src],
                       check=True)
    lib = C.CDLL(LIB)
    dp = C.POINTER(C.c_double)
    lib.host_membrane.argtypes = [C.c_int, C.c_int, dp, dp, dp] + [C.c_double] * 5 + [dp]
    lib.host_bending.argtypes = [C.c_int, C.c_int, dp, dp, C.c_int] + [C.c_double] * 5 + [dp]
    lib.host_contact.argtypes = [C.c_int, C.c_double, dp, dp] + [C.c_double] * 5 + [dp]
    return lib


def _p(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def _cases(golden_dir, key):
    return np.load(os.path.join(golden_dir, "elements.npz"))[key]


@pytest.mark.parametrize("prec,rtol", [(64, 1e-9), (32, 3e-4)])
def test_membrane(hostlib, golden_dir, prec, rtol):
    for r in _cases(golden_dir, "membrane"):
        X, Xp, pose = r[0:9], r[9:18], r[18:22]
        area, mu, lam, damping, dt, order = r[22:28]
        f_o, H_o = orc.element("membrane", 64, order, X, Xp, pose, area, mu, lam, damping, dt)
        out, op = _p(np.zeros(12))
        a, ap = _p(X)
        b, bp = _p(Xp)
        c, cp = _p(pose)
        hostlib.host_membrane(prec, int(order), ap, bp, cp, area, mu, lam, damping, dt, op)
        scale = max(np.abs(f_o).max(), np.abs(H_o).max())
        assert np.abs(out[:3] - f_o).max() <= rtol * scale
        assert np.abs(out[3:].reshape(3, 3) - H_o).max() <= rtol * scale


@pytest.mark.parametrize("prec,rtol", [(64, 1e-9), (32, 3e-4)])
def test_bending_closed_form(hostlib, golden_dir, prec, rtol):
    for r in _cases(golden_dir, "bending"):
        X, Xp = r[0:12], r[12:24]
        ra, rl, ke, kd, dt, order, boundary = r[24:31]
        f_o, H_o = orc.element("bending", 64, order, X, Xp, boundary, ra, rl, ke, kd, dt)
        out, op = _p(np.zeros(12))
        a, ap = _p(X)
        b, bp = _p(Xp)
        hostlib.host_bending(prec, int(order), ap, bp, int(boundary), ra, rl, ke, kd, dt, op)
        scale = max(np.abs(f_o).max(), np.abs(H_o).max(), 1e-30)
        assert np.abs(out[:3] - f_o).max() <= rtol * scale
        assert np.abs(out[3:].reshape(3, 3) - H_o).max() <= rtol * scale


@pytest.mark.parametrize("prec,rtol", [(64, 1e-9), (32, 3e-4)])
def test_contact(hostlib, golden_dir, prec, rtol):
    for r in _cases(golden_dir, "contact"):
        pen, n, rel = r[0], r[1:4], r[4:7]
        ke, kd, mu, eps, dt = r[7:12]
        f_o, H_o = orc.element("contact", 64, pen, n, rel, ke, kd, mu, eps, dt)
        out, op = _p(np.zeros(12))
        a, ap = _p(n)
        b, bp = _p(rel)
        hostlib.host_contact(prec, pen, ap, bp, ke, kd, mu, eps, dt, op)
        scale = max(np.abs(f_o).max(), np.abs(H_o).max())
        assert np.abs(out[:3] - f_o).max() <= rtol * scale
        assert np.abs(out[3:].reshape(3, 3) - H_o).max() <= rtol * scale


def _reexpress(order, X, pose):
    """The stencil record of vbd_b200.cu build_ell: the solved vertex renumbered as vertex 0."""
    D00, D01, D10, D11 = pose
    if order == 1:
        Xr = np.stack([X[1], X[2], X[0]])
        P = (D10, D11, -D00 - D10, -D01 - D11)
    elif order == 2:
        Xr = np.stack([X[2], X[0], X[1]])
        P = (-D00 - D10, -D01 - D11, D00, D01)
    else:
        Xr, P = X.copy(), (D00, D01, D10, D11)
    return Xr, np.array(P)


@pytest.mark.parametrize("prec,rtol", [(64, 1e-9), (32, 3e-4)])
def test_stencil_face_record_is_the_same_membrane(hostlib, golden_dir, prec, rtol):
    for r in _cases(golden_dir, "membrane"):
        X, Xp, pose = r[0:9].reshape(3, 3), r[9:18].reshape(3, 3), r[18:22]
        area, mu, lam, damping, dt, order = r[22:28]
        f_o, H_o = orc.element("membrane", 64, order, X.ravel(), Xp.ravel(), pose, area, mu, lam, damping, dt)
        Xr, P = _reexpress(int(order), X, pose)
        Xpr, _ = _reexpress(int(order), Xp, pose)
        out, op = _p(np.zeros(12))
        a, ap = _p(Xr.ravel())
        b, bp = _p(Xpr.ravel())
        c, cp = _p(P)
        hostlib.host_membrane(prec, 0, ap, bp, cp, 1.0, mu * area, lam * area, damping, dt, op)
        scale = max(np.abs(f_o).max(), np.abs(H_o).max())
        assert np.abs(out[:3] - f_o).max() <= rtol * scale
        assert np.abs(out[3:].reshape(3, 3) - H_o).max() <= rtol * scale
