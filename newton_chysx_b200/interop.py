"""Device arrays at the drop-in boundary.

The reference's Model, State and Contacts hold Warp arrays (``newton/_src/sim/model.py``, ``state.py``,
``contacts.py``); this package's own hold torch tensors. ``SolverVBD`` takes either, and any other object that
exposes ``__cuda_array_interface__`` (CuPy, Numba, ...), or a raw ``.ptr`` with ``.shape`` and a Warp-style
``.dtype``. Each array is checked for its element type, its element count and C-contiguity before its pointer
goes to the C ABI, in the way the reference's own ctypes plug-in hands Warp pointers to native code
(``newton/_src/solvers/chysx/solver_chysx.py:991-1039``: values copied, pointers referenced).
"""

from __future__ import annotations

import ctypes as C
import math
import sys
from typing import NamedTuple

import numpy as np
import torch

F32, F64, I32 = "<f4", "<f8", "<i4"
_TORCH_TYPESTR = {torch.float32: F32, torch.float64: F64, torch.int32: I32}
_NAME_TYPESTR = {"float32": F32, "float64": F64, "int32": I32}


class ArrayInfo(NamedTuple):
    ptr: int  # device address (0 for an empty array)
    typestr: str  # numpy array-interface element type of the scalars, e.g. "<f4"
    count: int  # number of scalars
    on_device: bool


def _c_contiguous(shape, strides, itemsize) -> bool:
    if strides is None:
        return True
    expect = itemsize
    for n, s in zip(reversed(shape), reversed(strides), strict=True):
        if n > 1 and s != expect:
            return False
        expect *= n
    return True


def describe(obj, what: str = "array") -> ArrayInfo | None:
    """Pointer, scalar type and scalar count of a torch tensor, an object with ``__cuda_array_interface__``
    (v2/v3: ``data``, ``shape``, ``typestr``, ``strides``) or one with ``.ptr``, ``.shape`` and ``.dtype``.
    Raises TypeError for a strided (non C-contiguous) array or an unknown type."""
    if obj is None:
        return None
    if isinstance(obj, torch.Tensor):
        if not obj.is_contiguous():
            raise TypeError(f"{what} must be contiguous")
        return ArrayInfo(obj.data_ptr(), _TORCH_TYPESTR.get(obj.dtype, str(obj.dtype)), obj.numel(), obj.is_cuda)
    cai = getattr(obj, "__cuda_array_interface__", None)
    if cai is not None:
        shape = tuple(int(n) for n in cai["shape"])
        typestr = str(cai["typestr"])
        if typestr[:1] == "=":
            typestr = "<" + typestr[1:]
        itemsize = int(typestr[2:]) if typestr[2:].isdigit() else 0
        if not _c_contiguous(shape, cai.get("strides"), itemsize):
            raise TypeError(f"{what} must be C-contiguous (strides {cai.get('strides')} for shape {shape})")
        return ArrayInfo(int(cai["data"][0] or 0), typestr, math.prod(shape), True)
    if hasattr(obj, "ptr") and hasattr(obj, "shape") and hasattr(obj, "dtype"):
        dt = obj.dtype
        scalar = getattr(dt, "_wp_scalar_type_", dt)
        name = getattr(scalar, "__name__", str(scalar))
        length = int(getattr(dt, "_length_", 1))
        if getattr(obj, "is_contiguous", True) is False:
            raise TypeError(f"{what} must be contiguous")
        count = math.prod(int(n) for n in obj.shape) * length
        dev = str(getattr(obj, "device", "cuda"))
        return ArrayInfo(int(obj.ptr or 0), _NAME_TYPESTR.get(name, name), count, dev.startswith("cuda"))
    raise TypeError(f"{what}: expected a torch tensor, an object with __cuda_array_interface__, or .ptr/.shape/.dtype")


def pointer(obj, what: str, typestr: str | None = None, count: int | None = None, at_least: int | None = None):
    """``ctypes.c_void_p`` of a device array after checking its element type and scalar count (exactly
    `count`, or at least `at_least`); None for None or an empty array."""
    info = describe(obj, what)
    if info is None:
        return None
    if typestr is not None and info.typestr != typestr:
        raise TypeError(f"{what} must hold {typestr} scalars, got {info.typestr}")
    if count is not None and info.count != count:
        raise ValueError(f"{what} must hold {count} scalars, got {info.count}")
    if at_least is not None and info.count < at_least:
        raise ValueError(f"{what} must hold at least {at_least} scalars, got {info.count}")
    if info.count and not info.on_device:
        raise TypeError(f"{what} must be in device memory")
    return C.c_void_p(info.ptr) if info.count else None


def to_host(obj) -> np.ndarray:
    """A host copy of a small array (color groups, world starts): torch tensors, Warp arrays (``.numpy()``),
    ``__cuda_array_interface__`` objects, numpy arrays and lists."""
    if isinstance(obj, torch.Tensor):
        return obj.detach().cpu().numpy()
    if isinstance(obj, (np.ndarray, list, tuple)):
        return np.asarray(obj)
    if getattr(obj, "__cuda_array_interface__", None) is not None:
        return torch.as_tensor(obj, device="cuda").cpu().numpy()
    if hasattr(obj, "numpy"):
        return np.asarray(obj.numpy())
    return np.asarray(obj)


def as_torch(obj, device) -> torch.Tensor:
    """A torch view of a device array (zero-copy for ``__cuda_array_interface__`` objects) or a device copy of
    a host one."""
    if isinstance(obj, torch.Tensor):
        return obj
    if getattr(obj, "__cuda_array_interface__", None) is not None:
        return torch.as_tensor(obj, device=device)
    return torch.as_tensor(to_host(obj), device=device)


def torch_device(dev) -> torch.device:
    """A torch device from a torch device, a Warp device (``str(dev) == "cuda:0"``) or a string."""
    if isinstance(dev, torch.device):
        return dev
    if dev is None:
        raise RuntimeError("the model has no device")
    return torch.device(str(dev))


def world_starts(model) -> np.ndarray | None:
    """Particle ranges of the model's worlds as starts [K+1] (first 0, last particle_count), or None for one
    world. This package's Model gives ``world_particle_start`` [world_count + 1]. The reference Model gives
    ``particle_world_start`` [world_count + 2] (``newton/_src/sim/model.py:172-187``): worlds 0..W-1, then the
    start of the global particles at [-2] and the particle count at [-1]; global particles may also sit before
    world 0. Global particle ranges become instances of their own, and empty worlds are dropped."""
    n = int(model.particle_count)
    ws = getattr(model, "world_particle_start", None)
    if ws is not None and int(getattr(model, "world_count", 0) or 0) > 1:
        return np.ascontiguousarray(to_host(ws), dtype=np.int32)
    ref = getattr(model, "particle_world_start", None)
    if ref is None or int(getattr(model, "world_count", 0) or 0) < 1:
        return None
    pws = to_host(ref).astype(np.int64).reshape(-1)
    if pws.size < 2 or pws.min() < 0 or pws.max() > n or np.any(np.diff(pws) < 0):
        raise ValueError(f"particle_world_start must be non-decreasing starts within [0, {n}], got {pws.tolist()}")
    bounds = np.unique(np.concatenate([[0], pws, [n]]))
    return None if len(bounds) < 3 else np.ascontiguousarray(bounds, dtype=np.int32)


def launch_stream(device: torch.device, arrays_from_warp: bool) -> int:
    """The CUDA stream a step launches on: Warp's current stream of the device when the caller's arrays are
    Warp arrays and Warp is loaded (the reference launches every kernel there), else torch's current stream."""
    if arrays_from_warp and "warp" in sys.modules:
        wp = sys.modules["warp"]
        return int(wp.get_stream(str(device)).cuda_stream)
    return int(torch.cuda.current_stream(device).cuda_stream)


def from_warp(obj) -> bool:
    return type(obj).__module__.split(".")[0] == "warp"
