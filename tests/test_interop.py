"""The drop-in boundary's array checks, without a GPU: torch tensors, objects that expose only
``__cuda_array_interface__`` (as Warp arrays do), Warp-style ``.ptr`` objects, and the reference Model's
``particle_world_start`` layout. No device memory is touched: the interface dictionaries carry made-up
addresses."""

import types

import numpy as np
import pytest
import torch

from newton_chysx_b200 import interop


class CAI:
    def __init__(self, shape, typestr="<f4", ptr=0x7F0000001000, strides=None):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": tuple(shape), "typestr": typestr,
                                         "strides": strides, "version": 3}  # fmt: skip


class WarpLike:
    """.ptr / .shape / .dtype as a Warp array has them (vec3 = 3 float32 scalars)."""

    def __init__(self, shape, scalar, length=1, ptr=0x7F0000002000, device="cuda:0", contiguous=True):
        self.ptr, self.shape, self.device, self.is_contiguous = ptr, tuple(shape), device, contiguous
        self.dtype = type("vec", (), {"_wp_scalar_type_": type(scalar, (), {}), "_length_": length})


def test_cuda_array_interface_is_read():
    info = interop.describe(CAI((10, 3)))
    assert info == interop.ArrayInfo(0x7F0000001000, "<f4", 30, True)
    p = interop.pointer(CAI((10, 3)), "q", interop.F32, 30)
    assert p.value == 0x7F0000001000
    # C-contiguous strides given explicitly are accepted; unit dimensions may carry any stride
    assert interop.describe(CAI((10, 3), strides=(12, 4))).count == 30
    assert interop.describe(CAI((1, 3), strides=(999, 4))).count == 3


def test_cuda_array_interface_rejects_wrong_type_size_and_strides():
    with pytest.raises(TypeError, match="<f8"):
        interop.pointer(CAI((10, 3)), "q", interop.F64, 30)
    with pytest.raises(ValueError, match="30 scalars"):
        interop.pointer(CAI((9, 3)), "q", interop.F32, 30)
    with pytest.raises(ValueError, match="at least 12"):
        interop.pointer(CAI((3, 3)), "c", interop.F32, at_least=12)
    with pytest.raises(TypeError, match="C-contiguous"):
        interop.describe(CAI((10, 3), strides=(4, 40)))  # a transposed view
    with pytest.raises(TypeError, match="C-contiguous"):
        interop.describe(CAI((10, 3), strides=(24, 4)))  # every other row


def test_empty_arrays_pass_as_null():
    assert interop.pointer(CAI((0, 3), ptr=0), "empty", interop.F32, 0) is None
    assert interop.pointer(None, "none") is None


def test_warp_style_ptr_objects():
    vec3 = WarpLike((5,), "float32", 3)
    assert interop.describe(vec3) == interop.ArrayInfo(0x7F0000002000, "<f4", 15, True)
    assert interop.pointer(vec3, "q", interop.F32, 15).value == 0x7F0000002000
    with pytest.raises(TypeError, match="<i4"):
        interop.pointer(WarpLike((5,), "float32"), "flags", interop.I32, 5)
    with pytest.raises(TypeError, match="device memory"):
        interop.pointer(WarpLike((5,), "int32", device="cpu"), "flags", interop.I32, 5)
    with pytest.raises(TypeError, match="contiguous"):
        interop.describe(WarpLike((5,), "int32", contiguous=False))


def test_torch_tensors():
    t = torch.zeros(4, 3)
    info = interop.describe(t)
    assert info.typestr == "<f4" and info.count == 12 and not info.on_device
    with pytest.raises(TypeError, match="device memory"):
        interop.pointer(t, "q", interop.F32, 12)
    with pytest.raises(TypeError, match="contiguous"):
        interop.describe(t.t())
    with pytest.raises(TypeError):
        interop.describe(object())


def test_reference_particle_world_start_layout():
    """[world_count + 2]: worlds, then the global particles' start, then the count
    (newton/_src/sim/model.py:172-187)."""
    m = types.SimpleNamespace(particle_count=10, world_count=3, particle_world_start=np.array([0, 4, 7, 10, 10]))
    assert interop.world_starts(m).tolist() == [0, 4, 7, 10]
    # global particles after the worlds and before world 0 become instances of their own
    m = types.SimpleNamespace(particle_count=12, world_count=2, particle_world_start=np.array([2, 6, 10, 12]))
    assert interop.world_starts(m).tolist() == [0, 2, 6, 10, 12]
    # one world and no global particles: a single instance
    m = types.SimpleNamespace(particle_count=5, world_count=1, particle_world_start=np.array([0, 5, 5]))
    assert interop.world_starts(m) is None
    # empty worlds are dropped
    m = types.SimpleNamespace(particle_count=6, world_count=3, particle_world_start=np.array([0, 3, 3, 6, 6]))
    assert interop.world_starts(m).tolist() == [0, 3, 6]
    with pytest.raises(ValueError):
        interop.world_starts(types.SimpleNamespace(particle_count=6, world_count=2,
                                                   particle_world_start=np.array([0, 4, 3, 6])))  # fmt: skip
    # this package's own layout [world_count + 1] is taken as it is
    m = types.SimpleNamespace(particle_count=6, world_count=2, world_particle_start=np.array([0, 2, 6]))
    assert interop.world_starts(m).tolist() == [0, 2, 6]


def test_devices():
    assert interop.torch_device("cuda:1") == torch.device("cuda", 1)
    assert interop.torch_device(type("Dev", (), {"__str__": lambda s: "cuda:0"})()) == torch.device("cuda", 0)
    assert interop.torch_device(torch.device("cpu")).type == "cpu"
