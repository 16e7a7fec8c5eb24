"""A model, states and contacts whose arrays expose only ``__cuda_array_interface__`` (as the reference's Warp
arrays do), laid out as the reference's Model (``particle_world_start`` [world_count + 2], a device object that
prints as "cuda:0", color groups as device arrays), step bit for bit as the same model built from torch
tensors."""

import types

import numpy as np
import pytest
import torch

from newton_chysx_b200 import CollisionPipeline, SolverVBD, sim
from tests.helpers import cloth_grid_builder

pytestmark = pytest.mark.gpu

MODEL_ARRAYS = ("particle_q", "particle_qd", "particle_mass", "particle_inv_mass", "particle_radius", "particle_flags",
                "tri_indices", "tri_poses", "tri_materials", "tri_areas", "edge_indices", "edge_rest_angle",
                "edge_rest_length", "edge_bending_properties", "gravity", "shape_material_ke", "shape_material_kd",
                "shape_material_mu", "shape_body")  # fmt: skip
CONTACT_ARRAYS = ("soft_contact_count", "soft_contact_particle", "soft_contact_shape", "soft_contact_body_pos",
                  "soft_contact_body_vel", "soft_contact_normal")  # fmt: skip


class CAIOnly:
    """Exposes a device tensor only through __cuda_array_interface__ (and keeps it alive)."""

    def __init__(self, t: torch.Tensor):
        self._t = t
        self.__cuda_array_interface__ = t.__cuda_array_interface__


class WarpDevice:
    def __str__(self):
        return "cuda:0"


def _reference_like(model: sim.Model):
    m = types.SimpleNamespace()
    for k in ("particle_count", "tri_count", "edge_count", "shape_count", "body_count", "world_count",
              "soft_contact_ke", "soft_contact_kd", "soft_contact_mu", "spring_count", "tet_count"):  # fmt: skip
        setattr(m, k, getattr(model, k, 0))
    for k in MODEL_ARRAYS:
        setattr(m, k, CAIOnly(getattr(model, k).clone()))
    m.particle_color_groups = [CAIOnly(g.clone()) for g in model.particle_color_groups]
    m.device = WarpDevice()
    if model.world_particle_start is not None:
        ws = np.asarray(model.world_particle_start, dtype=np.int32)
        pws = np.concatenate([ws, [model.particle_count]]).astype(np.int32)  # no global particles
        m.particle_world_start = CAIOnly(torch.as_tensor(pws, device="cuda"))
    return m


def _reference_state(s: sim.State):
    return types.SimpleNamespace(particle_q=CAIOnly(s.particle_q.clone()), particle_qd=CAIOnly(s.particle_qd.clone()),
                                 particle_f=CAIOnly(s.particle_f.clone()), body_q=None)  # fmt: skip


def _batch():
    top = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    for n, h in ((12, 0.3), (20, 0.004), (9, 0.004)):
        top.add_world(cloth_grid_builder(n=n, hanging=False, height=h, pin_top_corners=(n == 12)))
    top.add_ground_plane()
    m = top.finalize("cuda")
    m.soft_contact_ke, m.soft_contact_kd, m.soft_contact_mu = 1.0e3, 10.0, 0.5
    return m


@pytest.mark.parametrize("schedule", ["persistent", "per_color"])
def test_interface_only_arrays_step_like_torch_tensors(schedule):
    model = _batch()
    ref = _reference_like(model)
    kw = dict(iterations=10, schedule=schedule)
    a = SolverVBD(model, **kw)
    b = SolverVBD(ref, **kw)
    assert (a.layout, a.schedule) == (b.layout, b.schedule)
    pipe = CollisionPipeline(model, soft_contact_margin=0.01)
    c = pipe.contacts()
    rc = types.SimpleNamespace(soft_contact_max=c.soft_contact_max, **{k: CAIOnly(getattr(c, k)) for k in CONTACT_ARRAYS})
    sa = [model.state(), model.state()]
    sb = [_reference_state(sa[0]), _reference_state(sa[1])]
    for k in range(6):
        pipe.collide(sa[k % 2], c)
        a.step(sa[k % 2], sa[(k + 1) % 2], None, c, 1.0 / 600.0)
        b.step(sb[k % 2], sb[(k + 1) % 2], None, rc, 1.0 / 600.0)
    torch.cuda.synchronize()
    for k in range(2):
        assert torch.equal(sa[k].particle_q, sb[k].particle_q._t)
        assert torch.equal(sa[k].particle_qd, sb[k].particle_qd._t)
    assert int(c.soft_contact_count.item()) > 0


def test_interface_only_arrays_are_checked():
    model = _batch()
    ref = _reference_like(model)
    s = SolverVBD(ref, iterations=2)
    st = _reference_state(model.state())
    bad = types.SimpleNamespace(particle_q=CAIOnly(model.state().particle_q.double()), particle_qd=st.particle_qd,
                                particle_f=st.particle_f, body_q=None)  # fmt: skip
    with pytest.raises(TypeError, match="<f4"):
        s.step(bad, st, None, None, 1.0 / 600.0)
    short = types.SimpleNamespace(particle_q=CAIOnly(model.state().particle_q[:-1].clone()),
                                  particle_qd=st.particle_qd, particle_f=st.particle_f, body_q=None)  # fmt: skip
    with pytest.raises(ValueError):
        s.step(short, st, None, None, 1.0 / 600.0)
    strided = types.SimpleNamespace(particle_q=CAIOnly(torch.zeros(3, model.particle_count, device="cuda").t()),
                                    particle_qd=st.particle_qd, particle_f=st.particle_f, body_q=None)  # fmt: skip
    with pytest.raises(TypeError, match="contiguous"):
        s.step(strided, st, None, None, 1.0 / 600.0)
