"""B200-native cloth Vertex Block Descent: a drop-in for ``newton.solvers.SolverVBD``'s particle path.

Public API mirrors the reference names: ``ModelBuilder``, ``Model``, ``State``, ``Control``,
``Contacts``, ``CollisionPipeline``, ``ParticleFlags``, ``TriMeshCollisionDetector`` and ``SolverVBD``;
``solvers.SolverVBD`` is the same class. The solver runs in ``libvbd_b200.so`` (hand-written CUDA for sm_100a).
"""

from .sim import (
    CollisionPipeline,
    ColoringAlgorithm,
    Contacts,
    Control,
    GeoType,
    Heightfield,
    Mesh,
    Model,
    ModelBuilder,
    ParticleFlags,
    ShapeConfig,
    State,
    quat_from_axis_angle,
    quat_identity,
)
from .collision import TriMeshCollisionDetector
from .solver_vbd import SolverVBD


class solvers:  # noqa: N801 - mirrors ``newton.solvers``
    SolverVBD = SolverVBD


__all__ = [
    "CollisionPipeline",
    "ColoringAlgorithm",
    "Contacts",
    "Control",
    "GeoType",
    "Heightfield",
    "Mesh",
    "Model",
    "ModelBuilder",
    "ParticleFlags",
    "ShapeConfig",
    "SolverVBD",
    "State",
    "TriMeshCollisionDetector",
    "quat_from_axis_angle",
    "quat_identity",
    "solvers",
]
