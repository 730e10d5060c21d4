"""B200-native rigid-contact XPBD step: Newton's Model.collide + SolverXPBD.step
re-built as hand-written sm_100a CUDA behind a C ABI (libnewton_b200.so).

Public surface mirrors newton (newton/__init__.py, newton/solvers.py) for this path:
    ModelBuilder, Model, State, Control, Contacts, CollisionPipeline, SolverXPBD,
    GeoType, JointType, BodyFlags, ShapeFlags.
"""

from ._abi import BodyFlags, GeoType, JointType, ShapeFlags
from .builder import ModelBuilder
from .collide import CollisionPipeline
from .contacts import Contacts
from .model import Control, Model, State
from .solver_xpbd import SolverNotifyFlags, SolverXPBD

__all__ = [
    "BodyFlags",
    "CollisionPipeline",
    "Contacts",
    "Control",
    "GeoType",
    "JointType",
    "Model",
    "ModelBuilder",
    "ShapeFlags",
    "SolverNotifyFlags",
    "SolverXPBD",
    "State",
]

__version__ = "0.1.0"
