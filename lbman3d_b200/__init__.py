"""lbman3d_b200 -- B200 (sm_100a) implementation of lbman3d's per-timestep
hot path: D3Q15 lattice Boltzmann + Beris-Edwards Q-tensor active nematics,
with the reference's boundary rules and diagnostics, behind a C ABI
(include/lbman3d.h) and the reference's interface names.
"""
from . import _native
from .boundary import (Anchoring, BCConfig, ChannelConfig, FullyPeriodicConfig, MovingWall, Neumann,
                       NoSlip, Periodic, PeriodicBC, SimBC, SlitConfig, SlitNoSlipConfig,
                       SpecularReflection, WallSpec, from_face_tuples, is_wall_by_face,
                       periodicity_by_axis)
from .device import (DeviceFields, DeviceSolver, InitializeComputeBackend, LbmSolver, QTensorSolver,
                     Simulation, make_config)
from .fields import FluidFields, LocalGrid, QTensorFields
from .ensemble import Ensemble, ShardedEnsemble, draw_boxes, shard_boxes
from .params import Advection, EquilibriumScalarOrder, Params, Precision
from .slab import DistributedSlab, Slab, SlabBox, split_planes

__all__ = [
    "Anchoring", "BCConfig", "ChannelConfig", "FullyPeriodicConfig", "MovingWall", "Neumann", "NoSlip",
    "Periodic", "PeriodicBC", "SimBC", "SlitConfig", "SlitNoSlipConfig", "SpecularReflection", "WallSpec",
    "from_face_tuples", "is_wall_by_face", "periodicity_by_axis", "DeviceFields", "DeviceSolver",
    "InitializeComputeBackend", "LbmSolver", "QTensorSolver", "Simulation", "make_config", "FluidFields",
    "LocalGrid", "QTensorFields", "Advection", "EquilibriumScalarOrder", "Params", "Precision", "Ensemble",
    "draw_boxes", "ShardedEnsemble", "shard_boxes", "DistributedSlab", "Slab", "SlabBox", "split_planes",
]
