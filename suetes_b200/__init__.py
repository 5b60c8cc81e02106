"""B200 (sm_100a) implementation of the Suetes SISL timestep.

Public API mirrors the reference ``suetes.regional3d`` modules:
``RegionalGrid3D``, ``CGridOperator3D``, ``tensor_product_interp_3d``,
``Euler3D``, ``VerticalPreconditioner``, ``SemiLagrangianAdvector3D``,
``SemiImplicitSolver3D``, ``FluxFormAdvector``, ``SISLStepper3D`` and
``build_dynamical_core``.  The numerical work runs in ``libsisl_b200.so``
(C ABI in ``include/sisl_b200.h``).
"""

from .boundaries import BenchmarkSponge, DaviesSponge, LateralRelaxation, x_relaxation
from .driver import Simulation
from .euler import Euler3D
from .geometry import (GalChenSigma, HybridSigma, RegionalGrid3D, SleveSimple, StretchedSleveSimple)
from .operators import CGridOperator3D, map_coordinates_linear, tensor_product_interp_3d
from .output import AsyncSnapshotWriter, NetcdfSnapshots, SimulationOutputWriter, restart_seed
from .physics import PhysicsSuite
from .split_explicit import SplitExplicitStepper3D
from .steppers import (DeviceState, FluxFormAdvector, PingPong, SemiImplicitSolver3D, SemiLagrangianAdvector3D,
                       SISLStepper3D, StateRing, StepGraph, VerticalPreconditioner, build_dynamical_core)

__all__ = [
    "RegionalGrid3D", "GalChenSigma", "HybridSigma", "SleveSimple", "StretchedSleveSimple", "CGridOperator3D",
    "tensor_product_interp_3d", "map_coordinates_linear", "Euler3D", "VerticalPreconditioner",
    "SemiLagrangianAdvector3D", "SemiImplicitSolver3D", "FluxFormAdvector", "SISLStepper3D", "DeviceState",
    "StateRing", "StepGraph", "PingPong", "build_dynamical_core", "LateralRelaxation", "x_relaxation",
    "PhysicsSuite", "SplitExplicitStepper3D", "SimulationOutputWriter", "AsyncSnapshotWriter", "NetcdfSnapshots",
    "restart_seed", "DaviesSponge", "BenchmarkSponge", "Simulation",
]
