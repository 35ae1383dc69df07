"""cellgpu_b200: B200-native (sm_100a) implementation of cellGPU's per-timestep hot path.

The compute lives in ``libcellgpu_b200.so`` (hand-written CUDA behind the C ABI of
``include/cellgpu_b200.h``); this package is the Python mirror of the reference's class API.
"""
from ._lib import (CG_ERR_ARG, CG_ERR_CAPACITY, CG_ERR_CUDA, CG_ERR_STATE, CG_ERR_TIMEOUT,  # noqa: F401
                   CG_ERR_TOPOLOGY, CG_FP64, CG_MIXED, CG_OK, CellGPUError, load)
from ._lib import FireParams  # noqa: F401
from .models import (EnergyMinimizerFIRE, Simulation, VertexBatch, VertexQuadraticEnergy,  # noqa: F401
                     VertexQuadraticEnergyWithTension,
                     Voronoi2D, VoronoiBatch, VoronoiQuadraticEnergy, VoronoiQuadraticEnergyWithTension,
                     brownianParticleDynamics,
                     random_positions, restore, selfPropelledCellVertexDynamics,
                     selfPropelledParticleDynamics)

__all__ = [
    "CG_FP64", "CG_MIXED", "CellGPUError", "EnergyMinimizerFIRE", "FireParams", "load", "Simulation",
    "VertexBatch", "VertexQuadraticEnergy", "VertexQuadraticEnergyWithTension", "Voronoi2D", "VoronoiBatch", "VoronoiQuadraticEnergy",
    "VoronoiQuadraticEnergyWithTension", "brownianParticleDynamics", "random_positions", "restore", "selfPropelledCellVertexDynamics",
    "selfPropelledParticleDynamics",
]
