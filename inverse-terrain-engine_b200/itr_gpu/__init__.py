"""itr_gpu — B200 batched forward operator (and adjoint) for the inverse terrain engine.

The compute path is libitr_gpu.so (CUDA, sm_100a) behind the C ABI in include/itr_gpu.h;
this package is the host side mirroring the reference's batch-evaluator interface
(GpuSolver::run_batch, BatchBackend) plus the input builders (terrain, designs, scenes).
"""
from .solver import (Asset, BatchRun, DeviceError, GpuBackend, GpuRun, GpuSolver, Hyetograph, MonitorSet, Objective,
                     ObjectiveDef, SolverParams, UnsupportedError)
from .terrain import FineTerrain, GeoTransform, PreparedTerrain, Segment, TerrainBase, TerrainEdit, synthetic_terrain
from .design import Primitive, materialize

__all__ = [
    "Asset", "BatchRun", "DeviceError", "GpuBackend", "GpuRun", "GpuSolver", "Hyetograph", "MonitorSet", "Objective",
    "ObjectiveDef", "SolverParams", "UnsupportedError", "FineTerrain", "GeoTransform", "PreparedTerrain", "Segment",
    "TerrainBase", "TerrainEdit", "synthetic_terrain", "Primitive", "materialize",
]
