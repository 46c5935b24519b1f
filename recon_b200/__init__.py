"""B200-native MLEM cone-beam reconstruction on a Siddon projector pair.

The compute lives in ``librecon_b200.so`` (hand-written sm_100a CUDA behind the
C ABI of ``include/recon_b200.h``); this package is its Python face.
"""
from ._lib import (ARITH_COMPAT, ARITH_EXACT, BP_SIDDON, BP_VOXEL, FP_COLUMN_BLOCKS, FP_COLUMNS, FP_RAY_WALK, PROJECTOR_BACK, PROJECTOR_FORWARD, SIDDON_BP_AUTO,
                   SIDDON_BP_GATHER, SIDDON_BP_RAY, SIDDON_BP_TUNED, SINO_BF16, SINO_F32, SUM_KAHAN, SUM_PLAIN, VOXEL_GEOMETRIC,
                   VOXEL_REFERENCE, ReconError)
from .api import (Batch, Options, Plan, backward_projection_from_cfg, forward_projection_from_cfg, geometry,
                  geometry_from_cfg, mlem_from_cfg)

__all__ = [
    "ARITH_COMPAT", "ARITH_EXACT", "BP_SIDDON", "BP_VOXEL", "FP_COLUMN_BLOCKS", "FP_COLUMNS", "FP_RAY_WALK", "PROJECTOR_BACK", "PROJECTOR_FORWARD", "SIDDON_BP_AUTO", "SIDDON_BP_GATHER", "SIDDON_BP_RAY", "SIDDON_BP_TUNED",
    "SINO_BF16", "SINO_F32", "SUM_KAHAN", "SUM_PLAIN",
    "VOXEL_GEOMETRIC", "VOXEL_REFERENCE", "ReconError", "Batch", "Options", "Plan", "geometry", "geometry_from_cfg",
    "mlem_from_cfg", "forward_projection_from_cfg", "backward_projection_from_cfg",
]
