"""gbm3d_b200 — GBM3D two-step image denoising on NVIDIA B200 (sm_100a).

A from-scratch CUDA implementation of the hot path of toby-sanders/GBM3D
(block matching, global 3D wavelet hard thresholding, empirical Wiener
filtering, weighted aggregation) behind a C ABI (include/gbm3d.h) whose entry
points carry the reference's MATLAB function names.  This package is the
Python host side: option profiles (options), the reference-named calls (api)
and seeded synthetic images (synth).
"""
from .options import (checkBM3Dopts, getTau, getWaveFilters3Dbior, myMirrorPadImage, myPSNR,
                      resolve_opts, setBM3Dopts)
from ._lib import Context, GBM3DError, context
from .distributed import GBM3D_distributed, getBM3D_distribution, makeInterpWindow
from .api import (GBM3D, GBM3D_device, MatchSet, denoiseAndAggregateGPU, denoiseAndAggregateWie,
                  denoiseAndAggregateWieFast, matchBlocksCPU, matchBlocksGPU, matchBlocksWie)

__all__ = [
    "GBM3D", "GBM3D_device", "matchBlocksCPU", "matchBlocksGPU", "denoiseAndAggregateGPU", "matchBlocksWie",
    "denoiseAndAggregateWieFast", "denoiseAndAggregateWie", "MatchSet", "Context", "context",
    "GBM3DError", "setBM3Dopts", "checkBM3Dopts", "resolve_opts", "getTau", "getWaveFilters3Dbior",
    "myMirrorPadImage", "myPSNR", "GBM3D_distributed", "getBM3D_distribution", "makeInterpWindow",
]
