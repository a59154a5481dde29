"""rendervous_b200 -- B200-native (sm_100a) volumetric path integration.

A drop-in for rendervous's volume hot path: the map classes below keep the
reference's names and constructor signatures and run on hand-written CUDA
kernels in ``libvrt.so`` through the C ABI of ``include/vrt.h``.
"""
from ._lib import VrtError, context
from .maps import (
    ONE, ZERO, ConstantMap, DeltatrackingNEEPathIntegrator, DeltatrackingPathIntegrator, DeltatrackingTransmittance,
    DirectionalLight, DRTDSPathIntegrator, DRTPathIntegrator, DRTQPathIntegrator, Grid3D, GridDDATransmittance,
    GridMaximumMajorant, HenyeyGreensteinPhase, HenyeyGreensteinPhaseSampler, HGDirectionSampler, HGPhase,
    MajorantGrid, MapBase, ParametricMap, PerspectiveCameraSensor, RatiotrackingTransmittance, RayBoxIntersection,
    SPSPathIntegrator, UniformDirectionSampler, VHGPhaseSampler, _functionsampler, check, const, device, next_seed,
    normalized_box, parameter, ray_box_intersection, seed, set_sync_checks, vec3,
)
from . import objects, synthetic

__all__ = [n for n in dir() if not n.startswith("__")]
