"""gps-pbvr-web_b200: B200-native (sm_100a) stochastic particle renderer for 3D Gaussian splats.

A drop-in for the wgpu renderer of gps-pbvr-web's gps-render crate: the GPS, PBVR
(Proportional, Extinction C0-C3 / C3+R, ViewConditioned) and ScreenOccupancy particle methods,
the depth-sorted alpha path and the composite, as hand-written CUDA kernels behind the C ABI
of include/gpsb200.h. `gps` mirrors the reference's Rust renderer API in Python.
"""
from . import abi
from .gps import (Calibration, GpsError, GpsRenderer, GpuStats, Method, OracleCamera, OrbitCamera, PbvrParams,
                  RenderParams, RenderPath, debug_fmath, default_params, estimate_memory, load_ply, load_ply_device,
                  radius_lut)

__all__ = ["abi", "Calibration", "GpsError", "GpsRenderer", "GpuStats", "Method", "OracleCamera", "OrbitCamera",
           "PbvrParams", "RenderParams", "RenderPath", "debug_fmath", "default_params", "estimate_memory", "load_ply", "load_ply_device",
           "radius_lut"]
