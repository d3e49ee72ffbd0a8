"""rms_b200: a B200-native random-walk diffusion MRI engine.

Drop-in for the CUDA simulator of NYU-DiffusionMRI/monte-carlo-simulation-3D-RMS
(hpc_code/lib/main.cu, main_PGSE.cu): same run-directory inputs and outputs,
computed by hand-written sm_100a kernels behind the C ABI in include/rms.h.

Submodules:
  runio      run-directory text formats (inputs and outputs)
  geometry   seeded synthetic axon lattices
  analysis   the cumulant formulas of analysis/readRMS.m and readRMS_pgse.m
  engine     ctypes binding of the C ABI (librms.so)
"""
__all__ = ["runio", "geometry", "analysis", "engine"]
