"""B200 (sm_100a) implementation of HyDFT's nonlinear pseudo-spectral solver
step behind the reference's model_t / params_t API.

The compute path is libhydft_gpu.so (hand-written CUDA, built in-tree by
__graft_entry__.build()); this package is the host side over its C ABI.
"""
from .model import (Batch, HydftError, Model, Params, Server, default_params, fd_alpha, fd_table, footprint,
                    fourier_bessel, hnc_solve, lib, read_params)

__all__ = ["Batch", "HydftError", "Model", "Params", "Server", "default_params", "fd_alpha", "fd_table",
           "footprint", "fourier_bessel", "hnc_solve", "lib", "read_params"]
