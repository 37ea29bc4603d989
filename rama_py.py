"""`import rama_py` compatibility shim: the reference's module name, served by
rama_b200.rama_py."""
from rama_b200.rama_py import *  # noqa: F401,F403
from rama_b200.rama_py import multicut_solver_options, rama_cuda, rama_cuda_gpu_pointers, rama_torch, read_multicut_file  # noqa: F401
