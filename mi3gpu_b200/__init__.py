"""mi3gpu_b200 -- B200 (sm_100a) implementation of Mi3-GPU's inference inner
loop behind the reference's MCMCGPU / GPU_node / NewtonSteps interface.

    from mi3gpu_b200 import MCMCGPU, GPU_node, NewtonSteps

The compute runs in libmi3b200.so (hand-written CUDA, C ABI in
include/mi3b200.h); PyTorch tensors serve only as device buffers.
"""
from . import _lib
from .mcmcGPU import MCMCGPU, FutureBuf, initGPU, setup_GPU_context, histogram_heuristic, wgsize_heuristic
from .node_manager import GPU_node
from . import NewtonSteps, potts

__all__ = ["MCMCGPU", "FutureBuf", "GPU_node", "NewtonSteps", "potts", "initGPU", "setup_GPU_context",
           "histogram_heuristic", "wgsize_heuristic"]
