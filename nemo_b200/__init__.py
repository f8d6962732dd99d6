"""nemo_b200: B200-native spatial operator of nemo (DGSEM split form + FV blending + LSRK 5-4).

The compute path is libnemo_gpu.so (hand-written CUDA for sm_100a behind the C-ABI in
include/nemo_gpu.h); this package holds its ctypes binding, the host-side mirror of the reference's
hook interface (solver), the forest generator and adapt step (mesh), the initial conditions of the
benchmark workloads (setups), the element partition with its ghost exchange (partition), the
FLASH-layout checkpoints and restart (checkpoint) and the learned indicator's training (learned).
"""
from . import abi, mesh, setups  # noqa: F401

__all__ = ["abi", "mesh", "setups", "solver", "partition", "checkpoint", "learned"]
