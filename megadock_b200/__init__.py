"""megadock-b200: B200-native per-rotation FFT docking (MEGADOCK-compatible).

The docking path runs in libmd_b200.so (C ABI in include/md_b200.h): host C++
for the command line, PDB reading, grid sizing and receptor grids, and
hand-written sm_100a kernels for rotation, voxelization, the FFTs, the
receptor-spectrum product and the top-t search.
"""
from ._native import MdError, Pose, POSE_DTYPE, lib, rotation_matrix, rotation_matrices, sort_poses  # noqa: F401
from .fft_process import FFTProcess, Job  # noqa: F401
