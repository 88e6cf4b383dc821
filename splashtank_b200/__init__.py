"""B200-native FLIP water step of SplashTank: hand-written sm_100a kernels behind a C ABI (include/splashtank_cuda.h).

FlipSim mirrors the reference simulator's per-step API; SceneRunner and key_pose mirror its scene layer.
"""
from .flip import FlipSim, StError, load_library  # noqa: F401
from .scene import SceneRunner, key_pose, sphere_sdf, box_sdf, euler_mat  # noqa: F401
