"""B200-native geodesic spectral ray tracer (CUDA sm_100a behind a C ABI).

Host mirror of the reference's render call; the integrator runs in
librtw_b200.so (see include/rtw.h).
"""
from . import abi, configs
from .render import Renderer, gen_image, initialize_world, set_scene, xyz_to_srgb, available_worlds

__all__ = ["abi", "configs", "Renderer", "gen_image", "initialize_world", "set_scene", "xyz_to_srgb",
           "available_worlds"]
