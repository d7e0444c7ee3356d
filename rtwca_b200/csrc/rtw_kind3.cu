// Trace kernels of scene kind 3 (rtw_scene_kind).
#include "rtw_launch.cuh"
RTW_INSTANTIATE_KIND(3)
