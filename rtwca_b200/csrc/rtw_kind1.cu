// Trace kernels of scene kind 1 (rtw_scene_kind).
#include "rtw_launch.cuh"
RTW_INSTANTIATE_KIND(1)
