// Trace kernels of scene kind 2 (rtw_scene_kind).
#include "rtw_launch.cuh"
RTW_INSTANTIATE_KIND(2)
