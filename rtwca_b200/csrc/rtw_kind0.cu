// Trace kernels of scene kind 0 (rtw_scene_kind).
#include "rtw_launch.cuh"
RTW_INSTANTIATE_KIND(0)
