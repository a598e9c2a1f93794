// Stage kernels for the f32 precision combination (stored float, state arithmetic float, flux arithmetic float).
#include "od_launch_impl.cuh"

OD_INSTANTIATE(f32, float, float, float)
