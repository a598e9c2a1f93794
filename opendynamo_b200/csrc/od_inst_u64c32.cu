// Stage kernels for the u64c32 precision combination (stored double, state arithmetic float, flux arithmetic float).
#include "od_launch_impl.cuh"

OD_INSTANTIATE(u64c32, double, float, float)
