// Stage kernels for the mixed precision combination (stored double, state arithmetic double, flux arithmetic float).
#include "od_launch_impl.cuh"

OD_INSTANTIATE(mixed, double, double, float)
