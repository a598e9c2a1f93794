// Stage kernels for the f64 precision combination (stored double, state arithmetic double, flux arithmetic double).
#include "od_launch_impl.cuh"

OD_INSTANTIATE(f64, double, double, double)
