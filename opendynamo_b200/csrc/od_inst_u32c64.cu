// Stage kernels for the u32c64 precision combination (stored float, state arithmetic double, flux arithmetic double).
#include "od_launch_impl.cuh"

OD_INSTANTIATE(u32c64, float, double, double)
