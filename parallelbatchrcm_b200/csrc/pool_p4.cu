// pool_p4.cu -- batch kernels of pool shape 4: 128-thread CTAs of one group, four per SM.
#include "pool.cuh"

PBRCM_DEFINE_POOL(4, 128, 512, 128, 512, 4, 4)
