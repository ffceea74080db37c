// pool_p4.cu -- batch kernels of pool shape 4: 128-thread CTAs of one group (single requests of the serving session).
#include "pool.cuh"

PBRCM_DEFINE_POOL(4, 128, 512, 128, 512)
