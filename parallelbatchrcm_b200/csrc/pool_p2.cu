// pool_p2.cu -- batch kernels of pool shape 2: four groups of 128 threads per CTA.
#include "pool.cuh"

PBRCM_DEFINE_POOL(2, 512, 2048, 128, 512, 1, 1)
