// pool_p1.cu -- batch kernels of pool shape 1: two groups of 256 threads per CTA.
#include "pool.cuh"

PBRCM_DEFINE_POOL(1, 512, 2048, 256, 1024, 1, 1)
