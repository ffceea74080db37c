// pool_p3.cu -- batch kernels of pool shape 3: eight groups of 64 threads per CTA.
#include "pool.cuh"

PBRCM_DEFINE_POOL(3, 512, 2048, 64, 256, 1, 0)
