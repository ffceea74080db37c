// pool_p0.cu -- batch kernels of pool shape 0: one group per CTA (a matrix per 512-thread CTA).
#include "pool.cuh"

PBRCM_DEFINE_POOL(0, 512, 2048, 512, 2048, 1, 2)
