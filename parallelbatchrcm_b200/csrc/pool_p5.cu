// pool_p5.cu -- batch kernels of pool shape 5: 256-thread CTAs of one group with 512-edge chunks, three per SM (the solo engine's 76 registers).
#include "pool.cuh"

PBRCM_DEFINE_POOL(5, 256, 512, 256, 512, 3, 4)
