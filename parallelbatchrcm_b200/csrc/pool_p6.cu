// pool_p6.cu -- batch kernels of pool shape 6: 256-thread CTAs of one group with 1024-edge chunks, three per SM
// (the solo engine's shared memory packed to 72 KB, 80 registers).
#include "pool.cuh"

PBRCM_DEFINE_POOL(6, 256, 1024, 256, 1024, 3, 3)
