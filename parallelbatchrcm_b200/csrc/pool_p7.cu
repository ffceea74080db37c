// pool_p7.cu -- batch kernels of pool shape 7: 512-thread CTAs of two 256-thread groups with 2048-edge chunks
// (up to 256 parents a chunk at the engine's usual valences).
#include "pool.cuh"

PBRCM_DEFINE_POOL(7, 512, 2048, 256, 2048, 1, 1)
