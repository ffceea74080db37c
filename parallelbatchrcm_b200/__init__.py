"""parallelbatchrcm_b200 -- B200-native (sm_100a) Reverse Cuthill-McKee engine.

A drop-in for the GPU_BATCH path of GPUPeople/ParallelBatchRCM: the same CSR /
MatrixMarket input, the same options (reverse, start node, stable, bandwidth)
and a permutation bit-identical to the reference's serial stable RCM, computed
by hand-written CUDA kernels behind the C ABI of include/pbrcm.h
(libpbrcm.so, built in-tree by ``parallelbatchrcm_b200.build``).
"""
from .rcm import (  # noqa: F401
    AUTO_START, DEBUG_PHANTOM_CTA, GPU_BATCH, Context, Graph, PbrcmError, Session, SimplePeripheral, bandwidth,
    check_bandwidth, check_permutation, compute_bandwidth, connect_device, default_options, find_peripheral,
    load_hicsr, load_mtx,
    max_valency, store_hicsr, BatchResults, PreparedBatch,
    permute, permute_device, prepare_csr, reorder, reorder_batch, reorder_batch_device, reorder_device,
    reorder_device_noalloc, store_mtx, autotune, tuning_get, tuning_set, tuning_load,
)

__version__ = "0.1.0"
