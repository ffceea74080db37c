// ref_stubs.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's main.cpp (linked into oracle/_ref/ref_rcm only for its
// computeBandwidth / checkBandwidth / maxValency / checkPermutation helpers)
// also references the GPU and cuSOLVER implementations from its renamed
// main().  That main() is never called; these definitions only satisfy the
// linker so that the CPU-only driver needs no CUDA library.
#include <cstdlib>
#include <fstream>
#include <vector>

#include "Graph.h"

namespace CuSolverRCM {
void rcm(Graph<float>&, std::ofstream&, std::vector<unsigned>&) { std::abort(); }
void reorder(const Graph<float>&, const std::vector<unsigned>&) { std::abort(); }
}  // namespace CuSolverRCM

namespace GPU_SIMPLE {
template <typename T>
void rcm(Graph<T>&, std::ofstream&, std::vector<unsigned>&, unsigned) { std::abort(); }
template void rcm(Graph<float>&, std::ofstream&, std::vector<unsigned>&, unsigned);
}  // namespace GPU_SIMPLE

namespace GPU_BATCH {
template <typename T>
void rcm(Graph<T>&, std::ofstream&, std::vector<unsigned>&, unsigned) { std::abort(); }
template void rcm(Graph<float>&, std::ofstream&, std::vector<unsigned>&, unsigned);
}  // namespace GPU_BATCH
