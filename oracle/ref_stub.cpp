/*
 * Test infrastructure only. The reference's pairwise dispatcher names
 * needleman::hybrid (src/pairwise/pairwise.cpp:275-276), whose CUDA source
 * does not build with nvcc 12.9 as shipped (a narrowing error in
 * src/pairwise/needleman/impl/hybrid.cu). The oracle never selects it (the
 * harness always asks for "sequential"), so this stub supplies the symbol
 * without touching any reference file.
 */
#include "pairwise/pairwise.cuh"
#include "pairwise/needleman/needleman.cuh"

namespace museqa { namespace pairwise { namespace needleman {
    auto hybrid() -> pairwise::algorithm * { return sequential(); }
}}}
