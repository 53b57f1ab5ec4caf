// wfa_biwfa_packed_gen.cu -- BiWFA kernels with heuristic support, 2-bit packed sequences, a warp per pair.
#include "wfa_biwfa_kernels.cuh"

namespace wfab {

WFA_BIWFA_INSTANCE(WFA_SEQ_PACKED2, true, 32)

}  // namespace wfab
