// wfa_biwfa_ascii_gen.cu -- BiWFA kernels with heuristic support, ASCII sequences, a warp per pair.
#include "wfa_biwfa_kernels.cuh"

namespace wfab {

WFA_BIWFA_INSTANCE(WFA_SEQ_ASCII, true, 32)

}  // namespace wfab
