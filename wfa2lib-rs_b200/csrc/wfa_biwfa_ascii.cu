// wfa_biwfa_ascii.cu -- lean BiWFA kernels, ASCII sequences, a warp per pair.
#include "wfa_biwfa_kernels.cuh"

namespace wfab {

WFA_BIWFA_INSTANCE(WFA_SEQ_ASCII, false, 32)

}  // namespace wfab
