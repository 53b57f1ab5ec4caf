// wfa_biwfa_ascii_t512.cu -- lean BiWFA kernels, ASCII sequences, teams of 16 warps per pair.
#include "wfa_biwfa_kernels.cuh"

namespace wfab {

WFA_BIWFA_INSTANCE(WFA_SEQ_ASCII, false, 512)

}  // namespace wfab
