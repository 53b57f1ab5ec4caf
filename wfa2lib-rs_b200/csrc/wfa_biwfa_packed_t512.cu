// wfa_biwfa_packed_t512.cu -- lean BiWFA kernels, 2-bit packed sequences, teams of 16 warps per pair.
#include "wfa_biwfa_kernels.cuh"

namespace wfab {

WFA_BIWFA_INSTANCE(WFA_SEQ_PACKED2, false, 512)

}  // namespace wfab
