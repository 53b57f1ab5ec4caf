// wfa_biwfa_packed_gen.cu -- BiWFA kernels with heuristics, 2-bit packed sequences.
#include "wfa_biwfa_kernels.cuh"

namespace wfab {

template cudaError_t launch_biwfa_enc<WFA_SEQ_PACKED2, true>(const AlignParams&, int, int, size_t, cudaStream_t);

}  // namespace wfab
