// wfa_biwfa_ascii_gen.cu -- BiWFA kernels with heuristics, ASCII sequences.
#include "wfa_biwfa_kernels.cuh"

namespace wfab {

template cudaError_t launch_biwfa_enc<WFA_SEQ_ASCII, true>(const AlignParams&, int, int, size_t, cudaStream_t);

}  // namespace wfab
