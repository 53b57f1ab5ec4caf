// wfa_biwfa_ascii.cu -- lean BiWFA kernels for ASCII sequences.
#include "wfa_biwfa_kernels.cuh"

namespace wfab {

template cudaError_t launch_biwfa_enc<WFA_SEQ_ASCII, false>(const AlignParams&, int, int, size_t, cudaStream_t);

}  // namespace wfab
