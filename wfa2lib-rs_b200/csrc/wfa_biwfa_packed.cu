// wfa_biwfa_packed.cu -- lean BiWFA kernels for 2-bit packed sequences, and
// the launcher that picks the encoding and heuristic support.
#include "wfa_biwfa_kernels.cuh"

namespace wfab {

template cudaError_t launch_biwfa_enc<WFA_SEQ_PACKED2, false>(const AlignParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_biwfa_enc<WFA_SEQ_PACKED2, true>(const AlignParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_biwfa_enc<WFA_SEQ_ASCII, false>(const AlignParams&, int, int, size_t, cudaStream_t);
extern template cudaError_t launch_biwfa_enc<WFA_SEQ_ASCII, true>(const AlignParams&, int, int, size_t, cudaStream_t);

cudaError_t launch_biwfa(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st) {
  const bool gen = P.hkind != WFA_HEURISTIC_NONE;
  if (P.format == WFA_SEQ_PACKED2)
    return gen ? launch_biwfa_enc<WFA_SEQ_PACKED2, true>(P, cls, blocks, smem, st)
               : launch_biwfa_enc<WFA_SEQ_PACKED2, false>(P, cls, blocks, smem, st);
  return gen ? launch_biwfa_enc<WFA_SEQ_ASCII, true>(P, cls, blocks, smem, st)
             : launch_biwfa_enc<WFA_SEQ_ASCII, false>(P, cls, blocks, smem, st);
}

}  // namespace wfab
