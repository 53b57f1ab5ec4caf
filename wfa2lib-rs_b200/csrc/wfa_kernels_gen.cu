// wfa_kernels_gen.cu -- general (ends-free, heuristics, Corrected): the
// unidirectional kernel's instantiations for ends-free, heuristic and Corrected alignments in high memory or score only (whole warps), in a translation
// unit of their own so the kernel variants build in parallel.
#include "wfa_unialign.cuh"

namespace wfab {

template <int CLS>
static cudaError_t launch_c(const AlignParams& P, int blocks, size_t smem, cudaStream_t st) {
  return P.format == WFA_SEQ_PACKED2 ? launch_t<CLS, 1, true, 32>(P, blocks, smem, st)
                                     : launch_t<CLS, 0, true, 32>(P, blocks, smem, st);
}
template <int CLS>
static int occ_c(const AlignParams& P, size_t smem) {
  return P.format == WFA_SEQ_PACKED2 ? occ_t<CLS, 1, true, 32>(smem) : occ_t<CLS, 0, true, 32>(smem);
}

cudaError_t general_launch(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st) {
  switch (cls) {
    case kEditClass: return launch_c<kEditClass>(P, blocks, smem, st);
    case kLinearClass: return launch_c<kLinearClass>(P, blocks, smem, st);
    case kAffineClass: return launch_c<kAffineClass>(P, blocks, smem, st);
    default: return launch_c<kAffine2pClass>(P, blocks, smem, st);
  }
}

int general_occupancy(const AlignParams& P, int cls, size_t smem) {
  switch (cls) {
    case kEditClass: return occ_c<kEditClass>(P, smem);
    case kLinearClass: return occ_c<kLinearClass>(P, smem);
    case kAffineClass: return occ_c<kAffineClass>(P, smem);
    default: return occ_c<kAffine2pClass>(P, smem);
  }
}

}  // namespace wfab
