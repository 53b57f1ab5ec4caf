// wfa_kernels_medlow.cu -- med/low (the piggyback backtrace): the
// unidirectional kernel's instantiations for med/low memory with an alignment (whole warps; every span, heuristic and compat), in a translation
// unit of their own so the kernel variants build in parallel.
#include "wfa_unialign.cuh"

namespace wfab {

template <int CLS>
static cudaError_t launch_c(const AlignParams& P, int blocks, size_t smem, cudaStream_t st) {
  return P.format == WFA_SEQ_PACKED2 ? launch_t<CLS, 1, true, 32, true>(P, blocks, smem, st)
                                     : launch_t<CLS, 0, true, 32, true>(P, blocks, smem, st);
}
template <int CLS>
static int occ_c(const AlignParams& P, size_t smem) {
  return P.format == WFA_SEQ_PACKED2 ? occ_t<CLS, 1, true, 32, true>(smem) : occ_t<CLS, 0, true, 32, true>(smem);
}

cudaError_t medlow_launch(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st) {
  switch (cls) {
    case kEditClass: return launch_c<kEditClass>(P, blocks, smem, st);
    case kLinearClass: return launch_c<kLinearClass>(P, blocks, smem, st);
    case kAffineClass: return launch_c<kAffineClass>(P, blocks, smem, st);
    default: return launch_c<kAffine2pClass>(P, blocks, smem, st);
  }
}

int medlow_occupancy(const AlignParams& P, int cls, size_t smem) {
  switch (cls) {
    case kEditClass: return occ_c<kEditClass>(P, smem);
    case kLinearClass: return occ_c<kLinearClass>(P, smem);
    case kAffineClass: return occ_c<kAffineClass>(P, smem);
    default: return occ_c<kAffine2pClass>(P, smem);
  }
}

}  // namespace wfab
