// wfa_biwfa_packed.cu -- lean BiWFA kernels for 2-bit packed sequences (a
// warp per pair), and the launcher that picks the encoding, the heuristic
// support and the lane-group width (the kernels themselves in wfa_biwfa_*.cu).
#include "wfa_biwfa_kernels.cuh"

namespace wfab {

WFA_BIWFA_INSTANCE(WFA_SEQ_PACKED2, false, 32)
WFA_BIWFA_EXTERN(WFA_SEQ_PACKED2, true, 32)
WFA_BIWFA_EXTERN(WFA_SEQ_PACKED2, false, 128)
WFA_BIWFA_EXTERN(WFA_SEQ_PACKED2, false, 256)
WFA_BIWFA_EXTERN(WFA_SEQ_PACKED2, false, 512)
WFA_BIWFA_EXTERN(WFA_SEQ_ASCII, false, 32)
WFA_BIWFA_EXTERN(WFA_SEQ_ASCII, true, 32)
WFA_BIWFA_EXTERN(WFA_SEQ_ASCII, false, 128)
WFA_BIWFA_EXTERN(WFA_SEQ_ASCII, false, 256)
WFA_BIWFA_EXTERN(WFA_SEQ_ASCII, false, 512)

template <int ENC, bool GEN>
static cudaError_t launch_enc(const AlignParams& P, int cls, int lanes, int blocks, size_t smem,
                              cudaStream_t st) {
  if constexpr (!GEN) {
    if (lanes == 128) return launch_biwfa_lw<ENC, false, 128>(P, cls, blocks, smem, st);
    if (lanes == 256) return launch_biwfa_lw<ENC, false, 256>(P, cls, blocks, smem, st);
    if (lanes == 512) return launch_biwfa_lw<ENC, false, 512>(P, cls, blocks, smem, st);
  }
  return launch_biwfa_lw<ENC, GEN, 32>(P, cls, blocks, smem, st);
}

template <int ENC, bool GEN>
static int occupancy_enc(int cls, int lanes, size_t smem) {
  if constexpr (!GEN) {
    if (lanes == 128) return occupancy_biwfa_lw<ENC, false, 128>(cls, smem);
    if (lanes == 256) return occupancy_biwfa_lw<ENC, false, 256>(cls, smem);
    if (lanes == 512) return occupancy_biwfa_lw<ENC, false, 512>(cls, smem);
  }
  return occupancy_biwfa_lw<ENC, GEN, 32>(cls, smem);
}

cudaError_t launch_biwfa(const AlignParams& P, int cls, int lanes, int blocks, size_t smem, cudaStream_t st) {
  const bool gen = P.hkind != WFA_HEURISTIC_NONE;
  if (P.format == WFA_SEQ_PACKED2)
    return gen ? launch_enc<WFA_SEQ_PACKED2, true>(P, cls, lanes, blocks, smem, st)
               : launch_enc<WFA_SEQ_PACKED2, false>(P, cls, lanes, blocks, smem, st);
  return gen ? launch_enc<WFA_SEQ_ASCII, true>(P, cls, lanes, blocks, smem, st)
             : launch_enc<WFA_SEQ_ASCII, false>(P, cls, lanes, blocks, smem, st);
}

int occupancy_biwfa(const AlignParams& P, int cls, int lanes, size_t smem) {
  const bool gen = P.hkind != WFA_HEURISTIC_NONE;
  if (P.format == WFA_SEQ_PACKED2)
    return gen ? occupancy_enc<WFA_SEQ_PACKED2, true>(cls, lanes, smem)
               : occupancy_enc<WFA_SEQ_PACKED2, false>(cls, lanes, smem);
  return gen ? occupancy_enc<WFA_SEQ_ASCII, true>(cls, lanes, smem)
             : occupancy_enc<WFA_SEQ_ASCII, false>(cls, lanes, smem);
}

}  // namespace wfab
