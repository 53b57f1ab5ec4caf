// wfa_kernels.cu -- dispatch of the unidirectional kernel to its
// instantiations (wfa_kernels_lean4/8/16/32.cu, wfa_kernels_gen.cu,
// wfa_kernels_medlow.cu).
#include "wfa_kernels.h"

namespace wfab {

cudaError_t lean_w4_launch(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st);
cudaError_t lean_w8_launch(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st);
cudaError_t lean_w16_launch(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st);
cudaError_t lean_w32_launch(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st);
cudaError_t general_launch(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st);
cudaError_t medlow_launch(const AlignParams& P, int cls, int blocks, size_t smem, cudaStream_t st);
int lean_w4_occupancy(const AlignParams& P, int cls, size_t smem);
int lean_w8_occupancy(const AlignParams& P, int cls, size_t smem);
int lean_w16_occupancy(const AlignParams& P, int cls, size_t smem);
int lean_w32_occupancy(const AlignParams& P, int cls, size_t smem);
int general_occupancy(const AlignParams& P, int cls, size_t smem);
int medlow_occupancy(const AlignParams& P, int cls, size_t smem);

// The lean instantiation runs end-to-end high-memory (or score-only)
// alignments without a heuristic, with 4, 8, 16 or 32 lanes per pair;
// everything else (ends-free, heuristics, Corrected) runs the general one on
// whole warps, and med/low with an alignment its own instantiation of it.
bool needs_general(const AlignParams& P) {
  return P.span != WFA_SPAN_END2END || P.hkind != WFA_HEURISTIC_NONE || P.piggyback;
}

cudaError_t launch_unialign(const AlignParams& P, int metric_class, int lanes, int blocks, size_t smem,
                            cudaStream_t st) {
  if (P.piggyback && P.compute_alignment) return medlow_launch(P, metric_class, blocks, smem, st);
  if (needs_general(P)) return general_launch(P, metric_class, blocks, smem, st);
  if (lanes == 4) return lean_w4_launch(P, metric_class, blocks, smem, st);
  if (lanes == 8) return lean_w8_launch(P, metric_class, blocks, smem, st);
  if (lanes == 16) return lean_w16_launch(P, metric_class, blocks, smem, st);
  return lean_w32_launch(P, metric_class, blocks, smem, st);
}

int occupancy_blocks_per_sm(const AlignParams& P, int metric_class, int lanes, size_t smem) {
  if (P.piggyback && P.compute_alignment) return medlow_occupancy(P, metric_class, smem);
  if (needs_general(P)) return general_occupancy(P, metric_class, smem);
  if (lanes == 4) return lean_w4_occupancy(P, metric_class, smem);
  if (lanes == 8) return lean_w8_occupancy(P, metric_class, smem);
  if (lanes == 16) return lean_w16_occupancy(P, metric_class, smem);
  return lean_w32_occupancy(P, metric_class, smem);
}

}  // namespace wfab
