// wfa_params.h -- host-side penalty handling shared by the C ABI.
#pragma once
#include <stdint.h>

#include <algorithm>
#include <cstdlib>

#include "wfa_common.h"

namespace wfab {

// Validation and internal penalties of WavefrontPenalties::new_indel/new_edit/
// new_linear/new_affine/new_affine2p (src/penalties.rs:119-296), including
// Eizenga's transform for a match reward, and max_score_scope
// (src/components.rs:435-505).  Returns WFA_OK or WFA_ERR_PENALTIES.
inline int set_penalties(int metric, const wfa_penalties_t* u, AlignParams& P) {
  wfa_penalties_t z = {0, 0, 0, 0, 0, 0};
  if (!u) u = &z;
  P.metric = metric;
  for (int i = 0; i < 6; ++i) P.orig[i] = 0;
  P.o2 = -1;
  P.e2 = -1;
  switch (metric) {
    case WFA_METRIC_INDEL:
      P.match = 0; P.mismatch = -1; P.o1 = 1; P.e1 = -1;
      P.scope = 2;
      return WFA_OK;
    case WFA_METRIC_EDIT:
      P.match = 0; P.mismatch = 1; P.o1 = 1; P.e1 = -1;
      P.scope = 2;
      return WFA_OK;
    case WFA_METRIC_GAP_LINEAR: {
      int32_t m = u->match, x = u->mismatch, i = u->gap_opening1;
      if (m > 0 || !(x > 0 && i > 0)) return WFA_ERR_PENALTIES;
      if (m < 0) { P.match = m; P.mismatch = 2 * x - 2 * m; P.o1 = 2 * i - m; }
      else { P.match = 0; P.mismatch = x; P.o1 = i; }
      P.e1 = -1;
      P.orig[0] = m; P.orig[1] = x; P.orig[2] = i;
      P.scope = std::max(P.mismatch, P.o1) + 1;
      return WFA_OK;
    }
    case WFA_METRIC_GAP_AFFINE: {
      int32_t m = u->match, x = u->mismatch, o = u->gap_opening1, e = u->gap_extension1;
      if (m > 0 || !(x > 0 && o >= 0 && e > 0)) return WFA_ERR_PENALTIES;
      if (m < 0) { P.match = m; P.mismatch = 2 * x - 2 * m; P.o1 = 2 * o; P.e1 = 2 * e - m; }
      else { P.match = 0; P.mismatch = x; P.o1 = o; P.e1 = e; }
      P.orig[0] = m; P.orig[1] = x; P.orig[2] = o; P.orig[3] = e;
      P.scope = std::max(P.o1 + P.e1, P.mismatch) + 1;
      return WFA_OK;
    }
    case WFA_METRIC_GAP_AFFINE_2P: {
      int32_t m = u->match, x = u->mismatch, o1 = u->gap_opening1, e1 = u->gap_extension1;
      int32_t o2 = u->gap_opening2, e2 = u->gap_extension2;
      if (m > 0 || !(x > 0 && o1 >= 0 && e1 > 0 && o2 >= 0 && e2 > 0)) return WFA_ERR_PENALTIES;
      if (m < 0) {
        P.match = m; P.mismatch = 2 * x - 2 * m; P.o1 = 2 * o1; P.e1 = 2 * e1 - m;
        P.o2 = 2 * o2; P.e2 = 2 * e2 - m;
      } else {
        P.match = 0; P.mismatch = x; P.o1 = o1; P.e1 = e1; P.o2 = o2; P.e2 = e2;
      }
      P.orig[0] = m; P.orig[1] = x; P.orig[2] = o1; P.orig[3] = e1; P.orig[4] = o2; P.orig[5] = e2;
      P.scope = std::max(std::max(P.o1 + P.e1, P.o2 + P.e2), P.mismatch) + 1;
      return WFA_OK;
    }
    default:
      return WFA_ERR_ARGUMENT;
  }
}

inline int metric_class(int metric) {
  switch (metric) {
    case WFA_METRIC_INDEL: case WFA_METRIC_EDIT: return kEditClass;
    case WFA_METRIC_GAP_LINEAR: return kLinearClass;
    case WFA_METRIC_GAP_AFFINE: return kAffineClass;
    default: return kAffine2pClass;
  }
}
inline int metric_components(int metric) {
  int c = metric_class(metric);
  return c == kAffine2pClass ? 5 : c == kAffineClass ? 3 : 1;
}

}  // namespace wfab
