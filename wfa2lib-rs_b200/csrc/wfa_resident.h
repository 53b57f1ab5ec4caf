// wfa_resident.h -- what the host and the resident serving kernel share
// (wfa_resident.cu): the request ring in mapped host memory and the
// kernel's arguments.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/wfa_b200.h"
#include "wfa_common.h"

namespace wfab {

// Control block of a stream, in mapped host memory.
struct ResidentCtl {
  unsigned long long tail;  // requests published (host)
  int32_t stop;             // host: finish what was published, then return
  int32_t idle_exits;       // kernel: launches that ended for want of requests
  int32_t gave_up;          // kernel: lane groups that hit group_polls
  int32_t pad;
};

// One request slot: lengths (read by the kernel as one int2); its bytes
// (pattern then text) are at arena + slot * seq_stride.
struct alignas(8) ResidentReq {
  int32_t n, m;
};

struct ResidentArgs {
  ResidentCtl* ctl;           // mapped
  const ResidentReq* reqs;    // mapped, cap slots
  const uint8_t* arena;       // mapped, cap x seq_stride bytes
  wfa_result_t* results;      // mapped, cap records
  uint8_t* cigars;            // mapped, cap x cig_stride bytes
  uint32_t* done;             // mapped, cap marks: (slot / cap) + 1 once slot's result is written
  int64_t cap, seq_stride, cig_stride;
  unsigned long long* head;   // device: tickets handed out
  unsigned long long* dtail;  // device: the doorbell's copy of ctl->tail
  int32_t* dstop;             // device: 1 stopped by the host, 2 idle
  int64_t idle_polls;         // doorbell polls without a new request before the kernel ends
  int64_t group_polls;        // a lane group's polls without work before it gives up
};

// Lanes per request: 8 or 32.  Blocks of kWarpsPerBlock warps.
cudaError_t launch_resident(const AlignParams& P, const ResidentArgs& R, int cls, int lanes, int blocks,
                            size_t smem, cudaStream_t st);
int occupancy_resident(int cls, int lanes, size_t smem);

}  // namespace wfab
