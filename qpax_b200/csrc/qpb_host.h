// qpb_host.h -- launch planning shared by the uniform entry points
// (qpb_capi.cu) and the packed-batch plans (qpb_plan.cu).
#pragma once
#include <stddef.h>

#include "../../include/qpb.h"
#include "qpb_params.h"

namespace qpb {

constexpr size_t kCounterBytes = 256;  // work counter slot at the head of every workspace
constexpr int kMaxN = 256;

// One persistent launch: kernel, shape, shared memory, arena and workspace.
struct Plan {
  const void* fn;
  int NT, threads, teams, grid;
  size_t arena_bytes, smem_bytes, ws_bytes;
  int in_smem;
  int gstage_rows;  // rows of G per shared-memory chunk (arena in global memory), 0: none
};

int warp_np(const qpb_dims& d);
int chunks_for(int k);
int make_plan(int op, const qpb_dims& d, const qpb_config& cfg, Plan* pl);
qpb_config resolve_config(const qpb_config* c);
int check_common(int op, const qpb_dims* d, const qpb_config* cfg);
bool ok_ptr(const void* p, long count);

}  // namespace qpb
