// Spatial shard of one transform over several ranks (fgt_shard.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "fgt_device.hpp"
#include "fgt_plan.hpp"

namespace fgtb {

struct ShardInfo {
  int nranks = 1, rank = 0;
  std::vector<int> owner;                // per box: the rank that computes it
  std::vector<uint64_t> key_lo;          // first Morton key of each rank (nranks + 1)
  std::vector<std::vector<int>> send;    // per peer: own cut-level mp slots the peer reads
  std::vector<std::vector<int>> recv;    // per peer: the peer's mp slots this rank reads
  long long owned_src = 0, owned_trg = 0;
  bool large_delta_idle = false;         // large-delta plans run on rank 0 only
};

// Keeps in H only the tasks of the boxes rank `rank` of `nranks` owns and
// fills the exchange lists; 0 on success.
int shard_filter(HostPlan& H, int nranks, int rank, ShardInfo& S);

// Copies the nslot listed cut-level mp expansions (device slot list) of the
// plan into buf (pack) or from buf into the plan's pool (unpack); buf holds
// nslot * nd * nexp complex doubles.
cudaError_t shard_mp_copy(DevicePlan& D, const int* d_slots, int nslot, double* buf, bool pack,
                          cudaStream_t st);

}  // namespace fgtb
