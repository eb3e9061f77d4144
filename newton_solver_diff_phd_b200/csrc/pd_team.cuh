// Lanes of the persistent batched launch.
//
// The grid is cut into lanes, fixed ranges of blocks; each lane is one team
// of a size class and takes instances of its class from the class queue, one
// after the other. Rank 0 of a lane claims the next instance and publishes
// it in the lane's slot; the lane's barrier hands it to the other ranks.
#pragma once

#include "pd_device.cuh"
#include "pd_kernels.h"

namespace pdb200 {

// Lane of this block (binary search over the lane starts) and its rank/size.
__device__ __forceinline__ int lane_of_block(const TeamLaunch& launch, Team& team) {
  int lo = 0, hi = launch.lanes;  // lane_start[lo] <= block < lane_start[hi]
  const int block = static_cast<int>(blockIdx.x);
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (launch.lane_start[mid] <= block) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  team.rank = block - launch.lane_start[lo];
  team.size = launch.lane_start[lo + 1] - launch.lane_start[lo];
  return lo;
}

// Every block of the lane: the lane's next instance, or -1 when its class
// queue is empty (or a barrier gave up). Uses the whole block.
__device__ __forceinline__ int next_instance(const TeamLaunch& launch, int lane, Team team, int* status) {
  __shared__ int s_instance;
  if (team.rank == 0 && threadIdx.x == 0) {
    const int cls = launch.lane_class[lane];
    const unsigned position = atomicAdd(&launch.class_head[cls], 1u);
    const int begin = launch.class_begin[cls];
    const int end = launch.class_begin[cls + 1];
    launch.lane_slot[lane] = static_cast<int>(position) < end - begin ? launch.class_order[begin + position] : -1;
  }
  if (!grid_sync(&launch.lane_barrier[lane], status, team.size, team.rank)) return -1;
  if (threadIdx.x == 0) s_instance = *reinterpret_cast<volatile int*>(&launch.lane_slot[lane]);
  __syncthreads();
  return s_instance;
}

// Every thread of the block: the next instance of the one-block class for a
// block whose own lane has run out of work, or -1 when that queue is empty.
__device__ __forceinline__ int claim_solo(const TeamLaunch& launch) {
  __shared__ int s_instance;
  __syncthreads();
  if (threadIdx.x == 0) {
    const int cls = launch.solo_class;
    const unsigned position = atomicAdd(&launch.class_head[cls], 1u);
    const int begin = launch.class_begin[cls];
    const int end = launch.class_begin[cls + 1];
    s_instance = static_cast<int>(position) < end - begin ? launch.class_order[begin + position] : -1;
  }
  __syncthreads();
  return s_instance;
}

// The next instance of this block: its lane's queue first; when that is
// empty, one-block instances on its own (a lane of one block needs no barrier).
__device__ __forceinline__ int next_work(const TeamLaunch& launch, int lane, Team lane_team, bool& solo, Team& team) {
  if (!solo) {
    const int instance = next_instance(launch, lane, lane_team, launch.status);
    if (instance >= 0) {
      team = lane_team;
      return instance;
    }
    if (launch.solo_class < 0 || launch.lane_class[lane] == launch.solo_class) return -1;
    solo = true;
  }
  team = Team{0, 1};
  return claim_solo(launch);
}

// Block-wide copy of an argument block (a multiple of 8 bytes) into shared memory.
template <typename T>
__device__ __forceinline__ void copy_arguments(const T* source, T* target) {
  static_assert(sizeof(T) % 8 == 0, "argument blocks are 8-byte multiples");
  const unsigned long long* from = reinterpret_cast<const unsigned long long*>(source);
  unsigned long long* to = reinterpret_cast<unsigned long long*>(target);
  for (int k = threadIdx.x; k < static_cast<int>(sizeof(T) / 8); k += blockDim.x) to[k] = from[k];
}

__device__ __forceinline__ const void* state_offset(const void* base, int f64, long long offset) {
  if (base == nullptr) return nullptr;
  return f64 ? static_cast<const void*>(static_cast<const double*>(base) + offset)
             : static_cast<const void*>(static_cast<const float*>(base) + offset);
}
__device__ __forceinline__ void* state_offset(void* base, int f64, long long offset) {
  if (base == nullptr) return nullptr;
  return f64 ? static_cast<void*>(static_cast<double*>(base) + offset) : static_cast<void*>(static_cast<float*>(base) + offset);
}

}  // namespace pdb200
