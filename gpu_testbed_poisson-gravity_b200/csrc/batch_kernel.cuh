// batch_kernel.cuh -- one persistent launch for a batch of patches with mixed
// ghost sizes (groups of equal ghost size, each in the reference layout).
//
// Work queue: the batch is cut into units -- 4 patches at ghost 1 (teams of
// 32 threads), 2 at ghost 2 (64), 1 at ghost 3-5 (96/128) -- numbered group
// by group with the largest cubes first.  Every CTA of 128 threads takes the
// next unit from a device counter (one atomicAdd per unit), solves it and
// asks again, so patches whose sweep counts differ by 10x still keep all SMs
// busy to the end.  Each patch runs sor_solve_patch with the team shape and
// lane mapping of one of the per-ghost-size variants: two rows per lane and
// half a column in FP32 (teams of 32-128 threads, as in the fastest FP32
// variants), one row and a whole column in FP64 (the two-row FP64 layouts hold
// more registers than three resident CTAs allow).  The fields equal those of
// a patch solved alone whenever the sweep counts do.
#pragma once

#include "sor_kernel.cuh"

namespace gpg {

constexpr int kBatchMaxGroups = 8;
constexpr int kBatchThreads = 128;

// lane layout of the batch kernel: (lanes per pair column, rows per lane)
template <typename T>
struct BatchLayout {
  static constexpr int Z = sizeof(T) == 4 ? 2 : 1;
  static constexpr int Y = sizeof(T) == 4 ? 2 : 1;
};

template <typename T, int G>
struct BatchUnit {
  using L = BatchLayout<T>;
  static constexpr int TEAM = SorCfg<T, G, L::Z, L::Y>::TEAM;
  static constexpr int TEAMS = kBatchThreads / TEAM;  // patches per unit
  static constexpr size_t team_bytes = SorSmem<T, G, L::Z, L::Y>::team_bytes;
  static constexpr size_t smem = TEAMS * team_bytes;
  static_assert(TEAMS >= 1, "team larger than a batch CTA");
};

template <typename T>
struct BatchArgs {
  SolveArgs<T> grp[kBatchMaxGroups];          // per-group pointers and constants
  int ghost[kBatchMaxGroups];
  int64_t unit_start[kBatchMaxGroups + 1];    // first unit of each group
  int ngroup;
  int64_t nunit;
  unsigned int *counter;                      // next unit; zero at launch
};

template <typename T, int G>
__device__ __forceinline__ void batch_unit(const SolveArgs<T> &a, int64_t unit_in_group, unsigned char *smem) {
  using U = BatchUnit<T, G>;
  const int team = threadIdx.x / U::TEAM;
  if (team >= U::TEAMS) return;  // warps left over (ghost 3: one warp of four)
  const int tid = threadIdx.x - team * U::TEAM;
  const int64_t P = unit_in_group * U::TEAMS + team;
  if (P >= a.npatch) return;     // last unit of a group may be partial
  using L = BatchLayout<T>;
  sor_solve_patch<T, G, false, L::Z, L::Y>(a, P, team, tid, smem + team * U::team_bytes);
}

// Resident CTAs per SM the register allocation must allow (the five ghost
// sizes share one kernel; without the bound the allocator pads the merged
// code far beyond what any single ghost size needs).
template <typename T>
constexpr int batch_min_blocks() { return sizeof(T) == 8 ? 3 : 4; }

template <typename T>
__global__ void __launch_bounds__(kBatchThreads, batch_min_blocks<T>()) sor_batch_kernel(const BatchArgs<T> b) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // the unit's group arguments are copied to shared memory once, so the
  // solver reads them with static offsets instead of indexing kernel params
  __shared__ SolveArgs<T> s_args;
  __shared__ int64_t s_unit, s_k;
  __shared__ int s_ghost;
  for (;;) {
    if (threadIdx.x == 0) {
      const int64_t u = (int64_t)atomicAdd(b.counter, 1u);
      s_unit = u;
      if (u < b.nunit) {
        int gi = 0;
        while (gi + 1 < b.ngroup && u >= b.unit_start[gi + 1]) ++gi;
        s_args = b.grp[gi];
        s_ghost = b.ghost[gi];
        s_k = u - b.unit_start[gi];
      }
    }
    __syncthreads();
    if (s_unit >= b.nunit) break;
    switch (s_ghost) {
      case 1: batch_unit<T, 1>(s_args, s_k, smem_raw); break;
      case 2: batch_unit<T, 2>(s_args, s_k, smem_raw); break;
      case 3: batch_unit<T, 3>(s_args, s_k, smem_raw); break;
      case 4: batch_unit<T, 4>(s_args, s_k, smem_raw); break;
      default: batch_unit<T, 5>(s_args, s_k, smem_raw); break;
    }
    __syncthreads();  // shared memory free for the next unit; s_* read by all
  }
}

template <typename T>
constexpr size_t batch_smem_bytes() {
  size_t m = BatchUnit<T, 1>::smem;
  m = m > BatchUnit<T, 2>::smem ? m : BatchUnit<T, 2>::smem;
  m = m > BatchUnit<T, 3>::smem ? m : BatchUnit<T, 3>::smem;
  m = m > BatchUnit<T, 4>::smem ? m : BatchUnit<T, 4>::smem;
  m = m > BatchUnit<T, 5>::smem ? m : BatchUnit<T, 5>::smem;
  return m;
}

template <typename T>
__host__ __device__ constexpr int batch_patches_per_unit(int g) {
  return g == 1 ? BatchUnit<T, 1>::TEAMS
                : g == 2 ? BatchUnit<T, 2>::TEAMS
                         : g == 3 ? BatchUnit<T, 3>::TEAMS : g == 4 ? BatchUnit<T, 4>::TEAMS : BatchUnit<T, 5>::TEAMS;
}

}  // namespace gpg
