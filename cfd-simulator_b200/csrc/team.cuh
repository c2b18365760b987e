// team.cuh - a thread-block cluster working as one team: deterministic
// reductions (fixed-order warp trees, then ranks in order through DSMEM) and
// the std::max/min/clamp semantics the reference's arithmetic relies on.
#pragma once

#include <cooperative_groups.h>

#include <cmath>

namespace cfdb {

namespace cg = cooperative_groups;

#ifndef DEV
#define DEV __device__ __forceinline__
#endif

// std::max / std::min / std::clamp semantics, NaN behaviour included.
DEV double smax(double a, double b) { return (a < b) ? b : a; }
DEV double smin(double a, double b) { return (b < a) ? b : a; }
DEV double sclamp(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

constexpr int kMaxWarps = 32;
constexpr int kRedSlots = 8;

struct Shared {
  double warp[kMaxWarps][kRedSlots];
  double part[2][kRedSlots];
  double result[kRedSlots];
  // the chained k/omega sweeps: one mbarrier per ring slot, completed by the
  // bytes of a row the previous stage pushes (st.async), and the count of
  // rows the next stage has released, written by it through DSMEM; set up
  // at kernel start
  unsigned long long chainBar[4];
  unsigned chainAck;
  unsigned chainNever;  // stays 0: the wait test's condition
  // the split pressure CG: the barrier the neighbouring CTAs' halo rows
  // complete each iteration, its phase count and the bytes it expects
  unsigned long long haloBar;
  unsigned haloPhase;
  unsigned haloBytes;
};

struct Team {
  cg::cluster_group cl;
  unsigned rank, R;
  int tid, T;
  int c0, c1;
  int buf;
};

// ---- reductions -------------------------------------------------------------

enum RedOp : int { kSum = 0, kMax = 1 };

DEV double combine(int op, double a, double b) { return (op == kMax) ? smax(a, b) : a + b; }
DEV double identity(int op) { return (op == kMax) ? -INFINITY : 0.0; }

/// Reduce K values over every thread of the cluster. The result is the same
/// bits in every thread of every CTA: a fixed warp tree, the warp partials
/// in warp order, then warp 0 reads the ranks' partials in rank order from
/// distributed shared memory and reduces them with the same tree.
/// Contains two __syncthreads and one cluster barrier. (Having every warp
/// read the ranks' partials instead, to drop the second __syncthreads,
/// measured 0.65 us slower per reduction at 16 CTAs.)
template <int K>
DEV void teamReduce(Team& t, Shared& sh, double (&v)[K], const int (&op)[K]) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = (t.T + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      v[k] = combine(op[k], v[k], __shfl_down_sync(0xffffffffu, v[k], off));
    }
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) sh.warp[warp][k] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double a = (lane < nwarps) ? sh.warp[lane][k] : identity(op[k]);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) a = combine(op[k], a, __shfl_down_sync(0xffffffffu, a, off));
      if (lane == 0) sh.part[t.buf][k] = a;
    }
  }
  t.cl.sync();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double a = identity(op[k]);
      if (lane < static_cast<int>(t.R)) a = *t.cl.map_shared_rank(&sh.part[t.buf][k], lane);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) a = combine(op[k], a, __shfl_down_sync(0xffffffffu, a, off));
      if (lane == 0) sh.result[k] = a;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = sh.result[k];
  t.buf ^= 1;
}

}  // namespace cfdb
