// mldg_trsv_blk.cuh -- partitioned sparse unit-triangular solve.
//
// t = rhs - T_strict t for a strictly triangular factor T, in its "lower
// form" (an upper factor is walked with rows and columns reversed, so every
// dependency is an earlier row).  The rows are split into P contiguous
// blocks; CTA b solves block b by itself, walking the block's rows in steps:
// a step is a set of the block's rows on one global dependency level (or a
// part of one), so the rows of a step are independent of each other and one
// __syncthreads separates consecutive steps.  Dependencies are of two kinds:
//   * local: an earlier row of the same block, read from a shared-memory
//     ring of the block's last W solution values (indexed by the row's local
//     position mod W); the host checks that the slot has not been
//     overwritten yet (q >= end of the reading step - W), else the entry is
//     read as a remote one;
//   * remote: a row of an earlier block (or a local row older than the ring),
//     read from the exchange vector `cur` in global memory, which holds a
//     signalling-NaN sentinel until its row is solved; the reader re-polls,
//     bounded, while it sees the sentinel.
// With blocks that follow the matrix's own ordering, most dependencies are
// local: only rows on a block's upstream boundary wait for another CTA, and
// no grid-wide barrier is ever taken.  The CTAs take their block numbers from
// an atomic ticket in launch order, so a CTA only ever waits for blocks whose
// CTAs are already running (no co-residency assumption); the last CTA to
// finish resets the ticket for the next launch.
//
// Every step's plan (row descriptors, entry codes and values) is one
// 16-byte-aligned block in global memory, copied into a ring of kBlkD
// shared-memory stages by TMA bulk copies that one thread issues kBlkD-1
// steps ahead of use (an mbarrier per stage counts the bytes).  While a step
// is being solved, every thread already loads the right-hand side and the
// remote dependencies of its row of the next step, so the global-memory
// latency of those reads stays off the step-to-step critical path.
//
// Outputs: cur[orig] = t (the exchange vector, original row numbering);
// other[orig] = sentinel (the exchange vector of the previous solve, reset
// for the next one; it may be the right-hand side, each row reads its own
// entry before resetting it); out[orig] = alpha*t + beta*out[orig].
// Every wait is bounded: a sentinel poll gives up with 4020 (mldg_kernels.cuh
// wait_value), an mbarrier wait with 4021; a thread that gave up stops
// solving but keeps the barriers, and the issuing thread waits, bounded, for
// every stage copy still in flight before the CTA exits.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mldg_kernels.cuh"
#include "mldg_trsv_win.cuh"  // mbarrier and bulk-copy helpers

namespace mldg {

constexpr int kBlkThreads = 512;
constexpr int kBlkD = 4;   // plan stages in shared memory
constexpr int kBlkRE = 4;  // remote entries of the next row prefetched per thread

// Byte layout of one step's plan block (16-byte aligned):
//   int4 hdr        {nrows, nent, 0, 0}
//   int4 row[nrows] {orig, entry begin (within the step), entry count, local position}
//   int  code[nent] ring slot (>= 0) or -(orig + 1) of a remote dependency
//   T    val[nent]
__host__ __device__ inline int blk_al16(int x) { return (x + 15) & ~15; }
template <typename T>
__host__ __device__ inline int blk_off_val(int nrows, int nent) {
  return blk_al16(16 + 16 * nrows + 4 * nent);
}
template <typename T>
__host__ __device__ inline int blk_bytes(int nrows, int nent) {
  return blk_al16(blk_off_val<T>(nrows, nent) + (int)sizeof(T) * nent);
}

template <typename T>
struct BlkArgs {
  int nblocks;
  int wmask;          // ring size W - 1 (W a power of two)
  int stage_bytes;    // capacity of one stage (16-byte multiple)
  const int *bstep;   // [nblocks + 1] first step of each block
  const int2 *sdesc;  // [steps] {offset in 16-byte units, size in 16-byte units}
  const uint4 *plan;
  const T *src;    // right-hand side (original numbering)
  const T *scale;  // optional: rhs = scale[orig] * src[orig]
  T *cur;          // exchange vector: sentinel at launch, t afterwards
  T *other;        // optional: reset to the sentinel
  T *out;          // optional: out = alpha*t + beta*out
  T alpha, beta;
  int *ticket;     // [2] block ticket, CTAs finished (zero at launch, reset by the last CTA)
  int *err;
};

template <typename T>
__global__ void __launch_bounds__(kBlkThreads, 1) k_trsv_blk(BlkArgs<T> a) {
  extern __shared__ __align__(128) unsigned char smem[];
  typedef typename Bits<T>::U U;
  const U sent = (U)Sentinel<T>::bits;
  const int tid = threadIdx.x;
  T *ring = reinterpret_cast<T *>(smem);
  unsigned char *stages = smem + (size_t)(a.wmask + 1) * sizeof(T);
  uint64_t *full = reinterpret_cast<uint64_t *>(stages + (size_t)kBlkD * a.stage_bytes);
  __shared__ int s_blk;
  if (tid == 0) {
    s_blk = atomicAdd(&a.ticket[0], 1);
    for (int d = 0; d < kBlkD; ++d) mbar_init(&full[d], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int b = s_blk;
  const int s0 = a.bstep[b], ns = a.bstep[b + 1] - s0;
  bool live = true;
  int issued = 0, waited = 0;  // thread 0: stage copies issued / completed
  auto issue = [&](int k) {    // copy step s0 + k into stage k % kBlkD
    const int2 dsc = a.sdesc[s0 + k];
    uint64_t *bar = &full[k % kBlkD];
    mbar_expect_tx(bar, (unsigned)dsc.y * 16u);
    tma_bulk_g2s(stages + (size_t)(k % kBlkD) * a.stage_bytes, a.plan + dsc.x, (unsigned)dsc.y * 16u, bar);
    ++issued;
  };
  auto stage_ready = [&](int k) {  // bounded wait for the stage of step s0 + k (once per step)
    if (!live) return;
    if (!mbar_wait(&full[k % kBlkD], (unsigned)((k / kBlkD) & 1))) {
      atomicExch(a.err, 4021);
      live = false;
    } else {
      ++waited;
    }
  };
  // the next step's row of this thread: original row, right-hand side and
  // raw bits of its first kBlkRE remote dependencies (the sentinel if not yet written)
  int n_orig = -1;
  T n_src = T(0), n_sc = T(1), n_out = T(0);
  U n_raw[kBlkRE];
  auto prefetch = [&](int k) {  // step s0 + k, whose stage is ready
    n_orig = -1;
    if (!live) return;
    const unsigned char *st = stages + (size_t)(k % kBlkD) * a.stage_bytes;
    const int4 hdr = *reinterpret_cast<const int4 *>(st);
    if (tid >= hdr.x) return;
    const int4 rw = reinterpret_cast<const int4 *>(st + 16)[tid];
    const int *code = reinterpret_cast<const int *>(st + 16 + 16 * hdr.x);
    n_orig = rw.x;
    // loads only: nothing here waits for them (they are used in the next step)
    n_src = a.src[rw.x];
    if (a.scale) n_sc = a.scale[rw.x];
    if (a.out && a.beta != T(0)) n_out = a.out[rw.x];
#pragma unroll
    for (int e = 0; e < kBlkRE; ++e) {
      const int c = e < rw.z ? code[rw.y + e] : 0;
      n_raw[e] = c < 0 ? Bits<T>::load(a.cur + (-c - 1)) : (U)0;
    }
  };
  if (tid == 0)
    for (int k = 0; k < kBlkD - 1 && k < ns; ++k) issue(k);
  if (ns > 0) {
    stage_ready(0);
    prefetch(0);
  }
  for (int k = 0; k < ns; ++k) {
    // the stage of step k - 1 is free: every thread is past the barrier
    if (tid == 0 && live && k + kBlkD - 1 < ns) issue(k + kBlkD - 1);
    if (live) {
      const unsigned char *st = stages + (size_t)(k % kBlkD) * a.stage_bytes;
      const int4 hdr = *reinterpret_cast<const int4 *>(st);
      const int4 *rows = reinterpret_cast<const int4 *>(st + 16);
      const int *code = reinterpret_cast<const int *>(st + 16 + 16 * hdr.x);
      const T *val = reinterpret_cast<const T *>(st + blk_off_val<T>(hdr.x, hdr.y));
      for (int r = tid; r < hdr.x; r += kBlkThreads) {
        const int4 rw = rows[r];
        const bool pre = r == tid && n_orig == rw.x;
        const T rhs = pre ? (a.scale ? n_sc * n_src : n_src)
                          : (a.scale ? a.scale[rw.x] * a.src[rw.x] : a.src[rw.x]);
        T acc = T(0);
        for (int e = 0; e < rw.z; ++e) {
          const int c = code[rw.y + e];
          T dv;
          if (c >= 0)
            dv = ring[c];
          else if (pre && e < kBlkRE && n_raw[e] != sent)
            dv = Bits<T>::from(n_raw[e]);
          else
            dv = wait_value<T>(a.cur + (-c - 1), a.err);
          acc = fma(val[rw.y + e], dv, acc);
        }
        const T t = rhs - acc;
        ring[rw.w & a.wmask] = t;
        Bits<T>::store(a.cur + rw.x, Bits<T>::canon(t));
        if (a.other) Bits<T>::store(a.other + rw.x, Sentinel<T>::value());
        if (a.out) {
          if (a.beta == T(0))
            a.out[rw.x] = a.alpha * t;
          else
            a.out[rw.x] = fma(a.beta, pre ? n_out : a.out[rw.x], a.alpha * t);
        }
      }
    }
    // the next step's stage, then this thread's row of it
    if (k + 1 < ns) {
      stage_ready(k + 1);
      prefetch(k + 1);
    }
    __syncthreads();
  }
  // after a wait that gave up, no bulk copy may still be writing this CTA's
  // shared memory when it exits: wait (bounded) for every one issued
  if (tid == 0)
    for (int k = waited; k < issued; ++k) mbar_wait(&full[k % kBlkD], (unsigned)((k / kBlkD) & 1));
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(&a.ticket[1], 1) == a.nblocks - 1) {
      a.ticket[0] = 0;
      a.ticket[1] = 0;
      __threadfence();
    }
  }
}

}  // namespace mldg
