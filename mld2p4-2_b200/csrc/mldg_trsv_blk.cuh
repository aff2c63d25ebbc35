// mldg_trsv_blk.cuh -- partitioned sparse unit-triangular solve.
//
// t = rhs - T_strict t for a strictly triangular factor T, in its "lower
// form" (an upper factor is walked with rows and columns reversed, so every
// dependency is an earlier row).  The rows are split into P contiguous
// blocks; CTA b solves block b by itself, walking the block's rows in steps:
// a step is a set of the block's rows on one global dependency level (or a
// part of one), so the rows of a level are independent of each other and a
// barrier of the solving warps separates consecutive levels.  Dependencies
// are of two kinds:
//   * local: an earlier row of the same block, read from a shared-memory
//     ring of the block's last W solution values (indexed by the row's local
//     position mod W); the host checks that the slot cannot be overwritten
//     while the reading level runs (q >= end of the reading level - W), else
//     the entry is read as a remote one;
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
// 16-byte-aligned block in global memory.  The CTA splits into two roles so
// that a step touches only shared memory on its critical path:
//   * kBlkLoadWarps loader warps take the steps in turn (loader w the steps
//     w, w + kBlkLoadWarps, ...), up to kBlkD steps ahead of the solve: each
//     copies its step's plan into a stage of a kBlkD-deep shared-memory ring
//     by a TMA bulk copy, gathers the step's right-hand sides (and previous
//     outputs when beta != 0) into the stage's aux buffer, and polls the
//     step's remote dependencies on `cur` (bounded) into the aux buffer as
//     they land; then it publishes the stage (ready[stage] = step);
//   * the other warps solve the steps in order from the stage and the ring
//     and separate levels by a named barrier (steps that continue the same
//     level need none: their rows are independent), and thread 0 releases
//     each consumed stage to the loaders (done = step + 1).
// A block's time is thus the hand-offs along its upstream chain plus one
// shared-memory step per level, instead of a global-memory round trip per
// level.
//
// Outputs: cur[orig] = t (the exchange vector, original row numbering);
// other[orig] = sentinel (the exchange vector of the previous solve, reset
// for the next one; it may be the right-hand side, each row's loader reads
// its entry before the row is solved and reset); out[orig] = alpha*t +
// beta*out[orig].  Every wait is bounded: a sentinel poll gives up with
// 4020, an mbarrier or stage wait with 4021; after a give-up the roles stop
// loading and solving but keep stepping through the named barriers, and
// each loader waits, bounded, for the bulk copies it issued before the CTA
// exits.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mldg_kernels.cuh"
#include "mldg_trsv_win.cuh"  // mbarrier and bulk-copy helpers

namespace mldg {

constexpr int kBlkThreads = 512;
constexpr int kBlkLoadWarps = 8;                           // loader warps (the last ones)
constexpr int kBlkSolve = kBlkThreads - 32 * kBlkLoadWarps;  // solving threads
constexpr int kBlkD = 8;                                   // plan stages in shared memory
constexpr int kBlkLoadU = 4;                               // loads per lane issued together by a loader

// Byte layout of one step's plan block (16-byte aligned):
//   int4 hdr        {nrows, nent, same level as the block's previous step, 0}
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
// dynamic shared memory: ring, kBlkD plan stages, kBlkD aux buffers, mbarriers
template <typename T>
__host__ __device__ inline size_t blk_smem(int W, int stage_bytes, int aux_cap) {
  return (size_t)W * sizeof(T) + (size_t)kBlkD * stage_bytes + (size_t)kBlkD * aux_cap * sizeof(T) + 8 * kBlkD;
}

template <typename T>
struct BlkArgs {
  int nblocks;
  int wmask;          // ring size W - 1 (W a power of two)
  int stage_bytes;    // capacity of one stage (16-byte multiple)
  int aux_cap;        // aux elements per stage: >= 2 * nrows + nent of every step
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

__device__ __forceinline__ int blk_ld_volatile(const int *p) { return *reinterpret_cast<const volatile int *>(p); }
__device__ __forceinline__ void blk_st_volatile(int *p, int v) { *reinterpret_cast<volatile int *>(p) = v; }
constexpr int kBlkSolveWarps = kBlkSolve / 32;
constexpr int kBlkWaitLimit = 1 << 24;  // polls of a shared-memory flag before giving up

// bounded spin until *flag >= target (or the CTA's error flag is set)
__device__ __forceinline__ bool blk_wait_ge(const int *flag, int target, const int *s_err) {
  for (int it = 0; it < kBlkWaitLimit; ++it) {
    if (blk_ld_volatile(flag) >= target) return true;
    if (blk_ld_volatile(s_err)) return false;
    if ((it & 63) == 63) __nanosleep(32);
  }
  return false;
}

template <typename T>
__global__ void __launch_bounds__(kBlkThreads, 1) k_trsv_blk(BlkArgs<T> a) {
  extern __shared__ __align__(128) unsigned char smem[];
  typedef typename Bits<T>::U U;
  const U sent = (U)Sentinel<T>::bits;
  const int tid = threadIdx.x, lane = tid & 31;
  T *ring = reinterpret_cast<T *>(smem);
  unsigned char *stages = smem + (size_t)(a.wmask + 1) * sizeof(T);
  T *aux = reinterpret_cast<T *>(stages + (size_t)kBlkD * a.stage_bytes);
  uint64_t *full = reinterpret_cast<uint64_t *>(aux + (size_t)kBlkD * a.aux_cap);
  // s_ready[st]: the step whose plan and aux data the stage holds; s_cons[st]:
  // solving warps that have consumed the stage, over all its uses; s_lvl:
  // solving warps arrived at level barriers, over all of them
  __shared__ int s_blk, s_err, s_lvl;
  __shared__ int s_ready[kBlkD], s_cons[kBlkD];
  if (tid == 0) {
    s_blk = atomicAdd(&a.ticket[0], 1);
    s_err = 0;
    s_lvl = 0;
    for (int d = 0; d < kBlkD; ++d) {
      s_ready[d] = -1;
      s_cons[d] = 0;
      mbar_init(&full[d], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int b = s_blk;
  const int s0 = a.bstep[b], ns = a.bstep[b + 1] - s0;
  const bool has_out = a.out && a.beta != T(0);
  auto give_up = [&](int code) {
    if (!blk_ld_volatile(&s_err)) atomicExch(a.err, code);
    blk_st_volatile(&s_err, 1);
  };
  if (tid >= kBlkSolve) {
    // ---- loader warps: step k by warp k % kBlkLoadWarps, into stage k % kBlkD ----
    const int lw = (tid - kBlkSolve) >> 5;
    int issued = 0, waited = 0;  // lane 0: this warp's bulk copies issued / completed
    bool live = true;
    for (int k = lw; k < ns && live; k += kBlkLoadWarps) {
      const int st = k % kBlkD;
      // the stage is free once every solving warp has consumed step k - kBlkD
      if (!blk_wait_ge(&s_cons[st], kBlkSolveWarps * (k / kBlkD), &s_err)) {
        if (lane == 0) give_up(4021);
        live = false;
        break;
      }
      if (lane == 0) {
        const int2 dsc = a.sdesc[s0 + k];
        mbar_expect_tx(&full[st], (unsigned)dsc.y * 16u);
        tma_bulk_g2s(stages + (size_t)st * a.stage_bytes, a.plan + dsc.x, (unsigned)dsc.y * 16u, &full[st]);
        ++issued;
      }
      const bool got = mbar_wait(&full[st], (unsigned)((k / kBlkD) & 1));
      if (lane == 0 && got) ++waited;
      if (!got) {
        if (lane == 0) give_up(4021);
        live = false;
        break;
      }
      const unsigned char *sp = stages + (size_t)st * a.stage_bytes;
      const int4 hdr = *reinterpret_cast<const int4 *>(sp);
      const int4 *rows = reinterpret_cast<const int4 *>(sp + 16);
      const int *code = reinterpret_cast<const int *>(sp + 16 + 16 * hdr.x);
      T *ax = aux + (size_t)st * a.aux_cap;
      // the step's right-hand sides (and old outputs), kBlkLoadU rows per lane
      // loaded before any is stored, so a step costs one memory latency
      for (int r0 = 0; r0 < hdr.x; r0 += 32 * kBlkLoadU) {
        T sv[kBlkLoadU], ov[kBlkLoadU];
#pragma unroll
        for (int u = 0; u < kBlkLoadU; ++u) {
          const int r = r0 + u * 32 + lane;
          sv[u] = ov[u] = T(0);
          if (r < hdr.x) {
            const int o = rows[r].x;
            sv[u] = a.scale ? a.scale[o] * a.src[o] : a.src[o];
            if (has_out) ov[u] = a.out[o];
          }
        }
#pragma unroll
        for (int u = 0; u < kBlkLoadU; ++u) {
          const int r = r0 + u * 32 + lane;
          if (r < hdr.x) {
            ax[r] = sv[u];
            if (has_out) ax[hdr.x + r] = ov[u];
          }
        }
      }
      // remote dependencies: kBlkLoadU loads per lane issued together, a
      // missing value re-polled
      for (int e0 = 0; e0 < hdr.y; e0 += 32 * kBlkLoadU) {
        U rv[kBlkLoadU];
        int cv[kBlkLoadU];
#pragma unroll
        for (int u = 0; u < kBlkLoadU; ++u) {
          const int e = e0 + u * 32 + lane;
          cv[u] = e < hdr.y ? code[e] : 0;
          rv[u] = cv[u] < 0 ? Bits<T>::load(a.cur + (-cv[u] - 1)) : (U)0;
        }
#pragma unroll
        for (int u = 0; u < kBlkLoadU; ++u) {
          const int e = e0 + u * 32 + lane;
          if (cv[u] < 0)
            ax[2 * hdr.x + e] = rv[u] != sent ? Bits<T>::from(rv[u]) : wait_value<T>(a.cur + (-cv[u] - 1), a.err);
        }
      }
      __syncwarp();
      if (ld_relaxed_u32(a.err) != 0u) {
        if (lane == 0) blk_st_volatile(&s_err, 1);
        live = false;
        break;
      }
      __threadfence_block();
      if (lane == 0) blk_st_volatile(&s_ready[st], k);
    }
    // no bulk copy may still be writing shared memory when the CTA exits
    if (lane == 0)
      for (int k = lw + waited * kBlkLoadWarps; waited < issued; ++waited, k += kBlkLoadWarps)
        mbar_wait(&full[k % kBlkD], (unsigned)((k / kBlkD) & 1));
  } else {
    // ---- solving warps: the steps in order ----
    int nbar = 0;  // level barriers passed
    for (int k = 0; k < ns; ++k) {
      const int st = k % kBlkD;
      if (!blk_wait_ge(&s_ready[st], k, &s_err)) {
        if (lane == 0) give_up(4021);
        break;
      }
      // the stage's bulk copy has completed (its loader saw the same phase)
      if (!mbar_wait(&full[st], (unsigned)((k / kBlkD) & 1))) {
        if (lane == 0) give_up(4021);
        break;
      }
      __threadfence_block();
      const unsigned char *sp = stages + (size_t)st * a.stage_bytes;
      const int4 hdr = *reinterpret_cast<const int4 *>(sp);
      if (!hdr.z && k > 0) {
        // a new level: every warp's rows of the previous level are in the ring
        __syncwarp();
        ++nbar;
        if (lane == 0) {
          __threadfence_block();
          atomicAdd(&s_lvl, 1);
        }
        if (!blk_wait_ge(&s_lvl, nbar * kBlkSolveWarps, &s_err)) {
          if (lane == 0) give_up(4021);
          break;
        }
        __threadfence_block();
      }
      const int4 *rows = reinterpret_cast<const int4 *>(sp + 16);
      const int *code = reinterpret_cast<const int *>(sp + 16 + 16 * hdr.x);
      const T *val = reinterpret_cast<const T *>(sp + blk_off_val<T>(hdr.x, hdr.y));
      const T *ax = aux + (size_t)st * a.aux_cap;
      for (int r = tid; r < hdr.x; r += kBlkSolve) {
        const int4 rw = rows[r];
        T acc = T(0);
        for (int e = 0; e < rw.z; ++e) {
          const int c = code[rw.y + e];
          const T dv = c >= 0 ? ring[c] : ax[2 * hdr.x + rw.y + e];
          acc = fma(val[rw.y + e], dv, acc);
        }
        const T t = ax[r] - acc;
        ring[rw.w & a.wmask] = t;
        Bits<T>::store(a.cur + rw.x, Bits<T>::canon(t));
        if (a.other) Bits<T>::store(a.other + rw.x, Sentinel<T>::value());
        if (a.out) a.out[rw.x] = has_out ? fma(a.beta, ax[hdr.x + r], a.alpha * t) : a.alpha * t;
      }
      // this warp is done with the stage
      __syncwarp();
      if (lane == 0) atomicAdd(&s_cons[st], 1);
    }
  }
  __syncthreads();
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
