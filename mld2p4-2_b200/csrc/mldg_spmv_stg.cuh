// mldg_spmv_stg.cuh -- staged SELL-32 SpMV and Jacobi sweep: the matrix
// reaches the SMs by one TMA bulk copy per tile, not by per-thread loads.
//
// The operator's SELL-32 copy (slices of 32 rows stored slot by slot, see
// k_spmv_sell) is cut on the host, once, into tiles of consecutive slices,
// and every tile is packed into one 16-byte aligned block: a header, the
// slot offsets of its slices, its column offsets and its values.  Every warp
// of a persistent grid walks its own tiles (tile t goes to warp t mod (warps
// of the grid)) through a ring of `stages` shared-memory stages of its own:
// lane 0 copies a tile's whole block with one cp.async.bulk into a stage
// whose mbarrier counts the bytes, `stages - 1` tiles ahead of the tile the
// warp computes.  The warp computes StgRows slices at a time, one row per
// lane and slice: it loads the rows' vector operands (b, the old output, the
// Jacobi diagonal and iterate) with plain coalesced loads first, then, per
// batch of kStgU slots of every row, the column offsets and values from
// shared memory and the gathers, then the sums.  The bytes of the matrix are
// in flight a tile ahead on every warp, whatever the dependent load chain of
// a row.  A row's slots are summed in stored order from zero, padding
// included, exactly as k_spmv_sell / k_jacobi_sell (one slice per warp
// iteration) sum them: the results are bit for bit theirs.
//
// Packed block of a tile (all parts 16-byte aligned):
//   int  hdr[4]            {slices, slots, byte offset of col, byte offset of val}
//   int  soff[slices + 1]  slot offsets of the tile's slices, from its first slot
//   CI   col[slots]        int16 offsets from the row, or int32 columns
//   V    val[slots]        values (FP16 row-scaled values in the FP16 form)
// Tile descriptor: int4 {first slice, end slice, block offset / 16, block bytes / 16}.
//
// Every wait is bounded: an mbarrier wait that gives up sets error 4021 and
// the warp stops; lane 0 then waits (bounded) for every copy it issued before
// the warp exits.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mldg_kernels.cuh"
#include "mldg_trsv_win.cuh"  // mbar_init, mbar_expect_tx, mbar_wait, tma_bulk_g2s

namespace mldg {

constexpr int kStgWarps = 16;               // warps per CTA, each with its own ring
constexpr int kStgThreads = 32 * kStgWarps;
constexpr int kStgStages = 2;               // stages per warp the tiles are sized for
constexpr int kStgMaxStages = 4;            // MLDG_STG_S may ask for up to this many (fewer when they do not fit)
constexpr size_t kStgSmemMax = 227 * 1024;  // dynamic shared memory a CTA may opt in to
constexpr int kStgU = 8;                    // slots per row whose loads and gathers are issued together
// tile budget: kStgStages blocks for each of a CTA's warps, beside the mbarriers
constexpr int kStgBlockMax = (int)(((kStgSmemMax - 1024) / (kStgWarps * kStgStages)) & ~(size_t)15);

__host__ __device__ inline int stg_al16(int x) { return (x + 15) & ~15; }

// slices a warp holds in flight: 4 with 4-byte vectors, 2 with 8-byte ones
template <typename T>
struct StgRows {
  static constexpr int value = sizeof(T) == 8 ? 2 : 4;
};

// dynamic shared memory of a launch: every warp's stages and mbarriers
__host__ inline size_t stg_smem(int stages, int block_bytes) {
  return (size_t)kStgWarps * ((size_t)stages * block_bytes + 8 * (size_t)stages);
}

struct StgArgs {
  int ntiles, nr, stages, block_bytes;
  const int4 *tiles;
  const uint4 *pk;  // packed blocks
  const float *rs;  // FP16 values: row scales
  int *err;
};

// The tile loop of one warp: tile_fn(tile descriptor, its stage) runs on all
// 32 lanes once the tile's block has landed.
template <typename F>
__device__ __forceinline__ void stg_run(const StgArgs &a, F tile_fn) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = a.stages;
  unsigned char *ring = smem + (size_t)w * S * a.block_bytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + (size_t)kStgWarps * S * a.block_bytes) + (size_t)w * S;
  const int gw = blockIdx.x * kStgWarps + w, nw = gridDim.x * kStgWarps;
  auto issue = [&](int t, int s) {  // lane 0
    const int4 d = a.tiles[t];
    mbar_expect_tx(&full[s], (unsigned)d.w * 16u);
    tma_bulk_g2s(ring + (size_t)s * a.block_bytes, a.pk + d.z, (unsigned)d.w * 16u, &full[s]);
  };
  int issued = 0;  // lane 0: tiles of this warp whose copies were issued
  if (lane == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int s = 0; s < S && gw + s * nw < a.ntiles; ++s, ++issued) issue(gw + s * nw, s);
  }
  __syncwarp();
  int k = 0;
  for (; gw + k * nw < a.ntiles; ++k) {
    const int s = k % S;
    if (!mbar_wait(&full[s], (unsigned)((k / S) & 1))) {
      if (lane == 0) atomicExch(a.err, 4021);
      break;
    }
    tile_fn(a.tiles[gw + k * nw], ring + (size_t)s * a.block_bytes);
    __syncwarp();
    const int kn = k + S;
    if (lane == 0 && gw + kn * nw < a.ntiles) {
      // the warp's reads of this stage before the copy that overwrites it
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(gw + kn * nw, s);
      ++issued;
    }
  }
  // after a wait that gave up: every copy issued must land before the warp exits
  if (lane == 0)
    for (int j = k; j < issued; ++j) mbar_wait(&full[j % S], (unsigned)((j / S) & 1));
}

// The rows of one staged tile, StgRows slices at a time, one row per lane:
// pre(row) loads the row's vector operands, then the row's slots are summed
// (val * gather(col), in stored order, the loads of kStgU slots of every
// slice issued before their sums), then done(row, sum, operands).
template <typename T, typename V, typename CI, typename P, typename G, typename D>
__device__ __forceinline__ void stg_slices(const int4 d, const unsigned char *st, int nr,
                                           const float *__restrict__ rs, P pre, G gather, D done) {
  constexpr int R = StgRows<T>::value;
  const int lane = threadIdx.x & 31;
  const int *hdr = reinterpret_cast<const int *>(st);
  const int nsl = hdr[0];
  const int *so = hdr + 4;
  const CI *cs = reinterpret_cast<const CI *>(st + hdr[2]);
  const V *vs = reinterpret_cast<const V *>(st + hdr[3]);
  using Ops = decltype(pre(0));
  for (int q0 = 0; q0 < nsl; q0 += R) {
    int e[R], e1[R], row[R];
    T acc[R];
    Ops ops[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int q = q0 + r;
      const bool ok = q < nsl;
      row[r] = ((d.x + q) << 5) + lane;
      e[r] = ok ? so[q] + lane : 0;
      e1[r] = ok ? so[q + 1] : 0;
      acc[r] = T(0);
      if (ok && row[r] < nr) ops[r] = pre(row[r]);
    }
    for (;;) {
      bool more = false;
#pragma unroll
      for (int r = 0; r < R; ++r) more |= e[r] < e1[r];
      if (!more) break;
      T vv[R][kStgU], xv[R][kStgU];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int u = 0; u < kStgU; ++u) {
          const int k = e[r] + 32 * u;
          const bool ok = k < e1[r];
          vv[r][u] = ok ? ldval<T>(vs, k) : T(0);
          xv[r][u] = ok ? gather(sell_col(cs, k, row[r])) : T(0);
        }
#pragma unroll
      for (int r = 0; r < R; ++r) {
#pragma unroll
        for (int u = 0; u < kStgU; ++u)
          if (e[r] + 32 * u < e1[r]) acc[r] = fma(vv[r][u], xv[r][u], acc[r]);
        e[r] += 32 * kStgU;
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (q0 + r < nsl && row[r] < nr) done(row[r], row_scaled<T, V>(acc[r], rs, row[r]), ops[r]);
  }
}

template <typename T>
struct StgOps2 {
  T p, q;
};
template <typename T>
struct StgOps4 {
  T d, x, ty, o;
};

// out = a1*(A v) + a0*b + a2*out  (k_spmv_sell's operation)
template <typename T, typename V, typename CI>
__global__ void __launch_bounds__(kStgThreads, 1) k_spmv_stg(StgArgs a, const T *__restrict__ v, T a1,
                                                             const T *__restrict__ b, T a0, T *out, T a2) {
  stg_run(a, [&](const int4 d, const unsigned char *st) {
    stg_slices<T, V, CI>(
        d, st, a.nr, a.rs,
        [&](int row) {
          StgOps2<T> o;
          o.p = b ? b[row] : T(0);
          o.q = a2 != T(0) ? out[row] : T(0);
          return o;
        },
        [&](int j) { return __ldg(v + j); },
        [&](int row, T s, const StgOps2<T> &o) {
          T r = a1 * s;
          if (b) r = fma(a0, o.p, r);
          if (a2 != T(0)) r = fma(a2, o.q, r);
          out[row] = r;
        });
  });
}

// the Jacobi sweep of k_jacobi_sell
template <typename T, typename V, typename CI>
__global__ void __launch_bounds__(kStgThreads, 1) k_jacobi_stg(StgArgs a, const T *__restrict__ d,
                                                               const T *__restrict__ x, const T *__restrict__ ty,
                                                               int first, T omega, T alpha, T beta, T *out) {
  const bool use_ty = !first && omega != T(1);
  auto pre = [&](int row) {
    StgOps4<T> o;
    o.d = d[row];
    o.x = x[row];
    o.ty = use_ty ? ty[row] : T(0);
    o.o = beta != T(0) ? out[row] : T(0);
    return o;
  };
  auto done = [&](int row, T s, const StgOps4<T> &o) {
    out[row] = jac_row(o.d, o.x, s, o.ty, first != 0, omega, alpha, beta, o.o);
  };
  stg_run(a, [&](const int4 dd, const unsigned char *st) {
    if (first == 2)
      stg_slices<T, V, CI>(dd, st, a.nr, a.rs, pre, [&](int j) { return omega * __ldg(x + j); }, done);
    else if (first)
      stg_slices<T, V, CI>(dd, st, a.nr, a.rs, pre, [&](int j) { return omega * (__ldg(d + j) * __ldg(x + j)); },
                           done);
    else
      stg_slices<T, V, CI>(dd, st, a.nr, a.rs, pre, [&](int j) { return __ldg(ty + j); }, done);
  });
}

}  // namespace mldg
