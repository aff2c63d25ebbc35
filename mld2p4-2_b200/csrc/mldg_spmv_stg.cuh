// mldg_spmv_stg.cuh -- staged CSR SpMV and Jacobi sweep: the matrix and the
// row vectors reach the SMs by TMA bulk copies, not by per-thread loads.
//
// The rows of an operator are cut (on the host, once) into tiles of
// consecutive rows: at most rmax rows and emax entries each, described by
// int4 {first row, end row, first entry, end entry}, sized so that one
// warp's share of shared memory holds `stages` of them.  Every warp of a
// persistent grid walks its own tiles (tile t goes to warp t mod (warps of
// the grid)) through its own ring of `stages` shared-memory stages: lane 0
// copies a whole tile -- its slice of the row offsets, of the column indices,
// of the values and of up to kStgVecs row vectors (the right-hand side b,
// the output's old values, the Jacobi diagonal and iterate) -- with
// cp.async.bulk into a stage whose mbarrier counts the bytes, `stages - 1`
// tiles ahead of the one the warp computes.  The warp computes a tile's rows
// from shared memory, TPR lanes per row and StgRows rows per lane group at a
// time, every lane issuing the gathers of kStgU entries of each of its rows
// before it sums any of them.  So the DRAM stream is a few large contiguous
// requests per tile in flight on every warp, independent of the dependent
// load chain (row offsets, then entries, then gathers) that limits the
// per-thread CSR and SELL kernels, and the gathers of many rows overlap.
// A row's entries are summed per lane in stored order and the lanes combined
// by a butterfly, exactly as k_spmv / k_jacobi with the same lanes per row
// do: the results are bit for bit theirs.
//
// A bulk copy needs a 16-byte aligned source and a size that is a multiple
// of 16 bytes: every slice is widened to 16-byte boundaries (the arrays are
// cudaMalloc'd with slack past their end, so the widened slices stay inside
// the allocations), and the warp indexes the staged slices relative to the
// widened starts.  Before lane 0 refills a stage, the warp's reads of it are
// ordered before the asynchronous copy by __syncwarp and a proxy fence.
//
// Every wait is bounded: an mbarrier wait that gives up sets error 4021 and
// the warp stops; lane 0 then waits (bounded) for every copy it issued
// before the warp exits.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mldg_kernels.cuh"
#include "mldg_trsv_win.cuh"  // mbar_init, mbar_expect_tx, mbar_wait, tma_bulk_g2s

namespace mldg {

constexpr int kStgWarps = 16;               // warps per CTA, each with its own ring
constexpr int kStgThreads = 32 * kStgWarps;
constexpr int kStgVecs = 4;                 // row vectors staged per tile (at most)
constexpr int kStgStages = 2;     // stages per warp the plans are sized for
constexpr int kStgMaxStages = 4;  // MLDG_STG_S may ask for up to this many (fewer when they do not fit)
constexpr size_t kStgSmemMax = 227 * 1024;  // dynamic shared memory a CTA may opt in to
constexpr int kStgU = 8;                    // entries per lane and row whose gathers are issued together

// rows a lane group holds in flight: 4 with 4-byte vectors, 2 with 8-byte ones
template <typename T>
struct StgRows {
  static constexpr int value = sizeof(T) == 8 ? 2 : 4;
};

// Byte layout of one stage (all offsets 16-byte multiples):
//   int  irp[rmax + 8]                 row offsets of the tile (widened slice)
//   CI   col[emax + 16]                column indices / offsets
//   V    val[emax + 16]                values
//   T    vec[q][rmax + 8], q < nvec    row vectors
struct StgLayout {
  int rmax = 0, emax = 0, stages = 0, nvec = 0;
  int off_col = 0, off_val = 0, off_vec = 0, vec_bytes = 0, stage_bytes = 0;
};
__host__ __device__ inline int stg_al16(int x) { return (x + 15) & ~15; }
template <typename T, typename V, typename CI>
__host__ inline StgLayout stg_layout(int rmax, int emax, int stages, int nvec) {
  StgLayout L;
  L.rmax = rmax;
  L.emax = emax;
  L.stages = stages;
  L.nvec = nvec;
  L.off_col = stg_al16(4 * (rmax + 8));
  L.off_val = L.off_col + stg_al16((int)sizeof(CI) * (emax + 16));
  L.off_vec = L.off_val + stg_al16((int)sizeof(V) * (emax + 16));
  L.vec_bytes = stg_al16((int)sizeof(T) * (rmax + 8));
  L.stage_bytes = L.off_vec + nvec * L.vec_bytes;
  return L;
}
// dynamic shared memory of a launch: every warp's stages and mbarriers
__host__ inline size_t stg_smem(const StgLayout &L) {
  return (size_t)kStgWarps * ((size_t)L.stages * L.stage_bytes + 8 * (size_t)L.stages);
}

template <typename T, typename V, typename CI>
struct StgArgs {
  int ntiles;
  const int4 *tiles;
  const int *irp;
  const CI *cj;
  const V *val;
  const float *rs;  // FP16 values: row scales
  const T *vec[kStgVecs];
  StgLayout L;
  int *err;
};

// element index where a 16-byte aligned slice starting at or before i begins, and
// where one ending at or after i ends, for elements of E bytes
template <int E>
__device__ __forceinline__ int stg_lo(int i) { return i & ~(16 / E - 1); }
template <int E>
__device__ __forceinline__ int stg_hi(int i) { return (i + 16 / E - 1) & ~(16 / E - 1); }

__device__ __forceinline__ void stg_fence_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// lane 0: copy tile t into the stage st of the warp's ring, counted on bar
template <typename T, typename V, typename CI>
__device__ __forceinline__ void stg_issue(const StgArgs<T, V, CI> &a, int t, unsigned char *st, uint64_t *bar) {
  const StgLayout &L = a.L;
  const int4 d = a.tiles[t];
  const int ia0 = stg_lo<4>(d.x), ia1 = stg_hi<4>(d.y + 1);
  const int ec0 = stg_lo<sizeof(CI)>(d.z), ec1 = stg_hi<sizeof(CI)>(d.w);
  const int ev0 = stg_lo<sizeof(V)>(d.z), ev1 = stg_hi<sizeof(V)>(d.w);
  const int rv0 = stg_lo<sizeof(T)>(d.x), rv1 = stg_hi<sizeof(T)>(d.y);
  const unsigned bi = 4u * (unsigned)(ia1 - ia0), bc = (unsigned)sizeof(CI) * (unsigned)(ec1 - ec0),
                 bv = (unsigned)sizeof(V) * (unsigned)(ev1 - ev0), bw = (unsigned)sizeof(T) * (unsigned)(rv1 - rv0);
  mbar_expect_tx(bar, bi + bc + bv + (unsigned)L.nvec * bw);
  tma_bulk_g2s(st, a.irp + ia0, bi, bar);
  if (bc) tma_bulk_g2s(st + L.off_col, a.cj + ec0, bc, bar);
  if (bv) tma_bulk_g2s(st + L.off_val, a.val + ev0, bv, bar);
#pragma unroll
  for (int q = 0; q < kStgVecs; ++q)  // static indices: the arguments stay in the parameter space
    if (q < L.nvec) tma_bulk_g2s(st + L.off_vec + q * L.vec_bytes, a.vec[q] + rv0, bw, bar);
}

// The tile loop of one warp: tile_fn(tile descriptor, its stage) runs on all
// 32 lanes once the tile's copies have landed.
template <typename T, typename V, typename CI, typename F>
__device__ __forceinline__ void stg_run(const StgArgs<T, V, CI> &a, F tile_fn) {
  extern __shared__ __align__(128) unsigned char smem[];
  const StgLayout &L = a.L;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *ring = smem + (size_t)w * L.stages * L.stage_bytes;
  uint64_t *full =
      reinterpret_cast<uint64_t *>(smem + (size_t)kStgWarps * L.stages * L.stage_bytes) + (size_t)w * L.stages;
  const int gw = blockIdx.x * kStgWarps + w, nw = gridDim.x * kStgWarps;
  int issued = 0;  // lane 0: tiles of this warp whose copies were issued
  if (lane == 0) {
    for (int s = 0; s < L.stages; ++s) mbar_init(&full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int s = 0; s < L.stages && gw + s * nw < a.ntiles; ++s, ++issued)
      stg_issue(a, gw + s * nw, ring + (size_t)s * L.stage_bytes, &full[s]);
  }
  __syncwarp();
  int k = 0;
  for (; gw + k * nw < a.ntiles; ++k) {
    const int s = k % L.stages;
    if (!mbar_wait(&full[s], (unsigned)((k / L.stages) & 1))) {
      if (lane == 0) atomicExch(a.err, 4021);
      break;
    }
    tile_fn(a.tiles[gw + k * nw], ring + (size_t)s * L.stage_bytes);
    __syncwarp();
    const int kn = k + L.stages;
    if (lane == 0 && gw + kn * nw < a.ntiles) {
      stg_fence_async();  // the warp's reads of this stage before the copy that overwrites it
      stg_issue(a, gw + kn * nw, ring + (size_t)s * L.stage_bytes, &full[s]);
      ++issued;
    }
  }
  // after a wait that gave up: every copy issued must land before the warp exits
  if (lane == 0)
    for (int j = k; j < issued; ++j) mbar_wait(&full[j % L.stages], (unsigned)((j / L.stages) & 1));
}

// Rows of one staged tile: TPR lanes per row, StgRows rows per lane group at
// a time; per row each lane sums val * gather(col) over its entries k =
// first + lane, + TPR, ... in order (the loads and gathers of kStgU entries
// of every row of the group issued before the sums), then the butterfly,
// then done(row, the row's position in the staged vectors, sum) on the row's
// first lane.
template <typename T, typename V, typename CI, int TPR, typename G, typename D>
__device__ __forceinline__ void stg_rows(const StgLayout &L, const int4 d, const unsigned char *st,
                                         const float *__restrict__ rs, G gather, D done) {
  constexpr int R = StgRows<T>::value, NG = 32 / TPR;
  const int lane = threadIdx.x & 31, grp = lane / TPR, sub = lane % TPR;
  const int ia0 = stg_lo<4>(d.x), ec0 = stg_lo<sizeof(CI)>(d.z), ev0 = stg_lo<sizeof(V)>(d.z);
  const int rv0 = stg_lo<sizeof(T)>(d.x);
  const int *irs = reinterpret_cast<const int *>(st);
  const CI *cs = reinterpret_cast<const CI *>(st + L.off_col);
  // the value of staged column position k is at k + (ec0 - ev0) of the staged values
  const V *vs = reinterpret_cast<const V *>(st + L.off_val) + (ec0 - ev0);
  const int nrow = d.y - d.x;
  for (int p = 0; p < nrow; p += NG * R) {  // uniform over the warp: full-warp shuffles below
    int kb[R], ke[R], row[R];
    T s[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int lr = p + grp + r * NG;
      const bool ok = lr < nrow;
      row[r] = d.x + lr;
      kb[r] = ok ? irs[row[r] - ia0] + sub - ec0 : 0;  // staged column positions
      ke[r] = ok ? irs[row[r] + 1 - ia0] - ec0 : 0;
      s[r] = T(0);
    }
    for (;;) {
      bool more = false;
#pragma unroll
      for (int r = 0; r < R; ++r) more |= kb[r] < ke[r];
      if (!more) break;
      T vv[R][kStgU], xv[R][kStgU];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int u = 0; u < kStgU; ++u) {
          const int k = kb[r] + u * TPR;
          const bool ok = k < ke[r];
          vv[r][u] = ok ? ldval<T>(vs, k) : T(0);
          xv[r][u] = ok ? gather(colof(cs, k, row[r])) : T(0);
        }
#pragma unroll
      for (int r = 0; r < R; ++r) {
#pragma unroll
        for (int u = 0; u < kStgU; ++u)
          if (kb[r] + u * TPR < ke[r]) s[r] = fma(vv[r][u], xv[r][u], s[r]);
        kb[r] += kStgU * TPR;
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int o = TPR / 2; o > 0; o >>= 1) s[r] += __shfl_down_sync(0xffffffffu, s[r], o, TPR);
      if (row[r] < d.y && sub == 0) done(row[r], row[r] - rv0, row_scaled<T, V>(s[r], rs, row[r]));
    }
  }
}

// out = a1*(A v) + a0*b + a2*out  (k_spmv's operation); staged vectors:
// slot 0 = b when b is given, the next slot = out when a2 != 0
template <typename T, typename V, typename CI, int TPR>
__global__ void __launch_bounds__(kStgThreads, 1) k_spmv_stg(StgArgs<T, V, CI> a, const T *__restrict__ v, T a1,
                                                             int has_b, T a0, T *out, T a2) {
  const int sb = 0, so = has_b ? 1 : 0;
  stg_run<T, V, CI>(a, [&](const int4 d, const unsigned char *st) {
    const T *vb = reinterpret_cast<const T *>(st + a.L.off_vec + sb * a.L.vec_bytes);
    const T *vo = reinterpret_cast<const T *>(st + a.L.off_vec + so * a.L.vec_bytes);
    stg_rows<T, V, CI, TPR>(
        a.L, d, st, a.rs, [&](int j) { return __ldg(v + j); },
        [&](int row, int q, T s) {
          T r = a1 * s;
          if (has_b) r = fma(a0, vb[q], r);
          if (a2 != T(0)) r = fma(a2, vo[q], r);
          out[row] = r;
        });
  });
}

// the Jacobi sweep of k_jacobi; staged vectors: slot 0 = d, 1 = x, then ty
// (when !first and omega != 1), then out (when beta != 0)
template <typename T, typename V, typename CI, int TPR>
__global__ void __launch_bounds__(kStgThreads, 1) k_jacobi_stg(StgArgs<T, V, CI> a, const T *__restrict__ d,
                                                               const T *__restrict__ x, const T *__restrict__ ty,
                                                               int first, T omega, T alpha, T beta, T *out) {
  const bool use_ty = !first && omega != T(1);
  const int sty = 2, sout = use_ty ? 3 : 2;
  stg_run<T, V, CI>(a, [&](const int4 dd, const unsigned char *st) {
    const T *vd = reinterpret_cast<const T *>(st + a.L.off_vec);
    const T *vx = reinterpret_cast<const T *>(st + a.L.off_vec + a.L.vec_bytes);
    const T *vt = reinterpret_cast<const T *>(st + a.L.off_vec + sty * a.L.vec_bytes);
    const T *vo = reinterpret_cast<const T *>(st + a.L.off_vec + sout * a.L.vec_bytes);
    auto done = [&](int row, int q, T s) {
      out[row] = jac_row(vd[q], vx[q], s, use_ty ? vt[q] : T(0), first != 0, omega, alpha, beta,
                         beta != T(0) ? vo[q] : T(0));
    };
    if (first)
      stg_rows<T, V, CI, TPR>(a.L, dd, st, a.rs, [&](int j) { return omega * (__ldg(d + j) * __ldg(x + j)); },
                              done);
    else
      stg_rows<T, V, CI, TPR>(a.L, dd, st, a.rs, [&](int j) { return __ldg(ty + j); }, done);
  });
}

}  // namespace mldg
