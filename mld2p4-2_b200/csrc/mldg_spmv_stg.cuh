// mldg_spmv_stg.cuh -- staged CSR SpMV and Jacobi sweep: the matrix and the
// row vectors reach the SMs by TMA bulk copies, not by per-thread loads.
//
// The rows of an operator are cut (on the host, once) into tiles of
// consecutive rows: at most rmax rows and emax entries each, described by
// int4 {first row, end row, first entry, end entry}.  A persistent grid
// walks the tiles round robin (tile t goes to CTA t mod grid).  In each CTA
// one producer thread copies whole tiles -- the tile's slice of the row
// offsets, of the column indices, of the values and of up to kStgVecs row
// vectors (the right-hand side b, the output's old values, the Jacobi
// diagonal and iterate) -- into a ring of `stages` shared-memory stages with
// cp.async.bulk, each stage's full mbarrier counting the bytes; eight
// consumer warps compute the tile's rows from shared memory (TPR lanes per
// row, entries summed in stored order per lane, lanes combined by a
// butterfly exactly like k_spmv / k_jacobi) and gather the multiplied vector
// through L1/L2, then release the stage on its empty mbarrier.  The copies
// are large and contiguous (one to three requests of several KB per array
// and tile) and run `stages` tiles ahead of the compute, so the DRAM stream
// does not wait on the dependent load chain (row offsets, then entries, then
// gathers) that limits the per-thread CSR and SELL kernels.
//
// A bulk copy needs a 16-byte aligned source and a size that is a multiple
// of 16 bytes: every slice is widened to 16-byte boundaries (the arrays are
// cudaMalloc'd with slack past their end, so the widened slices stay inside
// the allocations), and the consumers index the staged slices relative to
// the widened starts.
//
// Every wait is bounded: an mbarrier wait that gives up sets error 4021; a
// consumer that gave up stops computing, the producer then gives up on its
// empty barrier, and before the CTA exits the producer waits (bounded) for
// every copy it issued.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mldg_kernels.cuh"
#include "mldg_trsv_win.cuh"  // mbar_init, mbar_expect_tx, mbar_wait, tma_bulk_g2s

namespace mldg {

constexpr int kStgConsumers = 8;                     // consumer warps
constexpr int kStgThreads = 32 * (kStgConsumers + 1);  // + one producer warp
constexpr int kStgVecs = 4;                          // row vectors staged per tile (at most)
constexpr int kStgMaxStages = 8;
constexpr size_t kStgSmemMax = 227 * 1024;  // dynamic shared memory a CTA may opt in to

__device__ __forceinline__ void stg_arrive(uint64_t *bar) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(smem_u32(bar))
               : "memory");
}

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
// dynamic shared memory of a launch: the stages and the 2 * stages mbarriers
__host__ inline size_t stg_smem(const StgLayout &L) { return (size_t)L.stages * L.stage_bytes + 16 * L.stages; }

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

// The tile loop shared by both kernels: tile_fn(tile descriptor, its stage)
// runs on every consumer thread once the tile's copies have landed.
template <typename T, typename V, typename CI, typename F>
__device__ __forceinline__ void stg_run(const StgArgs<T, V, CI> &a, F tile_fn) {
  extern __shared__ __align__(128) unsigned char smem[];
  const StgLayout &L = a.L;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + (size_t)L.stages * L.stage_bytes);
  uint64_t *empty = full + L.stages;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < L.stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kStgConsumers);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (warp == kStgConsumers) {
    // producer: one thread issues every copy of the CTA's tiles
    if (lane != 0) return;
    int i = 0;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++i) {
      const int s = i % L.stages;
      if (i >= L.stages && !mbar_wait(&empty[s], (unsigned)(((i / L.stages) - 1) & 1))) {
        atomicExch(a.err, 4021);
        break;
      }
      const int4 d = a.tiles[t];
      unsigned char *st = smem + (size_t)s * L.stage_bytes;
      const int ia0 = stg_lo<4>(d.x), ia1 = stg_hi<4>(d.y + 1);
      const int ec0 = stg_lo<sizeof(CI)>(d.z), ec1 = stg_hi<sizeof(CI)>(d.w);
      const int ev0 = stg_lo<sizeof(V)>(d.z), ev1 = stg_hi<sizeof(V)>(d.w);
      const int rv0 = stg_lo<sizeof(T)>(d.x), rv1 = stg_hi<sizeof(T)>(d.y);
      const unsigned bi = 4u * (unsigned)(ia1 - ia0), bc = (unsigned)sizeof(CI) * (unsigned)(ec1 - ec0),
                     bv = (unsigned)sizeof(V) * (unsigned)(ev1 - ev0), bw = (unsigned)sizeof(T) * (unsigned)(rv1 - rv0);
      mbar_expect_tx(&full[s], bi + bc + bv + (unsigned)L.nvec * bw);
      tma_bulk_g2s(st, a.irp + ia0, bi, &full[s]);
      if (bc) tma_bulk_g2s(st + L.off_col, a.cj + ec0, bc, &full[s]);
      if (bv) tma_bulk_g2s(st + L.off_val, a.val + ev0, bv, &full[s]);
#pragma unroll
      for (int q = 0; q < kStgVecs; ++q)  // static indices: the arguments stay in the parameter space
        if (q < L.nvec) tma_bulk_g2s(st + L.off_vec + q * L.vec_bytes, a.vec[q] + rv0, bw, &full[s]);
    }
    // every copy issued must land before the CTA exits
    for (int j = i > L.stages ? i - L.stages : 0; j < i; ++j)
      mbar_wait(&full[j % L.stages], (unsigned)((j / L.stages) & 1));
    return;
  }
  int i = 0;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++i) {
    const int s = i % L.stages;
    if (!mbar_wait(&full[s], (unsigned)((i / L.stages) & 1))) {
      if (lane == 0) atomicExch(a.err, 4021);
      break;
    }
    tile_fn(a.tiles[t], smem + (size_t)s * L.stage_bytes);
    __syncwarp();
    if (lane == 0) stg_arrive(&empty[s]);
  }
}

// Rows of one staged tile, TPR lanes per row: the row sum of val * gather(col)
// over the row's staged entries (csr_lane_sum per lane, then the butterfly),
// then done(row, the row's position in the staged vectors, sum) on the
// row's first lane.
template <typename T, typename V, typename CI, int TPR, typename G, typename D>
__device__ __forceinline__ void stg_rows(const StgLayout &L, const int4 d, const unsigned char *st,
                                         const float *__restrict__ rs, G gather, D done) {
  constexpr int RPP = 32 * kStgConsumers / TPR;  // rows per pass
  const int c = threadIdx.x;                     // consumer thread 0..255
  const int grp = c / TPR, sub = c % TPR;
  const int ia0 = stg_lo<4>(d.x), ec0 = stg_lo<sizeof(CI)>(d.z), ev0 = stg_lo<sizeof(V)>(d.z);
  const int rv0 = stg_lo<sizeof(T)>(d.x);
  const int *irs = reinterpret_cast<const int *>(st);
  const CI *cs = reinterpret_cast<const CI *>(st + L.off_col);
  const V *vs = reinterpret_cast<const V *>(st + L.off_val);
  const int nrow = d.y - d.x;
  for (int p = 0; p < nrow; p += RPP) {  // uniform over the CTA: full-warp shuffles below
    const int lr = p + grp;
    const bool ok = lr < nrow;
    const int row = d.x + lr;
    T s = T(0);
    if (ok) {
      // entry k of the row is staged at k - ec0 (columns) and k - ev0 (values)
      const int k0 = irs[row - ia0] + sub, k1 = irs[row + 1 - ia0];
      s = csr_lane_sum<T, TPR>(k0 - ec0, k1 - ec0, row, cs, vs + (ec0 - ev0), gather);
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    if (ok && sub == 0) done(row, row - rv0, row_scaled<T, V>(s, rs, row));
  }
}

// out = a1*(A v) + a0*b + a2*out  (k_spmv's operation); staged vectors:
// slot 0 = b when b is given, the next slot = out when a2 != 0
template <typename T, typename V, typename CI, int TPR>
__global__ void __launch_bounds__(kStgThreads) k_spmv_stg(StgArgs<T, V, CI> a, const T *__restrict__ v, T a1,
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
__global__ void __launch_bounds__(kStgThreads) k_jacobi_stg(StgArgs<T, V, CI> a, const T *__restrict__ d,
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
      const T di = vd[q], xi = vx[q];
      const T t = di * (xi - s);
      T vv;
      if (omega == T(1)) {
        vv = t;
      } else {
        const T tyi = first ? omega * (di * xi) : vt[q];
        vv = (T(1) - omega) * tyi + omega * t;
      }
      T r = alpha * vv;
      if (beta != T(0)) r = fma(beta, vo[q], r);
      out[row] = r;
    };
    if (first)
      stg_rows<T, V, CI, TPR>(a.L, dd, st, a.rs, [&](int j) { return omega * (__ldg(d + j) * __ldg(x + j)); },
                              done);
    else
      stg_rows<T, V, CI, TPR>(a.L, dd, st, a.rs, [&](int j) { return __ldg(ty + j); }, done);
  });
}

}  // namespace mldg
