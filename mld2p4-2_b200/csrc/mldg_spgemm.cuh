// mldg_spgemm.cuh -- sparse matrix products of the hierarchy set-up on the
// GPU, bit for bit the host build's.
//
// The host forms C = A B row by row (Gustavson): row i walks its entries a_ik
// in stored order and, for each, row k of B in stored order; a column j's
// first contribution a_ik*b_kj is assigned, every later one added
// (acc + p, each product and sum rounded on its own); the row's columns are
// then written in ascending order.  This stands in for psb_spspmm in the
// smoothed prolongator P = (I - omega D^{-1} A) P_tent and the Galerkin
// product R (A P) (mlprec/impl/mld_daggrmat_smth_asb.f90:316,345,399).
//
// On the GPU one warp forms one row of C.  The warp walks a_ik sequentially;
// its lanes take the entries of row k of B, whose columns are distinct, so
// no two lanes touch the same column in one step and every column receives
// its contributions in the host's order.  Columns and values live in a
// per-warp open-addressing hash table in shared memory (kSpgH slots); a row
// with more than kSpgMax distinct columns is left to the host (its count is
// -1).  The count pass sizes the rows; the fill pass accumulates, compacts
// the table, sorts the row's (column, value) pairs by column (odd-even
// transposition over the warp) and writes them.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mldg {

constexpr int kSpgH = 2048;                // hash slots per warp (power of two)
constexpr int kSpgMax = kSpgH * 3 / 4;     // distinct columns a warp takes
constexpr int kSpgWarps = 2;               // warps per block
constexpr int kSpgEmpty = -1;
// dynamic shared memory per warp: keys[H] int, vals[H] double, skey[Max] int, sval[Max] double
constexpr size_t kSpgWarpBytes = (size_t)kSpgH * 12 + (size_t)kSpgMax * 12;
constexpr size_t kSpgSmem = kSpgWarpBytes * kSpgWarps;

__device__ __forceinline__ unsigned spg_hash(int j) { return ((unsigned)j * 2654435761u) & (kSpgH - 1); }

// slot of column j (inserted if absent); *fresh = inserted by this call; -1 if full
__device__ __forceinline__ int spg_slot(int *keys, int j, bool *fresh) {
  unsigned h = spg_hash(j);
  *fresh = false;
  for (int probe = 0; probe < kSpgH; ++probe) {
    const int k = keys[h];
    if (k == j) return (int)h;
    if (k == kSpgEmpty) {
      const int old = atomicCAS(&keys[h], kSpgEmpty, j);
      if (old == kSpgEmpty) {
        *fresh = true;
        return (int)h;
      }
      if (old == j) return (int)h;
    }
    h = (h + 1) & (kSpgH - 1);
  }
  return -1;
}

struct SpgWarpMem {
  int *keys;
  double *vals;
  int *skey;
  double *sval;
};
__device__ __forceinline__ SpgWarpMem spg_mem(unsigned char *smem, int w) {
  unsigned char *b = smem + kSpgWarpBytes * w;
  SpgWarpMem m;
  m.vals = reinterpret_cast<double *>(b);
  m.sval = reinterpret_cast<double *>(b + (size_t)kSpgH * 8);
  m.keys = reinterpret_cast<int *>(b + (size_t)kSpgH * 8 + (size_t)kSpgMax * 8);
  m.skey = reinterpret_cast<int *>(b + (size_t)kSpgH * 12 + (size_t)kSpgMax * 8);
  return m;
}

// count pass: cnt[i] = entries of row i of C, or -1 when the row is left to the host
__global__ void __launch_bounds__(32 * kSpgWarps) k_spgemm_count(int m, const int *__restrict__ airp,
                                                                 const int *__restrict__ aja,
                                                                 const int *__restrict__ birp,
                                                                 const int *__restrict__ bja, int *cnt) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const SpgWarpMem mem = spg_mem(smem, w);
  for (int i = blockIdx.x * kSpgWarps + w; i < m; i += gridDim.x * kSpgWarps) {
    for (int s = lane; s < kSpgH; s += 32) mem.keys[s] = kSpgEmpty;
    __syncwarp();
    int c = 0;
    bool over = false;
    for (int ka = airp[i]; ka < airp[i + 1] && !over; ++ka) {
      const int k = aja[ka];
      for (int kb = birp[k] + lane; kb < birp[k + 1]; kb += 32) {
        bool fresh;
        const int h = spg_slot(mem.keys, bja[kb], &fresh);
        c += fresh;
        over |= h < 0;
      }
      __syncwarp();
      int tot = c;
      for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
      over = __any_sync(0xffffffffu, over) || tot > kSpgMax;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[i] = over ? -1 : c;
    __syncwarp();
  }
}

// fill pass: every row with cnt[i] >= 0 gets its sorted columns and values at cirp[i]
__global__ void __launch_bounds__(32 * kSpgWarps) k_spgemm_fill(int m, const int *__restrict__ airp,
                                                                const int *__restrict__ aja,
                                                                const double *__restrict__ aval,
                                                                const int *__restrict__ birp,
                                                                const int *__restrict__ bja,
                                                                const double *__restrict__ bval,
                                                                const int *__restrict__ cnt,
                                                                const int *__restrict__ cirp, int *cja,
                                                                double *cval) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const SpgWarpMem mem = spg_mem(smem, w);
  for (int i = blockIdx.x * kSpgWarps + w; i < m; i += gridDim.x * kSpgWarps) {
    if (cnt[i] < 0) continue;
    for (int s = lane; s < kSpgH; s += 32) mem.keys[s] = kSpgEmpty;
    __syncwarp();
    // contributions in the host's order: a_ik sequential, the distinct columns of row k across lanes
    for (int ka = airp[i]; ka < airp[i + 1]; ++ka) {
      const int k = aja[ka];
      const double av = aval[ka];
      for (int kb = birp[k] + lane; kb < birp[k + 1]; kb += 32) {
        const double p = __dmul_rn(av, bval[kb]);
        bool fresh;
        const int h = spg_slot(mem.keys, bja[kb], &fresh);
        if (h >= 0) mem.vals[h] = fresh ? p : __dadd_rn(mem.vals[h], p);  // always: the count pass bounds the row
      }
      __syncwarp();
    }
    // compact the table (order of slots), then sort by column
    int nd = 0;
    for (int s0 = 0; s0 < kSpgH; s0 += 32) {
      const int s = s0 + lane;
      const bool used = mem.keys[s] != kSpgEmpty;
      const unsigned bal = __ballot_sync(0xffffffffu, used);
      if (used) {
        const int q = nd + __popc(bal & ((1u << lane) - 1u));
        mem.skey[q] = mem.keys[s];
        mem.sval[q] = mem.vals[s];
      }
      nd += __popc(bal);
    }
    __syncwarp();
    for (int phase = 0; phase < nd; ++phase) {
      for (int t = 2 * lane + (phase & 1); t + 1 < nd; t += 64) {
        if (mem.skey[t] > mem.skey[t + 1]) {
          const int kt = mem.skey[t];
          mem.skey[t] = mem.skey[t + 1];
          mem.skey[t + 1] = kt;
          const double vt = mem.sval[t];
          mem.sval[t] = mem.sval[t + 1];
          mem.sval[t + 1] = vt;
        }
      }
      __syncwarp();
    }
    for (int t = lane; t < nd; t += 32) {
      cja[cirp[i] + t] = mem.skey[t];
      cval[cirp[i] + t] = mem.sval[t];
    }
    __syncwarp();
  }
}

}  // namespace mldg
