// mldg_multi.cuh -- multi-right-hand-side forms of the V-cycle kernels.
//
// Vectors of K right-hand sides are stored row-interleaved: v[i*K + c].  A
// thread owns one (row, column) pair, the column fastest, so every row's K
// values are one contiguous (coalesced) access while matrix entries are
// broadcast across the K lanes of the row.  K is a power of two <= 32.
#pragma once

#include "mldg_kernels.cuh"

namespace mldg {

// out[i,c] = a0*b[i,c] + a1*(A v)[i,c] + a2*out[i,c]
template <typename T, int K>
__global__ void __launch_bounds__(256) k_spmm(int nr, const int *__restrict__ irp, const int *__restrict__ ja,
                                              const T *__restrict__ val, const T *__restrict__ v, T a1,
                                              const T *__restrict__ b, T a0, T *out, T a2) {
  const long long total = (long long)nr * K;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(t / K), c = (int)(t % K);
    T s = T(0);
    const int e = irp[row + 1];
    for (int k = irp[row]; k < e; ++k) s = fma(val[k], __ldg(v + (size_t)ja[k] * K + c), s);
    T r = a1 * s;
    if (b) r = fma(a0, b[t], r);
    if (a2 != T(0)) r = fma(a2, out[t], r);
    out[t] = r;
  }
}

// FP32_P16 prolongation: out[i,c] += scale[i] * sum_k half(P_ik) v[j,c]
template <int K>
__global__ void __launch_bounds__(256) k_spmm_h(int nr, const int *__restrict__ irp, const int *__restrict__ ja,
                                                const __half *__restrict__ hval, const float *__restrict__ scale,
                                                const float *__restrict__ v, float *out) {
  const long long total = (long long)nr * K;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(t / K), c = (int)(t % K);
    float s = 0.f;
    const int e = irp[row + 1];
    for (int k = irp[row]; k < e; ++k) s = fmaf(__half2float(hval[k]), __ldg(v + (size_t)ja[k] * K + c), s);
    out[t] = fmaf(scale[row], s, out[t]);
  }
}

// multi-RHS point-Jacobi sweep (same algebra as k_jacobi)
template <typename T, int K>
__global__ void __launch_bounds__(256) k_jacobi_m(int nr, const int *__restrict__ irp, const int *__restrict__ ja,
                                                  const T *__restrict__ val, const T *__restrict__ d,
                                                  const T *__restrict__ x, const T *__restrict__ ty, int first,
                                                  T omega, T alpha, T beta, T *out) {
  const long long total = (long long)nr * K;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(t / K), c = (int)(t % K);
    T s = T(0);
    const int e = irp[row + 1];
    if (first == 2) {
      for (int k = irp[row]; k < e; ++k) s = fma(val[k], omega * __ldg(x + (size_t)ja[k] * K + c), s);
    } else if (first) {
      for (int k = irp[row]; k < e; ++k) {
        const int j = ja[k];
        s = fma(val[k], omega * (__ldg(d + j) * __ldg(x + (size_t)j * K + c)), s);
      }
    } else {
      for (int k = irp[row]; k < e; ++k) s = fma(val[k], __ldg(ty + (size_t)ja[k] * K + c), s);
    }
    out[t] = jac_row(d[row], x[t], s, (!first && omega != T(1)) ? ty[t] : T(0), first != 0, omega, alpha, beta,
                     beta != T(0) ? out[t] : T(0));
  }
}

// out[i,c] = alpha * d[i] * x[i,c] + beta * out[i,c]
template <typename T, int K>
__global__ void k_diag_m(int n, const T *__restrict__ d, const T *__restrict__ x, T alpha, T beta, T *out) {
  const long long total = (long long)n * K;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    T r = alpha * (d[t / K] * x[t]);
    if (beta != T(0)) r = fma(beta, out[t], r);
    out[t] = r;
  }
}

// dense coarsest solve for K right-hand sides: out = alpha*M x + beta*out
template <typename T, int K>
__global__ void __launch_bounds__(256) k_gemm_m(int n, const T *__restrict__ M, const T *__restrict__ x, T alpha,
                                                T beta, T *out) {
  const long long total = (long long)n * K;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / K), c = (int)(t % K);
    const T *row = M + (size_t)i * n;
    T s = T(0);
    for (int j = 0; j < n; ++j) s = fma(__ldg(row + j), __ldg(x + (size_t)j * K + c), s);
    T r = alpha * s;
    if (beta != T(0)) r = fma(beta, out[t], r);
    out[t] = r;
  }
}

// Multi-RHS sync-free triangular solve: the level-ordered factor of the
// single-vector solve (TriArgs), a warp block of 32/K rows, one lane per
// (row, column).  The exchange buffer holds K values per row, each the
// sentinel until produced; a lane waits only on its own column.
template <typename T, int K>
__global__ void __launch_bounds__(256) k_trsv_sf_m(TriArgs<T> a, int nblk_m, const int2 *blk_m) {
  const int lane = threadIdx.x & 31;
  const int c = lane % K;
  const int grp = lane / K;
  typedef typename Bits<T>::U U;
  const U sent = (U)Sentinel<T>::bits;
  for (;;) {
    int b = 0;
    if (lane == 0) b = atomicAdd(&a.counters[0], 1);
    b = __shfl_sync(0xffffffffu, b, 0);
    if (b >= nblk_m) break;
    const int2 be = blk_m[b];
    const int p = be.x + grp;
    if (p < be.y) {
      const int i = a.prow[p];
      const int o = a.rev ? (a.n - 1 - i) : i;
      const size_t oc = (size_t)o * K + c;
      T rhs = a.rhs_src[oc];
      if (a.rhs_scale) rhs = rhs * a.rhs_scale[o];
      T acc = T(0);
      const int k1 = a.pirp[p + 1];
      for (int k0 = a.pirp[p]; k0 < k1; k0 += 4) {
        // up to 4 dependency loads in flight, then re-poll the missing ones
        U raw[4];
        T vv[4];
        const T *src[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = k0 + e;
          const bool has = k < k1;
          const int j = has ? a.pja[k] : 0;
          const int oj = a.rev ? (a.n - 1 - j) : j;
          vv[e] = has ? a.pval[k] : T(0);
          src[e] = a.cur + (size_t)oj * K + c;
          raw[e] = has ? Bits<T>::load(src[e]) : (U)0;
        }
        const int lim = spin_limit();
        for (int it = 0;; ++it) {
          bool missing = false;
#pragma unroll
          for (int e = 0; e < 4; ++e) missing |= (raw[e] == sent);
          if (!missing) break;
          if (it >= lim) {
            atomicExch(a.err, kErrTimeout);
            break;
          }
          if ((it % kSpinCheck) == kSpinCheck - 1) {
            if (ld_relaxed_u32(a.err) != 0u) break;
            __nanosleep(32);
          }
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (raw[e] == sent) raw[e] = Bits<T>::load(src[e]);
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) acc = fma(vv[e], Bits<T>::from(raw[e] == sent ? (U)0 : raw[e]), acc);
      }
      const T t = Bits<T>::canon(rhs - acc);
      Bits<T>::store(a.cur + oc, t);
      if (a.other) a.other[oc] = Sentinel<T>::value();
      if (a.out) {
        T w = a.alpha * t;
        if (a.beta != T(0)) w = fma(a.beta, a.out[oc], w);
        a.out[oc] = w;
      }
    }
  }
  if (lane == 0) {
    const int nw = (int)(gridDim.x * (blockDim.x >> 5));
    const int done = atomicAdd(&a.counters[1], 1);
    if (done == nw - 1) {
      a.counters[0] = 0;
      a.counters[1] = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// ELL form of the multi-RHS sync-free solve.  The level-ordered rows are laid
// out in padded positions: every level starts at a multiple of RPW = 32/K, so
// the RPW rows of a warp task never straddle a level (no lane waits on its own
// warp).  Per padded position pp = t*RPW + g (task t, row g of the task): the
// original row prow[pp] (-1 = padding).  Task t owns E_t = toff[t].y entry
// slots per row (the longest row of the task, at most E), stored at
// ej/ev[toff[t].x + e*RPW + g]: the original index of the dependency row
// (-1 = empty) and the factor value, so padding costs no more than the
// longest row of each task.  A row's entries are ordered by the
// level of their dependency; rows longer than E keep their E most recent
// dependencies in the slots and the older ones in an overflow list
// (ovp/ovj/ovv), accumulated first.  All slot loads of a row are in flight at
// once, so a row costs one round trip once its last dependency is written.
//
// Tasks are claimed from S ticket streams (task k*S + s is ticket k of stream
// s, each stream a counter on its own 128-byte line), so that S atomics
// proceed in parallel.  A warp claims one ticket ahead and, for E <= 8 (PF),
// loads the next task's metadata while its current task waits.  Within a
// stream tickets are claimed in order and a warp finishes its current task
// before starting the next, so the lowest unfinished task is always being
// processed and only depends on finished tasks: every wait ends (each is
// bounded anyway).  The grid never exceeds the co-resident capacity, so every
// stream keeps running warps.
template <typename T>
struct EllArgs {
  int ntask, npad, S;
  const int2 *toff;  // per task: slot base, slots per row; null: uniform (t*E*RPW, E)
  int backoff;  // > 0: ns slept between polls after the first few (0: back to back)
  const int *prow;
  const int *ej;
  const T *ev;
  const int *ovp;  // npad + 1 overflow offsets, or null
  const int *ovj;
  const T *ovv;
  const T *rhs_src;
  const T *rhs_scale;
  T *cur;
  T *other;
  T *out;
  T alpha, beta;
  int *ctr;  // S ticket counters (stride 32 ints), then the finished-warp count
  int *err;
  unsigned long long *trace;  // diagnostics: per task [start, end] globaltimer ns, or null
};

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename T, int E>
struct EllMeta {
  int o, q0, q1;
  int j[E];
  T v[E];
};

template <typename T, int E, int RPW>
__device__ __forceinline__ void ell_meta(const EllArgs<T> &a, int t, int g, int2 to, EllMeta<T, E> &m) {
  const int pp = t * RPW + g;
  m.o = a.prow[pp];
  m.q0 = m.q1 = 0;
  if (a.ovp) {
    m.q0 = a.ovp[pp];
    m.q1 = a.ovp[pp + 1];
  }
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const bool has = e < to.y;
    const size_t q = (size_t)to.x + (size_t)e * RPW + g;
    m.j[e] = has ? a.ej[q] : -1;
    m.v[e] = has ? a.ev[q] : T(0);
  }
}

// wait until none of raw[0..N) holds the sentinel (bounded); returns false on failure
template <typename T, int N, int K>
__device__ __forceinline__ bool ell_wait(typename Bits<T>::U (&raw)[N], const int (&j)[N], const T *cur, int c,
                                         int *err, int backoff) {
  typedef typename Bits<T>::U U;
  const U sent = (U)Sentinel<T>::bits;
  const int lim = spin_limit();
  for (int it = 0;; ++it) {
    bool missing = false;
#pragma unroll
    for (int e = 0; e < N; ++e) missing |= (raw[e] == sent);
    if (!missing) return true;
    if (it >= lim) {
      atomicExch(err, kErrTimeout);
      return false;
    }
    if ((it % kSpinCheck) == kSpinCheck - 1) {
      if (ld_relaxed_u32(err) != 0u) return false;
      __nanosleep(32);
    } else if (backoff > 0 && it >= 2) {
      __nanosleep(backoff);  // measured: no gain on B200, off by default
    }
#pragma unroll
    for (int e = 0; e < N; ++e)
      if (raw[e] == sent) raw[e] = Bits<T>::load(cur + (size_t)j[e] * K + c);
  }
}

template <typename T, int K, int E, bool PF>
__global__ void __launch_bounds__(256) k_trsv_ell(EllArgs<T> a) {
  constexpr int RPW = 32 / K;
  typedef typename Bits<T>::U U;
  const U sent = (U)Sentinel<T>::bits;
  const int lane = threadIdx.x & 31;
  const int c = lane % K;
  const int grp = lane / K;
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int s = warp % a.S;
  int *ctr = a.ctr + 32 * s;
  int pend = 0;
  if (lane == 0) pend = atomicAdd(ctr, 1);
  int t = __shfl_sync(0xffffffffu, pend, 0) * a.S + s;
  if (lane == 0) pend = atomicAdd(ctr, 1);
  int tn = __shfl_sync(0xffffffffu, pend, 0) * a.S + s;
  if (lane == 0) pend = atomicAdd(ctr, 1);
  EllMeta<T, E> m, mn;
  auto slot_of = [&](int tt) {
    return a.toff ? (tt < a.ntask ? a.toff[tt] : make_int2(0, 0)) : make_int2(tt * E * RPW, E);
  };
  int2 to = slot_of(t);
  int2 ton = slot_of(tn);
  if (t < a.ntask) ell_meta<T, E, RPW>(a, t, grp, to, m);
  while (t < a.ntask) {
    if (PF && tn < a.ntask) ell_meta<T, E, RPW>(a, tn, grp, ton, mn);
    unsigned long long t0 = 0;
    if (a.trace) t0 = gtimer();
    if (m.o >= 0) {
      const size_t oc = (size_t)m.o * K + c;
      T rhs = a.rhs_src[oc];
      if (a.rhs_scale) rhs = rhs * a.rhs_scale[m.o];
      T acc = T(0);
      // older dependencies beyond the E slots, four loads in flight at a time
      for (int q = m.q0; q < m.q1; q += 4) {
        U raw[4];
        int jj[4];
        T vv[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const bool has = q + e < m.q1;
          jj[e] = has ? a.ovj[q + e] : 0;
          vv[e] = has ? a.ovv[q + e] : T(0);
          raw[e] = has ? Bits<T>::load(a.cur + (size_t)jj[e] * K + c) : (U)0;
        }
        ell_wait<T, 4, K>(raw, jj, a.cur, c, a.err, a.backoff);
#pragma unroll
        for (int e = 0; e < 4; ++e) acc = fma(vv[e], Bits<T>::from(raw[e] == sent ? (U)0 : raw[e]), acc);
      }
      U raw[E];
#pragma unroll
      for (int e = 0; e < E; ++e) raw[e] = m.j[e] >= 0 ? Bits<T>::load(a.cur + (size_t)m.j[e] * K + c) : (U)0;
      ell_wait<T, E, K>(raw, m.j, a.cur, c, a.err, a.backoff);
#pragma unroll
      for (int e = 0; e < E; ++e) acc = fma(m.v[e], Bits<T>::from(raw[e] == sent ? (U)0 : raw[e]), acc);
      const T r = Bits<T>::canon(rhs - acc);
      Bits<T>::store(a.cur + oc, r);
      if (a.other) a.other[oc] = Sentinel<T>::value();
      if (a.out) {
        T w = a.alpha * r;
        if (a.beta != T(0)) w = fma(a.beta, a.out[oc], w);
        a.out[oc] = w;
      }
    }
    if (a.trace) {
      __syncwarp();
      if (lane == 0) {
        a.trace[2 * (size_t)t] = t0;
        a.trace[2 * (size_t)t + 1] = gtimer();
      }
    }
    t = tn;
    to = ton;
    tn = __shfl_sync(0xffffffffu, pend, 0) * a.S + s;
    if (lane == 0) pend = atomicAdd(ctr, 1);
    ton = slot_of(tn);
    if (PF) {
      m = mn;
    } else if (t < a.ntask) {
      ell_meta<T, E, RPW>(a, t, grp, to, m);
    }
  }
  // the last warp to leave resets the ticket streams for the next launch
  if (lane == 0) {
    const int nw = (int)((gridDim.x * blockDim.x) >> 5);
    __threadfence();
    const int done = atomicAdd(a.ctr + 32 * a.S, 1);
    if (done == nw - 1) {
      for (int q = 0; q < a.S; ++q) a.ctr[32 * q] = 0;
      a.ctr[32 * a.S] = 0;
    }
  }
}

// column-major (ld) <-> row-interleaved (K) FP64 boundary conversions, with
// precision change; columns >= k are zero
template <typename T>
__global__ void k_to_interleaved(int n, int k, int K, int ld, const double *__restrict__ src, T *__restrict__ dst) {
  const long long total = (long long)n * K;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / K), c = (int)(t % K);
    dst[t] = c < k ? (T)src[(size_t)c * ld + i] : T(0);
  }
}
template <typename T>
__global__ void k_from_interleaved(int n, int k, int K, int ld, const T *__restrict__ src, double *__restrict__ dst) {
  const long long total = (long long)n * k;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / n), i = (int)(t % n);
    dst[(size_t)c * ld + i] = (double)src[(size_t)i * K + c];
  }
}

// ---------------------------------------------------------------------------
// Multi-column FP64 Krylov pieces: per-column dot products with fixed-order
// block partials (deterministic), per-column scalar updates.
constexpr int kRedBlocksM = 148;

// partial[b*2*K + q*K + c], q < 2: block b's share of sum_i x_q[i,c] * y_q[i,c]
template <int K>
__global__ void __launch_bounds__(256) k_dots_m(int n, int nq, const double *__restrict__ x0,
                                                const double *__restrict__ y0, const double *__restrict__ x1,
                                                const double *__restrict__ y1, double *partial) {
  __shared__ double sh[2][256];
  const int c = threadIdx.x % K;
  const int rl = threadIdx.x / K;          // row lane within the block
  constexpr int RPB = 256 / K;             // rows per block step
  double s0 = 0, s1 = 0;
  for (long long i = (long long)blockIdx.x * RPB + rl; i < n; i += (long long)gridDim.x * RPB) {
    const size_t t = (size_t)i * K + c;
    s0 = fma(x0[t], y0[t], s0);
    if (nq > 1) s1 = fma(x1[t], y1[t], s1);
  }
  sh[0][threadIdx.x] = s0;
  sh[1][threadIdx.x] = s1;
  __syncthreads();
  if (threadIdx.x < K) {
    double a0 = 0, a1 = 0;
    for (int r = 0; r < RPB; ++r) {
      a0 += sh[0][r * K + threadIdx.x];
      a1 += sh[1][r * K + threadIdx.x];
    }
    partial[(size_t)blockIdx.x * 2 * K + threadIdx.x] = a0;
    partial[(size_t)blockIdx.x * 2 * K + K + threadIdx.x] = a1;
  }
}

template <int K>
__global__ void k_dots_m_final(int nblocks, const double *partial, double *res) {
  // res[q*K + c], q < 2, summed over the blocks in a fixed order
  const int t = threadIdx.x;
  if (t >= 2 * K) return;
  double s = 0;
  for (int b = 0; b < nblocks; ++b) s += partial[(size_t)b * 2 * K + t];
  res[t] = s;
}

// Per-column FCG/CG state.  active[c] == 0 freezes a converged column;
// a column is active while ||r_c|| / ||b_c|| > tol (NaN stops it).
struct KrylovM {
  double dots[3 * 32];
  double beta_num[32], dq_prev[32], dq[32], dr[32], rr[32], rho[32], rho_old[32];
  double bn[32];
  double tol;
  int ncols;
  int active[32];
};

template <int K>
__global__ void k_scal_store_m(KrylovM *sc, int what) {
  const int c = threadIdx.x;
  if (c >= K) return;
  switch (what) {
    case 0:
      sc->beta_num[c] = sc->dots[c];
      sc->rho_old[c] = sc->rho[c];
      sc->rho[c] = sc->dots[c];
      break;
    case 1:
      sc->dq[c] = sc->dots[c];
      sc->dr[c] = sc->dots[K + c];
      break;
    case 2:
      sc->rr[c] = sc->dots[c];
      sc->dq_prev[c] = sc->dq[c];
      if (sc->active[c]) sc->active[c] = sqrt(fmax(sc->rr[c], 0.0)) / sc->bn[c] > sc->tol;
      break;
    case 3:  // after (b,b),(r,r): norms and the initial active set
      sc->bn[c] = sc->dots[c] == 0.0 ? 1.0 : sqrt(sc->dots[c]);
      sc->rr[c] = sc->dots[K + c];
      sc->active[c] = c < sc->ncols && sqrt(sc->rr[c]) / sc->bn[c] > sc->tol;
      break;
  }
}

template <int K>
__global__ void k_dir_update_m(int n, int method, int first, const double *__restrict__ z, double *d,
                               const KrylovM *sc) {
  const long long total = (long long)n * K;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t % K);
    if (first) {
      d[t] = z[t];
    } else if (sc->active[c]) {
      const double beta = (method == 1) ? -(sc->beta_num[c] / sc->dq_prev[c]) : (sc->rho[c] / sc->rho_old[c]);
      d[t] = fma(beta, d[t], z[t]);
    }
  }
}

template <int K>
__global__ void k_xr_update_m(int n, int method, const double *__restrict__ d, const double *__restrict__ q,
                              double *x, double *r, const KrylovM *sc) {
  const long long total = (long long)n * K;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t % K);
    if (!sc->active[c]) continue;
    const double alpha = (method == 1) ? sc->dr[c] / sc->dq[c] : sc->rho[c] / sc->dq[c];
    x[t] = fma(alpha, d[t], x[t]);
    r[t] = fma(-alpha, q[t], r[t]);
  }
}

}  // namespace mldg
