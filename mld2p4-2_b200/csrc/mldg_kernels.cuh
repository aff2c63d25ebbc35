// mldg_kernels.cuh -- sm_100a kernels of the multilevel V-cycle.
//
// Every kernel here is a memory-bound sparse or vector operation (no tensor
// cores).  Value type T is double (drop-in form) or float (precision form).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mldg {

// ---------------------------------------------------------------------------
// Sentinel values marking "not yet computed" entries of a triangular-solve
// exchange buffer.  They are signalling NaNs: arithmetic never produces them
// (results are canonical quiet NaNs), and the solve canonicalises any NaN it
// stores, so a computed value can never be mistaken for the sentinel.
template <typename T> struct Sentinel;
template <> struct Sentinel<double> {
  static constexpr unsigned long long bits = 0x7FF4DEADBEEF0001ull;
  __device__ __host__ static double value() {
    union { unsigned long long u; double d; } c{bits};
    return c.d;
  }
};
template <> struct Sentinel<float> {
  static constexpr unsigned int bits = 0x7FA0BEEFu;
  __device__ __host__ static float value() {
    union { unsigned int u; float f; } c{bits};
    return c.f;
  }
};

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const void *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int ld_relaxed_u32(const void *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(void *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u32(void *p, unsigned int v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename T> struct Bits;
template <> struct Bits<double> {
  typedef unsigned long long U;
  __device__ static U load(const double *p) { return ld_relaxed_u64(p); }
  __device__ static void store(double *p, double v) {
    st_relaxed_u64(p, __double_as_longlong(v));
  }
  __device__ static double from(U u) { return __longlong_as_double((long long)u); }
  __device__ static double canon(double v) {
    return isnan(v) ? __longlong_as_double(0x7FF8000000000000ll) : v;
  }
};
template <> struct Bits<float> {
  typedef unsigned int U;
  __device__ static U load(const float *p) { return ld_relaxed_u32(p); }
  __device__ static void store(float *p, float v) { st_relaxed_u32(p, __float_as_uint(v)); }
  __device__ static float from(U u) { return __uint_as_float(u); }
  __device__ static float canon(float v) { return isnan(v) ? __uint_as_float(0x7FC00000u) : v; }
};

// Spin-wait limits: a wait that exceeds kSpinLimit polls records
// MLDG_ERR_TIMEOUT in *err and returns 0; every other waiter checks *err every
// kSpinCheck polls and leaves at once, so a failed solve drains quickly.
constexpr int kSpinLimit = 1 << 22;
constexpr int kSpinCheck = 64;
constexpr int kErrTimeout = 4020;

template <typename T>
__device__ __forceinline__ T wait_value(const T *p, int *err) {
  typedef typename Bits<T>::U U;
  const U sent = (U)Sentinel<T>::bits;
  U v = Bits<T>::load(p);
  if (v != sent) return Bits<T>::from(v);
  for (int it = 1; it < kSpinLimit; ++it) {
    v = Bits<T>::load(p);
    if (v != sent) return Bits<T>::from(v);
    if ((it % kSpinCheck) == 0) {
      if (ld_relaxed_u32(err) != 0u) return T(0);
      __nanosleep(32);
    }
  }
  atomicExch(err, kErrTimeout);
  return T(0);
}

// ---------------------------------------------------------------------------
// CSR SpMV family:  out[i] = a0*b[i] + a1*(A v)[i] + a2*out[i]
// TPR lanes cooperate on one row (TPR in {1,2,4,8,16,32}); each warp walks a
// contiguous block of 32/TPR rows per step, so shuffles always see a full warp.
// Reference ops: psb_spmm (residual, mld_dmlprec_aply.f90:674,752),
// psb_map_X2Y / psb_map_Y2X (restriction :682, prolongation :707).
template <typename T, int TPR>
__global__ void __launch_bounds__(256) k_spmv(int nr, const int *__restrict__ irp,
                                              const int *__restrict__ ja,
                                              const T *__restrict__ val,
                                              const T *__restrict__ v, T a1,
                                              const T *__restrict__ b, T a0, T *out, T a2) {
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int grp = lane / TPR;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int r0 = warp * RPW; r0 < nr; r0 += nwarps * RPW) {
    const int row = r0 + grp;
    T s = T(0);
    if (row < nr) {
      const int e = irp[row + 1];
      for (int k = irp[row] + sub; k < e; k += TPR) s = fma(val[k], __ldg(v + ja[k]), s);
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    if (row < nr && sub == 0) {
      T r = a1 * s;
      if (b) r = fma(a0, b[row], r);
      if (a2 != T(0)) r = fma(a2, out[row], r);
      out[row] = r;
    }
  }
}

// FP16-valued prolongator with an FP32 per-row scale (precision form):
// out[i] += scale[i] * sum_j h_ij v_j
template <int TPR>
__global__ void __launch_bounds__(256) k_spmv_h(int nr, const int *__restrict__ irp,
                                                const int *__restrict__ ja,
                                                const __half *__restrict__ hval,
                                                const float *__restrict__ scale,
                                                const float *__restrict__ v, float *out) {
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int grp = lane / TPR;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int r0 = warp * RPW; r0 < nr; r0 += nwarps * RPW) {
    const int row = r0 + grp;
    float s = 0.f;
    if (row < nr) {
      const int e = irp[row + 1];
      for (int k = irp[row] + sub; k < e; k += TPR)
        s = fmaf(__half2float(hval[k]), __ldg(v + ja[k]), s);
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    if (row < nr && sub == 0) out[row] = fmaf(scale[row], s, out[row]);
  }
}

// ---------------------------------------------------------------------------
// Point-Jacobi sweep (jac smoother + diag solver,
// mld_d_jac_smoother_apply_vect.f90:161-175 with diag_solver :102):
//   t_i  = d_i * (x_i - sum_j ND_ij ty_j)
//   v_i  = (omega == 1) ? t_i : (1-omega)*ty_i + omega*t_i        (damping: extension)
//   out_i = alpha*v_i + beta*out_i
// When first != 0 the incoming iterate is ty = omega*d o x (the unrolled first
// sweep, :136), computed on the fly from x and d instead of being stored.
template <typename T, int TPR>
__global__ void __launch_bounds__(256) k_jacobi(int nr, const int *__restrict__ irp,
                                                const int *__restrict__ ja,
                                                const T *__restrict__ val,
                                                const T *__restrict__ d,
                                                const T *__restrict__ x,
                                                const T *__restrict__ ty, int first,
                                                T omega, T alpha, T beta, T *out) {
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int grp = lane / TPR;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int r0 = warp * RPW; r0 < nr; r0 += nwarps * RPW) {
    const int row = r0 + grp;
    T s = T(0);
    if (row < nr) {
      const int e = irp[row + 1];
      if (first) {
        for (int k = irp[row] + sub; k < e; k += TPR) {
          const int j = ja[k];
          s = fma(val[k], omega * (__ldg(d + j) * __ldg(x + j)), s);
        }
      } else {
        for (int k = irp[row] + sub; k < e; k += TPR) s = fma(val[k], __ldg(ty + ja[k]), s);
      }
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    if (row < nr && sub == 0) {
      const T di = d[row], xi = x[row];
      T t = di * (xi - s);
      T v;
      if (omega == T(1)) {
        v = t;
      } else {
        const T tyi = first ? omega * (di * xi) : ty[row];
        v = (T(1) - omega) * tyi + omega * t;
      }
      T r = alpha * v;
      if (beta != T(0)) r = fma(beta, out[row], r);
      out[row] = r;
    }
  }
}

// out = alpha * d o x + beta * out     (diag solver apply, :102)
template <typename T>
__global__ void k_diag(int n, const T *__restrict__ d, const T *__restrict__ x, T alpha, T beta,
                       T *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T r = alpha * (d[i] * x[i]);
    if (beta != T(0)) r = fma(beta, out[i], r);
    out[i] = r;
  }
}

template <typename A, typename B>
__global__ void k_cast(int n, const A *__restrict__ x, B *__restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = (B)x[i];
}

template <typename T>
__global__ void k_fill(int n, T v, T *__restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = v;
}

// ---------------------------------------------------------------------------
// Sparse unit-triangular solve, chunked and level-scheduled.
//
// The factor is stored "lower in internal numbering": for an upper factor the
// rows are reversed (internal i' = n-1-i), so every dependency j' < i'.  Rows
// are cut into chunks of R consecutive internal rows; inside a chunk they are
// permuted by dependency level (intra-chunk edges only) and stored in that
// order (prow/pirp/pja/pval).  A CTA takes chunks in increasing order from a
// ticket counter; it walks the chunk level by level with the chunk's partial
// solution in shared memory and one __syncthreads per level.  Dependencies on
// earlier chunks are read from the exchange buffer `cur`, whose entries hold
// the sentinel until produced (no flags, no fences: the value is the flag).
// Chunks only wait on earlier chunks, which were claimed earlier by CTAs that
// are running or finished, so the scheme cannot deadlock; every wait is
// bounded (wait_value).
//
// rhs_i = rhs_src[o] * (rhs_scale ? rhs_scale[o] : 1), o = original row.
// After the solve row o holds t_o in cur[o]; `other[o]` is reset to the
// sentinel (it is the exchange buffer of the previous solve, already
// consumed; when rhs_src == other it is read before being reset).
// When out != null: out[o] = alpha * t_o + beta * out[o].
// Reference op: psb_spsm on the ILU factors,
// mlprec/impl/solver/mld_d_ilu_solver_apply_vect.f90:130-142.
template <typename T>
struct TriArgs {
  int n;
  int rev;
  int R;
  int nchunks;
  const int *chunk_lvl;
  const int *lvl_ptr;
  const int *prow;
  const int *pirp;
  const int *pja;
  const T *pval;
  const T *rhs_src;
  const T *rhs_scale;
  T *cur;
  T *other;
  T *out;
  T alpha;
  T beta;
  int *counters;  // [0] = chunk ticket, [1] = finished CTAs (self-resetting)
  int *err;
};

template <typename T, int TPR>
__global__ void __launch_bounds__(256) k_trsv(TriArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *ysm = reinterpret_cast<T *>(smem_raw);
  __shared__ int s_chunk;
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int grp = lane / TPR;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const T sent = Sentinel<T>::value();
  for (;;) {
    if (threadIdx.x == 0) s_chunk = atomicAdd(&a.counters[0], 1);
    __syncthreads();
    const int c = s_chunk;
    __syncthreads();
    if (c >= a.nchunks) break;
    const int s = c * a.R;
    const int l0 = a.chunk_lvl[c], l1 = a.chunk_lvl[c + 1];
    for (int L = l0; L < l1; ++L) {
      const int p0 = a.lvl_ptr[L], p1 = a.lvl_ptr[L + 1];
      for (int q0 = p0 + warp * RPW; q0 < p1; q0 += nwarps * RPW) {
        const int p = q0 + grp;
        T acc = T(0);
        int i = 0;
        if (p < p1) {
          i = a.prow[p];
          const int e = a.pirp[p + 1];
          for (int k = a.pirp[p] + sub; k < e; k += TPR) {
            const int j = a.pja[k];
            T yj;
            if (j >= s) {
              yj = ysm[j - s];
            } else {
              const int oj = a.rev ? (a.n - 1 - j) : j;
              yj = wait_value<T>(a.cur + oj, a.err);
            }
            acc = fma(a.pval[k], yj, acc);
          }
        }
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, TPR);
        if (p < p1 && sub == 0) {
          const int o = a.rev ? (a.n - 1 - i) : i;
          T r = a.rhs_src[o];
          if (a.rhs_scale) r = r * a.rhs_scale[o];
          const T t = Bits<T>::canon(r - acc);
          ysm[i - s] = t;
          Bits<T>::store(a.cur + o, t);
          if (a.other) a.other[o] = sent;
          if (a.out) {
            T w = a.alpha * t;
            if (a.beta != T(0)) w = fma(a.beta, a.out[o], w);
            a.out[o] = w;
          }
        }
      }
      __syncthreads();
    }
  }
  // the last CTA to leave resets the counters for the next launch
  if (threadIdx.x == 0) {
    const int done = atomicAdd(&a.counters[1], 1);
    if (done == (int)gridDim.x - 1) {
      a.counters[0] = 0;
      a.counters[1] = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// Deterministic FP64 reductions for the Krylov loop: fixed grid, per-block
// partials, then one block sums the partials in a fixed order.
constexpr int kRedBlocks = 296;  // 2 x 148 SMs
constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
  if (w == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  return v;
}

// partial[b*np + k] for k < np: up to 3 dot products in one pass
__global__ void __launch_bounds__(kRedThreads) k_dots(int n, int np, const double *__restrict__ x0,
                                                     const double *__restrict__ y0,
                                                     const double *__restrict__ x1,
                                                     const double *__restrict__ y1,
                                                     const double *__restrict__ x2,
                                                     const double *__restrict__ y2,
                                                     double *partial) {
  __shared__ double sh[32];
  double s0 = 0, s1 = 0, s2 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    s0 = fma(x0[i], y0[i], s0);
    if (np > 1) s1 = fma(x1[i], y1[i], s1);
    if (np > 2) s2 = fma(x2[i], y2[i], s2);
  }
  s0 = block_sum(s0, sh);
  if (np > 1) s1 = block_sum(s1, sh);
  if (np > 2) s2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    partial[blockIdx.x * 3 + 0] = s0;
    partial[blockIdx.x * 3 + 1] = s1;
    partial[blockIdx.x * 3 + 2] = s2;
  }
}

__global__ void __launch_bounds__(kRedThreads) k_dots_final(int nblocks, const double *partial,
                                                           double *res) {
  __shared__ double sh[32];
  for (int k = 0; k < 3; ++k) {
    double s = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partial[b * 3 + k];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) res[k] = s;
  }
}

// Krylov scalar state kept on the device (no host round trip per kernel).
struct KrylovScalars {
  double dots[3];     // scratch results of the last k_dots_final
  double beta_num;    // (z, q_prev)
  double dq_prev;     // (d_prev, q_prev)
  double dq;          // (d, q)
  double dr;          // (d, r)
  double rr;          // (r, r)
  double rho, rho_old;
};

// FCG direction update: d = z - beta*d with beta = beta_num/dq_prev
// (first iteration: d = z).  CG: d = z + (rho/rho_old) d.
__global__ void k_dir_update(int n, int method, int first, const double *__restrict__ z,
                             double *d, const KrylovScalars *sc) {
  double beta = 0.0;
  if (!first) beta = (method == 1) ? -(sc->beta_num / sc->dq_prev) : (sc->rho / sc->rho_old);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    d[i] = first ? z[i] : fma(beta, d[i], z[i]);
}

// x += alpha d ; r -= alpha q ; alpha = num/dq, plus partial ||r||^2
__global__ void __launch_bounds__(kRedThreads) k_xr_update(int n, int method,
                                                          const double *__restrict__ d,
                                                          const double *__restrict__ q,
                                                          double *x, double *r,
                                                          const KrylovScalars *sc,
                                                          double *partial) {
  __shared__ double sh[32];
  const double alpha = (method == 1) ? sc->dr / sc->dq : sc->rho / sc->dq;
  double s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = fma(alpha, d[i], x[i]);
    const double ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    s = fma(ri, ri, s);
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    partial[blockIdx.x * 3 + 0] = s;
    partial[blockIdx.x * 3 + 1] = 0;
    partial[blockIdx.x * 3 + 2] = 0;
  }
}

// copy reduction results into named scalar slots
__global__ void k_scal_store(KrylovScalars *sc, int what) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  switch (what) {
    case 0:  // after (z,q_prev) [FCG] or (r,z) [CG]
      sc->beta_num = sc->dots[0];
      sc->rho_old = sc->rho;
      sc->rho = sc->dots[0];
      break;
    case 1:  // after (d,q),(d,r)
      sc->dq = sc->dots[0];
      sc->dr = sc->dots[1];
      break;
    case 2:  // after ||r||^2
      sc->rr = sc->dots[0];
      sc->dq_prev = sc->dq;
      break;
  }
}

}  // namespace mldg
