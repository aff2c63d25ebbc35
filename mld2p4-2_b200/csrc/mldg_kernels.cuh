// mldg_kernels.cuh -- sm_100a kernels of the multilevel V-cycle.
//
// Every kernel here is a memory-bound sparse or vector operation (no tensor
// cores).  Value type T is double (drop-in form) or float (precision form).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

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

// Programmatic dependent launch.  A kernel launched with the programmatic
// stream-serialization attribute may be scheduled while the kernel before it
// in the stream is still finishing; pdl_enter() first waits until that
// kernel has completed and its writes are visible (so it must run before
// the kernel touches any memory), then allows the next kernel in the stream
// to be scheduled early in turn.  Both instructions are no-ops in a kernel
// launched without the attribute.  Every kernel that the host may launch
// with the attribute calls it first, so completion stays transitive along
// the stream.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Spin-wait limits: a wait that exceeds kSpinLimit polls records
// MLDG_ERR_TIMEOUT in *err and returns 0; every other waiter checks *err every
// kSpinCheck polls and leaves at once, so a failed solve drains quickly.
constexpr int kSpinLimit = 1 << 22;
constexpr int kSpinCheck = 64;
constexpr int kErrTimeout = 4020;
// The limit in force (kSpinLimit unless a test lowers it through
// mldg_test_set_spin_limit to make waits run out on purpose).  Only these
// sentinel polls of global memory read it; the mbarrier waits of the window
// and cluster solves keep their fixed limit.
static __device__ int g_spin_limit = kSpinLimit;
__device__ __forceinline__ int spin_limit() { return *(volatile int *)&g_spin_limit; }

template <typename T>
__device__ __forceinline__ T wait_value(const T *p, int *err) {
  typedef typename Bits<T>::U U;
  const U sent = (U)Sentinel<T>::bits;
  U v = Bits<T>::load(p);
  if (v != sent) return Bits<T>::from(v);
  const int lim = spin_limit();
  for (int it = 1; it < lim; ++it) {
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
// Column of entry k of row `row`: absolute int32 indices, or int16 offsets
// from the row (square matrices whose entries all lie within 32767 of the
// diagonal: 2 bytes per entry instead of 4 on a bandwidth-bound sweep).
__device__ __forceinline__ int colof(const int *__restrict__ cj, int k, int) { return cj[k]; }
__device__ __forceinline__ int colof(const short *__restrict__ cj, int k, int row) { return row + (int)cj[k]; }
// Stored value of entry k widened to the vector type T: values of the
// matrix's own type, or FP16 values of a row-scaled copy (the FP16 operator
// form: a_ij = rs_i * h_ij, rs_i = max_j |a_ij| in FP32), whose row sum the
// epilogue multiplies by rs_i (row_scaled).
template <typename T, typename V>
__device__ __forceinline__ T ldval(const V *__restrict__ p, int64_t k) {
  if constexpr (std::is_same<V, __half>::value)
    return (T)__half2float(p[k]);
  else
    return p[k];
}
// (a rounded product that is never contracted into a later add: every
// kernel rounds the scaled row sum alike)
template <typename T, typename V>
__device__ __forceinline__ T row_scaled(T acc, const float *__restrict__ rs, int row) {
  if constexpr (std::is_same<V, __half>::value) {
    if constexpr (std::is_same<T, float>::value)
      return __fmul_rn(acc, rs[row]);
    else
      return __dmul_rn(acc, (double)rs[row]);
  } else {
    return acc;
  }
}

// The point-Jacobi update of one row from its off-diagonal sum s, every
// operation explicit (no multiply-add left to contraction), so that all the
// Jacobi kernels round alike: t = d_i (x_i - s); v = t when omega = 1, else
// (1 - omega) ty_i + omega t with ty_i = omega d_i x_i on the unrolled first
// sweep; result alpha v + beta out_i.
template <typename T>
__device__ __forceinline__ T jac_row(T di, T xi, T s, T tyi, bool first, T omega, T alpha, T beta, T outi) {
  const T t = di * (xi - s);
  T v = t;
  if (omega != T(1)) {
    const T ty0 = first ? omega * (di * xi) : tyi;
    v = fma(omega, t, (T(1) - omega) * ty0);
  }
  const T r = alpha * v;
  return beta != T(0) ? fma(beta, outi, r) : r;
}

// One lane's part of a CSR row sum: entries k = k0, k0 + TPR, ... < e,
// s = fma(val[k], g(col k), s) in that order from zero.  The loads are
// issued U entries at a time (column indices and values, then the gathers
// g, then the sums), so a long row costs two memory latencies per U entries
// instead of two per entry; the sums are the plain loop's.  U grows with the
// lanes per row, which the autotuner picks wide for long rows: 4 entries per
// lane below 4 lanes per row, 8 up to 8 lanes, 16 from 16 lanes (a coarse
// level's row of ~300 entries then takes one batch).
template <int TPR>
struct CsrU {
  static constexpr int value = TPR >= 16 ? 16 : (TPR >= 4 ? 8 : 4);
};
template <typename T, int TPR, typename CI, typename V, typename G>
__device__ __forceinline__ T csr_lane_sum(int k0, int e, int row, const CI *__restrict__ ja,
                                          const V *__restrict__ val, G g) {
  constexpr int kCsrU = CsrU<TPR>::value;
  T s = T(0);
  for (int k = k0; k < e; k += TPR * kCsrU) {
    T vv[kCsrU], xv[kCsrU];
#pragma unroll
    for (int u = 0; u < kCsrU; ++u) {
      const int kk = k + u * TPR;
      const bool ok = kk < e;
      vv[u] = ok ? ldval<T>(val, kk) : T(0);
      xv[u] = ok ? g(colof(ja, kk, row)) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kCsrU; ++u)
      if (k + u * TPR < e) s = fma(vv[u], xv[u], s);
  }
  return s;
}

template <typename T, int TPR, typename CI = int, typename V = T>
__global__ void __launch_bounds__(256) k_spmv(int nr, const int *__restrict__ irp,
                                              const CI *__restrict__ ja,
                                              const V *__restrict__ val,
                                              const T *__restrict__ v, T a1,
                                              const T *__restrict__ b, T a0, T *out, T a2,
                                              const float *__restrict__ rs = nullptr) {
  pdl_enter();
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int grp = lane / TPR;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int r0 = warp * RPW; r0 < nr; r0 += nwarps * RPW) {
    const int row = r0 + grp;
    T s = T(0);
    if (row < nr)
      s = csr_lane_sum<T, TPR>(irp[row] + sub, irp[row + 1], row, ja, val, [&](int j) { return __ldg(v + j); });
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    if (row < nr && sub == 0) {
      T r = a1 * row_scaled<T, V>(s, rs, row);
      if (b) r = fma(a0, b[row], r);
      if (a2 != T(0)) r = fma(a2, out[row], r);
      out[row] = r;
    }
  }
}

// ---------------------------------------------------------------------------
// The same operators on a sliced-ELL copy of the matrix (SELL-32): rows in
// slices of 32, slice s holding its rows' k-th entries at
// soff[s] + 32*k + lane (k < the slice's longest row; shorter rows padded
// with zero values on an in-range column).  One thread per row: the 32
// threads of a warp read 32 consecutive values and column indices per entry,
// and every thread issues SELL_U entries' loads before using them, so many
// more bytes are in flight per warp than with lanes sharing a short CSR row.
// A row's entries are summed in stored order from zero.
constexpr int kSellU = 8;

__device__ __forceinline__ int sell_col(const int *__restrict__ sj, int k, int) { return sj[k]; }
__device__ __forceinline__ int sell_col(const short *__restrict__ sj, int k, int row) { return row + (int)sj[k]; }

// acc[s] = sum over the slots of slice sl0 + s (s < S) for the thread's row
// of that slice, the S slices' loads of each block of kSellU entries issued
// together (S = 2 doubles the bytes in flight per warp, for short FP32 rows)
template <typename T, typename CI, int S, typename F, typename V>
__device__ __forceinline__ void sell_rows(const int *__restrict__ soff, const CI *__restrict__ sj,
                                          const V *__restrict__ sv, int sl0, int ns, int lane, F f,
                                          T (&acc)[S]) {
  int e[S], e1[S], row[S];
#pragma unroll
  for (int q = 0; q < S; ++q) {
    const int sl = sl0 + q;
    const bool ok = sl < ns;
    e[q] = ok ? soff[sl] + lane : 0;
    e1[q] = ok ? soff[sl + 1] : 0;
    row[q] = (sl << 5) + lane;
    acc[q] = T(0);
  }
  for (;;) {
    bool more = false;
#pragma unroll
    for (int q = 0; q < S; ++q) more |= e[q] < e1[q];
    if (!more) break;
    T vv[S][kSellU];
    int jj[S][kSellU];
#pragma unroll
    for (int q = 0; q < S; ++q)
#pragma unroll
      for (int u = 0; u < kSellU; ++u) {
        const int k = e[q] + 32 * u;
        const bool ok = k < e1[q];
        vv[q][u] = ok ? ldval<T>(sv, k) : T(0);
        jj[q][u] = ok ? sell_col(sj, k, row[q]) : 0;
      }
#pragma unroll
    for (int q = 0; q < S; ++q) {
#pragma unroll
      for (int u = 0; u < kSellU; ++u)
        if (e[q] + 32 * u < e1[q]) acc[q] = fma(vv[q][u], f(jj[q][u]), acc[q]);
      e[q] += 32 * kSellU;
    }
  }
}

// out[i] = a0*b[i] + a1*(A v)[i] + a2*out[i]; S slices per warp iteration
template <typename T, typename CI, int S, typename V = T>
__global__ void __launch_bounds__(256) k_spmv_sell(int nr, const int *__restrict__ soff,
                                                   const CI *__restrict__ sj, const V *__restrict__ sv,
                                                   const T *__restrict__ v, T a1, const T *__restrict__ b,
                                                   T a0, T *out, T a2,
                                                   const float *__restrict__ rs = nullptr) {
  pdl_enter();
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int ns = (nr + 31) >> 5;
  for (int sl0 = warp * S; sl0 < ns; sl0 += nwarps * S) {
    T acc[S];
    sell_rows<T, CI, S>(soff, sj, sv, sl0, ns, lane, [&](int j) { return __ldg(v + j); }, acc);
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const int row = ((sl0 + q) << 5) + lane;
      if (row < nr) {
        T r = a1 * row_scaled<T, V>(acc[q], rs, row);
        if (b) r = fma(a0, b[row], r);
        if (a2 != T(0)) r = fma(a2, out[row], r);
        out[row] = r;
      }
    }
  }
}

// SELL loop with the slices of a warp software-pipelined: the values and
// column indices of the warp's next slice (first kSellU entries) and the
// offsets of the one after are loaded before the current slice's vector
// gathers and sums, so a warp keeps two slices' loads in flight instead of
// waiting for each slice's offsets, then its entries, then its gathers.
// f(j): the vector entry an entry of column j multiplies; done(row, acc): the
// epilogue of a row (row < nr).
template <typename T, typename CI, typename F, typename D, typename V>
__device__ __forceinline__ void sellp_loop(int nr, const int *__restrict__ soff, const CI *__restrict__ sj,
                                           const V *__restrict__ sv, F f, D done) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int ns = (nr + 31) >> 5;
  int sl = warp;
  if (sl >= ns) return;
  auto load = [&](int e, int e1, int row, T (&vv)[kSellU], int (&jj)[kSellU]) {
#pragma unroll
    for (int u = 0; u < kSellU; ++u) {
      const int k = e + 32 * u;
      const bool ok = k < e1;
      vv[u] = ok ? ldval<T>(sv, k) : T(0);
      jj[u] = ok ? sell_col(sj, k, row) : 0;
    }
  };
  int ec = soff[sl] + lane, e1c = soff[sl + 1];
  T vc[kSellU];
  int jc[kSellU];
  load(ec, e1c, (sl << 5) + lane, vc, jc);
  int sn = sl + nwarps;
  int en = sn < ns ? soff[sn] + lane : 0, e1n = sn < ns ? soff[sn + 1] : 0;
  for (;;) {
    // next slice's first block and the offsets of the one after, issued now
    T vn[kSellU];
    int jn[kSellU];
    load(en, e1n, (sn << 5) + lane, vn, jn);
    const int snn = sn + nwarps;
    const int enn = snn < ns ? soff[snn] + lane : 0, e1nn = snn < ns ? soff[snn + 1] : 0;
    // the current slice
    const int row = (sl << 5) + lane;
    T acc = T(0);
#pragma unroll
    for (int u = 0; u < kSellU; ++u)
      if (ec + 32 * u < e1c) acc = fma(vc[u], f(jc[u]), acc);
    for (int e = ec + 32 * kSellU; e < e1c; e += 32 * kSellU) {  // slices wider than kSellU
      T vv[kSellU];
      int jj[kSellU];
      load(e, e1c, row, vv, jj);
#pragma unroll
      for (int u = 0; u < kSellU; ++u)
        if (e + 32 * u < e1c) acc = fma(vv[u], f(jj[u]), acc);
    }
    if (row < nr) done(row, acc);
    if (sn >= ns) break;
    sl = sn;
    ec = en;
    e1c = e1n;
#pragma unroll
    for (int u = 0; u < kSellU; ++u) {
      vc[u] = vn[u];
      jc[u] = jn[u];
    }
    sn = snn;
    en = enn;
    e1n = e1nn;
  }
}

template <typename T, typename CI, typename V = T>
__global__ void __launch_bounds__(256) k_spmv_sellp(int nr, const int *__restrict__ soff,
                                                    const CI *__restrict__ sj, const V *__restrict__ sv,
                                                    const T *__restrict__ v, T a1, const T *__restrict__ b,
                                                    T a0, T *out, T a2,
                                                    const float *__restrict__ rs = nullptr) {
  pdl_enter();
  sellp_loop<T, CI>(
      nr, soff, sj, sv, [&](int j) { return __ldg(v + j); },
      [&](int row, T acc) {
        T r = a1 * row_scaled<T, V>(acc, rs, row);
        if (b) r = fma(a0, b[row], r);
        if (a2 != T(0)) r = fma(a2, out[row], r);
        out[row] = r;
      });
}

// the Jacobi sweep of k_jacobi_sell, software-pipelined like k_spmv_sellp
template <typename T, typename CI, typename V = T>
__global__ void __launch_bounds__(256) k_jacobi_sellp(int nr, const int *__restrict__ soff,
                                                      const CI *__restrict__ sj, const V *__restrict__ sv,
                                                      const T *__restrict__ d, const T *__restrict__ x,
                                                      const T *__restrict__ ty, int first, T omega, T alpha,
                                                      T beta, T *out, const float *__restrict__ rs = nullptr) {
  pdl_enter();
  auto done = [&](int row, T acc) {
    out[row] = jac_row(d[row], x[row], row_scaled<T, V>(acc, rs, row), (!first && omega != T(1)) ? ty[row] : T(0),
                       first != 0, omega, alpha, beta, beta != T(0) ? out[row] : T(0));
  };
  if (first == 2)
    sellp_loop<T, CI>(nr, soff, sj, sv, [&](int j) { return omega * __ldg(x + j); }, done);
  else if (first)
    sellp_loop<T, CI>(
        nr, soff, sj, sv, [&](int j) { return omega * (__ldg(d + j) * __ldg(x + j)); }, done);
  else
    sellp_loop<T, CI>(nr, soff, sj, sv, [&](int j) { return __ldg(ty + j); }, done);
}

// the point-Jacobi sweep of k_jacobi on the SELL copy of ND
template <typename T, typename CI, int S, typename V = T>
__global__ void __launch_bounds__(256) k_jacobi_sell(int nr, const int *__restrict__ soff,
                                                     const CI *__restrict__ sj, const V *__restrict__ sv,
                                                     const T *__restrict__ d, const T *__restrict__ x,
                                                     const T *__restrict__ ty, int first, T omega, T alpha,
                                                     T beta, T *out, const float *__restrict__ rs = nullptr) {
  pdl_enter();
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int ns = (nr + 31) >> 5;
  for (int sl0 = warp * S; sl0 < ns; sl0 += nwarps * S) {
    T acc[S];
    if (first == 2)
      sell_rows<T, CI, S>(soff, sj, sv, sl0, ns, lane, [&](int j) { return omega * __ldg(x + j); }, acc);
    else if (first)
      sell_rows<T, CI, S>(soff, sj, sv, sl0, ns, lane,
                          [&](int j) { return omega * (__ldg(d + j) * __ldg(x + j)); }, acc);
    else
      sell_rows<T, CI, S>(soff, sj, sv, sl0, ns, lane, [&](int j) { return __ldg(ty + j); }, acc);
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const int row = ((sl0 + q) << 5) + lane;
      if (row < nr)
        out[row] = jac_row(d[row], x[row], row_scaled<T, V>(acc[q], rs, row),
                           (!first && omega != T(1)) ? ty[row] : T(0), first != 0, omega, alpha, beta,
                           beta != T(0) ? out[row] : T(0));
    }
  }
}

// ---------------------------------------------------------------------------
// The same operators on a hacked-diagonal copy (HDIA-32) of a square matrix:
// rows in slices of 32; slice s lists the distinct column offsets j - i of
// its rows' entries, ascending, in doff[dptr[s] .. dptr[s+1]), and stores the
// value of its k-th offset for row `lane` at hv[32*(dptr[s] + k) + lane]
// (zero where the row has no entry there).  No column index is stored per
// entry, so a level whose slices share a few diagonals (a stencil) moves
// only its values: 2 bytes per entry in the FP16 operator form instead of 4.
// A row's entries are summed in ascending column order from zero, the
// stored order of a column-sorted CSR row (the host builds the copy only for
// such matrices); a padding slot adds fma(0, v_j, s) = s for finite v_j, its
// column clamped into [0, n).  One warp per slice; the offsets are loaded by
// every lane (one broadcast access), kHdiaU diagonals' loads issued together.
// (Measured on the idim=160 level 0 against wider forms: 4 rows per thread
// with 8/16-byte accesses, 2 slices per warp, and offsets staged in shared
// memory per block all ran slower than this one-row-per-thread form, which
// the register limit of __launch_bounds__ keeps at full occupancy.)
// U = 4 for slices of a few diagonals (a stencil level), 16 for the long
// rows of a coarse level (more loads in flight per pass); the autotuner
// times both.
template <typename T, int U>
struct HdiaMinBlocks {  // 256-thread blocks per SM: 32 registers (FP32), 40 (FP64); U = 16 unbounded
  static constexpr int value = U > 4 ? 1 : (sizeof(T) == 8 ? 6 : 8);
};

template <typename T, int U = 4, typename F, typename V>
__device__ __forceinline__ T hdia_row(const int *__restrict__ dptr, const int *__restrict__ doff,
                                      const V *__restrict__ hv, int sl, int row, int n, int lane, F f) {
  constexpr int kHdiaU = U;
  int k = __ldg(dptr + sl);
  const int k1 = __ldg(dptr + sl + 1);
  T acc = T(0);
  for (; k < k1; k += kHdiaU) {  // k, k1 are the same in every lane of the warp
    T vv[kHdiaU], xv[kHdiaU];
#pragma unroll
    for (int u = 0; u < kHdiaU; ++u) {
      const bool ok = k + u < k1;
      const int off = ok ? __ldg(doff + k + u) : 0;
      vv[u] = ok ? ldval<T>(hv, ((k + u) << 5) + lane) : T(0);
      xv[u] = ok ? f(min(max(row + off, 0), n - 1)) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kHdiaU; ++u)
      if (k + u < k1) acc = fma(vv[u], xv[u], acc);
  }
  return acc;
}

// out[i] = a0*b[i] + a1*(A v)[i] + a2*out[i] on the HDIA copy of A
template <typename T, typename V = T, int U = 4>
__global__ void __launch_bounds__(256, (HdiaMinBlocks<T, U>::value))
    k_spmv_hdia(int nr, const int *__restrict__ dptr, const int *__restrict__ doff, const V *__restrict__ hv,
                const T *__restrict__ v, T a1, const T *__restrict__ b, T a0, T *out, T a2,
                const float *__restrict__ rs = nullptr) {
  pdl_enter();
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int ns = (nr + 31) >> 5;
  for (int sl = warp; sl < ns; sl += nwarps) {
    const int row = (sl << 5) + lane;
    const T acc = hdia_row<T, U>(dptr, doff, hv, sl, row, nr, lane, [&](int j) { return __ldg(v + j); });
    if (row < nr) {
      T r = a1 * row_scaled<T, V>(acc, rs, row);
      if (b) r = fma(a0, b[row], r);
      if (a2 != T(0)) r = fma(a2, out[row], r);
      out[row] = r;
    }
  }
}

// the point-Jacobi sweep of k_jacobi on the HDIA copy of ND
template <typename T, typename V = T, int U = 4>
__global__ void __launch_bounds__(256, (HdiaMinBlocks<T, U>::value))
    k_jacobi_hdia(int nr, const int *__restrict__ dptr, const int *__restrict__ doff, const V *__restrict__ hv,
                  const T *__restrict__ d, const T *__restrict__ x, const T *__restrict__ ty, int first, T omega,
                  T alpha, T beta, T *out, const float *__restrict__ rs = nullptr) {
  pdl_enter();
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int ns = (nr + 31) >> 5;
  for (int sl = warp; sl < ns; sl += nwarps) {
    const int row = (sl << 5) + lane;
    T acc;
    if (first == 2)
      acc = hdia_row<T, U>(dptr, doff, hv, sl, row, nr, lane, [&](int j) { return omega * __ldg(x + j); });
    else if (first)
      acc = hdia_row<T, U>(dptr, doff, hv, sl, row, nr, lane,
                           [&](int j) { return omega * (__ldg(d + j) * __ldg(x + j)); });
    else
      acc = hdia_row<T, U>(dptr, doff, hv, sl, row, nr, lane, [&](int j) { return __ldg(ty + j); });
    if (row < nr)
      out[row] = jac_row(d[row], x[row], row_scaled<T, V>(acc, rs, row),
                         (!first && omega != T(1)) ? ty[row] : T(0), first != 0, omega, alpha, beta,
                         beta != T(0) ? out[row] : T(0));
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
  pdl_enter();
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
// sweep, :136), computed on the fly from x and d instead of being stored;
// first == 2 says that ND's columns were scaled by d when it was stored
// (ND D), so the sweep gathers omega*x_j alone: one vector gather per entry
// instead of two.
template <typename T, int TPR, typename CI = int, typename V = T>
__global__ void __launch_bounds__(256) k_jacobi(int nr, const int *__restrict__ irp,
                                                const CI *__restrict__ ja,
                                                const V *__restrict__ val,
                                                const T *__restrict__ d,
                                                const T *__restrict__ x,
                                                const T *__restrict__ ty, int first,
                                                T omega, T alpha, T beta, T *out,
                                                const float *__restrict__ rs = nullptr) {
  pdl_enter();
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
      const int k0 = irp[row] + sub, e = irp[row + 1];
      if (first == 2)
        s = csr_lane_sum<T, TPR>(k0, e, row, ja, val, [&](int j) { return omega * __ldg(x + j); });
      else if (first)
        s = csr_lane_sum<T, TPR>(k0, e, row, ja, val, [&](int j) { return omega * (__ldg(d + j) * __ldg(x + j)); });
      else
        s = csr_lane_sum<T, TPR>(k0, e, row, ja, val, [&](int j) { return __ldg(ty + j); });
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    if (row < nr && sub == 0)
      out[row] = jac_row(d[row], x[row], row_scaled<T, V>(s, rs, row), (!first && omega != T(1)) ? ty[row] : T(0),
                         first != 0, omega, alpha, beta, beta != T(0) ? out[row] : T(0));
  }
}

// Dense coarsest-level solve: out = alpha * M x + beta * out with M the
// explicit inverse of the coarsest ILU(0) factorisation (row-major n x n),
// one warp per row.
template <typename T>
__global__ void __launch_bounds__(256) k_gemv(int n, const T *__restrict__ M, const T *__restrict__ x,
                                              T alpha, T beta, T *out) {
  pdl_enter();
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = warp; i < n; i += nwarps) {
    const T *row = M + (size_t)i * n;
    T s = T(0);
    for (int j = lane; j < n; j += 32) s = fma(row[j], __ldg(x + j), s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) {
      T r = alpha * s;
      if (beta != T(0)) r = fma(beta, out[i], r);
      out[i] = r;
    }
  }
}

// dL/dkappa of -div(kappa grad u) with harmonic-mean faces (see mldg.h)
__global__ void k_kappa_grad(int idim, double ih2, const double *__restrict__ kappa,
                             const double *__restrict__ x, const double *__restrict__ lam,
                             double *__restrict__ grad) {
  const long long s2 = (long long)idim * idim, n = s2 * idim;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(c / s2), iy = (int)((c / idim) % idim), iz = (int)(c % idim);
    const double kc = kappa[c], xc = x[c], lc = lam[c];
    const bool in[6] = {ix > 0, iy > 0, iz > 0, iz < idim - 1, iy < idim - 1, ix < idim - 1};
    const long long nb[6] = {c - s2, c - idim, c - 1, c + 1, c + idim, c + s2};
    double g = 0.0;
    for (int q = 0; q < 6; ++q) {
      if (in[q]) {
        const double ks = kappa[nb[q]], den = kc + ks;
        g += 2.0 * ks * ks / (den * den) * (lc - lam[nb[q]]) * (xc - x[nb[q]]);
      } else {
        g += lc * xc;
      }
    }
    grad[c] = -ih2 * g;
  }
}

// out = alpha * d o x + beta * out     (diag solver apply, :102)
template <typename T>
__global__ void k_diag(int n, const T *__restrict__ d, const T *__restrict__ x, T alpha, T beta,
                       T *out) {
  pdl_enter();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T r = alpha * (d[i] * x[i]);
    if (beta != T(0)) r = fma(beta, out[i], r);
    out[i] = r;
  }
}

template <typename A, typename B>
__global__ void k_cast(int n, const A *__restrict__ x, B *__restrict__ y) {
  pdl_enter();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = (B)x[i];
}

// Precision casts of the V-cycle's boundary vectors, four elements per
// thread with 16-byte loads and stores (both arrays 16-byte aligned; the
// host checks), the last n % 4 elements one per thread.
__device__ __forceinline__ void cast4_ld(const double *p, double (&v)[4]) {
  const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void cast4_ld(const float *p, float (&v)[4]) {
  const float4 a = *reinterpret_cast<const float4 *>(p);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void cast4_st(double *p, const double (&v)[4]) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void cast4_st(float *p, const float (&v)[4]) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
template <typename A, typename B>
__global__ void __launch_bounds__(256) k_cast4(int n, const A *__restrict__ x, B *__restrict__ y) {
  pdl_enter();
  const int n4 = n >> 2, stride = gridDim.x * blockDim.x, t = blockIdx.x * blockDim.x + threadIdx.x;
  for (int i = t; i < n4; i += stride) {
    A a[4];
    B b[4];
    cast4_ld(x + 4 * (int64_t)i, a);
#pragma unroll
    for (int u = 0; u < 4; ++u) b[u] = (B)a[u];
    cast4_st(y + 4 * (int64_t)i, b);
  }
  for (int i = 4 * n4 + t; i < n; i += stride) y[i] = (B)x[i];
}

template <typename T>
__global__ void k_fill(int n, T v, T *__restrict__ y) {
  pdl_enter();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = v;
}

// ---------------------------------------------------------------------------
// Sparse unit-triangular solve, level-scheduled.
//
// The factor is stored "lower in internal numbering": for an upper factor the
// rows are reversed (internal i' = n-1-i), so every dependency j' < i'.  Rows
// are sorted by dependency level (the longest chain of dependencies leading
// to them) and stored in that order (prow/pirp/pja/pval), so all rows of a
// level are independent and every dependency of a row sits at a smaller
// position.  Two kernels walk that order:
//   k_trsv_cta : one CTA, the whole solution in shared memory, one
//                __syncthreads per level, the next level's entries loaded
//                into registers while the current level is computed
//                (small levels).
//   k_trsv_sf  : all SMs, no barriers; warps claim consecutive blocks of
//                positions from a ticket counter, load their rows' entries,
//                then wait for each dependency on the exchange buffer `cur`,
//                whose entries hold a sentinel until produced (the value is
//                the flag).  Blocks are claimed in position order and every
//                dependency lies at an earlier position, so the waits always
//                end; each wait is bounded anyway (wait_value).
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
  int nlevels;
  const int *lvl_ptr;  // nlevels + 1 positions
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
  int *counters;  // [0] = block ticket, [1] = finished warps (self-resetting)
  int *err;
  // k_trsv_sf: warp blocks never straddle a level, so the rows of a block
  // are independent of one another (no lane waits on its own warp)
  int nblk;
  const int2 *blk;  // [first position, end position) per block
};

template <typename T>
__device__ __forceinline__ void tri_store(const TriArgs<T> &a, int o, T t) {
  Bits<T>::store(a.cur + o, t);
  if (a.other) a.other[o] = Sentinel<T>::value();
  if (a.out) {
    T w = a.alpha * t;
    if (a.beta != T(0)) w = fma(a.beta, a.out[o], w);
    a.out[o] = w;
  }
}

// One row's prefetched state: up to E entries per lane held in registers.
template <typename T, int E>
struct RowRegs {
  int i, o, k0, k1;  // internal row, original row, entry range of this lane
  T rhs;
  int j[E];
  T v[E];
};

template <typename T, int TPR, int E>
__device__ __forceinline__ void load_row(const TriArgs<T> &a, int p, int sub, RowRegs<T, E> &r) {
  r.i = a.prow[p];
  r.o = a.rev ? (a.n - 1 - r.i) : r.i;
  r.k0 = a.pirp[p] + sub;
  r.k1 = a.pirp[p + 1];
  r.rhs = a.rhs_src[r.o];
  if (a.rhs_scale) r.rhs = r.rhs * a.rhs_scale[r.o];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int k = r.k0 + e * TPR;
    if (k < r.k1) {
      r.j[e] = a.pja[k];
      r.v[e] = a.pval[k];
    } else {
      r.j[e] = 0;
      r.v[e] = T(0);
    }
  }
}

template <typename T, int TPR, int E>
__global__ void __launch_bounds__(512) k_trsv_cta(TriArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *ysm = reinterpret_cast<T *>(smem_raw);
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int slot = (threadIdx.x >> 5) * RPW + lane / TPR;  // row slot within a pass
  const int nslots = (blockDim.x >> 5) * RPW;
  RowRegs<T, E> cur, nxt;
  bool have = false, have_n = false;
  if (a.nlevels > 0) {
    const int p = a.lvl_ptr[0] + slot;
    have = p < a.lvl_ptr[1];
    if (have) load_row<T, TPR, E>(a, p, sub, cur);
  }
  for (int L = 0; L < a.nlevels; ++L) {
    const int p0 = a.lvl_ptr[L], p1 = a.lvl_ptr[L + 1];
    // prefetch the first pass of the next level
    if (L + 1 < a.nlevels) {
      const int pn = p1 + slot;
      have_n = pn < a.lvl_ptr[L + 2];
      if (have_n) load_row<T, TPR, E>(a, pn, sub, nxt);
    } else {
      have_n = false;
    }
    // first pass from registers
    {
      T acc = T(0);
      if (have) {
#pragma unroll
        for (int e = 0; e < E; ++e)
          if (cur.k0 + e * TPR < cur.k1) acc = fma(cur.v[e], ysm[cur.j[e]], acc);
        for (int k = cur.k0 + E * TPR; k < cur.k1; k += TPR) acc = fma(a.pval[k], ysm[a.pja[k]], acc);
      }
#pragma unroll
      for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, TPR);
      if (have && sub == 0) {
        const T t = Bits<T>::canon(cur.rhs - acc);
        ysm[cur.i] = t;
        tri_store(a, cur.o, t);
      }
    }
    // further passes of a wide level (not prefetched)
    for (int q0 = p0 + nslots; q0 < p1; q0 += nslots) {
      const int p = q0 + slot;
      T acc = T(0);
      RowRegs<T, 1> r;
      const bool ok = p < p1;
      if (ok) {
        load_row<T, TPR, 1>(a, p, sub, r);
        for (int k = r.k0; k < r.k1; k += TPR) acc = fma(a.pval[k], ysm[a.pja[k]], acc);
      }
#pragma unroll
      for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, TPR);
      if (ok && sub == 0) {
        const T t = Bits<T>::canon(r.rhs - acc);
        ysm[r.i] = t;
        tri_store(a, r.o, t);
      }
    }
    __syncthreads();
    cur = nxt;
    have = have_n;
  }
}

// ---------------------------------------------------------------------------
// Staged single-CTA solve (small levels).  The right-hand side is loaded once
// into the shared solution vector, which is then updated in place level by
// level; each level's rows and entries stream through a ring of D shared
// stages filled by cp.async D-1 levels ahead, so the only per-level costs
// are one barrier and the row arithmetic.  Results are written out
// (coalesced) at the end.
struct StageCfg {
  int D;       // ring depth
  int capR;    // rows per stage
  int capE;    // entries per stage
  int bytes;   // bytes per stage
  int off_y, off_desc, off_ring;  // byte offsets in dynamic shared memory
};

__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <typename T>
__device__ __forceinline__ void stage_issue(const TriArgs<T> &a, const StageCfg &c, unsigned char *ring,
                                            const int4 *desc, int l) {
  if (l >= a.nlevels) return;
  unsigned char *st = ring + (size_t)(l % c.D) * c.bytes;
  int *prow_s = reinterpret_cast<int *>(st);
  int *pirp_s = prow_s + c.capR;
  int *pja_s = pirp_s + c.capR + 1;
  T *pval_s = reinterpret_cast<T *>(st + (((size_t)(2 * c.capR + 1 + c.capE) * 4 + 15) & ~(size_t)15));
  const int4 d = desc[l];  // p0, p1, e0, e1
  const int nr = d.y - d.x, ne = d.w - d.z;
  if (nr > c.capR || ne > c.capE) return;  // oversized level: read from global at compute time
  for (int r = threadIdx.x; r < nr; r += blockDim.x) cp_async4(prow_s + r, a.prow + d.x + r);
  for (int r = threadIdx.x; r <= nr; r += blockDim.x) cp_async4(pirp_s + r, a.pirp + d.x + r);
  for (int k = threadIdx.x; k < ne; k += blockDim.x) {
    cp_async4(pja_s + k, a.pja + d.z + k);
    if (sizeof(T) == 8)
      cp_async8(pval_s + k, a.pval + d.z + k);
    else
      cp_async4(pval_s + k, a.pval + d.z + k);
  }
}

template <typename T, int TPR, int D>
__global__ void __launch_bounds__(512) k_trsv_stg(TriArgs<T> a, StageCfg c, const int4 *gdesc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *ysm = reinterpret_cast<T *>(smem_raw + c.off_y);
  int4 *desc = reinterpret_cast<int4 *>(smem_raw + c.off_desc);
  unsigned char *ring = smem_raw + c.off_ring;
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int slot = (threadIdx.x >> 5) * RPW + lane / TPR;
  const int nslots = (blockDim.x >> 5) * RPW;
  const T sent = Sentinel<T>::value();
  for (int l = threadIdx.x; l < a.nlevels; l += blockDim.x) desc[l] = gdesc[l];
  for (int i = threadIdx.x; i < a.n; i += blockDim.x) {
    const int o = a.rev ? (a.n - 1 - i) : i;
    T r = a.rhs_src[o];
    if (a.rhs_scale) r = r * a.rhs_scale[o];
    ysm[i] = r;
    if (a.other) a.other[o] = sent;
  }
  __syncthreads();
#pragma unroll
  for (int l = 0; l < D - 1; ++l) {
    stage_issue(a, c, ring, desc, l);
    cp_async_commit();
  }
  for (int L = 0; L < a.nlevels; ++L) {
    cp_async_wait<D - 2>();
    __syncthreads();  // level L staged; level L-1 finished (its stage is free)
    stage_issue(a, c, ring, desc, L + D - 1);
    cp_async_commit();
    const unsigned char *st = ring + (size_t)(L % D) * c.bytes;
    const int *prow_s = reinterpret_cast<const int *>(st);
    const int *pirp_s = prow_s + c.capR;
    const int *pja_s = pirp_s + c.capR + 1;
    const T *pval_s =
        reinterpret_cast<const T *>(st + (((size_t)(2 * c.capR + 1 + c.capE) * 4 + 15) & ~(size_t)15));
    const int4 d = desc[L];
    const int nr = d.y - d.x;
    const bool staged = nr <= c.capR && (d.w - d.z) <= c.capE;
    if (!staged) {
      prow_s = a.prow + d.x;
      pirp_s = a.pirp + d.x;
      pja_s = a.pja + d.z;
      pval_s = a.pval + d.z;
    }
    for (int r0 = 0; r0 < nr; r0 += nslots) {
      const int r = r0 + slot;
      T acc = T(0);
      int i = 0;
      if (r < nr) {
        i = prow_s[r];
        const int kb = pirp_s[r] - d.z, ke = pirp_s[r + 1] - d.z;
        for (int k = kb + sub; k < ke; k += TPR) acc = fma(pval_s[k], ysm[pja_s[k]], acc);
      }
#pragma unroll
      for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, TPR);
      if (r < nr && sub == 0) ysm[i] = Bits<T>::canon(ysm[i] - acc);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  for (int i = threadIdx.x; i < a.n; i += blockDim.x) {
    const int o = a.rev ? (a.n - 1 - i) : i;
    const T t = ysm[i];
    a.cur[o] = t;
    if (a.out) {
      T w = a.alpha * t;
      if (a.beta != T(0)) w = fma(a.beta, a.out[o], w);
      a.out[o] = w;
    }
  }
}

template <typename T, int TPR, int E>
__global__ void __launch_bounds__(256) k_trsv_sf(TriArgs<T> a) {
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int grp = lane / TPR;
  for (;;) {
    int b = 0;
    if (lane == 0) b = atomicAdd(&a.counters[0], 1);
    b = __shfl_sync(0xffffffffu, b, 0);
    if (b >= a.nblk) break;
    const int2 be = a.blk[b];
    const int p = be.x + grp;
    const bool ok = p < be.y;
    RowRegs<T, E> r;
    T acc = T(0);
    if (ok) {
      load_row<T, TPR, E>(a, p, sub, r);
      // all dependency loads in flight at once; re-poll only the missing ones
      typedef typename Bits<T>::U U;
      const U sent = (U)Sentinel<T>::bits;
      U raw[E];
      const T *src[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const bool has = r.k0 + e * TPR < r.k1;
        src[e] = a.cur + (a.rev ? (a.n - 1 - r.j[e]) : r.j[e]);
        raw[e] = has ? Bits<T>::load(src[e]) : (U)0;
      }
      const int lim = spin_limit();
      for (int it = 0;; ++it) {
        bool missing = false;
#pragma unroll
        for (int e = 0; e < E; ++e) missing |= (raw[e] == sent);
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
        for (int e = 0; e < E; ++e)
          if (raw[e] == sent) raw[e] = Bits<T>::load(src[e]);
      }
#pragma unroll
      for (int e = 0; e < E; ++e)
        if (r.k0 + e * TPR < r.k1) acc = fma(r.v[e], Bits<T>::from(raw[e] == sent ? (U)0 : raw[e]), acc);
      for (int k = r.k0 + E * TPR; k < r.k1; k += TPR) {
        const int j = a.pja[k];
        const int oj = a.rev ? (a.n - 1 - j) : j;
        acc = fma(a.pval[k], wait_value<T>(a.cur + oj, a.err), acc);
      }
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, TPR);
    if (ok && sub == 0) tri_store(a, r.o, Bits<T>::canon(r.rhs - acc));
  }
  // the last warp to leave resets the counters for the next launch
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

// ---------------------------------------------------------------------------
// One CG/FCG iteration after the preconditioner apply z = M^{-1} r (psb_dcg /
// psb_dfcg with istop = 2; FCG is Notay's flexible CG with truncation 1) in
// three kernels, every scalar kept on the device:
//   k_kry_beta   (z, q_prev) [FCG] or (r, z) [CG] -> beta
//   k_kry_spmv   d = z + beta d_prev (d = z on the first iteration), q = A d,
//                (d, q) and (d, r) -> alpha
//   k_kry_update x += alpha d, r -= alpha q, ||r||^2 -> ||r|| / ||b||, and the
//                stopping test, which also sets the CUDA-graph conditional
//                that repeats the iteration (a whole solve is one graph launch)
// Each kernel reduces deterministically: every block writes its partial sums,
// and the last block to finish (a ticket counter) adds them in block order.
// With an FP32 V-cycle the kernels read z as the V-cycle's FP32 output (ZT =
// float, widened exactly) and k_kry_update also writes the FP32 copy of r
// the next V-cycle starts from, so no separate precision casts run.
// The direction lives in two buffers used alternately (d0 on even, d1 on odd
// iterations), so q = A d reads the previous direction while the new one is
// written.
struct KState {
  double bn2;           // ||b||_2 (1 when b = 0)
  double tol;           // relative residual to reach
  double err;           // ||r||_2 / ||b||_2 after the last iteration
  double rr;            // ||r||_2^2
  double beta;          // direction coefficient of the current iteration
  double dq, dr;        // (d, A d), (d, r)
  double dq_prev;       // (d, A d) of the previous iteration (FCG)
  double rho, rho_old;  // (r, z) of this and the previous iteration (CG)
  double alpha;         // step of the current iteration
  int it;               // iterations done
  int itmax;
  int done;             // 1 once converged, at itmax or on a NaN residual
  int method;           // 0 CG, 1 FCG
  unsigned int ticket[4];
};

// True in exactly one block of the grid: the last one to arrive (after every
// block has written its partials).  The ticket is reset by that block.
__device__ __forceinline__ bool kry_last_block(unsigned int *ticket) {
  __shared__ int amlast;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) amlast = (atomicAdd(ticket, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (amlast) __threadfence();
  return amlast != 0;
}
// sum of partial[b*np + k] over the blocks, in a fixed order (one block)
__device__ __forceinline__ double kry_sum_partials(const double *partial, int nb, int np, int k,
                                                   double *sh) {
  double s = 0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += __ldcg(partial + (size_t)b * np + k);
  return block_sum(s, sh);
}

// Initial state after r = b - A x and the partials of (b, b), (r, r) from
// k_dots (one block).  ps: tol / itmax / method from the host.
struct KParams {
  double tol;
  int itmax;
  int method;
};
__global__ void __launch_bounds__(kRedThreads) k_kry_init(int nblocks, const double *partial,
                                                         const KParams *ps, KState *st,
                                                         cudaGraphConditionalHandle hc) {
  __shared__ double sh[32];
  const double bb = kry_sum_partials(partial, nblocks, 3, 0, sh);
  const double rr = kry_sum_partials(partial, nblocks, 3, 1, sh);
  if (threadIdx.x == 0) {
    double bn2 = sqrt(bb);
    if (bn2 == 0.0) bn2 = 1.0;
    const double err = sqrt(rr) / bn2;
    st->bn2 = bn2;
    st->tol = ps->tol;
    st->itmax = ps->itmax;
    st->method = ps->method;
    st->err = err;
    st->rr = rr;
    st->it = 0;
    st->beta = st->dq = st->dr = st->dq_prev = st->rho = st->rho_old = st->alpha = 0.0;
    for (int k = 0; k < 4; ++k) st->ticket[k] = 0u;
    const int done = (err > ps->tol && ps->itmax > 0) ? 0 : 1;
    st->done = done;
    if (hc) cudaGraphSetConditional(hc, done ? 0u : 1u);
  }
}

template <typename ZT>
__global__ void __launch_bounds__(kRedThreads) k_kry_beta(int n, const ZT *__restrict__ z,
                                                         const double *__restrict__ q,
                                                         const double *__restrict__ r, KState *st,
                                                         double *partial) {
  pdl_enter();
  __shared__ double sh[32];
  if (st->done) return;
  const int it = st->it, method = st->method;
  double s = 0;
  if (method == 1) {
    if (it > 0)
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        s = fma((double)z[i], q[i], s);
  } else {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
      s = fma(r[i], (double)z[i], s);
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (kry_last_block(&st->ticket[0])) {
    const double t = kry_sum_partials(partial, gridDim.x, 1, 0, sh);
    if (threadIdx.x == 0) {
      if (method == 1) {
        st->beta = it > 0 ? -(t / st->dq_prev) : 0.0;
      } else {
        st->rho_old = st->rho;
        st->rho = t;
        st->beta = it > 0 ? t / st->rho_old : 0.0;
      }
      st->ticket[0] = 0u;
    }
  }
}

// q = A d with d = z + beta*d_prev formed on the fly for every entry (the
// same fma as the stored d, so both agree bit for bit); TPR lanes per row as
// in k_spmv.  partial[2*b + {0,1}] = block sums of d_i q_i and d_i r_i.
template <int TPR, typename CI, typename ZT>
__global__ void __launch_bounds__(256) k_kry_spmv(int nr, const int *__restrict__ irp,
                                                  const CI *__restrict__ ja,
                                                  const double *__restrict__ val,
                                                  const ZT *__restrict__ z, double *d0, double *d1,
                                                  double *__restrict__ q, const double *__restrict__ r,
                                                  KState *st, double *partial) {
  pdl_enter();
  __shared__ double sh[32];
  if (st->done) return;
  constexpr int RPW = 32 / TPR;
  const int it = st->it;
  const bool first = it == 0;
  const double beta = st->beta;
  const double *dold = (it & 1) ? d0 : d1;
  double *dnew = (it & 1) ? d1 : d0;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int grp = lane / TPR;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double sdq = 0, sdr = 0;
  for (int r0 = warp * RPW; r0 < nr; r0 += nwarps * RPW) {
    const int row = r0 + grp;
    double s = 0;
    if (row < nr) {
      const int k0 = irp[row] + sub, e = irp[row + 1];
      if (first)
        s = csr_lane_sum<double, TPR>(k0, e, row, ja, val, [&](int j) { return (double)__ldg(z + j); });
      else
        s = csr_lane_sum<double, TPR>(k0, e, row, ja, val, [&](int j) { return fma(beta, dold[j], (double)__ldg(z + j)); });
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    if (row < nr && sub == 0) {
      const double di = first ? (double)z[row] : fma(beta, dold[row], (double)z[row]);
      dnew[row] = di;
      q[row] = s;
      sdq = fma(di, s, sdq);
      sdr = fma(di, r[row], sdr);
    }
  }
  sdq = block_sum(sdq, sh);
  sdr = block_sum(sdr, sh);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sdq;
    partial[2 * blockIdx.x + 1] = sdr;
  }
  if (kry_last_block(&st->ticket[1])) {
    const double dq = kry_sum_partials(partial, gridDim.x, 2, 0, sh);
    const double dr = kry_sum_partials(partial, gridDim.x, 2, 1, sh);
    if (threadIdx.x == 0) {
      st->dq = dq;
      st->dr = dr;
      st->alpha = (st->method == 1) ? dr / dq : st->rho / dq;
      st->ticket[1] = 0u;
    }
  }
}

// k_kry_spmv on the SELL copy of A (one thread per row)
template <typename CI, typename ZT>
__global__ void __launch_bounds__(256) k_kry_spmv_sell(int nr, const int *__restrict__ soff,
                                                       const CI *__restrict__ sj, const double *__restrict__ sv,
                                                       const ZT *__restrict__ z, double *d0, double *d1,
                                                       double *__restrict__ q, const double *__restrict__ r,
                                                       KState *st, double *partial) {
  pdl_enter();
  __shared__ double sh[32];
  if (st->done) return;
  const int it = st->it;
  const bool first = it == 0;
  const double beta = st->beta;
  const double *dold = (it & 1) ? d0 : d1;
  double *dnew = (it & 1) ? d1 : d0;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int ns = (nr + 31) >> 5;
  double sdq = 0, sdr = 0;
  for (int sl = warp; sl < ns; sl += nwarps) {
    const int row = (sl << 5) + lane;
    double acc[1];
    if (first)
      sell_rows<double, CI, 1>(soff, sj, sv, sl, ns, lane, [&](int j) { return (double)__ldg(z + j); }, acc);
    else
      sell_rows<double, CI, 1>(soff, sj, sv, sl, ns, lane, [&](int j) { return fma(beta, dold[j], (double)__ldg(z + j)); },
                               acc);
    const double s = acc[0];
    if (row < nr) {
      const double di = first ? (double)z[row] : fma(beta, dold[row], (double)z[row]);
      dnew[row] = di;
      q[row] = s;
      sdq = fma(di, s, sdq);
      sdr = fma(di, r[row], sdr);
    }
  }
  sdq = block_sum(sdq, sh);
  sdr = block_sum(sdr, sh);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sdq;
    partial[2 * blockIdx.x + 1] = sdr;
  }
  if (kry_last_block(&st->ticket[1])) {
    const double dq = kry_sum_partials(partial, gridDim.x, 2, 0, sh);
    const double dr = kry_sum_partials(partial, gridDim.x, 2, 1, sh);
    if (threadIdx.x == 0) {
      st->dq = dq;
      st->dr = dr;
      st->alpha = (st->method == 1) ? dr / dq : st->rho / dq;
      st->ticket[1] = 0u;
    }
  }
}

// k_kry_spmv on the HDIA copy of A (one thread per row, a warp per slice:
// the rows and the reduction order of k_kry_spmv_sell; two diagonals' loads
// per pass keep it at 40 registers, six 256-thread blocks per SM)
template <typename ZT>
__global__ void __launch_bounds__(256, 6) k_kry_spmv_hdia(int nr, const int *__restrict__ dptr,
                                                       const int *__restrict__ doff, const double *__restrict__ hv,
                                                       const ZT *__restrict__ z, double *d0, double *d1,
                                                       double *__restrict__ q, const double *__restrict__ r,
                                                       KState *st, double *partial) {
  pdl_enter();
  __shared__ double sh[32];
  if (st->done) return;
  const int it = st->it;
  const bool first = it == 0;
  const double beta = st->beta;
  const double *dold = (it & 1) ? d0 : d1;
  double *dnew = (it & 1) ? d1 : d0;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int ns = (nr + 31) >> 5;
  double sdq = 0, sdr = 0;
  for (int sl = warp; sl < ns; sl += nwarps) {
    const int row = (sl << 5) + lane;
    const double s =
        first ? hdia_row<double, 2>(dptr, doff, hv, sl, row, nr, lane, [&](int j) { return (double)__ldg(z + j); })
              : hdia_row<double, 2>(dptr, doff, hv, sl, row, nr, lane,
                                 [&](int j) { return fma(beta, dold[j], (double)__ldg(z + j)); });
    if (row < nr) {
      const double di = first ? (double)z[row] : fma(beta, dold[row], (double)z[row]);
      dnew[row] = di;
      q[row] = s;
      sdq = fma(di, s, sdq);
      sdr = fma(di, r[row], sdr);
    }
  }
  sdq = block_sum(sdq, sh);
  sdr = block_sum(sdr, sh);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sdq;
    partial[2 * blockIdx.x + 1] = sdr;
  }
  if (kry_last_block(&st->ticket[1])) {
    const double dq = kry_sum_partials(partial, gridDim.x, 2, 0, sh);
    const double dr = kry_sum_partials(partial, gridDim.x, 2, 1, sh);
    if (threadIdx.x == 0) {
      st->dq = dq;
      st->dr = dr;
      st->alpha = (st->method == 1) ? dr / dq : st->rho / dq;
      st->ticket[1] = 0u;
    }
  }
}

__global__ void __launch_bounds__(kRedThreads) k_kry_update(int n, const double *d0, const double *d1,
                                                           const double *__restrict__ q, double *x,
                                                           double *r, KState *st, double *partial,
                                                           cudaGraphConditionalHandle hc, float *r32) {
  pdl_enter();
  __shared__ double sh[32];
  if (st->done) return;
  const int it = st->it;
  const double *__restrict__ d = (it & 1) ? d1 : d0;
  const double alpha = st->alpha;
  double s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = fma(alpha, d[i], x[i]);
    const double ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    if (r32) r32[i] = (float)ri;  // the FP32 V-cycle's input, rounded as k_cast does
    s = fma(ri, ri, s);
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (kry_last_block(&st->ticket[2])) {
    const double rr = kry_sum_partials(partial, gridDim.x, 1, 0, sh);
    if (threadIdx.x == 0) {
      const double err = sqrt(rr < 0.0 ? 0.0 : rr) / st->bn2;  // NaN stays NaN
      st->rr = rr;
      st->err = err;
      st->it = it + 1;
      st->dq_prev = st->dq;
      const int done = (err > st->tol && it + 1 < st->itmax) ? 0 : 1;
      st->done = done;
      st->ticket[2] = 0u;
      if (hc) cudaGraphSetConditional(hc, done ? 0u : 1u);
    }
  }
}

// Independent systems solved in one graph: a WHILE loop whose body opens one
// IF branch (V-cycle + iteration) per unfinished system.  k_kry_gate sets
// every branch's conditional from its system's state at the top of the body;
// k_kry_any keeps the loop going while any system is unfinished.
__global__ void k_kry_gate(KState *const *st, const cudaGraphConditionalHandle *hc, int nsys) {
  for (int i = threadIdx.x; i < nsys; i += blockDim.x) cudaGraphSetConditional(hc[i], st[i]->done ? 0u : 1u);
}
__global__ void k_kry_any(KState *const *st, int nsys, cudaGraphConditionalHandle hw) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < nsys; i += blockDim.x)
    if (!st[i]->done) atomicOr(&any, 1);
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(hw, any ? 1u : 0u);
}

}  // namespace mldg
