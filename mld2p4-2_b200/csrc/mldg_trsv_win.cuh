// mldg_trsv_win.cuh -- windowed, cluster-cooperative sparse unit-triangular solve.
//
// Rows are processed in dependency-level order ("positions").  A cluster of C
// CTAs walks the levels in lock step: in every step each CTA solves its slice
// of the step's rows, then the cluster synchronises (barrier.cluster, or
// __syncthreads when C == 1).  The solution values of the last W positions
// live in a ring ("window") spread over the C CTAs' shared memory; every
// dependency of every row lies in the window (checked on the host), so a
// dependency read is a shared or distributed-shared load.  Each CTA streams its
// slice of rows, entries and right-hand side through a ring of D shared stages
// filled by TMA bulk copies (one thread issues, an mbarrier per stage signals
// completion) D-1 steps ahead of use.
//
// All vectors of the step are in position order, except the outputs: the
// result t_p of row p is written to
//   out[orig(p)] = alpha*t_p                         (when out != null)
//   tpos[p] = t_p                                    (when tpos != null)
//   next[nextpos[p]] = nextscale[p] * t_p            (when next != null)
// An update out = alpha*t + beta*out (beta != 0) goes through tpos and
// k_combine, so that no global read sits on the solve's critical path.
// where `next` is the right-hand side of the following solve in its own
// position order (the L solve feeds the U solve this way without a gather).
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mldg {

struct WinDesc {  // one CTA's slice of one step
  int r0, r1;     // positions
  int e0, e1;     // entries
};

template <typename T>
struct WinArgs {
  int n;
  int nsteps;
  int W;            // window size (power of two), slots per CTA = W / C
  int wshift;       // log2(W / C)
  int capR, capE;   // per-stage capacity (rows, entries)
  int D;            // stage count (== template D)
  int stage_bytes;
  int off_win, off_desc, off_bar, off_ring;  // dynamic shared memory layout
  const WinDesc *desc;  // [nsteps][C]
  const int *orig;      // orig row of each position            (out)
  const int *pirp;      // entry offsets per position (n + 1)
  const int *pja;       // dependency positions
  const T *pval;
  const T *rhs;         // right-hand side in position order
  const int *nextpos;   // position in the next solve (next != null)
  const T *nextscale;
  T *next;
  T *out;   // out[orig] = alpha * t (scattered; beta == 0 only)
  T *tpos;  // t in position order (for a separate beta != 0 combine)
  T alpha, beta;
  int *err;
  unsigned long long *trace;  // optional: cycles in wait / compute / barrier / issue (CTA 0, thread 0)
};

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile(
      "{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// bounded wait on an mbarrier phase; returns false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// explicit shared-space accesses through 32-bit shared addresses
__device__ __forceinline__ int lds_i32(unsigned a) {
  int v;
  asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ double lds_val(unsigned a, double) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ float lds_val(unsigned a, float) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ double ldc_val(unsigned a, double) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ float ldc_val(unsigned a, float) {
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ void stc_val(unsigned a, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void stc_val(unsigned a, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void sts_val(unsigned a, double v) {
  asm volatile("st.shared.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void sts_val(unsigned a, float v) {
  asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ unsigned mapa_u32(unsigned a, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Byte layout of one stage (all offsets 16-byte aligned):
//   orig[capR+8] int | pirp[capR+9] int | pja[capE+8] int | pval[capE+8] T |
//   rhs[capR+8] T | nextpos[capR+8] int | nextscale[capR+8] T
// Slices are copied from 16-byte-aligned global addresses, so each array in
// the stage starts at the element (start & ~(16/size-1)) and an in-stage
// offset `sk` locates the first element of the slice.
struct StageLayout {
  int o_orig, o_pirp, o_pja, o_pval, o_rhs, o_npos, o_nsc, bytes;
};

__host__ __device__ inline int al16(int x) { return (x + 15) & ~15; }

template <typename T>
__host__ __device__ inline StageLayout stage_layout(int capR, int capE) {
  StageLayout s;
  int o = 0;
  s.o_orig = o;
  o = al16(o + 4 * (capR + 8));
  s.o_pirp = o;
  o = al16(o + 4 * (capR + 9));
  s.o_pja = o;
  o = al16(o + 4 * (capE + 8));
  s.o_pval = o;
  o = al16(o + (int)sizeof(T) * (capE + 8));
  s.o_rhs = o;
  o = al16(o + (int)sizeof(T) * (capR + 8));
  s.o_npos = o;
  o = al16(o + 4 * (capR + 8));
  s.o_nsc = o;
  o = al16(o + (int)sizeof(T) * (capR + 8));
  s.bytes = o;
  return s;
}

// Aligned copy of elements [a, b) of a global array with element size es:
// the copy runs from a rounded down to b rounded up on 16-byte boundaries
// (global arrays carry 16 bytes of tail padding); `off` is the element offset
// of `a` inside the copy.
struct Slice {
  const unsigned char *src;
  unsigned bytes;
};
__device__ __forceinline__ Slice plan_slice(const void *base, int a, int b, int es, int *off) {
  const int per = 16 / es;
  const int a0 = a & ~(per - 1);
  const int b0 = (b + per - 1) & ~(per - 1);
  *off = a - a0;
  Slice s;
  s.src = (const unsigned char *)base + (size_t)a0 * es;
  s.bytes = (b > a) ? (unsigned)((b0 - a0) * es) : 0u;
  return s;
}

template <typename T, int TPR, int C, int D>
__global__ void __launch_bounds__(512, 1) k_trsv_win(WinArgs<T> a) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(128) unsigned char sm[];
  T *win = reinterpret_cast<T *>(sm + a.off_win);
  WinDesc *desc = reinterpret_cast<WinDesc *>(sm + a.off_desc);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + a.off_bar);
  unsigned char *ring = sm + a.off_ring;
  unsigned long long k_t0 = 0, k_ns0 = 0;
  if (a.trace && threadIdx.x == 0 && blockIdx.x == 0) {
    k_t0 = clock64();
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(k_ns0));
  }
  const StageLayout L = stage_layout<T>(a.capR, a.capE);
  const unsigned win_s = smem_u32(win);
  const unsigned ring_s = smem_u32(ring);
  unsigned rank = 0;
  if (C > 1) rank = cg::this_cluster().block_rank();
  const int wmask = (1 << a.wshift) - 1;
  const int tid = threadIdx.x;
  for (int s = tid; s < a.nsteps; s += blockDim.x) desc[s] = a.desc[(size_t)s * C + rank];
  if (tid == 0) {
    for (int d = 0; d < D; ++d) mbar_init(&bar[d], 7);  // one arrival per slice lane
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // offsets (in elements) of each slice inside its stage, per stage
  __shared__ int s_off[8][7];
  // The last warp is the producer: lanes 0..6 each stage one slice of a step
  // (arrive.expect_tx + TMA bulk copy); the other warps compute rows.
  const int warp = tid >> 5;
  const bool producer = warp == (int)(blockDim.x >> 5) - 1;
  auto issue = [&](int step) {
    const int i = tid & 31;
    if (step >= a.nsteps || i >= 7) return;
    const int d = step % D;
    unsigned char *st = ring + (size_t)d * L.bytes;
    const WinDesc w = desc[step];
    const int nr = w.r1 - w.r0;
    Slice sl{nullptr, 0u};
    int off = 0, dst = 0;
    switch (i) {
      case 0: sl = plan_slice(a.orig, w.r0, w.r1, 4, &off); dst = L.o_orig; break;
      case 1: sl = plan_slice(a.pirp, w.r0, w.r1 + (nr > 0 ? 1 : 0), 4, &off); dst = L.o_pirp; break;
      case 2: sl = plan_slice(a.pja, w.e0, w.e1, 4, &off); dst = L.o_pja; break;
      case 3: sl = plan_slice(a.pval, w.e0, w.e1, (int)sizeof(T), &off); dst = L.o_pval; break;
      case 4: sl = plan_slice(a.rhs, w.r0, w.r1, (int)sizeof(T), &off); dst = L.o_rhs; break;
      case 5:
        if (a.next) sl = plan_slice(a.nextpos, w.r0, w.r1, 4, &off);
        dst = L.o_npos;
        break;
      default:
        if (a.next) sl = plan_slice(a.nextscale, w.r0, w.r1, (int)sizeof(T), &off);
        dst = L.o_nsc;
        break;
    }
    s_off[d][i] = off;
    fence_proxy_async();
    mbar_expect_tx(&bar[d], sl.bytes);  // this lane's arrival (+ its bytes)
    if (sl.bytes) tma_bulk_g2s(st + dst, sl.src, sl.bytes, &bar[d]);
  };
  // The producer alone waits for each stage's TMA completion (mbarrier,
  // acquire) before the step barrier; the barrier then publishes the staged
  // data to the consumer warps, which never poll the mbarrier themselves.
  __shared__ int s_fail;  // set by the producer when a stage never completed
  if (tid == 0) s_fail = 0;
  __syncthreads();
  if (producer) {
    for (int s = 0; s < D - 1; ++s) issue(s);
    if (a.nsteps > 0 && !mbar_wait(&bar[0], 0u) && (tid & 31) == 0) {
      s_fail = 1;
      atomicExch(a.err, 4021);
    }
  }
  __syncthreads();
  constexpr int RPW = 32 / TPR;
  const int lane = tid & 31;
  const int sub = lane % TPR;
  const int slot = warp * RPW + lane / TPR;
  const int nslots = ((int)(blockDim.x >> 5) - 1) * RPW;
  const bool tr = a.trace && rank == 0 && tid == 0;
  unsigned long long c_wait = 0, c_comp = 0, c_bar = 0, t0 = 0, t1 = 0;
  const unsigned long long loop_t0 = tr ? clock64() : 0ull;
  for (int step = 0; step < a.nsteps; ++step) {
    const int d = step % D;
    if (producer) {
      issue(step + D - 1);  // stage (step-1) % D: its readers passed the last barrier
      const int nx = step + 1;
      if (nx < a.nsteps && !mbar_wait(&bar[nx % D], (unsigned)((nx / D) & 1)) && (tid & 31) == 0) {
        s_fail = 1;
        atomicExch(a.err, 4021);
      }
    } else {
      if (tr) t0 = clock64();
      if (tr) {
        t1 = clock64();
        c_wait += t1 - t0;
        t0 = t1;
      }
      // 32-bit shared addresses of this stage's arrays
      const unsigned st = ring_s + (unsigned)(d * L.bytes);
      const int *o = s_off[d];
      const unsigned a_orig = st + L.o_orig + 4u * o[0];
      const unsigned a_pirp = st + L.o_pirp + 4u * o[1];
      const unsigned a_pja = st + L.o_pja + 4u * o[2];
      const unsigned a_pval = st + L.o_pval + (unsigned)sizeof(T) * o[3];
      const unsigned a_rhs = st + L.o_rhs + (unsigned)sizeof(T) * o[4];
      const unsigned a_npos = st + L.o_npos + 4u * o[5];
      const unsigned a_nsc = st + L.o_nsc + (unsigned)sizeof(T) * o[6];
      const WinDesc w = desc[step];
      const int nr = w.r1 - w.r0;
      if (!s_fail) {
        for (int r0 = 0; r0 < nr; r0 += nslots) {
          const int r = r0 + slot;
          T acc = T(0);
          if (r < nr) {
            const int kb = lds_i32(a_pirp + 4u * r) - w.e0 + sub, ke = lds_i32(a_pirp + 4u * (r + 1)) - w.e0;
            // first 4 entries of this lane unrolled: every load issued before the FMAs
            constexpr int E = 4;
            unsigned qa[E];
            T pv[E], yv[E];
            bool valid[E];
#pragma unroll
            for (int e = 0; e < E; ++e) {
              const int k = kb + e * TPR;
              valid[e] = k < ke;
              qa[e] = valid[e] ? (unsigned)lds_i32(a_pja + 4u * k) & (unsigned)(a.W - 1) : 0u;
              pv[e] = valid[e] ? lds_val(a_pval + (unsigned)sizeof(T) * k, T(0)) : T(0);
            }
#pragma unroll
            for (int e = 0; e < E; ++e) {
              yv[e] = T(0);
              if (valid[e]) {
                if (C > 1)
                  yv[e] = ldc_val(
                      mapa_u32(win_s + (unsigned)sizeof(T) * (qa[e] & (unsigned)wmask), qa[e] >> a.wshift), T(0));
                else
                  yv[e] = lds_val(win_s + (unsigned)sizeof(T) * qa[e], T(0));
              }
            }
#pragma unroll
            for (int e = 0; e < E; ++e) acc = fma(pv[e], yv[e], acc);
            for (int k = kb + E * TPR; k < ke; k += TPR) {
              const unsigned q = (unsigned)lds_i32(a_pja + 4u * k) & (unsigned)(a.W - 1);
              const T v = lds_val(a_pval + (unsigned)sizeof(T) * k, T(0));
              T y;
              if (C > 1)
                y = ldc_val(mapa_u32(win_s + (unsigned)sizeof(T) * (q & (unsigned)wmask), q >> a.wshift), T(0));
              else
                y = lds_val(win_s + (unsigned)sizeof(T) * q, T(0));
              acc = fma(v, y, acc);
            }
          }
#pragma unroll
          for (int off = TPR / 2; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off, TPR);
          if (r < nr && sub == 0) {
            const int p = w.r0 + r;
            const T t = lds_val(a_rhs + (unsigned)sizeof(T) * r, T(0)) - acc;
            const unsigned q = (unsigned)p & (unsigned)(a.W - 1);
            if (C > 1)
              stc_val(mapa_u32(win_s + (unsigned)sizeof(T) * (q & (unsigned)wmask), q >> a.wshift), t);
            else
              sts_val(win_s + (unsigned)sizeof(T) * q, t);
            if (a.out) a.out[lds_i32(a_orig + 4u * r)] = a.alpha * t;
            if (a.tpos) a.tpos[p] = t;
            if (a.next) a.next[lds_i32(a_npos + 4u * r)] = lds_val(a_nsc + (unsigned)sizeof(T) * r, T(0)) * t;
          }
        }
      }
      if (tr) {
        t1 = clock64();
        c_comp += t1 - t0;
        t0 = t1;
      }
    }
    if (C > 1)
      asm volatile("barrier.cluster.arrive.release.aligned;\n barrier.cluster.wait.acquire.aligned;" ::: "memory");
    else
      __syncthreads();
    if (tr) c_bar += clock64() - t0;
  }
  if (tr) {
    unsigned long long ns1;
    a.trace[7] += clock64() - loop_t0;
    a.trace[8] += loop_t0 - k_t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(ns1));
    a.trace[0] += c_wait;
    a.trace[1] += c_comp;
    a.trace[2] += c_bar;
    a.trace[4] += (unsigned long long)a.nsteps;
    a.trace[5] += clock64() - k_t0;
    a.trace[6] += ns1 - k_ns0;
  }
  // keep this CTA's window alive until every peer has finished reading it
  if (C > 1)
    asm volatile("barrier.cluster.arrive.release.aligned;\n barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// out[orig[p]] = alpha * tpos[p] + beta * out[orig[p]]
template <typename T>
__global__ void k_combine(int n, const int *__restrict__ orig, const T *__restrict__ tpos, T alpha,
                          T beta, T *out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int o = orig[p];
    out[o] = fma(beta, out[o], alpha * tpos[p]);
  }
}

// rhs_p[p] = src[orig[p]] (* scale[orig[p]])
template <typename T>
__global__ void k_gather(int n, const int *__restrict__ orig, const T *__restrict__ src,
                         const T *__restrict__ scale, T *__restrict__ dst) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int o = orig[p];
    T v = src[o];
    if (scale) v = v * scale[o];
    dst[p] = v;
  }
}

}  // namespace mldg
