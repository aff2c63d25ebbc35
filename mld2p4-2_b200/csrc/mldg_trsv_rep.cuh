// mldg_trsv_rep.cuh -- level-synchronous cluster solve with a replicated window.
//
// A sparse unit-triangular solve t = rhs - T_strict t, rows in dependency-level
// order ("positions"), walked in steps (a step is a level or a part of one) by
// a cluster of C CTAs.  In each step every CTA solves its slice of the step's
// rows, one row per group of TPR lanes.  Every CTA keeps the last R solution
// values in its own shared memory (a ring indexed by position mod R): each
// value is sent to all C rings by st.async, which counts its bytes on the
// destination CTA's mbarrier for that step, so a dependency read is a local
// shared-memory load once the step's barrier phase has completed.  There is
// no per-step CTA or cluster barrier: a thread waits only for the values of
// the previous step.
//
// Only the dependencies of a row on the immediately preceding step sit on the
// critical path (from the arrival of that step's values to the send of the
// row's own).  The steps are dealt round-robin to kRepG groups of warps, so a
// group prepares its next step (older ring dependencies, far values) while
// the other groups solve theirs.  Dependencies older than the ring are read
// from a position-ordered copy of the solution in global memory that holds a
// signalling-NaN sentinel until the value is written (a reader re-reads,
// bounded, while it sees the sentinel) and is reset to the sentinel one step
// after its last read, so every launch starts from a clean copy.
//
// A value overwrites the ring slot of the position R earlier; the host checks
// that every ring dependency q of a row in step u has q >= end(u) - R, and a
// CTA cannot send the values of step w+2 before every row of step w+1 (whose
// reads are done before its own send) has been sent, so no slot is
// overwritten while a reader still needs it.
//
// The per-CTA, per-step plan (row descriptors, entry slots and values, the
// far entries of two steps later) is one 16-byte-aligned block in global
// memory.  Each block and the step's right-hand-side slice are copied into a
// ring of D shared-memory stages by two TMA bulk copies (one thread; a "full"
// mbarrier per stage counts the bytes, an "empty" one counts the warps done
// with it) D-1 steps ahead of use, after an L2 bulk prefetch RP steps ahead.
// Every wait is bounded (error 4021); a thread whose wait gave up stops
// reading and writing and only keeps the cluster barriers.
//
// Outputs, as in the windowed solve: out[orig(p)] = alpha*t_p (beta == 0),
// tpos[p] = t_p (an update with beta != 0 goes through k_combine), and
// next[npos(p)] = nsc(p)*t_p (the right-hand side of the following solve of a
// pair, in its own position order).
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mldg_trsv_win.cuh"  // mbarrier and bulk-copy helpers

namespace mldg {

// Byte layout of the plan block of one CTA for step t (arrays 16-byte aligned):
//   int4 hdr  {nr, ne, nf2, r0}
//   int4 cp   copy of the descriptor of step t + D - 1 (checked by the host emulation; the
//   int4 pf   producer warp reads the descriptor table) and of step t + RP
//   int4 h3   {nrG, nrst, 0, 0}: rows of this CTA in step t + kRepG, far-copy positions to reset
//   int4 row[nr]  {ebeg, cnt, 0, orig}      cnt = n1 | nm << 8 | no << 16 | feeds_far << 24
//   int  npos[nr], T nsc[nr]                (linked solves only)
//   u16  slot[ne], T val[ne]                (per row: previous step, 2..kRepG steps back, older)
//   int2 fr[nrG]  {fbeg, nf}                far entries of the rows of step t + kRepG
//   int  fq[nf2], T fv[nf2]                 (global positions, values)
//   int  rst[nrst]                          far-copy positions whose last reader is in step t - 1
struct RepLayout {
  int o_row, o_npos, o_nsc, o_slot, o_val, o_fr, o_fq, o_fv, o_rst, bytes;
};

__host__ __device__ inline int rep_al16(int x) { return (x + 15) & ~15; }

template <typename T>
__host__ __device__ inline RepLayout rep_layout(int nr, int ne, int nr2, int nf2, int nrst, bool linked) {
  RepLayout L;
  int o = 64;
  L.o_row = o;
  o += 16 * nr;
  L.o_npos = o;
  if (linked) o = rep_al16(o + 4 * nr);
  L.o_nsc = o;
  if (linked) o = rep_al16(o + (int)sizeof(T) * nr);
  L.o_slot = o;
  o = rep_al16(o + 2 * ne);
  L.o_val = o;
  o = rep_al16(o + (int)sizeof(T) * ne);
  L.o_fr = o;
  o = rep_al16(o + 8 * nr2);
  L.o_fq = o;
  o = rep_al16(o + 4 * nf2);
  L.o_fv = o;
  o = rep_al16(o + (int)sizeof(T) * nf2);
  L.o_rst = o;
  o = rep_al16(o + 4 * nrst);
  L.bytes = o;
  return L;
}

template <typename T>
struct RepArgs {
  int nsteps;
  int rmask;        // ring size R - 1 (R a power of two)
  int capB;         // stage bytes reserved for the block; the rhs slice follows
  int stage_bytes;  // capB + rhs capacity
  int ring_bytes;   // R * sizeof(T), 128-byte multiple
  int linked;
  const int4 *desc;    // [C][nsteps] {block offset in 16-byte units, block size in 16-byte units, r0, nr}
  const uint4 *blocks;
  const T *rhs;        // position order, 16-byte aligned, padded by 16 bytes
  T *next;
  T *out;
  T *tpos;
  T *xp;               // position-ordered copy for far readers: the sentinel until written, reset after its last read
  const int *tail_ptr;  // [C + 1] far-copy positions reset after the last step, per CTA
  const int *tail;
  T alpha;
  int off_bar;      // byte offset of the mbarriers in shared memory: full[D], empty[D], values[MV]
  const int *vbytes;  // [nsteps] bytes of the values of each step (every row of the cluster)
  int *err;
  unsigned long long *trace;  // optional [20]: per-phase cycles, steps, kernel cycles and ns of the first thread of groups 0 and 1 in CTA 0
};

__device__ __forceinline__ unsigned rep_smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void rep_prefetch_l2(const void *p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ unsigned rep_mapa(unsigned a, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ double rep_lds(unsigned a, double) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ float rep_lds(unsigned a, float) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}

// stage copies, value barriers, lookaheads, groups, per-lane register capacities
constexpr int kRepD = 8;        // plan stages in shared memory
constexpr int kRepMV = 8;       // value barriers (steps in flight)
constexpr int kRepPF = 16;      // L2 prefetch distance (steps)
constexpr int kRepAR = 4;       // value barriers armed this many steps ahead
constexpr int kRepG = 3;        // step groups: group g takes the steps s = g (mod kRepG)
constexpr int kRepGW = 5;       // warps per group
constexpr int kRepN1 = 2;       // previous-step entries per lane
constexpr int kRepNF = 4;       // far entries per lane
constexpr int kRepThreads = 512;
constexpr int kRepWarps = kRepThreads / 32;  // kRepG * kRepGW compute warps + one producer warp
// far dependencies at least this many steps back (checked on the host): the
// value has been written well before its load is issued, so a reader rarely
// sees the sentinel
constexpr int kRepFarMin = 2 * kRepG + 2;
static_assert(kRepG * kRepGW + 1 == kRepWarps, "thread layout");

template <int TPR>
constexpr int rep_rows() {  // row slots of one group
  return kRepGW * 32 / TPR;
}

__device__ __forceinline__ void rep_st_async(unsigned a, double v, unsigned mbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];" ::"r"(a), "d"(v),
               "r"(mbar)
               : "memory");
}
__device__ __forceinline__ void rep_st_async(unsigned a, float v, unsigned mbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f32 [%0], %1, [%2];" ::"r"(a), "f"(v),
               "r"(mbar)
               : "memory");
}
// bounded wait on an mbarrier phase with cluster-scope acquire (the bytes of
// st.async stores from other CTAs); false on timeout
__device__ __forceinline__ bool rep_wait_cluster(uint64_t *bar, unsigned parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(rep_smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void rep_arrive_cta(uint64_t *bar) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(rep_smem_u32(bar))
               : "memory");
}

template <typename T, int TPR, int C>
__global__ void __launch_bounds__(kRepThreads, 1) k_trsv_rep(RepArgs<T> a) {
  constexpr int D = kRepD, MV = kRepMV, G = kRepG, GT = kRepGW * 32;
  constexpr int PER = 16 / (int)sizeof(T);
  extern __shared__ __align__(128) unsigned char sm[];
  T *ring = reinterpret_cast<T *>(sm);
  unsigned char *stg = sm + a.ring_bytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + a.off_bar);  // [D] stage bytes landed
  uint64_t *empty = full + D;                                       // [D] stage released by its group
  uint64_t *vbar = empty + D;                                       // [MV] values of a step landed
  const int tid = threadIdx.x, lane = tid & 31;
  const bool producer = (tid >> 5) == kRepWarps - 1;
  unsigned rank = 0;
  if (C > 1) rank = cooperative_groups::this_cluster().block_rank();
  const int4 *desc = a.desc + (size_t)rank * a.nsteps;
  const int grp = producer ? 0 : tid / GT;
  const int slot = (tid - grp * GT) / TPR, sub = (tid - grp * GT) % TPR;
  const unsigned ring_s = rep_smem_u32(ring);
  const unsigned vbar_s = rep_smem_u32(vbar);
  const int4 zero4 = make_int4(0, 0, 0, 0);
  auto load_desc = [&](int t) { return t < a.nsteps ? desc[t] : zero4; };

  // After a wait that gave up (error 4021) a thread reads and writes nothing
  // more; it only keeps the cluster barriers, so the kernel still ends.
  bool live = true;
  auto give_up = [&]() {
    atomicExch(a.err, 4021);
    live = false;
  };
  auto cluster_sync = [&]() {
    __syncwarp();
    asm volatile("barrier.cluster.arrive.release.aligned;\n barrier.cluster.wait.acquire.aligned;" ::: "memory");
  };

  if (producer && lane == 0) {
    for (int d = 0; d < D; ++d) {
      mbar_init(&full[d], 1);
      mbar_init(&empty[d], kRepGW);
    }
    for (int m = 0; m < MV; ++m) mbar_init(&vbar[m], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // every CTA's barriers exist before any st.async reaches them
  cluster_sync();

  if (producer) {
    // ---- producer warp: lane 0 copies the plan and arms the value barriers ----
    // Descriptors and value bytes come 32 steps at a time, one step per lane,
    // loaded a chunk ahead; lane 0 takes each step's entries by shuffle.
    int last_issued = -1;  // lane 0: the last step whose stage copy was issued
    auto issue = [&](int t, int4 d) {
      if (lane != 0 || !live || t >= a.nsteps) return;
      if (t >= D && !mbar_wait(&empty[t % D], (unsigned)(((t - D) / D) & 1))) {
        give_up();
        return;
      }
      last_issued = t;
      unsigned char *dst = stg + (size_t)(t % D) * a.stage_bytes;
      const int r0a = d.z & ~(PER - 1);
      const int nrc = d.w > 0 ? (d.z + d.w - r0a + PER - 1) / PER : 0;
      mbar_expect_tx(&full[t % D], 16u * (unsigned)(d.y + nrc));
      tma_bulk_g2s(dst, a.blocks + d.x, 16u * (unsigned)d.y, &full[t % D]);
      if (nrc) tma_bulk_g2s(dst + a.capB, a.rhs + r0a, 16u * (unsigned)nrc, &full[t % D]);
    };
    auto prefetch = [&](int t, int4 d) {
      if (lane != 0 || t >= a.nsteps) return;
      rep_prefetch_l2(a.blocks + d.x, 16u * (unsigned)d.y);
      const int r0a = d.z & ~(PER - 1);
      const int nrc = d.w > 0 ? (d.z + d.w - r0a + PER - 1) / PER : 0;
      if (nrc) rep_prefetch_l2(a.rhs + r0a, 16u * (unsigned)nrc);
    };
    // expect the values of step t (every row of the cluster, one T each) once
    // the barrier's previous phase (step t - MV) has completed
    auto arm = [&](int t, int bytes) {
      if (lane != 0 || !live || t >= a.nsteps) return;
      if (t >= MV && !rep_wait_cluster(&vbar[t % MV], (unsigned)(((t - MV) / MV) & 1))) {
        give_up();
        return;
      }
      mbar_expect_tx(&vbar[t % MV], (unsigned)bytes);
    };
    auto vbytes_of = [&](int t) { return t < a.nsteps ? a.vbytes[t] : 0; };
    for (int t = 0; t < kRepAR; ++t) arm(t, vbytes_of(t));
    for (int t = 0; t < D - 1; ++t) issue(t, load_desc(t));
    for (int t = D - 1; t < kRepPF; ++t) prefetch(t, load_desc(t));
    // lane j of chunk c: the steps 32c + j + (D-1, kRepPF, kRepAR)
    int4 ci = load_desc(D - 1 + lane), cp = load_desc(kRepPF + lane);
    int cv = vbytes_of(kRepAR + lane);
    int4 ni = load_desc(32 + D - 1 + lane), np = load_desc(32 + kRepPF + lane);
    int nv = vbytes_of(32 + kRepAR + lane);
    for (int t = 0; t < a.nsteps; ++t) {
      const int j = t & 31;
      if (j == 0 && t > 0) {
        ci = ni;
        cp = np;
        cv = nv;
        ni = load_desc(t + 32 + D - 1 + lane);
        np = load_desc(t + 32 + kRepPF + lane);
        nv = vbytes_of(t + 32 + kRepAR + lane);
      }
      const int vb = __shfl_sync(0xffffffffu, cv, j);
      int4 di, dp;
      di.x = __shfl_sync(0xffffffffu, ci.x, j);
      di.y = __shfl_sync(0xffffffffu, ci.y, j);
      di.z = __shfl_sync(0xffffffffu, ci.z, j);
      di.w = __shfl_sync(0xffffffffu, ci.w, j);
      dp.x = __shfl_sync(0xffffffffu, cp.x, j);
      dp.y = __shfl_sync(0xffffffffu, cp.y, j);
      dp.z = __shfl_sync(0xffffffffu, cp.z, j);
      dp.w = __shfl_sync(0xffffffffu, cp.w, j);
      arm(t + kRepAR, vb);
      issue(t + D - 1, di);
      prefetch(t + kRepPF, dp);
    }
    // no bulk copy may still be writing this CTA's shared memory when it
    // exits: wait (bounded) for the last copy issued into every stage (on the
    // normal path the compute groups have already seen them all complete)
    if (lane == 0)
      for (int t = last_issued - D + 1; t <= last_issued; ++t)
        if (t >= 0) mbar_wait(&full[t % D], (unsigned)((t / D) & 1));
    cluster_sync();
    return;
  }

  // ---- compute groups ----
  // the rings (and value barriers) this lane sends to: CTAs sub, sub + TPR, ...
  constexpr int NP = C / TPR > 0 ? C / TPR : 1;
  static_assert(C % TPR == 0 || C < TPR, "cluster size and lanes per row");
  unsigned peer[NP], peerv[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const unsigned k = (unsigned)(sub + j * TPR) % (unsigned)C;
    peer[j] = rep_mapa(ring_s, k);
    peerv[j] = rep_mapa(vbar_s, k);
  }
  const bool sender = sub < C;  // fewer CTAs than lanes: the first C lanes send
  auto stage_ready = [&](int t) {
    if (live && !mbar_wait(&full[t % D], (unsigned)((t / D) & 1))) give_up();
    return live;
  };
  auto values_ready = [&](int t) {
    if (live && !rep_wait_cluster(&vbar[t % MV], (unsigned)((t / MV) & 1))) give_up();
  };

  // per-row state of this thread's next step
  T partial = T(0), rhs_r = T(0);
  T n1v[kRepN1];
  unsigned n1a[kRepN1];
  int n1c = 0, mbeg = 0, mend = 0;  // previous-step entries; mid entries [mbeg, mend) in the stage
  int nr_s = 0, r0_s = 0;           // rows and first position of this CTA's slice of the next step
  // far entries of this thread's next step, loaded a group cycle early (raw bits: the sentinel until written)
  typedef typename Bits<T>::U U;
  const U sent = (U)Sentinel<T>::bits;
  U farb[kRepNF];
  T farv[kRepNF];
  int farq[kRepNF], nfc = 0;
#pragma unroll
  for (int f = 0; f < kRepNF; ++f) {
    farb[f] = (U)0;
    farv[f] = T(0);
    farq[f] = 0;
  }

  // part A of step u (right after this group's previous step): older ring
  // entries (at least G + 1 steps back: their values have landed), far
  // entries, previous-step entries and right-hand side into registers, then
  // the far loads of step u + G
  auto prepare = [&](int u) {
    partial = T(0);
    rhs_r = T(0);
    n1c = 0;
    mbeg = mend = 0;
    nr_s = r0_s = 0;
    if (u >= a.nsteps || !stage_ready(u)) return;
    const unsigned char *sp = stg + (size_t)(u % D) * a.stage_bytes;
    const int4 hdr = *reinterpret_cast<const int4 *>(sp);
    nr_s = hdr.x;
    r0_s = hdr.w;
    const int4 h3 = reinterpret_cast<const int4 *>(sp)[3];
    const RepLayout L = rep_layout<T>(hdr.x, hdr.y, h3.x, hdr.z, h3.y, a.linked != 0);
    if (slot < hdr.x) {
      const int4 ri = *reinterpret_cast<const int4 *>(sp + L.o_row + 16 * slot);
      const int n1 = ri.y & 0xff, nm = (ri.y >> 8) & 0xff, no = (ri.y >> 16) & 0xff;
      const unsigned short *sl = reinterpret_cast<const unsigned short *>(sp + L.o_slot);
      const T *vl = reinterpret_cast<const T *>(sp + L.o_val);
      T acc = T(0);
      const int ob = ri.x + n1 + nm;
#pragma unroll 4
      for (int k = ob + sub; k < ob + no; k += TPR) acc = fma(vl[k], ring[sl[k] & a.rmask], acc);
#pragma unroll
      for (int f = 0; f < kRepNF; ++f)
        if (f < nfc) {
          U b = farb[f];
          if (b == sent) b = Bits<T>::load(a.xp + farq[f]);
          const T x = b == sent ? wait_value(a.xp + farq[f], a.err) : Bits<T>::from(b);
          acc = fma(farv[f], x, acc);
        }
      partial = acc;
#pragma unroll
      for (int e = 0; e < kRepN1; ++e) {
        const int k = ri.x + sub + e * TPR;
        if (k < ri.x + n1) {
          n1v[e] = vl[k];
          n1a[e] = ring_s + (unsigned)sizeof(T) * (sl[k] & a.rmask);
          n1c = e + 1;
        }
      }
      mbeg = ri.x + n1;
      mend = ri.x + n1 + nm;
      rhs_r = reinterpret_cast<const T *>(sp + a.capB)[(hdr.w & (PER - 1)) + slot];
    }
    nfc = 0;
    // far values of this slot's row in step u + G (listed in step u's block)
    if (hdr.z > 0 && slot < h3.x) {
      const int2 fr = reinterpret_cast<const int2 *>(sp + L.o_fr)[slot];
      const int *fq = reinterpret_cast<const int *>(sp + L.o_fq);
      const T *fv = reinterpret_cast<const T *>(sp + L.o_fv);
#pragma unroll
      for (int f = 0; f < kRepNF; ++f) {
        const int k = sub + f * TPR;
        if (k < fr.y) {
          farv[f] = fv[fr.x + k];
          farq[f] = fq[fr.x + k];
          farb[f] = Bits<T>::load(a.xp + farq[f]);
          nfc = f + 1;
        }
      }
    }
  };

  const bool tr = a.trace && rank == 0 && (tid == 0 || tid == GT);
  unsigned long long c_b = 0, c_crit = 0, c_st = 0, c_a = 0, c_sync = 0, c_w1 = 0, c_w2 = 0, tk0 = 0, tn0 = 0;
  if (tr) {
    tk0 = clock64();
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(tn0));
  }
  prepare(grp);
  for (int s = grp; s < a.nsteps; s += G) {
    const unsigned long long t0 = tr ? clock64() : 0ull;
    // ---- part B: entries 2 .. G steps back, once step s-2 has landed ----
    if (s >= 2) values_ready(s - 2);
    const unsigned long long t1 = tr ? clock64() : 0ull;
    if (live) {
      const unsigned char *sp = stg + (size_t)(s % D) * a.stage_bytes;
      const int4 hdr = *reinterpret_cast<const int4 *>(sp);
      const int4 h3 = reinterpret_cast<const int4 *>(sp)[3];
      const RepLayout L = rep_layout<T>(hdr.x, hdr.y, h3.x, hdr.z, h3.y, a.linked != 0);
      const unsigned short *sl = reinterpret_cast<const unsigned short *>(sp + L.o_slot);
      const T *vl = reinterpret_cast<const T *>(sp + L.o_val);
      T acc = partial;
      for (int k = mbeg + sub; k < mend; k += TPR) acc = fma(vl[k], ring[sl[k] & a.rmask], acc);
      partial = acc;
    }
    const unsigned long long t2 = tr ? clock64() : 0ull;
    // ---- critical part: previous-step entries, then send ----
    if (s >= 1) values_ready(s - 1);
    const unsigned long long t3 = tr ? clock64() : 0ull;
    const unsigned char *sp = stg + (size_t)(s % D) * a.stage_bytes;
    T acc = partial;
#pragma unroll
    for (int e = 0; e < kRepN1; ++e)
      if (e < n1c) acc = fma(n1v[e], rep_lds(n1a[e], T(0)), acc);
    // butterfly: every lane of the row ends with the same sum, bit for bit
#pragma unroll
    for (int off = TPR / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, TPR);
    const bool row = live && slot < nr_s;
    const bool mine = row && sub == 0;
    const int p = r0_s + slot;
    const T t = rhs_r - acc;
    if (row && sender) {
      // the row's lanes share the sends to the C rings
      const unsigned off = (unsigned)sizeof(T) * (unsigned)(p & a.rmask);
      const unsigned vo = 8u * (unsigned)(s % MV);
#pragma unroll
      for (int j = 0; j < NP; ++j) rep_st_async(peer[j] + off, t, peerv[j] + vo);
    }
    const int4 hdr = live ? *reinterpret_cast<const int4 *>(sp) : zero4;
    const unsigned long long t4 = tr ? clock64() : 0ull;
    // ---- outputs, then release the stage ----
    if (mine) {
      const RepLayout L = rep_layout<T>(hdr.x, 0, 0, 0, 0, a.linked != 0);  // row arrays only
      const int4 ri = *reinterpret_cast<const int4 *>(sp + L.o_row + 16 * slot);
      if (a.out) a.out[ri.w] = a.alpha * t;
      if (a.tpos) a.tpos[p] = t;
      if (a.next) a.next[reinterpret_cast<const int *>(sp + L.o_npos)[slot]] =
          reinterpret_cast<const T *>(sp + L.o_nsc)[slot] * t;
      if ((ri.y >> 24) & 1) Bits<T>::store(a.xp + p, Bits<T>::canon(t));
    }
    // far copies whose last reader was in step s-1: every read of them came
    // before that reader's send, and step s-1 has landed
    if (live) {
      const int4 h3 = reinterpret_cast<const int4 *>(sp)[3];
      if (h3.y > 0) {
        const RepLayout L = rep_layout<T>(hdr.x, hdr.y, h3.x, hdr.z, h3.y, a.linked != 0);
        const int *rst = reinterpret_cast<const int *>(sp + L.o_rst);
        for (int i = tid - grp * GT; i < h3.y; i += GT) Bits<T>::store(a.xp + rst[i], Sentinel<T>::value());
      }
    }
    __syncwarp();
    if (lane == 0) rep_arrive_cta(&empty[s % D]);
    const unsigned long long t5 = tr ? clock64() : 0ull;
    const unsigned long long t6 = t5;
    prepare(s + G);
    if (tr) {
      const unsigned long long t7 = clock64();
      c_w2 += t1 - t0;
      c_b += t2 - t1;
      c_w1 += t3 - t2;
      c_crit += t4 - t3;
      c_st += t5 - t4;
      c_sync += t6 - t5;
      c_a += t7 - t6;
    }
  }
  // every value sent to this CTA has landed before it exits: one thread waits
  // (bounded, also after a give-up) on the last phase of every value barrier,
  // so that no peer's st.async is still in flight into this CTA's memory
  values_ready(a.nsteps - 1);
  if (tid == 0)
    for (int t = a.nsteps - MV; t < a.nsteps; ++t)
      if (t >= 0) rep_wait_cluster(&vbar[t % MV], (unsigned)((t / MV) & 1));
  cluster_sync();
  // far copies read in the last step: every reader is done
  if (a.tail_ptr)
    for (int i = a.tail_ptr[rank] + tid; i < a.tail_ptr[rank + 1]; i += G * GT)
      Bits<T>::store(a.xp + a.tail[i], Sentinel<T>::value());
  if (tr) {
    unsigned long long tn1;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(tn1));
    unsigned long long *o = a.trace + (tid == 0 ? 0 : 10);
    o[0] += c_w2;
    o[1] += c_b;
    o[2] += c_w1;
    o[3] += c_crit;
    o[4] += c_st;
    o[5] += c_sync;
    o[6] += c_a;
    o[7] += (unsigned long long)((a.nsteps - grp + G - 1) / G);
    o[8] += clock64() - tk0;
    o[9] += tn1 - tn0;
  }
}

}  // namespace mldg
