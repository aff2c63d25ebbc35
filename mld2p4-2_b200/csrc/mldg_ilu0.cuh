// mldg_ilu0.cuh -- ILU(0) factorisation on the GPU, bit for bit the host's.
//
// The reference factorises row by row (mlprec/impl/mld_dilu0_fact.f90:284-477,
// ialg = ILU_N, with the row split of ilu_copyin :551-660): row i is split
// into its strict lower part (L), its diagonal and its strict upper part (U);
// then for every k in L's pattern of row i, in increasing column order,
//   l_ik <- l_ik * d_k,  and for every j in U's pattern of row k (ascending):
//     j < i:  l_ij <- l_ij - l_ik(old) * u_kj   if (i, j) is in L's pattern
//     j = i:  dia  <- dia  - l_ik(old) * u_kj
//     j > i:  u_ij <- u_ij - l_ik(old) * u_kj   if (i, j) is in U's pattern
// where l_ik(old) is the value before its scaling; finally d_i = 1 / dia and
// row i of U is scaled by d_i.  Row i reads only finished rows k < i (their
// U row and d_k), so all rows of one dependency level of L's pattern are
// factorised at once, one thread per row, each doing exactly the host's
// operations in the host's order with every product and difference rounded
// separately (__dmul_rn / __dsub_rn: no fused multiply-add), so the factors
// equal the host build's bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mldg {

// per row: entries of the strict lower and strict upper parts
__global__ void k_ilu0_count(int n, const int *__restrict__ irp, const int *__restrict__ ja, int *nl,
                             int *nu) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int a = 0, b = 0;
    for (int k = irp[i]; k < irp[i + 1]; ++k) {
      const int j = ja[k];
      a += j < i;
      b += j > i && j < n;
    }
    nl[i] = a;
    nu[i] = b;
  }
}

// the split: L and U patterns and values, the diagonal into d
__global__ void k_ilu0_split(int n, const int *__restrict__ irp, const int *__restrict__ ja,
                             const double *__restrict__ val, const int *__restrict__ lirp, int *lja,
                             double *lval, const int *__restrict__ uirp, int *uja, double *uval, double *d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int pl = lirp[i], pu = uirp[i];
    double dia = 0.0;
    for (int k = irp[i]; k < irp[i + 1]; ++k) {
      const int j = ja[k];
      if (j < i) {
        lja[pl] = j;
        lval[pl++] = val[k];
      } else if (j == i) {
        dia = val[k];
      } else if (j < n) {
        uja[pu] = j;
        uval[pu++] = val[k];
      }
    }
    d[i] = dia;
  }
}

// one dependency level: rows[r0..r1) are factorised; d holds the diagonal on
// entry and 1/pivot on exit; *bad receives the smallest row whose pivot is
// below eps (the host reports the first such row)
__global__ void k_ilu0_level(const int *__restrict__ rows, int r0, int r1, const int *__restrict__ lirp,
                             const int *__restrict__ lja, double *lval, const int *__restrict__ uirp,
                             const int *__restrict__ uja, double *uval, double *d, double eps, int *bad) {
  for (int r = r0 + blockIdx.x * blockDim.x + threadIdx.x; r < r1; r += gridDim.x * blockDim.x) {
    const int i = rows[r];
    const int le = lirp[i + 1], ue = uirp[i + 1];
    double dia = d[i];
    for (int kk = lirp[i]; kk < le; ++kk) {
      const int k = lja[kk];
      const double temp = lval[kk];
      lval[kk] = __dmul_rn(temp, d[k]);
      int p1 = kk + 1, p2 = uirp[i];
      for (int jj = uirp[k]; jj < uirp[k + 1]; ++jj) {
        const int j = uja[jj];
        if (j < i) {
          while (p1 < le && lja[p1] < j) ++p1;
          if (p1 < le && lja[p1] == j) {
            lval[p1] = __dsub_rn(lval[p1], __dmul_rn(temp, uval[jj]));
            ++p1;
          }
        } else if (j == i) {
          dia = __dsub_rn(dia, __dmul_rn(temp, uval[jj]));
        } else {
          while (p2 < ue && uja[p2] < j) ++p2;
          if (p2 < ue && uja[p2] == j) {
            uval[p2] = __dsub_rn(uval[p2], __dmul_rn(temp, uval[jj]));
            ++p2;
          }
        }
      }
    }
    if (fabs(dia) < eps) {
      atomicMin(bad, i);
      dia = 1.0;  // keeps the later rows finite; the host reports the failure
    }
    const double inv = __ddiv_rn(1.0, dia);
    d[i] = inv;
    for (int kk = uirp[i]; kk < ue; ++kk) uval[kk] = __dmul_rn(uval[kk], inv);
  }
}

}  // namespace mldg
