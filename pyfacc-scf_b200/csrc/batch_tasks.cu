// Task lists of the batched engine, built on the device.
//
// Pairs of a class are sorted by molecule, then by Schwarz factor Q
// (descending), so the kets a bra reaches are a prefix of its molecule's
// segment of the ket class: Q_bra Q_ket >= thresh, and in mixed precision
// the FP64 part the prefix with Q_bra Q_ket >= fp32_thresh (for the
// gradient, >= grad_fp32_thresh); for equal classes only kets up to the bra
// itself are canonical.  One thread per bra
// finds the prefixes by binary search (batch_ranges_kernel); one block per
// (class combination, precision, task width) turns the ket ranges into task
// offsets with a block-wide exclusive scan (batch_scan_kernel) and reports
// the task and quartet counts, which the host reads once.
#include <cuda_runtime.h>

#include "batch.h"

namespace pyfacc {

namespace {

__device__ __forceinline__ int q_prefix(const double4* __restrict__ geom, int base, int n, double qb, double t) {
  if (t <= 0) return n;
  int lo = 0, hi = n;  // count of j with qb * Q_j >= t, Q descending
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (qb * geom[base + mid].w >= t) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(256) batch_ranges_kernel(const BatchRangeArgs A) {
  const BatchRangeList& L = A.l[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.nb) return;
  const int bp = L.bra_base + i;
  const double qb = A.geom[bp].w;
  const int m = A.info2[bp].z;  // molecule of the bra
  const int ks = L.seg_k[m], nk = L.seg_k[m + 1] - ks;
  int mm = q_prefix(A.geom, L.ket_base + ks, nk, qb, A.thresh);
  if (L.same) mm = min(mm, i - L.seg_b[m] + 1);
  const int m64 = min(q_prefix(A.geom, L.ket_base + ks, nk, qb, A.fp32_thresh), mm);
  const int mg = min(q_prefix(A.geom, L.ket_base + ks, nk, qb, A.grad_fp32_thresh), mm);
  L.lo[3][i] = ks;
  L.hi[3][i] = ks + mg;
  L.lo[4][i] = ks + mg;
  L.hi[4][i] = ks + mm;
  L.lo[0][i] = ks;
  L.hi[0][i] = ks + mm;
  L.lo[1][i] = ks;
  L.hi[1][i] = ks + m64;
  L.lo[2][i] = ks + m64;
  L.hi[2][i] = ks + mm;
}

__global__ void __launch_bounds__(1024) batch_scan_kernel(const BatchScanArgs A) {
  const BatchScanList& L = A.l[blockIdx.x];
  __shared__ int wsum[32];
  __shared__ long long wq[32];
  __shared__ int carry;
  __shared__ long long qcarry;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) {
    carry = 0;
    qcarry = 0;
  }
  __syncthreads();
  for (int base = 0; base < L.nb; base += blockDim.x) {
    const int i = base + threadIdx.x;
    int cnt = 0;
    long long nq = 0;
    if (i < L.nb) {
      const int len = L.hi[i] - L.lo[i];
      cnt = (len + L.width - 1) / L.width;
      nq = len;
    }
    int v = cnt;
    long long vq = nq;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
      vq += __shfl_xor_sync(0xffffffffu, vq, o);
    }
    if (lane == 31) wsum[w] = v;
    if (lane == 0) wq[w] = vq;
    __syncthreads();
    if (w == 0) {
      int x = lane < nw ? wsum[lane] : 0;
      long long xq = lane < nw ? wq[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
        xq += __shfl_xor_sync(0xffffffffu, xq, o);
      }
      wsum[lane] = x;  // inclusive over warps
      if (lane == 0) wq[0] = xq;
    }
    __syncthreads();
    const int excl = carry + (w > 0 ? wsum[w - 1] : 0) + v - cnt;
    if (i < L.nb) L.toff[i] = excl;
    const int total = wsum[nw - 1];
    const long long tq = wq[0];
    __syncthreads();
    if (threadIdx.x == 0) {
      carry += total;
      qcarry += tq;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    L.toff[L.nb] = carry;
    A.ntasks[blockIdx.x] = carry;
    A.nquartets[blockIdx.x] = qcarry;
  }
}

}  // namespace

void launch_batch_ranges(const BatchRangeArgs& a, int nlists, int nb_max, cudaStream_t s) {
  if (nlists <= 0 || nb_max <= 0) return;
  dim3 grid((nb_max + 255) / 256, nlists), block(256);
  batch_ranges_kernel<<<grid, block, 0, s>>>(a);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

void launch_batch_scans(const BatchScanArgs& a, int nlists, cudaStream_t s) {
  if (nlists <= 0) return;
  batch_scan_kernel<<<nlists, 1024, 0, s>>>(a);
  PF_CUDA(cudaGetLastError());
  count_launch();
}

}  // namespace pyfacc
