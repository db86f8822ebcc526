// One-warp and grid-stride helper kernels of the plan's entry points
// (reductions' final merges, mean handling). Included by one translation unit only.
#pragma once
#include "pfc_kernels.cuh"

namespace pfc {

// ---------------------------------------------------------------- small kernels
// Merge of n compensated (sum, compensation) pairs at p[stride * b], b < n, by one
// warp in a fixed order: lane l merges b = l, l + 32, ... in turn, then the lanes
// combine in a fixed shuffle tree. The result (valid in lane 0) is deterministic.
__device__ KSum warp_merge(const double* p, int n, int stride) {
  const int lane = threadIdx.x & 31;
  KSum acc = {0.0, 0.0};
  for (int b = lane; b < n; b += 32) {
    const KSum o = {p[(size_t)stride * b], p[(size_t)stride * b + 1]};
    acc = ksum_merge(acc, o);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    KSum o;
    o.s = __shfl_down_sync(0xffffffffu, acc.s, off);
    o.c = __shfl_down_sync(0xffffffffu, acc.c, off);
    acc = ksum_merge(acc, o);
  }
  return acc;
}

// Final reduction of per-CTA compensated partials (one warp), in a fixed order.
// row partials: 3 sums (raw, fpoly, nonlin) x nrow; col partials: 1 sum x ncol.
// out3 = {F per site, mu per site, mean}.
__global__ void finalize_reduce_kernel(const double* rowp, int nrow, const double* colp, int ncol,
                                       const double* scal, double inv_sites, double lmu0, double lf0,
                                       int dev_form, double* out3, int* status) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  KSum q[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) q[k] = warp_merge(rowp + 2 * k, nrow, 6);
  const KSum p = warp_merge(colp, ncol, 2);
  if (threadIdx.x != 0) return;
  const double mean_dev = dev_form ? scal[kScalMean] : 0.0;
  const double raw_mean = (q[0].s + q[0].c) * inv_sites;
  double grad = (p.s + p.c) * inv_sites * inv_sites;
  if (dev_form) grad += lf0 * mean_dev * mean_dev;   // k = 0 term carried in FP64
  const double F = grad + (q[1].s + q[1].c) * inv_sites;
  const double mean = dev_form ? mean_dev : raw_mean;
  const double mu = lmu0 * mean + (q[2].s + q[2].c) * inv_sites;
  out3[0] = F;
  out3[1] = mu;
  out3[2] = mean;
  if (!isfinite(F) || !isfinite(mu) || !isfinite(raw_mean)) atomicOr(status, 1);
}

// Sum of materialise partials -> scal[kScalCorr] = sum / sites (deviation mean correction).
__global__ void finalize_mean_kernel(const double* p, int nb, double inv_sites, double* scal) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  const KSum acc = warp_merge(p, nb, 2);
  if (threadIdx.x == 0) scal[kScalCorr] = (acc.s + acc.c) * inv_sites;
}

__global__ void shift_kernel(double* x, size_t n, const double* by) {
  const double s = *by;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] -= s;
}

// Compensated sum of a real field (grid-stride), per-CTA partials.
__global__ void field_sum_kernel(const double* x, size_t n, double* partials) {
  KSum acc[1] = {{0.0, 0.0}};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    ksum_add(acc[0], x[i]);
  block_reduce_store<1>(acc, partials + 2 * blockIdx.x);
}

// Deviation-form scalars from the mean (std and log nonlinearities).
__global__ void set_scalars_kernel(const double* p, int nb, double inv_sites, int model, double g,
                                   double min_phi, double lmu0, double* scal) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  const KSum acc = warp_merge(p, nb, 2);
  if (threadIdx.x != 0) return;
  const double mu = (acc.s + acc.c) * inv_sites;
  scal[kScalMean] = mu;
  scal[kScalC1] = 2.0 * g * mu + 3.0 * mu * mu;
  scal[kScalC2] = g + 3.0 * mu;
  scal[kScalInvMean] = (mu != 0.0) ? 1.0 / mu : 0.0;
  double n0 = g * mu * mu + mu * mu * mu;
  if (model == kModelLog) n0 += log(mu);
  scal[kScalN0] = n0;
  scal[kScalLogMin] = (model == kModelLog && min_phi > 0.0 && mu > 0.0) ? log(min_phi) - log(mu) : 0.0;
  scal[kScalZero] = 0.0;
  scal[kScalCorr] = 0.0;
  scal[kScalMuConst] = lmu0 * mu + n0;
}

}  // namespace pfc
