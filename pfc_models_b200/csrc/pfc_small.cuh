// Single-thread and grid-stride helper kernels of the plan's entry points
// (reductions' final merges, mean handling). Included by one translation unit only.
#pragma once
#include "pfc_kernels.cuh"

namespace pfc {

// ---------------------------------------------------------------- small kernels
// Final reduction of per-CTA compensated partials, in a fixed order.
// row partials: 3 sums (raw, fpoly, nonlin) x nrow; col partials: 1 sum x ncol.
// out3 = {F per site, mu per site, mean}.
__global__ void finalize_reduce_kernel(const double* rowp, int nrow, const double* colp, int ncol,
                                       const double* scal, double inv_sites, double lmu0, double lf0,
                                       int dev_form, double* out3, int* status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  KSum q[3] = {{0, 0}, {0, 0}, {0, 0}};
  for (int b = 0; b < nrow; ++b)
    for (int k = 0; k < 3; ++k) {
      KSum o = {rowp[6 * b + 2 * k], rowp[6 * b + 2 * k + 1]};
      q[k] = ksum_merge(q[k], o);
    }
  KSum p = {0, 0};
  for (int b = 0; b < ncol; ++b) {
    KSum o = {colp[2 * b], colp[2 * b + 1]};
    p = ksum_merge(p, o);
  }
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
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  KSum acc = {0, 0};
  for (int b = 0; b < nb; ++b) {
    KSum o = {p[2 * b], p[2 * b + 1]};
    acc = ksum_merge(acc, o);
  }
  scal[kScalCorr] = (acc.s + acc.c) * inv_sites;
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
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  KSum acc = {0, 0};
  for (int b = 0; b < nb; ++b) {
    KSum o = {p[2 * b], p[2 * b + 1]};
    acc = ksum_merge(acc, o);
  }
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
