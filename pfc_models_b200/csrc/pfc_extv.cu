// Log PFC with an external potential and a re-optimised linear shift M (the reference's
// logpfc_extv model, models/logpfc_extv/simulation.py): the per-step decision and the
// coefficient rebuild, on the device, between the row and the column pass of a step.
//
// The reference's step (TimeStep :301-330) is ValidatePhiRange, then the ETD1 update
//   phi_hat' = A_M phi_hat + B_M (Gamma lap N_hat_M + lap V_hat),  N_M = N - M phi,
// with A_M, B_M from L_M = Gamma lap (beta (q0^2 + lap)^2 + eps + M). Because -M phi is
// linear it is folded into the coefficient of phi_hat: the column kernel applies
//   phi_hat' = phi_hat + (A_M - 1 - M Bg_M) phi_hat + Bg_M N_hat + F_M,
// Bg_M = B_M Gamma lap, F_M = B_M lap V_hat, so the row pass computes the plain clamped
// logPFC nonlinearity (plus the field's minimum and maximum) and the spectra it leaves in
// V stay those of the reference's nonlinearity without M, from which mu follows as in
// the reference (M cancels between its linear and nonlinear parts).
#include <algorithm>
#include <cmath>

#include <cuda_runtime.h>

#include "pfc_registry.h"

namespace pfc {

// ValidatePhiRange (:375-405) and OptimizeM (:332-373) on the row pass's per-CTA
// (min, max) pairs: one CTA; thread 0 applies the reference's rules in FP64.
__global__ void extv_decide_kernel(const double* __restrict__ minmax, int nparts, ExtvState* st, double g) {
  __shared__ double smin[256], smax[256];
  double lo = INFINITY, hi = -INFINITY;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    lo = fmin(lo, minmax[2 * i]);
    hi = fmax(hi, minmax[2 * i + 1]);
  }
  smin[threadIdx.x] = lo;
  smax[threadIdx.x] = hi;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  lo = smin[0];
  hi = smax[0];
  st->last_min = lo;
  st->last_max = hi;
  bool opt = !st->init;
  if (!opt) {
    const bool floor_breached = (st->phi_min - lo) / st->phi_min > st->floor_tol;
    const bool ceiling_breached = (hi - st->phi_max) / st->phi_max > st->ceil_tol;
    opt = floor_breached || ceiling_breached;
  }
  if (opt) {
    const double plo = lo > 0 ? lo : st->min_phi;
    const double nhi = g * hi * hi + hi * hi * hi + log(hi);
    const double nlo = g * plo * plo + plo * plo * plo + log(plo);
    st->M = (nhi - nlo) / (hi - plo);
    st->phi_min = plo;
    st->phi_max = hi;
    st->init = 1;
    st->count += 1;
  }
  st->changed = (opt || st->v_dirty) ? 1 : 0;
  st->v_dirty = 0;
}

// (A_M - 1 - M Bg_M, Bg_M) of every (kx <= m, ky <= ny/2) and F_M of every (kx <= m, ky),
// when the decision above changed M or V changed; the same expressions as the host build
// of the coefficients (kernel_etd, discretization/spectral/kernels.py:55-71).
__global__ void extv_coef_kernel(ExtvCoefArgs a, const ExtvState* __restrict__ st) {
  if (!st->changed) return;
  const double M = st->M;
  const double twopi = 6.283185307179586;
  const long long ncoef = (long long)(a.m + 1) * a.nyh, nforce = (long long)(a.m + 1) * a.ny;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ncoef + nforce;
       i += (long long)gridDim.x * blockDim.x) {
    int kx, ky;
    if (i < ncoef) {
      kx = (int)(i / a.nyh);
      ky = (int)(i - (long long)kx * a.nyh);
    } else {
      const long long j = i - ncoef;
      kx = (int)(j / a.ny);
      ky = (int)(j - (long long)kx * a.ny);
    }
    const int kys = (ky <= (a.ny - 1) / 2) ? ky : ky - a.ny;
    const double kyp = twopi * ((double)kys * a.fy);
    const double kxp = twopi * ((double)kx * a.fx);
    const double lap = -(kxp * kxp + kyp * kyp);
    const double t = a.q0 * a.q0 + lap;
    const double lmu = a.beta * (t * t) + a.epsilon + M;
    const double gl = a.gamma * lap;
    const double ln = gl * lmu;
    const double z = ln * a.dt;
    const double A = exp(z);
    const double B = (fabs(z) > a.small_z_tol) ? (A - 1) / ln : a.dt * (1 + z / 2 + z * z / 6);
    const double Bg = B * gl;
    if (i < ncoef) {
      a.coef[i] = make_double2(expm1(z) - M * Bg, Bg);
    } else {
      const double2 v = a.vhat[(size_t)ky * (a.m + 1) + kx];
      const double f = B * lap;
      a.forcing[i - ncoef] = make_double2(f * v.x, f * v.y);
    }
  }
}

cudaError_t launch_extv_decide(const double* minmax, int nparts, ExtvState* st, double g, cudaStream_t s) {
  extv_decide_kernel<<<1, 256, 0, s>>>(minmax, nparts, st, g);
  return cudaGetLastError();
}

cudaError_t launch_extv_coef(const ExtvCoefArgs& a, const ExtvState* st, cudaStream_t s) {
  const long long n = (long long)(a.m + 1) * (a.nyh + a.ny);
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4 * 148);
  extv_coef_kernel<<<blocks, 256, 0, s>>>(a, st);
  return cudaGetLastError();
}

}  // namespace pfc
