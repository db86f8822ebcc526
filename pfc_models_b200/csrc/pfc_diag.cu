// 3-mode fitness diagnostics of a crystal field on the device: the quantities the
// reference's phase-diagram adapters compute in `diagnose`
// (src/pfc_models/models/stdpfc_cpu/phase_diagram.py:178-215, the same code in
// logpfc_cpu/phase_diagram.py:182-240): the mean |n_hat| over each of three sets of mode
// indices (the amplitudes A, B, C), the mean squared deviation of n from the field those
// amplitudes and the mean rebuild (`_build3Mode`), and the count of strict local maxima
// over the 8 periodic neighbours (`_maxima_per_cell`).
//
// The reference rebuilds the 3-mode field with an inverse FFT and subtracts it in real
// space. Here the deviation comes from Parseval instead: the rebuilt field's spectrum is
// non-zero only at the DC entry and the mode entries, so
//   mean((n - n3)^2) = mean(n^2) - sum_e w_e (|n_hat_e|^2 - |n_hat_e - V_e|^2) / N^2
// over those entries e (w_e = 1 in the DC and Nyquist columns of the half spectrum, 2
// elsewhere; V_e the rebuilt value there). One pass over the field gives mean(n^2)
// (compensated) and the maxima count; a one-warp kernel gathers the entries.
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "pfc_kernels.cuh"
#include "pfc_registry.h"

namespace pfc {
namespace {

constexpr int kDiagBlocks = 256, kDiagThreads = 256;

// Compensated merge of n (s, c) pairs at p[stride * b] by one warp; lane 0 holds the total.
__device__ KSum diag_warp_merge(const double* p, int n, int stride) {
  const int lane = threadIdx.x & 31;
  KSum acc = {0.0, 0.0};
  for (int b = lane; b < n; b += 32) acc = ksum_merge(acc, KSum{p[(size_t)stride * b], p[(size_t)stride * b + 1]});
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    KSum o;
    o.s = __shfl_down_sync(0xffffffffu, acc.s, off);
    o.c = __shfl_down_sync(0xffffffffu, acc.c, off);
    acc = ksum_merge(acc, o);
  }
  return acc;
}

// Per CTA: compensated sum of n^2 (2 doubles) and the count of strict periodic
// 8-neighbour maxima (as a double, exact below 2^53), at partials[4 * blockIdx.x].
__global__ void __launch_bounds__(kDiagThreads) diag_field_kernel(const double* __restrict__ f, int nx, int ny,
                                                                   double* __restrict__ partials) {
  KSum acc[1] = {{0.0, 0.0}};
  unsigned long long count = 0;
  const size_t n = (size_t)nx * ny;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double v = f[i];
    ksum_add(acc[0], v * v);
    const int x = (int)(i % nx), y = (int)(i / nx);
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const double* rm = f + (size_t)ym * nx;
    const double* r0 = f + (size_t)y * nx;
    const double* rp = f + (size_t)yp * nx;
    const bool is_max = v > rm[xm] && v > rm[x] && v > rm[xp] && v > r0[xm] && v > r0[xp] && v > rp[xm] &&
                        v > rp[x] && v > rp[xp];
    count += is_max ? 1 : 0;
  }
  // integer counts: any summation order is exact
  __shared__ unsigned long long red[kDiagThreads / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) count += __shfl_down_sync(0xffffffffu, count, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = count;
  block_reduce_store<1>(acc, partials + 4 * blockIdx.x);   // synchronises the CTA
  if (threadIdx.x == 0) {
    unsigned long long c = 0;
    for (int w = 0; w < kDiagThreads / 32; ++w) c += red[w];
    partials[4 * blockIdx.x + 2] = (double)c;
  }
}

// out6 = {fitness, |A|, |B|, |C|, mean, maxima count}
__global__ void diag_finalize_kernel(const double* __restrict__ partials, int nb, const double* __restrict__ spec,
                                     DiagModes m, double n_sites, double* __restrict__ out6) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  const KSum sq = diag_warp_merge(partials, nb, 4);
  if (threadIdx.x != 0) return;
  double count = 0.0;
  for (int b = 0; b < nb; ++b) count += partials[4 * b + 2];
  const double mean_sq = (sq.s + sq.c) / n_sites;
  // amplitudes: NaN-skipping mean of |n_hat| over each set's entries (duplicates count),
  // signed, per site
  double amp[3];
  for (int s = 0; s < 3; ++s) {
    double sum = 0.0;
    int cnt = 0;
    for (int e = 0; e < m.n_list; ++e) {
      if (m.list_set[e] != s) continue;
      const double re = spec[2 * (size_t)m.list_flat[e]], im = spec[2 * (size_t)m.list_flat[e] + 1];
      const double a = hypot(re, im);
      if (isnan(a)) continue;
      sum += a;
      ++cnt;
    }
    amp[s] = cnt ? (m.sign * (sum / cnt)) / n_sites : NAN;
  }
  // the rebuilt spectrum V at the distinct entries; the DC entry carries n_hat(0, 0)
  double corr = 0.0;
  for (int e = 0; e < m.n_uniq; ++e) {
    const double re = spec[2 * (size_t)m.uniq_flat[e]], im = spec[2 * (size_t)m.uniq_flat[e] + 1];
    double vr, vi;
    if (m.uniq_set[e] < 0) {
      vr = spec[0];
      vi = spec[1];
    } else {
      vr = amp[m.uniq_set[e]] * n_sites;
      vi = 0.0;
    }
    const double dr = re - vr, di = im - vi;
    corr += m.uniq_w[e] * ((re * re + im * im) - (dr * dr + di * di));
  }
  const double dev = mean_sq - corr / (n_sites * n_sites);
  out6[0] = 1.0 - fabs(dev);
  out6[1] = fabs(amp[0]);
  out6[2] = fabs(amp[1]);
  out6[3] = fabs(amp[2]);
  out6[4] = spec[0] / n_sites;
  out6[5] = count;
}

// ---- frozen-field moments (logpfc_cpu/phase_diagram.py:465-505): per CTA, compensated
// sums of w |X_k|^2 K^n, n = 0, 1, 2, over the half spectrum (w = 1 in the DC and Nyquist
// columns, 2 elsewhere, so the sums equal those over the full fft2 grid), with
// K = |k_ref|^2 from NumPy's fftfreq ordering; at partials[6 * blockIdx.x].
constexpr int kFrozenBlocks = 128;

__global__ void __launch_bounds__(kDiagThreads) frozen_spectral_kernel(const double* __restrict__ spec, int nx,
                                                                        int ny, double fx, double fy,
                                                                        double* __restrict__ partials) {
  KSum acc[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
  const int nxh = nx / 2 + 1;
  const size_t n = (size_t)ny * nxh;
  const double two_pi = 6.283185307179586;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / nxh), c = (int)(i % nxh);
    const double re = spec[2 * i], im = spec[2 * i + 1];
    const int ky_i = r <= (ny - 1) / 2 ? r : r - ny;
    const double kx = two_pi * ((double)c * fx), ky = two_pi * ((double)ky_i * fy);
    const double K = kx * kx + ky * ky;
    const double w = (c == 0 || (nx % 2 == 0 && c == nx / 2)) ? 1.0 : 2.0;
    const double wp = w * (re * re + im * im);
    ksum_add(acc[0], wp);
    ksum_add(acc[1], wp * K);
    ksum_add(acc[2], wp * K * K);
  }
  block_reduce_store<3>(acc, partials + 6 * blockIdx.x);
}

// The local term phi ln phi + temp/2 phi^2 + g/3 phi^3 + v0/4 phi^4 summed over the field
// (compensated), at partials[2 * blockIdx.x].
__global__ void __launch_bounds__(kDiagThreads) frozen_local_kernel(const double* __restrict__ f, size_t n,
                                                                     double temp, double g, double v0,
                                                                     double* __restrict__ partials) {
  KSum acc[1] = {{0.0, 0.0}};
  const double ct = temp / 2, cg = g / 3, cv = v0 / 4;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double p = f[i], p2 = p * p;
    ksum_add(acc[0], p * log(p) + ct * p2 + cg * (p2 * p) + cv * (p2 * p2));
  }
  block_reduce_store<1>(acc, partials + 2 * blockIdx.x);
}

// out4 = {A0, A1, A2, local}
__global__ void frozen_finalize_kernel(const double* __restrict__ sp, const double* __restrict__ lp, int nb,
                                       double n_sites, double* __restrict__ out4) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  KSum s[3];
  for (int q = 0; q < 3; ++q) s[q] = diag_warp_merge(sp + 2 * q, nb, 6);
  const KSum l = diag_warp_merge(lp, nb, 2);
  if (threadIdx.x != 0) return;
  const double n2 = n_sites * n_sites;
  for (int q = 0; q < 3; ++q) out4[q] = (s[q].s + s[q].c) / n2;
  out4[3] = (l.s + l.c) / n_sites;
}

// ---- defect screen (logpfc_cpu/phase_diagram.py:512-528). Field pass, per CTA at
// partials[5 * b]: the count of sites >= their 8 periodic neighbours and above the mean,
// the compensated sum of their heights above the mean (2 doubles), the largest and the
// smallest height. The mean is the spectrum's DC entry over the site count.
constexpr int kDefectBlocks = 128;

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}

__global__ void __launch_bounds__(kDiagThreads) defect_field_kernel(const double* __restrict__ f, int nx, int ny,
                                                                     const double* __restrict__ spec,
                                                                     double* __restrict__ partials) {
  const double m = spec[0] / ((double)nx * (double)ny);
  KSum acc[1] = {{0.0, 0.0}};
  unsigned long long count = 0;
  double hmax = -INFINITY, hmin = INFINITY;
  const size_t n = (size_t)nx * ny;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double v = f[i];
    if (!(v > m)) continue;
    const int x = (int)(i % nx), y = (int)(i / nx);
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const double* rm = f + (size_t)ym * nx;
    const double* r0 = f + (size_t)y * nx;
    const double* rp = f + (size_t)yp * nx;
    if (v >= rm[xm] && v >= rm[x] && v >= rm[xp] && v >= r0[xm] && v >= r0[xp] && v >= rp[xm] && v >= rp[x] &&
        v >= rp[xp]) {
      const double h = v - m;
      ksum_add(acc[0], h);
      ++count;
      hmax = fmax(hmax, h);
      hmin = fmin(hmin, h);
    }
  }
  __shared__ unsigned long long rc[kDiagThreads / 32];
  __shared__ double rmax[kDiagThreads / 32], rmin[kDiagThreads / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) count += __shfl_down_sync(0xffffffffu, count, off);
  hmax = warp_max(hmax);
  hmin = warp_min(hmin);
  if ((threadIdx.x & 31) == 0) {
    rc[threadIdx.x >> 5] = count;
    rmax[threadIdx.x >> 5] = hmax;
    rmin[threadIdx.x >> 5] = hmin;
  }
  block_reduce_store<1>(acc, partials + 5 * blockIdx.x + 1);   // synchronises the CTA
  if (threadIdx.x == 0) {
    unsigned long long c = 0;
    double mx = -INFINITY, mn = INFINITY;
    for (int w = 0; w < kDiagThreads / 32; ++w) {
      c += rc[w];
      mx = fmax(mx, rmax[w]);
      mn = fmin(mn, rmin[w]);
    }
    partials[5 * blockIdx.x] = (double)c;
    partials[5 * blockIdx.x + 3] = mx;
    partials[5 * blockIdx.x + 4] = mn;
  }
}

// Spectral pass, per CTA at partials[2 * b]: the largest |X_k|^2 with 0 < |k_ref| < 0.95
// and the largest over k != 0 (the mean only moves the DC entry; the half spectrum
// holds every magnitude of the full grid).
__global__ void __launch_bounds__(kDiagThreads) defect_spectral_kernel(const double* __restrict__ spec, int nx,
                                                                        int ny, double fx, double fy,
                                                                        double* __restrict__ partials) {
  const int nxh = nx / 2 + 1;
  const size_t n = (size_t)ny * nxh;
  const double two_pi = 6.283185307179586;
  double psub = 0.0, pall = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if (i == 0) continue;
    const int r = (int)(i / nxh), c = (int)(i % nxh);
    const double re = spec[2 * i], im = spec[2 * i + 1];
    const double p = re * re + im * im;
    const int ky_i = r <= (ny - 1) / 2 ? r : r - ny;
    const double kx = two_pi * ((double)c * fx), ky = two_pi * ((double)ky_i * fy);
    const double kr = sqrt(kx * kx + ky * ky);
    pall = fmax(pall, p);
    if (kr > 1e-9 && kr < 0.95) psub = fmax(psub, p);
  }
  __shared__ double rs[kDiagThreads / 32], ra[kDiagThreads / 32];
  psub = warp_max(psub);
  pall = warp_max(pall);
  if ((threadIdx.x & 31) == 0) {
    rs[threadIdx.x >> 5] = psub;
    ra[threadIdx.x >> 5] = pall;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kDiagThreads / 32; ++w) {
      psub = fmax(psub, rs[w]);
      pall = fmax(pall, ra[w]);
    }
    partials[2 * blockIdx.x] = psub;
    partials[2 * blockIdx.x + 1] = pall;
  }
}

// out4 = {peak spread, sub-q ratio, peak count, 0}; NaN where the reference's is NaN
__global__ void defect_finalize_kernel(const double* __restrict__ fp, const double* __restrict__ sp, int nb,
                                       double* __restrict__ out4) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  const KSum hs = diag_warp_merge(fp + 1, nb, 5);
  if (threadIdx.x != 0) return;
  double count = 0.0, mx = -INFINITY, mn = INFINITY, psub = 0.0, pall = 0.0;
  for (int b = 0; b < nb; ++b) {
    count += fp[5 * b];
    mx = fmax(mx, fp[5 * b + 3]);
    mn = fmin(mn, fp[5 * b + 4]);
    psub = fmax(psub, sp[2 * b]);
    pall = fmax(pall, sp[2 * b + 1]);
  }
  out4[0] = count > 0 ? (mx - mn) / ((hs.s + hs.c) / count) : NAN;
  out4[1] = pall > 0 ? psub / pall : NAN;
  out4[2] = count;
  out4[3] = 0.0;
}

}  // namespace

cudaError_t launch_defect_screen(const double* field, const double* spec, int nx, int ny, double fx, double fy,
                                 double* partials, double* out4, cudaStream_t stream) {
  double* fp = partials;
  double* sp = partials + 5 * kDefectBlocks;
  defect_field_kernel<<<kDefectBlocks, kDiagThreads, 0, stream>>>(field, nx, ny, spec, fp);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  defect_spectral_kernel<<<kDefectBlocks, kDiagThreads, 0, stream>>>(spec, nx, ny, fx, fy, sp);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  defect_finalize_kernel<<<1, 32, 0, stream>>>(fp, sp, kDefectBlocks, out4);
  return cudaGetLastError();
}

cudaError_t launch_frozen_moments(const double* field, const double* spec, int nx, int ny, double fx, double fy,
                                  double temp, double g, double v0, double* partials, double* out4,
                                  cudaStream_t stream) {
  double* sp = partials;
  double* lp = partials + 6 * kFrozenBlocks;
  frozen_spectral_kernel<<<kFrozenBlocks, kDiagThreads, 0, stream>>>(spec, nx, ny, fx, fy, sp);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  frozen_local_kernel<<<kFrozenBlocks, kDiagThreads, 0, stream>>>(field, (size_t)nx * ny, temp, g, v0, lp);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  frozen_finalize_kernel<<<1, 32, 0, stream>>>(sp, lp, kFrozenBlocks, (double)nx * (double)ny, out4);
  return cudaGetLastError();
}

cudaError_t launch_diagnose_modes(const double* field, const double* spec, int nx, int ny, const DiagModes& m,
                                  double* partials, double* out6, cudaStream_t stream) {
  diag_field_kernel<<<kDiagBlocks, kDiagThreads, 0, stream>>>(field, nx, ny, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  diag_finalize_kernel<<<1, 32, 0, stream>>>(partials, kDiagBlocks, spec, m, (double)nx * (double)ny, out6);
  return cudaGetLastError();
}

// doubles of plan scratch the diagnostics use: the largest of their partial layouts
int diagnose_partials_needed() {
  const int a = 4 * kDiagBlocks, b = 8 * kFrozenBlocks, c = 7 * kDefectBlocks;
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}

}  // namespace pfc
