// Row and column kernels of the fused ETD1 step, plus the state, field and
// reduction kernels that share their transforms.
//
// Data layout in HBM. Every spectral array holds nx/2 "packed" columns of ny
// complex values, stored column-major ([kx][y], y fastest) so that a column
// transform reads one contiguous run. Column 0 packs the two real-valued
// columns of a real-input row transform: entry = X[0] + i X[nx/2] (DC and
// Nyquist). The 2-D spectrum of that packed column is P = H0 + i HM with H0, HM
// the Hermitian kx = 0 and kx = nx/2 columns of the true rfft2; every kernel
// unpacks them from the pair (ky, -ky) before applying a kx-dependent factor.
//
// Per step, with M = nx/2 (state: n_hat = packed rfft2 of n, W = its column
// inverse scaled by 1/(nx ny), so that the unnormalised row C2R of W is n):
//   row kernel    W  -> C2R -> N(n) -> R2C -> V        (read 1, write 1)
//   column kernel V  -> FFT_y -> n_hat' = A n_hat + Bg N_hat -> n_hat'
//                 n_hat' -> IFFT_y -> W'                 (read 2, write 2)
// FP32_MIXED runs the same kernels on delta = n - mean in float; the mean is an
// FP64 device scalar and the packed DC of delta_hat is held at exactly zero.
#pragma once
#include "pfc_fft.cuh"

namespace pfc {

enum : int { kModelStd = 0, kModelLog = 1 };
enum : int { kRowStep = 0, kRowForward = 1, kRowMaterialize = 2, kRowReduce = 3 };
enum : int { kColStep = 0, kColInit = 1, kColCombine = 2, kColParseval = 3, kColExport = 4 };
enum : int { kCombineMu = 0, kCombineLocalMu = 1, kCombineLocalN = 2, kCombineNonlin = 3, kCombineN = 4 };

// Slots of the device scalar block.
enum : int {
  kScalMean = 0,     // mean density (FP64); 0 for the plain form
  kScalC1 = 1,       // deviation form: N(mean + d) - N(mean) = d (c1 + d (c2 + d)) [+ log term]
  kScalC2 = 2,
  kScalInvMean = 3,  // 1 / mean (log model)
  kScalN0 = 4,       // N(mean): constant dropped from the deviation nonlinearity
  kScalLogMin = 5,   // log(min_phi) - log(mean) (clamped log, deviation form)
  kScalZero = 6,     // always 0
  kScalCorr = 7,     // mean correction of a materialised deviation field
  kScalMuConst = 8,  // L_mu(0) mean + N(mean): constant part of mu in the deviation form
  kScalCount = 12
};

// ---------------------------------------------------------------- compensated sums
struct KSum {
  double s, c;
};
__device__ __forceinline__ void ksum_add(KSum& a, double x) {
  const double t = a.s + x;
  if (fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x; else a.c += (x - t) + a.s;
  a.s = t;
}
__device__ __forceinline__ KSum ksum_merge(KSum a, KSum b) {
  KSum r;
  const double t = a.s + b.s;
  const double bp = t - a.s;
  const double e = (a.s - (t - bp)) + (b.s - bp);  // TwoSum error
  r.s = t;
  r.c = a.c + b.c + e;
  return r;
}

// Deterministic block reduction of NQ compensated sums; thread 0 writes
// (s, c) pairs to out[0 .. 2*NQ).
template <int NQ>
__device__ void block_reduce_store(KSum* v, double* out) {
  __shared__ KSum red[32][NQ];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      KSum o;
      o.s = __shfl_down_sync(0xffffffffu, v[q].s, off);
      o.c = __shfl_down_sync(0xffffffffu, v[q].c, off);
      v[q] = ksum_merge(v[q], o);
    }
  }
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) red[warp][q] = v[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      KSum acc = red[0][q];
      for (int w = 1; w < nw; ++w) acc = ksum_merge(acc, red[w][q]);
      out[2 * q] = acc.s;
      out[2 * q + 1] = acc.c;
    }
  }
}

// Block minimum and maximum; thread 0 writes (min, max) to out[0..1]. Every thread of the
// block calls it.
__device__ inline void block_minmax_store(double lo, double hi, double* out) {
  __shared__ double rmin[32], rmax[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, off));
    hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, off));
  }
  if (lane == 0) {
    rmin[warp] = lo;
    rmax[warp] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 1; w < nw; ++w) {
      lo = fmin(lo, rmin[w]);
      hi = fmax(hi, rmax[w]);
    }
    out[0] = lo;
    out[1] = hi;
  }
}

// ---------------------------------------------------------------- nonlinearity
// Plain FP64 form: the reference's expressions
// (models/stdpfc/simulation.py:297, models/logpfc/simulation.py:296).
template <int MODEL>
__device__ __forceinline__ double nonlin_plain(double n, double g, int clamp, double min_phi, double min_log) {
  const double n2 = n * n;
  double r = g * n2 + n2 * n;
  if (MODEL == kModelLog) r += (clamp && !(n > min_phi)) ? min_log : log(n);
  return r;
}

// FP32 deviation form: N(mean + d) - N(mean). The log term is
// log1p(d / mean); where 1 + d/mean < 1/8 it is evaluated in FP64.
template <int MODEL>
__device__ __forceinline__ float nonlin_dev(float d, float c1, float c2, float inv, double inv_d, int clamp,
                                            double min_phi_rel, float log_min) {
  float r = d * (c1 + d * (c2 + d));
  if (MODEL == kModelLog) {
    const float x = d * inv;
    float l;
    if (x > -0.875f) {
      l = log1pf(x);
    } else {
      const double xd = (double)d * inv_d;   // near-singular branch in FP64
      l = (clamp && !(1.0 + xd > min_phi_rel)) ? log_min : (float)log1p(xd);
    }
    r += l;
  }
  return r;
}

// ---------------------------------------------------------------- arguments
// Buffers of one plan of a batch (pfc_batch_*): the step kernels of a batched launch
// take their per-plan pointers from entry blockIdx.y of a device table of these.
struct BatchBufs {
  const void* w;        // W (row input, column output)
  void* v;              // V (row output, column input)
  const void* nin;      // n_hat of the current state (hi in the FP32 form)
  void* nout;           // n_hat of the next state
  const void* nin_lo;   // FP32 form: the residual arrays of the two states
  void* nout_lo;
  const void* coef;     // (A - 1, Bg), working precision
  const void* coef64;   // FP32 form: (A - 1, Bg) in FP64
  const double* scal;   // deviation-form scalars
};

template <class T>
struct RowArgs {
  int nx, ny, m, rows, tpf, ld;
  FftDesc fft;
  const cplx<T>* tw;
  const cplx<T>* rtw;       // exp(-2 pi i k / nx), k < m
  const cplx<T>* in;        // packed spectra [kx][y]
  cplx<T>* out;             // packed spectra [kx][y]
  const double* in_real;    // (ny, nx) FP64 (forward mode)
  double* out_real;         // (ny, nx) FP64 (materialise mode)
  const double* scal;       // device scalar block
  const double* add;        // materialise: constant added (device pointer), may be null
  double* partials;         // per-CTA compensated sums
  double* minmax;           // step mode, FP64 form: per-CTA (min, max) of the field, or null
  int clamp;
  double g, min_phi, min_log, epsilon;
  const BatchBufs* batch;   // step mode of a batch: per-plan W, V and scalars at [blockIdx.y]
};

// The spectral state and the update n_hat' = n_hat + (A - 1) n_hat + Bg N_hat.
// FP64 form: n_hat is complex128 and (A - 1, Bg) FP64. FP32 form: n_hat is a complex64
// "hi" array plus a complex64 "lo" array holding the rounding residual, and the update
// runs in FP64; for the slow modes (|A - 1| < slow_tau, where rounding errors would
// accumulate over many steps) it uses hi + lo and the FP64 coefficients, elsewhere hi and
// the FP32 coefficients, whose rounding is damped within a few steps. lo stays 0 outside
// the slow modes, so readers may always use hi + lo.
template <class T>
struct ColArgs {
  int nx, ny, m, cols, tpf, ld, nyh;
  FftDesc fft;
  const cplx<T>* tw;
  const cplx<T>* in;            // V (step/init/combine)
  const void* sin;              // n_hat (parseval/export): complex128, or hi (FP32 form)
  const cplx<float>* sin_lo;    //   its lo (FP32 form)
  const void* nin;              // n_hat (step/combine)
  const cplx<float>* nin_lo;
  void* nout;                   // n_hat' (step/init)
  cplx<float>* nout_lo;
  cplx<T>* wout;                // W' (step/init/combine)
  const cplx<T>* coef;          // (A - 1, Bg) [kx][ky], kx <= m, ky <= ny/2, working precision
  const cplx<double>* coef64;   // FP32 form: the same in FP64, read for the slow modes
  const cplx<double>* forcing;  // step mode, FP64 form: added to n_hat', [kx][ky] (kx <= m), or null
  float slow_tau;
  double* partials;
  double* out_c128;             // export: (ny, m+1) complex128
  int dev_form;                 // deviation form: keep the DC of column 0 at zero
  int combine;                  // kCombine*
  double scale;                 // 1 / (nx ny)
  double fx, fy;                // 1/(nx dx), 1/(ny dy): k = 2 pi idx f
  double beta, q0, epsilon, w;  // L_mu, L_f, Gaussian width
  const double* scal;           // device scalar block (export adds the deviation-form DC)
  const BatchBufs* batch;       // step mode of a batch: per-plan buffers at [blockIdx.y]
};

// Element i of a spectral state (hi + lo in the FP32 form when with_lo).
template <class T>
__device__ __forceinline__ cplx<double> state_ld(const void* s, const cplx<float>* lo, size_t i, bool with_lo) {
  if constexpr (sizeof(T) == 8) {
    return static_cast<const cplx<double>*>(s)[i];
  } else {
    const cplx<float> h = static_cast<const cplx<float>*>(s)[i];
    cplx<double> r = mk((double)h.x, (double)h.y);
    if (with_lo) {
      const cplx<float> l = lo[i];
      r.x += (double)l.x;
      r.y += (double)l.y;
    }
    return r;
  }
}

// Stores element i of a spectral state (the FP32 form keeps the residual in lo when with_lo).
template <class T>
__device__ __forceinline__ void state_st(void* s, cplx<float>* lo, size_t i, cplx<double> v, bool with_lo) {
  if constexpr (sizeof(T) == 8) {
    static_cast<cplx<double>*>(s)[i] = v;
  } else {
    const cplx<float> h = mk((float)v.x, (float)v.y);
    static_cast<cplx<float>*>(s)[i] = h;
    if (with_lo) lo[i] = mk((float)(v.x - (double)h.x), (float)(v.y - (double)h.y));
  }
}

// ETD coefficients (A - 1, Bg) of table entry ci in FP64; sets slow (always true in the
// FP64 form, where the state carries no separate residual).
template <class T>
__device__ __forceinline__ cplx<double> coef_ld(const cplx<T>* c, const cplx<double>* c64, size_t ci, float tau,
                                                bool force_slow, bool& slow) {
  const cplx<T> v = c[ci];
  if constexpr (sizeof(T) == 8) {
    slow = true;
    return v;
  } else {
    slow = force_slow || fabsf(v.x) < tau;
    if (slow) return c64[ci];
    return mk((double)v.x, (double)v.y);
  }
}

// wavenumber^2 of packed-column entry (kx, ky), numpy rfftfreq/fftfreq convention
__device__ __forceinline__ double ksq(int kx, int ky, int ny, double fx, double fy) {
  const double twopi = 6.283185307179586;
  const int kys = (ky <= (ny - 1) / 2) ? ky : ky - ny;
  const double kxp = twopi * ((double)kx * fx);
  const double kyp = twopi * ((double)kys * fy);
  return kxp * kxp + kyp * kyp;
}

// ---------------------------------------------------------------- row kernel
// rows transforms of length m per CTA, tpf threads each; smem = rows * ld complex.
template <class T, int MODE, int MODEL, int RSET, int LB = 256, int MINB = 1>
__global__ void __launch_bounds__(LB, MINB) row_kernel(RowArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* sm = reinterpret_cast<cplx<T>*>(smem_raw);
  const int m = a.m, ny = a.ny, rows = a.rows, tpf = a.tpf, ld = a.ld;
  const int y0 = blockIdx.x * rows;
  const int f = threadIdx.x / tpf, lt = threadIdx.x - f * tpf;
  const int y = y0 + f;
  const bool valid = (y < ny);
  const PadBuf<T> buf{sm + f * ld};   // padded exchange buffer of this transform
  const bool dev = (sizeof(T) == 4);
  // per-plan buffers: this plan's, or in a batched step launch plan blockIdx.y's
  const cplx<T>* a_in = a.in;
  cplx<T>* a_out = a.out;
  const double* a_scal = a.scal;
  if (a.batch) {
    const BatchBufs& bb = a.batch[blockIdx.y];
    a_in = static_cast<const cplx<T>*>(bb.w);
    a_out = static_cast<cplx<T>*>(bb.v);
    a_scal = bb.scal;
  }

  if (MODE != kRowForward) {
    // packed spectra, column-major [kx][y]: `rows` consecutive y per kx
    for (int i = threadIdx.x; i < rows * m; i += blockDim.x) {
      const int r = i % rows, kx = i / rows;
      cplx<T> v = mk(T(0), T(0));
      if (y0 + r < ny) v = a_in[(size_t)kx * ny + (y0 + r)];
      sm[r * ld + generic_pad(kx)] = v;
    }
    __syncthreads();
    // pre-process pairs (k, m-k) of the inverse real transform
    for (int k = lt; k <= m / 2; k += tpf) {
      if (k == 0) {
        const cplx<T> p = buf[0];
        buf[0] = mk(p.x + p.y, p.x - p.y);
      } else {
        const int kk = m - k;
        const cplx<T> xk = buf[k], xm = buf[kk];
        const cplx<T> s = xk + conj(xm), d = xk - conj(xm);
        const cplx<T> u = mul_i(cmul(conj(a.rtw[k]), d));
        buf[k] = s + u;
        if (kk != k) buf[kk] = conj(s - u);
      }
    }
    __syncthreads();
    fft_run<true, RSET>(buf, a.fft, a.tw, lt, tpf);
    // buf[j] = x[2j] + i x[2j+1]
  } else {
    // real FP64 field (ny, nx), row-major; deviation form subtracts the mean
    const double mean = dev ? a_scal[kScalMean] : 0.0;
    const double2* src = reinterpret_cast<const double2*>(a.in_real + (size_t)y * a.nx);
    for (int j = lt; j < m; j += tpf) {
      cplx<T> v = mk(T(0), T(0));
      if (valid) {
        const double2 p = src[j];
        v = mk((T)(p.x - mean), (T)(p.y - mean));
      }
      buf[j] = v;
    }
    __syncthreads();
  }

  if (MODE == kRowStep) {
    if (dev) {
      const float c1 = (float)a_scal[kScalC1], c2 = (float)a_scal[kScalC2];
      const float inv = (float)a_scal[kScalInvMean];
      const double inv_d = a_scal[kScalInvMean];
      const double mphi_rel = a.min_phi * inv_d;
      const float lmin = (float)a_scal[kScalLogMin];
      for (int j = lt; j < m; j += tpf) {
        const cplx<T> z = buf[j];
        buf[j] = mk((T)nonlin_dev<MODEL>((float)z.x, c1, c2, inv, inv_d, a.clamp, mphi_rel, lmin),
                    (T)nonlin_dev<MODEL>((float)z.y, c1, c2, inv, inv_d, a.clamp, mphi_rel, lmin));
      }
    } else {
      double lo = INFINITY, hi = -INFINITY;
      for (int j = lt; j < m; j += tpf) {
        const cplx<T> z = buf[j];
        if (valid) {
          lo = fmin(lo, fmin((double)z.x, (double)z.y));
          hi = fmax(hi, fmax((double)z.x, (double)z.y));
        }
        buf[j] = mk((T)nonlin_plain<MODEL>((double)z.x, a.g, a.clamp, a.min_phi, a.min_log),
                    (T)nonlin_plain<MODEL>((double)z.y, a.g, a.clamp, a.min_phi, a.min_log));
      }
      if (a.minmax) block_minmax_store(lo, hi, a.minmax + 2 * blockIdx.x);
    }
    __syncthreads();
  }

  if (MODE == kRowStep || MODE == kRowForward) {
    fft_run<false, RSET>(buf, a.fft, a.tw, lt, tpf);
    // post-process pairs (k, m-k) of the forward real transform
    for (int k = lt; k <= m / 2; k += tpf) {
      if (k == 0) {
        const cplx<T> z = buf[0];
        buf[0] = mk(z.x + z.y, z.x - z.y);
      } else {
        const int kk = m - k;
        const cplx<T> zk = buf[k], zm = buf[kk];
        const cplx<T> e = T(0.5) * (zk + conj(zm));
        const cplx<T> o = T(0.5) * rot4<false>(zk - conj(zm));
        const cplx<T> t = cmul(a.rtw[k], o);
        buf[k] = e + t;
        if (kk != k) buf[kk] = conj(e - t);
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < rows * m; i += blockDim.x) {
      const int r = i % rows, kx = i / rows;
      if (y0 + r < ny) a_out[(size_t)kx * ny + (y0 + r)] = sm[r * ld + generic_pad(kx)];
    }
    return;
  }

  if (MODE == kRowMaterialize) {
    const double add = a.add ? *a.add : 0.0;
    KSum acc[1] = {{0.0, 0.0}};
    if (valid) {
      double2* dst = reinterpret_cast<double2*>(a.out_real + (size_t)y * a.nx);
      for (int j = lt; j < m; j += tpf) {
        const cplx<T> z = buf[j];
        dst[j] = make_double2(add + (double)z.x, add + (double)z.y);
        ksum_add(acc[0], (double)z.x);
        ksum_add(acc[0], (double)z.y);
      }
    }
    if (a.partials) block_reduce_store<1>(acc, a.partials + 2 * blockIdx.x);
    return;
  }

  if (MODE == kRowReduce) {
    // sums of: raw value (mean), free-energy polynomial, nonlinear mu
    const double mean = dev ? a_scal[kScalMean] : 0.0;
    const double eps = a.epsilon, g = a.g;
    KSum acc[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    if (valid) {
      for (int j = lt; j < m; j += tpf) {
        const cplx<T> z = buf[j];
        const double vv[2] = {(double)z.x, (double)z.y};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const double n = mean + vv[h];
          const double n2 = n * n;
          double fpoly = (eps / 2.0) * n2 + (g / 3.0) * (n2 * n) + (1 / 4.0) * (n2 * n2);
          double nl = g * n2 + n2 * n;
          if (MODEL == kModelLog) {
            const double ln = (a.clamp && !(n > a.min_phi)) ? a.min_log : log(n);
            fpoly = n * log(n) + fpoly;
            nl += ln;
          }
          ksum_add(acc[0], vv[h]);
          ksum_add(acc[1], fpoly);
          ksum_add(acc[2], nl);
        }
      }
    }
    block_reduce_store<3>(acc, a.partials + 6 * blockIdx.x);
  }
}

// ---------------------------------------------------------------- column kernel
template <class T>
__device__ __forceinline__ void unpack_pair(cplx<T> pk, cplx<T> pkp, cplx<T>& h0, cplx<T>& hm) {
  h0 = T(0.5) * (pk + conj(pkp));
  hm = T(0.5) * rot4<false>(pk - conj(pkp));
}

// cols transforms of length ny per CTA, tpf threads each; smem = cols * ld complex.
template <class T, int MODE, int RSET, int LB = 256, int MINB = 1>
__global__ void __launch_bounds__(LB, MINB) col_kernel(ColArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* sm = reinterpret_cast<cplx<T>*>(smem_raw);
  const int ny = a.ny, m = a.m, cols = a.cols, tpf = a.tpf, ld = a.ld, nyh = a.nyh;
  const int c0 = blockIdx.x * cols;
  const int f = threadIdx.x / tpf, lt = threadIdx.x - f * tpf;
  const int kx = c0 + f;
  const bool valid = kx < m;
  const PadBuf<T> buf{sm + f * ld};   // padded exchange buffer of this transform
  // per-plan buffers: this plan's, or in a batched step launch plan blockIdx.y's
  const cplx<T>* a_in = a.in;
  const void* a_nin = a.nin;
  const cplx<float>* a_nin_lo = a.nin_lo;
  void* a_nout = a.nout;
  cplx<float>* a_nout_lo = a.nout_lo;
  cplx<T>* a_wout = a.wout;
  const cplx<T>* a_coef = a.coef;
  const cplx<double>* a_coef64 = a.coef64;
  if (a.batch) {
    const BatchBufs& bb = a.batch[blockIdx.y];
    a_in = static_cast<const cplx<T>*>(bb.v);
    a_nin = bb.nin;
    a_nin_lo = static_cast<const cplx<float>*>(bb.nin_lo);
    a_nout = bb.nout;
    a_nout_lo = static_cast<cplx<float>*>(bb.nout_lo);
    a_wout = static_cast<cplx<T>*>(const_cast<void*>(bb.w));
    a_coef = static_cast<const cplx<T>*>(bb.coef);
    a_coef64 = static_cast<const cplx<double>*>(bb.coef64);
  }

  if (MODE == kColParseval || MODE == kColExport) {
    // no transform: direct pass over n_hat
    KSum acc[1] = {{0.0, 0.0}};
    if (valid) {
      const size_t cb = (size_t)kx * ny;
      for (int ky = lt; ky < ny; ky += tpf) {
        const int kyp = ky == 0 ? 0 : ny - ky;
        if (kx == 0) {
          cplx<double> h0, hm;
          unpack_pair(state_ld<T>(a.sin, a.sin_lo, cb + ky, true), state_ld<T>(a.sin, a.sin_lo, cb + kyp, true), h0, hm);
          if (MODE == kColParseval) {
            const double k0 = ksq(0, ky, ny, a.fx, a.fy), kM = ksq(m, ky, ny, a.fx, a.fy);
            const double l0 = (a.beta / 2.0) * (a.q0 * a.q0 - k0) * (a.q0 * a.q0 - k0);
            const double lM = (a.beta / 2.0) * (a.q0 * a.q0 - kM) * (a.q0 * a.q0 - kM);
            ksum_add(acc[0], l0 * ((double)h0.x * h0.x + (double)h0.y * h0.y));
            ksum_add(acc[0], lM * ((double)hm.x * hm.x + (double)hm.y * hm.y));
          } else {
            double* o = a.out_c128 + 2 * ((size_t)ky * (m + 1));
            double dc = 0.0;
            if (a.dev_form && ky == 0) dc = a.scal[kScalMean] * ((double)a.nx * (double)a.ny);
            o[0] = (double)h0.x + dc; o[1] = h0.y;
            o[2 * m] = hm.x; o[2 * m + 1] = hm.y;
          }
        } else {
          const cplx<double> v = state_ld<T>(a.sin, a.sin_lo, cb + ky, true);
          if (MODE == kColParseval) {
            const double k2 = ksq(kx, ky, ny, a.fx, a.fy);
            const double l = (a.beta / 2.0) * (a.q0 * a.q0 - k2) * (a.q0 * a.q0 - k2);
            ksum_add(acc[0], 2.0 * l * ((double)v.x * v.x + (double)v.y * v.y));
          } else {
            double* o = a.out_c128 + 2 * ((size_t)ky * (m + 1) + kx);
            o[0] = v.x; o[1] = v.y;
          }
        }
      }
    }
    if (MODE == kColParseval) block_reduce_store<1>(acc, a.partials + 2 * blockIdx.x);
    return;
  }

  const bool need_v = !(MODE == kColCombine && a.combine == kCombineLocalN);
  if (need_v) {
    // contiguous columns c0 .. c0+cols-1
    for (int i = threadIdx.x; i < cols * ny; i += blockDim.x) {
      const int c = i / ny, ky = i - c * ny;
      cplx<T> v = mk(T(0), T(0));
      if (c0 + c < m) v = a_in[(size_t)c0 * ny + i];
      sm[c * ld + generic_pad(ky)] = v;
    }
    __syncthreads();
    fft_run<false, RSET>(buf, a.fft, a.tw, lt, tpf);
  }

  if (MODE == kColInit) {
    if (valid) {
      const size_t cb = (size_t)kx * ny;
      for (int ky = lt; ky < ny; ky += tpf) {
        cplx<T> v = buf[ky];
        if (a.dev_form && kx == 0 && ky == 0) { v.x = T(0); buf[0] = v; }
        state_st<T>(a_nout, a_nout_lo, cb + ky, mk((double)v.x, (double)v.y), true);   // lo = 0
      }
    }
    __syncthreads();
  } else if (MODE == kColStep) {
    if (valid && kx == 0) {
      const size_t cb = 0;
      for (int ky = lt; ky <= ny / 2; ky += tpf) {
        const int kyp = ky == 0 ? 0 : ny - ky;
        const cplx<T> qkt = buf[ky], qkpt = buf[kyp];
        const cplx<double> qk = mk((double)qkt.x, (double)qkt.y), qkp = mk((double)qkpt.x, (double)qkpt.y);
        // the packed column holds kx = 0 (slow near ky = 0): always at full precision
        bool s0, sM;
        const cplx<double> c0v = coef_ld<T>(a_coef, a_coef64, ky, a.slow_tau, true, s0);
        const cplx<double> cMv = coef_ld<T>(a_coef, a_coef64, (size_t)m * nyh + ky, a.slow_tau, true, sM);
        const cplx<double> pk = state_ld<T>(a_nin, a_nin_lo, cb + ky, true);
        const cplx<double> pkp = state_ld<T>(a_nin, a_nin_lo, cb + kyp, true);
        cplx<double> h0, hm, g0, gm;
        unpack_pair(pk, pkp, h0, hm);
        unpack_pair(qk, qkp, g0, gm);
        cplx<double> h0n = h0 + c0v.x * h0 + c0v.y * g0;
        cplx<double> hmn = hm + cMv.x * hm + cMv.y * gm;
        if (a.forcing) {
          h0n = h0n + a.forcing[ky];
          hmn = hmn + a.forcing[(size_t)m * ny + ky];
        }
        const cplx<double> ok = h0n + mul_i(hmn);
        const cplx<double> okp = conj(h0n) + mul_i(conj(hmn));
        state_st<T>(a_nout, a_nout_lo, cb + ky, ok, true);
        buf[ky] = mk((T)ok.x, (T)ok.y);
        if (kyp != ky) {
          state_st<T>(a_nout, a_nout_lo, cb + kyp, okp, true);
          buf[kyp] = mk((T)okp.x, (T)okp.y);
        }
      }
    } else if (valid) {
      // (ky, -ky) pairs in chunks of two, the coefficients and states of a chunk loaded
      // before any of its results is stored (the compiler keeps a later pair's loads
      // behind an earlier pair's stores); arithmetic as coef_ld / state_ld / state_st
      constexpr int CH = 2;
      const size_t cb = (size_t)kx * ny;
      const cplx<T>* nin = static_cast<const cplx<T>*>(a_nin);
      for (int ky0 = lt; ky0 <= ny / 2; ky0 += CH * tpf) {
        cplx<T> cw[CH], ph[CH], pph[CH];
#pragma unroll
        for (int j = 0; j < CH; ++j) {
          const int ky = ky0 + j * tpf;
          if (ky <= ny / 2) {
            const int kyp = ky == 0 ? 0 : ny - ky;
            cw[j] = a_coef[(size_t)kx * nyh + ky];
            ph[j] = nin[cb + ky];
            pph[j] = nin[cb + kyp];
          }
        }
#pragma unroll
        for (int j = 0; j < CH; ++j) {
          const int ky = ky0 + j * tpf;
          if (ky > ny / 2) break;
          const int kyp = ky == 0 ? 0 : ny - ky;
          const cplx<T> qkt = buf[ky], qkpt = buf[kyp];
          const cplx<double> qk = mk((double)qkt.x, (double)qkt.y), qkp = mk((double)qkpt.x, (double)qkpt.y);
          const bool slow = sizeof(T) == 8 || fabs((double)cw[j].x) < (double)a.slow_tau;
          const cplx<double> c = (sizeof(T) == 4 && slow) ? a_coef64[(size_t)kx * nyh + ky]
                                                           : mk((double)cw[j].x, (double)cw[j].y);
          cplx<double> pk = mk((double)ph[j].x, (double)ph[j].y), pkp = mk((double)pph[j].x, (double)pph[j].y);
          if (sizeof(T) == 4 && slow) {
            const cplx<float> l = a_nin_lo[cb + ky], lp = a_nin_lo[cb + kyp];
            pk.x += (double)l.x;
            pk.y += (double)l.y;
            pkp.x += (double)lp.x;
            pkp.y += (double)lp.y;
          }
          cplx<double> ok = pk + c.x * pk + c.y * qk;
          cplx<double> okp = pkp + c.x * pkp + c.y * qkp;
          if (a.forcing) {
            ok = ok + a.forcing[cb + ky];
            okp = okp + a.forcing[cb + kyp];
          }
          state_st<T>(a_nout, a_nout_lo, cb + ky, ok, slow);
          buf[ky] = mk((T)ok.x, (T)ok.y);
          if (kyp != ky) {
            state_st<T>(a_nout, a_nout_lo, cb + kyp, okp, slow);
            buf[kyp] = mk((T)okp.x, (T)okp.y);
          }
        }
      }
    }
    __syncthreads();
  } else if (MODE == kColCombine) {
    // mu_hat = L_mu n_hat + N_hat (optionally Gaussian-filtered), or G n_hat, or N_hat
    if (valid) {
      const size_t cb = (size_t)kx * ny;
      const double q2 = a.q0 * a.q0;
      for (int ky = lt; ky <= ny / 2; ky += tpf) {
        const int kyp = ky == 0 ? 0 : ny - ky;
        // multipliers for n_hat and N_hat at (kx, ky) and, for the packed column, (m, ky)
        double mn[2], mq[2];
        for (int h = 0; h < (kx == 0 ? 2 : 1); ++h) {
          const int kxx = (h == 0) ? kx : m;
          const double k2 = ksq(kxx, ky, ny, a.fx, a.fy);
          const double lmu = a.beta * (q2 - k2) * (q2 - k2) + a.epsilon;
          const double gs = exp(-k2 * a.w * a.w / 2);
          switch (a.combine) {
            case kCombineMu: mn[h] = lmu; mq[h] = 1.0; break;
            case kCombineLocalMu: mn[h] = gs * lmu; mq[h] = gs; break;
            case kCombineLocalN: mn[h] = gs; mq[h] = 0.0; break;
            case kCombineNonlin: mn[h] = 0.0; mq[h] = 1.0; break;
            default: mn[h] = 1.0; mq[h] = 0.0; break;
          }
        }
        const cplx<double> pk = state_ld<T>(a_nin, a_nin_lo, cb + ky, true);
        const cplx<double> pkp = state_ld<T>(a_nin, a_nin_lo, cb + kyp, true);
        cplx<double> qk = mk(0.0, 0.0), qkp = qk;
        if (need_v) {
          qk = mk((double)buf[ky].x, (double)buf[ky].y);
          qkp = mk((double)buf[kyp].x, (double)buf[kyp].y);
        }
        cplx<double> ok, okp;
        if (kx == 0) {
          cplx<double> h0, hm, g0, gm;
          unpack_pair(pk, pkp, h0, hm);
          unpack_pair(qk, qkp, g0, gm);
          const cplx<double> h0n = mn[0] * h0 + mq[0] * g0;
          const cplx<double> hmn = mn[1] * hm + mq[1] * gm;
          ok = h0n + mul_i(hmn);
          okp = conj(h0n) + mul_i(conj(hmn));
        } else {
          ok = mn[0] * pk + mq[0] * qk;
          okp = mn[0] * pkp + mq[0] * qkp;
        }
        buf[ky] = mk((T)ok.x, (T)ok.y);
        if (kyp != ky) buf[kyp] = mk((T)okp.x, (T)okp.y);
      }
    }
    __syncthreads();
  }

  fft_run<true, RSET>(buf, a.fft, a.tw, lt, tpf);
  const T s = (T)a.scale;
  for (int i = threadIdx.x; i < cols * ny; i += blockDim.x) {
    const int c = i / ny, ky = i - c * ny;
    if (c0 + c < m) {
      const cplx<T> v = sm[c * ld + generic_pad(ky)];
      a_wout[(size_t)c0 * ny + i] = mk(s * v.x, s * v.y);
    }
  }
}

}  // namespace pfc
