// Whole-grid step kernel for small FP64 mixed-radix plans (the phase-diagram cells,
// e.g. 28 x 24 or 32 x 56 sites).
//
// On such grids the two-kernel step (row pass, column pass) is bound by launch and
// barrier latency, not by HBM: a 28 x 24 step takes about 20 us while it moves 20 KB. Here
// one CTA holds one plan's whole grid in shared memory (the row buffers, the column
// buffers and the spectral state) and runs `nsteps` steps in a loop, so a block of steps
// is one launch; a batch of plans is one launch with one CTA per plan.
//
// Each step runs the same device functions, with the same arguments and in the same order,
// as row_kernel<kRowStep> followed by col_kernel<kColStep> (pfc_kernels.cuh): the packed
// inverse real transform of the rows, the nonlinearity, the forward real transform, the
// column transform, the ETD1 update n_hat' = n_hat + (A - 1) n_hat + Bg N_hat and the
// inverse column transform. On the last step of a launch it leaves in global memory what
// the two-kernel step leaves: V (the nonlinear spectrum of the state the step started
// from), that state, the new state and W (the new state's inverse column transforms).
#include "pfc_kernels.cuh"
#include "pfc_registry.h"

namespace pfc {

namespace {

// One Stockham pass from src to dst with one butterfly per thread at a time: the loads,
// twiddles, DFT and output positions of stockham_pass (pfc_fft.cuh), out of place, so a
// thread holds R values instead of all its butterflies and the pass needs one barrier.
template <int R, bool INV>
__device__ __forceinline__ void pass_oop(PadBuf<double> src, PadBuf<double> dst, int n, int ns,
                                         const cplx<double>* __restrict__ tw, const cplx<double>* __restrict__ roots,
                                         int lt, int tpf) {
  const int nr = n / R;
  for (int j = lt; j < nr; j += tpf) {
    cplx<double> v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = src[j + q * nr];
    const int k = j % ns;
    if (k != 0) {
      const cplx<double>* w = tw + k;   // table [q - 1][k]
#pragma unroll
      for (int q = 1; q < R; ++q) {
        cplx<double> t = w[(q - 1) * ns];
        if (INV) t.y = -t.y;
        v[q] = cmul(v[q], t);
      }
    }
    dft<R, INV>(v, roots);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int q = 0; q < R; ++q) dst[base + q * ns] = v[q];
  }
  __syncthreads();
}

// Every pass of d, alternating between buffers a and b (every thread of the CTA calls
// this); the result is in b when the pass count is odd, else in a. Out of line: the step
// calls each direction twice, and one copy of the butterflies per direction keeps the
// kernel's code small enough for the instruction cache.
template <bool INV, int RSET>
__device__ __noinline__ void fft_oop(PadBuf<double> a, PadBuf<double> b, const FftDesc& d,
                                        const cplx<double>* __restrict__ twbase, int lt, int tpf) {
  PadBuf<double> src = a, dst = b;
  for (int p = 0; p < d.npass; ++p) {
    const cplx<double>* tw = twbase + d.twoff[p];
    const cplx<double>* roots = d.rootoff[p] >= 0 ? twbase + d.rootoff[p] : nullptr;
    const int ns = d.ns[p];
    switch (d.radix[p]) {
      case 2: pass_oop<2, INV>(src, dst, d.n, ns, tw, roots, lt, tpf); break;
      case 4: pass_oop<4, INV>(src, dst, d.n, ns, tw, roots, lt, tpf); break;
      case 8: pass_oop<8, INV>(src, dst, d.n, ns, tw, roots, lt, tpf); break;
      case 16: pass_oop<16, INV>(src, dst, d.n, ns, tw, roots, lt, tpf); break;
      default:
        if constexpr (RSET != kRadixPow2) {
          switch (d.radix[p]) {
            case 3: pass_oop<3, INV>(src, dst, d.n, ns, tw, roots, lt, tpf); break;
            case 5: pass_oop<5, INV>(src, dst, d.n, ns, tw, roots, lt, tpf); break;
            case 7: pass_oop<7, INV>(src, dst, d.n, ns, tw, roots, lt, tpf); break;
            default:
              if constexpr (RSET == kRadixAll) {
                if (d.radix[p] == 11) pass_oop<11, INV>(src, dst, d.n, ns, tw, roots, lt, tpf);
                else if (d.radix[p] == 13) pass_oop<13, INV>(src, dst, d.n, ns, tw, roots, lt, tpf);
              }
              break;
          }
        }
        break;
    }
    const PadBuf<double> t = src;
    src = dst;
    dst = t;
  }
}

// MINB 1: all registers for one CTA per SM (single plans, small batches); MINB 2: two
// CTAs per SM (batches with more plans than SMs; a few spilled values).
template <int MODEL, int RSET, int MINB>
__global__ void __launch_bounds__(kOneCtaMaxThreads, MINB) onecta_step_kernel(RowArgs<double> ra, ColArgs<double> ca,
                                                                         const BatchBufs* table, long long nsteps) {
  using T = double;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int m = ra.m, ny = ra.ny, ldr = ra.ld, ldc = ca.ld, nyh = ca.nyh;
  const int spec = m * ny;
  cplx<T>* R = reinterpret_cast<cplx<T>*>(smem_raw);   // ny row buffers of ldr
  cplx<T>* R2 = R + (size_t)ny * ldr;                     // their pass partners
  cplx<T>* C = R2 + (size_t)ny * ldr;                     // m column buffers of ldc
  cplx<T>* C2 = C + (size_t)m * ldc;                      // their pass partners
  cplx<T>* S = C2 + (size_t)m * ldc;                      // n_hat, packed [kx][y]
  const BatchBufs& bb = table[blockIdx.x];
  cplx<T>* W = static_cast<cplx<T>*>(const_cast<void*>(bb.w));
  cplx<T>* V = static_cast<cplx<T>*>(bb.v);
  cplx<T>* P[2] = {static_cast<cplx<T>*>(const_cast<void*>(bb.nin)), static_cast<cplx<T>*>(bb.nout)};
  const cplx<T>* coef = static_cast<const cplx<T>*>(bb.coef);
  const int tid = threadIdx.x, nth = blockDim.x;

  for (int i = tid; i < spec; i += nth) {
    const int kx = i / ny, y = i - kx * ny;
    C[kx * ldc + generic_pad(y)] = W[i];
    S[i] = P[0][i];
  }
  // Roles: thread tid works on row tid / tpf_r and on column tid / tpf_c. A thread
  // without a row (or column) gets a lane index past every butterfly and pair loop, so
  // it touches no buffer there but still reaches every barrier of the transforms.
  const int tr = ra.tpf, tc = ca.tpf;
  const int fr = tid / tr, fc = tid / tc;
  const bool row_on = fr < ny, col_on = fc < m;
  constexpr int kIdle = 1 << 20;
  const int ltr = row_on ? tid - fr * tr : kIdle;
  const int ltc = col_on ? tid - fc * tc : kIdle;
  const PadBuf<T> rbuf{R + (size_t)(row_on ? fr : 0) * ldr}, rbuf2{R2 + (size_t)(row_on ? fr : 0) * ldr};
  const PadBuf<T> cbuf{C + (size_t)(col_on ? fc : 0) * ldc}, cbuf2{C2 + (size_t)(col_on ? fc : 0) * ldc};
  const int kx = col_on ? fc : 0;
  const T s = (T)ca.scale;
  const FftDesc& rfft = ra.fft;
  const FftDesc& cfft = ca.fft;
  // where a transform's result lands: the partner buffer after an odd pass count; an
  // inverse and a forward transform together always end in the main buffer
  const PadBuf<T> xr = (rfft.npass & 1) ? rbuf2 : rbuf, xr2 = (rfft.npass & 1) ? rbuf : rbuf2;
  const PadBuf<T> xc = (cfft.npass & 1) ? cbuf2 : cbuf, xc2 = (cfft.npass & 1) ? cbuf : cbuf2;
  __syncthreads();

  for (long long step = 0; step < nsteps; ++step) {
    const bool last = step == nsteps - 1;
    // ---- row pass (row_kernel<kRowStep>)
    for (int i = tid; i < spec; i += nth) {
      const int c = i / ny, y = i - c * ny;
      R[y * ldr + generic_pad(c)] = C[c * ldc + generic_pad(y)];
    }
    __syncthreads();
    for (int k = ltr; k <= m / 2; k += tr) {
      if (k == 0) {
        const cplx<T> p = rbuf[0];
        rbuf[0] = mk(p.x + p.y, p.x - p.y);
      } else {
        const int kk = m - k;
        const cplx<T> xk = rbuf[k], xm = rbuf[kk];
        const cplx<T> sm = xk + conj(xm), d = xk - conj(xm);
        const cplx<T> u = mul_i(cmul(conj(ra.rtw[k]), d));
        rbuf[k] = sm + u;
        if (kk != k) rbuf[kk] = conj(sm - u);
      }
    }
    __syncthreads();
    fft_oop<true, RSET>(rbuf, rbuf2, rfft, ra.tw, ltr, tr);
    for (int j = ltr; j < m; j += tr) {
      const cplx<T> z = xr[j];
      xr[j] = mk((T)nonlin_plain<MODEL>((double)z.x, ra.g, ra.clamp, ra.min_phi, ra.min_log),
                   (T)nonlin_plain<MODEL>((double)z.y, ra.g, ra.clamp, ra.min_phi, ra.min_log));
    }
    __syncthreads();
    fft_oop<false, RSET>(xr, xr2, rfft, ra.tw, ltr, tr);
    for (int k = ltr; k <= m / 2; k += tr) {
      if (k == 0) {
        const cplx<T> z = rbuf[0];
        rbuf[0] = mk(z.x + z.y, z.x - z.y);
      } else {
        const int kk = m - k;
        const cplx<T> zk = rbuf[k], zm = rbuf[kk];
        const cplx<T> e = T(0.5) * (zk + conj(zm));
        const cplx<T> o = T(0.5) * rot4<false>(zk - conj(zm));
        const cplx<T> t = cmul(ra.rtw[k], o);
        rbuf[k] = e + t;
        if (kk != k) rbuf[kk] = conj(e - t);
      }
    }
    __syncthreads();
    // ---- column pass (col_kernel<kColStep>)
    for (int i = tid; i < spec; i += nth) {
      const int c = i / ny, y = i - c * ny;
      const cplx<T> v = R[y * ldr + generic_pad(c)];
      C[c * ldc + generic_pad(y)] = v;
      if (last) V[i] = v;
    }
    if (last)   // the state this step starts from, in its ping-pong buffer
      for (int i = tid; i < spec; i += nth) P[step & 1][i] = S[i];
    __syncthreads();
    fft_oop<false, RSET>(cbuf, cbuf2, cfft, ca.tw, ltc, tc);
    if (col_on && kx == 0) {
      for (int ky = ltc; ky <= ny / 2; ky += tc) {
        const int kyp = ky == 0 ? 0 : ny - ky;
        const cplx<T> qkt = xc[ky], qkpt = xc[kyp];
        const cplx<double> qk = mk((double)qkt.x, (double)qkt.y), qkp = mk((double)qkpt.x, (double)qkpt.y);
        const cplx<double> c0v = coef[ky];
        const cplx<double> cMv = coef[(size_t)m * nyh + ky];
        const cplx<double> pk = S[ky];
        const cplx<double> pkp = S[kyp];
        cplx<double> h0, hm, g0, gm;
        unpack_pair(pk, pkp, h0, hm);
        unpack_pair(qk, qkp, g0, gm);
        const cplx<double> h0n = h0 + c0v.x * h0 + c0v.y * g0;
        const cplx<double> hmn = hm + cMv.x * hm + cMv.y * gm;
        const cplx<double> ok = h0n + mul_i(hmn);
        const cplx<double> okp = conj(h0n) + mul_i(conj(hmn));
        S[ky] = ok;
        xc[ky] = mk((T)ok.x, (T)ok.y);
        if (kyp != ky) {
          S[kyp] = okp;
          xc[kyp] = mk((T)okp.x, (T)okp.y);
        }
      }
    } else if (col_on) {
      const size_t cb = (size_t)kx * ny;
      for (int ky = ltc; ky <= ny / 2; ky += tc) {
        const int kyp = ky == 0 ? 0 : ny - ky;
        const cplx<T> cw = coef[(size_t)kx * nyh + ky];
        const cplx<T> ph = S[cb + ky], pph = S[cb + kyp];
        const cplx<T> qkt = xc[ky], qkpt = xc[kyp];
        const cplx<double> qk = mk((double)qkt.x, (double)qkt.y), qkp = mk((double)qkpt.x, (double)qkpt.y);
        const cplx<double> c = mk((double)cw.x, (double)cw.y);
        const cplx<double> pk = mk((double)ph.x, (double)ph.y), pkp = mk((double)pph.x, (double)pph.y);
        const cplx<double> ok = pk + c.x * pk + c.y * qk;
        const cplx<double> okp = pkp + c.x * pkp + c.y * qkp;
        S[cb + ky] = ok;
        xc[ky] = mk((T)ok.x, (T)ok.y);
        if (kyp != ky) {
          S[cb + kyp] = okp;
          xc[kyp] = mk((T)okp.x, (T)okp.y);
        }
      }
    }
    __syncthreads();
    fft_oop<true, RSET>(xc, xc2, cfft, ca.tw, ltc, tc);
    for (int ky = ltc; ky < ny; ky += tc) {
      const cplx<T> v = cbuf[ky];
      cbuf[ky] = mk(s * v.x, s * v.y);
    }
    __syncthreads();
    if (last) {
      for (int i = tid; i < spec; i += nth) {
        const int c = i / ny, y = i - c * ny;
        P[(step + 1) & 1][i] = S[i];
        W[i] = C[c * ldc + generic_pad(y)];
      }
    }
  }
}

template <int MODEL, int MINB>
void* pick_minb(int rset) {
  switch (rset) {
    case kRadixPow2: return (void*)onecta_step_kernel<MODEL, kRadixPow2, MINB>;
    case kRadixSmall: return (void*)onecta_step_kernel<MODEL, kRadixSmall, MINB>;
    case kRadixAll: return (void*)onecta_step_kernel<MODEL, kRadixAll, MINB>;
    default: return nullptr;
  }
}

template <int MODEL>
void* pick(int rset, bool dense) {
  return dense ? pick_minb<MODEL, 2>(rset) : pick_minb<MODEL, 1>(rset);
}

}  // namespace

size_t onecta_smem_bytes(int m, int ny, int row_ld, int col_ld) {
  return (2 * (size_t)ny * row_ld + 2 * (size_t)m * col_ld + (size_t)m * ny) * sizeof(cplx<double>);
}

cudaError_t onecta_allow_smem(size_t bytes) {
  for (int model : {kModelStd, kModelLog})
    for (int rset : {kRadixPow2, kRadixSmall, kRadixAll})
      for (bool dense : {false, true}) {
        void* fn = model == kModelLog ? pick<kModelLog>(rset, dense) : pick<kModelStd>(rset, dense);
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
      }
  return cudaSuccess;
}

bool onecta_supported(int rset) { return rset == kRadixPow2 || rset == kRadixSmall || rset == kRadixAll; }

cudaError_t launch_onecta_step(const RowArgs<double>& ra, const ColArgs<double>& ca, const BatchBufs* table,
                               int count, long long nsteps, int model, int rset, bool dense, int threads,
                               size_t smem, cudaStream_t stream) {
  void* fn = model == kModelLog ? pick<kModelLog>(rset, dense) : pick<kModelStd>(rset, dense);
  if (!fn) return cudaErrorInvalidValue;
  RowArgs<double> r = ra;
  ColArgs<double> c = ca;
  void* args[] = {(void*)&r, (void*)&c, (void*)&table, (void*)&nsteps};
  return cudaLaunchKernel(fn, dim3(count), dim3(threads), args, smem, stream);
}

}  // namespace pfc
