// Two-lane packed FP32 step kernels for power-of-two grids (FP32-mixed form).
//
// The same step as row_step_fast / col_step_fast (pfc_fast.cuh), with the same buffers
// and layouts, but every thread advances two independent transforms at once in the
// two lanes of packed f32x2 instructions (pfc_pack.cuh): the row kernel pairs rows
// y0 + 2p and y0 + 2p + 1, the column kernel pairs columns 2c and 2c + 1. The butterflies,
// twiddle products, real-packing twiddles and the nonlinearity of two transforms then
// cost the issue slots of one, which is what bounded the one-lane kernels (about 139
// instructions per complex value in the row pass).
//
// Transforms: radix-16 Stockham passes (FastSeq with radix cap 16), sequence A then B
// with the last pass of A and the first of B in the same registers, as in pfc_fast.cuh.
// Exchange buffers hold one 16-byte `pc` per index, padded one slot per 16 (the Stockham
// stores of a radix-16 pass then hit distinct bank groups per quarter warp).
// Pass twiddles are float4 (c, c, s, s) tables, [q-1][k] per pass, s = sin of the
// forward angle; inverse passes conjugate them.
#pragma once
#include <cuda.h>

#include "pfc_fast.cuh"
#include "pfc_pack.cuh"

namespace pfc {

constexpr int kPkPad = 4;  // one pad slot per 16 pc slots

template <int N, int EE_REQ> using PkSeq = FastSeq<N, EE_REQ, 16>;

__device__ __forceinline__ pc pk_ld(const float4* p) {
  const float4 v = *p;
  return mkpc(make_float2(v.x, v.y), make_float2(v.z, v.w));
}
__device__ __forceinline__ void pk_st(float4* p, pc v) { *p = make_float4(v.r.x, v.r.y, v.i.x, v.i.y); }

// v * w (forward) or v * conj(w) (inverse), w = (c, s) broadcast to both lanes as (C, S)
template <bool INV>
__device__ __forceinline__ pc pk_tw(pc v, float2 C, float2 S) {
  if (INV) return mkpc(fma2(v.i, S, mul2(v.r, C)), sub2(mul2(v.i, C), mul2(v.r, S)));
  return mkpc(sub2(mul2(v.r, C), mul2(v.i, S)), fma2(v.r, S, mul2(v.i, C)));
}

template <int N, int EE, int R, int NS>
struct PkPass {
  static constexpr int P = kPkPad;
  static_assert(R <= (1 << P), "a butterfly's consecutive outputs must not straddle a pad");
  static constexpr int TPF = N / EE, NB = EE / R, NR = N / R;
  static constexpr int NRP = NR + (NR >> P);
  static constexpr bool LIN_LOAD = (NR % (1 << P)) == 0;
  static constexpr bool LIN_STORE = (NS % (1 << P)) == 0 || NS == 1;
  static constexpr int NSP = NS == 1 ? 1 : NS + (NS >> P);
  static __device__ __forceinline__ void load(const float4* buf, pc* v, int t) {
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const int j = t + b * TPF;
      if constexpr (LIN_LOAD) {
        const float4* p = buf + padi<P>(j);
#pragma unroll
        for (int q = 0; q < R; ++q) v[b * R + q] = pk_ld(p + q * NRP);
      } else {
#pragma unroll
        for (int q = 0; q < R; ++q) v[b * R + q] = pk_ld(buf + padi<P>(j + q * NR));
      }
    }
  }
  template <bool INV>
  static __device__ __forceinline__ void compute(pc* v, int t, const float4* __restrict__ tw) {
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      if constexpr (NS > 1) {
        const int j = t + b * TPF;
        const int k = j % NS;   // NS need not be a power of two (mixed sequences)
        const float4* w = tw + k;
        float4 wq[R];
#pragma unroll
        for (int q = 1; q < R; ++q) wq[q] = ld_keep(w + (q - 1) * NS);
#pragma unroll
        for (int q = 1; q < R; ++q)
          v[b * R + q] = pk_tw<INV>(v[b * R + q], make_float2(wq[q].x, wq[q].y), make_float2(wq[q].z, wq[q].w));
      }
      pdft<R, INV>(v + b * R);
    }
  }
  static __device__ __forceinline__ void store(float4* buf, const pc* v, int t) {
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const int j = t + b * TPF;
      const int k = j % NS;   // NS need not be a power of two (mixed sequences)
      const int base = (j - k) * R + k;
      if constexpr (LIN_STORE) {
        float4* p = buf + padi<P>(base);
#pragma unroll
        for (int q = 0; q < R; ++q) pk_st(p + q * NSP, v[b * R + q]);
      } else {
#pragma unroll
        for (int q = 0; q < R; ++q) pk_st(buf + padi<P>(base + q * NS), v[b * R + q]);
      }
    }
  }
  static __device__ __forceinline__ int out_index(int t, int b, int q) { return t + b * TPF + q * NR; }
};

// Middle passes [PA, PB) of sequence A (SEQB = false) or B, in place through buf.
template <int N, int EE_REQ, bool SEQB, bool INV, int PA, int PB>
__device__ __forceinline__ void pk_mid(float4* buf, pc* v, int t, int g, const float4* __restrict__ tw) {
  if constexpr (PA < PB) {
    using S = PkSeq<N, EE_REQ>;
    constexpr int R = SEQB ? S::radB(PA) : S::radA(PA);
    constexpr int NS = SEQB ? S::nsB(PA) : S::nsA(PA);
    constexpr int OFF = SEQB ? S::twB(PA) : S::twA(PA);
    using PS = PkPass<N, S::EE, R, NS>;
    PS::load(buf, v, t);
    group_sync<S::TPF>(g);
    PS::template compute<INV>(v, t, tw + OFF);
    PS::store(buf, v, t);
    group_sync<S::TPF>(g);
    pk_mid<N, EE_REQ, SEQB, INV, PA + 1, PB>(buf, v, t, g, tw);
  }
}

// Raw tile entry (row a: re, im; row b: re, im) <-> two-lane value.
__device__ __forceinline__ pc raw2pc(float4 x) { return mkpc(make_float2(x.x, x.z), make_float2(x.y, x.w)); }
__device__ __forceinline__ float4 pc2raw(pc v) { return make_float4(v.r.x, v.i.x, v.r.y, v.i.y); }

// launch bounds: at least 256 threads (one group if larger); two CTAs per SM (128 registers)
// unless a group alone needs more than 256 threads
template <int TPF> struct PkBound { static constexpr int value = TPF > 256 ? TPF : 256; };
template <int TPF> struct PkMinB { static constexpr int value = TPF > 256 ? 1 : 2; };

// Byte offset of tile entry (p, kx) in a TMA-staged tile: the box lands as [kx][rows]
// (8-byte complex per row, ib = rows * 8 bytes per kx) with the hardware swizzle of its
// inner width, XOR of the 16-byte chunk index (bits 4..) with bits 7.. of the offset
// (smask = 0, 1, 3, 7 for no swizzle, 32-, 64- and 128-byte swizzle; the tile starts on a
// 1024-byte boundary, so the offset's bits are the address bits the hardware uses).
__device__ __forceinline__ unsigned tma_tile_off(int kx, int p, int ib, unsigned smask) {
  const unsigned o = (unsigned)kx * (unsigned)ib + 16u * (unsigned)p;
  return o ^ (((o >> 7) & smask) << 4);
}

constexpr long long kTmaWaitLimit = 1LL << 22;

// ------------------------------------------------------------------ row kernel
// CTA: `rows` consecutive rows (a.rows even), `rows / 2` groups of TPF threads, group p
// owning rows y0 + 2p, y0 + 2p + 1. Entry (p, kx) of the tile is W[kx][y0 + 2p] and
// W[kx][y0 + 2p + 1], the 16 contiguous bytes of the column-major array. The tile is staged
// either by the tensor memory accelerator (a.tma_box > 0: one thread issues
// cp.async.bulk.tensor boxes of rows x tma_box from the tensor map of W, completion counted
// on an mbarrier, swizzled [kx][rows] layout in shared memory), or with 16-byte
// asynchronous copies into a padded [p][kx] layout (consecutive threads take consecutive p
// of one kx: runs of rows * 8 bytes per kx).
template <int M, int EE_REQ, int MODEL>
__global__ void __launch_bounds__(PkBound<PkSeq<M, EE_REQ>::TPF>::value, PkMinB<PkSeq<M, EE_REQ>::TPF>::value)
row_step_pk(FastRowArgs<float> a, const __grid_constant__ CUtensorMap tmap) {
  using S = PkSeq<M, EE_REQ>;
  constexpr int EE = S::EE, TPF = S::TPF, NP = S::NPASS;
  constexpr int P = kPkPad;
  constexpr int LD = M + (M >> P);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // 1024-byte aligned start (the plan requests 1 KB more when it stages with TMA)
  const unsigned raw_s = (unsigned)__cvta_generic_to_shared(smem_raw);
  const unsigned pad_s = a.tma_box ? ((1024u - (raw_s & 1023u)) & 1023u) : 0u;
  float4* sm = reinterpret_cast<float4*>(smem_raw + pad_s);
  const int ny = a.ny, rows = a.rows, pairs = rows >> 1;
  const int y0 = blockIdx.x * rows;
  const int g = threadIdx.x / TPF, t = threadIdx.x - g * TPF;
  const float2* gin = reinterpret_cast<const float2*>(a.in);
  float2* gout = reinterpret_cast<float2*>(a.out);
  const double* scal = a.scal;
  if (a.batch) {
    const BatchBufs& b = a.batch[blockIdx.y];
    gin = static_cast<const float2*>(b.w);
    gout = static_cast<float2*>(b.v);
    scal = b.scal;
  }
  const float4* twA = reinterpret_cast<const float4*>(a.twA);
  const float4* twB = reinterpret_cast<const float4*>(a.twB);
  const float4* rtw = reinterpret_cast<const float4*>(a.rtw);   // (c, c, s, s) of exp(-2 pi i k / nx)

  pdl_wait();
  pdl_trigger();

  // ---- tile load: entry (p, kx) <- 16 bytes at W[kx][y0 + 2p]
  const int tp = threadIdx.x % pairs, kx0 = threadIdx.x / pairs, kstep = blockDim.x / pairs;
  const bool tma = a.tma_box > 0;
  const int ib = rows * 8;
  const unsigned smask = ib >= 128 ? 7u : ib == 64 ? 3u : ib == 32 ? 1u : 0u;
  if (tma) {
    __shared__ __align__(8) unsigned long long tbar;
    const unsigned bar = (unsigned)__cvta_generic_to_shared(&tbar);
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned bytes = (unsigned)M * (unsigned)ib + a.tma_extra_tx;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
      const unsigned base = raw_s + pad_s;
      // x (the innermost coordinate, rows) = y0 is even: 16-byte aligned; kx is the outer one
      for (int kx = 0; kx < M; kx += a.tma_box) {
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
            ::"r"(base + (unsigned)kx * (unsigned)ib), "l"(reinterpret_cast<unsigned long long>(&tmap)), "r"(y0),
              "r"(kx), "r"(bar)
            : "memory");
      }
    }
    unsigned done = 0;
    const long long limit = a.tma_wait_limit > 0 ? a.tma_wait_limit : kTmaWaitLimit;
    for (long long it = 0; !done && it < limit; ++it) {
      asm volatile(
          "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(done)
          : "r"(bar)
          : "memory");
    }
    if (!done) {
      // the barrier did not complete within the limit: report and leave (nothing else reads
      // the tile; the boxes themselves were issued before the wait)
      if (threadIdx.x == 0 && a.err) atomicOr(a.err, (int)kStatusTimeout);
      return;
    }
  } else {
    float4* drow = sm + tp * LD;
    const float2* src = gin + (size_t)kx0 * ny + (y0 + 2 * tp);
    const size_t gstep = (size_t)kstep * ny;
    for (int kx = kx0; kx < M; kx += kstep, src += gstep) {
      const unsigned sdst = (unsigned)__cvta_generic_to_shared(drow + padi<P>(kx));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sdst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
  }

  // nonlinearity parameters (deviation form)
  const float c1 = (float)scal[kScalC1], c2 = (float)scal[kScalC2];
  const float inv = (float)scal[kScalInvMean];
  const double inv_d = scal[kScalInvMean];
  const double mphi_rel = a.min_phi * inv_d;
  const float lmin = (float)scal[kScalLogMin];

  float4* row = sm + g * LD;
  pc v[EE];
  // ---- inverse-real pre-twiddle fused with the first pass's load: element k of this
  // thread's butterflies, Z[k] = S + U, S = X[k] + conj X[M-k], U = i conj(r_k) (X[k] - conj X[M-k]);
  // Z[0] = (X0.re + X0.im, X0.re - X0.im) (DC and Nyquist packed in column 0)
  {
    using P0 = PkPass<M, EE, S::radA(0), 1>;
#pragma unroll
    for (int b = 0; b < P0::NB; ++b)
#pragma unroll
      for (int q = 0; q < S::radA(0); ++q) {
        const int k = t + b * TPF + q * P0::NR;
        const float4* xk = tma ? reinterpret_cast<const float4*>(reinterpret_cast<const char*>(sm) +
                                                                  tma_tile_off(k, g, ib, smask))
                               : row + padi<P>(k);
        const pc x = raw2pc(*xk);
        if (k == 0) {
          v[b * S::radA(0) + q] = mkpc(add2(x.r, x.i), sub2(x.r, x.i));
        } else {
          const float4* xm = tma ? reinterpret_cast<const float4*>(reinterpret_cast<const char*>(sm) +
                                                                    tma_tile_off(M - k, g, ib, smask))
                                 : row + padi<P>(M - k);
          const pc y = raw2pc(*xm);
          const float4 r = ld_keep(rtw + k);
          const float2 C = make_float2(r.x, r.y), Sn = make_float2(r.z, r.w);
          const pc s = mkpc(add2(x.r, y.r), sub2(x.i, y.i));
          const pc d = mkpc(sub2(x.r, y.r), add2(x.i, y.i));
          // U = d * (s_k + i c_k): conj(r_k) = c_k - i s_k, times i
          const pc u = mkpc(sub2(mul2(d.r, Sn), mul2(d.i, C)), fma2(d.i, Sn, mul2(d.r, C)));
          v[b * S::radA(0) + q] = s + u;
        }
      }
  }
  // every partner read of the tile done before the exchange writes (a TMA tile interleaves
  // the groups' rows, so then the whole CTA)
  if (tma) __syncthreads(); else group_sync<TPF>(g);
  if constexpr (NP == 1) {
    PkPass<M, EE, S::radA(0), 1>::template compute<true>(v, t, twA);
  } else {
    using P0 = PkPass<M, EE, S::radA(0), 1>;
    P0::template compute<true>(v, t, twA);
    P0::store(row, v, t);
    group_sync<TPF>(g);
    pk_mid<M, EE_REQ, false, true, 1, NP - 1>(row, v, t, g, twA);
    using PL = PkPass<M, EE, S::radA(NP - 1), S::nsA(NP - 1)>;
    PL::load(row, v, t);
    group_sync<TPF>(g);
    PL::template compute<true>(v, t, twA + S::twA(NP - 1));
  }
  // ---- v holds z[e] = d[2e] + i d[2e+1] of both rows: the deviation-form nonlinearity
  if constexpr (MODEL == kModelStd) {
    const float2 C1 = bc2(c1), C2 = bc2(c2);
#pragma unroll
    for (int e = 0; e < EE; ++e) {
      v[e].r = mul2(v[e].r, fma2(v[e].r, add2(v[e].r, C2), C1));
      v[e].i = mul2(v[e].i, fma2(v[e].i, add2(v[e].i, C2), C1));
    }
  } else {
#pragma unroll
    for (int e = 0; e < EE; ++e) {
      v[e].r.x = nonlin_dev<MODEL>(v[e].r.x, c1, c2, inv, inv_d, a.clamp, mphi_rel, lmin);
      v[e].r.y = nonlin_dev<MODEL>(v[e].r.y, c1, c2, inv, inv_d, a.clamp, mphi_rel, lmin);
      v[e].i.x = nonlin_dev<MODEL>(v[e].i.x, c1, c2, inv, inv_d, a.clamp, mphi_rel, lmin);
      v[e].i.y = nonlin_dev<MODEL>(v[e].i.y, c1, c2, inv, inv_d, a.clamp, mphi_rel, lmin);
    }
  }
  // ---- forward sequence B
  constexpr int RL = S::radB(NP - 1);
  if constexpr (NP == 1) {
    PkPass<M, EE, S::radB(0), 1>::template compute<false>(v, t, twB);
  } else {
    using Q0 = PkPass<M, EE, S::radB(0), 1>;
    Q0::template compute<false>(v, t, twB);
    Q0::store(row, v, t);
    group_sync<TPF>(g);
    pk_mid<M, EE_REQ, true, false, 1, NP - 1>(row, v, t, g, twB);
    using QL = PkPass<M, EE, RL, S::nsB(NP - 1)>;
    QL::load(row, v, t);
    group_sync<TPF>(g);
    QL::template compute<false>(v, t, twB + S::twB(NP - 1));
  }
  // ---- publish Z (natural order) for the post-twiddle store
  {
    using QO = PkPass<M, EE, RL, M / RL>;
    constexpr int NBL = EE / RL;
#pragma unroll
    for (int b = 0; b < NBL; ++b)
#pragma unroll
      for (int q = 0; q < RL; ++q) pk_st(row + padi<P>(QO::out_index(t, b, q)), v[b * RL + q]);
  }
  __syncthreads();
  // ---- forward-real post-twiddle fused with the transposing store: one (k, M - k) pair per
  // step, Y[k] = E + r_k O, Y[M - k] = conj(E - r_k O), E = (Z[k] + conj Z[M-k]) / 2,
  // O = -i (Z[k] - conj Z[M-k]) / 2; 16 bytes (both rows) per k
  {
    const float4* srow = sm + tp * LD;
    float4* col0 = reinterpret_cast<float4*>(gout + (y0 + 2 * tp));
    const size_t cstride = (size_t)ny / 2;   // float4 entries per column
    const float2 H = bc2(0.5f);
    for (int k = kx0; k <= M / 2; k += kstep) {
      const pc zk = pk_ld(srow + padi<P>(k));
      if (k == 0) {
        col0[0] = pc2raw(mkpc(add2(zk.r, zk.i), sub2(zk.r, zk.i)));
      } else {
        const pc zm = pk_ld(srow + padi<P>(M - k));
        const float4 r = ld_keep(rtw + k);
        const float2 C = make_float2(r.x, r.y), Sn = make_float2(r.z, r.w);
        const pc es = mkpc(add2(zk.r, zm.r), sub2(zk.i, zm.i));       // 2E
        const pc d = mkpc(sub2(zk.r, zm.r), add2(zk.i, zm.i));        // 2iO
        // 2 r_k O = r_k (d.i - i d.r)
        const pc ro = mkpc(fma2(d.r, Sn, mul2(d.i, C)), sub2(mul2(d.i, Sn), mul2(d.r, C)));
        col0[(size_t)k * cstride] = pc2raw(mkpc(mul2(add2(es.r, ro.r), H), mul2(add2(es.i, ro.i), H)));
        if (k != M / 2)
          col0[(size_t)(M - k) * cstride] = pc2raw(mkpc(mul2(sub2(es.r, ro.r), H), mul2(sub2(ro.i, es.i), H)));
      }
    }
  }
}

// ------------------------------------------------------------------ column kernel
// CTA: ngroups consecutive column pairs, one group of TPF threads per pair (columns 2c and
// 2c + 1 in lanes 0 and 1). Pair 0 holds the packed DC/Nyquist column in lane 0, updated
// from (ky, -ky) pairs at full precision as in col_step_fast.
template <int NY, int EE_REQ>
__global__ void __launch_bounds__(PkBound<PkSeq<NY, EE_REQ>::TPF>::value, PkMinB<PkSeq<NY, EE_REQ>::TPF>::value)
col_step_pk(FastColArgs<float> a) {
  using S = PkSeq<NY, EE_REQ>;
  constexpr int EE = S::EE, TPF = S::TPF, NP = S::NPASS;
  constexpr int P = kPkPad;
  constexpr int PADN = NY + (NY >> P) + 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* sm = reinterpret_cast<float4*>(smem_raw);
  const int ngroups = blockDim.x / TPF;
  const int g = threadIdx.x / TPF, t = threadIdx.x - g * TPF;
  const int c = blockIdx.x * ngroups + g;      // column pair
  const int kx0 = 2 * c, kx1 = 2 * c + 1;
  const float4* twA = reinterpret_cast<const float4*>(a.twA);
  const float4* twB = reinterpret_cast<const float4*>(a.twB);
  float4* buf = sm + g * PADN;
  const int m = a.m, nyh = a.nyh;
  const float2* gin = reinterpret_cast<const float2*>(a.in);
  const void* gnin = a.nin;
  void* gnout = a.nout;
  const cplx<float>* gnin_lo = a.nin_lo;
  cplx<float>* gnout_lo = a.nout_lo;
  float2* gwout = reinterpret_cast<float2*>(a.wout);
  const cplx<float>* gcoef = a.coef;
  const cplx<double>* gcoef64 = a.coef64;
  if (a.batch) {
    const BatchBufs& b = a.batch[blockIdx.y];
    gin = static_cast<const float2*>(b.v);
    gnin = b.nin;
    gnout = b.nout;
    gnin_lo = static_cast<const cplx<float>*>(b.nin_lo);
    gnout_lo = static_cast<cplx<float>*>(b.nout_lo);
    gwout = static_cast<float2*>(const_cast<void*>(b.w));
    gcoef = static_cast<const cplx<float>*>(b.coef);
    gcoef64 = static_cast<const cplx<double>*>(b.coef64);
  }
  pc v[EE];

  // ---- both columns' n_hat and coefficients towards L2 while the forward transform runs
  l2_prefetch_range(static_cast<const char*>(gnin) + (size_t)kx0 * NY * sizeof(float2), 2 * NY * sizeof(float2), t,
                    TPF);
  {
    const uintptr_t q0 = reinterpret_cast<uintptr_t>(gcoef + (size_t)kx0 * nyh) & ~(uintptr_t)15;
    const uintptr_t q1 = (reinterpret_cast<uintptr_t>(gcoef + (size_t)(kx1 + 1) * nyh) + 15) & ~(uintptr_t)15;
    l2_prefetch_range(reinterpret_cast<const void*>(q0), (unsigned)(q1 - q0), t, TPF);
  }

  pdl_wait();
  pdl_trigger();

  // ---- forward sequence A; pass 0 reads both columns of V
  {
    constexpr int R = S::radA(0), NR = NY / R, NB = EE / R;
    const float2* col0 = gin + (size_t)kx0 * NY;
    const float2* col1 = gin + (size_t)kx1 * NY;
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int y = t + b * TPF + q * NR;
        v[b * R + q] = mkpc2(ld_stream(col0 + y), ld_stream(col1 + y));
      }
  }
  if constexpr (NP == 1) {
    PkPass<NY, EE, S::radA(0), 1>::template compute<false>(v, t, twA);
  } else {
    using P0 = PkPass<NY, EE, S::radA(0), 1>;
    P0::template compute<false>(v, t, twA);
    P0::store(buf, v, t);
    group_sync<TPF>(g);
    pk_mid<NY, EE_REQ, false, false, 1, NP - 1>(buf, v, t, g, twA);
    using PL = PkPass<NY, EE, S::radA(NP - 1), S::nsA(NP - 1)>;
    PL::load(buf, v, t);
    group_sync<TPF>(g);
    PL::template compute<false>(v, t, twA + S::twA(NP - 1));
  }
  // ---- publish the natural-order spectra of both columns
  constexpr int RL = S::radA(NP - 1), NBL = EE / RL;
  {
    using PO = PkPass<NY, EE, RL, NY / RL>;
#pragma unroll
    for (int b = 0; b < NBL; ++b)
#pragma unroll
      for (int q = 0; q < RL; ++q) pk_st(buf + padi<P>(PO::out_index(t, b, q)), v[b * RL + q]);
  }
  group_sync<TPF>(g);

  // ---- ETD1 update n_hat' = n_hat + (A - 1) n_hat + Bg N_hat of both columns
  const float tau = a.slow_tau;
  const float2* nin = static_cast<const float2*>(gnin);
  float2* nout = static_cast<float2*>(gnout);
  float* bf = reinterpret_cast<float*>(buf);   // lane l of slot i: re at 4 i + l, im at 4 i + 2 + l
  {
    // the regular lanes: both of pair c > 0, lane 1 of pair 0
    const int lfirst = c == 0 ? 1 : 0;
    constexpr int CH = 4;
    static_assert(EE % CH == 0, "chunks tile the modes of a thread");
#pragma unroll 1
    for (int j0 = 0; j0 < EE; j0 += CH) {
      float2 cw[2][CH], p[2][CH];
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        const int ky = t + (j0 + j) * TPF;
        const int kh = ky <= NY / 2 ? ky : NY - ky;
#pragma unroll
        for (int l = 0; l < 2; ++l) {
          const int kx = kx0 + l;
          if (l >= lfirst) {
            cw[l][j] = ld_stream(reinterpret_cast<const float2*>(gcoef) + (size_t)kx * nyh + kh);
            p[l][j] = ld_stream(nin + (size_t)kx * NY + ky);
          } else {
            cw[l][j] = make_float2(0.f, 0.f);
            p[l][j] = make_float2(0.f, 0.f);
          }
        }
      }
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        const int ky = t + (j0 + j) * TPF;
        const int kh = ky <= NY / 2 ? ky : NY - ky;
        float4* slot = buf + padi<P>(ky);
        const pc gv = pk_ld(slot);
        const bool fast0 = lfirst == 0 && fabsf(cw[0][j].x) >= tau;
        const bool fast1 = fabsf(cw[1][j].x) >= tau;
        if (fast0 && fast1) {
          // both lanes fast: the FP32 update on hi alone, packed
          const float2 CX = make_float2(cw[0][j].x, cw[1][j].x), CY = make_float2(cw[0][j].y, cw[1][j].y);
          const float2 PR = make_float2(p[0][j].x, p[1][j].x), PI = make_float2(p[0][j].y, p[1][j].y);
          const pc o = mkpc(fma2(CY, gv.r, fma2(CX, PR, PR)), fma2(CY, gv.i, fma2(CX, PI, PI)));
          nout[(size_t)kx0 * NY + ky] = lane0(o);
          nout[(size_t)kx1 * NY + ky] = lane1(o);
          pk_st(slot, o);
        } else {
          float* sf = bf + 4 * padi<P>(ky);
#pragma unroll
          for (int l = 0; l < 2; ++l) {
            if (l < lfirst) continue;
            const size_t si = (size_t)(kx0 + l) * NY + ky;
            const float gr = l ? gv.r.y : gv.r.x, gi = l ? gv.i.y : gv.i.x;
            if ((l ? fast1 : fast0)) {
              const float2 o = make_float2(fmaf(cw[l][j].y, gr, fmaf(cw[l][j].x, p[l][j].x, p[l][j].x)),
                                           fmaf(cw[l][j].y, gi, fmaf(cw[l][j].x, p[l][j].y, p[l][j].y)));
              nout[si] = o;
              sf[l] = o.x;
              sf[2 + l] = o.y;
            } else {
              // slow mode: FP64 coefficients and the state with its residual
              const cplx<double> cc = gcoef64[(size_t)(kx0 + l) * nyh + kh];
              const cplx<float> lo = gnin_lo[si];
              cplx<double> pd = mk((double)p[l][j].x + (double)lo.x, (double)p[l][j].y + (double)lo.y);
              const cplx<double> o = pd + cc.x * pd + cc.y * mk((double)gr, (double)gi);
              state_st<float>(gnout, gnout_lo, si, o, true);
              sf[l] = (float)o.x;
              sf[2 + l] = (float)o.y;
            }
          }
        }
      }
    }
  }
  if (c == 0) {
    // lane 0 of pair 0: the packed DC/Nyquist column (kx = 0 and kx = m), one (ky, -ky)
    // pair per step at full precision
    const size_t cmb = (size_t)m * nyh;
#pragma unroll 1
    for (int ky = t; ky <= NY / 2; ky += TPF) {
      const int kyp = ky == 0 ? 0 : NY - ky;
      bool s0, sm;
      const cplx<double> pk = state_ld<float>(gnin, gnin_lo, ky, true);
      const cplx<double> pkp = state_ld<float>(gnin, gnin_lo, kyp, true);
      const cplx<double> a0 = coef_ld<float>(gcoef, gcoef64, ky, tau, true, s0);
      const cplx<double> am = coef_ld<float>(gcoef, gcoef64, cmb + ky, tau, true, sm);
      float* sk = bf + 4 * padi<P>(ky);
      float* skp = bf + 4 * padi<P>(kyp);
      const cplx<double> qk = mk((double)sk[0], (double)sk[2]), qkp = mk((double)skp[0], (double)skp[2]);
      cplx<double> h0, hm, g0, gm;
      unpack_pair(pk, pkp, h0, hm);
      unpack_pair(qk, qkp, g0, gm);
      const cplx<double> h0n = h0 + a0.x * h0 + a0.y * g0;
      const cplx<double> hmn = hm + am.x * hm + am.y * gm;
      const cplx<double> ok = h0n + mul_i(hmn), okp = conj(h0n) + mul_i(conj(hmn));
      state_st<float>(gnout, gnout_lo, ky, ok, true);
      sk[0] = (float)ok.x;
      sk[2] = (float)ok.y;
      if (kyp != ky) {
        state_st<float>(gnout, gnout_lo, kyp, okp, true);
        skp[0] = (float)okp.x;
        skp[2] = (float)okp.y;
      }
    }
  }
  group_sync<TPF>(g);
  PkPass<NY, EE, S::radB(0), 1>::load(buf, v, t);
  group_sync<TPF>(g);

  // ---- inverse sequence B; the last pass writes W of both columns
  if constexpr (NP == 1) {
    PkPass<NY, EE, S::radB(0), 1>::template compute<true>(v, t, twB);
  } else {
    using Q0 = PkPass<NY, EE, S::radB(0), 1>;
    Q0::template compute<true>(v, t, twB);
    Q0::store(buf, v, t);
    group_sync<TPF>(g);
    pk_mid<NY, EE_REQ, true, true, 1, NP - 1>(buf, v, t, g, twB);
    using QL = PkPass<NY, EE, S::radB(NP - 1), S::nsB(NP - 1)>;
    QL::load(buf, v, t);
    QL::template compute<true>(v, t, twB + S::twB(NP - 1));
  }
  {
    constexpr int RB = S::radB(NP - 1), NBB = EE / RB;
    using QO = PkPass<NY, EE, RB, NY / RB>;
    float2* col0 = gwout + (size_t)kx0 * NY;
    float2* col1 = gwout + (size_t)kx1 * NY;
    const float2 SC = bc2((float)a.scale);
#pragma unroll
    for (int b = 0; b < NBB; ++b)
#pragma unroll
      for (int q = 0; q < RB; ++q) {
        const pc x = mkpc(mul2(v[b * RB + q].r, SC), mul2(v[b * RB + q].i, SC));
        const int y = QO::out_index(t, b, q);
        col0[y] = lane0(x);
        col1[y] = lane1(x);
      }
  }
}

}  // namespace pfc
