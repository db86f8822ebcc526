// Shared-memory mixed-radix Stockham FFT engine for sm_100a.
//
// A CTA owns a batch of equal-length transforms (rows or columns) resident in
// shared memory. Each pass p has radix R_p and stride Ns_p (the product of the
// previous radices). Thread `lt` of a transform executes butterflies
// j = lt, lt + tpf, ...: it reads x[j + q*n/R] (q < R), multiplies by the pass
// twiddles w^(q*k), k = j mod Ns, runs an R-point DFT in registers and writes
// y[(j - k)*R + k + q*Ns]. All reads of a pass complete before the barrier and
// all writes after it, so a pass runs in place and needs one buffer.
// Natural order in and out (decimation in time, autosort).
//
// Twiddles are precomputed on the host in extended precision and stored in the
// working precision: per pass a table tw[k*(R-1) + q-1] = exp(-2 pi i q k/(Ns R)).
// The inverse transform (unnormalised) conjugates them.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef PFC_MAXE_F
#define PFC_MAXE_F 16
#endif
#ifndef PFC_MAXE_D
#define PFC_MAXE_D 8
#endif

namespace pfc {

template <class T>
struct alignas(2 * sizeof(T)) cplx {
  T x, y;
};

template <class T> __device__ __forceinline__ cplx<T> mk(T a, T b) { cplx<T> r; r.x = a; r.y = b; return r; }
template <class T> __device__ __forceinline__ cplx<T> operator+(cplx<T> a, cplx<T> b) { return mk(a.x + b.x, a.y + b.y); }
template <class T> __device__ __forceinline__ cplx<T> operator-(cplx<T> a, cplx<T> b) { return mk(a.x - b.x, a.y - b.y); }
template <class T> __device__ __forceinline__ cplx<T> operator*(T s, cplx<T> a) { return mk(s * a.x, s * a.y); }
template <class T> __device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class T> __device__ __forceinline__ cplx<T> conj(cplx<T> a) { return mk(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse): the radix-4 rotation
template <bool INV, class T> __device__ __forceinline__ cplx<T> rot4(cplx<T> a) {
  return INV ? mk(-a.y, a.x) : mk(a.y, -a.x);
}
template <class T> __device__ __forceinline__ cplx<T> mul_i(cplx<T> a) { return mk(-a.y, a.x); }

constexpr int kMaxPass = 10;

// Per-transform pass description (passed by value in kernel arguments).
struct FftDesc {
  int n;
  int npass;
  int radix[kMaxPass];
  int ns[kMaxPass];
  int twoff[kMaxPass];    // offset (complex elements) of the pass twiddles
  int rootoff[kMaxPass];  // offset of the R roots of unity (odd radices > 3), else -1
};

// ---------------------------------------------------------------- small DFTs
template <bool INV, class T> __device__ __forceinline__ void dft2(cplx<T>& a, cplx<T>& b) {
  cplx<T> t = a - b; a = a + b; b = t;
}

template <bool INV, class T> __device__ __forceinline__ void dft4(cplx<T>* v) {
  cplx<T> t0 = v[0] + v[2], t1 = v[0] - v[2];
  cplx<T> t2 = v[1] + v[3], t3 = rot4<INV>(v[1] - v[3]);
  v[0] = t0 + t2; v[2] = t0 - t2; v[1] = t1 + t3; v[3] = t1 - t3;
}

// multiply by exp(-+ 2 pi i k / 8)
template <bool INV, int K, class T> __device__ __forceinline__ cplx<T> w8(cplx<T> a) {
  const T c = T(0.70710678118654752440084436210485);
  if (K == 0) return a;
  if (K == 2) return rot4<INV>(a);
  if (K == 1) return INV ? mk(c * (a.x - a.y), c * (a.x + a.y)) : mk(c * (a.x + a.y), c * (a.y - a.x));
  /* K == 3 */ return INV ? mk(-c * (a.x + a.y), c * (a.x - a.y)) : mk(c * (a.y - a.x), -c * (a.x + a.y));
}

template <bool INV, class T> __device__ __forceinline__ void dft8(cplx<T>* v) {
  cplx<T> e[4] = {v[0], v[2], v[4], v[6]};
  cplx<T> o[4] = {v[1], v[3], v[5], v[7]};
  dft4<INV>(e); dft4<INV>(o);
  o[1] = w8<INV, 1>(o[1]); o[2] = w8<INV, 2>(o[2]); o[3] = w8<INV, 3>(o[3]);
#pragma unroll
  for (int k = 0; k < 4; ++k) { v[k] = e[k] + o[k]; v[k + 4] = e[k] - o[k]; }
}

template <bool INV, class T> __device__ __forceinline__ void dft16(cplx<T>* v) {
  cplx<T> e[8], o[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) { e[k] = v[2 * k]; o[k] = v[2 * k + 1]; }
  dft8<INV>(e); dft8<INV>(o);
  // o[k] *= exp(-+ 2 pi i k / 16), cos/sin of k*pi/8
  const T c1 = T(0.92387953251128675612818318939679), s1 = T(0.38268343236508977172845998403040);
  const T c2 = T(0.70710678118654752440084436210485);
  const T cs[8] = {T(1), c1, c2, s1, T(0), -s1, -c2, -c1};
  const T sn[8] = {T(0), s1, c2, c1, T(1), c1, c2, s1};
#pragma unroll
  for (int k = 1; k < 8; ++k) {
    if (k == 4) { o[k] = rot4<INV>(o[k]); continue; }
    cplx<T> w = mk(cs[k], INV ? sn[k] : -sn[k]);
    o[k] = cmul(o[k], w);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) { v[k] = e[k] + o[k]; v[k + 8] = e[k] - o[k]; }
}

// 32 points: two 16-point DFTs of the even and odd elements, twiddles
// exp(-+ 2 pi i k / 32), k = 0..15, and a final radix-2 combination.
template <bool INV, class T> __device__ __forceinline__ void dft32(cplx<T>* v) {
  cplx<T> e[16], o[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) { e[k] = v[2 * k]; o[k] = v[2 * k + 1]; }
  dft16<INV>(e); dft16<INV>(o);
  // cos and sin of k pi / 16, k = 0..15
  const T cs[16] = {T(1.0), T(0.98078528040323044912618223613424), T(0.92387953251128675612818318939679),
                    T(0.83146961230254523707878837761791), T(0.70710678118654752440084436210485),
                    T(0.55557023301960222474283081394853), T(0.38268343236508977172845998403040),
                    T(0.19509032201612826784828486847702), T(0.0), T(-0.19509032201612826784828486847702),
                    T(-0.38268343236508977172845998403040), T(-0.55557023301960222474283081394853),
                    T(-0.70710678118654752440084436210485), T(-0.83146961230254523707878837761791),
                    T(-0.92387953251128675612818318939679), T(-0.98078528040323044912618223613424)};
#pragma unroll
  for (int k = 1; k < 16; ++k) {
    if (k == 8) { o[k] = rot4<INV>(o[k]); continue; }
    const T s = cs[(k + 8) & 15] * (k < 8 ? T(-1) : T(1));  // sin(k pi / 16) = -cos((k + 8) pi / 16), k < 8
    cplx<T> w = mk(cs[k], INV ? s : -s);
    o[k] = cmul(o[k], w);
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) { v[k] = e[k] + o[k]; v[k + 16] = e[k] - o[k]; }
}

template <bool INV, class T> __device__ __forceinline__ void dft3(cplx<T>* v) {
  const T h = T(0.86602540378443864676372317075294);  // sqrt(3)/2
  cplx<T> s = v[1] + v[2], d = v[1] - v[2];
  cplx<T> m = v[0] - T(0.5) * s;
  cplx<T> t = h * rot4<INV>(d);
  v[0] = v[0] + s; v[1] = m + t; v[2] = m - t;
}

// Odd prime radix R: with s_b = v_b + v_{R-b}, d_b = v_b - v_{R-b} (b = 1..(R-1)/2),
// y_a = v_0 + sum_b s_b cos(t_ab) -+ i sum_b d_b sin(t_ab), y_{R-a} the conjugate
// combination, t_ab = 2 pi (a b mod R) / R. roots[m] = exp(-2 pi i m / R).
template <int R, bool INV, class T> __device__ __forceinline__ void dft_odd(cplx<T>* v, const cplx<T>* __restrict__ roots) {
  constexpr int H = (R - 1) / 2;
  T cs[H + 1], sn[H + 1];
#pragma unroll
  for (int m = 1; m <= H; ++m) { const cplx<T> r = roots[m]; cs[m] = r.x; sn[m] = -r.y; }
  cplx<T> s[H + 1], d[H + 1];
#pragma unroll
  for (int b = 1; b <= H; ++b) { s[b] = v[b] + v[R - b]; d[b] = v[b] - v[R - b]; }
  const cplx<T> v0 = v[0];
  cplx<T> tot = v0;
#pragma unroll
  for (int b = 1; b <= H; ++b) tot = tot + s[b];
#pragma unroll
  for (int a = 1; a <= H; ++a) {
    cplx<T> A = v0, B = mk(T(0), T(0));
#pragma unroll
    for (int b = 1; b <= H; ++b) {
      const int t = (a * b) % R;
      // cos/sin of 2 pi t / R from the first half of the circle
      const T c = (t <= H) ? cs[t] : cs[R - t];
      const T sgn_s = (t <= H) ? sn[t] : -sn[R - t];
      A = A + c * s[b];
      B = B + sgn_s * d[b];
    }
    // forward: y_a = A - i B, y_{R-a} = A + i B; inverse swaps the signs
    const cplx<T> iB = mul_i(B);
    v[a] = INV ? A + iB : A - iB;
    v[R - a] = INV ? A - iB : A + iB;
  }
  v[0] = tot;
}

template <int R, bool INV, class T> __device__ __forceinline__ void dft(cplx<T>* v, const cplx<T>* roots) {
  if constexpr (R == 2) dft2<INV>(v[0], v[1]);
  else if constexpr (R == 3) dft3<INV>(v);
  else if constexpr (R == 4) dft4<INV>(v);
  else if constexpr (R == 8) dft8<INV>(v);
  else if constexpr (R == 16) dft16<INV>(v);
  else if constexpr (R == 32) dft32<INV>(v);
  else dft_odd<R, INV>(v, roots);
}

// Odd-radix DFT with compile-time roots (R = 5 or 7): cos and sin of 2 pi m / R are
// literal constants (to 20 digits) instead of a table in memory; the same
// (s, d)-symmetric evaluation as dft_odd.
template <int R> __device__ __forceinline__ double root_cos(int m) {
  if (R == 5) return m == 1 ? 0.30901699437494742410 : -0.80901699437494742410;
  // R == 7
  return m == 1 ? 0.62348980185873353053 : m == 2 ? -0.22252093395631440429 : -0.90096886790241912624;
}
template <int R> __device__ __forceinline__ double root_sin(int m) {
  if (R == 5) return m == 1 ? 0.95105651629515357212 : 0.58778525229247312917;
  return m == 1 ? 0.78183148246802980871 : m == 2 ? 0.97492791218182360702 : 0.43388373911755812048;
}
template <int R, bool INV, class T> __device__ __forceinline__ void dft_odd_c(cplx<T>* v) {
  constexpr int H = (R - 1) / 2;
  cplx<T> s[H + 1], d[H + 1];
#pragma unroll
  for (int b = 1; b <= H; ++b) { s[b] = v[b] + v[R - b]; d[b] = v[b] - v[R - b]; }
  const cplx<T> v0 = v[0];
  cplx<T> tot = v0;
#pragma unroll
  for (int b = 1; b <= H; ++b) tot = tot + s[b];
#pragma unroll
  for (int a = 1; a <= H; ++a) {
    cplx<T> A = v0, B = mk(T(0), T(0));
#pragma unroll
    for (int b = 1; b <= H; ++b) {
      const int t = (a * b) % R;
      const T c = (T)root_cos<R>(t <= H ? t : R - t);
      const T sg = (T)(t <= H ? root_sin<R>(t) : -root_sin<R>(R - t));
      A = A + c * s[b];
      B = B + sg * d[b];
    }
    // forward: y_a = A - i B, y_{R-a} = A + i B; inverse swaps the signs
    const cplx<T> iB = mul_i(B);
    v[a] = INV ? A + iB : A - iB;
    v[R - a] = INV ? A - iB : A + iB;
  }
  v[0] = tot;
}

// DFT of a compile-time radix without a root table (powers of two up to 32, 3, 5, 7).
template <int R, bool INV, class T> __device__ __forceinline__ void dft_c(cplx<T>* v) {
  if constexpr (R == 1) return;
  else if constexpr (R == 5 || R == 7) dft_odd_c<R, INV>(v);
  else dft<R, INV>(v, (const cplx<T>*)nullptr);
}

// Elements a thread may hold in registers during one pass.
template <class T> struct MaxElems { static constexpr int value = PFC_MAXE_F; };
template <> struct MaxElems<double> { static constexpr int value = PFC_MAXE_D; };
template <int R, class T> struct MaxBfly {
  // odd radices hold one butterfly at a time (their DFT needs 2R live values)
  static constexpr int value = (R % 2 == 1 && R > 3) ? 1
                             : ((MaxElems<T>::value / R) > 0 ? (MaxElems<T>::value / R) : 1);
};

// Radix sets compiled into a kernel: powers of two only, every supported radix, or the
// radices of grids with prime factors 2, 3, 5 and 7 only (a smaller kernel than the full
// set, which also carries the radix-11 and radix-13 butterflies).
enum : int { kRadixPow2 = 0, kRadixAll = 1, kRadixSmall = 4 };

// One transform's exchange buffer in shared memory, with one pad element per 16 (index i
// lives at i + i / 16): the stores of a small-stride pass, R elements apart across lanes,
// then fall on different banks for the 16 lanes an 8-byte access serves at once.
constexpr int kGenericPadShift = 4;
__host__ __device__ constexpr int generic_pad(int i) { return i + (i >> kGenericPadShift); }
template <class T>
struct PadBuf {
  cplx<T>* p;
  __device__ __forceinline__ cplx<T>& operator[](int i) const { return p[generic_pad(i)]; }
};

// One in-place Stockham pass over a transform of length n at `buf`.
template <int R, bool INV, class T>
__device__ __forceinline__ void stockham_pass(PadBuf<T> buf, int n, int ns, const cplx<T>* __restrict__ tw,
                                              const cplx<T>* __restrict__ roots, int lt, int tpf) {
  constexpr int MB = MaxBfly<R, T>::value;
  const int nr = n / R;
  cplx<T> v[MB][R];
#pragma unroll
  for (int b = 0; b < MB; ++b) {
    const int j = lt + b * tpf;
    if (j < nr) {
#pragma unroll
      for (int q = 0; q < R; ++q) v[b][q] = buf[j + q * nr];
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < MB; ++b) {
    const int j = lt + b * tpf;
    if (j < nr) {
      const int k = j % ns;
      if (k != 0) {
        const cplx<T>* w = tw + k;   // table [q - 1][k]
#pragma unroll
        for (int q = 1; q < R; ++q) {
          cplx<T> t = w[(q - 1) * ns];
          if (INV) t.y = -t.y;
          v[b][q] = cmul(v[b][q], t);
        }
      }
      dft<R, INV>(v[b], roots);
      const int base = (j - k) * R + k;
#pragma unroll
      for (int q = 0; q < R; ++q) buf[base + q * ns] = v[b][q];
    }
  }
  __syncthreads();
}

// Runs every pass of `d` on buf. All threads of the CTA must call this with the same d.
template <bool INV, int RSET, class T>
__device__ __forceinline__ void fft_run(PadBuf<T> buf, const FftDesc& d, const cplx<T>* __restrict__ twbase, int lt, int tpf) {
  for (int p = 0; p < d.npass; ++p) {
    const cplx<T>* tw = twbase + d.twoff[p];
    const cplx<T>* roots = d.rootoff[p] >= 0 ? twbase + d.rootoff[p] : nullptr;
    const int ns = d.ns[p];
    if constexpr (RSET == kRadixPow2) {
      switch (d.radix[p]) {
        case 2: stockham_pass<2, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 4: stockham_pass<4, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 8: stockham_pass<8, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 16: stockham_pass<16, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        default: break;  // rejected on the host
      }
    } else if constexpr (RSET == kRadixSmall) {
      switch (d.radix[p]) {
        case 2: stockham_pass<2, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 3: stockham_pass<3, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 4: stockham_pass<4, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 5: stockham_pass<5, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 7: stockham_pass<7, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 8: stockham_pass<8, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 16: stockham_pass<16, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        default: break;  // rejected on the host
      }
    } else {
      switch (d.radix[p]) {
        case 2: stockham_pass<2, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 3: stockham_pass<3, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 4: stockham_pass<4, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 5: stockham_pass<5, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 7: stockham_pass<7, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 8: stockham_pass<8, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 11: stockham_pass<11, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 13: stockham_pass<13, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        case 16: stockham_pass<16, INV>(buf, d.n, ns, tw, roots, lt, tpf); break;
        default: break;  // rejected on the host
      }
    }
  }
}

}  // namespace pfc
