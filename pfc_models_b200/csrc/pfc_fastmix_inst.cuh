// Register-resident step kernels (pfc_fast.cuh) for transform lengths with one odd
// factor, N = ODD * 2^k (ODD = 3, 5, 7; 2^k = 16 .. 512): the grids of phase-diagram
// boxes and other sizes that are not powers of two. Included by one .cu file per
// precision. The power-of-two part of the values per thread is fixed per precision and
// odd factor (FastSeq: EE = ODD * E2), so that every pass's radix divides it.
#pragma once
#include <cmath>

#include "pfc_fast.cuh"
#include "pfc_registry.h"

namespace pfc {

namespace mix_detail {

// E2 by precision and odd factor: FP32 values per thread 24 (3 x 8), 20 (5 x 4) or
// 28 (7 x 4); FP64 12, 20, 28.
template <class T, int ODD> constexpr int mix_e2() { return ODD == 3 ? (sizeof(T) == 4 ? 8 : 4) : 4; }

template <int ODD, int K> constexpr int mixn() { return ODD << K; }

template <class T, int N>
void seq_tables(std::vector<long double>& tw, int& offA, int& offB) {
  using S = FastSeq<N, mix_e2<T, FastSeq<N, 1, 1>::ODD>(), RadixCap<T>::value>;
  const long double twopi = 6.283185307179586476925286766559L;
  for (int seq = 0; seq < 2; ++seq) {
    (seq == 0 ? offA : offB) = (int)(tw.size() / 2);
    for (int p = 1; p < S::NPASS; ++p) {
      const int R = seq == 0 ? S::radA(p) : S::radB(p);
      const int ns = seq == 0 ? S::nsA(p) : S::nsB(p);
      for (int q = 1; q < R; ++q)
        for (int k = 0; k < ns; ++k) {
          const long double ang = -twopi * (long double)((long long)q * k) / (long double)(ns * R);
          tw.push_back(cosl(ang));
          tw.push_back(sinl(ang));
        }
    }
  }
}

template <class T, int N> constexpr int e2_of() { return mix_e2<T, FastSeq<N, 1, 1>::ODD>(); }

template <class T, int ODD, int K>
bool one(int n, int model, bool col, std::vector<long double>* tw, int* a, int* b, FastKernel* out) {
  constexpr int N = ODD << K;
  if (n != N) return false;
  constexpr int E2 = e2_of<T, N>();
  if (tw) {
    seq_tables<T, N>(*tw, *a, *b);
    return true;
  }
  using S = FastSeq<N, E2, RadixCap<T>::value>;
  out->tpf = S::TPF;
  if (col) out->fn = (void*)col_step_fast<T, N, E2>;
  else out->fn = model == kModelLog ? (void*)row_step_fast<T, N, E2, kModelLog> : (void*)row_step_fast<T, N, E2, kModelStd>;
  return true;
}

template <class T, int ODD, int K>
bool find(int n, int model, bool col, std::vector<long double>* tw, int* a, int* b, FastKernel* out) {
  if constexpr (K > kMixMaxLog2) {
    return false;
  } else {
    if (one<T, ODD, K>(n, model, col, tw, a, b, out)) return true;
    return find<T, ODD, K + 1>(n, model, col, tw, a, b, out);
  }
}

template <class T>
bool find_any(int n, int model, bool col, std::vector<long double>* tw, int* a, int* b, FastKernel* out) {
  return find<T, 3, kMixMinLog2>(n, model, col, tw, a, b, out) ||
         find<T, 5, kMixMinLog2>(n, model, col, tw, a, b, out) ||
         find<T, 7, kMixMinLog2>(n, model, col, tw, a, b, out);
}

}  // namespace mix_detail

template <class T>
bool MixInst<T>::row(int n, int model, FastKernel* out) {
  return mix_detail::find_any<T>(n, model, false, nullptr, nullptr, nullptr, out);
}

template <class T>
bool MixInst<T>::col(int n, FastKernel* out) {
  return mix_detail::find_any<T>(n, kModelStd, true, nullptr, nullptr, nullptr, out);
}

template <class T>
bool MixInst<T>::tables(int n, std::vector<long double>& tw, int& offA, int& offB) {
  return mix_detail::find_any<T>(n, kModelStd, true, &tw, &offA, &offB, nullptr);
}

template <class T>
int MixInst<T>::values_per_thread(int n) {
  FastKernel k;
  if (!col(n, &k)) return 0;
  return n / k.tpf;
}

}  // namespace pfc
