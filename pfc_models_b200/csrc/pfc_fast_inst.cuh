// Definitions of FastInst (pfc_registry.h): included by the .cu file of each
// (precision, elements-per-thread) variant, which instantiates one FastInst.
#pragma once
#include <cmath>

#include "pfc_fast.cuh"
#include "pfc_registry.h"

namespace pfc {

namespace fast_detail {

// Pass tables of sequences A and B for an N-point transform, laid out as FastSeq
// expects: for p = 1 .. NPASS-1, (R(p) - 1) x ns(p) entries exp(-2 pi i q k / (ns R)),
// [q-1][k], so that the lanes of a warp (consecutive k) read consecutive entries.
template <class T, int N, int EE>
void seq_tables(std::vector<long double>& tw, int& offA, int& offB) {
  using S = FastSeq<N, EE, RadixCap<T>::value>;
  const long double twopi = 6.283185307179586476925286766559L;
  for (int seq = 0; seq < 2; ++seq) {
    if (seq == 1 && S::symmetric()) {   // B's table is A's: one copy (half the L1 footprint)
      offB = offA;
      break;
    }
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

template <class T, int EE, int L>
bool tables_l(int lg, std::vector<long double>& tw, int& a, int& b) {
  if constexpr (L <= kFastMaxLogCol) {
    if (lg == L) { seq_tables<T, (1 << L), EE>(tw, a, b); return true; }
    return tables_l<T, EE, L + 1>(lg, tw, a, b);
  } else {
    return false;
  }
}

template <class T, int EE, int MODEL, int L>
bool row_l(int lg, FastKernel* out) {
  if constexpr (L <= kFastMaxLogRow) {
    if (lg == L) {
      out->fn = (void*)row_step_fast<T, (1 << L), EE, MODEL>;
      out->tpf = FastSeq<(1 << L), EE, RadixCap<T>::value>::TPF;
      return true;
    }
    return row_l<T, EE, MODEL, L + 1>(lg, out);
  } else {
    return false;
  }
}

template <class T, int EE, int L>
bool col_l(int lg, FastKernel* out) {
  if constexpr (L <= kFastMaxLogCol) {
    if (lg == L) {
      out->fn = (void*)col_step_fast<T, (1 << L), EE>;
      out->tpf = FastSeq<(1 << L), EE, RadixCap<T>::value>::TPF;
      return true;
    }
    return col_l<T, EE, L + 1>(lg, out);
  } else {
    return false;
  }
}

}  // namespace fast_detail

template <class T, int EE>
bool FastInst<T, EE>::row(int lg, int model, FastKernel* out) {
  return model == kModelLog ? fast_detail::row_l<T, EE, kModelLog, kFastMinLog>(lg, out)
                            : fast_detail::row_l<T, EE, kModelStd, kFastMinLog>(lg, out);
}

template <class T, int EE>
bool FastInst<T, EE>::col(int lg, FastKernel* out) {
  return fast_detail::col_l<T, EE, kFastMinLog>(lg, out);
}

template <class T, int EE>
bool FastInst<T, EE>::tables(int lg, std::vector<long double>& tw, int& offA, int& offB) {
  return fast_detail::tables_l<T, EE, kFastMinLog>(lg, tw, offA, offB);
}

}  // namespace pfc
