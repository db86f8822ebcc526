// Two-lane packed FP32 step kernels (pfc_pack_step.cuh): instantiation and lookup by
// transform size, and their float4 twiddle tables.
#include <cmath>

#include "pfc_pack_step.cuh"
#include "pfc_registry.h"

namespace pfc {

namespace pack_detail {

// (c, c, s, s) of exp(-2 pi i num / den): two complex slots (c, c), (s, s)
void push4(std::vector<long double>& tw, long long num, long long den) {
  const long double twopi = 6.283185307179586476925286766559L;
  const long double ang = -twopi * (long double)num / (long double)den;
  const long double c = cosl(ang), s = sinl(ang);
  tw.push_back(c); tw.push_back(c);
  tw.push_back(s); tw.push_back(s);
}

void align4(std::vector<long double>& tw) {
  if ((tw.size() / 2) % 2) { tw.push_back(0); tw.push_back(0); }   // float4 alignment
}

template <int N, int EE>
void seq_tables(std::vector<long double>& tw, int& offA, int& offB) {
  using S = PkSeq<N, EE>;
  for (int seq = 0; seq < 2; ++seq) {
    if (seq == 1 && S::symmetric()) {   // B's table is A's: one copy (half the L1 footprint)
      offB = offA;
      break;
    }
    align4(tw);
    (seq == 0 ? offA : offB) = (int)(tw.size() / 2);
    for (int p = 1; p < S::NPASS; ++p) {
      const int R = seq == 0 ? S::radA(p) : S::radB(p);
      const int ns = seq == 0 ? S::nsA(p) : S::nsB(p);
      for (int q = 1; q < R; ++q)
        for (int k = 0; k < ns; ++k) push4(tw, (long long)q * k, (long long)ns * R);
    }
  }
}

template <int EE, int L>
bool tables_l(int lg, std::vector<long double>& tw, int& a, int& b) {
  if constexpr (L <= kPackMaxLogCol) {
    if (lg == L) { seq_tables<(1 << L), EE>(tw, a, b); return true; }
    return tables_l<EE, L + 1>(lg, tw, a, b);
  } else {
    return false;
  }
}

template <int EE, int MODEL, int L>
bool row_l(int lg, FastKernel* out) {
  if constexpr (L <= kPackMaxLogRow) {
    if (lg == L) {
      out->fn = (void*)row_step_pk<(1 << L), EE, MODEL>;
      out->tpf = PkSeq<(1 << L), EE>::TPF;
      return true;
    }
    return row_l<EE, MODEL, L + 1>(lg, out);
  } else {
    return false;
  }
}

template <int EE, int L>
bool col_l(int lg, FastKernel* out) {
  if constexpr (L <= kPackMaxLogCol) {
    if (lg == L) {
      out->fn = (void*)col_step_pk<(1 << L), EE>;
      out->tpf = PkSeq<(1 << L), EE>::TPF;
      return true;
    }
    return col_l<EE, L + 1>(lg, out);
  } else {
    return false;
  }
}

}  // namespace pack_detail

bool pack_row(int lg, int ee, int model, FastKernel* out) {
  if (ee == 8)
    return model == kModelLog ? pack_detail::row_l<8, kModelLog, kPackMinLog>(lg, out)
                              : pack_detail::row_l<8, kModelStd, kPackMinLog>(lg, out);
  if (ee == 16)
    return model == kModelLog ? pack_detail::row_l<16, kModelLog, kPackMinLog>(lg, out)
                              : pack_detail::row_l<16, kModelStd, kPackMinLog>(lg, out);
  return false;
}

bool pack_col(int lg, int ee, FastKernel* out) {
  if (ee == 8) return pack_detail::col_l<8, kPackMinLog>(lg, out);
  if (ee == 16) return pack_detail::col_l<16, kPackMinLog>(lg, out);
  return false;
}

bool pack_tables(int lg, int ee, std::vector<long double>& tw, int& offA, int& offB) {
  if (ee == 8) return pack_detail::tables_l<8, kPackMinLog>(lg, tw, offA, offB);
  if (ee == 16) return pack_detail::tables_l<16, kPackMinLog>(lg, tw, offA, offB);
  return false;
}

void pack_real_table(int nx, std::vector<long double>& tw, int& off) {
  pack_detail::align4(tw);
  off = (int)(tw.size() / 2);
  for (int k = 0; k < nx / 2; ++k) pack_detail::push4(tw, k, nx);
}

}  // namespace pfc
