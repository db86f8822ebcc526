// Definitions of GenericInst (pfc_registry.h): included by the .cu file of each precision.
#pragma once
#include "pfc_kernels.cuh"
#include "pfc_registry.h"

namespace pfc {

namespace generic_detail {

// The nonlinearity only matters in the step and reduce modes; other modes use the std instance.
template <int MODE> constexpr bool row_uses_model() { return MODE == kRowStep || MODE == kRowReduce; }

template <class T, int MODE>
void* pick_row(int model, int rset) {
  const bool log = row_uses_model<MODE>() && model == kModelLog;
  if (rset == kRadixAllDense) {
    if constexpr (sizeof(T) == 4 && MODE == kRowStep)
      return log ? (void*)row_kernel<T, MODE, kModelLog, kRadixAll, 256, 2>
                 : (void*)row_kernel<T, MODE, kModelStd, kRadixAll, 256, 2>;
    rset = kRadixAll;
  }
  if (rset == kRadixSmallDense) {
    if constexpr (sizeof(T) == 4 && MODE == kRowStep)
      return log ? (void*)row_kernel<T, MODE, kModelLog, kRadixSmall, 256, 2>
                 : (void*)row_kernel<T, MODE, kModelStd, kRadixSmall, 256, 2>;
    rset = kRadixSmall;
  }
  if (rset == kRadixSmall)
    return log ? (void*)row_kernel<T, MODE, kModelLog, kRadixSmall, 256>
               : (void*)row_kernel<T, MODE, kModelStd, kRadixSmall, 256>;
  if (rset == kRadixSmallBig)
    return log ? (void*)row_kernel<T, MODE, kModelLog, kRadixSmall, 1024>
               : (void*)row_kernel<T, MODE, kModelStd, kRadixSmall, 1024>;
  if (rset == kRadixPow2Big)
    return log ? (void*)row_kernel<T, MODE, kModelLog, kRadixPow2, 1024>
               : (void*)row_kernel<T, MODE, kModelStd, kRadixPow2, 1024>;
  if (rset == kRadixPow2)
    return log ? (void*)row_kernel<T, MODE, kModelLog, kRadixPow2, 256>
               : (void*)row_kernel<T, MODE, kModelStd, kRadixPow2, 256>;
  return log ? (void*)row_kernel<T, MODE, kModelLog, kRadixAll, 256>
             : (void*)row_kernel<T, MODE, kModelStd, kRadixAll, 256>;
}

template <class T, int MODE>
void* pick_col(int rset) {
  if (rset == kRadixAllDense) {
    if constexpr (sizeof(T) == 4 && MODE == kColStep) return (void*)col_kernel<T, MODE, kRadixAll, 256, 2>;
    rset = kRadixAll;
  }
  if (rset == kRadixSmallDense) {
    if constexpr (sizeof(T) == 4 && MODE == kColStep) return (void*)col_kernel<T, MODE, kRadixSmall, 256, 2>;
    rset = kRadixSmall;
  }
  if (rset == kRadixSmall && MODE != kColParseval && MODE != kColExport) return (void*)col_kernel<T, MODE, kRadixSmall, 256>;
  if (rset == kRadixPow2Big) return (void*)col_kernel<T, MODE, kRadixPow2, 1024>;
  if (rset == kRadixSmallBig)   // (the Parseval and export modes transform nothing)
    return (MODE == kColParseval || MODE == kColExport) ? (void*)col_kernel<T, MODE, kRadixPow2, 1024>
                                                        : (void*)col_kernel<T, MODE, kRadixSmall, 1024>;
  if (MODE == kColParseval || MODE == kColExport || rset == kRadixPow2) return (void*)col_kernel<T, MODE, kRadixPow2, 256>;
  return (void*)col_kernel<T, MODE, kRadixAll, 256>;
}

}  // namespace generic_detail

template <class T>
void* GenericInst<T>::row(int mode, int model, int rset) {
  using namespace generic_detail;
  switch (mode) {
    case kRowStep: return pick_row<T, kRowStep>(model, rset);
    case kRowForward: return pick_row<T, kRowForward>(model, rset);
    case kRowMaterialize: return pick_row<T, kRowMaterialize>(model, rset);
    case kRowReduce: return pick_row<T, kRowReduce>(model, rset);
    default: return nullptr;
  }
}

template <class T>
void* GenericInst<T>::col(int mode, int rset) {
  using namespace generic_detail;
  switch (mode) {
    case kColStep: return pick_col<T, kColStep>(rset);
    case kColInit: return pick_col<T, kColInit>(rset);
    case kColCombine: return pick_col<T, kColCombine>(rset);
    case kColParseval: return pick_col<T, kColParseval>(rset);
    case kColExport: return pick_col<T, kColExport>(rset);
    default: return nullptr;
  }
}

}  // namespace pfc
