// Host side of the C ABI declared in include/pfc_b200.h: plan construction
// (factorisation, twiddles, FP64 ETD1 coefficients, launch shapes), buffer
// ownership and the launch sequences of each entry point.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include "pfc_b200.h"
#include "pfc_fast.cuh"
#include "pfc_kernels.cuh"
#include "pfc_queue.cuh"
#include "pfc_registry.h"
#include "pfc_small.cuh"

using namespace pfc;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define PFC_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(PFC_E_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                  __FILE__, __LINE__);                                                  \
  } while (0)

#define PFC_LAUNCHED()                                                                  \
  do {                                                                                  \
    cudaError_t e_ = cudaGetLastError();                                                \
    if (e_ != cudaSuccess)                                                              \
      return fail(PFC_E_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                  \
  } while (0)

// Largest radix first for the power-of-two part (16 in FP32, 8 in FP64, which
// bounds the registers one butterfly needs), then the odd primes.
bool factorize(int n, bool fp32, std::vector<int>& radices) {
  radices.clear();
  int p2 = 0;
  while (n % 2 == 0) { n /= 2; ++p2; }
  if (fp32)
    while (p2 >= 4) { radices.push_back(16); p2 -= 4; }
  while (p2 >= 3) { radices.push_back(8); p2 -= 3; }
  if (p2 == 2) radices.push_back(4);
  if (p2 == 1) radices.push_back(2);
  for (int r : {3, 5, 7, 11, 13})
    while (n % r == 0) { radices.push_back(r); n /= r; }
  return n == 1 && (int)radices.size() <= kMaxPass;
}

constexpr int kBlockMax = 256;  // default launch bound of the generic kernels
constexpr int pfc_block_max = kBlockMax;
constexpr int kMaxElemsF = PFC_MAXE_F, kMaxElemsD = PFC_MAXE_D;  // as MaxElems in pfc_fft.cuh

// must match MaxBfly in pfc_fft.cuh
int max_bfly(int radix, bool fp32) {
  if (radix % 2 == 1 && radix > 3) return 1;
  const int e = fp32 ? kMaxElemsF : kMaxElemsD;
  return e / radix > 0 ? e / radix : 1;
}

bool all_pow2(const std::vector<int>& radices) {
  for (int r : radices)
    if (r & (r - 1)) return false;
  return true;
}

// Appends the pass tables of an n-point transform to `tw` (complex, long double
// accuracy rounded once) and fills `d`.
void build_fft(int n, const std::vector<int>& radices, std::vector<long double>& tw, FftDesc& d) {
  const long double twopi = 6.283185307179586476925286766559L;
  d.n = n;
  d.npass = (int)radices.size();
  int ns = 1;
  for (int p = 0; p < d.npass; ++p) {
    const int R = radices[p];
    d.radix[p] = R;
    d.ns[p] = ns;
    d.twoff[p] = (int)(tw.size() / 2);
    // [q - 1][k]: the lanes of a warp (consecutive k) read consecutive entries
    for (int q = 1; q < R; ++q)
      for (int k = 0; k < ns; ++k) {
        const long long num = (long long)q * k % ((long long)ns * R);
        const long double ang = -twopi * (long double)num / (long double)(ns * R);
        tw.push_back(cosl(ang));
        tw.push_back(sinl(ang));
      }
    if (R >= 5) {
      d.rootoff[p] = (int)(tw.size() / 2);
      for (int mm = 0; mm < R; ++mm) {
        const long double ang = -twopi * (long double)mm / (long double)R;
        tw.push_back(cosl(ang));
        tw.push_back(sinl(ang));
      }
    } else {
      d.rootoff[p] = -1;
    }
    ns *= R;
  }
  for (int p = d.npass; p < kMaxPass; ++p) { d.radix[p] = 0; d.ns[p] = 0; d.twoff[p] = 0; d.rootoff[p] = -1; }
}

int threads_per_fft(const std::vector<int>& radices, int n, bool fp32) {
  int need = 1;
  for (int R : radices) {
    const int nr = n / R;
    const int mb = max_bfly(R, fp32);
    need = std::max(need, (nr + mb - 1) / mb);
  }
  int t = 1;
  while (t < need) t <<= 1;
  return t;
}

}  // namespace

struct pfc_plan {
  pfc_problem prob;
  int device = 0;
  bool fp32 = false;
  int nx = 0, ny = 0, m = 0, nyh = 0;
  size_t nspec = 0;     // m * ny complex elements per spectral array
  size_t elt = 0;       // bytes per complex element
  // device buffers
  void* nhat[2] = {nullptr, nullptr};     // complex128, or hi (complex64) in the FP32 form
  void* nhat_lo[2] = {nullptr, nullptr};  // FP32 form: residuals of the slow modes
  void* W = nullptr;
  void* V = nullptr;
  void* W2 = nullptr;
  void* coef = nullptr;    // (A - 1, Bg), working precision
  void* coef64 = nullptr;  // FP32 form: (A - 1, Bg) in FP64 for the slow modes
  void* tw = nullptr;
  double* partials = nullptr;
  size_t npartials = 0;
  double* scal = nullptr;
  int* status = nullptr;
  // transforms and launch shapes
  FftDesc rowfft{}, colfft{};
  int rt_off = 0;       // offset of the real-packing twiddles in tw
  int row_tpf = 0, rows = 0, row_ld = 0, row_grid = 0, row_rset = kRadixPow2;
  int col_tpf = 0, cols = 0, col_ld = 0, col_grid = 0, col_rset = kRadixPow2;
  size_t row_smem = 0, col_smem = 0;
  int cur = 0;
  bool state_set = false;
  long long steps_since_set = 0;
  long long launches = 0;
  std::vector<double> hostA, hostBg;  // FP64 coefficients, (ny, m+1)
  // specialised power-of-two step kernels (pfc_fast.cuh)
  bool fast = false;
  void* fast_row_fn = nullptr;
  void* fast_col_fn = nullptr;
  int fr_rows = 0, fr_threads = 0, fr_ld = 0, fr_grid = 0;
  int ee_row = 0, ee_col = 0;  // elements per thread of the fast kernels (per lane when packed)
  bool packed = false;         // two-lane packed FP32 step kernels (pfc_pack_step.cuh) on either pass
  bool packed_row = false, packed_col = false;
  // log PFC with an external potential (PFC_FLAG_EXTV, pfc_extv.cu)
  bool extv = false;
  pfc::ExtvState* extv_st = nullptr;   // device
  double* extv_minmax = nullptr;       // per row-CTA (min, max) of the field
  double2* vhat = nullptr;             // rfft2 of V, (ny, m + 1)
  double2* forcing = nullptr;          // B lap V_hat, [kx][ky]
  void* scratch_state = nullptr;       // a spectral state for transforming V
  int rt4_off = 0;             // packed kernels: offset of the float4 real-packing table in tw
  int tma_box = 0;             // packed row kernel staged by TMA: kx extent of a box (0: cp.async)
  CUtensorMap tmap{};          // its tensor map of W ([kx][y], 8-byte elements)
  unsigned tma_extra_tx = 0;   // pfc_test_tma_wait: bytes its barrier waits for beyond the tile
  int tma_wait_limit = 0;      //   and the polls before it gives up
  int fc_threads = 0, fc_grid = 0;
  size_t fr_smem = 0, fc_smem = 0;
  int tw_ra = 0, tw_rb = 0, tw_ca = 0, tw_cb = 0;  // table offsets (complex elements)
  double lmu0 = 0, lf0 = 0;
  // CUDA graphs of kGraphBlock steps and of one step, one per starting ping-pong parity
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t graph1[2] = {nullptr, nullptr};
  // small FP64 mixed-radix grids: whole steps in one CTA (pfc_onecta.cu), reading this
  // plan's buffers from a one-entry table per parity of cur
  bool onecta = false;
  int oc_threads = 0, oc_rset = kRadixPow2, oc_tpf_r = 0, oc_tpf_c = 0, oc_sms = 0;
  size_t oc_smem = 0;
  pfc::BatchBufs* oc_table[2] = {nullptr, nullptr};
};

// A batch of plans stepped in lockstep: plans with the same step kernels, sizes and
// nonlinearity parameters form a class, stepped by one launch per pass with
// gridDim.y = plans in the class.
struct pfc_batch_class {
  std::vector<pfc_plan*> plans;
  pfc::BatchBufs* table[2] = {nullptr, nullptr};  // device tables, by parity of cur
  cudaStream_t stream = nullptr;                  // classes run concurrently (fork/join)
  cudaEvent_t done = nullptr;
};

struct pfc_batch {
  std::vector<pfc_batch_class> classes;
  bool fp32 = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  cudaEvent_t fork = nullptr;
  long long launches = 0;
};

// Work-queue batch (pfc_queue.cuh): members in the caller's order, their classes, the
// device copies of the class descriptions, one step's item list and the counters.
struct pfc_queue {
  bool fp32 = false;
  std::vector<pfc_plan*> plans;
  std::vector<std::vector<int>> classes;   // member indices of each class
  void* cls_dev = nullptr;                 // QueueClass<T>[classes]
  std::vector<void*> tables;               // BatchBufs arrays, two per class
  int4* items = nullptr;
  int nitems = 0;
  int first_col_item = 0;
  unsigned* counters = nullptr;            // rows done [n], columns done [n], ticket
  int* flags = nullptr;                    // status word, abort flag
  void* fn = nullptr;
  int grid = 0, per_sm = 0;
  size_t smem = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long long launches = 0;
  long long wait_limit = kQueueWaitLimit;
  int extra = 0;
};

// FP32 form: modes with |A - 1| below this are "slow" and keep an FP64-accurate state
// (hi + lo) and FP64 coefficients; the rounding of the others is damped by at least
// this factor every step.
constexpr float kSlowTau = 0.25f;

namespace {

template <class T>
RowArgs<T> row_args(const pfc_plan* h) {
  RowArgs<T> a{};
  a.nx = h->nx; a.ny = h->ny; a.m = h->m; a.rows = h->rows; a.tpf = h->row_tpf; a.ld = h->row_ld;
  a.fft = h->rowfft;
  a.tw = reinterpret_cast<const cplx<T>*>(h->tw);
  a.rtw = reinterpret_cast<const cplx<T>*>(h->tw) + h->rt_off;
  a.scal = h->scal;
  a.clamp = h->prob.clamp_log;
  a.g = h->prob.g;
  a.min_phi = h->prob.min_phi;
  a.min_log = (h->prob.min_phi > 0) ? std::log(h->prob.min_phi) : -INFINITY;
  a.epsilon = h->prob.epsilon;
  return a;
}

template <class T>
ColArgs<T> col_args(const pfc_plan* h) {
  ColArgs<T> a{};
  a.nx = h->nx; a.ny = h->ny; a.m = h->m; a.cols = h->cols; a.tpf = h->col_tpf; a.ld = h->col_ld;
  a.nyh = h->nyh;
  a.fft = h->colfft;
  a.tw = reinterpret_cast<const cplx<T>*>(h->tw);
  a.coef = static_cast<const cplx<T>*>(h->coef);
  a.coef64 = static_cast<const cplx<double>*>(h->coef64);
  a.slow_tau = kSlowTau;
  a.dev_form = h->fp32 ? 1 : 0;
  a.scale = 1.0 / ((double)h->nx * (double)h->ny);
  const double dx = h->prob.lx / h->nx, dy = h->prob.ly / h->ny;
  a.fx = 1.0 / (h->nx * dx);
  a.fy = 1.0 / (h->ny * dy);
  a.beta = h->prob.beta; a.q0 = h->prob.q0; a.epsilon = h->prob.epsilon;
  a.scal = h->scal;
  return a;
}

template <class T, int MODE>
void* pick_row(int model, int rset) { return GenericInst<T>::row(MODE, model, rset); }

template <class T, int MODE>
void* pick_col(int rset) { return GenericInst<T>::col(MODE, rset); }

template <class T, int MODE>
int launch_row(pfc_plan* h, const RowArgs<T>& a, cudaStream_t s, int count = 1) {
  void* fn = pick_row<T, MODE>(h->prob.model, h->row_rset);
  void* args[] = {(void*)&a};
  cudaError_t e = cudaLaunchKernel(fn, dim3(h->row_grid, count), dim3(h->rows * h->row_tpf), args, h->row_smem, s);
  ++h->launches;
  if (e != cudaSuccess) return fail(PFC_E_CUDA, "row kernel launch failed: %s", cudaGetErrorString(e));
  return PFC_OK;
}

template <class T, int MODE>
int launch_col(pfc_plan* h, const ColArgs<T>& a, cudaStream_t s, int count = 1) {
  void* fn = pick_col<T, MODE>(h->col_rset);
  void* args[] = {(void*)&a};
  cudaError_t e = cudaLaunchKernel(fn, dim3(h->col_grid, count), dim3(h->cols * h->col_tpf), args, h->col_smem, s);
  ++h->launches;
  if (e != cudaSuccess) return fail(PFC_E_CUDA, "column kernel launch failed: %s", cudaGetErrorString(e));
  return PFC_OK;
}

// The dynamic shared-memory limit belongs to the kernel function on the device and is
// shared by every plan that launches it: only ever raise it, so that creating a plan
// that needs less cannot break the launches of one that needs more.
int raise_smem_limit(const void* fn, size_t bytes) {
  cudaFuncAttributes fa{};
  PFC_CUDA(cudaFuncGetAttributes(&fa, fn));
  if ((size_t)fa.maxDynamicSharedSizeBytes < bytes)
    PFC_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return PFC_OK;
}

template <class T>
int set_smem_attrs(pfc_plan* h) {
#define PFC_ATTR(fn, bytes) do { int rc_ = raise_smem_limit((const void*)(fn), (bytes)); if (rc_) return rc_; } while (0)
  const int md = h->prob.model, rr = h->row_rset, cr = h->col_rset;
  PFC_ATTR((pick_row<T, kRowStep>(md, rr)), h->row_smem);
  PFC_ATTR((pick_row<T, kRowForward>(md, rr)), h->row_smem);
  PFC_ATTR((pick_row<T, kRowMaterialize>(md, rr)), h->row_smem);
  PFC_ATTR((pick_row<T, kRowReduce>(md, rr)), h->row_smem);
  PFC_ATTR((pick_col<T, kColStep>(cr)), h->col_smem);
  PFC_ATTR((pick_col<T, kColInit>(cr)), h->col_smem);
  PFC_ATTR((pick_col<T, kColCombine>(cr)), h->col_smem);
  PFC_ATTR((pick_col<T, kColParseval>(cr)), h->col_smem);
  PFC_ATTR((pick_col<T, kColExport>(cr)), h->col_smem);
#undef PFC_ATTR
  return PFC_OK;
}

// ---- specialised power-of-two path (pfc_fast.cuh)
int ilog2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return (1 << l) == n ? l : -1;
}

// Elements per thread of the step kernels built for each precision (the first is the default).
template <class T> constexpr int fast_ee_default() { return sizeof(T) == 4 ? 32 : 16; }
template <class T> bool fast_ee_valid(int ee) {
  return sizeof(T) == 4 ? (ee == 8 || ee == 16 || ee == 32) : (ee == 8 || ee == 16);
}

template <class T>
bool fast_lookup(bool col, int lg, int ee, int model, FastKernel* k) {
  if (sizeof(T) == 4) {
    if (ee == 8) return col ? FastInst<float, 8>::col(lg, k) : FastInst<float, 8>::row(lg, model, k);
    if (ee == 16) return col ? FastInst<float, 16>::col(lg, k) : FastInst<float, 16>::row(lg, model, k);
    return col ? FastInst<float, 32>::col(lg, k) : FastInst<float, 32>::row(lg, model, k);
  }
  if (ee == 8) return col ? FastInst<double, 8>::col(lg, k) : FastInst<double, 8>::row(lg, model, k);
  return col ? FastInst<double, 16>::col(lg, k) : FastInst<double, 16>::row(lg, model, k);
}

template <class T>
bool fast_seq_tables(int lg, int ee, std::vector<long double>& tw, int& a, int& b) {
  if (sizeof(T) == 4) {
    if (ee == 8) return FastInst<float, 8>::tables(lg, tw, a, b);
    return ee == 16 ? FastInst<float, 16>::tables(lg, tw, a, b) : FastInst<float, 32>::tables(lg, tw, a, b);
  }
  return ee == 8 ? FastInst<double, 8>::tables(lg, tw, a, b) : FastInst<double, 16>::tables(lg, tw, a, b);
}

// Launch shape of the power-of-two row kernel (one side of the fast step).
struct FastRowSide {
  bool ok = false, packed = false;
  void* fn = nullptr;
  int ee = 0, rows = 0, threads = 0, ld = 0, grid = 0, tw_a = 0, tw_b = 0, rt4 = 0;
  size_t smem = 0;
};
struct FastColSide {
  bool ok = false, packed = false;
  void* fn = nullptr;
  int ee = 0, threads = 0, grid = 0, tw_a = 0, tw_b = 0;
  size_t smem = 0;
};

// One-lane row kernel (pfc_fast.cuh): tile of rows (>= 64 B per kx run by default).
template <class T>
int fast_row_side(pfc_plan* h, int ee, int tile, std::vector<long double>& tw, FastRowSide& o) {
  const int lm = ilog2_exact(h->m);
  FastKernel kr;
  if (lm >= 0) {
    if (lm < kFastMinLog || lm > kFastMaxLogRow || !fast_lookup<T>(false, lm, ee, h->prob.model, &kr)) return PFC_OK;
  } else {
    // one odd factor: the kernel's values per thread are fixed by the transform length
    if (!MixInst<T>::row(h->m, h->prob.model, &kr)) return PFC_OK;
    ee = h->m / kr.tpf;
  }
  // pad shift of the row tile as the kernel uses it (for length / threads per transform)
  const int P = fast_pad_shift(sizeof(T) == 8, h->m / kr.tpf);
  const int elt = (int)sizeof(cplx<T>);
  const int tpr = kr.tpf;
  int ngr = std::max(1, 256 / tpr);
  int rows = tile ? tile : (sizeof(T) == 4 ? 8 : 4);
  // smaller tiles for long rows so that the tile fits the shared-memory budget
  while (rows > 1 && (size_t)rows * (h->m + (h->m >> P) + (1 << P)) * elt > 200 * 1024) rows /= 2;
  ngr = std::min(ngr, rows);
  rows = std::max(rows, ngr);
  // row stride in shared memory: with S = 128 B / element slots per bank cycle,
  // ld = S / rows (mod S) makes the transposing loads and stores of a warp hit
  // distinct banks
  const int slots = 128 / elt;
  const int want = (slots / rows) % slots;
  int ld = h->m + (h->m >> P);
  while (ld % slots != want) ++ld;
  const size_t smem = (size_t)rows * ld * elt;
  // a row count other than a power of two needs the CTA to be whole multiples of it (the
  // transposing tile copies give each thread one row)
  if (ngr * tpr > 1024 || smem > 200 * 1024 || (ilog2_exact(rows) < 0 && (ngr * tpr) % rows)) return PFC_OK;
  o.rows = rows;
  o.threads = ngr * tpr;
  o.ld = ld;
  o.grid = (h->ny + rows - 1) / rows;
  o.smem = smem;
  o.fn = kr.fn;
  o.ee = ee;
  if (lm >= 0) fast_seq_tables<T>(lm, ee, tw, o.tw_a, o.tw_b);
  else MixInst<T>::tables(h->m, tw, o.tw_a, o.tw_b);
  o.ok = true;
  return PFC_OK;
}

// One-lane column kernel: one group of tpc threads per column.
template <class T>
int fast_col_side(pfc_plan* h, int ee, int col_cta, std::vector<long double>& tw, FastColSide& o) {
  const int ly = ilog2_exact(h->ny);
  FastKernel kc;
  if (ly >= 0) {
    if (ly < kFastMinLog || ly > kFastMaxLogCol || !fast_lookup<T>(true, ly, ee, h->prob.model, &kc)) return PFC_OK;
  } else {
    if (!MixInst<T>::col(h->ny, &kc)) return PFC_OK;
    ee = h->ny / kc.tpf;
  }
  const int Pc = fast_pad_shift(sizeof(T) == 8, h->ny / kc.tpf);
  const int elt = (int)sizeof(cplx<T>);
  const int tpc = kc.tpf;
  // (the kernels are built for at most 256 threads per CTA, or one group if larger)
  const int ngc_max = std::max(1, 256 / tpc);
  int ngc = std::min(col_cta ? std::min(col_cta, ngc_max) : ngc_max, h->m);
  while (h->m % ngc) ngc /= 2;
  const size_t smem = (size_t)ngc * (h->ny + (h->ny >> Pc) + 2) * elt;   // one exchange buffer per column
  if (ngc * tpc > 1024 || smem > 200 * 1024) return PFC_OK;
  o.threads = ngc * tpc;
  o.grid = h->m / ngc;
  o.smem = smem;
  o.fn = kc.fn;
  o.ee = ee;
  if (ly >= 0) fast_seq_tables<T>(ly, ee, tw, o.tw_a, o.tw_b);
  else MixInst<T>::tables(h->ny, tw, o.tw_a, o.tw_b);
  o.ok = true;
  return PFC_OK;
}

// Two-lane packed FP32 row kernel (pfc_pack_step.cuh): tiles of `rows` rows, rows / 2
// groups of one row pair; float4 pass tables and the float4 real-packing table.
int pack_row_side(pfc_plan* h, int ee, int tile, std::vector<long double>& tw, FastRowSide& o) {
  const int lm = ilog2_exact(h->m);
  if (lm < kPackMinLog || lm > kPackMaxLogRow) return PFC_OK;
  FastKernel kr;
  if (!pack_row(lm, ee, h->prob.model, &kr)) return PFC_OK;
  const size_t slot = 16;   // one pc (two complex floats)
  const size_t ld = (size_t)h->m + (h->m >> 4);
  int rows = tile ? tile : 8;
  // the kernels are built for max(256, threads per transform) threads per CTA; at most
  // about half the shared memory of an SM per CTA
  const int max_threads = std::max(256, kr.tpf);
  while (rows > 2 && ((size_t)(rows / 2) * ld * slot > 110 * 1024 || (rows / 2) * kr.tpf > max_threads)) rows /= 2;
  if (h->ny % rows || (rows / 2) * kr.tpf > max_threads || (size_t)(rows / 2) * ld * slot > 200 * 1024)
    return PFC_OK;
  o.rows = rows;
  o.threads = (rows / 2) * kr.tpf;
  o.ld = (int)ld;
  o.grid = h->ny / rows;
  o.smem = (size_t)(rows / 2) * ld * slot;
  o.fn = kr.fn;
  o.ee = ee;
  o.packed = true;
  pack_tables(lm, ee, tw, o.tw_a, o.tw_b);
  pack_real_table(h->nx, tw, o.rt4);
  o.ok = true;
  return PFC_OK;
}

// Two-lane packed FP32 column kernel: ngc column pairs per CTA.
int pack_col_side(pfc_plan* h, int ee, int col_cta, std::vector<long double>& tw, FastColSide& o) {
  const int ly = ilog2_exact(h->ny);
  if (ly < kPackMinLog || ly > kPackMaxLogCol || h->m % 2) return PFC_OK;
  FastKernel kc;
  if (!pack_col(ly, ee, &kc)) return PFC_OK;
  const size_t slot = 16;
  const int ngc_max = std::max(1, 256 / kc.tpf);
  const int npairs = h->m / 2;
  int ngc = std::min(col_cta ? std::min(col_cta, ngc_max) : ngc_max, npairs);
  while (npairs % ngc) ngc /= 2;
  const size_t padn = (size_t)h->ny + (h->ny >> 4) + 2;
  const size_t smem = (size_t)ngc * padn * slot;
  if (ngc * kc.tpf > std::max(256, kc.tpf) || smem > 200 * 1024) return PFC_OK;
  o.threads = ngc * kc.tpf;
  o.grid = npairs / ngc;
  o.smem = smem;
  o.fn = kc.fn;
  o.ee = ee;
  o.packed = true;
  pack_tables(ly, ee, tw, o.tw_a, o.tw_b);
  o.ok = true;
  return PFC_OK;
}

// The tensor map through which the packed row kernel stages its tile (PFC_FLAG_TMA):
// W as a 2-D array of 8-byte elements, y innermost (ny, stride 8 B) and kx outer (m,
// stride ny * 8 B); boxes of fr_rows x min(m, 256) with the swizzle of the box's inner
// width. The box's x coordinate is the tile's first row, always even (16-byte aligned).
int setup_tma(pfc_plan* h) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", reinterpret_cast<void**>(&encode), cudaEnableDefault,
                                &q) != cudaSuccess || q != cudaDriverEntryPointSuccess || !encode)
      return fail(PFC_E_CUDA, "pfc_plan_create: cuTensorMapEncodeTiled is not available");
  }
  const int ib = h->fr_rows * 8;
  CUtensorMapSwizzle sw = CU_TENSOR_MAP_SWIZZLE_NONE;
  if (ib == 32) sw = CU_TENSOR_MAP_SWIZZLE_32B;
  else if (ib == 64) sw = CU_TENSOR_MAP_SWIZZLE_64B;
  else if (ib == 128) sw = CU_TENSOR_MAP_SWIZZLE_128B;
  else if (ib != 16) return fail(PFC_E_ARG, "pfc_plan_create: TMA staging takes row tiles of 2 to 16 rows");
  const int box = std::min(h->m, 256);
  cuuint64_t dims[2] = {(cuuint64_t)h->ny, (cuuint64_t)h->m};
  cuuint64_t strides[1] = {(cuuint64_t)h->ny * 8};
  cuuint32_t boxd[2] = {(cuuint32_t)h->fr_rows, (cuuint32_t)box};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode(&h->tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, h->W, dims, strides, boxd, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(PFC_E_CUDA, "pfc_plan_create: cuTensorMapEncodeTiled failed (%d)", (int)r);
  h->tma_box = box;
  h->fr_smem += 1024;   // room to start the tile on a 1024-byte boundary
  return raise_smem_limit(h->fast_row_fn, h->fr_smem);
}

// Chooses the fast kernels and their launch shapes; appends their twiddle tables to tw.
// problem.flags may pick each kernel's values per thread (with PFC_EE_PACKED, or
// PFC_FLAG_PACKED for both, the two-lane packed FP32 kernel of that pass), the row tile
// and the columns per CTA. Both passes must have a fast kernel, else the plan uses the
// mixed-radix kernels.
template <class T>
int setup_fast(pfc_plan* h, std::vector<long double>& tw) {
  const int flags = h->prob.flags;
  const int fr = PFC_FLAG_ROW_EE_OF(flags), fc = PFC_FLAG_COL_EE_OF(flags);
  const bool all_packed = (flags & PFC_FLAG_PACKED) != 0;
  const bool row_packed = all_packed || (fr & PFC_EE_PACKED), col_packed = all_packed || (fc & PFC_EE_PACKED);
  if ((row_packed || col_packed) && sizeof(T) != 4)
    return fail(PFC_E_ARG, "pfc_plan_create: the packed kernels are built for the FP32-mixed form only");
  const int er = fr & ~PFC_EE_PACKED, ec = fc & ~PFC_EE_PACKED;
  const int ee_r = er ? er : (row_packed ? 16 : fast_ee_default<T>());
  const int ee_c = ec ? ec : (col_packed ? 16 : fast_ee_default<T>());
  if (row_packed ? (ee_r != 8 && ee_r != 16) : !fast_ee_valid<T>(ee_r))
    return fail(PFC_E_ARG, "pfc_plan_create: row kernel values per thread %d not built (FP32: 8, 16 or 32; "
                "FP64: 8 or 16; packed: 8 or 16 per lane)", ee_r);
  if (col_packed ? (ee_c != 8 && ee_c != 16) : !fast_ee_valid<T>(ee_c))
    return fail(PFC_E_ARG, "pfc_plan_create: column kernel values per thread %d not built (FP32: 8, 16 or 32; "
                "FP64: 8 or 16; packed: 8 or 16 per lane)", ee_c);
  const int tile = PFC_FLAG_ROW_TILE_OF(flags);
  if (tile && (tile > 16 || (row_packed && ((tile & (tile - 1)) || tile < 2))))
    return fail(PFC_E_ARG, "pfc_plan_create: row tile %d: at most 16 rows (packed: a power of two >= 2)", tile);
  if (flags & PFC_FLAG_GENERIC_ONLY) return PFC_OK;
  const int col_cta = PFC_FLAG_COL_CTA_OF(flags);
  FastRowSide r;
  FastColSide c;
  int rc = row_packed ? pack_row_side(h, ee_r, tile, tw, r) : fast_row_side<T>(h, ee_r, tile, tw, r);
  if (rc) return rc;
  rc = col_packed ? pack_col_side(h, ee_c, col_cta, tw, c) : fast_col_side<T>(h, ee_c, col_cta, tw, c);
  if (rc) return rc;
  if (!r.ok || !c.ok) return PFC_OK;   // generic path
  h->fr_rows = r.rows;
  h->fr_threads = r.threads;
  h->fr_ld = r.ld;
  h->fr_grid = r.grid;
  h->fr_smem = r.smem;
  h->fc_threads = c.threads;
  h->fc_grid = c.grid;
  h->fc_smem = c.smem;
  h->fast_row_fn = r.fn;
  h->fast_col_fn = c.fn;
  h->ee_row = r.ee;
  h->ee_col = c.ee;
  h->tw_ra = r.tw_a; h->tw_rb = r.tw_b;
  h->tw_ca = c.tw_a; h->tw_cb = c.tw_b;
  h->rt4_off = r.rt4;
  h->packed_row = r.packed;
  h->packed_col = c.packed;
  h->packed = r.packed || c.packed;
  if (int e = raise_smem_limit(h->fast_row_fn, h->fr_smem)) return e;
  if (int e = raise_smem_limit(h->fast_col_fn, h->fc_smem)) return e;
  h->fast = true;
  return PFC_OK;
}

// One row pass of a step: W -> V (of every plan in `table` when batched).
// Launches a power-of-two step kernel, with PFC_FLAG_PDL (or, for the column kernel,
// PFC_FLAG_PDL_COL) as a programmatic dependent launch (the kernel may start while the
// previous kernel of the stream drains; it waits for it with griddepcontrol.wait before
// reading its outputs).
inline cudaError_t launch_step_kernel(const pfc_plan* h, const void* fn, dim3 grid, dim3 block, void** args,
                                      size_t smem, cudaStream_t s, bool col = false) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = ((h->prob.flags & PFC_FLAG_PDL) || (col && (h->prob.flags & PFC_FLAG_PDL_COL))) ? 1 : 0;
  return cudaLaunchKernelExC(&cfg, fn, args);
}

ExtvCoefArgs extv_coef_args(const pfc_plan* h) {
  ExtvCoefArgs a{};
  a.nx = h->nx; a.ny = h->ny; a.m = h->m; a.nyh = h->nyh;
  const double dx = h->prob.lx / h->nx, dy = h->prob.ly / h->ny;
  a.fx = 1.0 / (h->nx * dx);
  a.fy = 1.0 / (h->ny * dy);
  a.gamma = h->prob.gamma; a.beta = h->prob.beta; a.q0 = h->prob.q0; a.epsilon = h->prob.epsilon;
  a.dt = h->prob.dt; a.small_z_tol = h->prob.small_z_tol;
  a.coef = static_cast<double2*>(h->coef);
  a.vhat = h->vhat;
  a.forcing = h->forcing;
  return a;
}

// launches of one step of this plan (row and column kernels, plus the external-potential
// decision and coefficient kernels)
int launches_per_step(const pfc_plan* h) { return h->extv ? 4 : 2; }

// Arguments of the fast row kernel for plan h (a batch's members from `table`).
template <class T>
FastRowArgs<T> fast_row_args(const pfc_plan* h, const BatchBufs* table) {
  FastRowArgs<T> a{};
  a.batch = table;
  a.ny = h->ny; a.rows = h->fr_rows; a.ld = h->fr_ld; a.rows_log2 = ilog2_exact(h->fr_rows);
  a.in = reinterpret_cast<const cplx<T>*>(h->W);
  a.out = reinterpret_cast<cplx<T>*>(h->V);
  const cplx<T>* tw = reinterpret_cast<const cplx<T>*>(h->tw);
  a.twA = tw + h->tw_ra; a.twB = tw + h->tw_rb; a.rtw = tw + (h->packed_row ? h->rt4_off : h->rt_off);
  a.scal = h->scal;
  a.clamp = h->prob.clamp_log;
  a.g = h->prob.g; a.min_phi = h->prob.min_phi;
  a.min_log = (h->prob.min_phi > 0) ? std::log(h->prob.min_phi) : -INFINITY;
  a.err = h->status;
  a.tma_box = table ? 0 : h->tma_box;   // a batch's plans each have their own W: copies
  a.tma_extra_tx = h->tma_extra_tx;
  a.tma_wait_limit = h->tma_wait_limit;
  return a;
}

// Arguments of the fast column kernel for plan h (a batch's members from `table`).
template <class T>
FastColArgs<T> fast_col_args(const pfc_plan* h, const BatchBufs* table) {
  FastColArgs<T> a{};
  a.batch = table;
  a.m = h->m; a.ny = h->ny; a.nyh = h->nyh;
  a.in = reinterpret_cast<const cplx<T>*>(h->V);
  a.nin = h->nhat[h->cur];
  a.nout = h->nhat[h->cur ^ 1];
  a.nin_lo = static_cast<const cplx<float>*>(h->nhat_lo[h->cur]);
  a.nout_lo = static_cast<cplx<float>*>(h->nhat_lo[h->cur ^ 1]);
  a.coef64 = static_cast<const cplx<double>*>(h->coef64);
  a.slow_tau = kSlowTau;
  a.wout = reinterpret_cast<cplx<T>*>(h->W);
  a.coef = static_cast<const cplx<T>*>(h->coef);
  const cplx<T>* tw = reinterpret_cast<const cplx<T>*>(h->tw);
  a.twA = tw + h->tw_ca; a.twB = tw + h->tw_cb;
  a.scale = (T)(1.0 / ((double)h->nx * (double)h->ny));
  return a;
}

template <class T>
int launch_step_row(pfc_plan* h, cudaStream_t s, const BatchBufs* table = nullptr, int count = 1) {
  if (h->fast) {
    FastRowArgs<T> a = fast_row_args<T>(h, table);
    void* args_pk[] = {(void*)&a, (void*)&h->tmap};
    void* args1[] = {(void*)&a};
    void** args = h->packed_row ? args_pk : args1;
    cudaError_t e = launch_step_kernel(h, h->fast_row_fn, dim3(h->fr_grid, count), dim3(h->fr_threads), args,
                                       h->fr_smem, s);
    ++h->launches;
    if (e != cudaSuccess) return fail(PFC_E_CUDA, "row step launch failed: %s", cudaGetErrorString(e));
    return PFC_OK;
  }
  RowArgs<T> ra = row_args<T>(h);
  ra.in = reinterpret_cast<const cplx<T>*>(h->W);
  ra.out = reinterpret_cast<cplx<T>*>(h->V);
  ra.batch = table;
  if (!h->extv) return launch_row<T, kRowStep>(h, ra, s, count);
  // external potential: the field's range, the M decision and (when M or V changed) the
  // coefficients and the forcing, before the column pass
  ra.minmax = h->extv_minmax;
  int rc = launch_row<T, kRowStep>(h, ra, s, count);
  if (rc) return rc;
  cudaError_t e = launch_extv_decide(h->extv_minmax, h->row_grid, h->extv_st, h->prob.g, s);
  if (e == cudaSuccess) e = launch_extv_coef(extv_coef_args(h), h->extv_st, s);
  h->launches += 2;
  if (e != cudaSuccess) return fail(PFC_E_CUDA, "external-potential step launch failed: %s", cudaGetErrorString(e));
  return PFC_OK;
}

// One column pass of a step: V, n_hat[cur] -> n_hat[cur ^ 1], W (batched as above).
template <class T>
int launch_step_col(pfc_plan* h, cudaStream_t s, const BatchBufs* table = nullptr, int count = 1) {
  if (h->fast) {
    FastColArgs<T> a = fast_col_args<T>(h, table);
    void* args[] = {(void*)&a};
    cudaError_t e = launch_step_kernel(h, h->fast_col_fn, dim3(h->fc_grid, count), dim3(h->fc_threads), args,
                                       h->fc_smem, s, true);
    ++h->launches;
    if (e != cudaSuccess) return fail(PFC_E_CUDA, "column step launch failed: %s", cudaGetErrorString(e));
    return PFC_OK;
  }
  ColArgs<T> ca = col_args<T>(h);
  ca.in = reinterpret_cast<const cplx<T>*>(h->V);
  ca.wout = reinterpret_cast<cplx<T>*>(h->W);
  ca.nin = h->nhat[h->cur];
  ca.nout = h->nhat[h->cur ^ 1];
  ca.nin_lo = static_cast<const cplx<float>*>(h->nhat_lo[h->cur]);
  ca.nout_lo = static_cast<cplx<float>*>(h->nhat_lo[h->cur ^ 1]);
  ca.batch = table;
  if (h->extv) ca.forcing = reinterpret_cast<const cplx<double>*>(h->forcing);
  return launch_col<T, kColStep>(h, ca, s, count);
}

// ---- entry point bodies, templated on the working precision
template <class T>
int do_set_state(pfc_plan* h, const double* field, cudaStream_t s) {
  const size_t sites = (size_t)h->nx * h->ny;
  if (h->fp32) {
    field_sum_kernel<<<256, 256, 0, s>>>(field, sites, h->partials);
    ++h->launches;
    PFC_LAUNCHED();
    set_scalars_kernel<<<1, 32, 0, s>>>(h->partials, 256, 1.0 / (double)sites, h->prob.model, h->prob.g,
                                        h->prob.min_phi, h->lmu0, h->scal);
    ++h->launches;
    PFC_LAUNCHED();
  }
  RowArgs<T> ra = row_args<T>(h);
  ra.in_real = field;
  ra.out = reinterpret_cast<cplx<T>*>(h->V);
  int rc = launch_row<T, kRowForward>(h, ra, s);
  if (rc) return rc;
  ColArgs<T> ca = col_args<T>(h);
  ca.in = reinterpret_cast<const cplx<T>*>(h->V);
  ca.nout = h->nhat[h->cur];
  ca.nout_lo = static_cast<cplx<float>*>(h->nhat_lo[h->cur]);
  ca.wout = reinterpret_cast<cplx<T>*>(h->W);
  rc = launch_col<T, kColInit>(h, ca, s);
  if (rc) return rc;
  h->state_set = true;
  h->steps_since_set = 0;
  return PFC_OK;
}

constexpr int kGraphBlock = 16;   // steps per captured graph (even: the parity returns)

// Records `fn(capture_stream)` into an executable graph.
template <class F>
int capture_graph(F&& fn, cudaGraphExec_t* out) {
  cudaStream_t cs = nullptr;
  PFC_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t g = nullptr;
  int rc = PFC_OK;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = fn(cs);
    cudaError_t e2 = cudaStreamEndCapture(cs, &g);
    if (rc == PFC_OK && e2 != cudaSuccess) rc = fail(PFC_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e2));
  } else {
    rc = fail(PFC_E_CUDA, "cudaStreamBeginCapture failed: %s", cudaGetErrorString(e));
  }
  if (rc == PFC_OK) {
    e = cudaGraphInstantiate(out, g, 0);
    if (e != cudaSuccess) rc = fail(PFC_E_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(e));
  }
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  return rc;
}

// ---- one-CTA steps (small FP64 mixed-radix grids)
// Steps per launch of the one-CTA kernel (a launch of 2048 steps of a 28 x 24 grid runs
// a few milliseconds).
constexpr long long kOneCtaChunk = 2048;

// The radix set that holds every radix of both transforms.
int onecta_rset(int a, int b) {
  if (a == kRadixAll || b == kRadixAll) return kRadixAll;
  if (a == kRadixSmall || b == kRadixSmall) return kRadixSmall;
  return (a == kRadixPow2 && b == kRadixPow2) ? kRadixPow2 : -1;
}

// Largest butterfly count of a pass of d: threads per transform for one butterfly each.
int max_butterflies(const FftDesc& d) {
  int r = 1;
  for (int p = 0; p < d.npass; ++p) r = std::max(r, d.n / d.radix[p]);
  return r;
}

// Chooses the one-CTA path for FP64 mixed-radix plans whose grid fits one CTA: every row
// (and every column) transform at once within kOneCtaMaxThreads threads, up to one
// butterfly per thread and pass, and the buffers within kOneCtaMaxSmem of shared memory.
// PFC_FLAG_NO_ONE_CTA keeps the two-kernel step.
int setup_onecta(pfc_plan* h) {
  h->onecta = false;
  if (h->fp32 || h->fast || (h->prob.flags & PFC_FLAG_NO_ONE_CTA)) return PFC_OK;
  const int rset = onecta_rset(h->row_rset, h->col_rset);
  if (rset < 0 || !onecta_supported(rset)) return PFC_OK;
  const int tpf_r = std::min(max_butterflies(h->rowfft), std::max(1, kOneCtaMaxThreads / h->ny));
  const int tpf_c = std::min(max_butterflies(h->colfft), std::max(1, kOneCtaMaxThreads / h->m));
  const int need = std::max(h->ny * tpf_r, h->m * tpf_c);
  const int threads = (need + 31) / 32 * 32;
  const size_t smem = onecta_smem_bytes(h->m, h->ny, h->row_ld, h->col_ld);
  if (threads > kOneCtaMaxThreads || smem > kOneCtaMaxSmem) return PFC_OK;
  if (smem > 48 * 1024) {
    cudaError_t e = onecta_allow_smem(kOneCtaMaxSmem);
    if (e != cudaSuccess) return fail(PFC_E_CUDA, "pfc_plan_create: one-CTA shared memory: %s", cudaGetErrorString(e));
  }
  for (int p = 0; p < 2; ++p) {
    BatchBufs b{};
    b.w = h->W; b.v = h->V; b.nin = h->nhat[p]; b.nout = h->nhat[p ^ 1];
    b.coef = h->coef; b.scal = h->scal;
    cudaError_t e = cudaMalloc(&h->oc_table[p], sizeof(BatchBufs));
    if (e == cudaSuccess) e = cudaMemcpy(h->oc_table[p], &b, sizeof(BatchBufs), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(PFC_E_CUDA, "pfc_plan_create: one-CTA table: %s", cudaGetErrorString(e));
  }
  h->onecta = true;
  h->oc_threads = threads;
  h->oc_tpf_r = tpf_r;
  h->oc_tpf_c = tpf_c;
  cudaDeviceGetAttribute(&h->oc_sms, cudaDevAttrMultiProcessorCount, h->device);
  h->oc_rset = rset;
  h->oc_smem = smem;
  return PFC_OK;
}

// `nsteps` steps of `count` plans of one class (table: their buffers at the current parity).
int launch_onecta(pfc_plan* h, cudaStream_t s, const BatchBufs* table, int count, long long nsteps) {
  RowArgs<double> ra = row_args<double>(h);
  ColArgs<double> ca = col_args<double>(h);
  ra.tpf = h->oc_tpf_r;
  ca.tpf = h->oc_tpf_c;
  // more plans than SMs: the build that fits two CTAs per SM
  const bool dense = count > h->oc_sms;
  cudaError_t e = launch_onecta_step(ra, ca, table, count, nsteps, h->prob.model, h->oc_rset, dense,
                                     h->oc_threads, h->oc_smem, s);
  ++h->launches;
  if (e != cudaSuccess) return fail(PFC_E_CUDA, "one-CTA step launch failed: %s", cudaGetErrorString(e));
  return PFC_OK;
}

int onecta_steps(pfc_plan* h, long long nsteps, cudaStream_t s) {
  for (long long done = 0; done < nsteps;) {
    const long long k = std::min(nsteps - done, kOneCtaChunk);
    int rc = launch_onecta(h, s, h->oc_table[h->cur], 1, k);
    if (rc) return rc;
    if (k & 1) h->cur ^= 1;
    h->steps_since_set += k;
    done += k;
  }
  return PFC_OK;
}

template <class T>
int step_direct(pfc_plan* h, long long nsteps, cudaStream_t s) {
  for (long long i = 0; i < nsteps; ++i) {
    int rc = launch_step_row<T>(h, s);
    if (rc) return rc;
    rc = launch_step_col<T>(h, s);
    if (rc) return rc;
    h->cur ^= 1;
    ++h->steps_since_set;
  }
  return PFC_OK;
}

// Replays `count` times a graph of `len` steps that starts at the current parity
// (captured on first use) and updates cur and the counters as direct stepping would.
// A graph of odd length flips the parity, so it is replayed once per call (count = 1).
template <class T>
int replay_steps(pfc_plan* h, cudaGraphExec_t* slot, int len, long long count, cudaStream_t s) {
  const int p = h->cur;
  if (!slot[p]) {
    const long long launches = h->launches, since = h->steps_since_set;
    int rc = capture_graph([&](cudaStream_t cs) { return step_direct<T>(h, len, cs); }, &slot[p]);
    h->launches = launches;
    h->steps_since_set = since;
    h->cur = p;
    if (rc) return rc;
  }
  for (long long b = 0; b < count; ++b) {
    cudaError_t e = cudaGraphLaunch(slot[p], s);
    if (e != cudaSuccess) return fail(PFC_E_CUDA, "cudaGraphLaunch failed: %s", cudaGetErrorString(e));
  }
  h->launches += (long long)launches_per_step(h) * len * count;
  h->steps_since_set += (long long)len * count;
  if ((len * count) & 1) h->cur ^= 1;
  return PFC_OK;
}

// Whole blocks of kGraphBlock steps and the remaining single steps replay graphs captured
// once per starting parity (smaller gaps between the kernels than direct launches).
template <class T>
int do_step(pfc_plan* h, long long nsteps, cudaStream_t s) {
  if (h->onecta) return onecta_steps(h, nsteps, s);
  if (h->prob.flags & PFC_FLAG_NO_GRAPHS) return step_direct<T>(h, nsteps, s);
  const long long blocks = nsteps / kGraphBlock;
  if (blocks > 0) {
    int rc = replay_steps<T>(h, h->graph, kGraphBlock, blocks, s);
    if (rc) return rc;
  }
  for (long long i = blocks * kGraphBlock; i < nsteps; ++i) {
    int rc = replay_steps<T>(h, h->graph1, 1, 1, s);
    if (rc) return rc;
  }
  return PFC_OK;
}

// ---- batches
// The classes are independent: each runs its nsteps on its own stream, forked from and
// joined back to `s` (in a capture this makes parallel branches of the graph).
template <class T>
int batch_step_direct(pfc_batch* b, int parity, long long nsteps, cudaStream_t s) {
  if (nsteps <= 0) return PFC_OK;
  const bool fork = b->classes.size() > 1;
  if (fork) PFC_CUDA(cudaEventRecord(b->fork, s));
  for (auto& c : b->classes) {
    cudaStream_t cs = fork ? c.stream : s;
    if (fork) PFC_CUDA(cudaStreamWaitEvent(cs, b->fork, 0));
    pfc_plan* h = c.plans[0];
    const int n = (int)c.plans.size();
    int p = parity;
    for (long long done = 0; h->onecta && done < nsteps;) {
      const long long k = std::min(nsteps - done, kOneCtaChunk);
      int rc = launch_onecta(h, cs, c.table[p], n, k);
      if (rc) return rc;
      b->launches += 1;
      if (k & 1) p ^= 1;
      done += k;
    }
    for (long long i = 0; !h->onecta && i < nsteps; ++i) {
      int rc = launch_step_row<T>(h, cs, c.table[p], n);
      if (rc) return rc;
      rc = launch_step_col<T>(h, cs, c.table[p], n);
      if (rc) return rc;
      b->launches += 2;
      p ^= 1;
    }
    if (fork) PFC_CUDA(cudaEventRecord(c.done, cs));
  }
  if (fork)
    for (auto& c : b->classes) PFC_CUDA(cudaStreamWaitEvent(s, c.done, 0));
  return PFC_OK;
}

template <class T>
int do_batch_step(pfc_batch* b, long long nsteps, cudaStream_t s) {
  const int parity = b->classes[0].plans[0]->cur;
  for (auto& c : b->classes)
    for (pfc_plan* h : c.plans) {
      if (!h->state_set) return fail(PFC_E_STATE, "pfc_batch_step: a plan has no state");
      if (h->cur != parity)
        return fail(PFC_E_STATE, "pfc_batch_step: plans must have taken the same number of steps mod 2");
    }
  bool all_onecta = true;
  for (auto& c : b->classes) all_onecta = all_onecta && c.plans[0]->onecta;
  const long long blocks = all_onecta ? 0 : nsteps / kGraphBlock;
  if (blocks > 0) {
    if (!b->graph[parity]) {
      const long long launches = b->launches;
      int rc = capture_graph([&](cudaStream_t cs) { return batch_step_direct<T>(b, parity, kGraphBlock, cs); },
                             &b->graph[parity]);
      b->launches = launches;
      if (rc) return rc;
    }
    for (long long k = 0; k < blocks; ++k) {
      cudaError_t e = cudaGraphLaunch(b->graph[parity], s);
      if (e != cudaSuccess) return fail(PFC_E_CUDA, "cudaGraphLaunch failed: %s", cudaGetErrorString(e));
    }
    long long per_block = 0;
    for (auto& c : b->classes) per_block += c.plans[0]->onecta ? 1 : 2LL * kGraphBlock;
    b->launches += per_block * blocks;
  }
  const long long rest = nsteps - blocks * kGraphBlock;
  int rc = batch_step_direct<T>(b, parity, rest, s);   // kGraphBlock is even: parity unchanged
  if (rc) return rc;
  for (auto& c : b->classes)
    for (pfc_plan* h : c.plans) {
      h->cur ^= (int)(nsteps & 1);
      h->steps_since_set += nsteps;
    }
  return PFC_OK;
}

template <class T>
int do_step_timed(pfc_plan* h, long long nsteps, double* ms_row, double* ms_col, cudaStream_t s) {
  std::vector<cudaEvent_t> ev(3 * (size_t)nsteps, nullptr);
  int rc = PFC_OK;
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) { rc = fail(PFC_E_CUDA, "cudaEventCreate failed"); break; }
  for (long long i = 0; i < nsteps && rc == PFC_OK; ++i) {
    cudaEventRecord(ev[3 * i], s);
    rc = launch_step_row<T>(h, s);
    if (rc) break;
    cudaEventRecord(ev[3 * i + 1], s);
    rc = launch_step_col<T>(h, s);
    if (rc) break;
    cudaEventRecord(ev[3 * i + 2], s);
    h->cur ^= 1;
    ++h->steps_since_set;
  }
  double tr = 0, tc = 0;
  if (rc == PFC_OK) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(PFC_E_CUDA, "pfc_step_timed: %s", cudaGetErrorString(e));
    for (long long i = 0; i < nsteps && rc == PFC_OK; ++i) {
      float a = 0, b = 0;
      cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]);
      cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]);
      tr += a; tc += b;
    }
  }
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  if (ms_row) *ms_row = tr;
  if (ms_col) *ms_col = tc;
  return rc;
}

template <class T>
int do_materialize(pfc_plan* h, const void* spec, const double* add, double* out, bool correct_mean,
                   cudaStream_t s) {
  RowArgs<T> ra = row_args<T>(h);
  ra.in = reinterpret_cast<const cplx<T>*>(spec);
  ra.out_real = out;
  ra.add = add;
  ra.partials = correct_mean ? h->partials : nullptr;
  int rc = launch_row<T, kRowMaterialize>(h, ra, s);
  if (rc) return rc;
  if (correct_mean) {
    const size_t sites = (size_t)h->nx * h->ny;
    finalize_mean_kernel<<<1, 32, 0, s>>>(h->partials, h->row_grid, 1.0 / (double)sites, h->scal);
    ++h->launches;
    PFC_LAUNCHED();
    shift_kernel<<<1024, 256, 0, s>>>(out, sites, h->scal + kScalCorr);
    ++h->launches;
    PFC_LAUNCHED();
  }
  return PFC_OK;
}

template <class T>
int do_get_state(pfc_plan* h, double* out, cudaStream_t s) {
  return do_materialize<T>(h, h->W, h->scal + (h->fp32 ? kScalMean : kScalZero), out, h->fp32, s);
}

template <class T>
int do_reduce(pfc_plan* h, double* out3, cudaStream_t s) {
  double* rowp = h->partials;
  double* colp = h->partials + 6 * (size_t)h->row_grid;
  RowArgs<T> ra = row_args<T>(h);
  ra.in = reinterpret_cast<const cplx<T>*>(h->W);
  ra.partials = rowp;
  int rc = launch_row<T, kRowReduce>(h, ra, s);
  if (rc) return rc;
  ColArgs<T> ca = col_args<T>(h);
  ca.sin = h->nhat[h->cur];
  ca.sin_lo = static_cast<const cplx<float>*>(h->nhat_lo[h->cur]);
  ca.partials = colp;
  rc = launch_col<T, kColParseval>(h, ca, s);
  if (rc) return rc;
  const double sites = (double)h->nx * (double)h->ny;
  finalize_reduce_kernel<<<1, 32, 0, s>>>(rowp, h->row_grid, colp, h->col_grid, h->scal, 1.0 / sites, h->lmu0,
                                          h->lf0, h->fp32 ? 1 : 0, out3, h->status);
  ++h->launches;
  PFC_LAUNCHED();
  return PFC_OK;
}

// Nonlinear row spectra V of the "previous" state, and the index of that state's n_hat.
template <class T>
int prepare_previous(pfc_plan* h, bool current, int* old_buf, cudaStream_t s) {
  if (h->steps_since_set > 0 && !current) {
    *old_buf = h->cur ^ 1;
    return PFC_OK;
  }
  RowArgs<T> ra = row_args<T>(h);
  ra.in = reinterpret_cast<const cplx<T>*>(h->W);
  ra.out = reinterpret_cast<cplx<T>*>(h->V);
  int rc = launch_row<T, kRowStep>(h, ra, s);
  if (rc) return rc;
  *old_buf = h->cur;
  return PFC_OK;
}

template <class T>
int do_get_field(pfc_plan* h, int which, double w, double* out, cudaStream_t s) {
  const bool current = (which & PFC_FIELD_OF_CURRENT) != 0;
  which &= ~PFC_FIELD_OF_CURRENT;
  if (which == PFC_FIELD_N) return do_get_state<T>(h, out, s);
  if (!h->W2) {
    PFC_CUDA(cudaMalloc(&h->W2, h->nspec * h->elt));
  }
  int old_buf = 0;
  int rc = prepare_previous<T>(h, current, &old_buf, s);
  if (rc) return rc;
  ColArgs<T> ca = col_args<T>(h);
  ca.in = reinterpret_cast<const cplx<T>*>(h->V);
  ca.nin = h->nhat[old_buf];
  ca.nin_lo = static_cast<const cplx<float>*>(h->nhat_lo[old_buf]);
  ca.wout = reinterpret_cast<cplx<T>*>(h->W2);
  ca.w = w;
  int addslot = kScalZero;
  switch (which) {
    case PFC_FIELD_MU: ca.combine = kCombineMu; addslot = h->fp32 ? kScalMuConst : kScalZero; break;
    case PFC_FIELD_LOCAL_MU: ca.combine = kCombineLocalMu; addslot = h->fp32 ? kScalMuConst : kScalZero; break;
    case PFC_FIELD_LOCAL_N: ca.combine = kCombineLocalN; addslot = h->fp32 ? kScalMean : kScalZero; break;
    case PFC_FIELD_NONLIN_MU: ca.combine = kCombineNonlin; addslot = h->fp32 ? kScalN0 : kScalZero; break;
    default: return fail(PFC_E_ARG, "pfc_get_field: unknown field %d", which);
  }
  rc = launch_col<T, kColCombine>(h, ca, s);
  if (rc) return rc;
  return do_materialize<T>(h, h->W2, h->scal + addslot, out, false, s);
}

template <class T>
int do_get_spectrum(pfc_plan* h, int which, double* out, cudaStream_t s) {
  int buf = h->cur;
  if (which == PFC_SPEC_N_HAT && h->steps_since_set > 0) buf = h->cur ^ 1;
  ColArgs<T> ca = col_args<T>(h);
  ca.sin = h->nhat[buf];
  ca.sin_lo = static_cast<const cplx<float>*>(h->nhat_lo[buf]);
  ca.out_c128 = out;
  int rc = launch_col<T, kColExport>(h, ca, s);
  if (rc) return rc;
  return PFC_OK;
}

}  // namespace

// ---------------------------------------------------------------- C ABI
extern "C" {

int pfc_abi_version(void) { return PFC_ABI_VERSION; }

int pfc_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return PFC_E_ARG;
  snprintf(buf, len, "%s", g_last_error.c_str());
  return PFC_OK;
}

int pfc_plan_create(const pfc_problem* p, pfc_plan** out) {
  if (!p || !out) return fail(PFC_E_ARG, "pfc_plan_create: null argument");
  *out = nullptr;
  if (p->nx < 4 || p->ny < 2 || (p->nx & 1))
    return fail(PFC_E_ARG, "pfc_plan_create: nx must be even and >= 4, ny >= 2 (got %d x %d)", p->nx, p->ny);
  if (p->model != PFC_MODEL_STD && p->model != PFC_MODEL_LOG)
    return fail(PFC_E_ARG, "pfc_plan_create: unknown model %d", p->model);
  if (p->precision != PFC_FP64_PLAIN && p->precision != PFC_FP32_MIXED)
    return fail(PFC_E_ARG, "pfc_plan_create: unknown precision %d", p->precision);
  if (!(p->lx > 0) || !(p->ly > 0) || !(p->dt > 0))
    return fail(PFC_E_ARG, "pfc_plan_create: lx, ly, dt must be positive");
  std::vector<int> rrow, rcol;
  const int m = p->nx / 2;
  const bool fp32 = (p->precision == PFC_FP32_MIXED);
  if (!factorize(m, fp32, rrow))
    return fail(PFC_E_ARG, "pfc_plan_create: nx/2 = %d has a prime factor other than 2,3,5,7,11,13", m);
  if (!factorize(p->ny, fp32, rcol))
    return fail(PFC_E_ARG, "pfc_plan_create: ny = %d has a prime factor other than 2,3,5,7,11,13", p->ny);

  if ((p->flags & PFC_FLAG_EXTV) && (fp32 || p->model != PFC_MODEL_LOG || !p->clamp_log || !(p->min_phi > 0)))
    return fail(PFC_E_ARG, "pfc_plan_create: PFC_FLAG_EXTV needs the FP64 plain log model with the clamped log "
                "(clamp_log = 1, min_phi > 0)");

  pfc_plan* h = new pfc_plan();
  h->prob = *p;
  // the external-potential step runs on the mixed-radix kernels and the two-kernel step
  if (p->flags & PFC_FLAG_EXTV) h->prob.flags |= PFC_FLAG_GENERIC_ONLY | PFC_FLAG_NO_ONE_CTA;
  h->extv = (p->flags & PFC_FLAG_EXTV) != 0;
  h->fp32 = (p->precision == PFC_FP32_MIXED);
  h->nx = p->nx; h->ny = p->ny; h->m = m; h->nyh = p->ny / 2 + 1;
  h->nspec = (size_t)m * p->ny;
  auto rset_of = [](const std::vector<int>& r) {
    if (all_pow2(r)) return (int)kRadixPow2;
    for (int x : r)
      if (x == 11 || x == 13) return (int)kRadixAll;
    return (int)kRadixSmall;
  };
  h->row_rset = rset_of(rrow);
  h->col_rset = rset_of(rcol);
  if (h->fp32 && (long long)p->nx * p->ny >= kDenseMinSites) {
    for (int* r : {&h->row_rset, &h->col_rset}) {
      if (*r == kRadixAll) *r = kRadixAllDense;
      else if (*r == kRadixSmall) *r = kRadixSmallDense;
    }
  }
  h->elt = h->fp32 ? sizeof(float2) : sizeof(double2);
  cudaGetDevice(&h->device);

  auto cleanup_fail = [&](int rc) { pfc_plan_destroy(h); return rc; };

  // ---- twiddles: row passes, column passes, real-packing table
  std::vector<long double> tw;
  build_fft(m, rrow, tw, h->rowfft);
  build_fft(p->ny, rcol, tw, h->colfft);
  h->rt_off = (int)(tw.size() / 2);
  {
    const long double twopi = 6.283185307179586476925286766559L;
    for (int k = 0; k < m; ++k) {
      const long double ang = -twopi * (long double)k / (long double)p->nx;
      tw.push_back(cosl(ang));
      tw.push_back(sinl(ang));
    }
  }
  {
    const int rc = h->fp32 ? setup_fast<float>(h, tw) : setup_fast<double>(h, tw);
    if (rc) return cleanup_fail(rc);
  }

  // ---- launch shapes
  const int cbytes = (int)h->elt;
  int smem_opt = 0;
  cudaDeviceGetAttribute(&smem_opt, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  if (smem_opt <= 0) smem_opt = 227 * 1024;
  const int budget = std::min(smem_opt - 8 * 1024, 200 * 1024);
  // at least two CTAs per SM where the grid allows it: larger tiles coalesce better, but
  // on small and medium grids they left most SMs idle
  int n_sm = 0;
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, h->device);
  const int min_ctas = 2 * std::max(n_sm, 1);
  {
    h->row_tpf = threads_per_fft(rrow, m, h->fp32);
    // padded row (generic_pad) plus one, odd, so that the transposing tile accesses of
    // consecutive rows start on different banks
    h->row_ld = generic_pad(m - 1) + 2;
    if (h->row_ld % 2 == 0) ++h->row_ld;
    if (h->row_tpf > kBlockMax && h->row_rset == kRadixPow2 && h->row_tpf <= 1024) h->row_rset = kRadixPow2Big;
    if (h->row_tpf > kBlockMax && (h->row_rset == kRadixSmall || h->row_rset == kRadixSmallDense) &&
        h->row_tpf <= 1024)
      h->row_rset = kRadixSmallBig;
    const int kBlockMax = (h->row_rset == kRadixPow2Big || h->row_rset == kRadixSmallBig) ? 1024 : pfc_block_max;
    if (h->row_tpf > kBlockMax)
      return cleanup_fail(fail(PFC_E_ARG, "pfc_plan_create: row transform of %d points needs %d threads", m, h->row_tpf));
    const int rows_min = std::max(1, 32 / h->row_tpf);       // whole warps
    const int rows_cap = std::max(rows_min, kBlockMax / h->row_tpf);
    const int coalesce = std::max(1, 64 / cbytes);           // >= 64 B per kx run
    int rows = std::max(rows_min, std::min(coalesce, rows_cap));
    while (2 * rows <= rows_cap && (size_t)(2 * rows) * h->row_ld * cbytes <= (size_t)budget / 2 && rows < p->ny)
      rows *= 2;
    while ((size_t)rows * h->row_ld * cbytes > (size_t)budget && rows > std::max(1, 32 / h->row_tpf)) rows /= 2;
    while (rows > rows_min && (p->ny + rows - 1) / rows < min_ctas) rows /= 2;
    if ((size_t)rows * h->row_ld * cbytes > (size_t)budget || rows * h->row_tpf > kBlockMax)
      return cleanup_fail(fail(PFC_E_ARG, "pfc_plan_create: row transform of %d points does not fit", m));
    h->rows = rows;
    h->row_grid = (p->ny + rows - 1) / rows;
    h->row_smem = (size_t)rows * h->row_ld * cbytes;
  }
  {
    h->col_tpf = threads_per_fft(rcol, p->ny, h->fp32);
    h->col_ld = generic_pad(p->ny - 1) + 2;   // padded column plus one
    if (h->col_ld % 2 == 0) ++h->col_ld;
    if (h->col_tpf > kBlockMax && h->col_rset == kRadixPow2 && h->col_tpf <= 1024) h->col_rset = kRadixPow2Big;
    if (h->col_tpf > kBlockMax && (h->col_rset == kRadixSmall || h->col_rset == kRadixSmallDense) &&
        h->col_tpf <= 1024)
      h->col_rset = kRadixSmallBig;
    const int kBlockMax = (h->col_rset == kRadixPow2Big || h->col_rset == kRadixSmallBig) ? 1024 : pfc_block_max;
    if (h->col_tpf > kBlockMax)
      return cleanup_fail(fail(PFC_E_ARG, "pfc_plan_create: column transform of %d points needs %d threads", p->ny, h->col_tpf));
    int cols = std::max(1, 32 / h->col_tpf);
    while (2 * cols * h->col_tpf <= kBlockMax && (size_t)(2 * cols) * h->col_ld * cbytes <= (size_t)budget / 2 && cols < m)
      cols *= 2;
    while (cols > std::max(1, 32 / h->col_tpf) && (m + cols - 1) / cols < min_ctas) cols /= 2;
    if ((size_t)cols * h->col_ld * cbytes > (size_t)budget || cols * h->col_tpf > kBlockMax)
      return cleanup_fail(fail(PFC_E_ARG, "pfc_plan_create: column transform of %d points does not fit", p->ny));
    h->cols = cols;
    h->col_grid = (m + cols - 1) / cols;
    h->col_smem = (size_t)cols * h->col_ld * cbytes;
  }

  // ---- FP64 ETD1 coefficients (kernels.py:55-71) and the update factor Gamma*lap
  const double dx = p->lx / p->nx, dy = p->ly / p->ny;
  const double fx = 1.0 / (p->nx * dx), fy = 1.0 / (p->ny * dy);
  const double twopi = 6.283185307179586;
  h->hostA.assign((size_t)p->ny * (m + 1), 0.0);
  h->hostBg.assign((size_t)p->ny * (m + 1), 0.0);
  std::vector<double> coefA(2 * (size_t)(m + 1) * h->nyh);   // (A - 1, Bg) pairs
  for (int ky = 0; ky < p->ny; ++ky) {
    const int kys = (ky <= (p->ny - 1) / 2) ? ky : ky - p->ny;
    const double kyp = twopi * ((double)kys * fy);
    for (int kx = 0; kx <= m; ++kx) {
      const double kxp = twopi * ((double)kx * fx);
      const double lap = -(kxp * kxp + kyp * kyp);
      const double t = p->q0 * p->q0 + lap;
      const double lmu = p->beta * (t * t) + p->epsilon;
      const double gl = p->gamma * lap;
      const double ln = gl * lmu;
      const double z = ln * p->dt;
      const double A = std::exp(z);
      const double B = (std::fabs(z) > p->small_z_tol) ? (A - 1) / ln : p->dt * (1 + z / 2 + z * z / 6);
      const double Bg = B * gl;
      h->hostA[(size_t)ky * (m + 1) + kx] = A;
      h->hostBg[(size_t)ky * (m + 1) + kx] = Bg;
      // the device applies n' = n + (A - 1) n + Bg N in FP64, with A - 1 = expm1(z)
      if (ky < h->nyh) {
        coefA[2 * ((size_t)kx * h->nyh + ky)] = std::expm1(z);
        coefA[2 * ((size_t)kx * h->nyh + ky) + 1] = Bg;
      }
    }
  }
  h->lmu0 = p->beta * (p->q0 * p->q0) * (p->q0 * p->q0) + p->epsilon;
  h->lf0 = (p->beta / 2.0) * (p->q0 * p->q0) * (p->q0 * p->q0);

  // ---- device buffers
  const size_t specb = h->nspec * h->elt;
  // the spectral state: complex128 (FP64 form), or hi + lo complex64 arrays (FP32 form)
  const size_t stateb = h->nspec * (h->fp32 ? sizeof(float2) : sizeof(double2));
  const size_t ncoef = (size_t)(m + 1) * h->nyh;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaMalloc(&h->nhat[i], stateb);
  for (int i = 0; i < 2 && e == cudaSuccess && h->fp32; ++i) e = cudaMalloc(&h->nhat_lo[i], stateb);
  if (e == cudaSuccess && h->fp32) e = cudaMalloc(&h->coef64, ncoef * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc(&h->W, specb);
  if (e == cudaSuccess) e = cudaMalloc(&h->V, specb);
  if (e == cudaSuccess) e = cudaMalloc(&h->coef, ncoef * h->elt);
  if (e == cudaSuccess) e = cudaMalloc(&h->tw, tw.size() / 2 * h->elt);
  h->npartials = 6 * (size_t)h->row_grid + 2 * (size_t)h->col_grid + 2 * 1024;
  if (e == cudaSuccess) e = cudaMalloc(&h->partials, h->npartials * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&h->scal, kScalCount * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&h->status, sizeof(int));
  if (h->extv) {
    if (e == cudaSuccess) e = cudaMalloc(&h->extv_st, sizeof(ExtvState));
    if (e == cudaSuccess) e = cudaMalloc(&h->extv_minmax, 2 * (size_t)h->row_grid * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&h->vhat, (size_t)p->ny * (m + 1) * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&h->forcing, (size_t)(m + 1) * p->ny * sizeof(double2));
    if (e == cudaSuccess) e = cudaMemset(h->vhat, 0, (size_t)p->ny * (m + 1) * sizeof(double2));
    if (e == cudaSuccess) e = cudaMemset(h->forcing, 0, (size_t)(m + 1) * p->ny * sizeof(double2));
    if (e == cudaSuccess) {
      // ValidatePhiRange's state as the reference builds it (logpfc_extv/simulation.py:130-144)
      ExtvState st{};
      st.floor_tol = 0.1;
      st.ceil_tol = 0.1;
      st.min_phi = p->min_phi;
      e = cudaMemcpy(h->extv_st, &st, sizeof(st), cudaMemcpyHostToDevice);
    }
  }
  if (e != cudaSuccess)
    return cleanup_fail(fail(e == cudaErrorMemoryAllocation ? PFC_E_NOMEM : PFC_E_CUDA,
                             "pfc_plan_create: cudaMalloc failed: %s", cudaGetErrorString(e)));

  // upload the twiddle tables in the working precision, the coefficients (A - 1, Bg) in FP64
  {
    std::vector<unsigned char> host;
    const size_t ntw = tw.size() / 2;
    host.resize(ntw * h->elt);
    for (size_t i = 0; i < ntw; ++i) {
      if (h->fp32) { float2 v = make_float2((float)tw[2 * i], (float)tw[2 * i + 1]); memcpy(&host[i * 8], &v, 8); }
      else { double2 v = make_double2((double)tw[2 * i], (double)tw[2 * i + 1]); memcpy(&host[i * 16], &v, 16); }
    }
    e = cudaMemcpy(h->tw, host.data(), host.size(), cudaMemcpyHostToDevice);
    if (h->fp32) {
      std::vector<float2> c32(ncoef);
      for (size_t i = 0; i < ncoef; ++i) c32[i] = make_float2((float)coefA[2 * i], (float)coefA[2 * i + 1]);
      if (e == cudaSuccess) e = cudaMemcpy(h->coef, c32.data(), ncoef * sizeof(float2), cudaMemcpyHostToDevice);
      if (e == cudaSuccess)
        e = cudaMemcpy(h->coef64, coefA.data(), coefA.size() * sizeof(double), cudaMemcpyHostToDevice);
    } else if (e == cudaSuccess) {
      e = cudaMemcpy(h->coef, coefA.data(), coefA.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
    std::vector<double> sc(kScalCount, 0.0);
    if (e == cudaSuccess) e = cudaMemcpy(h->scal, sc.data(), sc.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(h->status, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->W, 0, specb);
    for (int i = 0; i < 2; ++i) {
      if (e == cudaSuccess) e = cudaMemset(h->nhat[i], 0, stateb);
      if (e == cudaSuccess && h->nhat_lo[i]) e = cudaMemset(h->nhat_lo[i], 0, stateb);
    }
    if (e != cudaSuccess)
      return cleanup_fail(fail(PFC_E_CUDA, "pfc_plan_create: upload failed: %s", cudaGetErrorString(e)));
  }
  int rc = h->fp32 ? set_smem_attrs<float>(h) : set_smem_attrs<double>(h);
  if (rc) return cleanup_fail(rc);
  if (h->packed_row && (p->flags & PFC_FLAG_TMA)) {
    rc = setup_tma(h);
    if (rc) return cleanup_fail(rc);
  }
  rc = setup_onecta(h);
  if (rc) return cleanup_fail(rc);
  *out = h;
  return PFC_OK;
}

int pfc_plan_destroy(pfc_plan* h) {
  if (!h) return PFC_OK;
  for (auto& g : h->graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto& g : h->graph1)
    if (g) cudaGraphExecDestroy(g);
  for (void* p : {h->nhat[0], h->nhat[1], h->nhat_lo[0], h->nhat_lo[1], h->W, h->V, h->W2, h->coef, h->coef64, h->tw})
    if (p) cudaFree(p);
  if (h->partials) cudaFree(h->partials);
  for (void* q : {(void*)h->extv_st, (void*)h->extv_minmax, (void*)h->vhat, (void*)h->forcing, h->scratch_state})
    if (q) cudaFree(q);
  if (h->scal) cudaFree(h->scal);
  if (h->status) cudaFree(h->status);
  for (auto* t : h->oc_table)
    if (t) cudaFree(t);
  delete h;
  return PFC_OK;
}

int pfc_set_state(pfc_plan* h, const double* field, void* stream) {
  if (!h || !field) return fail(PFC_E_ARG, "pfc_set_state: null argument");
  if (reinterpret_cast<uintptr_t>(field) % 16)
    return fail(PFC_E_ARG, "pfc_set_state: field must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  return h->fp32 ? do_set_state<float>(h, field, s) : do_set_state<double>(h, field, s);
}

int pfc_get_state(pfc_plan* h, double* field, void* stream) {
  if (!h || !field) return fail(PFC_E_ARG, "pfc_get_state: null argument");
  if (!h->state_set) return fail(PFC_E_STATE, "pfc_get_state: no state has been set");
  if (reinterpret_cast<uintptr_t>(field) % 16)
    return fail(PFC_E_ARG, "pfc_get_state: field must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  return h->fp32 ? do_get_state<float>(h, field, s) : do_get_state<double>(h, field, s);
}

int pfc_step(pfc_plan* h, int64_t nsteps, void* stream) {
  if (!h) return fail(PFC_E_ARG, "pfc_step: null plan");
  if (nsteps < 0) return fail(PFC_E_ARG, "pfc_step: negative step count");
  if (!h->state_set) return fail(PFC_E_STATE, "pfc_step: no state has been set");
  cudaStream_t s = (cudaStream_t)stream;
  return h->fp32 ? do_step<float>(h, nsteps, s) : do_step<double>(h, nsteps, s);
}

int pfc_step_timed(pfc_plan* h, int64_t nsteps, double* ms_row, double* ms_col, void* stream) {
  if (!h) return fail(PFC_E_ARG, "pfc_step_timed: null plan");
  if (nsteps < 0) return fail(PFC_E_ARG, "pfc_step_timed: negative step count");
  if (!h->state_set) return fail(PFC_E_STATE, "pfc_step_timed: no state has been set");
  cudaStream_t s = (cudaStream_t)stream;
  return h->fp32 ? do_step_timed<float>(h, nsteps, ms_row, ms_col, s)
                 : do_step_timed<double>(h, nsteps, ms_row, ms_col, s);
}

int pfc_reduce(pfc_plan* h, double* out3, void* stream) {
  if (!h || !out3) return fail(PFC_E_ARG, "pfc_reduce: null argument");
  if (!h->state_set) return fail(PFC_E_STATE, "pfc_reduce: no state has been set");
  cudaStream_t s = (cudaStream_t)stream;
  return h->fp32 ? do_reduce<float>(h, out3, s) : do_reduce<double>(h, out3, s);
}

int pfc_get_field(pfc_plan* h, int which, double w, double* field, void* stream) {
  if (!h || !field) return fail(PFC_E_ARG, "pfc_get_field: null argument");
  if (!h->state_set) return fail(PFC_E_STATE, "pfc_get_field: no state has been set");
  if (reinterpret_cast<uintptr_t>(field) % 16)
    return fail(PFC_E_ARG, "pfc_get_field: field must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  return h->fp32 ? do_get_field<float>(h, which, w, field, s) : do_get_field<double>(h, which, w, field, s);
}

int pfc_get_spectrum(pfc_plan* h, int which, double* out, void* stream) {
  if (!h || !out) return fail(PFC_E_ARG, "pfc_get_spectrum: null argument");
  if (!h->state_set) return fail(PFC_E_STATE, "pfc_get_spectrum: no state has been set");
  if (which != PFC_SPEC_N_HAT && which != PFC_SPEC_N_HAT_NOW)
    return fail(PFC_E_ARG, "pfc_get_spectrum: unknown spectrum %d", which);
  cudaStream_t s = (cudaStream_t)stream;
  return h->fp32 ? do_get_spectrum<float>(h, which, out, s) : do_get_spectrum<double>(h, which, out, s);
}

int pfc_get_coefficients(pfc_plan* h, double* a, double* bg) {
  if (!h) return fail(PFC_E_ARG, "pfc_get_coefficients: null plan");
  const size_t n = h->hostA.size();
  if (a) memcpy(a, h->hostA.data(), n * sizeof(double));
  if (bg) memcpy(bg, h->hostBg.data(), n * sizeof(double));
  return PFC_OK;
}

int pfc_status(pfc_plan* h, int32_t* out) {
  if (!h || !out) return fail(PFC_E_ARG, "pfc_status: null argument");
  int v = 0;
  PFC_CUDA(cudaMemcpy(&v, h->status, sizeof(int), cudaMemcpyDeviceToHost));
  *out = v;
  return PFC_OK;
}

int pfc_plan_info(pfc_plan* h, int64_t* o) {
  if (!h || !o) return fail(PFC_E_ARG, "pfc_plan_info: null argument");
  o[0] = h->rows; o[1] = h->row_tpf; o[2] = h->row_grid;
  o[3] = h->cols; o[4] = h->col_tpf; o[5] = h->col_grid;
  o[6] = (int64_t)h->row_smem; o[7] = (int64_t)h->col_smem;
  o[8] = h->fast ? 1 : 0;
  o[9] = h->fr_rows; o[10] = h->fr_threads; o[11] = h->fr_grid; o[12] = (int64_t)h->fr_smem;
  o[13] = h->fc_threads; o[14] = h->fc_grid; o[15] = (int64_t)h->fc_smem;
  return PFC_OK;
}

int64_t pfc_launch_count(pfc_plan* h) { return h ? h->launches : 0; }

int pfc_plan_variant(pfc_plan* h, int32_t* o) {
  if (!h || !o) return fail(PFC_E_ARG, "pfc_plan_variant: null argument");
  o[0] = h->fast ? h->ee_row : 0;
  o[1] = h->fast ? h->ee_col : 0;
  o[2] = h->fast ? h->fr_rows : 0;
  // fast: 1 one-lane kernels, 2 packed row and column, 3 packed row only, 4 packed column only
  o[3] = !h->fast ? 0 : h->packed_row && h->packed_col ? 2 : h->packed_row ? 3 : h->packed_col ? 4 : 1;
  return PFC_OK;
}

int pfc_plan_path(pfc_plan* h, int32_t* path) {
  if (!h || !path) return fail(PFC_E_ARG, "pfc_plan_path: null argument");
  *path = h->onecta ? PFC_PATH_ONE_CTA
          : h->fast ? ((ilog2_exact(h->m) >= 0 && ilog2_exact(h->ny) >= 0) ? PFC_PATH_POW2 : PFC_PATH_FAST_MIXED)
                    : PFC_PATH_MIXED_RADIX;
  return PFC_OK;
}

int pfc_batch_create(pfc_plan* const* plans, int32_t count, pfc_batch** out) {
  if (!plans || count <= 0 || !out) return fail(PFC_E_ARG, "pfc_batch_create: need plans and an output");
  *out = nullptr;
  for (int i = 0; i < count; ++i) {
    if (!plans[i]) return fail(PFC_E_ARG, "pfc_batch_create: null plan %d", i);
    if (plans[i]->fp32 != plans[0]->fp32) return fail(PFC_E_ARG, "pfc_batch_create: plans mix precisions");
    if (plans[i]->device != plans[0]->device) return fail(PFC_E_ARG, "pfc_batch_create: plans on different devices");
    if (plans[i]->extv) return fail(PFC_E_ARG, "pfc_batch_create: plans with an external potential step alone");
    for (int j = 0; j < i; ++j)
      if (plans[j] == plans[i]) return fail(PFC_E_ARG, "pfc_batch_create: plan %d appears twice", i);
  }
  if (count > 65535) return fail(PFC_E_ARG, "pfc_batch_create: at most 65535 plans");
  pfc_batch* b = new pfc_batch();
  b->fp32 = plans[0]->fp32;
  for (int i = 0; i < count; ++i) {
    pfc_plan* h = plans[i];
    pfc_batch_class* cls = nullptr;
    for (auto& c : b->classes) {
      // everything the step kernels take from the plan besides the per-plan table entries
      const pfc_plan* r = c.plans[0];
      // (mixed-radix plans of one size and precision share the FFT description, twiddle
      // tables and launch shape, all of which come from plans[0] of the class)
      if (r->fast == h->fast && r->onecta == h->onecta && r->fast_row_fn == h->fast_row_fn &&
          r->fast_col_fn == h->fast_col_fn && r->packed_row == h->packed_row && r->fr_rows == h->fr_rows &&
          r->fc_threads == h->fc_threads &&
          r->row_rset == h->row_rset && r->col_rset == h->col_rset && r->prob.model == h->prob.model &&
          r->nx == h->nx && r->ny == h->ny && r->prob.g == h->prob.g && r->prob.clamp_log == h->prob.clamp_log &&
          r->prob.min_phi == h->prob.min_phi) {
        cls = &c;
        break;
      }
    }
    if (!cls) {
      b->classes.emplace_back();
      cls = &b->classes.back();
    }
    cls->plans.push_back(h);
  }
  cudaError_t es = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (auto& c : b->classes) {
    if (es == cudaSuccess) es = cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking);
    if (es == cudaSuccess) es = cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming);
  }
  if (es != cudaSuccess) {
    pfc_batch_destroy(b);
    return fail(PFC_E_CUDA, "pfc_batch_create: %s", cudaGetErrorString(es));
  }
  for (auto& c : b->classes) {
    const size_t n = c.plans.size();
    std::vector<BatchBufs> host(n);
    for (int p = 0; p < 2; ++p) {
      for (size_t i = 0; i < n; ++i) {
        pfc_plan* h = c.plans[i];
        host[i].w = h->W;
        host[i].v = h->V;
        host[i].nin = h->nhat[p];
        host[i].nout = h->nhat[p ^ 1];
        host[i].nin_lo = h->nhat_lo[p];
        host[i].nout_lo = h->nhat_lo[p ^ 1];
        host[i].coef = h->coef;
        host[i].coef64 = h->coef64;
        host[i].scal = h->scal;
      }
      cudaError_t e = cudaMalloc(&c.table[p], n * sizeof(BatchBufs));
      if (e == cudaSuccess) e = cudaMemcpy(c.table[p], host.data(), n * sizeof(BatchBufs), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        pfc_batch_destroy(b);
        return fail(PFC_E_CUDA, "pfc_batch_create: %s", cudaGetErrorString(e));
      }
    }
  }
  *out = b;
  return PFC_OK;
}

int pfc_batch_step(pfc_batch* b, int64_t nsteps, void* stream) {
  if (!b) return fail(PFC_E_ARG, "pfc_batch_step: null batch");
  if (nsteps < 0) return fail(PFC_E_ARG, "pfc_batch_step: negative step count");
  if (nsteps == 0) return PFC_OK;
  cudaStream_t s = (cudaStream_t)stream;
  return b->fp32 ? do_batch_step<float>(b, nsteps, s) : do_batch_step<double>(b, nsteps, s);
}

int pfc_batch_destroy(pfc_batch* b) {
  if (!b) return PFC_OK;
  for (auto& g : b->graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto& c : b->classes) {
    for (auto& tb : c.table)
      if (tb) cudaFree(tb);
    if (c.done) cudaEventDestroy(c.done);
    if (c.stream) cudaStreamDestroy(c.stream);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  delete b;
  return PFC_OK;
}

int64_t pfc_batch_launch_count(pfc_batch* b) { return b ? b->launches : 0; }

int pfc_batch_classes(pfc_batch* b) { return b ? (int)b->classes.size() : 0; }

}  // extern "C"

// ---------------------------------------------------------------------------
// pfc_field_mean_noalloc: the compensated mean of a real FP64 field, with its
// per-CTA partial sums in a fixed device array instead of memory it allocates.
namespace {

constexpr int kNoallocThreads = 256;
constexpr int kNoallocChunk = kNoallocThreads * 32;     // contiguous sites per CTA
constexpr int kNoallocMaxBlocks = 8192;                 // CTA partials the array holds
constexpr long long kNoallocMaxSites = (long long)kNoallocChunk * kNoallocMaxBlocks;  // 2^26 = 8192 x 8192
constexpr int kNoallocMaxDevices = 64;

// (sum, compensation) of CTA b at [2b, 2b + 2); the completion counter (an unsigned
// int) at [2 * kNoallocMaxBlocks]. 128 KiB + 256 B on every GPU that loads the library.
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoallocMaxBlocks + 32];

// Each CTA sums one chunk, the last CTA to finish merges the partials in CTA order
// (the result does not depend on which CTA that is) and puts the counter back to 0.
__global__ void __launch_bounds__(kNoallocThreads)
noalloc_mean_kernel(const double* __restrict__ x, long long n, double inv_n, double* scratch, double* out) {
  KSum acc[1] = {{0.0, 0.0}};
  const long long base = (long long)blockIdx.x * kNoallocChunk;
  const long long end = base + kNoallocChunk < n ? base + kNoallocChunk : n;
  for (long long i = base + threadIdx.x; i < end; i += kNoallocThreads) ksum_add(acc[0], x[i]);
  block_reduce_store<1>(acc, scratch + 2 * blockIdx.x);  // thread 0 writes the pair
  unsigned int* done = reinterpret_cast<unsigned int*>(scratch + 2 * kNoallocMaxBlocks);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  const volatile double* p = scratch;
  KSum tot = {0.0, 0.0};
  for (unsigned int b = 0; b < gridDim.x; ++b) {
    KSum o = {p[2 * b], p[2 * b + 1]};
    tot = ksum_merge(tot, o);
  }
  out[0] = (tot.s + tot.c) * inv_n;
  *done = 0u;
}

std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kNoallocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once per device.
int noalloc_scratch(double** out) {
  int dev = 0;
  PFC_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocMaxDevices)
    return fail(PFC_E_ARG, "pfc_field_mean_noalloc: device %d is beyond the %d devices it supports", dev,
                kNoallocMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(PFC_E_CUDA, "pfc_field_mean_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                  cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return PFC_OK;
}

}  // namespace

extern "C" int pfc_field_mean_noalloc(const double* dev_field, int64_t count, double* dev_mean, void* stream) {
  if (!dev_field || !dev_mean) return fail(PFC_E_ARG, "pfc_field_mean_noalloc: null argument");
  if (count <= 0) return fail(PFC_E_ARG, "pfc_field_mean_noalloc: count must be positive, got %lld", (long long)count);
  if (count > kNoallocMaxSites)
    return fail(PFC_E_ARG,
                "pfc_field_mean_noalloc: %lld sites exceed the maximum of %lld (an 8192 x 8192 field) "
                "that its fixed scratch array holds",
                (long long)count, kNoallocMaxSites);
  double* scratch = nullptr;
  if (int rc = noalloc_scratch(&scratch)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  // the completion counter must start at zero
  PFC_CUDA(cudaMemsetAsync(scratch + 2 * kNoallocMaxBlocks, 0, sizeof(unsigned int), s));
  const int blocks = (int)((count + kNoallocChunk - 1) / kNoallocChunk);
  noalloc_mean_kernel<<<blocks, kNoallocThreads, 0, s>>>(dev_field, (long long)count, 1.0 / (double)count, scratch,
                                                         dev_mean);
  PFC_LAUNCHED();
  return PFC_OK;
}

extern "C" int pfc_locate_vacancies(const double* dev_field, int32_t nx, int32_t ny, double dx, double dy,
                                    double* dev_xy, int32_t count, int32_t* dev_status, void* stream) {
  if (count < 0) return fail(PFC_E_ARG, "pfc_locate_vacancies: count %d < 0", count);
  if (nx < 1 || ny < 1) return fail(PFC_E_ARG, "pfc_locate_vacancies: grid %d x %d", nx, ny);
  if (!(dx > 0.0) || !(dy > 0.0) || !std::isfinite(dx) || !std::isfinite(dy))
    return fail(PFC_E_ARG, "pfc_locate_vacancies: spacings dx = %g, dy = %g must be finite and > 0", dx, dy);
  if (count == 0) return PFC_OK;
  if (!dev_field || !dev_xy || !dev_status) return fail(PFC_E_ARG, "pfc_locate_vacancies: null pointer");
  cudaError_t e = launch_locate_vacancies(dev_field, nx, ny, dx, dy, dev_xy, count, dev_status,
                                          static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(PFC_E_CUDA, "pfc_locate_vacancies: launch failed: %s", cudaGetErrorString(e));
  return PFC_OK;
}

extern "C" int pfc_diagnose_modes(pfc_plan* h, const double* dev_field, const double* dev_spectrum,
                                  const int32_t* mode_rc, const int32_t* mode_set, int32_t n_modes,
                                  double amplitude_sign, double* dev_out6, void* stream) {
  if (!h) return fail(PFC_E_ARG, "pfc_diagnose_modes: null plan");
  if (!dev_field || !dev_spectrum || !dev_out6) return fail(PFC_E_ARG, "pfc_diagnose_modes: null device pointer");
  if (n_modes < 0 || n_modes > kDiagMaxModes)
    return fail(PFC_E_ARG, "pfc_diagnose_modes: %d modes (0 .. %d)", n_modes, kDiagMaxModes);
  if (n_modes > 0 && (!mode_rc || !mode_set)) return fail(PFC_E_ARG, "pfc_diagnose_modes: null mode table");
  if (h->npartials < (size_t)diagnose_partials_needed())
    return fail(PFC_E_STATE, "pfc_diagnose_modes: plan scratch too small");
  const int nx = h->nx, ny = h->ny, nxh = nx / 2 + 1;
  DiagModes m{};
  m.sign = amplitude_sign;
  // the rebuilt spectrum as _build3Mode assigns it: the DC entry, then the 1-, 2- and
  // 3-mode sets in turn, a later assignment to an entry replacing an earlier one
  m.uniq_flat[0] = 0;
  m.uniq_set[0] = -1;
  m.uniq_w[0] = 1.0;
  m.n_uniq = 1;
  for (int s = 0; s < 3; ++s)
    for (int i = 0; i < n_modes; ++i) {
      if (mode_set[i] < 0 || mode_set[i] > 2)
        return fail(PFC_E_ARG, "pfc_diagnose_modes: mode %d has set %d (0, 1 or 2)", i, mode_set[i]);
      if (mode_set[i] != s) continue;
      const int r = mode_rc[2 * i], c = mode_rc[2 * i + 1];
      const int rw = r < 0 ? r + ny : r, cw = c < 0 ? c + nxh : c;
      if (rw < 0 || rw >= ny || cw < 0 || cw >= nxh)
        return fail(PFC_E_ARG, "pfc_diagnose_modes: mode (%d, %d) lies outside the %d x %d half spectrum", r, c, ny,
                    nxh);
      const int flat = rw * nxh + cw;
      int e = 0;
      while (e < m.n_uniq && m.uniq_flat[e] != flat) ++e;
      if (e == m.n_uniq) {
        m.uniq_flat[e] = flat;
        m.uniq_w[e] = (cw == 0 || (nx % 2 == 0 && cw == nx / 2)) ? 1.0 : 2.0;
        ++m.n_uniq;
      }
      m.uniq_set[e] = s;
    }
  // the entries each set's amplitude averages, repeats included, in the given order
  for (int i = 0; i < n_modes; ++i) {
    const int r = mode_rc[2 * i], c = mode_rc[2 * i + 1];
    m.list_flat[i] = (r < 0 ? r + ny : r) * nxh + (c < 0 ? c + nxh : c);
    m.list_set[i] = mode_set[i];
  }
  m.n_list = n_modes;
  cudaError_t e = launch_diagnose_modes(dev_field, dev_spectrum, nx, ny, m, h->partials, dev_out6,
                                        static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(PFC_E_CUDA, "pfc_diagnose_modes: launch failed: %s", cudaGetErrorString(e));
  return PFC_OK;
}

extern "C" int pfc_frozen_moments(pfc_plan* h, const double* dev_field, const double* dev_spectrum, double lx_ref,
                                  double ly_ref, double temp, double g, double v0, double* dev_out4, void* stream) {
  if (!h) return fail(PFC_E_ARG, "pfc_frozen_moments: null plan");
  if (!dev_field || !dev_spectrum || !dev_out4) return fail(PFC_E_ARG, "pfc_frozen_moments: null device pointer");
  if (!(lx_ref > 0.0) || !(ly_ref > 0.0) || !std::isfinite(lx_ref) || !std::isfinite(ly_ref))
    return fail(PFC_E_ARG, "pfc_frozen_moments: box %g x %g must be finite and > 0", lx_ref, ly_ref);
  if (h->npartials < (size_t)diagnose_partials_needed())
    return fail(PFC_E_STATE, "pfc_frozen_moments: plan scratch too small");
  // NumPy's fftfreq(n, d = L / n) spacing: 1 / (n * d)
  const double fx = 1.0 / (h->nx * (lx_ref / h->nx)), fy = 1.0 / (h->ny * (ly_ref / h->ny));
  cudaError_t e = launch_frozen_moments(dev_field, dev_spectrum, h->nx, h->ny, fx, fy, temp, g, v0, h->partials,
                                        dev_out4, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(PFC_E_CUDA, "pfc_frozen_moments: launch failed: %s", cudaGetErrorString(e));
  return PFC_OK;
}

extern "C" int pfc_defect_screen(pfc_plan* h, const double* dev_field, const double* dev_spectrum, double lx_ref,
                                 double ly_ref, double* dev_out4, void* stream) {
  if (!h) return fail(PFC_E_ARG, "pfc_defect_screen: null plan");
  if (!dev_field || !dev_spectrum || !dev_out4) return fail(PFC_E_ARG, "pfc_defect_screen: null device pointer");
  if (!(lx_ref > 0.0) || !(ly_ref > 0.0) || !std::isfinite(lx_ref) || !std::isfinite(ly_ref))
    return fail(PFC_E_ARG, "pfc_defect_screen: box %g x %g must be finite and > 0", lx_ref, ly_ref);
  if (h->npartials < (size_t)diagnose_partials_needed())
    return fail(PFC_E_STATE, "pfc_defect_screen: plan scratch too small");
  const double fx = 1.0 / (h->nx * (lx_ref / h->nx)), fy = 1.0 / (h->ny * (ly_ref / h->ny));
  cudaError_t e = launch_defect_screen(dev_field, dev_spectrum, h->nx, h->ny, fx, fy, h->partials, dev_out4,
                                       static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(PFC_E_CUDA, "pfc_defect_screen: launch failed: %s", cudaGetErrorString(e));
  return PFC_OK;
}

// ---- log PFC with an external potential
extern "C" int pfc_set_potential(pfc_plan* h, const double* dev_v, void* stream) {
  if (!h || !dev_v) return fail(PFC_E_ARG, "pfc_set_potential: null argument");
  if (!h->extv) return fail(PFC_E_ARG, "pfc_set_potential: the plan was not created with PFC_FLAG_EXTV");
  if (reinterpret_cast<uintptr_t>(dev_v) % 16) return fail(PFC_E_ARG, "pfc_set_potential: V must be 16-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  if (!h->W2) PFC_CUDA(cudaMalloc(&h->W2, h->nspec * h->elt));
  if (!h->scratch_state) PFC_CUDA(cudaMalloc(&h->scratch_state, h->nspec * sizeof(double2)));
  // rfft2 of V through the plan's own forward transform: row pass into W2, column pass
  // into the scratch state, exported unpacked as (ny, m + 1)
  RowArgs<double> ra = row_args<double>(h);
  ra.in_real = dev_v;
  ra.out = reinterpret_cast<cplx<double>*>(h->W2);
  int rc = launch_row<double, kRowForward>(h, ra, s);
  if (rc) return rc;
  ColArgs<double> ca = col_args<double>(h);
  ca.in = reinterpret_cast<const cplx<double>*>(h->W2);
  ca.nout = h->scratch_state;
  ca.wout = reinterpret_cast<cplx<double>*>(h->W2);
  rc = launch_col<double, kColInit>(h, ca, s);
  if (rc) return rc;
  ColArgs<double> ce = col_args<double>(h);
  ce.sin = h->scratch_state;
  ce.out_c128 = reinterpret_cast<double*>(h->vhat);
  rc = launch_col<double, kColExport>(h, ce, s);
  if (rc) return rc;
  // the next step rebuilds the forcing B lap V_hat
  PFC_CUDA(cudaMemsetAsync(&h->extv_st->v_dirty, 0xff, sizeof(int), s));
  return PFC_OK;
}

extern "C" int pfc_extv_state(pfc_plan* h, double* out6) {
  if (!h || !out6) return fail(PFC_E_ARG, "pfc_extv_state: null argument");
  if (!h->extv) return fail(PFC_E_ARG, "pfc_extv_state: the plan was not created with PFC_FLAG_EXTV");
  ExtvState st{};
  PFC_CUDA(cudaMemcpy(&st, h->extv_st, sizeof(st), cudaMemcpyDeviceToHost));
  out6[0] = st.M;
  out6[1] = st.init ? st.phi_min : NAN;
  out6[2] = st.init ? st.phi_max : NAN;
  out6[3] = st.last_min;
  out6[4] = st.last_max;
  out6[5] = (double)st.count;
  return PFC_OK;
}

extern "C" int pfc_extv_set_tolerances(pfc_plan* h, double floor_tol, double ceiling_tol) {
  if (!h) return fail(PFC_E_ARG, "pfc_extv_set_tolerances: null plan");
  if (!h->extv) return fail(PFC_E_ARG, "pfc_extv_set_tolerances: the plan was not created with PFC_FLAG_EXTV");
  if (!(floor_tol >= 0) || !(ceiling_tol >= 0)) return fail(PFC_E_ARG, "pfc_extv_set_tolerances: negative tolerance");
  ExtvState st{};
  PFC_CUDA(cudaMemcpy(&st, h->extv_st, sizeof(st), cudaMemcpyDeviceToHost));
  st.floor_tol = floor_tol;
  st.ceil_tol = ceiling_tol;
  PFC_CUDA(cudaMemcpy(h->extv_st, &st, sizeof(st), cudaMemcpyHostToDevice));
  return PFC_OK;
}

extern "C" int pfc_test_tma_wait(pfc_plan* h, int32_t extra_bytes, int32_t wait_limit) {
  if (!h) return fail(PFC_E_ARG, "pfc_test_tma_wait: null plan");
  if (!h->tma_box) return fail(PFC_E_ARG, "pfc_test_tma_wait: the plan's row pass is not staged by TMA");
  if (extra_bytes < 0 || extra_bytes % 16 || wait_limit < 0)
    return fail(PFC_E_ARG, "pfc_test_tma_wait: extra bytes must be a non-negative multiple of 16, limit >= 0");
  h->tma_extra_tx = (unsigned)extra_bytes;
  h->tma_wait_limit = wait_limit;
  // graphs recorded with the old arguments would replay them
  for (auto& g : h->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto& g : h->graph1)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return PFC_OK;
}

// ---------------------------------------------------------------------------
// Work-queue batches: the members' row and column tiles of a block of steps as the items
// of one cooperative launch (pfc_queue.cuh).
namespace {

constexpr size_t kQueueSmemMax = 48 * 1024;
constexpr int kQueueItemsPerPass = 8;

// Why plan h cannot join a work-queue batch, or nullptr.
const char* queue_refusal(const pfc_plan* h) {
  const int lr = ilog2_exact(h->m), lc = ilog2_exact(h->ny);
  if (lr < 0 || lc < 0) return "the work-queue kernel steps power-of-two grids";
  if (!h->fast || h->packed || h->onecta || h->extv) return "plans must use the one-lane power-of-two step kernels";
  if (h->prob.model != PFC_MODEL_STD) return "the work-queue kernel steps stdPFC plans";
  if (lr < kQueueMinLogRow || lr > kQueueMaxLogRow || lc < kQueueMinLogCol || lc > kQueueMaxLogCol)
    return "grid sides must be 64 .. 1024";
  if (h->ee_row != queue_row_ee(!h->fp32, h->m) || h->ee_col != queue_col_ee(!h->fp32, h->ny))
    return "the plan's values per thread differ from the work-queue kernel's";
  if (h->fr_threads > kQueueThreads || h->fc_threads > kQueueThreads || h->fr_threads % 32 || h->fc_threads % 32)
    return "a pass's CTA is not whole warps of at most 256 threads";
  if (h->fr_smem > kQueueSmemMax || h->fc_smem > kQueueSmemMax) return "a pass needs more than 48 KiB of shared memory";
  return nullptr;
}

template <class T>
int queue_build(pfc_queue* q) {
  const int n = (int)q->plans.size();
  // classes: the batch's (everything the kernels take from the plan besides the table)
  for (int i = 0; i < n; ++i) {
    const pfc_plan* h = q->plans[i];
    int c = 0;
    for (; c < (int)q->classes.size(); ++c) {
      const pfc_plan* r = q->plans[q->classes[c][0]];
      if (r->fast_row_fn == h->fast_row_fn && r->fast_col_fn == h->fast_col_fn && r->fr_rows == h->fr_rows &&
          r->fc_threads == h->fc_threads && r->nx == h->nx && r->ny == h->ny && r->prob.g == h->prob.g &&
          r->prob.clamp_log == h->prob.clamp_log && r->prob.min_phi == h->prob.min_phi)
        break;
    }
    if (c == (int)q->classes.size()) q->classes.emplace_back();
    q->classes[c].push_back(i);
  }
  const int ncls = (int)q->classes.size();
  std::vector<QueueClass<T>> host(ncls);
  std::vector<int4> items;
  for (int c = 0; c < ncls; ++c) {
    const std::vector<int>& mem = q->classes[c];
    const pfc_plan* r = q->plans[mem[0]];
    QueueClass<T>& k = host[c];
    k.row = fast_row_args<T>(r, nullptr);
    k.col = fast_col_args<T>(r, nullptr);
    k.row_log = ilog2_exact(r->m);
    k.col_log = ilog2_exact(r->ny);
    k.row_threads = r->fr_threads;
    k.col_threads = r->fc_threads;
    // a few items per member and pass: each item pays one dependency check and one
    // completion, and a pass of more, smaller items gains little from the finer grain
    k.row_group = std::max(1, r->fr_grid / kQueueItemsPerPass);
    k.col_group = std::max(1, r->fc_grid / kQueueItemsPerPass);
    k.row_items = r->fr_grid / k.row_group;
    k.col_items = r->fc_grid / k.col_group;
    q->smem = std::max(q->smem, std::max(r->fr_smem, r->fc_smem));
    for (int p = 0; p < 2; ++p) {
      std::vector<BatchBufs> tb(mem.size());
      for (size_t j = 0; j < mem.size(); ++j) {
        const pfc_plan* h = q->plans[mem[j]];
        tb[j].w = h->W;
        tb[j].v = h->V;
        tb[j].nin = h->nhat[p];
        tb[j].nout = h->nhat[p ^ 1];
        tb[j].nin_lo = h->nhat_lo[p];
        tb[j].nout_lo = h->nhat_lo[p ^ 1];
        tb[j].coef = h->coef;
        tb[j].coef64 = h->coef64;
        tb[j].scal = h->scal;
      }
      void* d = nullptr;
      PFC_CUDA(cudaMalloc(&d, tb.size() * sizeof(BatchBufs)));
      q->tables.push_back(d);
      PFC_CUDA(cudaMemcpy(d, tb.data(), tb.size() * sizeof(BatchBufs), cudaMemcpyHostToDevice));
      k.table[p] = static_cast<const BatchBufs*>(d);
    }
  }
  // one step: every row tile (class by class), then every column tile
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) q->first_col_item = (int)items.size();
    for (int c = 0; c < ncls; ++c)
      for (size_t j = 0; j < q->classes[c].size(); ++j) {
        const int nit = pass ? host[c].col_items : host[c].row_items;
        for (int t = 0; t < nit; ++t)
          items.push_back(make_int4(q->classes[c][j], c, (int)j, t | (pass ? kQueueColBit : 0)));
      }
  }
  q->nitems = (int)items.size();
  PFC_CUDA(cudaMalloc(&q->cls_dev, ncls * sizeof(QueueClass<T>)));
  PFC_CUDA(cudaMemcpy(q->cls_dev, host.data(), ncls * sizeof(QueueClass<T>), cudaMemcpyHostToDevice));
  PFC_CUDA(cudaMalloc(&q->items, items.size() * sizeof(int4)));
  PFC_CUDA(cudaMemcpy(q->items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
  PFC_CUDA(cudaMalloc(&q->counters, (2 * (size_t)n + 1) * sizeof(unsigned)));
  PFC_CUDA(cudaMalloc(&q->flags, 2 * sizeof(int)));
  PFC_CUDA(cudaMemset(q->flags, 0, 2 * sizeof(int)));
  q->fn = QueueInst<T>::kernel();
  PFC_CUDA(cudaFuncSetAttribute(q->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)q->smem));
  int dev = 0, n_sm = 0;
  PFC_CUDA(cudaGetDevice(&dev));
  PFC_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  PFC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&q->per_sm, q->fn, kQueueThreads, q->smem));
  if (q->per_sm < 1) return fail(PFC_E_ARG, "pfc_queue_create: the work-queue kernel does not fit an SM");
  q->grid = q->per_sm * n_sm;
  return PFC_OK;
}

template <class T>
int queue_launch(pfc_queue* q, int parity, int nsteps, cudaStream_t s) {
  const size_t n = q->plans.size();
  PFC_CUDA(cudaMemsetAsync(q->counters, 0, (2 * n + 1) * sizeof(unsigned), s));
  PFC_CUDA(cudaMemsetAsync(q->flags + 1, 0, sizeof(int), s));
  QueueArgs<T> a{};
  a.classes = static_cast<const QueueClass<T>*>(q->cls_dev);
  a.items = q->items;
  a.nitems = q->nitems;
  a.nsteps = nsteps;
  a.parity0 = parity;
  a.rows_done = q->counters;
  a.cols_done = q->counters + n;
  a.ticket = q->counters + 2 * n;
  a.status = q->flags;
  a.abort = q->flags + 1;
  a.wait_limit = q->wait_limit;
  a.extra_item = q->extra ? q->first_col_item : -1;
  a.extra = q->extra;
  void* args[] = {(void*)&a};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(q->grid);
  cfg.blockDim = dim3(kQueueThreads);
  cfg.dynamicSmemBytes = q->smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelExC(&cfg, q->fn, args);
  ++q->launches;
  if (e != cudaSuccess) return fail(PFC_E_CUDA, "work-queue launch failed: %s", cudaGetErrorString(e));
  return PFC_OK;
}

template <class T>
int do_queue_step(pfc_queue* q, long long nsteps, cudaStream_t s) {
  const int parity = q->plans[0]->cur;
  for (pfc_plan* h : q->plans) {
    if (!h->state_set) return fail(PFC_E_STATE, "pfc_queue_step: a plan has no state");
    if (h->cur != parity)
      return fail(PFC_E_STATE, "pfc_queue_step: plans must have taken the same number of steps mod 2");
  }
  const long long blocks = nsteps / kGraphBlock;
  if (blocks > 0) {
    if (!q->graph[parity]) {
      const long long launches = q->launches;
      int rc = capture_graph([&](cudaStream_t cs) { return queue_launch<T>(q, parity, kGraphBlock, cs); },
                             &q->graph[parity]);
      q->launches = launches;
      if (rc) return rc;
    }
    for (long long k = 0; k < blocks; ++k) {
      cudaError_t e = cudaGraphLaunch(q->graph[parity], s);
      if (e != cudaSuccess) return fail(PFC_E_CUDA, "cudaGraphLaunch failed: %s", cudaGetErrorString(e));
    }
    q->launches += blocks;
  }
  const long long rest = nsteps - blocks * kGraphBlock;   // kGraphBlock is even: parity unchanged
  if (rest > 0) {
    int rc = queue_launch<T>(q, parity, (int)rest, s);
    if (rc) return rc;
  }
  for (pfc_plan* h : q->plans) {
    h->cur ^= (int)(nsteps & 1);
    h->steps_since_set += nsteps;
  }
  return PFC_OK;
}

void queue_drop_graphs(pfc_queue* q) {
  for (auto& g : q->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

}  // namespace

extern "C" int pfc_queue_destroy(pfc_queue* q) {
  if (!q) return PFC_OK;
  queue_drop_graphs(q);
  for (void* t : q->tables)
    if (t) cudaFree(t);
  if (q->cls_dev) cudaFree(q->cls_dev);
  if (q->items) cudaFree(q->items);
  if (q->counters) cudaFree(q->counters);
  if (q->flags) cudaFree(q->flags);
  delete q;
  return PFC_OK;
}

extern "C" int pfc_queue_create(pfc_plan* const* plans, int32_t count, pfc_queue** out) {
  if (!plans || count <= 0 || !out) return fail(PFC_E_ARG, "pfc_queue_create: need plans and an output");
  *out = nullptr;
  for (int i = 0; i < count; ++i) {
    if (!plans[i]) return fail(PFC_E_ARG, "pfc_queue_create: null plan %d", i);
    if (plans[i]->fp32 != plans[0]->fp32) return fail(PFC_E_ARG, "pfc_queue_create: plans mix precisions");
    if (plans[i]->device != plans[0]->device) return fail(PFC_E_ARG, "pfc_queue_create: plans on different devices");
    if (const char* why = queue_refusal(plans[i])) return fail(PFC_E_ARG, "pfc_queue_create: plan %d: %s", i, why);
    for (int j = 0; j < i; ++j)
      if (plans[j] == plans[i]) return fail(PFC_E_ARG, "pfc_queue_create: plan %d appears twice", i);
  }
  pfc_queue* q = new pfc_queue();
  q->fp32 = plans[0]->fp32;
  q->plans.assign(plans, plans + count);
  const int rc = q->fp32 ? queue_build<float>(q) : queue_build<double>(q);
  if (rc) {
    pfc_queue_destroy(q);
    return rc;
  }
  *out = q;
  return PFC_OK;
}

extern "C" int pfc_queue_step(pfc_queue* q, int64_t nsteps, void* stream) {
  if (!q) return fail(PFC_E_ARG, "pfc_queue_step: null queue");
  if (nsteps < 0) return fail(PFC_E_ARG, "pfc_queue_step: negative step count");
  if (nsteps == 0) return PFC_OK;
  cudaStream_t s = (cudaStream_t)stream;
  return q->fp32 ? do_queue_step<float>(q, nsteps, s) : do_queue_step<double>(q, nsteps, s);
}

extern "C" int pfc_queue_status(pfc_queue* q, int32_t* status) {
  if (!q || !status) return fail(PFC_E_ARG, "pfc_queue_status: null argument");
  PFC_CUDA(cudaDeviceSynchronize());
  int v = 0;
  PFC_CUDA(cudaMemcpy(&v, q->flags, sizeof(int), cudaMemcpyDeviceToHost));
  *status = v;
  return PFC_OK;
}

extern "C" int pfc_queue_info(pfc_queue* q, int32_t* out4) {
  if (!q || !out4) return fail(PFC_E_ARG, "pfc_queue_info: null argument");
  out4[0] = q->grid;
  out4[1] = q->per_sm;
  out4[2] = q->nitems;
  out4[3] = (int32_t)q->classes.size();
  return PFC_OK;
}

extern "C" int64_t pfc_queue_launch_count(pfc_queue* q) { return q ? q->launches : 0; }

extern "C" int pfc_test_queue_wait(pfc_queue* q, int32_t extra, int64_t wait_limit) {
  if (!q) return fail(PFC_E_ARG, "pfc_test_queue_wait: null queue");
  if (extra < 0 || wait_limit < 0) return fail(PFC_E_ARG, "pfc_test_queue_wait: negative argument");
  q->extra = extra;
  q->wait_limit = wait_limit ? wait_limit : kQueueWaitLimit;
  queue_drop_graphs(q);   // graphs recorded with the old arguments would replay them
  return PFC_OK;
}
