// Kernel lookup across translation units. The step kernels are instantiated in
// several .cu files (one per precision and variant) that compile in parallel; the
// plan code finds them through these functions.
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace pfc {

// Radix-set code of the generic kernels built for 1024-thread blocks, used when one
// transform needs more than 256 threads (>= 8192 points in FP32); kRadixPow2 and
// kRadixAll (pfc_fft.cuh) select the 256-thread kernels.
constexpr int kRadixPow2Big = 2;
// The all-radix step kernels (row and column) built for two CTAs per SM (at most 128
// registers, with some spills) instead of one: faster for large FP32 grids, slower for
// small grids and in FP64 (measured on B200). Modes other than the step use kRadixAll.
constexpr int kRadixAllDense = 3;
// Grids with prime factors 2, 3, 5, 7 only: the smaller radix set (kRadixSmall), and its
// two-CTA step build as above.
constexpr int kRadixSmallDense = 5;
// The small-radix generic kernels built for 1024-thread blocks: transforms whose radix-5 or
// radix-7 pass has more than 256 butterflies (2560 = 5 x 512, 3584 = 7 x 512, 5120 points);
// they hold one butterfly of such a pass per thread, so the block grows with the length.
constexpr int kRadixSmallBig = 6;
constexpr long long kDenseMinSites = 1LL << 20;

// log2 sizes of the power-of-two step kernels: row transforms of M = nx/2 points,
// column transforms of ny points
constexpr int kFastMinLog = 5, kFastMaxLogRow = 12, kFastMaxLogCol = 13;

// Work-queue step kernel of one precision (pfc_queue.cuh; pfc_queue_f32.cu, pfc_queue_f64.cu).
template <class T>
struct QueueInst {
  static void* kernel();
};

struct FastKernel {
  void* fn = nullptr;  // kernel entry, for cudaLaunchKernel
  int tpf = 0;         // threads per transform
};

// Power-of-two step kernels with EE complex values per thread (pfc_fast.cuh).
template <class T, int EE>
struct FastInst {
  static bool row(int lg, int model, FastKernel* out);
  static bool col(int lg, FastKernel* out);
  // appends the pass tables of sequences A and B of a 2^lg-point transform
  static bool tables(int lg, std::vector<long double>& tw, int& offA, int& offB);
};

// Register-resident step kernels for transforms of N = ODD * 2^k points, ODD = 3, 5, 7
// and k = kMixMinLog2 .. kMixMaxLog2 (pfc_fastmix_inst.cuh), by transform length.
constexpr int kMixMinLog2 = 4, kMixMaxLog2 = 9;
template <class T>
struct MixInst {
  static bool row(int n, int model, FastKernel* out);
  static bool col(int n, FastKernel* out);
  static bool tables(int n, std::vector<long double>& tw, int& offA, int& offB);
  static int values_per_thread(int n);
};

// Two-lane packed FP32 step kernels (pfc_pack_step.cuh), `ee` = 8 or 16 complex values
// per lane and thread: row transforms of 2^lg points (M = nx/2), column transforms of
// 2^lg points (ny). Their pass tables are float4 entries (c, c, s, s), appended to `tw`
// as two complex slots each, at even (16-byte aligned) offsets; pack_real_table appends
// the real-packing table exp(-2 pi i k / nx), k < nx/2, in the same form.
constexpr int kPackMinLog = 6, kPackMaxLogRow = 12, kPackMaxLogCol = 13;
bool pack_row(int lg, int ee, int model, FastKernel* out);
bool pack_col(int lg, int ee, FastKernel* out);
bool pack_tables(int lg, int ee, std::vector<long double>& tw, int& offA, int& offB);
void pack_real_table(int nx, std::vector<long double>& tw, int& off);

// Mixed-radix kernels (pfc_kernels.cuh), by mode (kRow* / kCol*) and radix set.
template <class T>
struct GenericInst {
  static void* row(int mode, int model, int rset);
  static void* col(int mode, int rset);
};

// Mode entries of the 3-mode diagnostics (pfc_diag.cu), built on the host from the
// reference's k-vector sets: the list (with repeats) whose |n_hat| each set averages,
// and the distinct entries of the rebuilt spectrum with their half-spectrum weights
// (set -1: the DC entry, which keeps n_hat(0, 0)). Indices are flat in the
// (ny, nx / 2 + 1) half spectrum.
constexpr int kDiagMaxModes = 64;
struct DiagModes {
  double sign;
  int n_list, n_uniq;
  int list_flat[kDiagMaxModes], list_set[kDiagMaxModes];
  int uniq_flat[kDiagMaxModes + 1], uniq_set[kDiagMaxModes + 1];
  double uniq_w[kDiagMaxModes + 1];
};
cudaError_t launch_diagnose_modes(const double* field, const double* spec, int nx, int ny, const DiagModes& m,
                                  double* partials, double* out6, cudaStream_t stream);
cudaError_t launch_frozen_moments(const double* field, const double* spec, int nx, int ny, double fx, double fy,
                                  double temp, double g, double v0, double* partials, double* out4,
                                  cudaStream_t stream);
cudaError_t launch_defect_screen(const double* field, const double* spec, int nx, int ny, double fx, double fy,
                                 double* partials, double* out4, cudaStream_t stream);
int diagnose_partials_needed();

// Whole-grid step kernel for small FP64 mixed-radix grids (pfc_onecta.cu): one CTA per
// plan runs nsteps steps with the grid in shared memory; `table` holds the plans'
// buffers (BatchBufs) at the starting parity, `count` entries.
template <class T> struct RowArgs;
template <class T> struct ColArgs;
struct BatchBufs;
constexpr int kOneCtaMaxThreads = 256;
constexpr size_t kOneCtaMaxSmem = 96 * 1024;   // two CTAs per SM
size_t onecta_smem_bytes(int m, int ny, int row_ld, int col_ld);
cudaError_t onecta_allow_smem(size_t bytes);     // raises the kernels' dynamic shared memory limit
bool onecta_supported(int rset);
cudaError_t launch_onecta_step(const RowArgs<double>& ra, const ColArgs<double>& ca, const BatchBufs* table,
                               int count, long long nsteps, int model, int rset, bool dense, int threads,
                               size_t smem, cudaStream_t stream);

// Log PFC with an external potential (pfc_extv.cu): the state of the M shift, kept in
// device memory, and the arguments of the coefficient rebuild.
struct ExtvState {
  double M, phi_min, phi_max;   // shift and the range it was optimised for
  double floor_tol, ceil_tol;   // relative tolerances of ValidatePhiRange (0.1, 0.1)
  double min_phi;               // replaces a non-positive minimum in OptimizeM
  double last_min, last_max;    // the field's range seen by the last step
  int init, changed, count;
  int v_dirty;                  // nonzero: V changed since the forcing was built
};
struct ExtvCoefArgs {
  int nx, ny, m, nyh;
  double fx, fy, gamma, beta, q0, epsilon, dt, small_z_tol;
  double2* coef;          // (A - 1 - M Bg, Bg), [kx][ky <= ny/2]
  const double2* vhat;    // rfft2 of V, (ny, m + 1) row-major
  double2* forcing;       // B lap V_hat, [kx][ky], kx <= m
};
cudaError_t launch_extv_decide(const double* minmax, int nparts, ExtvState* st, double g, cudaStream_t s);
cudaError_t launch_extv_coef(const ExtvCoefArgs& a, const ExtvState* st, cudaStream_t s);

// Vacancy location on a local density field (pfc_track.cu), count > 0.
cudaError_t launch_locate_vacancies(const double* field, int nx, int ny, double dx, double dy, double* xy,
                                    int count, int32_t* status, cudaStream_t stream);

}  // namespace pfc
