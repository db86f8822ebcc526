// Vacancy location on a local (coarse-grained) density field, on the device: the
// computation of the reference's _VacancyTracker.LocateVacancy
// (src/pfc_models/analysis/vacancy_tracker.py:22-60) for many vacancies in one launch,
// so that tracking needs no copy of the field to the host.
//
// One thread per vacancy. The arithmetic is the reference's FP64 sequence with every
// operation rounded on its own (no fused multiply-add), and the index rules are
// NumPy's: the nearest pixel by round-half-to-even, the 3 x 3 neighbourhood as a slice
// cuts it (a negative start wraps, a stop past the end clips, an empty slice is an
// error), the first minimum in row-major order (a NaN, if any, wins), and the 5-point
// cross read with integer indices (-1 wraps, one past the end is an error). Where the
// reference raises, the thread leaves the position unchanged and writes status 1 where
// it raises ValueError (a non-finite position, an empty neighbourhood) or 2 where it
// raises IndexError (a cross neighbour past the last row or column).
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "pfc_registry.h"

namespace pfc {
namespace {

// NumPy integer index on an axis of length n; false where NumPy raises IndexError
__device__ __forceinline__ bool np_index(long long i, long long n, long long* out) {
  const long long j = i < 0 ? i + n : i;
  if (j < 0 || j >= n) return false;
  *out = j;
  return true;
}

// [lo, hi) of the unit-step slice start:stop on an axis of length n (Python's
// slice.indices for step 1)
__device__ __forceinline__ void np_slice(long long start, long long stop, long long n, long long* lo,
                                         long long* hi) {
  if (start < 0) start = start + n < 0 ? 0 : start + n;
  else if (start > n) start = n;
  if (stop < 0) stop = stop + n < 0 ? 0 : stop + n;
  else if (stop > n) stop = n;
  *lo = start;
  *hi = stop > start ? stop : start;
}

__global__ void locate_vacancies_kernel(const double* __restrict__ f, int nx, int ny, double dx, double dy,
                                        double* __restrict__ xy, int count, int32_t* __restrict__ status) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= count) return;
  const double x0 = xy[2 * v], y0 = xy[2 * v + 1];
  status[v] = 1;
  if (!isfinite(x0) || !isfinite(y0)) return;
  const double rx = rint(__ddiv_rn(x0, dx)), ry = rint(__ddiv_rn(y0, dy));
  // far outside any grid: the neighbourhood is empty there, as for any start below -1
  if (fabs(rx) > 4.0e15 || fabs(ry) > 4.0e15) return;
  long long px = (long long)rx, py = (long long)ry;
  const long long NX = nx, NY = ny;
  long long r0, r1, c0, c1;
  np_slice(py - 1, py + 2, NY, &r0, &r1);
  np_slice(px - 1, px + 2, NX, &c0, &c1);
  if (r0 == r1 || c0 == c1) return;
  double best = 0.0;
  long long bi = 0, bj = 0;
  bool have = false;
  for (long long r = r0; r < r1; ++r)
    for (long long c = c0; c < c1; ++c) {
      const double val = f[r * NX + c];
      const bool take = !have || (isnan(val) && !isnan(best)) || (!isnan(best) && val < best);
      if (take) {
        best = val;
        bi = r - r0;
        bj = c - c0;
        have = true;
      }
    }
  py += bi - 1;
  px += bj - 1;
  long long ym, yu, yd, xm, xl, xr;
  if (!np_index(py, NY, &ym) || !np_index(py - 1, NY, &yu) || !np_index(py + 1, NY, &yd) ||
      !np_index(px, NX, &xm) || !np_index(px - 1, NX, &xl) || !np_index(px + 1, NX, &xr)) {
    status[v] = 2;
    return;
  }
  const double f_mid = f[ym * NX + xm];
  const double f_left = f[ym * NX + xl], f_right = f[ym * NX + xr];
  const double f_up = f[yu * NX + xm], f_down = f[yd * NX + xm];
  // 2 (f_left - 2 f_mid + f_right), each operation rounded as the reference rounds it
  const double two_mid = __dmul_rn(2.0, f_mid);
  const double denom_x = __dmul_rn(2.0, __dadd_rn(__dsub_rn(f_left, two_mid), f_right));
  const double denom_y = __dmul_rn(2.0, __dadd_rn(__dsub_rn(f_up, two_mid), f_down));
  const double delta_x = denom_x != 0.0 ? __ddiv_rn(__dsub_rn(f_left, f_right), denom_x) : 0.0;
  const double delta_y = denom_y != 0.0 ? __ddiv_rn(__dsub_rn(f_up, f_down), denom_y) : 0.0;
  xy[2 * v] = __dmul_rn(__dadd_rn((double)px, delta_x), dx);
  xy[2 * v + 1] = __dmul_rn(__dadd_rn((double)py, delta_y), dy);
  status[v] = 0;
}

}  // namespace

cudaError_t launch_locate_vacancies(const double* field, int nx, int ny, double dx, double dy, double* xy,
                                    int count, int32_t* status, cudaStream_t stream) {
  constexpr int kThreads = 128;
  locate_vacancies_kernel<<<(count + kThreads - 1) / kThreads, kThreads, 0, stream>>>(field, nx, ny, dx, dy, xy,
                                                                                      count, status);
  return cudaGetLastError();
}

}  // namespace pfc
