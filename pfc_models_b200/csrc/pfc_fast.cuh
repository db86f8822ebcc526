// Specialised step kernels for power-of-two grids (compile-time transform sizes).
//
// Each transform of length N is owned by a group of TPF = N/EE threads; a thread
// holds EE complex values in registers. Sequence A runs radices (EE, ..., EE, LAST)
// and sequence B (LAST, EE, ..., EE), so that the last pass of A and the first pass
// of B touch the same elements in the same thread: the row kernel applies the
// nonlinearity between them (inverse A, forward B) and the column kernel applies the
// ETD1 update between them (forward A, inverse B) without a shared-memory round trip.
//
// Shared-memory exchanges between passes use the padded index i + (i >> P), one pad
// element per 2^P. Shared memory serves 8-byte accesses per half-warp (16 lanes, bank
// pair = index mod 16) and 16-byte accesses per quarter-warp (8 lanes, index mod 8);
// P is chosen per element size and values per thread so that the Stockham loads and
// stores of every pass need the fewest wavefronts under that rule (fast_pad_shift).
// Every radix R of a sequence satisfies R <= 2^P, so the R consecutive outputs of an
// NS = 1 pass never straddle a pad.
// A transform group synchronises with __syncwarp when it fits in a warp, otherwise
// with its own named barrier, so groups never wait for each other.
#pragma once
#include <cstdint>
#include <type_traits>

#include "pfc_kernels.cuh"

namespace pfc {

// Radix sequence of an N-point transform held EE values per thread. N = ODD * 2^K2 with
// ODD = 1, 3, 5 or 7: EE_REQ is then the power-of-two part of the values per thread
// (EE = ODD * E2), sequence A runs the radix-RC passes of the power-of-two part (the last
// of them radix LAST2) and then one radix-ODD pass, sequence B the same in reverse, so
// that every radix divides EE (each pass gives a thread EE / R whole butterflies) and the
// last pass of A and the first of B still touch the same elements in the same thread.
template <int N, int EE_REQ, int RMAX>
struct FastSeq {
  __host__ __device__ static constexpr int lg(int x) { return x <= 1 ? 0 : 1 + lg(x >> 1); }
  __host__ __device__ static constexpr int ctz(int x) { return (x & 1) ? 0 : 1 + ctz(x >> 1); }
  static constexpr int K2 = ctz(N), ODD = N >> K2;        // N = ODD * 2^K2
  static constexpr int P2 = 1 << K2;
  static constexpr int E2 = EE_REQ < P2 ? EE_REQ : P2;    // power-of-two part of the values per thread
  static constexpr int EE = ODD * E2;                     // elements per thread
  static constexpr int TPF = N / EE;                      // threads per transform
  static constexpr int RC = RMAX < E2 ? RMAX : E2;        // radix of the full power-of-two passes
  static constexpr int LN = K2, LE = lg(RC);
  static constexpr int NP2 = LE > 0 ? (LN + LE - 1) / LE : 0;
  static constexpr int LAST2 = NP2 > 0 ? 1 << (LN - (NP2 - 1) * LE) : 1;
  static constexpr int NPASS = NP2 + (ODD > 1 ? 1 : 0);
  static constexpr int LAST = ODD > 1 ? ODD : LAST2;      // radix of A's last (B's first) pass
  __host__ __device__ static constexpr int radA(int p) {
    return p == NPASS - 1 ? LAST : (p == NP2 - 1 ? LAST2 : RC);
  }
  __host__ __device__ static constexpr int radB(int p) { return radA(NPASS - 1 - p); }
  __host__ __device__ static constexpr int nsA(int p) { return p == 0 ? 1 : nsA(p - 1) * radA(p - 1); }
  __host__ __device__ static constexpr int nsB(int p) { return p == 0 ? 1 : nsB(p - 1) * radB(p - 1); }
  // offset of pass p's twiddle table ([q-1][k], q < R, k < ns) within the sequence table
  __host__ __device__ static constexpr int twA(int p) { return p <= 1 ? 0 : twA(p - 1) + nsA(p - 1) * (radA(p - 1) - 1); }
  __host__ __device__ static constexpr int twB(int p) { return p <= 1 ? 0 : twB(p - 1) + nsB(p - 1) * (radB(p - 1) - 1); }
  __host__ __device__ static constexpr int sizeA() { return twA(NPASS); }
  __host__ __device__ static constexpr int sizeB() { return twB(NPASS); }
  // A and B run the same radices in the same order (all passes of one radix): their pass
  // tables are equal, and the plans keep one copy for both
  __host__ __device__ static constexpr bool symmetric(int p = 0) {
    return p >= NPASS ? true : (radA(p) == radB(p) && symmetric(p + 1));
  }
};

// Pad shift of the exchange buffers for EE values per thread (the effective EE of the
// transform). Complex float: radix-32 passes (EE = 32) need a pad per 32 elements,
// radix-16 and radix-8 passes one per 16; complex double: one per 16 for radix 16,
// one per 8 for radix 8. (With one pad per 32 the radix-16 FP32 column transform
// stored 1.5 wavefronts per 128 bytes in three of its four exchanges.)
__host__ __device__ constexpr int fast_pad_shift(bool fp64, int ee) {
  return fp64 ? (ee >= 16 ? 4 : 3) : (ee >= 32 ? 5 : 4);
}
template <class T, int EE> struct FastPad { static constexpr int value = fast_pad_shift(sizeof(T) == 8, EE); };

template <int P> __device__ __forceinline__ int padi(int i) { return i + (i >> P); }

// largest radix of a pass: 32 complex floats or 16 complex doubles per thread
template <class T> struct RadixCap { static constexpr int value = sizeof(T) == 4 ? 32 : 16; };

__device__ __forceinline__ float2 ldg2(const float2* p) { return __ldg(p); }
__device__ __forceinline__ double2 ldg2(const double2* p) { return __ldg(p); }
template <class T> __device__ __forceinline__ cplx<T> ldgc(const cplx<T>* p) {
  using V = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
  const V v = ldg2(reinterpret_cast<const V*>(p));
  return mk((T)v.x, (T)v.y);
}

// L1 eviction priorities. The step kernels stream every field element through the SM
// once (the row tile's 8-byte asynchronous copies, the column loads), which would evict
// the small twiddle tables that every transform re-reads: the tables are loaded
// evict_last, streamed field data without allocating in L1.
// Tables: written before the first launch and never again, so the load may be moved or
// merged freely.
__device__ __forceinline__ float2 ld_keep(const float2* p) {
  float2 v;
  asm("ld.global.nc.L1::evict_last.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ double2 ld_keep(const double2* p) {
  double2 v;
  asm("ld.global.nc.L1::evict_last.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ float4 ld_keep(const float4* p) {
  float4 v;
  asm("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}
template <class T> __device__ __forceinline__ cplx<T> ldkc(const cplx<T>* p) {
  using V = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
  const V v = ld_keep(reinterpret_cast<const V*>(p));
  return mk((T)v.x, (T)v.y);
}
// Field data read once per launch and not written by it. Volatile: the loads keep their
// place after griddepcontrol.wait (the data is the previous launch's output).
__device__ __forceinline__ float2 ld_stream(const float2* p) {
  float2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ double2 ld_stream(const double2* p) {
  double2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
template <class T> __device__ __forceinline__ cplx<T> ldsc(const cplx<T>* p) {
  using V = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
  const V v = ld_stream(reinterpret_cast<const V*>(p));
  return mk((T)v.x, (T)v.y);
}

// Synchronisation of one transform group (TPF threads, group index g within the CTA).
template <int TPF>
__device__ __forceinline__ void group_sync(int g) {
  if constexpr (TPF < 32) {
    // lanes of this group only, so groups sharing a warp may branch differently
    const unsigned lane0 = (threadIdx.x & 31u) & ~(unsigned)(TPF - 1);
    __syncwarp(((1u << TPF) - 1u) << lane0);
  } else if constexpr (TPF == 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(TPF) : "memory");
  }
}

// One Stockham pass of radix R, stride NS, on a length-N transform whose group has
// TPF threads holding EE = R * NB values each (v[b * R + q], butterfly j = t + b * TPF).
template <class T, int N, int EE, int R, int NS, int P>
struct FastPass {
  static_assert(R <= (1 << P), "the padded exchange assumes radices up to 2^P");
  static constexpr int TPF = N / EE, NB = EE / R, NR = N / R;
  // padi(x + q * S) = padi(x) + q * (S + S / 2^P) whenever 2^P divides S
  static constexpr int NRP = NR + (NR >> P);
  static constexpr bool LIN_LOAD = (NR % (1 << P)) == 0;
  // the R consecutive outputs of an NS = 1 pass stay inside one pad block when R divides 2^P
  static constexpr bool LIN_STORE = (NS % (1 << P)) == 0 || (NS == 1 && ((1 << P) % R) == 0);
  static constexpr int NSP = NS == 1 ? 1 : NS + (NS >> P);
  static __device__ __forceinline__ void load(const cplx<T>* buf, cplx<T>* v, int t) {
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const int j = t + b * TPF;
      if constexpr (LIN_LOAD) {
        const cplx<T>* p = buf + padi<P>(j);
#pragma unroll
        for (int q = 0; q < R; ++q) v[b * R + q] = p[q * NRP];
      } else {
#pragma unroll
        for (int q = 0; q < R; ++q) v[b * R + q] = buf[padi<P>(j + q * NR)];
      }
    }
  }
  template <bool INV>
  static __device__ __forceinline__ void compute(cplx<T>* v, int t, const cplx<T>* __restrict__ tw) {
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      if constexpr (NS > 1) {
        const int j = t + b * TPF;
        const int k = j % NS;   // NS need not be a power of two (mixed sequences)
        // table [q-1][k]: consecutive lanes read consecutive entries
        const cplx<T>* w = tw + k;
        cplx<T> wq[R];
#pragma unroll
        for (int q = 1; q < R; ++q) wq[q] = ldkc(w + (q - 1) * NS);
#pragma unroll
        for (int q = 1; q < R; ++q) {
          cplx<T> x = wq[q];
          if (INV) x.y = -x.y;
          v[b * R + q] = cmul(v[b * R + q], x);
        }
      }
      dft_c<R, INV>(v + b * R);
    }
  }
  // NS == 1: the R outputs of a butterfly are consecutive and R divides 2^P, so they
  // never straddle a pad
  static __device__ __forceinline__ void store(cplx<T>* buf, const cplx<T>* v, int t) {
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const int j = t + b * TPF;
      const int k = j % NS;   // NS need not be a power of two (mixed sequences)
      const int base = (j - k) * R + k;
      if constexpr (LIN_STORE) {
        cplx<T>* p = buf + padi<P>(base);
#pragma unroll
        for (int q = 0; q < R; ++q) p[q * NSP] = v[b * R + q];
      } else {
#pragma unroll
        for (int q = 0; q < R; ++q) buf[padi<P>(base + q * NS)] = v[b * R + q];
      }
    }
  }
  // natural-order index of register v[b * R + q] after the last pass (NS = N / R)
  static __device__ __forceinline__ int out_index(int t, int b, int q) { return t + b * TPF + q * NR; }
};

// Middle passes [PA, PB) of sequence A (SEQB = false) or B, in place through buf.
template <class T, int N, int EE_REQ, bool SEQB, bool INV, int PA, int PB>
__device__ __forceinline__ void fast_mid(cplx<T>* buf, cplx<T>* v, int t, int g, const cplx<T>* __restrict__ tw) {
  if constexpr (PA < PB) {
    using S = FastSeq<N, EE_REQ, RadixCap<T>::value>;
    constexpr int P = FastPad<T, S::EE>::value;
    constexpr int R = SEQB ? S::radB(PA) : S::radA(PA);
    constexpr int NS = SEQB ? S::nsB(PA) : S::nsA(PA);
    constexpr int OFF = SEQB ? S::twB(PA) : S::twA(PA);
    using PS = FastPass<T, N, S::EE, R, NS, P>;
    PS::load(buf, v, t);
    group_sync<S::TPF>(g);
    PS::template compute<INV>(v, t, tw + OFF);
    PS::store(buf, v, t);
    group_sync<S::TPF>(g);
    fast_mid<T, N, EE_REQ, SEQB, INV, PA + 1, PB>(buf, v, t, g, tw);
  }
}


constexpr unsigned kStatusTimeout = 2;   // PFC_STATUS_TIMEOUT: a bounded wait gave up

template <class T>
struct FastRowArgs {
  int ny, rows, ld;
  int rows_log2;             // rows = 1 << rows_log2, or -1 when rows is not a power of two
  const BatchBufs* batch;    // null: one plan, the pointers below
  const cplx<T>* in;         // W, column-major [kx][y]
  cplx<T>* out;              // V, column-major
  const cplx<T>* twA;        // row sequence A table (inverse uses conjugates)
  const cplx<T>* twB;        // row sequence B table
  const cplx<T>* rtw;        // exp(-2 pi i k / nx), k < m
  const double* scal;
  int clamp;
  double g, min_phi, min_log;
  int tma_box;               // packed row kernel: kx extent of a TMA box (0: asynchronous copies)
  int* err;                  // status word; a bounded wait that gave up ORs PFC_STATUS_TIMEOUT
  unsigned tma_extra_tx;     // bytes the TMA barrier expects beyond the tile (0; a test sets more)
  int tma_wait_limit;        // polls of that barrier before giving up (0: the default)
};

template <class T>
struct FastColArgs {
  int m, ny, nyh;
  const BatchBufs* batch;    // null: one plan, the pointers below
  const cplx<T>* in;         // V
  const void* nin;           // n_hat: complex128, or hi (FP32 form; see ColArgs)
  const cplx<float>* nin_lo;
  void* nout;                // n_hat'
  cplx<float>* nout_lo;
  cplx<T>* wout;             // W'
  const cplx<T>* coef;       // (A - 1, Bg) [kx][ky <= ny/2], working precision
  const cplx<double>* coef64;  // FP32 form: FP64 copy, read for the slow modes
  float slow_tau;
  const cplx<T>* twA;        // column sequence A (forward)
  const cplx<T>* twB;        // column sequence B (inverse uses conjugates)
  T scale;
};

// Bulk prefetch of [p, p + bytes) into L2 (p and bytes multiples of 16), in chunks
// issued by the threads of a transform group.
__device__ __forceinline__ void l2_prefetch_range(const void* p, unsigned bytes, int t, int nthreads) {
  constexpr unsigned kChunk = 4096;
  const char* c = static_cast<const char*>(p);
  for (unsigned off = (unsigned)t * kChunk; off < bytes; off += (unsigned)nthreads * kChunk) {
    const unsigned n = bytes - off < kChunk ? bytes - off : kChunk;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(c + off), "r"(n) : "memory");
  }
}

// Programmatic dependent launch. A step kernel launched with programmatic stream
// serialisation may start while the kernel before it in the stream is still running:
// pdl_wait() returns once that kernel has completed and its writes are visible (at
// once for a kernel launched without the attribute). Each step kernel calls
// pdl_trigger() right after pdl_wait(), so the code a kernel runs before its own
// pdl_wait() starts only after the kernel two launches back has completed; that code
// reads only buffers written two or more launches back and writes nothing.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Synchronisation hook of the step bodies: in the step kernels, the point where a kernel
// launched with programmatic dependent launch waits for its predecessor; in the work-queue
// kernel, whose items wait for their dependencies before the body starts, nothing.
struct PdlSync {
  __device__ __forceinline__ void operator()() const { pdl_wait(); pdl_trigger(); }
};
struct NoSync {
  __device__ __forceinline__ void operator()() const {}
};

// CTA-wide barrier of the threads that run a step body: the whole CTA in the step kernels,
// the first `nthreads` threads (whole warps) in the work-queue kernel, on named barrier 15,
// which no transform group uses (group barriers are 1 + group index, at most 4 groups).
__device__ __forceinline__ void body_sync(int nthreads) {
  if (nthreads == (int)blockDim.x) __syncthreads();
  else asm volatile("bar.sync 15, %0;" ::"r"(nthreads) : "memory");
}

template <int TPF> struct FastBound { static constexpr int value = TPF > 256 ? TPF : 256; };
// minimum resident CTAs per SM requested from the register allocator (256-thread CTAs)
// from the registers the values held take (2 per real): with up to 32 of them the
// kernels fit 64 registers without spilling (4 CTAs per SM), with 64 they need 128
template <class T, int EE, int TPF> struct FastMinBlocks {
  static constexpr int data_regs = 2 * EE * (int)(sizeof(T) / 4);
  static constexpr int value = TPF > 256 ? 1 : (data_regs <= 32 ? 4 : 2);
};

// Chunk of the column kernel's ETD1 update: the modes whose coefficients and states are
// loaded together (4 registers per mode in FP32, 8 in FP64), a power of two dividing EE:
// 8 for FP32 transforms of 16 or 24 values per thread, 4 for 32 (with 8 the in-register
// update spilled 16 bytes per thread and ran 0.5-1 % slower), else 4 or 2. The update
// runs in registers (REG) where the launch bounds leave room for the chunk on top of the
// EE values held and about 28 registers of addresses and indices (the 128-register
// kernels); in the 64-register kernels the values wait in the exchange buffer instead.
template <class T, int EE, int TPF>
struct ColChunk {
  using MB = FastMinBlocks<T, EE, TPF>;
  static constexpr int value =
      (sizeof(T) == 4 && EE == 32) ? 4 : ((sizeof(T) == 4 && EE >= 16 && EE % 8 == 0) ? 8 : (EE % 4 == 0 ? 4 : 2));
  static constexpr int limit0 = 65536 / (MB::value * FastBound<TPF>::value);
  static constexpr int limit = limit0 > 255 ? 255 : limit0;
  static constexpr int per_mode = 4 * (int)(sizeof(T) / 4);
  static constexpr bool REG = (EE & (EE - 1)) == 0 && limit >= 128 && value * per_mode <= limit - MB::data_regs - 28;
};
// the 2048-point columns: FP32 with 16 values per thread (64 registers) buffered, with 32 in
// registers; FP64 with 8 buffered, with 16 in registers
static_assert(!ColChunk<float, 16, 128>::REG && ColChunk<float, 32, 64>::REG, "FP32 column update forms");
static_assert(!ColChunk<double, 8, 256>::REG && ColChunk<double, 16, 128>::REG, "FP64 column update forms");

// ------------------------------------------------------------------ row kernel
// CTA: `rows` consecutive rows (tile), groups of TPF threads each process rows
// g, g + ngroups, ... The tile is staged through shared memory with a transposing
// load/store (global layout is column-major). The body runs row tile `tile` of batch member
// `member` (of `batch`, or the plan in `a` when null) on the CTA's first `nthreads` threads.
// COHERENT: W may have been written by another CTA of the same launch (the work-queue
// kernel), so the tile is not read through the non-coherent path.
template <class T, int M, int EE_REQ, int MODEL, bool COHERENT = false, class Sync>
__device__ __forceinline__ void row_step_body(const FastRowArgs<T>& a, const BatchBufs* batch, int tile, int member,
                                              int nthreads, Sync sync) {
  using S = FastSeq<M, EE_REQ, RadixCap<T>::value>;
  constexpr int P = FastPad<T, S::EE>::value;
  constexpr int EE = S::EE, TPF = S::TPF, NP = S::NPASS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* sm = reinterpret_cast<cplx<T>*>(smem_raw);
  const int ny = a.ny, rows = a.rows, ld = a.ld, rl2 = a.rows_log2;
  const int y0 = tile * rows;
  const int ngroups = nthreads / TPF;
  const int g = threadIdx.x / TPF, t = threadIdx.x - g * TPF;
  const bool dev = (sizeof(T) == 4);
  const cplx<T>* gin = a.in;
  cplx<T>* gout = a.out;
  const double* scal = a.scal;
  if (batch) {
    const BatchBufs& b = batch[member];
    gin = static_cast<const cplx<T>*>(b.w);
    gout = static_cast<cplx<T>*>(b.v);
    scal = b.scal;
  }

  // W is the previous column pass's output
  sync();

  // ---- transposing tile load: element (kx, y0 + r) -> sm[r * ld + pad(kx)], issued as
  // asynchronous global->shared copies so that every load of the tile is in flight at once.
  // nthreads is a multiple of rows: each thread keeps one row and walks kx with a fixed
  // stride, so the addresses advance by constants. (A tile of a row count other than a
  // power of two spreads a grid's rows evenly over the SMs: 2048 rows in 293 tiles of 7,
  // two per SM, where 256 tiles of 8 leave 40 SMs with one.)
  const int tr = rl2 >= 0 ? (int)(threadIdx.x & (rows - 1)) : (int)threadIdx.x % rows;
  const int kx0 = rl2 >= 0 ? (int)(threadIdx.x >> rl2) : (int)threadIdx.x / rows;
  const int kstep = rl2 >= 0 ? nthreads >> rl2 : nthreads / rows;
  const bool rvalid = y0 + tr < ny;
  const size_t gstep = (size_t)kstep * ny;
  // With one row per transform group (rows == groups, the usual tile) the stride is TPF:
  // the loops over a thread's elements then have compile-time trip counts and unroll.
  const bool unit = kstep == TPF;
  {
    cplx<T>* drow = sm + tr * ld;
    const cplx<T>* src0 = gin + (size_t)kx0 * ny + (y0 + tr);
    auto copy = [&](int kx, const cplx<T>* src) {
      cplx<T>* dst = drow + padi<P>(kx);
      if (rvalid) {
        const unsigned sdst = (unsigned)__cvta_generic_to_shared(dst);
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(sdst), "l"(src), "n"(sizeof(cplx<T>))
                     : "memory");
      } else {
        *dst = mk(T(0), T(0));
      }
    };
    if (!COHERENT && unit && rvalid) {
      // a thread's elements as loads that do not allocate in L1 (the tile passes through
      // once; the twiddle tables keep the L1), all in flight before the shared stores:
      // 2048^2 FP32 step 34.1 -> 33.2 us against the asynchronous copies below
      cplx<T> tmp[M / TPF];
#pragma unroll
      for (int j = 0; j < M / TPF; ++j) tmp[j] = ldsc(src0 + (size_t)j * gstep);
#pragma unroll
      for (int j = 0; j < M / TPF; ++j) drow[padi<P>(kx0 + j * TPF)] = tmp[j];
    } else if (unit) {
#pragma unroll
      for (int j = 0; j < M / TPF; ++j) copy(kx0 + j * TPF, src0 + (size_t)j * gstep);
    } else if (!COHERENT && rvalid) {
      // several rows per transform group: the same loads, eight in flight at a time
      constexpr int B = 8;
      const cplx<T>* src = src0;
      int kx = kx0;
      for (; kx + (B - 1) * kstep < M; kx += B * kstep, src += (size_t)B * gstep) {
        cplx<T> tmp[B];
#pragma unroll
        for (int b = 0; b < B; ++b) tmp[b] = ldsc(src + (size_t)b * gstep);
#pragma unroll
        for (int b = 0; b < B; ++b) drow[padi<P>(kx + b * kstep)] = tmp[b];
      }
      for (; kx < M; kx += kstep, src += gstep) drow[padi<P>(kx)] = ldsc(src);
    } else {
      const cplx<T>* src = src0;
      for (int kx = kx0; kx < M; kx += kstep, src += gstep) copy(kx, src);
    }
  }
  // twiddle tables are read through the L1 cache
  const cplx<T>* twA_s = a.twA;
  const cplx<T>* twB_s = a.twB;
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  body_sync(nthreads);

  // nonlinearity parameters
  float c1 = 0.f, c2 = 0.f, inv = 0.f, lmin = 0.f;
  double inv_d = 0.0, mphi_rel = 0.0;
  if (dev) {
    c1 = (float)scal[kScalC1];
    c2 = (float)scal[kScalC2];
    inv = (float)scal[kScalInvMean];
    inv_d = scal[kScalInvMean];
    mphi_rel = a.min_phi * inv_d;
    lmin = (float)scal[kScalLogMin];
  }

  for (int r = g; r < rows; r += ngroups) {
    cplx<T>* row = sm + r * ld;
    cplx<T> v[EE];
    // ---- inverse-real pre-twiddle, in place, one (k, M - k) pair per step:
    // Z[k] = S + U, Z[M - k] = conj(S - U), S = X[k] + conj X[M-k], U = i conj(r_k) (X[k] - conj X[M-k])
    // (k = t + j TPF, j < M / (2 TPF) + 1, the last only while k <= M / 2)
#pragma unroll
    for (int j = 0; j <= M / (2 * TPF); ++j) {
      const int k = t + j * TPF;
      if (k > M / 2) break;
      if (k == 0) {
        const cplx<T> x0 = row[0];
        row[0] = mk(x0.x + x0.y, x0.x - x0.y);
      } else {
        const cplx<T> xk = row[padi<P>(k)], xm = row[padi<P>(M - k)];
        const cplx<T> s = xk + conj(xm), d = xk - conj(xm);
        const cplx<T> u = mul_i(cmul(conj(ldkc(a.rtw + k)), d));
        row[padi<P>(k)] = s + u;
        if (k != M / 2) row[padi<P>(M - k)] = conj(s - u);
      }
    }
    group_sync<TPF>(g);
    FastPass<T, M, EE, S::radA(0), 1, P>::load(row, v, t);
    group_sync<TPF>(g);
    if constexpr (NP == 1) {
      FastPass<T, M, EE, S::radA(0), 1, P>::template compute<true>(v, t, twA_s);
    } else {
      using P0 = FastPass<T, M, EE, S::radA(0), 1, P>;
      P0::template compute<true>(v, t, twA_s);
      P0::store(row, v, t);
      group_sync<TPF>(g);
      fast_mid<T, M, EE_REQ, false, true, 1, NP - 1>(row, v, t, g, twA_s);
      using PL = FastPass<T, M, EE, S::radA(NP - 1), S::nsA(NP - 1), P>;
      PL::load(row, v, t);
      group_sync<TPF>(g);
      PL::template compute<true>(v, t, twA_s + S::twA(NP - 1));
    }
    // ---- v holds z[e] = n[2e] + i n[2e+1]: the nonlinearity, in registers
#pragma unroll
    for (int e = 0; e < EE; ++e) {
      const cplx<T> z = v[e];
      if (dev) {
        v[e] = mk((T)nonlin_dev<MODEL>((float)z.x, c1, c2, inv, inv_d, a.clamp, mphi_rel, lmin),
                  (T)nonlin_dev<MODEL>((float)z.y, c1, c2, inv, inv_d, a.clamp, mphi_rel, lmin));
      } else {
        v[e] = mk((T)nonlin_plain<MODEL>((double)z.x, a.g, a.clamp, a.min_phi, a.min_log),
                  (T)nonlin_plain<MODEL>((double)z.y, a.g, a.clamp, a.min_phi, a.min_log));
      }
    }
    // ---- forward sequence B
    constexpr int RL = S::radB(NP - 1);
    if constexpr (NP == 1) {
      FastPass<T, M, EE, S::radB(0), 1, P>::template compute<false>(v, t, twB_s);
    } else {
      using Q0 = FastPass<T, M, EE, S::radB(0), 1, P>;
      Q0::template compute<false>(v, t, twB_s);
      Q0::store(row, v, t);
      group_sync<TPF>(g);
      fast_mid<T, M, EE_REQ, true, false, 1, NP - 1>(row, v, t, g, twB_s);
      using QL = FastPass<T, M, EE, RL, S::nsB(NP - 1), P>;
      QL::load(row, v, t);
      group_sync<TPF>(g);
      QL::template compute<false>(v, t, twB_s + S::twB(NP - 1));
    }
    // ---- publish Z (the forward transform, natural order) for the fused post-twiddle store
    using QO = FastPass<T, M, EE, RL, M / RL, P>;
    constexpr int NBL = EE / RL;
#pragma unroll
    for (int b = 0; b < NBL; ++b)
#pragma unroll
      for (int q = 0; q < RL; ++q) row[padi<P>(QO::out_index(t, b, q))] = v[b * RL + q];
  }
  body_sync(nthreads);
  // ---- forward-real post-twiddle fused with the transposing tile store: one (k, M - k)
  // pair per step, Y[k] = E + r_k O, Y[M - k] = conj(E - r_k O), with
  // E = (Z[k] + conj Z[M-k]) / 2, O = -i (Z[k] - conj Z[M-k]) / 2, written to V[k][y]
  // and V[M - k][y] (consecutive threads take consecutive y of one k: coalesced)
  if (rvalid) {
    const cplx<T>* srow = sm + tr * ld;
    cplx<T>* col0 = gout + (y0 + tr);
    auto post = [&](int k) {
      if (k == 0) {
        const cplx<T> z0 = srow[0];
        col0[0] = mk(z0.x + z0.y, z0.x - z0.y);
      } else {
        const cplx<T> zk = srow[padi<P>(k)], zm = srow[padi<P>(M - k)];
        const cplx<T> e = T(0.5) * (zk + conj(zm));
        const cplx<T> o = cmul(ldkc(a.rtw + k), T(0.5) * rot4<false>(zk - conj(zm)));
        col0[(size_t)k * ny] = e + o;
        if (k != M / 2) col0[(size_t)(M - k) * ny] = conj(e - o);
      }
    };
    if (unit) {
#pragma unroll
      for (int j = 0; j <= M / (2 * TPF); ++j) {
        const int k = kx0 + j * TPF;
        if (k > M / 2) break;
        post(k);
      }
    } else {
#pragma unroll 2
      for (int k = kx0; k <= M / 2; k += kstep) post(k);
    }
  }
}

template <class T, int M, int EE_REQ, int MODEL>
__global__ void __launch_bounds__(FastBound<FastSeq<M, EE_REQ, RadixCap<T>::value>::TPF>::value,
                  FastMinBlocks<T, FastSeq<M, EE_REQ, RadixCap<T>::value>::EE,
                                FastSeq<M, EE_REQ, RadixCap<T>::value>::TPF>::value)
row_step_fast(FastRowArgs<T> a) {
  row_step_body<T, M, EE_REQ, MODEL>(a, a.batch, blockIdx.x, blockIdx.y, blockDim.x, PdlSync{});
}

// Loads of field data in the column body. The step kernels read V and n_hat, outputs of
// earlier launches, without allocating in L1 through the non-coherent path; the work-queue
// kernel reads them while other CTAs of the same launch write them, so through L2 only.
template <bool COHERENT, class T>
__device__ __forceinline__ cplx<T> ld_field(const cplx<T>* p) {
  if constexpr (!COHERENT) {
    return ldsc(p);
  } else {
    using V = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
    V v;
    if constexpr (sizeof(T) == 4)
      asm volatile("ld.global.cg.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    else
      asm volatile("ld.global.cg.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return mk((T)v.x, (T)v.y);
  }
}

// ------------------------------------------------------------------ column kernel
// CTA: ngroups consecutive columns, one group of TPF threads per column. Global
// reads and writes go straight between registers and HBM (the first pass of each
// sequence reads, and the last pass writes, consecutive elements per lane). The body runs
// column tile `tile` of member `member` on the CTA's first `nthreads` threads.
template <class T, int NY, int EE_REQ, bool COHERENT, class Sync>
__device__ __forceinline__ void col_step_body(const FastColArgs<T>& a, const BatchBufs* batch, int tile, int member,
                                              int nthreads, Sync sync) {
  using S = FastSeq<NY, EE_REQ, RadixCap<T>::value>;
  constexpr int P = FastPad<T, S::EE>::value;
  constexpr int EE = S::EE, TPF = S::TPF, NP = S::NPASS;
  constexpr int PADN = NY + (NY >> P) + 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* sm = reinterpret_cast<cplx<T>*>(smem_raw);
  const int ngroups = nthreads / TPF;
  const int g = threadIdx.x / TPF, t = threadIdx.x - g * TPF;
  const int kx = tile * ngroups + g;      // m is a multiple of ngroups
  const cplx<T>* twA_s = a.twA;                   // twiddle tables, read through L1
  const cplx<T>* twB_s = a.twB;
  cplx<T>* buf = sm + g * PADN;                   // exchange buffer of this column
  const int m = a.m, nyh = a.nyh;
  const cplx<T>* gin = a.in;
  const void* gnin = a.nin;
  void* gnout = a.nout;
  const cplx<float>* gnin_lo = a.nin_lo;
  cplx<float>* gnout_lo = a.nout_lo;
  cplx<T>* gwout = a.wout;
  const cplx<T>* gcoef = a.coef;
  const cplx<double>* gcoef64 = a.coef64;
  if (batch) {
    const BatchBufs& b = batch[member];
    gin = static_cast<const cplx<T>*>(b.v);
    gnin = b.nin;
    gnout = b.nout;
    gnin_lo = static_cast<const cplx<float>*>(b.nin_lo);
    gnout_lo = static_cast<cplx<float>*>(b.nout_lo);
    gwout = static_cast<cplx<T>*>(const_cast<void*>(b.w));
    gcoef = static_cast<const cplx<T>*>(b.coef);
    gcoef64 = static_cast<const cplx<double>*>(b.coef64);
  }
  cplx<T> v[EE];

  // ---- start this column's n_hat and coefficients towards L2 while the forward
  // transform runs (the coefficient range is widened to 16-byte boundaries; it stays
  // inside the table, which has a row after every column a CTA handles)
  constexpr unsigned kStateElt = sizeof(T) == 8 ? sizeof(cplx<double>) : sizeof(cplx<float>);
  l2_prefetch_range(static_cast<const char*>(gnin) + (size_t)kx * NY * kStateElt, NY * kStateElt, t, TPF);
  {
    const uintptr_t c0 = reinterpret_cast<uintptr_t>(gcoef + (size_t)kx * nyh) & ~(uintptr_t)15;
    const uintptr_t c1 = (reinterpret_cast<uintptr_t>(gcoef + (size_t)(kx + 1) * nyh) + 15) & ~(uintptr_t)15;
    l2_prefetch_range(reinterpret_cast<const void*>(c0), (unsigned)(c1 - c0), t, TPF);
  }

  // V is the row pass's output (n_hat and the coefficients above were written two or
  // more launches back)
  sync();

  // ---- forward sequence A; pass 0 reads the column of V from HBM
  {
    constexpr int R = S::radA(0), NR = NY / R, NB = EE / R;
    const cplx<T>* col = gin + (size_t)kx * NY;
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int q = 0; q < R; ++q) v[b * R + q] = ld_field<COHERENT>(col + t + b * TPF + q * NR);
  }
  if constexpr (NP == 1) {
    FastPass<T, NY, EE, S::radA(0), 1, P>::template compute<false>(v, t, twA_s);
  } else {
    using P0 = FastPass<T, NY, EE, S::radA(0), 1, P>;
    P0::template compute<false>(v, t, twA_s);
    P0::store(buf, v, t);
    group_sync<TPF>(g);
    fast_mid<T, NY, EE_REQ, false, false, 1, NP - 1>(buf, v, t, g, twA_s);
    using PL = FastPass<T, NY, EE, S::radA(NP - 1), S::nsA(NP - 1), P>;
    PL::load(buf, v, t);
    group_sync<TPF>(g);
    PL::template compute<false>(v, t, twA_s + S::twA(NP - 1));
  }

  // ---- ETD1 update. After A's last pass register v[b * RL + q] holds mode
  // ky = t + (b + q NBL) TPF (its natural-order index), the element B's first pass loads
  // into the same register. Where the registers allow (ColChunk::REG) the columns other
  // than the packed one update in registers; otherwise, and for the packed column, which
  // pairs ky with NY - ky held by another thread, the spectrum goes through the exchange
  // buffer in natural order and is reloaded for sequence B.
  constexpr int RL = S::radA(NP - 1), NBL = EE / RL;
  using PO = FastPass<T, NY, EE, RL, NY / RL, P>;
  using CC = ColChunk<T, EE, TPF>;
  const size_t cb = (size_t)kx * NY;
  const float tau = a.slow_tau;
  const bool packed = kx == 0;
  if (!CC::REG || packed) {
#pragma unroll
    for (int b = 0; b < NBL; ++b)
#pragma unroll
      for (int q = 0; q < RL; ++q) buf[padi<P>(PO::out_index(t, b, q))] = v[b * RL + q];
    group_sync<TPF>(g);
  }
  if (!packed) {
    const size_t ccb = (size_t)kx * nyh;
    // mode ky of coefficient cw, state p, transformed nonlinearity gv (updated in place)
    auto update = [&](int ky, const cplx<T>& cw, const cplx<T>& p, cplx<T>& gv) {
      const int kh = ky <= NY / 2 ? ky : NY - ky;
      if constexpr (sizeof(T) == 4) {
        if (fabsf(cw.x) >= tau) {
          // fast modes (|A - 1| >= tau): the update in FP32 on hi alone; their rounding
          // errors are damped by at least tau every step
          const cplx<float> o = mk(fmaf(cw.x, p.x, p.x) + cw.y * gv.x, fmaf(cw.x, p.y, p.y) + cw.y * gv.y);
          static_cast<cplx<float>*>(gnout)[cb + ky] = o;
          gv = o;
        } else {
          // slow modes: FP64 coefficients and the state with its residual
          const cplx<double> c = gcoef64[ccb + kh];
          const cplx<float> l = gnin_lo[cb + ky];
          cplx<double> pd = mk((double)p.x, (double)p.y);
          pd.x += (double)l.x;
          pd.y += (double)l.y;
          const cplx<double> o = pd + c.x * pd + c.y * mk((double)gv.x, (double)gv.y);
          state_st<T>(gnout, gnout_lo, cb + ky, o, true);
          gv = mk((T)o.x, (T)o.y);
        }
      } else {
        const cplx<double> c = cw, pd = p;
        const cplx<double> o = pd + c.x * pd + c.y * mk((double)gv.x, (double)gv.y);
        state_st<T>(gnout, gnout_lo, cb + ky, o, true);
        gv = mk((T)o.x, (T)o.y);
      }
    };
    // Each thread updates its modes ky = t + j TPF, j < EE, in chunks: the coefficients
    // and states of a whole chunk are loaded before any of its results is stored (the
    // compiler may not move a load above an earlier store to memory it cannot tell
    // apart), so the chunk's loads are in flight together.
    constexpr int CH = CC::value;
    static_assert(EE % CH == 0, "chunks tile the modes of a thread");
    auto chunk_loads = [&](int j0, cplx<T>* cw, cplx<T>* p) {
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        const int ky = t + (j0 + j) * TPF;
        const int kh = ky <= NY / 2 ? ky : NY - ky;
        cw[j] = ldgc(gcoef + ccb + kh);   // cached: modes ky and NY - ky share an entry
        p[j] = ld_field<COHERENT>(static_cast<const cplx<T>*>(gnin) + cb + ky);
      }
    };
    if constexpr (CC::REG) {
#pragma unroll
      for (int j0 = 0; j0 < EE; j0 += CH) {
        cplx<T> cw[CH], p[CH];
        chunk_loads(j0, cw, p);
#pragma unroll
        for (int j = 0; j < CH; ++j) {
          const int jj = j0 + j;
          update(t + jj * TPF, cw[j], p[j], v[(jj % NBL) * RL + jj / NBL]);
        }
      }
    } else {
#pragma unroll 1
      for (int j0 = 0; j0 < EE; j0 += CH) {
        cplx<T> cw[CH], p[CH];
        chunk_loads(j0, cw, p);
#pragma unroll
        for (int j = 0; j < CH; ++j) {
          const int ky = t + (j0 + j) * TPF;
          cplx<T> gv = buf[padi<P>(ky)];
          update(ky, cw[j], p[j], gv);
          buf[padi<P>(ky)] = gv;
        }
      }
    }
  } else {
    // packed DC/Nyquist column (kx = 0 and kx = M): one (ky, -ky) pair per step, always
    // at full precision
    const size_t cmb = (size_t)m * nyh;
    // two pairs per chunk, both loaded before either is stored (as above)
    constexpr int CP = 2;
#pragma unroll 1
    for (int i0 = 0; t + i0 * TPF <= NY / 2; i0 += CP) {
      cplx<double> pk[CP], pkp[CP], a0[CP], am[CP];
#pragma unroll
      for (int j = 0; j < CP; ++j) {
        const int ky = t + (i0 + j) * TPF;
        if (ky <= NY / 2) {
          const int kyp = ky == 0 ? 0 : NY - ky;
          bool s0, sm;
          pk[j] = state_ld<T>(gnin, gnin_lo, cb + ky, true);
          pkp[j] = state_ld<T>(gnin, gnin_lo, cb + kyp, true);
          a0[j] = coef_ld<T>(gcoef, gcoef64, ky, tau, true, s0);
          am[j] = coef_ld<T>(gcoef, gcoef64, cmb + ky, tau, true, sm);
        }
      }
#pragma unroll
      for (int j = 0; j < CP; ++j) {
        const int ky = t + (i0 + j) * TPF;
        if (ky > NY / 2) break;
        const int kyp = ky == 0 ? 0 : NY - ky;
        const cplx<T> qkt = buf[padi<P>(ky)], qkpt = buf[padi<P>(kyp)];
        const cplx<double> qk = mk((double)qkt.x, (double)qkt.y), qkp = mk((double)qkpt.x, (double)qkpt.y);
        cplx<double> h0, hm, g0, gm;
        unpack_pair(pk[j], pkp[j], h0, hm);
        unpack_pair(qk, qkp, g0, gm);
        const cplx<double> h0n = h0 + a0[j].x * h0 + a0[j].y * g0;
        const cplx<double> hmn = hm + am[j].x * hm + am[j].y * gm;
        const cplx<double> ok = h0n + mul_i(hmn), okp = conj(h0n) + mul_i(conj(hmn));
        state_st<T>(gnout, gnout_lo, cb + ky, ok, true);
        buf[padi<P>(ky)] = mk((T)ok.x, (T)ok.y);
        if (kyp != ky) {
          state_st<T>(gnout, gnout_lo, cb + kyp, okp, true);
          buf[padi<P>(kyp)] = mk((T)okp.x, (T)okp.y);
        }
      }
    }
  }
  if (!CC::REG || packed) {
    group_sync<TPF>(g);
    FastPass<T, NY, EE, S::radB(0), 1, P>::load(buf, v, t);
    group_sync<TPF>(g);
  }

  // ---- inverse sequence B; the last pass writes W to HBM
  if constexpr (NP == 1) {
    FastPass<T, NY, EE, S::radB(0), 1, P>::template compute<true>(v, t, twB_s);
  } else {
    using Q0 = FastPass<T, NY, EE, S::radB(0), 1, P>;
    Q0::template compute<true>(v, t, twB_s);
    Q0::store(buf, v, t);
    group_sync<TPF>(g);
    fast_mid<T, NY, EE_REQ, true, true, 1, NP - 1>(buf, v, t, g, twB_s);
    using QL = FastPass<T, NY, EE, S::radB(NP - 1), S::nsB(NP - 1), P>;
    QL::load(buf, v, t);
    QL::template compute<true>(v, t, twB_s + S::twB(NP - 1));
  }
  {
    constexpr int RB = S::radB(NP - 1), NBB = EE / RB;
    using QO = FastPass<T, NY, EE, RB, NY / RB, P>;
    cplx<T>* col = gwout + (size_t)kx * NY;
    const T s = a.scale;
#pragma unroll
    for (int b = 0; b < NBB; ++b)
#pragma unroll
      for (int q = 0; q < RB; ++q) {
        const cplx<T> x = v[b * RB + q];
        col[QO::out_index(t, b, q)] = mk(s * x.x, s * x.y);
      }
  }
}

template <class T, int NY, int EE_REQ>
__global__ void __launch_bounds__(FastBound<FastSeq<NY, EE_REQ, RadixCap<T>::value>::TPF>::value,
                                  FastMinBlocks<T, FastSeq<NY, EE_REQ, RadixCap<T>::value>::EE,
                                                FastSeq<NY, EE_REQ, RadixCap<T>::value>::TPF>::value)
col_step_fast(FastColArgs<T> a) {
  col_step_body<T, NY, EE_REQ, false>(a, a.batch, blockIdx.x, blockIdx.y, blockDim.x, PdlSync{});
}

}  // namespace pfc
