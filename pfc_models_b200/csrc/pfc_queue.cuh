// Work-queue step kernel: many independent plans of several power-of-two sizes advanced
// by a block of steps in ONE persistent launch.
//
// The unit of work (an item) is one row tile or one column tile of one plan at one step,
// the same tiles the step kernels of pfc_fast.cuh run as CTAs, through the same bodies
// (row_step_body / col_step_body), so a plan stepped here computes bit for bit what its
// own launches compute. An item's dependencies are the plan's own: its row tiles of step
// s need all of its column tiles of step s - 1 (W, and V free to overwrite), its column
// tiles of step s all of its row tiles of step s (V; n_hat of step s - 1 follows). Each
// plan keeps two completion counters (row tiles done, column tiles done) that only grow
// within a launch, so there is no grid-wide barrier: a plan waits only for itself, and the
// CTAs move on to other plans' items meanwhile.
//
// Schedule: the items of one step are listed once (row tiles of every plan, class by
// class, then the column tiles); the launch walks `nsteps` copies of the list, each CTA
// taking the next item from a ticket counter when it finishes one. An item depends only on
// items earlier in the walk, and tickets are handed out in order to CTAs that are running,
// so the earliest unfinished item always has its dependencies done and a running CTA at
// it: the walk cannot deadlock (the launch is also cooperative: every CTA resident). The
// waits are bounded all the same: a wait that exceeds its poll limit sets
// PFC_STATUS_TIMEOUT in the status word and the abort flag, and every CTA returns at its
// next item.
//
// Memory ordering (the pattern of CUTLASS's inter-CTA barriers): an item's threads finish
// their stores, the CTA synchronises, and its first thread issues fence.acq_rel.gpu and a
// relaxed add to the plan's counter; a waiting CTA's first thread polls the counter with
// ld.acquire.gpu, and the CTA synchronises before the body reads. Data written within the launch (V, W, n_hat) is read with
// coherent loads: the column body's non-coherent (ld.global.nc) loads of V and n_hat
// become ld.global.cg here (COHERENT = true); tables and coefficients, written before the
// launch, keep their loads.
#pragma once
#include "pfc_fast.cuh"

namespace pfc {

// Values per thread of the bodies compiled into the work-queue kernels: at most 16 complex
// floats or 8 complex doubles, so that every body fits the 64 registers of four 256-thread
// CTAs per SM.
__host__ __device__ constexpr int queue_row_ee(bool fp64, int m) { return fp64 ? 8 : (m <= 128 ? 8 : 16); }
__host__ __device__ constexpr int queue_col_ee(bool fp64, int ny) { return fp64 ? 8 : (ny <= 512 ? 8 : 16); }
// log2 range of the transforms compiled in: rows of M = nx/2 = 32 .. 512 points (grids 64
// .. 1024 wide), columns of 64 .. 1024 points
constexpr int kQueueMinLogRow = 5, kQueueMaxLogRow = 9, kQueueMinLogCol = 6, kQueueMaxLogCol = 10;
constexpr int kQueueThreads = 256;
constexpr long long kQueueWaitLimit = 1LL << 20;   // polls (an L2 round trip and 64 ns each): about a second

// One size class: plans of one grid and one step variant.
template <class T>
struct QueueClass {
  FastRowArgs<T> row;          // the class's row-pass arguments (members' buffers from `table`)
  FastColArgs<T> col;
  const BatchBufs* table[2];   // the members' buffers, by the parity of the step
  int row_log, col_log;        // log2 of the row (M) and column (ny) transform lengths
  int row_threads, col_threads;
  int row_items, col_items;    // items of one member's pass
  int row_group, col_group;    // consecutive tiles per item (a member's tiles = items x group)
};

// item: x = member (counter index), y = class, z = member within its class,
// w = item index within the member's pass (tiles w * group ...) | kQueueColBit for columns
constexpr int kQueueColBit = 1 << 30;

template <class T>
struct QueueArgs {
  const QueueClass<T>* classes;
  const int4* items;      // one step's items
  int nitems;
  int nsteps;
  int parity0;            // the members' common ping-pong parity at the start of the launch
  unsigned* rows_done;    // per member, zero at the start of the launch
  unsigned* cols_done;
  unsigned* ticket;       // next item of the walk, zero at the start of the launch
  int* status;            // PFC_STATUS_TIMEOUT when a wait gave up
  int* abort;             // set with it: every CTA returns
  long long wait_limit;
  int extra_item;         // an item (index within a step, at step 0) that waits for `extra`
  int extra;              //   completions more than it needs (0: none); a test sets it
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Waits (one thread) until *cnt >= target; false when the launch is aborted or the limit ran out.
__device__ __forceinline__ bool queue_wait(const unsigned* cnt, unsigned target, int* status, int* abort,
                                           long long limit) {
  for (long long polls = 0;; ++polls) {
    if (ld_acquire_u32(cnt) >= target) return true;
    if (*reinterpret_cast<volatile int*>(abort)) return false;
    if (polls >= limit) {
      atomicOr(status, (int)kStatusTimeout);
      atomicExch(abort, 1);
      return false;
    }
    __nanosleep(64);
  }
}

// One body per transform length, each compiled as its own function: inlined into one
// kernel, the ten bodies spilled over a kilobyte per thread; called, each keeps the
// registers and unrolling of its step kernel (plus the saved registers of the call).
template <class T, int M>
__device__ __noinline__ void queue_row_body(const QueueClass<T>* C, const BatchBufs* table, int tile, int local) {
  row_step_body<T, M, queue_row_ee(sizeof(T) == 8, M), kModelStd, true>(C->row, table, tile, local,
                                                                        C->row_threads, NoSync{});
}
template <class T, int NY>
__device__ __noinline__ void queue_col_body(const QueueClass<T>* C, const BatchBufs* table, int tile, int local) {
  constexpr int EE = queue_col_ee(sizeof(T) == 8, NY);
  // the queue kernel runs in 64 registers: its column bodies keep the buffered ETD1 update
  static_assert(!ColChunk<T, FastSeq<NY, EE, RadixCap<T>::value>::EE,
                          FastSeq<NY, EE, RadixCap<T>::value>::TPF>::REG,
                "queue column bodies update through the exchange buffer");
  col_step_body<T, NY, EE, true>(C->col, table, tile, local, C->col_threads, NoSync{});
}

template <class T, int L>
__device__ __forceinline__ void queue_row_item(const QueueClass<T>& C, const BatchBufs* table, int local, int tile) {
  if constexpr (L <= kQueueMaxLogRow) {
    if (C.row_log == L) {
      constexpr int M = 1 << L;
      queue_row_body<T, M>(&C, table, tile, local);
      return;
    }
    queue_row_item<T, L + 1>(C, table, local, tile);
  }
}

template <class T, int L>
__device__ __forceinline__ void queue_col_item(const QueueClass<T>& C, const BatchBufs* table, int local, int tile) {
  if constexpr (L <= kQueueMaxLogCol) {
    if (C.col_log == L) {
      constexpr int NY = 1 << L;
      queue_col_body<T, NY>(&C, table, tile, local);
      return;
    }
    queue_col_item<T, L + 1>(C, table, local, tile);
  }
}

template <class T>
__global__ void __launch_bounds__(kQueueThreads, 4) queue_step_kernel(QueueArgs<T> q) {
  __shared__ int go, item;
  const unsigned total = (unsigned)q.nitems * (unsigned)q.nsteps;
  // the first thread takes the next ticket while the current item runs (its round trip to
  // L2 then overlaps the body); items are still claimed in order, and a claimed item waits
  // only for earlier ones, so the walk stays free of deadlock
  unsigned next = 0;
  if (threadIdx.x == 0) next = atomicAdd(q.ticket, 1u);
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned gi = next;
      bool ok = gi < total && !*reinterpret_cast<volatile int*>(q.abort);
      if (ok) {
        const int s = (int)(gi / (unsigned)q.nitems), i = (int)(gi - (unsigned)s * (unsigned)q.nitems);
        const int4 it = q.items[i];
        const unsigned rt = (unsigned)q.classes[it.y].row_items, ct = (unsigned)q.classes[it.y].col_items;
        const bool col = (it.w & kQueueColBit) != 0;
        // rows of step s: every column item of step s - 1; columns of step s: every row item of step s
        unsigned target = col ? (unsigned)(s + 1) * rt : (unsigned)s * ct;
        if (s == 0 && i == q.extra_item) target += (unsigned)q.extra;
        if (target > 0)
          ok = queue_wait(col ? q.rows_done + it.x : q.cols_done + it.x, target, q.status, q.abort, q.wait_limit);
      }
      go = ok;
      item = (int)gi;
      if (ok) next = atomicAdd(q.ticket, 1u);
    }
    __syncthreads();
    if (!go) return;
    const unsigned gi = (unsigned)item;
    const int s = (int)(gi / (unsigned)q.nitems), i = (int)(gi - (unsigned)s * (unsigned)q.nitems);
    const int4 it = q.items[i];
    const QueueClass<T>& C = q.classes[it.y];
    const bool col = (it.w & kQueueColBit) != 0;
    const int group = col ? C.col_group : C.row_group;
    const int tile0 = (it.w & (kQueueColBit - 1)) * group;
    const BatchBufs* table = C.table[(q.parity0 + s) & 1];
    for (int k = 0; k < group; ++k) {
      if (k) __syncthreads();   // the previous tile's shared-memory reads are done
      if (!col) {
        if ((int)threadIdx.x < C.row_threads) queue_row_item<T, kQueueMinLogRow>(C, table, it.z, tile0 + k);
      } else {
        if ((int)threadIdx.x < C.col_threads) queue_col_item<T, kQueueMinLogCol>(C, table, it.z, tile0 + k);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned* cnt = col ? q.cols_done + it.x : q.rows_done + it.x;
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      asm volatile("red.relaxed.gpu.global.add.u32 [%0], 1;" ::"l"(cnt) : "memory");
    }
  }
}

}  // namespace pfc
