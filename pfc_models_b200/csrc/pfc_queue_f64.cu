// Work-queue step kernel, FP64 working precision (pfc_queue.cuh).
#include "pfc_queue.cuh"
#include "pfc_registry.h"

namespace pfc {
template <>
void* QueueInst<double>::kernel() {
  return (void*)queue_step_kernel<double>;
}
}  // namespace pfc
