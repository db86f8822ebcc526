// Work-queue step kernel, FP32 working precision (pfc_queue.cuh).
#include "pfc_queue.cuh"
#include "pfc_registry.h"

namespace pfc {
template <>
void* QueueInst<float>::kernel() {
  return (void*)queue_step_kernel<float>;
}
}  // namespace pfc
