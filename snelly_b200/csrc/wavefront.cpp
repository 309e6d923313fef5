// wavefront.cpp - host side of the wavefront integrator: path-state buffers and stage launches.
#include "runtime_internal.h"

namespace snelly {

int Context::alloc_wavefront(Job& j) {
  (void)j;
  return SNELLY_OK;
}

void Context::release_wavefront(Job& j) { release(j.wf); }

int Context::enqueue_wavefront_frame(Job& j) {
  (void)j;
  return fail(SNELLY_EINVAL, "wavefront integrator not available");
}

}  // namespace snelly
