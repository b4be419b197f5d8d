// shadow_host.h — what the batched launch needs of a prepared per-face shadow cull pass
// (helio_shadow_cull_*), so that the batch can run the pass's three stages as units of
// its own phases (helio_batch_attach_shadow).
#pragma once

#include "shadow_device.cuh"

struct helio_shadow_cull_pass;

namespace helio {

// The device view of a prepared pass; false when the pass is not prepared or has no
// face or no draw in use, in which case the pass does nothing at all (lib.rs:261-263).
bool shadow_dev(const helio_shadow_cull_pass* p, ShadowDev* out);

}  // namespace helio
