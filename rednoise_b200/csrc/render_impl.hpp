// Shared host helpers of the physical-mode entry points.
#pragma once

#include "physical.cuh"
#include "rednoise/rednoise_pt.h"

struct rn_scene;

namespace rnb {

// Validate the public camera/settings, prepare the scene and fill the kernel inputs.
rn_status make_phys_inputs(rn_scene *s, const rn_pt_camera *c, const rn_pt_settings *st, unsigned flags,
                           PhysScene &ps, PhysCamera &pc, PhysSettings &pst);

} // namespace rnb
