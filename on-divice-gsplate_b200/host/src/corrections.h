// The per-view correction state of gs::Trainer (its private `Corrections`).
#pragma once

#include "gs/trainer.h"
#include "node_rig.h"
#include "refinement.h"

namespace gs {

struct Trainer::Corrections {
  refine::CaptureOrder order;  // the trained frames in capture order
  refine::PoseTable poses;     // camera correction per dataset frame
  refine::GainTable gains;     // exposure gains per dataset frame
  refine::NodeRig rig;         // subject motion (empty without refine_motion)
};

}  // namespace gs
