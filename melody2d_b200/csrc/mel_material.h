// Host-side matrix updates of Body::Update_material, applied once when a model is created.
#pragma once
#include "melgpu.h"

// Rebuilds the MATRICES entries of every deformable body from its material, as
// Body::Update_material does at set-up (Code/Body.h:2784-2875), in place:
//  - d->flags[5] == 1: mk (n_matrix stiffness entries) re-assembled from the Gauss points;
//  - d->flags[6] == 1: mc (n_matrix damping entries) = alpha K (+ beta m on the diagonal), with the
//    masses in node_mass (2 per node, global order; the rebuilt ones when flags[4] == 1).
// mk and mc hold the description's entries on entry.  Returns MEL_OK, or MEL_ERR_INVALID with the
// error set when a Gauss point names a node outside its body.
extern "C" mel_status mel_update_matrices(const mel_model_desc* d, const double* node_mass, double* mk, double* mc);
