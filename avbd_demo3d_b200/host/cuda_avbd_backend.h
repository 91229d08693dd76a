// CUDA AVBD physics backend for the reference solver (ts-jls/avbd-demo3d).
//
// Drop-in for the reference's backend seam `struct PhysicsBackend` (source/solver.h:410-417):
//     host.solver().physicsBackend = makeCudaAvbdPhysicsBackend(0);
// after which Solver::step (solver.cpp:934-937) runs the whole step on the GPU through the
// C ABI in include/avbd_cuda.h. Compile this file inside the reference tree (it includes
// the reference's solver.h) and link libavbd_cuda.so.
#pragma once

#include <memory>

#include "solver.h"

struct AvbdContext;

std::unique_ptr<PhysicsBackend> makeCudaAvbdPhysicsBackend(int device = 0);

// The device context behind a backend made by makeCudaAvbdPhysicsBackend (null for any
// other backend), for callers that query the ABI directly (colouring, profiles).
AvbdContext *cudaAvbdBackendContext(PhysicsBackend *backend);

// Whole-world uploads and joint-edit calls made so far by a backend made by
// makeCudaAvbdPhysicsBackend (0 for any other backend): a session whose only changes
// are drags and parameter commands uploads once.
int cudaAvbdBackendUploads(PhysicsBackend *backend);
int cudaAvbdBackendJointEdits(PhysicsBackend *backend);
