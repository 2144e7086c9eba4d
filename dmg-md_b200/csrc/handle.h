// handle.h -- the opaque handle behind nepx_t (include/nepx.h).
#pragma once

#include <string>

#include "engine.h"

struct nepx_handle {
  nepx::Engine engine;
  nepx::NeighborState* h_state = nullptr;   // pinned mirror of the device flags
  cudaEvent_t state_ready = nullptr;
  bool state_pending = false;
  std::string error;
};

namespace nepx {

// Error code and message of a set of device flags (overflow of the Verlet,
// radial or angular rows, non-finite output, unsupported box, tensor-core
// timeout); NEPX_OK when none is set.  Shared by every force entry point so
// they report the same codes and messages.
int decode_state(nepx_handle* h, const NeighborState& s);

// Flags of the handle's previous asynchronous call, once its copy into the
// pinned mirror has landed (at once when `wait`): decode_state of them.
int check_state(nepx_handle* h, bool wait);

}  // namespace nepx
