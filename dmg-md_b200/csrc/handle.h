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
