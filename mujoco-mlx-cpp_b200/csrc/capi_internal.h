// Definitions behind the opaque C handles.
#pragma once
#include <memory>
#include <string>

#include "../../include/mjmlx/mjb200.h"
#include "model.h"

struct MjmlxModel {
  mjb::Model model;
  mjb::LoadOptions options;
};

namespace mjb {
void set_error(const std::string& msg);
class Engine;
}  // namespace mjb

struct MjmlxBatchedSim {
  std::unique_ptr<mjb::Engine> engine;
};
