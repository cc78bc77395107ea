// persist.h — the exact model as it is stored on disk (persist.cpp).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "gprx_cuda.h"

namespace gprx {

struct Mapped;

struct PersistModel {
  long long n = 0, d = 0;
  std::vector<gprx_kernel_node> nodes;
  std::vector<double> theta;  // kernel log-parameters, depth-first
  double log_noise = 0.0;
  gprx_options jitter{};      // only the jitter fields are stored
  bool has_factor = false;
  bool ldlt = false;          // factor_kind "ldlt" (unit L below, D on the diagonal)
  double factor_jitter = 0.0;
  std::vector<double> x, y, l, alpha;  // column-major, as the files hold them
  const double* l_map = nullptr;       // read: l inside the file mapping
  std::shared_ptr<Mapped> mapping;     // keeps l_map valid
  std::vector<uint64_t> ids;
  uint64_t next_id = 0;
};

gprx_status persist_write(const std::string& dir, const PersistModel& m);
// with_factor_data: map l (l_map) as well as reading the rest
gprx_status persist_read(const std::string& dir, PersistModel& m, bool with_factor_data);

}  // namespace gprx
