// Autotuner of the batched CV grids: per (device, grid shape, precision) it
// times the candidate kernel configurations on the caller's own data the first
// time the shape is seen, keeps those whose results equal the default
// configuration's, and caches the fastest for every later call of that shape.
//
// Knobs: the row Gram's output tile width (128 x 128 or 128 x 64, two-plane
// split), the row-space step layout (512 threads x 2 rows or 256 x 8 rows per
// CTA of a 4-CTA cluster) and the merged refresh (on / off).  The number of
// INT8 digit slices of the K products is part of the configuration but is not
// searched: it sets the accuracy of the products, so each precision mode keeps
// its own.  A switch set in the environment (FASTPLS_GRAM_TILE,
// FASTPLS_DUAL_STEP, FASTPLS_DUAL_MERGE, FASTPLS_OZAKI_SLICES) wins over the
// tuned value.
#pragma once

#include <string>

namespace fpls {

struct TuneConfig {
  int gram_tile = 0;      // 0: default (128), else 64 or 128
  int step_layout = -1;   // -1: default, 0: 512 x 2 rows, 1: 256 x 8 rows
  int merge = -1;         // -1: default (on), 0 off, 1 on
  int ozaki_slices = 0;   // 0: default (5), else 4..7
  std::string str() const;
};

// The configuration in force for the running call (default: all defaults).
TuneConfig& active_tune();

// RAII: sets the active configuration for a scope and restores the previous one.
struct TuneScope {
  TuneConfig saved;
  explicit TuneScope(const TuneConfig& c) : saved(active_tune()) { active_tune() = c; }
  ~TuneScope() { active_tune() = saved; }
};

bool autotune_enabled();
void set_autotune(bool on);

struct TuneKey {
  int device, n, p, F, L, K, m, precision, scaling;
  bool operator<(const TuneKey& o) const;
};

// The cached choice for a shape, or null when it has not been tuned.
const TuneConfig* tuned_lookup(const TuneKey& k);
void tuned_store(const TuneKey& k, const TuneConfig& c, const std::string& report);
// One line per tuned shape: key, the chosen configuration and each
// candidate's device time (JSON objects, newline separated).
std::string tune_report();

}  // namespace fpls
