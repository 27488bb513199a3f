#include "autotune.cuh"

#include <map>
#include <sstream>

namespace fpls {

namespace {
TuneConfig g_active;
bool g_enabled = false;
struct Entry {
  TuneConfig cfg;
  std::string report;
};
std::map<TuneKey, Entry>& cache() {
  static std::map<TuneKey, Entry> c;
  return c;
}
}  // namespace

std::string TuneConfig::str() const {
  std::ostringstream s;
  s << "{\"gram_tile\": " << (gram_tile ? gram_tile : 128) << ", \"step_layout\": \""
    << (step_layout == 1 ? "256x8" : (step_layout == 0 ? "512x2" : "default")) << "\", \"merge\": "
    << (merge == 0 ? "false" : "true") << ", \"ozaki_slices\": ";
  if (ozaki_slices)
    s << ozaki_slices;
  else
    s << "\"mode default\"";
  s << "}";
  return s.str();
}

TuneConfig& active_tune() { return g_active; }
bool autotune_enabled() { return g_enabled; }
void set_autotune(bool on) { g_enabled = on; }

bool TuneKey::operator<(const TuneKey& o) const {
  const int a[] = {device, n, p, F, L, K, m, precision, scaling};
  const int b[] = {o.device, o.n, o.p, o.F, o.L, o.K, o.m, o.precision, o.scaling};
  for (int i = 0; i < 9; ++i)
    if (a[i] != b[i]) return a[i] < b[i];
  return false;
}

const TuneConfig* tuned_lookup(const TuneKey& k) {
  auto it = cache().find(k);
  return it == cache().end() ? nullptr : &it->second.cfg;
}

void tuned_store(const TuneKey& k, const TuneConfig& c, const std::string& report) {
  cache()[k] = Entry{c, report};
}

std::string tune_report() {
  std::ostringstream s;
  for (const auto& kv : cache()) {
    const TuneKey& k = kv.first;
    s << "{\"device\": " << k.device << ", \"n\": " << k.n << ", \"p\": " << k.p << ", \"fits\": " << k.F
      << ", \"ncomp_slices\": " << k.L << ", \"kmax\": " << k.K << ", \"classes\": " << k.m
      << ", \"precision\": " << k.precision << ", \"scaling\": " << k.scaling << ", \"chosen\": "
      << kv.second.cfg.str() << ", \"candidates\": " << kv.second.report << "}\n";
  }
  return s.str();
}

}  // namespace fpls
