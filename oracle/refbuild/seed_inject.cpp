// Seed injection for the reference build (test infrastructure).
//
// The reference draws every seed from std::random_device on rank 0
// (mdrpt.cpp:402-416): one seed for the global projection matrix
// (mdrpt.cpp:55), then `ntrees` seeds for the local matrices (mdrpt.cpp:341).
// To run it reproducibly without editing its sources, this translation unit
// supplies the libstdc++ member that random_device::operator() forwards to;
// the static link resolves the reference's calls to it.  Values come, in
// order, from the comma-separated unsigned list in DRPT_REF_SEEDS.  Running
// out of values is a hard error, so a run can never fall back to entropy.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

namespace {
std::vector<unsigned> &seed_list() {
  static std::vector<unsigned> v;
  static bool parsed = false;
  if (!parsed) {
    parsed = true;
    const char *env = std::getenv("DRPT_REF_SEEDS");
    if (env) {
      std::string s(env);
      size_t pos = 0;
      while (pos < s.size()) {
        size_t comma = s.find(',', pos);
        std::string tok = s.substr(pos, comma == std::string::npos ? std::string::npos : comma - pos);
        if (!tok.empty()) v.push_back((unsigned)std::strtoul(tok.c_str(), nullptr, 0));
        if (comma == std::string::npos) break;
        pos = comma + 1;
      }
    }
  }
  return v;
}
size_t next_seed = 0;
}  // namespace

namespace std {
random_device::result_type random_device::_M_getval() {
  std::vector<unsigned> &v = seed_list();
  if (next_seed >= v.size()) {
    std::fprintf(stderr,
                 "seed_inject: random_device called %zu times but DRPT_REF_SEEDS holds %zu "
                 "values\n",
                 next_seed + 1, v.size());
    std::abort();
  }
  return v[next_seed++];
}
}  // namespace std

extern "C" size_t drpt_ref_seeds_consumed(void) { return next_seed; }
