// Test harness (tests only): exposes the host symbolic phase of the
// smoothed-aggregation hierarchy (openaccel_b200/csrc/oa_amg_symbolic.h) to
// ctypes so that tests/test_amg_symbolic.py can check its structure and term
// lists against scipy sparse products.
#include <cstring>

#include "../openaccel_b200/csrc/oa_amg_symbolic.h"

static oa::sa::Level g_level;

extern "C" int sa_build(int n, const int* rp, const int* cols) {
  std::vector<int> R(rp, rp + n + 1), C(cols, cols + rp[n]);
  return oa::sa::build(n, R, C, g_level) ? g_level.nc : -1;
}

#define OA_SA_FIELD(name)                                                     \
  extern "C" long sa_len_##name() { return (long)g_level.name.size(); }     \
  extern "C" void sa_get_##name(int* out) {                                  \
    std::memcpy(out, g_level.name.data(), sizeof(int) * g_level.name.size()); \
  }
OA_SA_FIELD(agg)
OA_SA_FIELD(prp)
OA_SA_FIELD(pcols)
OA_SA_FIELD(pdiag)
OA_SA_FIELD(pgptr)
OA_SA_FIELD(pglist)
OA_SA_FIELD(ptrp)
OA_SA_FIELD(ptrows)
OA_SA_FIELD(ptsrc)
OA_SA_FIELD(trp)
OA_SA_FIELD(tcols)
OA_SA_FIELD(ttptr)
OA_SA_FIELD(tta)
OA_SA_FIELD(ttp)
OA_SA_FIELD(crp)
OA_SA_FIELD(ccols)
OA_SA_FIELD(cdg)
OA_SA_FIELD(ctptr)
OA_SA_FIELD(ctp)
OA_SA_FIELD(ctt)
