// CPU harness over the tet4 assembly's contribution-list builder
// (openaccel_b200/csrc/oa_tet4_lists.h): builds the lists for a mesh handed
// in as plain arrays and exposes them to tests/test_tet4_lists.py.
#include <vector>

#include "../openaccel_b200/csrc/oa_tet4_lists.h"

static std::vector<int> g_eptr, g_eidx;
static std::vector<uint8_t> g_ediag;

extern "C" {
int tl_build(int nn, int ne, int nf, const int* row_ptr, const int* cols, const int* diag, const int* conn,
             const int* face_side, const int* face_opp, const unsigned char* face_fixed) {
  oa::tet4lists::Input in;
  in.nn = nn;
  in.ne = ne;
  in.nf = nf;
  in.row_ptr = row_ptr;
  in.cols = cols;
  in.diag = diag;
  in.conn = conn;
  in.face_side = face_side;
  in.face_opp = face_opp;
  in.face_fixed = face_fixed;
  return oa::tet4lists::build(in, g_eptr, g_eidx, g_ediag) ? 0 : 1;
}
long tl_len_eidx() { return (long)g_eidx.size(); }
void tl_get(int* eptr, int* eidx, unsigned char* ediag) {
  for (size_t i = 0; i < g_eptr.size(); ++i) eptr[i] = g_eptr[i];
  for (size_t i = 0; i < g_eidx.size(); ++i) eidx[i] = g_eidx[i];
  for (size_t i = 0; i < g_ediag.size(); ++i) ediag[i] = g_ediag[i];
}
}
