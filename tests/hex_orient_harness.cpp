// CPU harness over the hex8 relabelling (openaccel_b200/csrc/oa_hex_orient.h):
// orients a mesh handed in as plain arrays for tests/test_hex_orient.py.
#include <string>
#include <vector>

#include "../openaccel_b200/csrc/oa_hex_orient.h"

extern "C" {
// 0: oriented; 1: not a block (the row kernels take the incident-list lanes);
// 2: not a valid hex mesh
int ho_orient(int nn, int ne, const int* conn, int* out_conn, unsigned char* rot) {
  std::vector<int> oc;
  std::vector<uint8_t> r;
  std::string why;
  bool invalid = false;
  if (!oa::hexorient::orient(nn, ne, conn, oc, r, &why, &invalid)) return invalid ? 2 : 1;
  for (size_t i = 0; i < oc.size(); ++i) out_conn[i] = oc[i];
  for (size_t i = 0; i < r.size(); ++i) rot[i] = r[i];
  return 0;
}
int ho_rotation(int r, int* perm) {
  const auto& R = oa::hexorient::rotations();
  if (r < 0 || r >= (int)R.size()) return 1;
  for (int k = 0; k < 8; ++k) perm[k] = R[r][k];
  return 0;
}
int ho_count() { return (int)oa::hexorient::rotations().size(); }
void ho_ip_map(int r, int q, int* old_ip, int* sign) { oa::hexorient::ip_map(r, q, old_ip, sign); }
int ho_face_map(int r, int f) { return oa::hexorient::face_map(r, f); }
}
