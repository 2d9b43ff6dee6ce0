// Host-side relabelling of hex8 elements into a consistently oriented block
// (internal; plain C++, no CUDA).
//
// The hex8 row kernels take, for every node, the element in which it is local
// corner c, for c = 0..7: around every node the elements must sit in the
// 2x2x2 arrangement of a block whose elements share one local orientation.
// Meshes written by other tools number the corners of some elements from a
// different starting corner or axis (the reference's own cavity example does).
// Any proper rotation of the reference cube maps an element onto itself with
// its corners relabelled and the Jacobian sign kept, so each element can be
// rotated (24 choices) until its neighbours agree: a breadth-first walk across
// shared faces fixes the rotation of each element from an already oriented
// neighbour, whose face is the opposite face of the neighbour's (same
// positions in the other two axes). A mesh where two walks disagree is not a
// block (for instance a node where 3 or 5 elements meet around an edge): the
// row kernels then run with 16 lanes per row on the caller's labelling.
#pragma once
#include <algorithm>
#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace oa {
namespace hexorient {

// Nalu hex8 corner signs (-1 / +1 per axis), faces and SCS ip edges.
constexpr int SIGN[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                            {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
constexpr int FACE[6][4] = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
constexpr int LR[12][2] = {{0, 1}, {1, 2}, {2, 3}, {0, 3}, {4, 5}, {5, 6},
                           {6, 7}, {4, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

inline int corner_of(const int s[3]) {
  for (int c = 0; c < 8; ++c)
    if (SIGN[c][0] == s[0] && SIGN[c][1] == s[1] && SIGN[c][2] == s[2]) return c;
  return -1;
}

// The 24 proper rotations of the cube as corner permutations: P[r][k] is the
// old corner that becomes new corner k (new_conn[k] = old_conn[P[r][k]]).
// Generated from the signed permutation matrices of determinant +1.
inline const std::vector<std::array<int, 8>>& rotations() {
  static const std::vector<std::array<int, 8>> R = [] {
    std::vector<std::array<int, 8>> out;
    const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    const int parity[6] = {1, -1, -1, 1, 1, -1};
    for (int p = 0; p < 6; ++p)
      for (int sg = 0; sg < 8; ++sg) {
        const int s[3] = {(sg & 1) ? -1 : 1, (sg & 2) ? -1 : 1, (sg & 4) ? -1 : 1};
        if (parity[p] * s[0] * s[1] * s[2] != 1) continue;  // proper rotations only
        std::array<int, 8> P{};
        for (int k = 0; k < 8; ++k) {
          // new corner k sits where the rotation takes old corner P[k]:
          // x_new = M x_old with M[i][perm[i]] = s[i]
          int old[3];
          for (int i = 0; i < 3; ++i) old[perms[p][i]] = s[i] * SIGN[k][i];
          P[k] = corner_of(old);
        }
        out.push_back(P);
      }
    // identity first
    std::stable_partition(out.begin(), out.end(), [](const std::array<int, 8>& P) {
      for (int k = 0; k < 8; ++k)
        if (P[k] != k) return false;
      return true;
    });
    return out;
  }();
  return R;
}

// Old SCS ip (and its orientation, +1 or -1) of new ip q under rotation r.
inline void ip_map(int r, int q, int* old_ip, int* sign) {
  const auto& P = rotations()[r];
  const int a = P[LR[q][0]], b = P[LR[q][1]];
  for (int o = 0; o < 12; ++o) {
    if (LR[o][0] == a && LR[o][1] == b) {
      *old_ip = o;
      *sign = 1;
      return;
    }
    if (LR[o][0] == b && LR[o][1] == a) {
      *old_ip = o;
      *sign = -1;
      return;
    }
  }
  *old_ip = -1;
  *sign = 0;
}

// New face ordinal of old face f under rotation r.
inline int face_map(int r, int f) {
  const auto& P = rotations()[r];
  int inv[8];
  for (int k = 0; k < 8; ++k) inv[P[k]] = k;
  int c[4];
  for (int k = 0; k < 4; ++k) c[k] = inv[FACE[f][k]];
  std::sort(c, c + 4);
  for (int g = 0; g < 6; ++g) {
    int d[4] = {FACE[g][0], FACE[g][1], FACE[g][2], FACE[g][3]};
    std::sort(d, d + 4);
    if (std::equal(c, c + 4, d)) return g;
  }
  return -1;
}

// Orient every element. conn [ne][8] in, out_conn / rot [ne] out (rot = index
// into rotations(), 0 = unchanged). Returns false with a reason when the mesh
// is not a consistently orientable block; *invalid (when given) is then set if
// the mesh is not a valid hex mesh at all (a face shared by three elements)
// rather than only not a block.
inline bool orient(int nn, int ne, const int* conn, std::vector<int>& out_conn, std::vector<uint8_t>& rot,
                   std::string* why, bool* invalid = nullptr) {
  if (invalid) *invalid = false;
  const auto& R = rotations();
  out_conn.assign(conn, conn + 8L * ne);
  rot.assign(ne, 0);
  std::vector<char> done(ne, 0);
  // face -> elements, keyed by its sorted node ids
  std::map<std::array<int, 4>, std::vector<std::pair<int, int>>> faces;
  for (int e = 0; e < ne; ++e)
    for (int f = 0; f < 6; ++f) {
      std::array<int, 4> k;
      for (int j = 0; j < 4; ++j) k[j] = conn[8L * e + FACE[f][j]];
      std::sort(k.begin(), k.end());
      faces[k].push_back({e, f});
    }
  for (auto& kv : faces)
    if (kv.second.size() > 2) {
      if (why) *why = "a face is shared by more than two elements";
      if (invalid) *invalid = true;
      return false;
    }
  std::vector<int> queue;
  for (int root = 0; root < ne; ++root) {
    if (done[root]) continue;
    done[root] = 1;  // a component's first element keeps its labelling
    queue.assign(1, root);
    for (size_t qi = 0; qi < queue.size(); ++qi) {
      const int e = queue[qi];
      const int* ec = &out_conn[8L * e];
      for (int f = 0; f < 6; ++f) {
        std::array<int, 4> k;
        for (int j = 0; j < 4; ++j) k[j] = ec[FACE[f][j]];
        std::sort(k.begin(), k.end());
        const auto& sh = faces[k];
        if (sh.size() != 2) continue;
        const int g = sh[0].first == e ? sh[1].first : sh[0].first;
        // axis and side of face f of e; the neighbour's copy of each shared
        // node sits at the same signs in the other two axes, opposite side
        int ax = 0;
        for (int a = 0; a < 3; ++a) {
          int s0 = SIGN[FACE[f][0]][a];
          bool same = true;
          for (int j = 1; j < 4; ++j) same = same && SIGN[FACE[f][j]][a] == s0;
          if (same) ax = a;
        }
        int want[8];  // want[new corner of g] = node id, -1 unknown
        for (int c = 0; c < 8; ++c) want[c] = -1;
        for (int j = 0; j < 4; ++j) {
          const int ce = FACE[f][j];
          int s[3] = {SIGN[ce][0], SIGN[ce][1], SIGN[ce][2]};
          s[ax] = -s[ax];
          want[corner_of(s)] = ec[ce];
        }
        // the rotation of g's original labelling that puts those nodes there
        const int* gc = conn + 8L * g;
        int found = -1;
        for (int r = 0; r < (int)R.size() && found < 0; ++r) {
          bool ok = true;
          for (int c = 0; c < 8 && ok; ++c)
            if (want[c] >= 0 && gc[R[r][c]] != want[c]) ok = false;
          if (ok) found = r;
        }
        if (found < 0) {
          if (why) *why = "two neighbouring elements share a face in an incompatible way";
          return false;
        }
        if (done[g]) {
          if ((int)rot[g] != found) {
            if (why) *why = "elements cannot be given one consistent orientation (not a block-structured mesh)";
            return false;
          }
          continue;
        }
        done[g] = 1;
        rot[g] = (uint8_t)found;
        for (int c = 0; c < 8; ++c) out_conn[8L * g + c] = gc[R[found][c]];
        queue.push_back(g);
      }
    }
  }
  (void)nn;
  return true;
}

}  // namespace hexorient
}  // namespace oa
