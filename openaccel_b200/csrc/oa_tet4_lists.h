// Contribution lists of the tet4 diffusion assembly (internal, plain C++).
//
// The assembly stages, per element e and corner a, the corner's coefficient
// of every element node k at staged index 16 e + 4 a + k, and per fixed-value
// boundary face f the coefficient of the face's opposite node for side node q
// at 16 ne + 3 f + q. These lists are the element-to-CSR slot map turned
// around: for every CSR entry, the staged indices that sum into it, in
// ascending order (elements in order, then faces), so that the device gather
// is an owner sum in a fixed order. A column missing from its row, which a
// conforming mesh cannot produce (its graph holds every element pair), is
// lumped into the row's diagonal.
#pragma once
#include <algorithm>
#include <climits>
#include <cstdint>
#include <thread>
#include <vector>

namespace oa {
namespace tet4lists {

struct Input {
  int nn = 0, ne = 0, nf = 0;
  const int* row_ptr = nullptr;  // [nn+1] CSR graph, columns ascending per row
  const int* cols = nullptr;     // [nnz]
  const int* diag = nullptr;     // [nn] offset of the diagonal within its row
  const int* conn = nullptr;     // [ne][4]
  const int* face_side = nullptr;   // [nf][3] global side nodes in side order
  const int* face_opp = nullptr;    // [nf] global node opposite the face
  const uint8_t* face_fixed = nullptr;  // [nf] 1: fixed-value face (contributes)
};

// Returns false when the staged indices would not fit 32-bit integers.
inline bool build(const Input& in, std::vector<int>& eptr, std::vector<int>& eidx, std::vector<uint8_t>& ediag) {
  const long long ne = in.ne, nf = in.nf, nnz = in.row_ptr[in.nn];
  if (16 * ne + 3 * nf >= INT_MAX) return false;
  auto slot = [&](int row, int col) -> int {
    const int *b = in.cols + in.row_ptr[row], *e = in.cols + in.row_ptr[row + 1];
    const int* p = std::lower_bound(b, e, col);
    return (p != e && *p == col) ? (int)(p - in.cols) : in.row_ptr[row] + in.diag[row];
  };
  // CSR slot of every staged contribution (-1: a face that is not fixed-value)
  std::vector<int> sl(16 * ne + 3 * nf, -1);
  const int nt = std::max(1, std::min<int>(16, (int)std::thread::hardware_concurrency()));
  auto work = [&](int t) {
    const long long lo = ne * t / nt, hi = ne * (t + 1) / nt;
    for (long long e = lo; e < hi; ++e)
      for (int a = 0; a < 4; ++a)
        for (int k = 0; k < 4; ++k) sl[16 * e + 4 * a + k] = slot(in.conn[4 * e + a], in.conn[4 * e + k]);
  };
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) th.emplace_back(work, t);
  for (auto& t : th) t.join();
  for (long long f = 0; f < nf; ++f)
    if (in.face_fixed[f])
      for (int q = 0; q < 3; ++q) sl[16 * ne + 3 * f + q] = slot(in.face_side[3 * f + q], in.face_opp[f]);
  eptr.assign(nnz + 1, 0);
  for (const int s : sl)
    if (s >= 0) ++eptr[s + 1];
  for (long long s = 0; s < nnz; ++s) eptr[s + 1] += eptr[s];
  eidx.assign(eptr[nnz], 0);
  std::vector<int> pos(eptr.begin(), eptr.end() - 1);
  for (size_t i = 0; i < sl.size(); ++i)
    if (sl[i] >= 0) eidx[pos[sl[i]]++] = (int)i;
  ediag.assign(nnz, 0);
  for (int r = 0; r < in.nn; ++r) ediag[in.row_ptr[r] + in.diag[r]] = 1;
  return true;
}

}  // namespace tet4lists
}  // namespace oa
