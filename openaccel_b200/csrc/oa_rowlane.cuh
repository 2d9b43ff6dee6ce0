// Row-owner ("corner-lane") execution model shared by the hex8 kernels.
//
// Eight (or sixteen) consecutive lanes own one CSR row (mesh node). Each lane
// handles one incident element, in the canonical frame of oa_hex8.cuh that
// puts the row node at corner 0. Per-lane partial sums are combined in a fixed
// order — xor-butterflies for the diagonal block and the rhs, and an ordered
// shared-memory gather for off-diagonal slots — so every CSR entry is written
// exactly once, deterministically, without atomics and without a zero fill.
#pragma once
#include <cstdint>

#include "oa_hex8.cuh"
#include "oa_internal.h"

namespace oa {

constexpr unsigned FULL_MASK = 0xffffffffu;

// Lanes per row: 8 on consistently oriented block meshes, where lane c takes
// the element in which the node is corner c, and 16 on other hex meshes
// (3, 5, ... elements around an edge), where the lanes take the node's
// incident (element, corner) pairs in element order. n2e holds LPR entries per
// node, element * 8 + corner, or -1.
template <int LPR>
struct RowLane {
  int row, li, e, c;
  bool rv;
};

template <int LPR>
__device__ __forceinline__ RowLane<LPR> row_lane(const MeshView& m) {
  static_assert(LPR == 8 || LPR == 16, "8 or 16 lanes per row");
  RowLane<LPR> r;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  r.row = (int)(t / LPR);
  r.li = threadIdx.x & (LPR - 1);
  r.rv = r.row < m.nn;
  const int ec = r.rv ? __ldg(m.n2e + (size_t)LPR * r.row + r.li) : -1;
  r.e = ec >= 0 ? (ec >> 3) : -1;
  r.c = ec >= 0 ? (ec & 7) : 0;
  return r;
}

// ROT_PERM / ROT_IP / ROT_FACE rows packed into one word so a lane can select
// its row without an indexed constant load (8 distinct addresses per warp).
__device__ __forceinline__ uint32_t perm_word(int c) {
  // 3 bits per canonical node k = 0..7
  switch (c) {
    case 0: return 0u | 1u << 3 | 2u << 6 | 3u << 9 | 4u << 12 | 5u << 15 | 6u << 18 | 7u << 21;
    case 1: return 1u | 0u << 3 | 4u << 6 | 5u << 9 | 2u << 12 | 3u << 15 | 7u << 18 | 6u << 21;
    case 2: return 2u | 3u << 3 | 0u << 6 | 1u << 9 | 6u << 12 | 7u << 15 | 4u << 18 | 5u << 21;
    case 3: return 3u | 2u << 3 | 6u << 6 | 7u << 9 | 0u << 12 | 1u << 15 | 5u << 18 | 4u << 21;
    case 4: return 4u | 5u << 3 | 1u << 6 | 0u << 9 | 7u << 12 | 6u << 15 | 2u << 18 | 3u << 21;
    case 5: return 5u | 4u << 3 | 7u << 6 | 6u << 9 | 1u << 12 | 0u << 15 | 3u << 18 | 2u << 21;
    case 6: return 6u | 7u << 3 | 3u << 6 | 2u << 9 | 5u << 12 | 4u << 15 | 0u << 18 | 1u << 21;
    default: return 7u | 6u << 3 | 5u << 6 | 4u << 9 | 3u << 12 | 2u << 15 | 1u << 18 | 0u << 21;
  }
}
// 5 bits per canonical ip q = 0..2: original ip * 2 + (sign < 0)
__device__ __forceinline__ uint32_t ip_word(int c) {
  switch (c) {
    case 0: return 0u | 6u << 5 | 16u << 10;
    case 1: return 1u | 18u << 5 | 2u << 10;
    case 2: return 4u | 3u << 5 | 20u << 10;
    case 3: return 5u | 22u << 5 | 7u << 10;
    case 4: return 8u | 17u << 5 | 14u << 10;
    case 5: return 9u | 10u << 5 | 19u << 10;
    case 6: return 12u | 21u << 5 | 11u << 10;
    default: return 13u | 15u << 5 | 23u << 10;
  }
}
// 3 bits per canonical face q = 0..2 (faces 0, 3, 4): original face ordinal
__device__ __forceinline__ uint32_t face_word(int c) {
  switch (c) {
    case 0: return 0u | 3u << 3 | 4u << 6;
    case 1: return 4u | 1u << 3 | 0u << 6;
    case 2: return 2u | 1u << 3 | 4u << 6;
    case 3: return 4u | 3u << 3 | 2u << 6;
    case 4: return 5u | 3u << 3 | 0u << 6;
    case 5: return 0u | 1u << 3 | 5u << 6;
    case 6: return 5u | 1u << 3 | 2u << 6;
    default: return 2u | 3u << 3 | 5u << 6;
  }
}

__device__ __forceinline__ int perm_at(uint32_t w, int k) { return (w >> (3 * k)) & 7; }

// sum over a row's lanes (xor butterflies: every lane gets the same value)
template <int LPR, class T>
__device__ __forceinline__ T rowsum(T v) {
  v += __shfl_xor_sync(FULL_MASK, v, 1);
  v += __shfl_xor_sync(FULL_MASK, v, 2);
  v += __shfl_xor_sync(FULL_MASK, v, 4);
  if (LPR == 16) v += __shfl_xor_sync(FULL_MASK, v, 8);
  return v;
}

// Canonical target of element column a for the row at canonical corner 0 in
// the reduced (edge) stencil: 1, 3, 4 are edge neighbours (slots 0, 1, 2);
// 0 is the row itself and 2, 5, 6, 7 (face/body diagonals) are lumped into the
// diagonal block, as applyCoeff_'s deductUnfound does (assembler.h:423-445).
__host__ __device__ constexpr int nb_slot(int a) { return a == 1 ? 0 : (a == 3 ? 1 : (a == 4 ? 2 : -1)); }

// Edge neighbours of corner c in the order of a lane's neighbour slots
// (canonical nodes 1, 3, 4 of the rotation that maps c to corner 0).
__host__ __device__ constexpr int edge_nbr(int c, int s) {
  constexpr int T[8][3] = {{1, 3, 4}, {0, 5, 2}, {3, 1, 6}, {2, 7, 0}, {5, 0, 7}, {4, 6, 1}, {7, 2, 5}, {6, 4, 3}};
  return T[c][s];
}

}  // namespace oa
