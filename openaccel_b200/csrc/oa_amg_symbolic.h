// Host symbolic phase of the smoothed-aggregation hierarchy (internal, plain
// C++): for one level's CSR graph it builds the aggregates, the structure of
// the smoothed prolongation P = (I - w Dinv A) P_tent and of its transpose,
// and the fixed term lists with which the device recomputes, every time the
// fine values change, P, T = A P and the coarse operator A_c = P^T T as
// deterministic owner sums (one output entry, one ordered list of products).
#pragma once
#include <algorithm>
#include <cstdint>
#include <thread>
#include <utility>
#include <vector>

namespace oa {
namespace sa {

// Greedy aggregation of a CSR graph: a row whose neighbours are all free
// becomes a root and takes them; leftover rows join an adjacent aggregate.
inline int aggregate(int n, const std::vector<int>& rp, const std::vector<int>& cols, std::vector<int>& agg) {
  agg.assign(n, -1);
  int nc = 0;
  for (int i = 0; i < n; ++i) {
    if (agg[i] != -1) continue;
    bool free_nb = true;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (cols[k] != i && agg[cols[k]] != -1) {
        free_nb = false;
        break;
      }
    if (!free_nb) continue;
    agg[i] = nc;
    for (int k = rp[i]; k < rp[i + 1]; ++k) agg[cols[k]] = nc;
    ++nc;
  }
  std::vector<int> pass1(agg);
  for (int i = 0; i < n; ++i) {
    if (agg[i] != -1) continue;
    int best = -1;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (pass1[cols[k]] != -1) {
        best = pass1[cols[k]];
        break;
      }
    agg[i] = best >= 0 ? best : nc++;
  }
  return nc;
}

// Rows of a CSR output built independently: each row appends its entries
// (column, number of terms) and the terms (two indices each); blocks of rows
// run on host threads and are concatenated in row order, so the result does
// not depend on the thread count.
struct RowOut {
  std::vector<int> cols, cnt, ta, tb, rowlen, diag;
};

template <class F>
inline bool build_rows(int nrows, F row_fn, std::vector<int>& rp, std::vector<int>& cols, std::vector<int>& ptr,
                       std::vector<int>& ta, std::vector<int>& tb, std::vector<int>* diag) {
  const int nt = std::max(1, std::min<int>(16, (int)std::thread::hardware_concurrency()));
  const int nb = nrows < 4096 ? 1 : nt;
  std::vector<RowOut> out(nb);
  auto work = [&](int b) {
    const int lo = (int)((long long)nrows * b / nb), hi = (int)((long long)nrows * (b + 1) / nb);
    for (int r = lo; r < hi; ++r) row_fn(r, out[b]);
  };
  if (nb == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (int b = 0; b < nb; ++b) th.emplace_back(work, b);
    for (auto& t : th) t.join();
  }
  size_t ncols = 0, nterms = 0;
  for (const RowOut& o : out) {
    ncols += o.cols.size();
    nterms += o.ta.size();
  }
  if (ncols > (size_t)INT32_MAX / 2 || nterms > (size_t)INT32_MAX / 2) return false;
  rp.assign(nrows + 1, 0);
  cols.clear();
  cols.reserve(ncols);
  ptr.assign(1, 0);
  ptr.reserve(ncols + 1);
  ta.clear();
  tb.clear();
  ta.reserve(nterms);
  tb.reserve(nterms);
  if (diag) diag->assign(nrows, 0);
  int r = 0;
  for (const RowOut& o : out) {
    for (size_t q = 0; q < o.rowlen.size(); ++q, ++r) {
      rp[r + 1] = rp[r] + o.rowlen[q];
      if (diag) (*diag)[r] = o.diag[q];
    }
    cols.insert(cols.end(), o.cols.begin(), o.cols.end());
    for (int c : o.cnt) ptr.push_back(ptr.back() + c);
    ta.insert(ta.end(), o.ta.begin(), o.ta.end());
    tb.insert(tb.end(), o.tb.begin(), o.tb.end());
  }
  return true;
}

struct Level {
  int n = 0, nc = 0;
  std::vector<int> agg;
  // P (n x nc): row pointers, coarse columns, position of the row's own
  // aggregate within the row, and per entry the A entries of the row whose
  // column lies in that aggregate
  std::vector<int> prp, pcols, pdiag, pgptr, pglist;
  // P^T by coarse row: fine rows (ascending) and the P entry of each
  std::vector<int> ptrp, ptrows, ptsrc;
  // T = A P: structure and, per entry, the (A entry, P entry) products
  std::vector<int> trp, tcols, ttptr, tta, ttp;
  // A_c = P^T T: structure, diagonal offsets and the (P entry, T entry) products
  std::vector<int> crp, ccols, cdg, ctptr, ctp, ctt;
};

// Returns false when a term list would overflow 32-bit offsets.
inline bool build(int n, const std::vector<int>& rp, const std::vector<int>& cols, Level& L) {
  L.n = n;
  L.nc = aggregate(n, rp, cols, L.agg);
  const std::vector<int>& agg = L.agg;
  struct Term {
    int col, a, b;
  };
  auto by_col = [](const Term& x, const Term& y) { return x.col < y.col; };
  // append the row's terms grouped by column (stable: list order kept within
  // a column); own = the column whose offset is recorded as the row's diagonal
  auto emit = [](std::vector<Term>& tt, int own, RowOut& o, bool two) {
    int last = -1, len = 0, dg = 0;
    for (const Term& t : tt) {
      if (t.col != last) {
        if (t.col == own) dg = len;
        o.cols.push_back(t.col);
        o.cnt.push_back(0);
        last = t.col;
        ++len;
      }
      o.ta.push_back(t.a);
      if (two) o.tb.push_back(t.b);
      o.cnt.back() += 1;
    }
    o.rowlen.push_back(len);
    o.diag.push_back(dg);
  };
  // P structure and gather lists (term a: the A entry)
  std::vector<int> unused;
  bool ok = build_rows(
      n,
      [&](int i, RowOut& o) {
        thread_local std::vector<Term> tt;
        tt.clear();
        for (int k = rp[i]; k < rp[i + 1]; ++k) tt.push_back({agg[cols[k]], k, 0});
        std::stable_sort(tt.begin(), tt.end(), by_col);
        emit(tt, agg[i], o, false);
      },
      L.prp, L.pcols, L.pgptr, L.pglist, unused, &L.pdiag);
  if (!ok) return false;
  const int nnzP = L.prp[n];
  // P^T
  L.ptrp.assign(L.nc + 1, 0);
  for (int e = 0; e < nnzP; ++e) L.ptrp[L.pcols[e] + 1] += 1;
  for (int c = 0; c < L.nc; ++c) L.ptrp[c + 1] += L.ptrp[c];
  L.ptrows.assign(nnzP, 0);
  L.ptsrc.assign(nnzP, 0);
  {
    std::vector<int> pos(L.ptrp.begin(), L.ptrp.end() - 1);
    for (int i = 0; i < n; ++i)
      for (int e = L.prp[i]; e < L.prp[i + 1]; ++e) {
        const int q = pos[L.pcols[e]]++;
        L.ptrows[q] = i;
        L.ptsrc[q] = e;
      }
  }
  // T = A P (terms: A entry, P entry)
  ok = build_rows(
      n,
      [&](int i, RowOut& o) {
        thread_local std::vector<Term> tt;
        tt.clear();
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
          const int j = cols[k];
          for (int e = L.prp[j]; e < L.prp[j + 1]; ++e) tt.push_back({L.pcols[e], k, e});
        }
        std::stable_sort(tt.begin(), tt.end(), by_col);
        emit(tt, -1, o, true);
      },
      L.trp, L.tcols, L.ttptr, L.tta, L.ttp, nullptr);
  if (!ok) return false;
  // A_c = P^T T (terms: P entry, T entry), coarse rows
  ok = build_rows(
      L.nc,
      [&](int c, RowOut& o) {
        thread_local std::vector<Term> tt;
        tt.clear();
        for (int q = L.ptrp[c]; q < L.ptrp[c + 1]; ++q) {
          const int i = L.ptrows[q], e = L.ptsrc[q];
          for (int t = L.trp[i]; t < L.trp[i + 1]; ++t) tt.push_back({L.tcols[t], e, t});
        }
        std::stable_sort(tt.begin(), tt.end(), by_col);
        emit(tt, c, o, true);
      },
      L.crp, L.ccols, L.ctptr, L.ctp, L.ctt, &L.cdg);
  return ok;
}

}  // namespace sa
}  // namespace oa
