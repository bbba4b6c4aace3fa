// Host symbolic analysis (ordering, etree, supernodes, contribution rows).
//
// Each routine restates the step of the reference's symbolic phase named in
// its comment. The integer results are the contract (they fix the front
// structure of every supernode, hence the delayed pivots and the inertia
// bookkeeping), so the order of operations - including tie-breaking in
// degree lists and sorts - follows the reference step for step.
#include "symbolic.h"

#include <algorithm>
#include <cmath>
#include <climits>
#include <cstdint>
#include <utility>
#include <cstdio>
#include <numeric>
#include <stdexcept>

namespace b200ldl {

namespace {

// Sort, drop negative entries and duplicates; returns the new length
// (block_amd.h:459-477).
int sort_unique_nonneg(int len, int* a) {
  std::sort(a, a + len);
  int i = 0;
  int j = 0;
  while (i < len && a[i] < 0) i++;
  for (; i < len; i++, j++) {
    while (i < len - 1 && a[i] == a[i + 1]) i++;
    if (i != j) a[j] = a[i];
  }
  return j;
}

// element lists up to this length test every pair directly
constexpr int kMergeScanMax = 48;
// re-keyed positions looked up linearly before the sorted keys are rebuilt
constexpr size_t kMergeExtraMax = 64;
// rows longer than this at the start (a dense row, e.g. a constraint
// coupled to every design variable) keep their slen sum and row hash up to
// date instead of rescanning the row at every pivot that touches it
constexpr int kTrackRow = 256;
constexpr int kTrackMaxRows = 64;

// a 64-bit mixing function (splitmix64's finalizer)
inline uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

// Bucketed degree lists with LIFO buckets and a monotonically non-increasing
// minimum pointer (block_amd.h:687-812).
struct DegreeBuckets {
  int size;
  int min_degree = 0;
  std::vector<int> degree, first, next, prev;

  DegreeBuckets(int size_, const int* rowp)
      : size(size_), degree(size_), first(size_ + 1, -1), next(size_ + 1, -1),
        prev(size_ + 1, -1) {
    for (int i = 0; i < size; i++) {
      degree[i] = rowp[i + 1] - rowp[i];
      if (i == 0 || degree[i] < min_degree) min_degree = degree[i];
    }
    for (int i = 0; i < size; i++) push_front(i, degree[i]);
  }
  void push_front(int i, int d) {
    if (first[d] != -1) {
      prev[first[d]] = i;
      next[i] = first[d];
    }
    first[d] = i;
  }
  void unlink(int i) {
    const int d = degree[i];
    if (first[d] == i) first[d] = next[i];
    if (next[i] != -1) prev[next[i]] = prev[i];
    if (prev[i] != -1) next[prev[i]] = next[i];
    prev[i] = -1;
    next[i] = -1;
  }
  void set(int i, int d) {
    if (d < min_degree) min_degree = d;
    unlink(i);
    push_front(i, d);
    degree[i] = d;
  }
  int pick() const {
    for (int d = min_degree; d <= size; d++)
      if (first[d] != -1) return first[d];
    return -1;
  }
};

// Quotient graph stored in one CSR-like array: row r holds elen[r] element
// ids followed by (alen[r] - elen[r]) variable ids in cols[rowp[r]..].
struct QuotientGraph {
  int n;
  int* rowp;
  int* cols;
  std::vector<int> alen, elen;

  // Make room for `need` more entries at the end of row r by compacting the
  // rows before it (towards lower addresses), then, if that is not enough,
  // the rows after it (towards higher addresses) (block_amd.h:531-581).
  void make_room(int r, int need) {
    int got = 0;
    if (r > 0) {
      int s = r - 1;
      for (; got < need && s >= 0; s--) got += (rowp[s + 1] - rowp[s]) - alen[s];
      s++;
      int dst = rowp[s] + alen[s];
      for (int i = s + 1; i <= r; i++) {
        int src = rowp[i];
        const int new_start = dst;
        const int stop = src + alen[i];
        for (; src < stop; src++, dst++) cols[dst] = cols[src];
        rowp[i] = new_start;
      }
    }
    if (got < need) {
      int s = r + 1;
      for (; got < need && s < n; s++) got += (rowp[s + 1] - rowp[s]) - alen[s];
      s--;
      if (s >= n) {
        s = n - 1;
        std::fprintf(stderr, "b200ldl: quotient graph out of space\n");
      }
      int dst = rowp[s + 1] - 1;
      for (int i = s; i > r; i--) {
        const int lo = rowp[i];
        for (int src = lo + alen[i] - 1; src >= lo; src--, dst--) cols[dst] = cols[src];
        rowp[i] = rowp[i + 1] - alen[i];
      }
    }
  }

  // Indistinguishable-variable test (block_amd.h:600-630); it walks both
  // lists in lock step, skipping the other variable once on each side.
  bool same_adjacency(int a, int b) const {
    if (a == b) return false;
    if (alen[a] != alen[b] || elen[a] != elen[b]) return false;
    int pa = rowp[a];
    int pb = rowp[b];
    const int ea = pa + alen[a];
    const int eb = pb + alen[b];
    for (int k = 0; k < alen[a]; k++, pa++, pb++) {
      if (cols[pa] == b) pa++;
      if (cols[pb] == a) pb++;
      if (cols[pa] != cols[pb]) break;
    }
    return pa == ea && pb == eb;
  }

  // Delete variable v from the rows of its elements and neighbours
  // (block_amd.h:637-681).
  void drop_variable(int v) {
    int i = rowp[v];
    for (; i < rowp[v] + elen[v]; i++) {
      const int e = cols[i];
      int j = rowp[e];
      const int last = rowp[e] + alen[e] - 1;
      while (j < last && cols[j] != v) j++;
      for (; j < last; j++) cols[j] = cols[j + 1];
      alen[e]--;
    }
    for (; i < rowp[v] + alen[v]; i++) {
      const int w = cols[i];
      int j = rowp[w] + elen[w];
      const int last = rowp[w] + alen[w] - 1;
      while (j < last && cols[j] != v) j++;
      for (; j < last; j++) cols[j] = cols[j + 1];
      alen[w]--;
    }
    elen[v] = 0;
    alen[v] = 0;
  }
};

}  // namespace

// Approximate minimum degree with element absorption and supervariables,
// as BlockAMD::amd with no forced-last multipliers and the approximate
// degree (block_amd.h:27-452, called from ordering_utils.h:202-221).
int amd_order(int n, int* rowp, int* cols, int* perm) {
  QuotientGraph g{n, rowp, cols, std::vector<int>(n), std::vector<int>(n, 0)};
  std::vector<int> slen(n, 1), state(n, 1), elem_deg(n, -1), Lp(n);
  for (int i = 0; i < n; i++) {
    perm[i] = i;
    g.alen[i] = rowp[i + 1] - rowp[i];
  }
  // input format check (strictly increasing, non-negative rows)
  for (int i = 0; i < n; i++) {
    for (int j = rowp[i]; j < rowp[i] + g.alen[i] - 1; j++) {
      if (cols[j] < 0 || cols[j + 1] < 0 || cols[j + 1] <= cols[j]) return i + 1;
    }
  }

  DegreeBuckets deg(n, rowp);
  // Long rows: vsum[v] = sum of slen over v's variable part, rhash[v] = sum
  // of mix64 over v's whole row, kept exact through every change to the row
  // (prune, new element, variable drop) and to slen (merge).
  std::vector<char> tracked(n, 0);
  std::vector<long long> vsum(n, 0);
  std::vector<uint64_t> rhash(n, 0);
  std::vector<int> tracked_list;
  // esum[e] = sum of slen over the row of live element e, kept with the row
  std::vector<long long> esum(n, 0);
  // slen summed over element e's row (the running sum of a live element)
  auto element_size = [&](int e) {
    if (state[e] == 0) return (int)esum[e];
    int t = 0;
    for (int p = rowp[e]; p < rowp[e] + g.alen[e]; p++) t += slen[cols[p]];
    return t;
  };
  // For a long row T: esumT[T] = sum over T's elements of their slen sums
  // (0 for a dead element), kept with T's element part and with esum.
  std::vector<long long> esumT(n, 0), corr(n, 0);
  std::vector<int> tl;  // long rows in the current Lp
  // held[e] bit b: the long row tracked_list[b] holds element e (set and
  // cleared with the row's element part: insertion of a new element, prune
  // of absorbed ones)
  std::vector<uint64_t> held(n, 0);
  std::vector<int> tbit(n, -1);
  auto elem_in = [&](int t, int e) { return (held[e] >> tbit[t]) & 1u; };
  auto elem_value = [&](int e) { return state[e] == 0 ? esum[e] : 0LL; };
  auto elem_has = [&](int e, int x) {
    const int* b = cols + rowp[e];
    return std::binary_search(b, b + g.alen[e], x);
  };
  for (int v = 0; v < n; v++)
    if (g.alen[v] > kTrackRow) tracked_list.push_back(v);
  // the longest few only: every merge checks each tracked row
  std::stable_sort(tracked_list.begin(), tracked_list.end(),
                   [&](int x, int y) { return g.alen[x] > g.alen[y]; });
  if (tracked_list.size() > (size_t)kTrackMaxRows) tracked_list.resize(kTrackMaxRows);
  for (size_t b = 0; b < tracked_list.size(); b++) tbit[tracked_list[b]] = (int)b;
  for (const int v : tracked_list) {
    tracked[v] = 1;
    for (int q = rowp[v]; q < rowp[v] + g.alen[v]; q++) {
      vsum[v] += slen[cols[q]];
      rhash[v] += mix64((uint64_t)cols[q]);
    }
  }
  auto in_vars = [&](int v, int x) {
    const int* b = cols + rowp[v] + g.elen[v];
    const int* e = cols + rowp[v] + g.alen[v];
    return std::binary_search(b, e, x);
  };
  // supervariable detection on long lists (see the merge step)
  std::vector<int> lp_pos(n, -1), touched;
  std::vector<uint64_t> merge_keys;
  std::vector<int> head[2], chain[2], extra[2];
  int nsv = 0;
  for (int i = 0; i < n; nsv++) {
    const int piv = deg.pick();
    deg.unlink(piv);
    perm[nsv] = piv;
    state[piv] = 0;
    tracked[piv] = 0;  // its row becomes the new element's

    // Lp = {piv} U adj(piv) U adj(elements of piv)
    int len = 0;
    Lp[len++] = piv;
    for (int j = rowp[piv] + g.elen[piv]; j < rowp[piv] + g.alen[piv]; j++)
      if (cols[j] != piv) Lp[len++] = cols[j];
    for (int j = rowp[piv]; j < rowp[piv] + g.elen[piv]; j++) {
      const int e = cols[j];
      for (int k = rowp[e] + g.elen[e]; k < rowp[e] + g.alen[e]; k++) {
        if (len >= n) len = sort_unique_nonneg(len, Lp.data());
        if (cols[k] != piv) Lp[len++] = cols[k];
      }
    }
    len = sort_unique_nonneg(len, Lp.data());

    // prune absorbed elements and Lp members from every row in Lp
    for (int j = 0; j < len; j++) {
      const int v = Lp[j];
      if (v == piv) continue;
      int removed_e = 0;
      if (tracked[v]) {
        // the same entries by binary search over v's (sorted) element part
        int* eb = cols + rowp[v];
        int* ee = cols + rowp[v] + g.elen[v];
        for (int k = rowp[piv]; k < rowp[piv] + g.elen[piv]; k++) {
          int* it = std::lower_bound(eb, ee, cols[k]);
          if (it != ee && *it == cols[k]) {
            rhash[v] -= mix64((uint64_t)*it);
            esumT[v] -= elem_value(*it);
            held[*it] &= ~(1ull << tbit[v]);
            *it = -1;
            removed_e++;
            eb = it + 1;
          } else {
            eb = it;
          }
        }
      } else {
        int k = rowp[piv];
        const int kend = rowp[piv] + g.elen[piv];
        for (int c = rowp[v]; k < kend && c < rowp[v] + g.elen[v]; c++) {
          while (k < kend && cols[k] < cols[c]) k++;
          if (k < kend && cols[k] == cols[c]) {
            if (tracked[v]) rhash[v] -= mix64((uint64_t)cols[c]);
            cols[c] = -1;
            removed_e++;
          }
        }
      }
      int removed_v = 0;
      if (tracked[v]) {
        // the same entries by binary search over the (sorted) variable part
        int* vb = cols + rowp[v] + g.elen[v];
        int* ve = cols + rowp[v] + g.alen[v];
        for (int k = 0; k < len; k++) {
          int* it = std::lower_bound(vb, ve, Lp[k]);
          if (it != ve && *it == Lp[k]) {
            vsum[v] -= slen[Lp[k]];
            rhash[v] -= mix64((uint64_t)Lp[k]);
            *it = -1;
            removed_v++;
            vb = it + 1;
          } else {
            vb = it;
          }
        }
      } else {
        int k = 0;
        for (int c = rowp[v] + g.elen[v]; k < len && c < rowp[v] + g.alen[v]; c++) {
          while (k < len && Lp[k] < cols[c]) k++;
          if (k < len && cols[c] == Lp[k]) {
            cols[c] = -1;
            removed_v++;
          }
        }
      }
      if (removed_e > 0 || removed_v > 0) {
        const int stop = rowp[v] + g.alen[v];
        int k = rowp[v];
        int dst = k;
        for (; k < stop; k++, dst++) {
          while (k < stop && cols[k] == -1) k++;
          if (k < stop) cols[dst] = cols[k];
        }
        g.elen[v] -= removed_e;
        g.alen[v] -= removed_e + removed_v;
      }
    }

    // piv becomes an element of every row in Lp \ {piv}, kept sorted
    for (int j = 0; j < len; j++) {
      const int v = Lp[j];
      if (v == piv) continue;
      if (g.alen[v] == rowp[v + 1] - rowp[v]) g.make_room(v, 1);
      int k = rowp[v];
      const int kend = k + g.elen[v];
      while (k < kend && cols[k] < piv) k++;
      if (cols[k] != piv) {
        for (int p = rowp[v] + g.alen[v] - 1; p >= k; p--) cols[p + 1] = cols[p];
        cols[k] = piv;
        g.alen[v] += 1;
        g.elen[v] += 1;
        if (tracked[v]) {
          rhash[v] += mix64((uint64_t)piv);
          held[piv] |= 1ull << tbit[v];
        }
      }
    }

    // the elements adjacent to piv are absorbed into it
    for (int j = rowp[piv]; j < rowp[piv] + g.elen[piv]; j++) {
      const int e = cols[j];
      for (uint64_t m = held[e]; m; m &= m - 1) {
        const int t = tracked_list[__builtin_ctzll(m)];
        if (tracked[t]) esumT[t] -= elem_value(e);
      }
      g.alen[e] = 0;
      g.elen[e] = 0;
      state[e] = -1;
    }

    // row piv now lists the variables of the new element
    const int cap = rowp[piv + 1] - rowp[piv];
    if (len - 1 > cap) g.make_room(piv, len - 1 - (rowp[piv + 1] - rowp[piv]));
    g.elen[piv] = 0;
    g.alen[piv] = len - 1;
    for (int j = rowp[piv], k = 0; k < len; k++, j++) {
      if (Lp[k] == piv) {
        k++;
        if (k == len) break;
      }
      cols[j] = Lp[k];
    }
    esum[piv] = 0;
    for (int k = 0; k < len; k++)
      if (Lp[k] != piv) esum[piv] += slen[Lp[k]];
    for (int k = 0; k < len; k++)
      if (Lp[k] != piv && tracked[Lp[k]]) esumT[Lp[k]] += esum[piv];

    // approximate external degrees |A_v \ v| + |Lp \ v| + sum_e |L_e \ Lp|.
    // elem_deg[e] = |L_e| minus slen of every member of Lp holding e. A long
    // row T in Lp does not walk its elements: each element's first visitor
    // subtracts slen[T] when T holds it, and T's own sum comes from esumT
    // minus corr[T] = sum over T's elements of the slen of the Lp members
    // that hold them.
    tl.clear();
    for (int j = 0; j < len; j++)
      if (Lp[j] != piv && tracked[Lp[j]]) tl.push_back(Lp[j]);
    for (const int t : tl) {
      corr[t] = (long long)slen[t] * g.elen[t];
      for (const int u : tl) {
        if (u == t) continue;
        // |elements(t) and elements(u)| by a merge of the sorted lists
        long long both = 0;
        int x = rowp[t], y = rowp[u];
        const int xe = rowp[t] + g.elen[t], ye = rowp[u] + g.elen[u];
        while (x < xe && y < ye) {
          if (cols[x] < cols[y])
            x++;
          else if (cols[y] < cols[x])
            y++;
          else {
            both++;
            x++;
            y++;
          }
        }
        corr[t] += (long long)slen[u] * both;
      }
    }
    for (int j = 0; j < len; j++) {
      const int v = Lp[j];
      if (v != piv && tracked[v]) continue;
      for (int k = rowp[v]; k < rowp[v] + g.elen[v]; k++) {
        const int e = cols[k];
        if (elem_deg[e] < 0) {
          elem_deg[e] = element_size(e);
          for (const int t : tl)
            if (elem_in(t, e)) elem_deg[e] -= slen[t];
        }
        elem_deg[e] -= slen[v];
        for (const int t : tl)
          if (elem_in(t, e)) corr[t] += slen[v];
      }
    }
    int deg_lp = 0;
    for (int j = 0; j < len; j++)
      if (Lp[j] != piv) deg_lp += slen[Lp[j]];

    for (int j = 0; j < len; j++) {
      const int v = Lp[j];
      if (v == piv) continue;
      int est = deg_lp;
      if (tracked[v])
        est += (int)vsum[v];
      else
        for (int k = rowp[v] + g.elen[v]; k < rowp[v] + g.alen[v]; k++) est += slen[cols[k]];
      const int vs = rowp[v] + g.elen[v];
      const int vl = g.alen[v] - g.elen[v];
      if (vl > 0 && std::binary_search(cols + vs, cols + vs + vl, v)) est -= slen[v];
      if (std::binary_search(Lp.data(), Lp.data() + len, v)) est -= slen[v];
      if (tracked[v]) {
        // piv's own term is |L_piv| - deg_lp, zero, and is excluded
        est += (int)(esumT[v] - corr[v] - (esum[piv] - deg_lp));
      } else {
        for (int k = rowp[v]; k < rowp[v] + g.elen[v]; k++) {
          const int e = cols[k];
          if (e == piv) continue;
          if (elem_deg[e] < 0) {
            elem_deg[e] = element_size(e);
          }
          est += elem_deg[e];
        }
      }
      est = std::min(est, n - i);
      const int d = std::min(est, deg.degree[v] + deg_lp);
      deg.set(v, d);
    }
    for (int j = 0; j < len; j++) {
      const int v = Lp[j];
      if (v != piv && tracked[v]) continue;  // its elements were set by others, if at all
      for (int k = rowp[v]; k < rowp[v] + g.elen[v]; k++) elem_deg[cols[k]] = -1;
    }

    // merge indistinguishable variables of Lp into supervariables: pairs
    // (Lp[j], Lp[k]), k > j, are tested in order and a match is merged at
    // once (later tests see the merged graph)
    auto merge = [&](int a, int b) {
      const int sb = slen[b];
      const int nb = -(a + 1);  // slen[b] after the merge
      // the long rows that hold a or b see their slen change
      for (const int t : tracked_list) {
        if (!tracked[t]) continue;
        if (in_vars(t, a)) vsum[t] += sb;
        if (in_vars(t, b)) vsum[t] += (long long)nb - sb;
      }
      // live elements holding a or b see their slen change; every element
      // that holds a variable is in that variable's element list
      for (int q = rowp[a]; q < rowp[a] + g.elen[a]; q++) {
        const int e = cols[q];
        if (state[e] == 0 && elem_has(e, a)) {
          esum[e] += sb;
          for (uint64_t m = held[e]; m; m &= m - 1) {
            const int t = tracked_list[__builtin_ctzll(m)];
            if (tracked[t]) esumT[t] += sb;
          }
        }
      }
      for (int q = rowp[b]; q < rowp[b] + g.elen[b]; q++) {
        const int e = cols[q];
        if (state[e] != 0) continue;
        long long delta = 0;
        if (elem_has(e, b)) delta += (long long)nb - sb;
        // the entry drop_variable(b) removes from e's row
        int j = rowp[e];
        const int last = rowp[e] + g.alen[e] - 1;
        if (last >= j) {
          while (j < last && cols[j] != b) j++;
          const int x = cols[j];
          delta -= (x == b) ? nb : (x == a ? slen[a] + sb : slen[x]);
        }
        esum[e] += delta;
        if (delta != 0)
          for (uint64_t m = held[e]; m; m &= m - 1) {
            const int t = tracked_list[__builtin_ctzll(m)];
            if (tracked[t]) esumT[t] += delta;
          }
      }
      // the entry drop_variable(b) removes from each neighbour's variable
      // part: b where it is found before the last entry, else the last entry
      for (int q = rowp[b] + g.elen[b]; q < rowp[b] + g.alen[b]; q++) {
        const int w = cols[q];
        if (w < 0 || w >= n || !tracked[w]) continue;
        int j = rowp[w] + g.elen[w];
        const int last = rowp[w] + g.alen[w] - 1;
        while (j < last && cols[j] != b) j++;
        const int x = cols[j];
        vsum[w] -= (x == b) ? nb : (x == a ? slen[a] + sb : slen[x]);
        rhash[w] -= mix64((uint64_t)x);
      }
      tracked[b] = 0;
      slen[a] += slen[b];
      deg.set(a, deg.degree[a] - slen[b]);
      slen[b] = -(a + 1);
      state[b] = -1;
      g.drop_variable(b);
      deg.unlink(b);
    };
    if (len <= kMergeScanMax) {
      for (int j = 0; j < len; j++) {
        const int a = Lp[j];
        if (a == piv || slen[a] < 0) continue;
        for (int k = j + 1; k < len; k++) {
          const int b = Lp[k];
          if (b == piv || slen[b] < 0) continue;
          if (g.same_adjacency(a, b)) merge(a, b);
        }
      }
    } else {
      // Same tests, same order, without the pairs that cannot match. The
      // test holds only when the lengths agree and either the rows are
      // equal, or each row holds the other variable and the rows agree
      // without them. So with R(v) the sum of a hash over v's row, a match
      // needs R(a) = R(b) or R(a) + h(a) = R(b) + h(b). Positions are kept
      // in two ordered sets by those keys; the next candidate after k is a
      // lookup. A merge changes the rows of the dropped variable's
      // neighbours, whose keys are then recomputed.
      merge_keys.assign(2 * len, 0);
      for (int p = 0; p < len; p++) lp_pos[Lp[p]] = p;
      auto compute_keys = [&](int p) {
        const int v = Lp[p];
        uint64_t r = 0;
        if (tracked[v])
          r = rhash[v];
        else
          for (int q = rowp[v]; q < rowp[v] + g.alen[v]; q++) r += mix64((uint64_t)cols[q]);
        const uint64_t shape = ((uint64_t)(uint32_t)g.alen[v] << 32) | (uint32_t)g.elen[v];
        merge_keys[2 * p] = mix64(r ^ mix64(shape));
        merge_keys[2 * p + 1] = mix64((r + mix64((uint64_t)v)) ^ mix64(shape));
      };
      auto active = [&](int p) { return Lp[p] != piv && slen[Lp[p]] >= 0; };
      // Per key kind: a hash table of chains of positions in increasing
      // order (filled from the back), plus the positions re-keyed since it
      // was filled. An entry whose key is no longer its position's current
      // key is stale and skipped.
      int tsize = 1;
      while (tsize < 2 * len) tsize <<= 1;
      auto rebuild = [&]() {
        for (int t = 0; t < 2; t++) {
          head[t].assign(tsize, -1);
          chain[t].assign(len, -1);
          extra[t].clear();
          for (int p = len - 1; p >= 0; p--) {
            if (!active(p)) continue;
            const int slot = (int)(merge_keys[2 * p + t] & (uint64_t)(tsize - 1));
            chain[t][p] = head[t][slot];
            head[t][slot] = p;
          }
        }
      };
      for (int p = 0; p < len; p++)
        if (active(p)) compute_keys(p);
      rebuild();
      auto next_candidate = [&](int j, int k) {
        int c = INT_MAX;
        for (int t = 0; t < 2; t++) {
          const uint64_t key = merge_keys[2 * j + t];
          for (int p = head[t][(int)(key & (uint64_t)(tsize - 1))]; p >= 0 && p < c;
               p = chain[t][p]) {
            if (p > k && merge_keys[2 * p + t] == key && active(p)) {
              c = p;
              break;
            }
          }
          for (const int p : extra[t])
            if (p > k && p < c && merge_keys[2 * p + t] == key && active(p)) c = p;
        }
        return c;
      };
      for (int j = 0; j < len; j++) {
        const int a = Lp[j];
        if (a == piv || slen[a] < 0) continue;
        int k = j;
        for (;;) {
          const int c = next_candidate(j, k);
          if (c == INT_MAX) break;
          k = c;
          const int b = Lp[k];
          if (!g.same_adjacency(a, b)) continue;
          // the neighbours of b in Lp whose rows the drop shortens
          touched.clear();
          for (int q = rowp[b] + g.elen[b]; q < rowp[b] + g.alen[b]; q++) {
            const int w = cols[q];
            if (w >= 0 && w < n && lp_pos[w] >= 0 && w != piv && slen[w] >= 0 && w != b)
              touched.push_back(lp_pos[w]);
          }
          merge(a, b);
          for (const int p : touched) {
            compute_keys(p);
            extra[0].push_back(p);
            extra[1].push_back(p);
          }
          if (extra[0].size() > kMergeExtraMax) rebuild();
        }
      }
      for (int p = 0; p < len; p++) lp_pos[Lp[p]] = -1;
    }
    i += slen[piv];
  }

  // expand supervariables: principal variable first, then its members in
  // increasing index
  int end = n;
  for (int j = nsv - 1; j >= 0; j--) {
    const int sv = perm[j];
    end -= slen[sv];
    perm[end] = sv;
    state[sv] = end + 1;
  }
  for (int k = 0; k < n; k++) {
    if (slen[k] < 0) {
      int j = k;
      while (slen[j] < 0) j = -(slen[j] + 1);
      perm[state[j]] = k;
      state[j]++;
    }
  }
  return 0;
}

namespace {

// parts of at most this many vertices are ordered by AMD on their subgraph
constexpr int kNdLeaf = 256;

// AMD on the subgraph induced by `verts` (adjacency adj/adj_ptr, global
// ids); appends the vertices in elimination order to `out`.
void amd_subgraph(const std::vector<int>& verts, const std::vector<int>& adj_ptr,
                  const std::vector<int>& adj, std::vector<int>& local,
                  std::vector<int>& out) {
  const int m = (int)verts.size();
  for (int i = 0; i < m; i++) local[verts[i]] = i;
  std::vector<int> rp(m + 1, 0), cc;
  for (int i = 0; i < m; i++) {
    const int v = verts[i];
    const size_t start = cc.size();
    cc.push_back(i);
    for (int q = adj_ptr[v]; q < adj_ptr[v + 1]; q++) {
      const int w = local[adj[q]];
      if (w >= 0) cc.push_back(w);
    }
    std::sort(cc.begin() + start, cc.end());
    cc.erase(std::unique(cc.begin() + start, cc.end()), cc.end());
    rp[i + 1] = (int)cc.size();
  }
  std::vector<int> p(m);
  if (amd_order(m, rp.data(), cc.data(), p.data()) != 0) std::iota(p.begin(), p.end(), 0);
  for (int i = 0; i < m; i++) out.push_back(verts[p[i]]);
  for (int i = 0; i < m; i++) local[verts[i]] = -1;
}

}  // namespace

// Nested dissection without METIS (our own ordering, not the reference's:
// without METIS the reference's nested dissection is the identity). Rows
// far denser than the rest (e.g. a constraint on every design variable) are
// set aside and ordered last. The rest is split recursively: a breadth-first
// level structure from a pseudo-peripheral vertex, the level that halves
// the part as the separator, thinned to the vertices with a neighbour in
// the next level. Each separator follows its two parts; parts of at most
// kNdLeaf vertices are ordered by AMD on their subgraph.
void nd_order(int n, const int* rowp, const int* cols, int* perm) {
  // adjacency without the diagonal
  std::vector<int> adj_ptr(n + 1, 0), adj;
  adj.reserve(rowp[n]);
  for (int i = 0; i < n; i++) {
    for (int q = rowp[i]; q < rowp[i + 1]; q++)
      if (cols[q] != i && cols[q] >= 0 && cols[q] < n) adj.push_back(cols[q]);
    adj_ptr[i + 1] = (int)adj.size();
  }
  long long total = adj_ptr[n];
  const double avg = n > 0 ? (double)total / n : 0.0;
  const int dense_min = std::max(64, (int)std::max(10.0 * avg, 10.0 * std::sqrt((double)n)));
  std::vector<int> part(n, 0), level(n, -1), local(n, -1), dense;
  for (int v = 0; v < n; v++) {
    if (adj_ptr[v + 1] - adj_ptr[v] > dense_min) {
      part[v] = -1;  // set aside
      dense.push_back(v);
    }
  }
  std::vector<int> out;
  out.reserve(n);
  // explicit stack of tasks: a part to split (verts, id) or a separator to emit
  struct Task {
    std::vector<int> verts;
    int id;
    bool emit;
  };
  std::vector<Task> stack;
  {
    Task t{{}, 0, false};
    for (int v = 0; v < n; v++)
      if (part[v] == 0) t.verts.push_back(v);
    stack.push_back(std::move(t));
  }
  int next_id = 1;
  std::vector<int> queue;
  auto bfs = [&](int root, int id, std::vector<int>& order) {
    order.clear();
    order.push_back(root);
    level[root] = 0;
    for (size_t h = 0; h < order.size(); h++) {
      const int v = order[h];
      for (int q = adj_ptr[v]; q < adj_ptr[v + 1]; q++) {
        const int w = adj[q];
        if (part[w] == id && level[w] < 0) {
          level[w] = level[v] + 1;
          order.push_back(w);
        }
      }
    }
  };
  auto clear_levels = [&](const std::vector<int>& vs) {
    for (const int v : vs) level[v] = -1;
  };
  while (!stack.empty()) {
    Task t = std::move(stack.back());
    stack.pop_back();
    if (t.emit) {
      for (const int v : t.verts) out.push_back(v);
      continue;
    }
    const int m = (int)t.verts.size();
    if (m == 0) continue;
    if (m <= kNdLeaf) {
      amd_subgraph(t.verts, adj_ptr, adj, local, out);
      for (const int v : t.verts) part[v] = -2;  // done
      continue;
    }
    // the component of t.verts[0]; other components become their own part
    bfs(t.verts[0], t.id, queue);
    if ((int)queue.size() < m) {
      Task rest{{}, next_id++, false};
      for (const int v : t.verts)
        if (level[v] < 0) {
          part[v] = rest.id;
          rest.verts.push_back(v);
        }
      Task comp{queue, next_id++, false};
      clear_levels(queue);
      for (const int v : comp.verts) part[v] = comp.id;
      stack.push_back(std::move(rest));
      stack.push_back(std::move(comp));
      continue;
    }
    // pseudo-peripheral root: restart from a far vertex of least degree
    int height = level[queue.back()];
    for (int it = 0; it < 4; it++) {
      int best = queue.back();
      for (size_t h = queue.size(); h-- > 0;) {
        const int v = queue[h];
        if (level[v] < height) break;
        if (adj_ptr[v + 1] - adj_ptr[v] < adj_ptr[best + 1] - adj_ptr[best]) best = v;
      }
      clear_levels(queue);
      bfs(best, t.id, queue);
      const int h2 = level[queue.back()];
      if (h2 <= height) break;
      height = h2;
    }
    // among the levels that leave 35-65% of the part on their lower side,
    // the one with the fewest vertices touching the next level
    int mid = 0;
    {
      std::vector<int> below(height + 2, 0), thin(height + 2, 0);
      for (const int v : queue) {
        const int l = level[v];
        below[l + 1]++;
        bool touches_next = false;
        for (int q = adj_ptr[v]; q < adj_ptr[v + 1] && !touches_next; q++) {
          const int w = adj[q];
          touches_next = (part[w] == t.id && level[w] == l + 1);
        }
        thin[l] += touches_next;
      }
      for (int l = 1; l <= height + 1; l++) below[l] += below[l - 1];
      int best = -1;
      for (int l = 1; l < height; l++) {
        const long long lo = below[l];  // vertices in levels < l
        if (20 * lo < 7 * (long long)m || 20 * lo > 13 * (long long)m) continue;
        if (best < 0 || thin[l] < thin[best]) best = l;
      }
      if (best < 0) {
        int cum = 0;
        for (size_t h = 0; h < queue.size(); h++) {
          cum++;
          if (2 * cum >= m) {
            best = level[queue[h]];
            break;
          }
        }
      }
      mid = best;
    }
    if (mid == 0 || mid >= height) {  // no useful split: order the part by AMD
      clear_levels(queue);
      amd_subgraph(t.verts, adj_ptr, adj, local, out);
      for (const int v : t.verts) part[v] = -2;
      continue;
    }
    Task a{{}, next_id++, false}, b{{}, next_id++, false}, sep{{}, -1, true};
    for (const int v : queue) {
      const int l = level[v];
      if (l < mid) {
        a.verts.push_back(v);
      } else if (l > mid) {
        b.verts.push_back(v);
      } else {
        bool touches_next = false;
        for (int q = adj_ptr[v]; q < adj_ptr[v + 1] && !touches_next; q++) {
          const int w = adj[q];
          touches_next = (part[w] == t.id && level[w] == mid + 1);
        }
        (touches_next ? sep.verts : a.verts).push_back(v);
      }
    }
    clear_levels(queue);
    for (const int v : a.verts) part[v] = a.id;
    for (const int v : b.verts) part[v] = b.id;
    for (const int v : sep.verts) part[v] = -2;
    stack.push_back(std::move(sep));  // emitted after both parts
    stack.push_back(std::move(b));
    stack.push_back(std::move(a));
  }
  for (const int v : dense) out.push_back(v);
  for (int i = 0; i < n; i++) perm[i] = out[i];
}

// copy_for_reorder (ordering_utils.h:313-360) + reorder (38-56): AMD sees the
// pattern with the diagonal added, rows sorted and de-duplicated in place;
// nested dissection without METIS is the identity (189-194).
void compute_ordering(Ordering order, int n, const int* rowp, const int* cols,
                      std::vector<int>& perm, std::vector<int>& iperm) {
  perm.assign(n, 0);
  iperm.assign(n, 0);
  if (order == Ordering::Amd) {
    const int nnz = rowp[n];
    std::vector<int> rp(n + 1), cc(static_cast<size_t>(nnz) + n);
    int ptr = 0;
    rp[0] = 0;
    for (int i = 0; i < n; i++) {
      cc[ptr++] = i;
      for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) cc[ptr++] = cols[jp];
      rp[i + 1] = ptr;
    }
    // sort_and_uniquify_csr (ordering_utils.h:812-838): rows compacted left
    int start = rp[0];
    for (int i = 0; i < n; i++) {
      const int size = rp[i + 1] - start;
      int* a = &cc[start];
      std::sort(a, a + size);
      int m = 0;
      if (size > 0) {
        cc[rp[i]] = a[0];
        m = 1;
        for (int r = 1; r < size; r++) {
          if (a[r] != cc[rp[i] + m - 1]) cc[rp[i] + m++] = a[r];
        }
      }
      start = rp[i + 1];
      rp[i + 1] = rp[i] + m;
    }
    const int flag = amd_order(n, rp.data(), cc.data(), perm.data());
    if (flag != 0) {
      std::fprintf(stderr, "b200ldl: AMD input format error at row %d\n", flag - 1);
      std::iota(perm.begin(), perm.end(), 0);
    }
  } else if (order == Ordering::GraphNd) {
    nd_order(n, rowp, cols, perm.data());
  } else if (order == Ordering::MultiColor) {
    throw std::invalid_argument("multicolor ordering is not supported");
  } else {
    std::iota(perm.begin(), perm.end(), 0);
  }
  for (int i = 0; i < n; i++) iperm[perm[i]] = i;
}

// compute_etree (sparse_ldl.h:2393-2458), post_order_etree +
// depth_first_search (2473-2536), count_column_nonzeros with
// init_column_count_data and find_root (2545-2719).
void etree_postorder_colcount(int n, const int* rowp, const int* cols,
                              const int* perm, const int* iperm,
                              std::vector<int>& parent, std::vector<int>& post,
                              std::vector<int>& colcount) {
  parent.assign(n, -1);
  post.assign(n, 0);
  colcount.assign(n, 0);
  std::vector<int> anc(n, -1);
  for (int k = 0; k < n; k++) {
    const int ka = perm ? perm[k] : k;
    for (int ip = rowp[ka]; ip < rowp[ka + 1]; ip++) {
      int i = iperm ? iperm[cols[ip]] : cols[ip];
      while (i < k) {
        const int up = anc[i];
        anc[i] = k;
        if (up == -1) {
          parent[i] = k;
          break;
        }
        i = up;
      }
    }
  }

  // postorder: children visited in increasing index, roots in increasing index
  std::vector<int> head(n, -1), next(n, -1), stack(n);
  for (int j = n - 1; j >= 0; j--) {
    if (parent[j] != -1) {
      next[j] = head[parent[j]];
      head[parent[j]] = j;
    }
  }
  for (int j = 0, k = 0; j < n; j++) {
    if (parent[j] != -1) continue;
    int top = 0;
    stack[0] = j;
    while (top >= 0) {
      const int p = stack[top];
      const int c = head[p];
      if (c == -1) {
        post[k++] = p;
        top--;
      } else {
        head[p] = next[c];
        stack[++top] = c;
      }
    }
  }

  // column counts (skeleton-graph leaves with path-compressed ancestors)
  std::vector<int> first(n, -1), prevleaf(n, -1), maxfirst(n, -1), ancestor(n);
  for (int k = 0; k < n; k++) {
    int j = post[k];
    if (first[j] == -1) colcount[j] = 1;
    while (j != -1 && first[j] == -1) {
      first[j] = k;
      j = parent[j];
    }
  }
  std::iota(ancestor.begin(), ancestor.end(), 0);
  auto root_of = [&](int p) {
    int r = p;
    while (ancestor[r] != r) r = ancestor[r];
    while (ancestor[p] != p) {
      const int nx = ancestor[p];
      ancestor[p] = r;
      p = nx;
    }
    return r;
  };
  for (int k = 0; k < n; k++) {
    const int j = post[k];
    const int ja = perm ? perm[j] : j;
    if (parent[j] != -1) colcount[parent[j]]--;
    for (int ip = rowp[ja]; ip < rowp[ja + 1]; ip++) {
      const int i = iperm ? iperm[cols[ip]] : cols[ip];
      if (i <= j) continue;
      if (first[j] <= maxfirst[i]) continue;
      colcount[j]++;
      maxfirst[i] = first[j];
      const int jprev = prevleaf[i];
      prevleaf[i] = j;
      if (jprev != -1) colcount[root_of(jprev)]--;
    }
    if (parent[j] != -1) ancestor[j] = parent[j];
  }
  for (int k = 0; k < n; k++) {
    const int j = post[k];
    if (parent[j] != -1) colcount[parent[j]] += colcount[j];
  }
}

namespace {

// count_node_children (sparse_ldl.h:2978-3014): CSR of children in
// increasing id, roots appended in slot num_nodes.
void child_lists(int nn, const std::vector<int>& parent, std::vector<int>& ptr,
                 std::vector<int>& kids) {
  ptr.assign(nn + 2, 0);
  kids.assign(std::max(nn, 1), 0);
  for (int i = 0; i < nn; i++) {
    const int p = parent[i];
    ptr[(p != -1 ? p : nn) + 1]++;
  }
  for (int i = 0; i < nn + 1; i++) ptr[i + 1] += ptr[i];
  for (int i = 0; i < nn; i++) {
    const int p = parent[i];
    const int slot = p != -1 ? p : nn;
    kids[ptr[slot]++] = i;
  }
  for (int i = nn; i >= 0; i--) ptr[i + 1] = ptr[i];
  ptr[0] = 0;
  kids.resize(nn);
}

}  // namespace

Symbolic analyze(Ordering order, int n, const int* rowp, const int* cols) {
  Symbolic s;
  s.n = n;
  compute_ordering(order, n, rowp, cols, s.perm, s.iperm);
  s.permuted = (order != Ordering::Natural);
  const int* P = s.permuted ? s.perm.data() : nullptr;
  const int* IP = s.permuted ? s.iperm.data() : nullptr;

  std::vector<int> parent, post, colcount;
  etree_postorder_colcount(n, rowp, cols, P, IP, parent, post, colcount);

  // fundamental supernodes along the postorder (sparse_ldl.h:2734-2765)
  std::vector<int> vtosn(n), sntov(n);
  int nsn = 0;
  for (int i = 0; i < n; nsn++) {
    int var = post[i];
    vtosn[var] = nsn;
    sntov[i] = var;
    i++;
    int nv = i < n ? post[i] : n;
    while (i < n && parent[var] == nv && colcount[nv] == colcount[var] - 1) {
      var = nv;
      vtosn[var] = nsn;
      sntov[i] = var;
      i++;
      if (i < n) nv = post[i];
    }
  }
  std::vector<int> sn_ptr(nsn + 1, 0);
  for (int i = 0; i < n; i++) sn_ptr[vtosn[i] + 1]++;
  for (int i = 0; i < nsn; i++) sn_ptr[i + 1] += sn_ptr[i];
  std::vector<int> sn_parent(nsn);
  for (int is = 0; is < nsn; is++) {
    const int p = parent[sntov[sn_ptr[is + 1] - 1]];
    sn_parent[is] = p >= 0 ? vtosn[p] : -1;
  }
  std::vector<int> sn_kptr, sn_kids;
  child_lists(nsn, sn_parent, sn_kptr, sn_kids);

  // relaxed amalgamation (sparse_ldl.h:2786-2967): children visited by
  // increasing width of the group of the snode whose id equals the child's
  // slot in the child array, merged while width <= 64 and the zeros added to
  // the group stay <= 256.
  const int max_width = 64;
  const int max_zeros = 256;
  std::vector<int> grp(nsn), gcount(nsn), width(nsn), zeros(nsn, 0);
  for (int is = 0; is < nsn; is++) {
    width[is] = sn_ptr[is + 1] - sn_ptr[is];
    gcount[is] = colcount[sntov[sn_ptr[is]]];
    grp[is] = is;
  }
  auto find = [&](int x) {
    while (grp[x] != x) {
      grp[x] = grp[grp[x]];
      x = grp[x];
    }
    return x;
  };
  std::vector<int> order_buf;
  for (int is = 0; is < nsn; is++) {
    const int b = sn_kptr[is];
    const int e = sn_kptr[is + 1];
    order_buf.resize(e - b);
    for (int ip = b; ip < e; ip++) order_buf[ip - b] = ip;
    std::sort(order_buf.begin(), order_buf.end(),
              [&](int x, int y) { return width[find(x)] < width[find(y)]; });
    for (int ip : order_buf) {
      const int child = sn_kids[ip];
      const int rp = find(is);
      const int rc = find(child);
      const int w = width[rc] + width[rp];
      if (rc != rp && w <= max_width) {
        const int extra = std::max(0, gcount[rp] - (gcount[rc] - width[rp]));
        const int added = extra * width[rc];
        if (zeros[rp] + zeros[rc] + added <= max_zeros) {
          gcount[rp] = w + gcount[rp] - width[rp];
          width[rp] = w;
          grp[rc] = rp;
          zeros[rp] += added + zeros[rc];
        }
      }
    }
  }
  std::vector<int> to_node(nsn, -1), new_id(nsn, -1);
  int nn = 0;
  for (int is = 0; is < nsn; is++)
    if (find(is) == is) new_id[is] = nn++;
  for (int is = 0; is < nsn; is++) to_node[is] = new_id[find(is)];

  s.num_nodes = nn;
  s.node_ptr.assign(nn + 1, 0);
  s.node_to_var.assign(n, 0);
  std::vector<int> var_to_node(n), node_count(nn);
  for (int is = 0; is < nsn; is++) s.node_ptr[to_node[is] + 1] += sn_ptr[is + 1] - sn_ptr[is];
  for (int k = 0; k < nn; k++) s.node_ptr[k + 1] += s.node_ptr[k];
  {
    std::vector<int> fill(s.node_ptr.begin(), s.node_ptr.end() - 1);
    for (int is = 0; is < nsn; is++) {
      const int k = to_node[is];
      for (int ip = sn_ptr[is]; ip < sn_ptr[is + 1]; ip++) {
        const int var = sntov[ip];
        s.node_to_var[fill[k]++] = var;
        var_to_node[var] = k;
      }
    }
  }
  for (int is = 0; is < nsn; is++) node_count[to_node[is]] = gcount[find(is)];
  s.parent.assign(nn, -1);
  for (int is = 0; is < nsn; is++) {
    if (find(is) != is) continue;
    const int k = to_node[is];
    const int ps = sn_parent[is];
    if (ps >= 0) {
      const int kp = to_node[find(ps)];
      if (kp != k) s.parent[k] = kp;
    }
  }
  child_lists(nn, s.parent, s.children_ptr, s.children);

  // contribution rows (sparse_ldl.h:2323-2348, build_nonzero_pattern
  // 3036-3122): walk each row's subtree upward, one visit per node per row
  s.contrib_ptr.assign(nn + 1, 0);
  for (int k = 0; k < nn; k++) s.contrib_ptr[k + 1] = node_count[k] - (s.node_ptr[k + 1] - s.node_ptr[k]);
  for (int k = 0; k < nn; k++) s.contrib_ptr[k + 1] += s.contrib_ptr[k];
  s.contrib_rows.assign(s.contrib_ptr[nn], 0);
  {
    std::vector<int> filled(nn, 0), flag(nn, -1), up(nn);
    for (int k = 0; k < nn; k++) {
      const int last = s.node_to_var[s.node_ptr[k + 1] - 1];
      const int p = parent[last];
      up[k] = p >= 0 ? var_to_node[p] : -1;
    }
    for (int k = 0; k < n; k++) {
      const int ks = var_to_node[k];
      const int ka = P ? P[k] : k;
      for (int ip = rowp[ka]; ip < rowp[ka + 1]; ip++) {
        const int i = IP ? IP[cols[ip]] : cols[ip];
        if (i >= k) continue;
        for (int is = var_to_node[i]; is >= 0 && is != ks; is = up[is]) {
          if (flag[is] == k) break;
          flag[is] = k;
          const int pos = s.contrib_ptr[is] + filled[is];
          if (pos >= s.contrib_ptr[is + 1])
            throw std::runtime_error("symbolic: contribution row overflow");
          s.contrib_rows[pos] = ka;
          filled[is]++;
        }
      }
    }
  }
  if (P) {
    for (int i = 0; i < n; i++) s.node_to_var[i] = P[s.node_to_var[i]];
  }
  return s;
}

}  // namespace b200ldl
