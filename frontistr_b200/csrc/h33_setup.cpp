// h33_setup.cpp -- host-side symbolic setup of the B200 3x3 solver.
//
// The orderings must reproduce the reference's colour schedule exactly (the same
// permutation and COLORindex), so their steps follow the reference algorithms:
//   RCM   hecmw1/src/solver/matrix/hecmw_matrix_ordering_CM.f90:18-245
//   MC    hecmw1/src/solver/matrix/hecmw_matrix_ordering_MC.f90:15-72
//   reorder hecmw1/src/solver/matrix/hecmw_matrix_reorder.f90:20-158
//   ILU(0) hecmw1/src/solver/precond/bilu/hecmw_precond_BILU_33.f90:185-362,1493-1596
// Everything here is 0-based; node ids in the input profile are 1-based.
#include "h33_setup.h"

#include <omp.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>
#include <stdexcept>

namespace h33 {

std::string check_profile(int N, int NP, int NPL, int NPU, const int *indexL, const int *itemL,
                          const int *indexU, const int *itemU) {
  if (N <= 0) return "N must be positive";
  if (NP < N) return "NP < N";
  if (!indexL || !indexU || (NPL > 0 && !itemL) || (NPU > 0 && !itemU)) return "null profile array";
  if (indexL[0] != 0 || indexU[0] != 0 || indexL[NP] != NPL || indexU[NP] != NPU)
    return "indexL/indexU inconsistent with NPL/NPU";
  for (int i = 0; i < NP; i++) {
    if (indexL[i + 1] < indexL[i] || indexU[i + 1] < indexU[i]) return "index arrays must be non-decreasing";
    int prev = 0;
    for (int j = indexL[i]; j < indexL[i + 1]; j++) {
      const int c = itemL[j];
      if (c <= prev || c >= i + 1) return "itemL must be ascending ids < row";
      prev = c;
    }
    prev = i + 1;
    for (int j = indexU[i]; j < indexU[i + 1]; j++) {
      const int c = itemU[j];
      if (c <= prev || c > NP) return "itemU must be ascending ids in (row, NP]";
      prev = c;
    }
  }
  return "";
}

namespace {

// Degree = lower neighbours + upper neighbours inside the domain (count_degrees).
std::vector<int> degrees(const Profile &p) {
  std::vector<int> deg(p.N);
  for (int i = 0; i < p.N; i++) {
    int d = p.indexL[i + 1] - p.indexL[i];
    for (int j = p.indexU[i]; j < p.indexU[i + 1]; j++)
      if (p.itemU[j] <= p.N) d++;
    deg[i] = d;
  }
  return deg;
}

// Middle-pivot Hoare partition sort of a level by degree (sort_nodes_by_degree).
// Unstable; the order of equal degrees is part of the reference's result.
void sort_level(int *item, int lo, int hi, const std::vector<int> &deg) {
  while (lo < hi) {
    const int pivot = deg[item[(lo + hi) / 2]];
    int l = lo, r = hi;
    for (;;) {
      while (deg[item[l]] < pivot) l++;
      while (pivot < deg[item[r]]) r--;
      if (l >= r) break;
      std::swap(item[l], item[r]);
      l++;
      r--;
    }
    // recurse into the left part, iterate on the right part (same order of work)
    sort_level(item, lo, l - 1, deg);
    lo = r + 1;
  }
}

// One Cuthill-McKee sweep from `seed`; returns the number of levels and fills order.
int cm_from_seed(const Profile &p, const std::vector<int> &deg, int seed, std::vector<int> &order) {
  const int N = p.N;
  std::vector<int> level_of(N, 0);
  order.assign(N, 0);
  int prev_begin = 0, prev_end = 1, count = 1;
  order[0] = seed;
  level_of[seed] = 1;
  if (count == N) return 1;
  for (int level = 2; level <= N; level++) {
    const int begin = count;
    for (int j = prev_begin; j < prev_end; j++) {
      const int node = order[j];
      for (int k = p.indexL[node]; k < p.indexL[node + 1]; k++) {
        const int nb = p.itemL[k] - 1;
        if (level_of[nb] == 0) {
          level_of[nb] = level;
          order[count++] = nb;
        }
      }
      for (int k = p.indexU[node]; k < p.indexU[node + 1]; k++) {
        const int nb1 = p.itemU[k];
        if (nb1 > N) continue;
        const int nb = nb1 - 1;
        if (level_of[nb] == 0) {
          level_of[nb] = level;
          order[count++] = nb;
        }
      }
    }
    if (count == begin) {  // disconnected: start the next component at the lowest id
      for (int nb = 0; nb < N; nb++)
        if (level_of[nb] == 0) {
          level_of[nb] = level;
          order[count++] = nb;
          break;
        }
    }
    sort_level(order.data(), begin, count - 1, deg);
    if (count == N) return level;
    prev_begin = begin;
    prev_end = count;
  }
  return N;
}

}  // namespace

void ordering_rcm(const Profile &p, std::vector<int> &perm, std::vector<int> &iperm) {
  const int N = p.N;
  const std::vector<int> deg = degrees(p);
  // up to five minimum-degree seeds in index order (find_minimum_degrees)
  std::vector<int> seeds;
  int degmin = N, nmin = 0;
  for (int i = 0; i < N; i++) {
    if (deg[i] == 0) continue;
    if (deg[i] < degmin) {
      degmin = deg[i];
      nmin = 1;
      seeds.assign(1, i);
    } else if (deg[i] == degmin) {
      nmin++;
      if (nmin <= 5) seeds.push_back(i);
    }
  }
  if (seeds.empty()) seeds.push_back(0);  // no edges at all: start from node 0
  std::vector<std::vector<int>> orders(seeds.size());
  std::vector<int> nlevel(seeds.size());
#pragma omp parallel for schedule(static, 1)
  for (int s = 0; s < int(seeds.size()); s++) nlevel[s] = cm_from_seed(p, deg, seeds[s], orders[s]);
  size_t best = 0;
  for (size_t s = 1; s < seeds.size(); s++)
    if (nlevel[s] > nlevel[best]) best = s;
  // reverse the chosen Cuthill-McKee order
  perm.assign(N, 0);
  iperm.assign(N, 0);
  for (int pos = 0; pos < N; pos++) {
    const int node = orders[best][pos];
    const int rpos = N - 1 - pos;
    iperm[node] = rpos;
    perm[rpos] = node;
  }
}

namespace {

// First-fit colouring in `order` (null: the input order): each node takes the smallest
// colour that none of its already coloured neighbours has.  Returns the colour count.
int first_fit(const Profile &p, const std::vector<int> *order, std::vector<int> &colour) {
  const int N = p.N;
  colour.assign(static_cast<size_t>(N), -1);
  std::vector<int> seen;
  int ncolor = 0;
  for (int t = 0; t < N; t++) {
    const int i = order ? (*order)[static_cast<size_t>(t)] : t;
    seen.resize(static_cast<size_t>(ncolor) + 1, -1);
    for (int k = p.indexL[i]; k < p.indexL[i + 1]; k++) {
      const int c = colour[static_cast<size_t>(p.itemL[k] - 1)];
      if (c >= 0) seen[static_cast<size_t>(c)] = t;
    }
    for (int k = p.indexU[i]; k < p.indexU[i + 1]; k++) {
      const int c = colour[static_cast<size_t>(p.itemU[k] - 1)];
      if (c >= 0) seen[static_cast<size_t>(c)] = t;
    }
    int c = 0;
    while (seen[static_cast<size_t>(c)] == t) c++;
    colour[static_cast<size_t>(i)] = c;
    ncolor = std::max(ncolor, c + 1);
  }
  return ncolor;
}

// Smallest-last order (Matula and Beck, 1983): repeatedly remove a node of least
// remaining degree; the reverse of the removal order.  Bucket queue with lazy entries.
std::vector<int> smallest_last(const Profile &p) {
  const int N = p.N;
  std::vector<int> deg(static_cast<size_t>(N));
  std::vector<char> removed(static_cast<size_t>(N), 0);
  int maxd = 0;
  for (int i = 0; i < N; i++) {
    deg[static_cast<size_t>(i)] = (p.indexL[i + 1] - p.indexL[i]) + (p.indexU[i + 1] - p.indexU[i]);
    maxd = std::max(maxd, deg[static_cast<size_t>(i)]);
  }
  std::vector<std::vector<int>> bucket(static_cast<size_t>(maxd) + 1);
  for (int i = 0; i < N; i++) bucket[static_cast<size_t>(deg[static_cast<size_t>(i)])].push_back(i);
  std::vector<int> order;
  order.reserve(static_cast<size_t>(N));
  int d = 0;
  for (int cnt = 0; cnt < N; cnt++) {
    d = std::max(0, d - 1);  // a removal lowers a neighbour's degree by one at most
    int v;
    for (;;) {
      while (bucket[static_cast<size_t>(d)].empty()) d++;
      v = bucket[static_cast<size_t>(d)].back();
      bucket[static_cast<size_t>(d)].pop_back();
      if (!removed[static_cast<size_t>(v)] && deg[static_cast<size_t>(v)] == d) break;  // else stale
    }
    removed[static_cast<size_t>(v)] = 1;
    order.push_back(v);
    auto drop = [&](int u) {
      if (removed[static_cast<size_t>(u)]) return;
      const int du = --deg[static_cast<size_t>(u)];
      bucket[static_cast<size_t>(du)].push_back(u);
    };
    for (int k = p.indexL[v]; k < p.indexL[v + 1]; k++) drop(p.itemL[k] - 1);
    for (int k = p.indexU[v]; k < p.indexU[v + 1]; k++) drop(p.itemU[k] - 1);
  }
  std::reverse(order.begin(), order.end());
  return order;
}

}  // namespace

int ordering_greedy(const Profile &p, std::vector<int> &colorindex, std::vector<int> &perm,
                    std::vector<int> &iperm) {
  const int N = p.N;
  std::vector<int> c_in, c_sl;
  int n_in = 0, n_sl = 0;
  // the two candidate colourings are independent: one thread each
#pragma omp parallel sections num_threads(2)
  {
#pragma omp section
    n_in = first_fit(p, nullptr, c_in);
#pragma omp section
    {
      const std::vector<int> sl = smallest_last(p);
      n_sl = first_fit(p, &sl, c_sl);
    }
  }
  const bool use_sl = n_sl < n_in;
  const std::vector<int> &colour = use_sl ? c_sl : c_in;
  const int ncolor = use_sl ? n_sl : n_in;
  colorindex.assign(static_cast<size_t>(ncolor) + 1, 0);
  for (int i = 0; i < N; i++) colorindex[static_cast<size_t>(colour[static_cast<size_t>(i)]) + 1]++;
  for (int c = 0; c < ncolor; c++) colorindex[static_cast<size_t>(c) + 1] += colorindex[static_cast<size_t>(c)];
  perm.assign(static_cast<size_t>(N), 0);
  iperm.assign(static_cast<size_t>(N), 0);
  std::vector<int> at(colorindex.begin(), colorindex.end() - 1);
  for (int i = 0; i < N; i++) {
    const int pos = at[static_cast<size_t>(colour[static_cast<size_t>(i)])]++;
    perm[static_cast<size_t>(pos)] = i;
    iperm[static_cast<size_t>(i)] = pos;
  }
  return ncolor;
}

int ordering_mc(const Profile &p, const std::vector<int> &perm_cur, int ncolor_in,
                std::vector<int> &colorindex, std::vector<int> &perm, std::vector<int> &iperm) {
  const int N = p.N;
  if (ncolor_in < 1) ncolor_in = 1;
  const int per_colour = N / ncolor_in;  // colour size cap (0 = no cap)
  // Everything below works on positions in perm_cur (the order the reference scans):
  // a node's neighbours are near it in that (banded) order, so the marks stay in cache.
  std::vector<int> pos_of(static_cast<size_t>(N));
#pragma omp parallel for schedule(static)
  for (int k = 0; k < N; k++) pos_of[static_cast<size_t>(perm_cur[static_cast<size_t>(k)])] = k;
  std::vector<int64_t> aptr(static_cast<size_t>(N) + 1, 0);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < N; k++) {
    const int node = perm_cur[static_cast<size_t>(k)];
    int c = p.indexL[node + 1] - p.indexL[node];
    for (int j = p.indexU[node]; j < p.indexU[node + 1]; j++) c += p.itemU[j] <= N;
    aptr[static_cast<size_t>(k) + 1] = c;
  }
  for (int k = 0; k < N; k++) aptr[static_cast<size_t>(k) + 1] += aptr[static_cast<size_t>(k)];
  // left uninitialised: the parallel fill below writes every entry (and first-touches
  // the pages on many threads instead of one zero-filling pass)
  std::unique_ptr<int[]> adj(new int[static_cast<size_t>(aptr[static_cast<size_t>(N)]) + 1]);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < N; k++) {
    const int node = perm_cur[static_cast<size_t>(k)];
    int64_t w = aptr[static_cast<size_t>(k)];
    for (int j = p.indexL[node]; j < p.indexL[node + 1]; j++) adj[static_cast<size_t>(w++)] = pos_of[static_cast<size_t>(p.itemL[j] - 1)];
    for (int j = p.indexU[node]; j < p.indexU[node + 1]; j++)
      if (p.itemU[j] <= N) adj[static_cast<size_t>(w++)] = pos_of[static_cast<size_t>(p.itemU[j] - 1)];
  }
  std::vector<int> mark(static_cast<size_t>(N), 0);  // >0 colour, -1 neighbour of this colour
  perm.assign(static_cast<size_t>(N), 0);
  colorindex.assign(1, 0);
  // the positions not yet coloured, ascending: every colour scans them from the start
  // as the reference scans perm_cur (coloured nodes, which it skips, are left out), so
  // the same nodes are taken in the same order
  std::vector<int> rest(static_cast<size_t>(N));
  for (int k = 0; k < N; k++) rest[static_cast<size_t>(k)] = k;
  int done = 0, ncolor = 0;
  for (int colour = 1; colour <= N; colour++) {
    int taken = 0;
    for (const int k : rest) {
      if (mark[static_cast<size_t>(k)] != 0) continue;
      mark[static_cast<size_t>(k)] = colour;
      perm[static_cast<size_t>(done++)] = perm_cur[static_cast<size_t>(k)];
      taken++;
      if (taken == per_colour || done == N) break;
      for (int64_t e = aptr[static_cast<size_t>(k)]; e < aptr[static_cast<size_t>(k) + 1]; e++) {
        int &m = mark[static_cast<size_t>(adj[static_cast<size_t>(e)])];
        if (m == 0) m = -1;
      }
    }
    colorindex.push_back(done);
    if (done == N) {
      ncolor = colour;
      break;
    }
    // only uncoloured positions carry -1 marks: clear them and drop the coloured ones
    size_t w = 0;
    for (const int k : rest) {
      if (mark[static_cast<size_t>(k)] > 0) continue;
      mark[static_cast<size_t>(k)] = 0;
      rest[w++] = k;
    }
    rest.resize(w);
  }
  iperm.assign(static_cast<size_t>(N), 0);
  for (int i = 0; i < N; i++) iperm[static_cast<size_t>(perm[static_cast<size_t>(i)])] = i;
  return ncolor;
}

void unified_rows(const Profile &p, BlockRows &out) {
  const int N = p.N, NPL = p.NPL();
  const int64_t nz = int64_t(N) + NPL + p.NPU();
  out.ptr.assign(size_t(N) + 1, 0);
  out.col.resize(size_t(nz));
  out.src.resize(size_t(nz));
  for (int i = 0; i < N; i++)
    out.ptr[i + 1] = out.ptr[i] + (p.indexL[i + 1] - p.indexL[i]) + 1 + (p.indexU[i + 1] - p.indexU[i]);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    int64_t w = out.ptr[i];
    for (int j = p.indexL[i]; j < p.indexL[i + 1]; j++) {
      out.col[w] = p.itemL[j] - 1;
      out.src[w++] = N + j;
    }
    out.col[w] = i;
    out.src[w++] = i;
    for (int j = p.indexU[i]; j < p.indexU[i + 1]; j++) {
      out.col[w] = p.itemU[j] - 1;
      out.src[w++] = N + NPL + j;
    }
  }
}

void reordered_rows(const Profile &p, const std::vector<int> &perm, const std::vector<int> &iperm,
                    BlockRows &lower, BlockRows &upper) {
  const int N = p.N, NPL = p.NPL();
  lower.ptr.assign(size_t(N) + 1, 0);
  upper.ptr.assign(size_t(N) + 1, 0);
  // rows are visited in their old (input) order, so the profile and the neighbours'
  // new indices are read from nearby memory; each finished row goes to its new place
  // counts per new row
#pragma omp parallel for schedule(static)
  for (int iold = 0; iold < N; iold++) {
    const int inew = iperm[iold];
    int nl = 0, nu = 0;
    for (int j = p.indexL[iold]; j < p.indexL[iold + 1]; j++)
      (iperm[p.itemL[j] - 1] < inew ? nl : nu)++;
    for (int j = p.indexU[iold]; j < p.indexU[iold + 1]; j++) {
      if (p.itemU[j] > N) continue;
      (iperm[p.itemU[j] - 1] < inew ? nl : nu)++;
    }
    lower.ptr[inew + 1] = nl;
    upper.ptr[inew + 1] = nu;
  }
  for (int inew = 0; inew < N; inew++) {
    lower.ptr[inew + 1] += lower.ptr[inew];
    upper.ptr[inew + 1] += upper.ptr[inew];
  }
  lower.col.resize(size_t(lower.ptr[N]));
  lower.src.resize(size_t(lower.ptr[N]));
  upper.col.resize(size_t(upper.ptr[N]));
  upper.src.resize(size_t(upper.ptr[N]));
  struct Entry {
    int jnew, src, jold;  // new column, raw block, old column (the node id kept in col)
  };
#pragma omp parallel
  {
    std::vector<Entry> lo, up;
#pragma omp for schedule(static)
    for (int iold = 0; iold < N; iold++) {
      const int inew = iperm[iold];
      lo.clear();
      up.clear();
      for (int j = p.indexL[iold]; j < p.indexL[iold + 1]; j++) {
        const int jold = p.itemL[j] - 1, jnew = iperm[jold];
        (jnew < inew ? lo : up).push_back(Entry{jnew, N + j, jold});
      }
      for (int j = p.indexU[iold]; j < p.indexU[iold + 1]; j++) {
        if (p.itemU[j] > N) continue;
        const int jold = p.itemU[j] - 1, jnew = iperm[jold];
        (jnew < inew ? lo : up).push_back(Entry{jnew, N + NPL + j, jold});
      }
      // new columns are distinct within a row: the order is total
      auto by_new = [](const Entry &a, const Entry &b) { return a.jnew < b.jnew; };
      std::sort(lo.begin(), lo.end(), by_new);
      std::sort(up.begin(), up.end(), by_new);
      int64_t w = lower.ptr[inew];
      for (const Entry &e : lo) {
        lower.col[w] = e.jold;
        lower.src[w++] = e.src;
      }
      w = upper.ptr[inew];
      for (const Entry &e : up) {
        upper.col[w] = e.jold;
        upper.src[w++] = e.src;
      }
    }
  }
}

void sell_shape(const int *count, const std::vector<int> &group_rows, SellLayout &out, int lanes, int max_runs) {
  if (lanes < 1 || lanes > 32 || (32 % lanes) != 0) throw std::runtime_error("lanes per row must divide 32");
  out = SellLayout();
  out.lanes = lanes;
  const int per_slice = 32 / lanes;
  const int ngroups = int(group_rows.size()) - 1;
  out.group_slice.assign(size_t(ngroups) + 1, 0);
  if (max_runs > 0) out.run_ptr.assign(size_t(ngroups) + 1, 0);
  std::vector<int> lens;
  for (int g = 0; g < ngroups; g++) {
    // natural slot count of each slice of the group
    lens.clear();
    for (int r0 = group_rows[g]; r0 < group_rows[g + 1]; r0 += per_slice) {
      const int nr = std::min(per_slice, group_rows[g + 1] - r0);
      int len = 0;
      for (int l = 0; l < nr; l++) len = std::max(len, (count[r0 + l] + lanes - 1) / lanes);
      lens.push_back(len);
    }
    if (max_runs > 0) {
      // runs of equal slot counts; while there are too many, merge the adjacent pair
      // whose merge adds the fewest padding slots
      std::vector<std::pair<int, int>> runs;  // (slices, slot count)
      for (int len : lens) {
        if (!runs.empty() && runs.back().second == len) runs.back().first++;
        else runs.emplace_back(1, len);
      }
      while (int(runs.size()) > max_runs) {
        size_t best = 0;
        int64_t best_cost = -1;
        for (size_t i = 0; i + 1 < runs.size(); i++) {
          const auto &a = runs[i], &b = runs[i + 1];
          const int64_t cost = a.second < b.second ? int64_t(a.first) * (b.second - a.second)
                                                   : int64_t(b.first) * (a.second - b.second);
          if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = i;
          }
        }
        runs[best].first += runs[best + 1].first;
        runs[best].second = std::max(runs[best].second, runs[best + 1].second);
        runs.erase(runs.begin() + int64_t(best) + 1);
      }
      int at = 0;
      for (const auto &rn : runs) {
        out.run_slice.push_back(at);
        out.run_slot.push_back(0);  // set below, when the run's first slice is laid out
        out.run_len.push_back(rn.second);
        for (int k = 0; k < rn.first; k++) lens[size_t(at + k)] = rn.second;
        at += rn.first;
      }
      out.run_ptr[size_t(g) + 1] = int(out.run_slice.size());
    }
    size_t k = 0;
    int run = max_runs > 0 ? out.run_ptr[size_t(g)] : 0;
    for (int r0 = group_rows[g]; r0 < group_rows[g + 1]; r0 += per_slice, k++) {
      if (max_runs > 0 && run < out.run_ptr[size_t(g) + 1] && out.run_slice[size_t(run)] == int(k))
        out.run_slot[size_t(run++)] = int(out.nslots);
      out.row0.push_back(r0);
      out.nrows.push_back(std::min(per_slice, group_rows[g + 1] - r0));
      out.slot0.push_back(int(out.nslots));
      out.len.push_back(lens[k]);
      out.nslots += lens[k];
      if (out.nslots > (int64_t(1) << 31) / 32 / 9)
        throw std::runtime_error("matrix too large for 32-bit slot offsets");
    }
    out.group_slice[g + 1] = int(out.row0.size());
  }
  out.nslices = int(out.row0.size());
  out.rowlen.assign(size_t(out.nslices) * 32, 0);
  for (int s = 0; s < out.nslices; s++)
    for (int r = 0; r < out.nrows[s]; r++) out.rowlen[size_t(s) * 32 + r] = count[out.row0[s] + r];
}

void build_sell(const BlockRows &rows, const std::vector<int> &group_rows, SellLayout &out, int lanes,
                int max_runs) {
  const int nrows = int(rows.ptr.size()) - 1;
  std::vector<int> count(size_t(std::max(nrows, 0)));
  for (int r = 0; r < nrows; r++) count[size_t(r)] = int(rows.ptr[r + 1] - rows.ptr[r]);
  sell_shape(count.data(), group_rows, out, lanes, max_runs);
  out.col.assign(size_t(out.nslots) * 32, 0);
  out.src.assign(size_t(out.nslots) * 32, -1);
  // block k of the row at offset r of slice s sits in slot k / lanes, lane r*lanes + k % lanes
#pragma omp parallel for schedule(static)
  for (int s = 0; s < out.nslices; s++) {
    for (int r = 0; r < out.nrows[s]; r++) {
      const int row = out.row0[s] + r;
      const int64_t b = rows.ptr[row];
      const int n = int(rows.ptr[row + 1] - b);
      for (int k = 0; k < n; k++) {
        const size_t at = (size_t(out.slot0[s]) + k / lanes) * 32 + size_t(r) * lanes + k % lanes;
        out.col[at] = rows.col[b + k];
        out.src[at] = rows.src[b + k];
      }
    }
  }
}

void element_profile(int n_node, int n_elem, int nn, const int *conn, std::vector<int> &indexL,
                     std::vector<int> &itemL, std::vector<int> &indexU, std::vector<int> &itemU) {
  // node -> elements, then the neighbour sets of each node (independent per node)
  std::vector<int> eptr(size_t(n_node) + 1, 0), elist(size_t(n_elem) * nn);
  for (int64_t k = 0; k < int64_t(n_elem) * nn; k++) {
    const int v = conn[k];
    if (v < 1 || v > n_node) throw std::runtime_error("element node id out of range");
    eptr[size_t(v)]++;
  }
  for (int i = 0; i < n_node; i++) eptr[size_t(i) + 1] += eptr[size_t(i)];
  {
    std::vector<int> at(eptr.begin(), eptr.end() - 1);
    for (int e = 0; e < n_elem; e++)
      for (int a = 0; a < nn; a++) elist[size_t(at[size_t(conn[size_t(e) * nn + a] - 1)]++)] = e;
  }
  std::vector<std::vector<int>> lo(static_cast<size_t>(n_node)), up(static_cast<size_t>(n_node));
#pragma omp parallel for schedule(dynamic, 1024)
  for (int i = 0; i < n_node; i++) {
    auto &l = lo[size_t(i)], &u = up[size_t(i)];
    for (int k = eptr[size_t(i)]; k < eptr[size_t(i) + 1]; k++) {
      const int e = elist[size_t(k)];
      for (int a = 0; a < nn; a++) {
        const int j = conn[size_t(e) * nn + a];
        if (j < i + 1) l.push_back(j);
        else if (j > i + 1) u.push_back(j);
      }
    }
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
  }
  indexL.assign(size_t(n_node) + 1, 0);
  indexU.assign(size_t(n_node) + 1, 0);
  for (int i = 0; i < n_node; i++) {
    indexL[size_t(i) + 1] = indexL[size_t(i)] + int(lo[size_t(i)].size());
    indexU[size_t(i) + 1] = indexU[size_t(i)] + int(up[size_t(i)].size());
  }
  itemL.resize(size_t(indexL[size_t(n_node)]));
  itemU.resize(size_t(indexU[size_t(n_node)]));
  for (int i = 0; i < n_node; i++) {
    std::copy(lo[size_t(i)].begin(), lo[size_t(i)].end(), itemL.begin() + indexL[size_t(i)]);
    std::copy(up[size_t(i)].begin(), up[size_t(i)].end(), itemU.begin() + indexU[size_t(i)]);
  }
}

void element_contributions(int n_node, int n_elem, int nn, const int *conn, const std::vector<int> &indexL,
                           const std::vector<int> &itemL, const std::vector<int> &indexU,
                           const std::vector<int> &itemU, std::vector<int64_t> &ptr, std::vector<int> &code) {
  if (int64_t(n_elem) * nn * nn >= (int64_t(1) << 31)) throw std::runtime_error("too many elements");
  const int64_t NPL = indexL[size_t(n_node)], NPU = indexU[size_t(n_node)];
  const int64_t nb = int64_t(n_node) + NPL + NPU;
  // raw block id of (row i, column j), both 0-based
  auto block_of = [&](int i, int j) -> int64_t {
    if (i == j) return i;
    if (j < i) {
      const int *b = itemL.data() + indexL[size_t(i)], *e = itemL.data() + indexL[size_t(i) + 1];
      return int64_t(n_node) + (std::lower_bound(b, e, j + 1) - itemL.data());
    }
    const int *b = itemU.data() + indexU[size_t(i)], *e = itemU.data() + indexU[size_t(i) + 1];
    return int64_t(n_node) + NPL + (std::lower_bound(b, e, j + 1) - itemU.data());
  };
  std::vector<int64_t> blk(size_t(n_elem) * nn * nn);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < n_elem; e++)
    for (int a = 0; a < nn; a++)
      for (int b = 0; b < nn; b++)
        blk[(size_t(e) * nn + a) * nn + b] = block_of(conn[size_t(e) * nn + a] - 1, conn[size_t(e) * nn + b] - 1);
  ptr.assign(size_t(nb) + 1, 0);
  for (int64_t v : blk) ptr[size_t(v) + 1]++;
  for (int64_t i = 0; i < nb; i++) ptr[size_t(i) + 1] += ptr[size_t(i)];
  code.resize(blk.size());
  std::vector<int64_t> at(ptr.begin(), ptr.end() - 1);
  // element order inside every block's list (e ascending, then a, b as in the scatter loop)
  for (size_t k = 0; k < blk.size(); k++) code[size_t(at[size_t(blk[k])]++)] = int(k);
}

void order_rows_by_length(const BlockRows &lower, const BlockRows &upper, const std::vector<int> &group_rows,
                          int lanes, std::vector<int> &order) {
  const int n = int(lower.ptr.size()) - 1;
  std::vector<int> nl(size_t(std::max(n, 0))), nu(size_t(std::max(n, 0)));
  for (int r = 0; r < n; r++) {
    nl[size_t(r)] = int(lower.ptr[r + 1] - lower.ptr[r]);
    nu[size_t(r)] = int(upper.ptr[r + 1] - upper.ptr[r]);
  }
  order_rows_by_counts(nl.data(), nu.data(), n, group_rows, lanes, order);
}

void order_rows_by_counts(const int *nl, const int *nu, int n, const std::vector<int> &group_rows, int lanes,
                          std::vector<int> &order) {
  order.resize(size_t(n));
  auto cls = [lanes](const int *c, int r) { return (c[r] + lanes - 1) / lanes; };
  int maxu = 0;
  for (int r = 0; r < n; r++) maxu = std::max(maxu, cls(nu, r));
  // a stable counting sort of each group by the key (lower slots, upper slots)
  const int ng = int(group_rows.size()) - 1;
#pragma omp parallel for schedule(dynamic, 1)
  for (int g = 0; g < ng; g++) {
    const int r0 = group_rows[size_t(g)], r1 = group_rows[size_t(g) + 1];
    std::vector<int> key(size_t(r1 - r0));
    int kmax = 0;
    for (int r = r0; r < r1; r++) {
      key[size_t(r - r0)] = cls(nl, r) * (maxu + 1) + cls(nu, r);
      kmax = std::max(kmax, key[size_t(r - r0)]);
    }
    std::vector<int> start(size_t(kmax) + 2, 0);
    for (int k : key) start[size_t(k) + 1]++;
    for (int k = 0; k <= kmax; k++) start[size_t(k) + 1] += start[size_t(k)];
    for (int r = r0; r < r1; r++) order[size_t(r0 + start[size_t(key[size_t(r - r0)])]++)] = r;
  }
}

void permute_rows(const BlockRows &in, const std::vector<int> &order, const std::vector<int> &iorder,
                  BlockRows &out) {
  const int n = int(order.size());
  out.ptr.assign(size_t(n) + 1, 0);
  for (int i = 0; i < n; i++) out.ptr[size_t(i) + 1] = out.ptr[size_t(i)] + in.ptr[order[i] + 1] - in.ptr[order[i]];
  out.col.resize(in.col.size());
  out.src.resize(in.src.size());
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    int64_t w = out.ptr[size_t(i)];
    for (int64_t k = in.ptr[order[i]]; k < in.ptr[order[i] + 1]; k++, w++) {
      out.col[size_t(w)] = iorder[size_t(in.col[size_t(k)])];
      out.src[size_t(w)] = in.src[size_t(k)];
    }
  }
}

namespace {

// In-place 3x3 LU with reciprocal pivots (the reference's ALU / ILU1a33 form).
bool lu33_inplace(double *a) {
  double T[3][3] = {{a[0], a[1], a[2]}, {a[3], a[4], a[5]}, {a[6], a[7], a[8]}};
  bool zero = false;
  for (int k = 0; k < 3; k++) {
    if (T[k][k] == 0.0) zero = true;
    T[k][k] = 1.0 / T[k][k];
    for (int i = k + 1; i < 3; i++) {
      T[i][k] = T[i][k] * T[k][k];
      double PW[3];
      for (int j = k + 1; j < 3; j++) PW[j] = T[i][j] - T[i][k] * T[k][j];
      for (int j = k + 1; j < 3; j++) T[i][j] = PW[j];
    }
  }
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) a[3 * r + c] = T[r][c];
  return zero;
}

// RHS = Aik * Dk^-1 * Akj with Dk in reciprocal-pivot LU form (ILU1b33).
void aik_dinv_akj(double *RHS, const double *Dk, const double *Aik, const double *Akj) {
  for (int c = 0; c < 3; c++) {
    double x1 = Akj[c], x2 = Akj[3 + c], x3 = Akj[6 + c];
    x2 = x2 - Dk[3] * x1;
    x3 = x3 - Dk[6] * x1 - Dk[7] * x2;
    x3 = Dk[8] * x3;
    x2 = Dk[4] * (x2 - Dk[5] * x3);
    x1 = Dk[0] * (x1 - Dk[2] * x3 - Dk[1] * x2);
    RHS[c] = Aik[0] * x1 + Aik[1] * x2 + Aik[2] * x3;
    RHS[3 + c] = Aik[3] * x1 + Aik[4] * x2 + Aik[5] * x3;
    RHS[6 + c] = Aik[6] * x1 + Aik[7] * x2 + Aik[8] * x3;
  }
}

}  // namespace

int factor_bilu0(const Profile &p, const double *D, const double *AL, const double *AU,
                 double sigma_diag, std::vector<double> &Dlu0, std::vector<double> &ALlu0,
                 std::vector<double> &AUlu0) {
  Dlu0.assign(D, D + 9 * size_t(p.N));
  ALlu0.assign(AL, AL + 9 * size_t(p.NPL()));
  AUlu0.assign(AU, AU + 9 * size_t(p.NPU()));
  return factor_bilu0_inplace(p, Dlu0.data(), ALlu0.data(), AUlu0.data(), sigma_diag);
}

int factor_bilu0_inplace(const Profile &p, double *Dlu0, double *ALlu0, double *AUlu0, double sigma_diag) {
  const int N = p.N;
  for (int i = 0; i < N; i++) {
    Dlu0[9 * size_t(i)] *= sigma_diag;
    Dlu0[9 * size_t(i) + 4] *= sigma_diag;
    Dlu0[9 * size_t(i) + 8] *= sigma_diag;
  }
  // Row i reads only rows k of its lower list (their final U blocks and diagonal LU)
  // and writes only its own blocks, so the rows of one level of the lower pattern are
  // factored in parallel; each row's arithmetic is the natural-order sweep's, in the
  // same order, so the factors are the serial ones bit for bit.  Level order reads the
  // neighbours' rows from farther back than the natural order (on a 101^3 27-point
  // profile one thread takes 5.5 s against 3.0 s in natural order), so with fewer
  // than four threads the rows go in natural order.
  std::vector<int> order, level_ptr;
  if (omp_get_max_threads() >= 4) {
    level_schedule(p, true, order, level_ptr);
  } else {
    order.resize(size_t(N));
    for (int i = 0; i < N; i++) order[size_t(i)] = i;
    level_ptr = {0, N};  // one "level": the loop below then runs the rows in order on one thread
  }
  const int nlev = int(level_ptr.size()) - 1;
  const bool serial = nlev == 1 && omp_get_max_threads() < 4;
  int bad = 0;
#pragma omp parallel if (!serial)
  {
    // position markers of row i's lower / upper entries (0 = absent), per thread
    std::vector<int> posL(static_cast<size_t>(N), 0), posU(static_cast<size_t>(N), 0);
    double RHS[9];
    for (int lv = 0; lv < nlev; lv++) {
#pragma omp for schedule(static)
      for (int t = level_ptr[size_t(lv)]; t < level_ptr[size_t(lv) + 1]; t++) {
        const int i = order[size_t(t)];
        for (int k = p.indexL[i]; k < p.indexL[i + 1]; k++) posL[size_t(p.itemL[k] - 1)] = k + 1;
        for (int k = p.indexU[i]; k < p.indexU[i + 1]; k++)
          if (p.itemU[k] <= N) posU[size_t(p.itemU[k] - 1)] = k + 1;
        for (int kk = p.indexL[i]; kk < p.indexL[i + 1]; kk++) {
          const int k = p.itemL[kk] - 1;
          double Aik[9];
          std::memcpy(Aik, &ALlu0[9 * size_t(kk)], sizeof(Aik));
          const double *Dk = &Dlu0[9 * size_t(k)];
          for (int jj = p.indexU[k]; jj < p.indexU[k + 1]; jj++) {
            const int j = p.itemU[jj] - 1;
            if (j >= N) continue;
            // a row's own id is in neither of its lists, so j == i never passes here and
            // the diagonal block is left as it is (as in the reference)
            if (posL[size_t(j)] == 0 && posU[size_t(j)] == 0) continue;
            aik_dinv_akj(RHS, Dk, Aik, &AUlu0[9 * size_t(jj)]);
            double *dst = j < i ? &ALlu0[9 * size_t(posL[size_t(j)] - 1)] : &AUlu0[9 * size_t(posU[size_t(j)] - 1)];
            for (int q = 0; q < 9; q++) dst[q] = dst[q] - RHS[q];
          }
        }
        if (lu33_inplace(&Dlu0[9 * size_t(i)])) {
#pragma omp atomic write
          bad = 1;
        }
        for (int k = p.indexL[i]; k < p.indexL[i + 1]; k++) posL[size_t(p.itemL[k] - 1)] = 0;
        for (int k = p.indexU[i]; k < p.indexU[i + 1]; k++)
          if (p.itemU[k] <= N) posU[size_t(p.itemU[k] - 1)] = 0;
      }
    }
  }
  return bad ? 9001 : 0;
}

void bilu_fill(const Profile &p, int level, FilledProfile &f) {
  const int N = p.N;
  // per row: fill columns (0-based) with their level, collected as the reference
  // scans (the order of collection is undone by the sort)
  std::vector<std::vector<std::pair<int, int>>> fill(static_cast<size_t>(N));
  std::vector<int> mark(static_cast<size_t>(N), 0);
  std::vector<int> touched;
  auto reset = [&]() {
    for (int c : touched) mark[size_t(c)] = 0;
    touched.clear();
  };
  auto set = [&](int c) {
    if (!mark[size_t(c)]) touched.push_back(c);
    mark[size_t(c)] = 1;
  };
  // level 1
  for (int i = 1; i < N; i++) {
    set(i);
    for (int k = p.indexL[i]; k < p.indexL[i + 1]; k++) set(p.itemL[k] - 1);
    for (int k = p.indexU[i]; k < p.indexU[i + 1]; k++)
      if (p.itemU[k] <= N) set(p.itemU[k] - 1);
    for (int kk = p.indexL[i]; kk < p.indexL[i + 1]; kk++) {
      const int k = p.itemL[kk] - 1;
      for (int j = p.indexU[k]; j < p.indexU[k + 1]; j++) {
        const int c = p.itemU[j] - 1;
        if (c >= N || mark[size_t(c)]) continue;
        fill[size_t(i)].push_back({c, 1});
        set(c);
      }
    }
    reset();
  }
  // level 2: original L x level-1 U, then level-1 L x original U
  if (level >= 2) {
    std::vector<std::vector<std::pair<int, int>>> fill2(static_cast<size_t>(N));
    for (int i = 1; i < N; i++) {
      set(i);
      for (int k = p.indexL[i]; k < p.indexL[i + 1]; k++) set(p.itemL[k] - 1);
      for (int k = p.indexU[i]; k < p.indexU[i + 1]; k++)
        if (p.itemU[k] <= N) set(p.itemU[k] - 1);
      for (const auto &e : fill[size_t(i)]) set(e.first);
      for (int kk = p.indexL[i]; kk < p.indexL[i + 1]; kk++) {
        const int k = p.itemL[kk] - 1;
        for (const auto &e : fill[size_t(k)]) {
          const int c = e.first;
          if (c <= k || mark[size_t(c)]) continue;  // level-1 U entries of row k
          fill2[size_t(i)].push_back({c, 2});
          set(c);
        }
      }
      for (const auto &fe : fill[size_t(i)]) {
        const int k = fe.first;
        if (k >= i) continue;  // level-1 L entries of row i
        for (int j = p.indexU[k]; j < p.indexU[k + 1]; j++) {
          const int c = p.itemU[j] - 1;
          if (c >= N || mark[size_t(c)]) continue;
          fill2[size_t(i)].push_back({c, 2});
          set(c);
        }
      }
      reset();
    }
    for (int i = 0; i < N; i++)
      fill[size_t(i)].insert(fill[size_t(i)].end(), fill2[size_t(i)].begin(), fill2[size_t(i)].end());
  }
  f = FilledProfile();
  f.N = N;
  f.indexL.assign(size_t(N) + 1, 0);
  f.indexU.assign(size_t(N) + 1, 0);
  struct E {
    int col, lev, src;
  };
  std::vector<E> lo, up;
  for (int i = 0; i < N; i++) {
    lo.clear();
    up.clear();
    for (int k = p.indexL[i]; k < p.indexL[i + 1]; k++) lo.push_back({p.itemL[k] - 1, 0, k});
    for (int k = p.indexU[i]; k < p.indexU[i + 1]; k++)
      if (p.itemU[k] <= N) up.push_back({p.itemU[k] - 1, 0, k});
    for (const auto &e : fill[size_t(i)]) (e.first < i ? lo : up).push_back({e.first, e.second, -1});
    auto by_col = [](const E &a, const E &b) { return a.col < b.col; };
    std::sort(lo.begin(), lo.end(), by_col);  // distinct columns: any sort gives the reference's order
    std::sort(up.begin(), up.end(), by_col);
    for (const auto &e : lo) {
      f.itemL.push_back(e.col + 1);
      f.levL.push_back(e.lev);
      f.srcL.push_back(e.src);
    }
    for (const auto &e : up) {
      f.itemU.push_back(e.col + 1);
      f.levU.push_back(e.lev);
      f.srcU.push_back(e.src);
    }
    f.indexL[size_t(i) + 1] = int(f.itemL.size());
    f.indexU[size_t(i) + 1] = int(f.itemU.size());
  }
}

int factor_bilu_fill(const FilledProfile &f, int level, const double *D, const double *AL, const double *AU,
                     double sigma_diag, std::vector<double> &Dlu, std::vector<double> &ALlu,
                     std::vector<double> &AUlu) {
  const int N = f.N;
  const size_t nL = f.itemL.size(), nU = f.itemU.size();
  Dlu.assign(D, D + 9 * size_t(N));
  ALlu.assign(9 * nL, 0.0);
  AUlu.assign(9 * nU, 0.0);
  for (size_t k = 0; k < nL; k++)
    if (f.srcL[k] >= 0) std::memcpy(&ALlu[9 * k], AL + 9 * size_t(f.srcL[k]), 9 * sizeof(double));
  for (size_t k = 0; k < nU; k++)
    if (f.srcU[k] >= 0) std::memcpy(&AUlu[9 * k], AU + 9 * size_t(f.srcU[k]), 9 * sizeof(double));
  for (int i = 0; i < N; i++) {
    Dlu[9 * size_t(i)] *= sigma_diag;
    Dlu[9 * size_t(i) + 4] *= sigma_diag;
    Dlu[9 * size_t(i) + 8] *= sigma_diag;
  }
  if (N > 0 && lu33_inplace(Dlu.data())) return 9001;
  std::vector<int> posL(static_cast<size_t>(N), 0), posU(static_cast<size_t>(N), 0);
  double RHS[9];
  for (int i = 1; i < N; i++) {
    for (int k = f.indexL[i]; k < f.indexL[i + 1]; k++) posL[size_t(f.itemL[k] - 1)] = k + 1;
    for (int k = f.indexU[i]; k < f.indexU[i + 1]; k++) posU[size_t(f.itemU[k] - 1)] = k + 1;
    for (int kk = f.indexL[i]; kk < f.indexL[i + 1]; kk++) {
      const int lik = f.levL[size_t(kk)];
      if (lik >= level) continue;
      const int k = f.itemL[kk] - 1;
      double Aik[9];
      std::memcpy(Aik, &ALlu[9 * size_t(kk)], sizeof(Aik));
      const double *Dk = &Dlu[9 * size_t(k)];
      for (int jj = f.indexU[k]; jj < f.indexU[k + 1]; jj++) {
        if (lik + f.levU[size_t(jj)] >= level) continue;
        const int j = f.itemU[jj] - 1;
        aik_dinv_akj(RHS, Dk, Aik, &AUlu[9 * size_t(jj)]);
        double *dst = j == i ? &Dlu[9 * size_t(i)]
                             : (j < i ? &ALlu[9 * size_t(posL[size_t(j)] - 1)] : &AUlu[9 * size_t(posU[size_t(j)] - 1)]);
        for (int e = 0; e < 9; e++) dst[e] = dst[e] - RHS[e];
      }
    }
    if (lu33_inplace(&Dlu[9 * size_t(i)])) return 9001;
    for (int k = f.indexL[i]; k < f.indexL[i + 1]; k++) posL[size_t(f.itemL[k] - 1)] = 0;
    for (int k = f.indexU[i]; k < f.indexU[i + 1]; k++) posU[size_t(f.itemU[k] - 1)] = 0;
  }
  return 0;
}

void level_schedule(const Profile &p, bool lower, std::vector<int> &order,
                    std::vector<int> &level_ptr) {
  const int N = p.N;
  std::vector<int> lev(N, 0);
  int maxlev = 0;
  if (lower) {
    for (int i = 0; i < N; i++) {
      int l = 0;
      for (int k = p.indexL[i]; k < p.indexL[i + 1]; k++) l = std::max(l, lev[p.itemL[k] - 1] + 1);
      lev[i] = l;
      maxlev = std::max(maxlev, l);
    }
  } else {
    for (int i = N - 1; i >= 0; i--) {
      int l = 0;
      for (int k = p.indexU[i]; k < p.indexU[i + 1]; k++) {
        if (p.itemU[k] > N) continue;
        l = std::max(l, lev[p.itemU[k] - 1] + 1);
      }
      lev[i] = l;
      maxlev = std::max(maxlev, l);
    }
  }
  // The backward sweep walks its groups from the last to the first (as the SSOR
  // backward sweep walks the colours), so the upper schedule numbers its groups
  // from the highest level down: group maxlev - l holds level l.
  if (!lower)
    for (int i = 0; i < N; i++) lev[i] = maxlev - lev[i];
  level_ptr.assign(size_t(maxlev) + 2, 0);
  for (int i = 0; i < N; i++) level_ptr[lev[i] + 1]++;
  for (int l = 0; l <= maxlev; l++) level_ptr[l + 1] += level_ptr[l];
  order.assign(N, 0);
  std::vector<int> fill(level_ptr.begin(), level_ptr.end() - 1);
  for (int i = 0; i < N; i++) order[fill[lev[i]]++] = i;
  if (!lower) {
    // the backward sweep visits higher ids first inside a level; keep descending ids
    for (int l = 0; l <= maxlev; l++) std::reverse(order.begin() + level_ptr[l], order.begin() + level_ptr[l + 1]);
  }
}

namespace {

// Compressed adjacency lists (row r: col[ptr[r] .. ptr[r+1]), ascending, no self).
struct Csr {
  std::vector<int64_t> ptr;
  std::vector<int> col;
  int n() const { return int(ptr.size()) - 1; }
};

// One greedy distance-1 aggregation pass.
int aggregate_pass(const Csr &g, std::vector<int> &agg) {
  const int n = g.n();
  agg.assign(size_t(n), -1);
  int na = 0;
  for (int i = 0; i < n; i++) {
    if (agg[size_t(i)] >= 0) continue;
    bool free_nbhd = true;
    for (int64_t k = g.ptr[size_t(i)]; k < g.ptr[size_t(i) + 1]; k++)
      if (agg[size_t(g.col[size_t(k)])] >= 0) {
        free_nbhd = false;
        break;
      }
    if (!free_nbhd) continue;
    agg[size_t(i)] = na;
    for (int64_t k = g.ptr[size_t(i)]; k < g.ptr[size_t(i) + 1]; k++) agg[size_t(g.col[size_t(k)])] = na;
    na++;
  }
  std::vector<int> root_agg(agg);  // the aggregates the roots formed
  for (int i = 0; i < n; i++) {
    if (agg[size_t(i)] >= 0) continue;
    for (int64_t k = g.ptr[size_t(i)]; k < g.ptr[size_t(i) + 1]; k++)
      if (root_agg[size_t(g.col[size_t(k)])] >= 0) {
        agg[size_t(i)] = root_agg[size_t(g.col[size_t(k)])];
        break;
      }
    if (agg[size_t(i)] < 0) agg[size_t(i)] = na++;  // no aggregated neighbour (isolated node)
  }
  return na;
}

// The graph of aggregates: a ~ b when a node of a neighbours a node of b.
Csr coarse_graph(const Csr &g, const std::vector<int> &a, int na) {
  const int n = g.n();
  std::vector<int64_t> mptr(size_t(na) + 1, 0);
  for (int u = 0; u < n; u++) mptr[size_t(a[size_t(u)]) + 1]++;
  for (int c = 0; c < na; c++) mptr[size_t(c) + 1] += mptr[size_t(c)];
  std::vector<int> members(static_cast<size_t>(n));
  {
    std::vector<int64_t> fill(mptr.begin(), mptr.end() - 1);
    for (int u = 0; u < n; u++) members[size_t(fill[size_t(a[size_t(u)])]++)] = u;
  }
  Csr h;
  h.ptr.assign(size_t(na) + 1, 0);
  std::vector<int> mark(size_t(na), -1);
  for (int c = 0; c < na; c++) {
    for (int64_t m = mptr[size_t(c)]; m < mptr[size_t(c) + 1]; m++) {
      const int u = members[size_t(m)];
      for (int64_t k = g.ptr[size_t(u)]; k < g.ptr[size_t(u) + 1]; k++) {
        const int b = a[size_t(g.col[size_t(k)])];
        if (b != c && mark[size_t(b)] != c) {
          mark[size_t(b)] = c;
          h.col.push_back(b);
        }
      }
    }
    h.ptr[size_t(c) + 1] = int64_t(h.col.size());
  }
  for (int c = 0; c < na; c++) std::sort(h.col.begin() + h.ptr[size_t(c)], h.col.begin() + h.ptr[size_t(c) + 1]);
  return h;
}

// For every row r: the sorted union of the values lists[q] (each in 0 .. nvals-1) over
// q in items(r); distinct values found with a marker array per thread; two passes
// (count, fill), rows in parallel.
template <class Items, class Lists>
void row_unions(int nrows, int nvals, Items items, Lists lists, std::vector<int> &ptr, std::vector<int> &out) {
  std::vector<int> cnt(size_t(nrows) + 1, 0);
  ptr.assign(size_t(nrows) + 1, 0);
  for (int pass = 0; pass < 2; pass++) {
#pragma omp parallel
    {
      std::vector<int> tmp, mark(size_t(nvals), -1);
#pragma omp for schedule(dynamic, 1024)
      for (int r = 0; r < nrows; r++) {
        tmp.clear();
        items(r, [&](int q) {
          lists(q, [&](int v) {
            if (mark[size_t(v)] != r) {
              mark[size_t(v)] = r;
              tmp.push_back(v);
            }
          });
        });
        if (pass == 0) {
          cnt[size_t(r) + 1] = int(tmp.size());
        } else {
          std::sort(tmp.begin(), tmp.end());
          std::copy(tmp.begin(), tmp.end(), out.begin() + ptr[size_t(r)]);
        }
      }
    }
    if (pass == 0) {
      for (int r = 0; r < nrows; r++) ptr[size_t(r) + 1] = ptr[size_t(r)] + cnt[size_t(r) + 1];
      out.assign(size_t(ptr[size_t(nrows)]), 0);
    }
  }
}

}  // namespace

void aggregate_nodes(const Profile &p, int max_aggregates, Aggregation &out) {
  const int N = p.N;
  // the node graph: row i's own neighbours (its L and U items, ascending; the blocks
  // the device kernels read for row i), in-range and not i
  Csr adj;
  adj.ptr.assign(size_t(N) + 1, 0);
  auto keep = [&](int i, int c) { return c >= 0 && c < N && c != i; };
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    int64_t k = 0;
    for (int j = p.indexL[i]; j < p.indexL[i + 1]; j++) k += keep(i, p.itemL[j] - 1);
    for (int j = p.indexU[i]; j < p.indexU[i + 1]; j++) k += keep(i, p.itemU[j] - 1);
    adj.ptr[size_t(i) + 1] = k;
  }
  for (int i = 0; i < N; i++) adj.ptr[size_t(i) + 1] += adj.ptr[size_t(i)];
  adj.col.assign(size_t(adj.ptr[size_t(N)]), 0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    int64_t w = adj.ptr[size_t(i)];
    for (int j = p.indexL[i]; j < p.indexL[i + 1]; j++)
      if (keep(i, p.itemL[j] - 1)) adj.col[size_t(w++)] = p.itemL[j] - 1;
    for (int j = p.indexU[i]; j < p.indexU[i + 1]; j++)
      if (keep(i, p.itemU[j] - 1)) adj.col[size_t(w++)] = p.itemU[j] - 1;
  }
  std::vector<int> agg(static_cast<size_t>(N));
  for (int i = 0; i < N; i++) agg[size_t(i)] = i;
  int n = N;
  const Csr *g = &adj;  // the graph of the current level (the node graph itself first: no copy)
  Csr level;
  for (int pass = 0; pass == 0 || n > max_aggregates; pass++) {
    std::vector<int> a;
    const int na = aggregate_pass(*g, a);
    if (2 * na > n) break;  // no longer coarsening
    for (int i = 0; i < N; i++) agg[size_t(i)] = a[size_t(agg[size_t(i)])];
    level = coarse_graph(*g, a, na);
    g = &level;
    n = na;
  }
  out.n_agg = n;
  out.agg = agg;
  // prolongator pattern: aggregates of each closed neighbourhood
  row_unions(
      N, n,
      [&](int i, auto f) {
        f(i);
        for (int64_t k = adj.ptr[size_t(i)]; k < adj.ptr[size_t(i) + 1]; k++) f(adj.col[size_t(k)]);
      },
      [&](int j, auto f) { f(agg[size_t(j)]); }, out.pptr, out.pagg);
  // two-ring pattern (rows of A P): the union of the neighbours' prolongator patterns
  row_unions(
      N, n,
      [&](int i, auto f) {
        f(i);
        for (int64_t k = adj.ptr[size_t(i)]; k < adj.ptr[size_t(i) + 1]; k++) f(adj.col[size_t(k)]);
      },
      [&](int j, auto f) {
        for (int q = out.pptr[size_t(j)]; q < out.pptr[size_t(j) + 1]; q++) f(out.pagg[size_t(q)]);
      },
      out.qptr, out.qagg);
  // restriction gather: per aggregate its (node, entry) pairs, ascending node
  out.rptr.assign(size_t(n) + 1, 0);
  for (int a : out.pagg) out.rptr[size_t(a) + 1]++;
  for (int a = 0; a < n; a++) out.rptr[size_t(a) + 1] += out.rptr[size_t(a)];
  out.rnode.assign(out.pagg.size(), 0);
  out.rpos.assign(out.pagg.size(), 0);
  {
    std::vector<int> fill(out.rptr.begin(), out.rptr.end() - 1);
    for (int i = 0; i < N; i++)
      for (int q = out.pptr[size_t(i)]; q < out.pptr[size_t(i) + 1]; q++) {
        const int a = out.pagg[size_t(q)];
        out.rnode[size_t(fill[size_t(a)])] = i;
        out.rpos[size_t(fill[size_t(a)]++)] = q;
      }
  }
  // coarse pattern: row a = union of the two-ring patterns of a's restriction nodes
  row_unions(
      n, n,
      [&](int a, auto f) {
        for (int t = out.rptr[size_t(a)]; t < out.rptr[size_t(a) + 1]; t++) f(out.rnode[size_t(t)]);
      },
      [&](int i, auto f) {
        for (int q = out.qptr[size_t(i)]; q < out.qptr[size_t(i) + 1]; q++) f(out.qagg[size_t(q)]);
      },
      out.cptr, out.cagg);
}

}  // namespace h33
