// Host check of the layout split used by the device fill: sell_shape (the layout's
// shape from row counts) against build_sell, the placement rule of the fill kernels
// (block k of the row at offset r of slice s: slot slot0[s] + k / lanes, lane
// r * lanes + k % lanes) against build_sell's col/src, order_rows_by_counts against
// order_rows_by_length, and the reordered layouts built the device's way (counts per
// part, row order and shape from counts, each block placed by its rank among the
// part's smaller new columns, columns renamed to layout rows) against the host chain
// reordered_rows -> permute_rows -> build_sell, on seeded random profiles.
// Prints "ok" and exits 0, or names the first difference and exits 1.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <random>
#include <set>
#include <vector>

#include "h33_setup.h"

using namespace h33;

namespace {

int fail(const char *what, int seed) {
  std::printf("mismatch: %s (seed %d)\n", what, seed);
  return 1;
}

bool same_shape(const SellLayout &a, const SellLayout &b) {
  return a.nslices == b.nslices && a.lanes == b.lanes && a.nslots == b.nslots && a.row0 == b.row0 &&
         a.nrows == b.nrows && a.slot0 == b.slot0 && a.len == b.len && a.rowlen == b.rowlen &&
         a.group_slice == b.group_slice && a.run_ptr == b.run_ptr && a.run_slice == b.run_slice &&
         a.run_slot == b.run_slot && a.run_len == b.run_len;
}

std::vector<int> random_groups(int n, std::mt19937 &g) {
  std::vector<int> groups{0};
  while (groups.back() < n) groups.push_back(std::min(n, groups.back() + 1 + int(g() % 40)));
  return groups;
}

size_t place(const SellLayout &L, int s, int r, int k) {
  return (size_t(L.slot0[size_t(s)]) + size_t(k / L.lanes)) * 32 + size_t(r) * L.lanes + size_t(k % L.lanes);
}

// layout row -> slice
std::vector<int> row_slices(const SellLayout &L, int n) {
  std::vector<int> rs(size_t(n), -1);
  for (int s = 0; s < L.nslices; s++)
    for (int r = 0; r < L.nrows[size_t(s)]; r++) rs[size_t(L.row0[size_t(s)] + r)] = s;
  return rs;
}

// A random symmetric profile of n nodes (1-based items, ascending, no diagonal).
void random_profile(int n, std::mt19937 &g, std::vector<int> &indexL, std::vector<int> &itemL,
                    std::vector<int> &indexU, std::vector<int> &itemU) {
  std::vector<std::set<int>> adj(static_cast<size_t>(n));
  for (int i = 0; i < n; i++) {
    const int deg = int(g() % 12);
    for (int d = 0; d < deg; d++) {
      const int j = int(g() % unsigned(n));
      if (j == i) continue;
      adj[size_t(i)].insert(j);
      adj[size_t(j)].insert(i);
    }
  }
  indexL.assign(size_t(n) + 1, 0);
  indexU.assign(size_t(n) + 1, 0);
  itemL.clear();
  itemU.clear();
  for (int i = 0; i < n; i++) {
    for (int j : adj[size_t(i)]) (j < i ? itemL : itemU).push_back(j + 1);
    indexL[size_t(i) + 1] = int(itemL.size());
    indexU[size_t(i) + 1] = int(itemU.size());
  }
}

}  // namespace

int main() {
  for (int seed = 1; seed <= 40; seed++) {
    std::mt19937 g{static_cast<unsigned>(seed)};
    const int n = 1 + int(g() % 700);
    const int lanes_opts[] = {1, 4, 8, 16};
    const int lanes = lanes_opts[g() % 4];
    const int max_runs = int(g() % 3) == 0 ? 0 : 1 + int(g() % 24);
    // 1. shape from counts, and the fill's placement rule
    BlockRows rows;
    rows.ptr.assign(size_t(n) + 1, 0);
    std::vector<int> count(static_cast<size_t>(n));
    for (int i = 0; i < n; i++) {
      count[size_t(i)] = int(g() % 41);
      rows.ptr[size_t(i) + 1] = rows.ptr[size_t(i)] + count[size_t(i)];
    }
    for (int64_t k = 0; k < rows.ptr[size_t(n)]; k++) {
      rows.col.push_back(int(g() % unsigned(n)));
      rows.src.push_back(int(g() % 100000));
    }
    const std::vector<int> groups = random_groups(n, g);
    SellLayout a, b;
    build_sell(rows, groups, a, lanes, max_runs);
    sell_shape(count.data(), groups, b, lanes, max_runs);
    if (!same_shape(a, b)) return fail("sell_shape != build_sell", seed);
    const std::vector<int> rs = row_slices(b, n);
    std::vector<int> col(size_t(b.nslots) * 32, 0), src(size_t(b.nslots) * 32, -1);
    for (int i = 0; i < n; i++) {
      const int s = rs[size_t(i)], r = i - b.row0[size_t(s)];
      for (int k = 0; k < count[size_t(i)]; k++) {
        col[place(b, s, r, k)] = rows.col[size_t(rows.ptr[size_t(i)] + k)];
        src[place(b, s, r, k)] = rows.src[size_t(rows.ptr[size_t(i)] + k)];
      }
    }
    if (col != a.col || src != a.src) return fail("placement rule != build_sell", seed);

    // 2. the reordered layouts, host chain against the device's way
    std::vector<int> indexL, itemL, indexU, itemU;
    random_profile(n, g, indexL, itemL, indexU, itemU);
    const Profile prof{n, indexL.data(), itemL.data(), indexU.data(), itemU.data()};
    std::vector<int> perm(static_cast<size_t>(n)), iperm(static_cast<size_t>(n));
    for (int i = 0; i < n; i++) perm[size_t(i)] = i;
    std::shuffle(perm.begin(), perm.end(), g);
    for (int i = 0; i < n; i++) iperm[size_t(perm[size_t(i)])] = i;
    const std::vector<int> cgroups = random_groups(n, g);
    const int K = lanes == 1 ? 4 : lanes;
    // host chain (setup_ssor with HECMW33_HOST_LAYOUT=1)
    BlockRows lo_ref, up_ref, lo_h, up_h;
    reordered_rows(prof, perm, iperm, lo_ref, up_ref);
    for (auto *br : {&lo_ref, &up_ref})
      for (int &c : br->col) c = iperm[size_t(c)];
    std::vector<int> order_h, iorder_h(static_cast<size_t>(n));
    order_rows_by_length(lo_ref, up_ref, cgroups, K, order_h);
    for (int i = 0; i < n; i++) iorder_h[size_t(order_h[size_t(i)])] = i;
    permute_rows(lo_ref, order_h, iorder_h, lo_h);
    permute_rows(up_ref, order_h, iorder_h, up_h);
    SellLayout lo_a, up_a;
    build_sell(lo_h, cgroups, lo_a, K, 24);
    build_sell(up_h, cgroups, up_a, K, 24);
    // the device's way
    std::vector<int> nl(size_t(n), 0), nu(size_t(n), 0);
    for (int iold = 0; iold < n; iold++) {
      const int inew = iperm[size_t(iold)];
      for (int j = indexL[size_t(iold)]; j < indexL[size_t(iold) + 1]; j++)
        (iperm[size_t(itemL[size_t(j)] - 1)] < inew ? nl : nu)[size_t(inew)]++;
      for (int j = indexU[size_t(iold)]; j < indexU[size_t(iold) + 1]; j++)
        (iperm[size_t(itemU[size_t(j)] - 1)] < inew ? nl : nu)[size_t(inew)]++;
    }
    std::vector<int> order, iorder(static_cast<size_t>(n)), cl(static_cast<size_t>(n)), cu(static_cast<size_t>(n));
    order_rows_by_counts(nl.data(), nu.data(), n, cgroups, K, order);
    if (order != order_h) return fail("order_rows_by_counts != order_rows_by_length", seed);
    for (int q = 0; q < n; q++) {
      iorder[size_t(order[size_t(q)])] = q;
      cl[size_t(q)] = nl[size_t(order[size_t(q)])];
      cu[size_t(q)] = nu[size_t(order[size_t(q)])];
    }
    SellLayout lo_b, up_b;
    sell_shape(cl.data(), cgroups, lo_b, K, 24);
    sell_shape(cu.data(), cgroups, up_b, K, 24);
    if (!same_shape(lo_a, lo_b) || !same_shape(up_a, up_b)) return fail("reordered shape", seed);
    const std::vector<int> rsl = row_slices(lo_b, n);
    for (int part = 0; part < 2; part++) {
      const SellLayout &B = part == 0 ? lo_b : up_b;
      const SellLayout &A = part == 0 ? lo_a : up_a;
      std::vector<int> dcol(size_t(B.nslots) * 32, 0), dsrc(size_t(B.nslots) * 32, -1);
      for (int q = 0; q < n; q++) {
        const int inew = order[size_t(q)], iold = perm[size_t(inew)];
        const int s = rsl[size_t(q)], r = q - B.row0[size_t(s)];
        std::vector<std::pair<int, int>> blocks;  // (new column, raw id) of the row's stored blocks
        for (int j = indexL[size_t(iold)]; j < indexL[size_t(iold) + 1]; j++)
          blocks.emplace_back(iperm[size_t(itemL[size_t(j)] - 1)], n + j);
        for (int j = indexU[size_t(iold)]; j < indexU[size_t(iold) + 1]; j++)
          blocks.emplace_back(iperm[size_t(itemU[size_t(j)] - 1)], n + indexL[size_t(n)] + j);
        for (const auto &e : blocks) {
          const bool mine = part == 0 ? e.first < inew : e.first > inew;
          if (!mine) continue;
          int rank = 0;
          for (const auto &f : blocks)
            if ((part == 0 ? f.first < inew : f.first > inew) && f.first < e.first) rank++;
          dcol[place(B, s, r, rank)] = iorder[size_t(e.first)];
          dsrc[place(B, s, r, rank)] = e.second;
        }
      }
      if (dcol != A.col || dsrc != A.src) return fail(part == 0 ? "reordered lower blocks" : "reordered upper blocks", seed);
    }
  }
  std::printf("ok\n");
  return 0;
}
