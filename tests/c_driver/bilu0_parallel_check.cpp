// Host check of factor_bilu0's level-parallel factorisation: on seeded random
// symmetric profiles (and a 27-point box) with diagonally dominant 3x3 blocks, the
// factors computed with one thread (rows in natural order) and with several threads
// (rows of one level of the lower pattern in parallel) are equal bit for bit, and a
// zero pivot gives 9001 either way.  Prints "ok" and exits 0, or names the first
// difference and exits 1.
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <random>
#include <set>
#include <vector>

#include "h33_setup.h"

using namespace h33;

namespace {

struct System {
  std::vector<int> indexL, itemL, indexU, itemU;
  std::vector<double> D, AL, AU;
  Profile prof() const { return Profile{int(indexL.size()) - 1, indexL.data(), itemL.data(), indexU.data(), itemU.data()}; }
};

void fill_values(System &s, std::mt19937 &g) {
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  const size_t n = s.indexL.size() - 1;
  s.D.resize(9 * n);
  for (size_t i = 0; i < s.D.size(); i++) s.D[i] = (i % 9 == 0 || i % 9 == 4 || i % 9 == 8) ? 60.0 + u(g) : 0.1 * u(g);
  s.AL.resize(9 * s.itemL.size());
  s.AU.resize(9 * s.itemU.size());
  for (auto &v : s.AL) v = u(g);
  for (auto &v : s.AU) v = u(g);
}

System random_system(int n, std::mt19937 &g) {
  std::vector<std::set<int>> adj(static_cast<size_t>(n));
  for (int i = 0; i < n; i++) {
    const int deg = int(g() % 10);
    for (int d = 0; d < deg; d++) {
      const int j = int(g() % unsigned(n));
      if (j == i) continue;
      adj[size_t(i)].insert(j);
      adj[size_t(j)].insert(i);
    }
  }
  System s;
  s.indexL.assign(size_t(n) + 1, 0);
  s.indexU.assign(size_t(n) + 1, 0);
  for (int i = 0; i < n; i++) {
    for (int j : adj[size_t(i)]) (j < i ? s.itemL : s.itemU).push_back(j + 1);
    s.indexL[size_t(i) + 1] = int(s.itemL.size());
    s.indexU[size_t(i) + 1] = int(s.itemU.size());
  }
  fill_values(s, g);
  return s;
}

System box_system(int m, std::mt19937 &g) {
  System s;
  const int n = m * m * m;
  s.indexL.assign(size_t(n) + 1, 0);
  s.indexU.assign(size_t(n) + 1, 0);
  for (int k = 0; k < m; k++)
    for (int j = 0; j < m; j++)
      for (int i = 0; i < m; i++) {
        const int r = (k * m + j) * m + i;
        for (int dk = -1; dk <= 1; dk++)
          for (int dj = -1; dj <= 1; dj++)
            for (int di = -1; di <= 1; di++) {
              const int a = i + di, b = j + dj, c = k + dk;
              if (a < 0 || b < 0 || c < 0 || a >= m || b >= m || c >= m) continue;
              const int q = (c * m + b) * m + a;
              if (q < r) s.itemL.push_back(q + 1);
              else if (q > r) s.itemU.push_back(q + 1);
            }
        s.indexL[size_t(r) + 1] = int(s.itemL.size());
        s.indexU[size_t(r) + 1] = int(s.itemU.size());
      }
  fill_values(s, g);
  return s;
}

int factor(const System &s, int threads, std::vector<double> &d, std::vector<double> &l, std::vector<double> &u) {
  omp_set_num_threads(threads);
  return factor_bilu0(s.prof(), s.D.data(), s.AL.data(), s.AU.data(), 1.0, d, l, u);
}

bool same_bits(const std::vector<double> &a, const std::vector<double> &b) {
  return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(double)) == 0);
}

}  // namespace

int main() {
  for (int seed = 1; seed <= 12; seed++) {
    std::mt19937 g{static_cast<unsigned>(seed)};
    System s = seed <= 10 ? random_system(1 + int(g() % 3000), g) : box_system(12 + seed, g);
    std::vector<double> d1, l1, u1, d8, l8, u8;
    const int rc1 = factor(s, 1, d1, l1, u1), rc8 = factor(s, 8, d8, l8, u8);
    if (rc1 != 0 || rc8 != 0) {
      std::printf("mismatch: unexpected zero pivot (seed %d)\n", seed);
      return 1;
    }
    if (!same_bits(d1, d8) || !same_bits(l1, l8) || !same_bits(u1, u8)) {
      std::printf("mismatch: factors differ between 1 and 8 threads (seed %d)\n", seed);
      return 1;
    }
    // a zero pivot in a row of a late level
    const int n = s.prof().N;
    const int bad = n - 1 - int(g() % unsigned(std::max(1, n / 4)));
    for (int e = 0; e < 9; e++) s.D[9 * size_t(bad) + size_t(e)] = 0.0;
    if (factor(s, 1, d1, l1, u1) != 9001 || factor(s, 8, d8, l8, u8) != 9001) {
      std::printf("mismatch: zero pivot not reported (seed %d)\n", seed);
      return 1;
    }
  }
  std::printf("ok\n");
  return 0;
}
