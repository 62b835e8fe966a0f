// Integer-partition basis of the edge sectors (host only).
//
// Semantics follow the reference's iparts::integer_partitions:
//  - generation: the accelerated ascending algorithm (Kelleher & O'Sullivan,
//    "Generating all partitions: a comparison of two encodings", 2009),
//    reference modules/partitions/integer_partitions.cu:10-47;
//  - filter: at most N parts (integer_partitions.cu:108-114);
//  - compression: (part, multiplicity) pairs by ascending part, then stably
//    ordered by ascending multiplicity (integer_partitions.cu:64-77, :117-137);
//  - sector ordering: the order of the requested dL list (:162-171);
//  - dL = 0 yields the single partition {0} whose polynomial is p_0 = N.
#pragma once
#include <cstdint>
#include <vector>

namespace lemc {

struct PartPair {
  int part;
  int mult;
};

struct BasisRow {
  int dL;
  int sector_index;   // index into the requested sector list
  int sector_size;    // number of rows of this sector
  std::vector<PartPair> pairs;  // compressed, reference order
};

// All partitions of n as ascending sequences, in generation order.
inline std::vector<std::vector<int>> partitions_ascending(int n) {
  std::vector<std::vector<int>> out;
  if (n < 0) return out;
  std::vector<int> a(n + 2, 0);
  int k = 1;
  int y = n - 1;
  while (k != 0) {
    int x = a[k - 1] + 1;
    k -= 1;
    while (2 * x <= y) {
      a[k] = x;
      y -= x;
      k += 1;
    }
    int l = k + 1;
    while (x <= y) {
      a[k] = x;
      a[l] = y;
      out.emplace_back(a.begin(), a.begin() + k + 2);
      x += 1;
      y -= 1;
    }
    a[k] = x + y;
    y = x + y - 1;
    out.emplace_back(a.begin(), a.begin() + k + 1);
  }
  return out;
}

// Compress an ascending partition into (part, multiplicity) pairs, ordered by
// ascending multiplicity with ties kept in ascending part order.
inline std::vector<PartPair> compress_partition(const std::vector<int>& p) {
  std::vector<PartPair> v;
  for (size_t i = 0; i < p.size();) {
    size_t j = i;
    while (j < p.size() && p[j] == p[i]) ++j;
    v.push_back({p[i], int(j - i)});
    i = j;
  }
  // stable insertion sort on multiplicity (equivalent to a stable bubble sort)
  for (size_t i = 1; i < v.size(); ++i) {
    PartPair t = v[i];
    size_t j = i;
    while (j > 0 && v[j - 1].mult > t.mult) {
      v[j] = v[j - 1];
      --j;
    }
    v[j] = t;
  }
  return v;
}

struct Basis {
  std::vector<int> sectors;       // requested dL list
  std::vector<int> sector_dim;    // rows per sector
  std::vector<int> sector_first;  // first row of each sector
  std::vector<BasisRow> rows;
  int max_degree = 0;             // largest part over all rows
  int longest = 0;                // longest compressed partition
};

inline Basis build_basis(int particles, const std::vector<int>& sectors) {
  Basis b;
  b.sectors = sectors;
  for (size_t s = 0; s < sectors.size(); ++s) {
    const int n = sectors[s];
    b.sector_first.push_back(int(b.rows.size()));
    int dim = 0;
    for (const auto& p : partitions_ascending(n)) {
      if (int(p.size()) > particles) continue;
      BasisRow r;
      r.dL = n;
      r.sector_index = int(s);
      r.pairs = compress_partition(p);
      for (const auto& pp : r.pairs)
        if (pp.part > b.max_degree) b.max_degree = pp.part;
      if (int(r.pairs.size()) > b.longest) b.longest = int(r.pairs.size());
      b.rows.push_back(r);
      ++dim;
    }
    b.sector_dim.push_back(dim);
    for (int i = b.sector_first.back(); i < int(b.rows.size()); ++i)
      b.rows[i].sector_size = dim;
  }
  return b;
}

}  // namespace lemc
