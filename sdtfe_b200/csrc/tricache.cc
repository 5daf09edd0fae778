// tricache.cc - the triangulation cache behind triangulate().
//
// Host Qhull dominates a map's end-to-end time (seconds to minutes against
// milliseconds of GPU work), and callers often triangulate the same particles
// again: one map per projection axis or resolution, a density and a grid of
// the same cutout, a serving process that reloads a cutout.  triangulate()
// therefore keeps its recent results, keyed by the exact input: the particle
// count, the options string and every coordinate (x, y, z of each row; column
// 3 does not take part in the triangulation).  A call whose input matches an
// entry bit for bit gets a copy of that entry's tetra_data without running
// the backend; Qhull is deterministic for a given input order and options, so
// the copy is exactly what it would have returned.  Entries hold a copy of
// the coordinates (compared in full on a hash match) and the rows; the least
// recently used ones are dropped beyond the byte limit.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <list>
#include <mutex>
#include <string>
#include <vector>

#include "sdtfe_b200.h"

namespace sdtfe {
namespace {

struct Entry {
  uint64_t hash;
  int n;
  std::string options;
  std::vector<double> xyz;  // 3 per particle
  std::vector<int> tetra;   // 8 per tet
  size_t bytes() const { return xyz.size() * sizeof(double) + tetra.size() * sizeof(int); }
};

struct Cache {
  std::mutex mu;
  bool configured = false;
  size_t limit = 0, bytes = 0;
  unsigned long long hits = 0, misses = 0;
  std::list<Entry> lru;  // most recent first
};

Cache& cache() {
  static Cache c;
  return c;
}

// with c.mu held: the limit from SDTFE_TRI_CACHE_MB (default 1024 MB) until set
void configure(Cache& c) {
  if (c.configured) return;
  c.configured = true;
  const char* e = getenv("SDTFE_TRI_CACHE_MB");
  c.limit = (size_t)(e ? strtoull(e, nullptr, 10) : 1024ull) << 20;
}

void trim(Cache& c) {
  while (c.bytes > c.limit && !c.lru.empty()) {
    c.bytes -= c.lru.back().bytes();
    c.lru.pop_back();
  }
}

// FNV-1a over the coordinates' bytes, the count and the options
uint64_t key_hash(const double* xyz4, int n, const char* options) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](const void* p, size_t len) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < len; ++i) {
      h ^= b[i];
      h *= 1099511628211ull;
    }
  };
  mix(&n, sizeof(n));
  if (options) mix(options, strlen(options));
  for (int i = 0; i < n; ++i) mix(xyz4 + 4 * (size_t)i, 3 * sizeof(double));
  return h;
}

bool same_input(const Entry& e, uint64_t h, const double* xyz4, int n, const char* options) {
  if (e.hash != h || e.n != n || e.options != (options ? options : "")) return false;
  for (int i = 0; i < n; ++i)
    if (memcmp(&e.xyz[3 * (size_t)i], xyz4 + 4 * (size_t)i, 3 * sizeof(double)) != 0) return false;
  return true;
}

}  // namespace

int* tri_cache_lookup(const double* xyz4, int n, const char* options, size_t* n_tetra) {
  Cache& c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  configure(c);
  if (c.limit == 0 || n <= 0) return nullptr;
  const uint64_t h = key_hash(xyz4, n, options);
  for (auto it = c.lru.begin(); it != c.lru.end(); ++it) {
    if (!same_input(*it, h, xyz4, n, options)) continue;
    const size_t nt = it->tetra.size() / 8;
    int* out = static_cast<int*>(malloc(sizeof(int) * 8 * (nt ? nt : 1)));
    if (!out) return nullptr;
    memcpy(out, it->tetra.data(), sizeof(int) * 8 * nt);
    *n_tetra = nt;
    c.lru.splice(c.lru.begin(), c.lru, it);
    ++c.hits;
    return out;
  }
  ++c.misses;
  return nullptr;
}

void tri_cache_insert(const double* xyz4, int n, const char* options, const int* tetra,
                      size_t n_tetra) {
  Cache& c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  configure(c);
  const size_t need = 3 * (size_t)n * sizeof(double) + 8 * n_tetra * sizeof(int);
  if (c.limit == 0 || n <= 0 || need > c.limit) return;
  Entry e;
  e.hash = key_hash(xyz4, n, options);
  e.n = n;
  e.options = options ? options : "";
  try {
    e.xyz.resize(3 * (size_t)n);
    for (int i = 0; i < n; ++i) memcpy(&e.xyz[3 * (size_t)i], xyz4 + 4 * (size_t)i, 3 * sizeof(double));
    e.tetra.assign(tetra, tetra + 8 * n_tetra);
    c.lru.push_front(std::move(e));
  } catch (...) {
    return;  // no room on the host: the result is simply not kept
  }
  c.bytes += c.lru.front().bytes();
  trim(c);
}

}  // namespace sdtfe

extern "C" {

void dtfe_set_triangulation_cache(size_t max_bytes) {
  sdtfe::Cache& c = sdtfe::cache();
  std::lock_guard<std::mutex> lk(c.mu);
  c.configured = true;
  c.limit = max_bytes;
  sdtfe::trim(c);
}

void dtfe_triangulation_cache_stats(unsigned long long* hits, unsigned long long* misses,
                                    size_t* entries, size_t* bytes) {
  sdtfe::Cache& c = sdtfe::cache();
  std::lock_guard<std::mutex> lk(c.mu);
  if (hits) *hits = c.hits;
  if (misses) *misses = c.misses;
  if (entries) *entries = c.lru.size();
  if (bytes) *bytes = c.bytes;
}

}  // extern "C"
