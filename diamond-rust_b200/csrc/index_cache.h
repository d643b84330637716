// Seed index cache of a resident database.
//
// A search enumerates and sorts the reference seeds of every index chunk it
// covers (the reference rebuilds them on every run, search.rs:104-126).  For
// a database that stays in HBM across searches the sorted seeds of one
// (shape set, reduction, complexity cut, chunk) are a property of the
// database, so they can stay resident too: this cache keeps them, shared by
// every context that searches the database, and evicts the least recently
// used when the held bytes pass the budget.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <list>
#include <memory>
#include <mutex>
#include <string>

namespace drg {

// Sorted reference seeds of one index chunk under one seed configuration:
// keys[0, n) ascending (or keys32, when the seed key fits 32 bits), vals
// their letter indices.
struct SeedIndex {
  std::string key;
  int device = 0;
  uint64_t* keys = nullptr;
  uint32_t* keys32 = nullptr;
  uint32_t* vals = nullptr;
  uint64_t n = 0;
  uint64_t bytes = 0;
  SeedIndex() = default;
  SeedIndex(const SeedIndex&) = delete;
  SeedIndex& operator=(const SeedIndex&) = delete;
  ~SeedIndex();
};

class IndexCache {
 public:
  explicit IndexCache(int device) : device_(device) {}
  // Sets the budget and evicts down to it; 0 drops every entry.
  void set_budget(uint64_t bytes);
  uint64_t budget() const;
  // The entry under `key`, most recently used from now on; null on a miss.
  std::shared_ptr<SeedIndex> find(const std::string& key);
  // Copies n sorted seeds (device arrays, ready once `stream` reaches this
  // point; 64-bit keys or 32-bit keys32, the other null) into a new entry;
  // returns null when the budget cannot hold it.
  std::shared_ptr<SeedIndex> insert(const std::string& key, const uint64_t* keys, const uint32_t* keys32,
                                    const uint32_t* vals, uint64_t n, cudaStream_t stream);
  struct Stats {
    uint64_t entries, bytes, hits, misses, evictions;
  };
  Stats stats() const;

 private:
  // Moves entries past `limit` bytes into `out` (caller holds mu_ and frees
  // them after unlocking).
  void evict_to(uint64_t limit, std::list<std::shared_ptr<SeedIndex>>* out);
  int device_;
  mutable std::mutex mu_;
  uint64_t budget_ = 0, bytes_ = 0, hits_ = 0, misses_ = 0, evictions_ = 0;
  std::list<std::shared_ptr<SeedIndex>> lru_;  // front: most recently used
};

}  // namespace drg
