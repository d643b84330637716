// Seed index cache of a resident database (LRU under a byte budget).
#include "common.cuh"
#include "index_cache.h"

namespace drg {

SeedIndex::~SeedIndex() {
  // cudaFree waits for the device, so no search still reads the arrays
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  cudaFree(keys);
  cudaFree(keys32);
  cudaFree(vals);
  if (cur != device) cudaSetDevice(cur);
}

void IndexCache::evict_to(uint64_t limit, std::list<std::shared_ptr<SeedIndex>>* out) {
  while (bytes_ > limit && !lru_.empty()) {
    bytes_ -= lru_.back()->bytes;
    out->splice(out->end(), lru_, std::prev(lru_.end()));  // freed when the last search holding it lets go
    ++evictions_;
  }
}

void IndexCache::set_budget(uint64_t bytes) {
  std::list<std::shared_ptr<SeedIndex>> dropped;  // released after the lock
  std::lock_guard<std::mutex> g(mu_);
  budget_ = bytes;
  evict_to(budget_, &dropped);
}

uint64_t IndexCache::budget() const {
  std::lock_guard<std::mutex> g(mu_);
  return budget_;
}

std::shared_ptr<SeedIndex> IndexCache::find(const std::string& key) {
  std::lock_guard<std::mutex> g(mu_);
  for (auto it = lru_.begin(); it != lru_.end(); ++it) {
    if ((*it)->key == key) {
      lru_.splice(lru_.begin(), lru_, it);
      ++hits_;
      return lru_.front();
    }
  }
  ++misses_;
  return nullptr;
}

std::shared_ptr<SeedIndex> IndexCache::insert(const std::string& key, const uint64_t* keys, const uint32_t* keys32,
                                              const uint32_t* vals, uint64_t n, cudaStream_t stream) {
  const uint64_t key_bytes = keys ? sizeof(uint64_t) : sizeof(uint32_t);
  const uint64_t bytes = n * (key_bytes + sizeof(uint32_t));
  {
    std::lock_guard<std::mutex> g(mu_);
    if (bytes > budget_ || bytes == 0) return nullptr;
    for (auto& e : lru_)
      if (e->key == key) return e;  // another context built it meanwhile
  }
  auto e = std::make_shared<SeedIndex>();
  e->key = key;
  e->device = device_;
  e->n = n;
  e->bytes = bytes;
  void** kp = keys ? reinterpret_cast<void**>(&e->keys) : reinterpret_cast<void**>(&e->keys32);
  if (cudaMalloc(kp, n * key_bytes) != cudaSuccess || cudaMalloc(&e->vals, n * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();  // out of memory: the search goes on without caching
    return nullptr;
  }
  DRG_CUDA(cudaMemcpyAsync(*kp, keys ? static_cast<const void*>(keys) : static_cast<const void*>(keys32),
                           n * key_bytes, cudaMemcpyDeviceToDevice, stream));
  DRG_CUDA(cudaMemcpyAsync(e->vals, vals, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream));
  DRG_CUDA(cudaStreamSynchronize(stream));  // other contexts read it from their own streams
  std::list<std::shared_ptr<SeedIndex>> dropped;  // released after the lock (declared first)
  std::lock_guard<std::mutex> g(mu_);
  for (auto& x : lru_)
    if (x->key == key) return x;
  lru_.push_front(e);
  bytes_ += bytes;
  evict_to(budget_, &dropped);
  return e;
}

IndexCache::Stats IndexCache::stats() const {
  std::lock_guard<std::mutex> g(mu_);
  return Stats{(uint64_t)lru_.size(), bytes_, hits_, misses_, evictions_};
}

}  // namespace drg
