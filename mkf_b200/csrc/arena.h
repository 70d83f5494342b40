// arena.h - sub-allocator of one memory range for the request loop's device-memory budget:
// 256-byte-aligned blocks, best fit, neighbouring free blocks merged on release. Host code only (it
// never touches the memory it hands out), not thread-safe: the server's worker thread owns it.
#pragma once
#include <cstddef>
#include <iterator>
#include <map>

namespace mkf {

class Arena
{
 public:
   // Manage [base, base + bytes); the caller owns the memory.
   void init(void *base, size_t bytes)
   {
      base_ = static_cast<char *>(base);
      size_ = bytes;
      used_ = 0;
      free_.clear();
      if (bytes) { free_[0] = bytes; }
   }
   static size_t round(size_t n) { return (n + 255) & ~(size_t)255; }
   // A block of at least n bytes (the smallest free block that fits), or nullptr.
   void *alloc(size_t n)
   {
      n = round(n);
      if (n == 0) { n = 256; }
      auto best = free_.end();
      for (auto it = free_.begin(); it != free_.end(); ++it) {
         if (it->second >= n && (best == free_.end() || it->second < best->second)) { best = it; }
      }
      if (best == free_.end()) { return nullptr; }
      const size_t off = best->first, sz = best->second;
      free_.erase(best);
      if (sz > n) { free_[off + n] = sz - n; }
      used_ += n;
      return base_ + off;
   }
   // Give back a block alloc(n) returned (same n).
   void release(void *p, size_t n)
   {
      if (!p) { return; }
      n = round(n);
      if (n == 0) { n = 256; }
      const size_t off = (size_t)(static_cast<char *>(p) - base_);
      used_ -= n;
      auto next = free_.lower_bound(off);
      if (next != free_.end() && off + n == next->first) {
         n += next->second;
         next = free_.erase(next);
      }
      if (next != free_.begin()) {
         auto prev = std::prev(next);
         if (prev->first + prev->second == off) {
            prev->second += n;
            return;
         }
      }
      free_[off] = n;
   }
   size_t size() const { return size_; }
   size_t used() const { return used_; }
   size_t freeBlocks() const { return free_.size(); }
   char *base() const { return base_; }

 private:
   char *base_ = nullptr;
   size_t size_ = 0, used_ = 0;
   std::map<size_t, size_t> free_;  // offset -> bytes
};

}  // namespace mkf
