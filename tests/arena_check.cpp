// Randomised check of the request loop's device-memory sub-allocator (mkf_b200/csrc/arena.h)
// against a model of the live blocks: alignment and bounds, no overlap, the used byte count, best
// fit (a block comes from the smallest free gap that holds it), a failure only when no gap holds
// the request, and full merging of free neighbours. Exit status 0 when every check holds.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
#include "arena.h"

struct Block { size_t off, size; };

static int fail(const char *what, long step)
{
   std::printf("arena check failed at step %ld: %s\n", step, what);
   return 1;
}

// Free gaps between the live blocks (the arena must hold exactly these as merged free blocks).
static std::vector<Block> gaps(std::vector<Block> live, size_t total)
{
   std::sort(live.begin(), live.end(), [](const Block &a, const Block &b) { return a.off < b.off; });
   std::vector<Block> g;
   size_t at = 0;
   for (const Block &b : live) {
      if (b.off > at) { g.push_back({at, b.off - at}); }
      at = b.off + b.size;
   }
   if (total > at) { g.push_back({at, total - at}); }
   return g;
}

int main()
{
   const size_t total = (size_t)1 << 20;
   std::vector<char> mem(total);
   mkf::Arena A;
   A.init(mem.data(), total);
   std::mt19937_64 rng(12345);
   std::vector<Block> live;
   size_t used = 0;
   for (long step = 0; step < 200000; ++step) {
      const bool doAlloc = live.empty() || (rng() % 100) < 55;
      if (doAlloc) {
         const size_t n = 1 + rng() % (48 * 1024);
         const size_t r = mkf::Arena::round(n);
         const std::vector<Block> g = gaps(live, total);
         size_t bestSize = 0;
         for (const Block &b : g) {
            if (b.size >= r && (bestSize == 0 || b.size < bestSize)) { bestSize = b.size; }
         }
         char *p = static_cast<char *>(A.alloc(n));
         if (!p) {
            if (bestSize) { return fail("alloc failed although a free gap holds the request", step); }
            continue;
         }
         if (!bestSize) { return fail("alloc succeeded with no free gap large enough", step); }
         const size_t off = (size_t)(p - mem.data());
         if (off % 256 || off + r > total) { return fail("misaligned or out of range", step); }
         bool inBest = false;
         for (const Block &b : g) {
            if (off >= b.off && off + r <= b.off + b.size) { inBest = b.size == bestSize; }
         }
         if (!inBest) { return fail("not the best-fitting gap", step); }
         live.push_back({off, r});
         used += r;
      } else {
         const size_t i = rng() % live.size();
         A.release(mem.data() + live[i].off, live[i].size);
         used -= live[i].size;
         live[i] = live.back();
         live.pop_back();
      }
      if (A.used() != used) { return fail("used byte count", step); }
      if (A.freeBlocks() != gaps(live, total).size()) { return fail("free neighbours not merged", step); }
   }
   for (const Block &b : live) { A.release(mem.data() + b.off, b.size); }
   if (A.used() != 0 || A.freeBlocks() != 1) { return fail("not one free block after releasing everything", -1); }
   std::printf("arena check ok\n");
   return 0;
}
