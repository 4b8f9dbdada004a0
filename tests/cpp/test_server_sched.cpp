// Host test of the serving loop's admission and step-forming rules
// (curplsh_b200/csrc/server_sched.h); no GPU involved.
#include <cassert>
#include <cstdio>
#include <deque>
#include <map>
#include <vector>

#include "server_sched.h"

using namespace curplsh_b200;

#define CHECK(c)                                                  \
  do {                                                            \
    if (!(c)) {                                                   \
      std::printf("check failed: %s (line %d)\n", #c, __LINE__);  \
      return 1;                                                   \
    }                                                             \
  } while (0)

int main() {
  // ---- arena: first fit, 256-byte granules, coalescing on release
  Arena a;
  a.reset(4096);
  size_t o1 = 0, o2 = 0, o3 = 0, o4 = 0;
  CHECK(a.alloc(100, &o1) && o1 == 0);       // rounds to 256
  CHECK(a.alloc(1000, &o2) && o2 == 256);    // rounds to 1024
  CHECK(a.alloc(512, &o3) && o3 == 1280);
  CHECK(a.in_use() == 256 + 1024 + 512);
  CHECK(!a.alloc(4096, &o4));                // does not fit
  a.release(o2, 1000);                        // hole [256, 1280)
  CHECK(a.alloc(900, &o4) && o4 == 256);      // first fit reuses the hole
  a.release(o4, 900);
  a.release(o1, 100);
  a.release(o3, 512);
  CHECK(a.in_use() == 0 && a.free_blocks() == 1 && a.largest_free() == 4096);  // fully coalesced

  // ---- step forming: first come first served under the query cap
  std::map<int64_t, int64_t> num = {{1, 100}, {2, 300}, {3, 50}, {4, 700}, {5, 10}};
  auto num_of = [&](int64_t t) { return num[t]; };
  std::deque<int64_t> pending = {1, 2, 3, 4, 5};
  std::vector<int64_t> take = take_step(pending, 500, num_of);
  CHECK((take == std::vector<int64_t>{1, 2, 3}));  // 450; adding 700 would exceed 500
  std::deque<int64_t> big = {4, 1};
  take = take_step(big, 500, num_of);
  CHECK((take == std::vector<int64_t>{4}));         // the head is always taken

  // ---- admission by memory: halve (keeping arrival order) until it fits
  Arena m;
  m.reset(64 * 1024);
  auto bytes_for = [&](const std::vector<int64_t>& tk, size_t* b) -> int {
    size_t s = 0;
    for (int64_t t : tk) s += (size_t)num[t] * 64;  // 64 bytes per query
    *b = s;
    return 0;
  };
  std::vector<int64_t> tk = {1, 2, 3};  // 450 queries -> 28,800 bytes
  size_t off = 0, bytes = 0;
  CHECK(admit_step(tk, m, &off, &bytes, bytes_for) == 1 && tk.size() == 3 && bytes == 28800);
  size_t off_b = 0, bytes_b = 0;           // 28,928 bytes in use, 36,608 free
  num[4] = 570;                             // {4, 5}: 36,480 + 640 bytes do not fit
  std::vector<int64_t> tk2 = {4, 5};
  CHECK(admit_step(tk2, m, &off_b, &bytes_b, bytes_for) == 1);
  CHECK((tk2 == std::vector<int64_t>{4}) && bytes_b == 36480);  // halved, head kept
  std::vector<int64_t> tk3 = {5};           // the arena is full now: wait
  size_t off_c = 0, bytes_c = 0;
  CHECK(admit_step(tk3, m, &off_c, &bytes_c, bytes_for) == 0);
  m.release(off, bytes);                    // a running step finishes
  CHECK(admit_step(tk3, m, &off_c, &bytes_c, bytes_for) == 1 && off_c == 0);
  num[2] = 2000;                            // 128,000 bytes: never fits the 64 KiB arena
  std::vector<int64_t> tk4 = {2};
  size_t off_d = 0, bytes_d = 0;
  CHECK(admit_step(tk4, m, &off_d, &bytes_d, bytes_for) == 0);
  auto failing = [&](const std::vector<int64_t>&, size_t*) -> int { return 7; };
  std::vector<int64_t> tk5 = {1};
  CHECK(admit_step(tk5, m, &off_d, &bytes_d, failing) < 0);     // a planning error is reported
  std::printf("server sched ok\n");
  return 0;
}
