// TEST INFRASTRUCTURE: replays "a <n>" / "f <start> <n>" commands from stdin against
// gpq::RangeAlloc (gpupq_b200/csrc/range_alloc.h) and prints each alloc's start or -1,
// and "used <n>" at the end.
#include <cstdio>

#include "range_alloc.h"

int main() {
  unsigned long long size = 0;
  if (scanf("%llu", &size) != 1) return 1;
  gpq::RangeAlloc r;
  r.reset(size);
  char op;
  while (scanf(" %c", &op) == 1) {
    if (op == 'a') {
      unsigned long long n;
      if (scanf("%llu", &n) != 1) return 1;
      uint64_t s = 0;
      if (r.alloc(n, &s)) printf("%llu\n", (unsigned long long)s);
      else printf("-1\n");
    } else {
      unsigned long long s, n;
      if (scanf("%llu %llu", &s, &n) != 2) return 1;
      r.free(s, n);
    }
  }
  printf("used %llu\n", (unsigned long long)r.used());
  return 0;
}
