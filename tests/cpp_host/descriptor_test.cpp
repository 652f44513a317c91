// Host check of the look-back descriptor algebra: the packed branch-free
// composition equals the field-wise one, and composition is associative.
#include "descriptor.cuh"

#include <cstdio>

using namespace gpjb;

static unsigned long long state = 88172645463325252ull;
static uint64_t rnd() {
  state ^= state << 13;
  state ^= state >> 7;
  state ^= state << 17;
  return state;
}
static Agg random_agg() {
  Agg a;
  a.p = uint32_t(rnd() & 1u);
  a.d0 = uint32_t(rnd() & 0xFFu);
  a.d1 = uint32_t(rnd() & 0xFFu);
  a.c = (rnd() % 5) == 0 ? 1u : 0u;
  if (a.c) a.d1 = a.d0;
  a.n = rnd() & ((1ull << 36) - 1);
  return a;
}

int main() {
  int bad = 0;
  for (int t = 0; t < 2000000; ++t) {
    const Agg a = random_agg(), b = random_agg(), c = random_agg();
    const uint64_t pa = agg_pack(rnd() & 3u, a), pb = agg_pack(rnd() & 3u, b),
                   pc = agg_pack(rnd() & 3u, c);
    if (desc_combine(pa, pb) != agg_pack(0, agg_combine(a, b))) ++bad;
    if (desc_combine(desc_combine(pa, pb), pc) != desc_combine(pa, desc_combine(pb, pc))) ++bad;
    if (desc_combine(0, pa) != (pa & ~uint64_t(3)) || desc_combine(pa, 0) != (pa & ~uint64_t(3)))
      ++bad;
  }
  std::printf("%s %d\n", bad ? "MISMATCH" : "OK", bad);
  return bad ? 1 : 0;
}
