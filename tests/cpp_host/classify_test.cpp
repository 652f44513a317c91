// Host check of the bit-sliced classifier: every byte value at every one of
// the 32 positions of a group, against a plain per-byte classification.
#include "classify.cuh"

#include <cstdio>

using namespace gpjb;

static void ref(const unsigned char *b, GroupClasses &g) {
  g = GroupClasses{0, 0, 0, 0, 0, 0};
  for (int j = 0; j < 32; ++j) {
    const unsigned c = b[j];
    const uint32_t bit = 1u << j;
    if (c == '\\') g.bs |= bit;
    if (c == '"') g.qt |= bit;
    if (c == '\n') g.nl |= bit;
    if (c == '{' || c == '[') g.op |= bit;
    if (c == '}' || c == ']') g.cl |= bit;
    if (c == ':' || c == ',') g.sp |= bit;
  }
}

static int check(const unsigned char *b) {
  uint32_t r[8];
  for (int m = 0; m < 8; ++m)
    r[m] = uint32_t(b[4 * m]) | uint32_t(b[4 * m + 1]) << 8 | uint32_t(b[4 * m + 2]) << 16 |
           uint32_t(b[4 * m + 3]) << 24;
  GroupClasses want, got = classify32(r);
  ref(b, want);
  return want.bs != got.bs || want.qt != got.qt || want.nl != got.nl || want.op != got.op ||
         want.cl != got.cl || want.sp != got.sp;
}

int main() {
  unsigned char b[32];
  int bad = 0;
  // every value at every position, the other positions holding a rotating filler
  for (int pos = 0; pos < 32; ++pos)
    for (int v = 0; v < 256; ++v) {
      for (int j = 0; j < 32; ++j) b[j] = (unsigned char)(v + 37 * j + pos);
      b[pos] = (unsigned char)v;
      bad += check(b);
    }
  // random groups
  unsigned s = 12345u;
  for (int t = 0; t < 200000; ++t) {
    for (int j = 0; j < 32; ++j) {
      s = s * 1103515245u + 12345u;
      b[j] = (unsigned char)(s >> 16);
    }
    bad += check(b);
  }
  std::printf("%s %d\n", bad ? "MISMATCH" : "OK", bad);
  return bad ? 1 : 0;
}
