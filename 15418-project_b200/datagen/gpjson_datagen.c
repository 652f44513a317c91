/*
 * Seeded synthetic JSON corpora for benchmarks and tests.
 *
 * Two invented record families stand in for the GpJSON evaluation datasets
 * (no dataset ships with the engine and none is reproduced here):
 *   - "tweets": social-post-like objects, one per line (NDJSON), ~40 keys with
 *     nested "user", "place", "entities" (0..8 hashtag objects) and, in 30%
 *     of records, a nested "retweeted_status" that repeats the structure one
 *     level deeper;
 *   - "products": catalogue-item-like objects with 25 keys, a "categoryPath"
 *     array of 2..6 {id,name} objects and an "offers" array, written as one
 *     top-level JSON array with one element per line.
 * Record sizes are log-normal (mean ~2 KiB, sigma 0.5).  5% of string values
 * carry escaped quotes or backslash runs of length 1..4 (always valid JSON
 * escapes); 2% carry 2..4-byte UTF-8 characters.  Output is compact (no
 * whitespace) and fully determined by the seed.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef struct {
  uint64_t s;
} rng_t;

static uint64_t next_u64(rng_t *r) {
  uint64_t z = (r->s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static double next_unit(rng_t *r) { return (double)(next_u64(r) >> 11) * (1.0 / 9007199254740992.0); }
static uint32_t below(rng_t *r, uint32_t n) { return (uint32_t)(next_unit(r) * n); }
static double normal(rng_t *r) {
  double u1 = next_unit(r), u2 = next_unit(r);
  if (u1 < 1e-300) u1 = 1e-300;
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

typedef struct {
  uint8_t *p;
  uint64_t len, cap;
  int overflow;
} buf_t;

static void put(buf_t *b, const char *s, uint64_t n) {
  if (b->len + n > b->cap) {
    b->overflow = 1;
    return;
  }
  memcpy(b->p + b->len, s, n);
  b->len += n;
}
static void puts_(buf_t *b, const char *s) { put(b, s, strlen(s)); }
static void putc_(buf_t *b, char c) { put(b, &c, 1); }
static void put_u64(buf_t *b, uint64_t v) {
  char tmp[24];
  int i = 23;
  tmp[i] = 0;
  do {
    tmp[--i] = (char)('0' + v % 10);
    v /= 10;
  } while (v);
  puts_(b, tmp + i);
}
static void put_fixed(buf_t *b, double v, int decimals) {
  if (v < 0) {
    putc_(b, '-');
    v = -v;
  }
  uint64_t scale = 1;
  for (int i = 0; i < decimals; ++i) scale *= 10;
  uint64_t x = (uint64_t)(v * (double)scale + 0.5);
  put_u64(b, x / scale);
  putc_(b, '.');
  char tmp[24];
  uint64_t f = x % scale;
  for (int i = decimals - 1; i >= 0; --i) {
    tmp[i] = (char)('0' + f % 10);
    f /= 10;
  }
  put(b, tmp, (uint64_t)decimals);
}

static const char *kSyll[] = {"ka", "lo", "mi", "ne", "ru", "ta", "vo", "si", "de", "pa",
                              "zu", "qi", "ben", "tor", "lux", "fen", "gra", "mon", "dex", "ri"};
static const char *kLang[] = {"en", "es", "fr", "de", "ja", "pt", "nl", "it", "ko", "tr"};
static const char *kCountry[] = {"US", "GB", "FR", "DE", "JP", "BR", "NL", "IT", "KR", "ES"};
static const char *kUtf8[] = {"\xC3\xA9", "\xC3\xBC", "\xE4\xB8\xAD", "\xE2\x82\xAC",
                              "\xF0\x9F\x98\x80", "\xF0\x9F\x8C\x8D"};

static void word(buf_t *b, rng_t *r) {
  const uint32_t k = 1 + below(r, 3);
  for (uint32_t i = 0; i < k; ++i) puts_(b, kSyll[below(r, 20)]);
}

/* A quoted string of roughly `len` bytes of words; 5% carry an escape
 * sequence with a backslash run of 1..4, 2% carry a UTF-8 character. */
static void str_value(buf_t *b, rng_t *r, uint32_t len) {
  putc_(b, '"');
  const uint64_t start = b->len;
  const uint32_t dice = below(r, 100);
  const int esc = dice < 5, utf = dice >= 5 && dice < 7;
  const uint32_t at = len ? below(r, len) : 0;
  int done = 0;
  while (b->len - start < len && !b->overflow) {
    if (!done && b->len - start >= at) {
      done = 1;
      if (esc) {
        const uint32_t run = 1 + below(r, 4);
        for (uint32_t i = 0; i < run; ++i) putc_(b, '\\');
        if (run & 1u) {
          /* odd run: the last backslash escapes the next character */
          static const char *kTail[] = {"\"", "n", "t", "/", "u00e9"};
          puts_(b, kTail[below(r, 5)]);
        }
        continue;
      }
      if (utf) {
        puts_(b, kUtf8[below(r, 6)]);
        continue;
      }
    }
    word(b, r);
    if (b->len - start < len) putc_(b, ' ');
  }
  putc_(b, '"');
}

static void key(buf_t *b, const char *k) {
  putc_(b, '"');
  puts_(b, k);
  puts_(b, "\":");
}

static void user_obj(buf_t *b, rng_t *r, uint32_t desc_len) {
  putc_(b, '{');
  key(b, "id"); put_u64(b, next_u64(r) >> 12); putc_(b, ',');
  key(b, "name"); str_value(b, r, 8 + below(r, 10)); putc_(b, ',');
  key(b, "screen_name"); str_value(b, r, 6 + below(r, 8)); putc_(b, ',');
  key(b, "location"); str_value(b, r, 5 + below(r, 20)); putc_(b, ',');
  key(b, "description"); str_value(b, r, desc_len); putc_(b, ',');
  key(b, "verified"); puts_(b, below(r, 10) ? "false" : "true"); putc_(b, ',');
  key(b, "followers_count"); put_u64(b, below(r, 100000)); putc_(b, ',');
  key(b, "friends_count"); put_u64(b, below(r, 5000)); putc_(b, ',');
  key(b, "statuses_count"); put_u64(b, below(r, 90000)); putc_(b, ',');
  key(b, "created_at"); str_value(b, r, 24); putc_(b, ',');
  key(b, "lang"); putc_(b, '"'); puts_(b, kLang[below(r, 10)]); putc_(b, '"'); putc_(b, ',');
  key(b, "profile_color"); str_value(b, r, 6);
  putc_(b, '}');
}

static void hashtags(buf_t *b, rng_t *r) {
  const uint32_t k = below(r, 9); /* 0..8 */
  putc_(b, '[');
  for (uint32_t i = 0; i < k; ++i) {
    if (i) putc_(b, ',');
    putc_(b, '{');
    key(b, "text"); str_value(b, r, 4 + below(r, 12)); putc_(b, ',');
    key(b, "indices"); putc_(b, '[');
    const uint32_t a = below(r, 120);
    put_u64(b, a); putc_(b, ','); put_u64(b, a + 2 + below(r, 14));
    puts_(b, "]}");
  }
  putc_(b, ']');
}

static void place_obj(buf_t *b, rng_t *r, int deep) {
  if (below(r, 4) == 0) {
    puts_(b, "null");
    return;
  }
  putc_(b, '{');
  key(b, "id"); str_value(b, r, 16); putc_(b, ',');
  key(b, "place_type"); puts_(b, "\"city\",");
  key(b, "full_name"); str_value(b, r, 10 + below(r, 12)); putc_(b, ',');
  key(b, "country_code"); putc_(b, '"'); puts_(b, kCountry[below(r, 10)]); puts_(b, "\",");
  key(b, "bounding_box"); putc_(b, '{');
  key(b, "type"); puts_(b, "\"Polygon\","); key(b, "coordinates");
  puts_(b, deep ? "[[[" : "[[");
  for (int i = 0; i < 4; ++i) {
    if (i) putc_(b, ',');
    putc_(b, '[');
    put_fixed(b, -180.0 + 360.0 * next_unit(r), 6); putc_(b, ',');
    put_fixed(b, -90.0 + 180.0 * next_unit(r), 6);
    putc_(b, ']');
  }
  puts_(b, deep ? "]]]}" : "]]}");
  putc_(b, '}');
}

static void entities(buf_t *b, rng_t *r) {
  putc_(b, '{');
  key(b, "hashtags"); hashtags(b, r); putc_(b, ',');
  key(b, "urls"); putc_(b, '[');
  const uint32_t u = below(r, 3);
  for (uint32_t i = 0; i < u; ++i) {
    if (i) putc_(b, ',');
    putc_(b, '{'); key(b, "url"); str_value(b, r, 23); putc_(b, ',');
    key(b, "indices"); puts_(b, "[0,23]}");
  }
  puts_(b, "],");
  key(b, "symbols"); puts_(b, "[]");
  putc_(b, '}');
}

/* The body of one post; `nest` > 0 adds a retweeted_status one level down. */
static void post(buf_t *b, rng_t *r, uint32_t text_len, int nest, int deep) {
  putc_(b, '{');
  key(b, "created_at"); str_value(b, r, 30); putc_(b, ',');
  key(b, "id"); put_u64(b, next_u64(r) >> 4); putc_(b, ',');
  key(b, "id_str"); putc_(b, '"'); put_u64(b, next_u64(r) >> 4); puts_(b, "\",");
  key(b, "text"); str_value(b, r, text_len); putc_(b, ',');
  key(b, "source"); str_value(b, r, 20 + below(r, 40)); putc_(b, ',');
  key(b, "truncated"); puts_(b, "false,");
  key(b, "in_reply_to_status_id"); if (below(r, 5)) puts_(b, "null"); else put_u64(b, next_u64(r) >> 4); putc_(b, ',');
  key(b, "in_reply_to_user_id"); puts_(b, "null,");
  key(b, "user"); user_obj(b, r, 20 + below(r, 100)); putc_(b, ',');
  key(b, "geo"); puts_(b, "null,");
  key(b, "coordinates");
  if (below(r, 3) == 0) {
    putc_(b, '{'); key(b, "type"); puts_(b, "\"Point\","); key(b, "coordinates"); putc_(b, '[');
    put_fixed(b, -180.0 + 360.0 * next_unit(r), 8); putc_(b, ',');
    put_fixed(b, -90.0 + 180.0 * next_unit(r), 8); puts_(b, "]}");
  } else {
    puts_(b, "null");
  }
  putc_(b, ',');
  key(b, "place"); place_obj(b, r, deep); putc_(b, ',');
  key(b, "is_quote_status"); puts_(b, "false,");
  key(b, "quote_count"); put_u64(b, below(r, 100)); putc_(b, ',');
  key(b, "reply_count"); put_u64(b, below(r, 100)); putc_(b, ',');
  key(b, "retweet_count"); put_u64(b, below(r, 1000)); putc_(b, ',');
  key(b, "favorite_count"); put_u64(b, below(r, 5000)); putc_(b, ',');
  key(b, "entities"); entities(b, r); putc_(b, ',');
  key(b, "favorited"); puts_(b, "false,");
  key(b, "retweeted"); puts_(b, "false,");
  key(b, "score"); put_fixed(b, 100.0 * next_unit(r) - 50.0, 3); putc_(b, ',');
  if (nest > 0) {
    key(b, "retweeted_status");
    post(b, r, text_len / 2 + 10, nest - 1, deep);
    putc_(b, ',');
  }
  key(b, "filter_level"); puts_(b, "\"low\",");
  key(b, "lang"); putc_(b, '"'); puts_(b, kLang[below(r, 10)]); puts_(b, "\",");
  key(b, "timestamp_ms"); putc_(b, '"'); put_u64(b, 1500000000000ull + below(r, 1000000000)); putc_(b, '"');
  putc_(b, '}');
}

static uint32_t lognormal_size(rng_t *r, double mean, double sigma) {
  const double mu = log(mean) - 0.5 * sigma * sigma;
  double v = exp(mu + sigma * normal(r));
  if (v < 256.0) v = 256.0;
  if (v > 65536.0) v = 65536.0;
  return (uint32_t)v;
}

/* NDJSON of post records until target_bytes is reached.  deep != 0 nests
 * place coordinates one level deeper (depth up to 8 instead of 6).  Returns
 * the bytes written (the output ends with '\n'). */
uint64_t gdg_tweets(uint64_t seed, uint64_t target_bytes, int deep, uint8_t *out,
                    uint64_t cap) {
  rng_t r = {seed * 0x2545F4914F6CDD1Dull + 1};
  buf_t b = {out, 0, cap, 0};
  while (b.len < target_bytes) {
    const uint32_t size = lognormal_size(&r, 2048.0, 0.5);
    const int nest = below(&r, 10) < 3;
    /* the skeleton without text is ~1.65 KiB (~2.7 KiB with a retweet) */
    const uint32_t skel = nest ? 2700u : 1650u;
    const uint32_t text = size > skel + 16u ? size - skel : 16u;
    const uint64_t before = b.len;
    post(&b, &r, text, nest, deep);
    putc_(&b, '\n');
    if (b.overflow) {
      b.len = before;
      break;
    }
  }
  return b.len;
}

static void product(buf_t *b, rng_t *r, uint32_t desc_len, uint64_t sku) {
  putc_(b, '{');
  key(b, "sku"); put_u64(b, sku); putc_(b, ',');
  key(b, "productId"); put_u64(b, 1000000 + sku * 7); putc_(b, ',');
  key(b, "name"); str_value(b, r, 20 + below(r, 40)); putc_(b, ',');
  key(b, "type"); puts_(b, "\"HardGood\",");
  key(b, "regularPrice"); put_fixed(b, 5.0 + 2000.0 * next_unit(r), 2); putc_(b, ',');
  key(b, "salePrice"); put_fixed(b, 5.0 + 2000.0 * next_unit(r), 2); putc_(b, ',');
  key(b, "onSale"); puts_(b, below(r, 2) ? "true," : "false,");
  key(b, "url"); str_value(b, r, 60); putc_(b, ',');
  key(b, "categoryPath"); putc_(b, '[');
  const uint32_t cats = 2 + below(r, 5); /* 2..6 */
  for (uint32_t i = 0; i < cats; ++i) {
    if (i) putc_(b, ',');
    putc_(b, '{');
    key(b, "id"); puts_(b, "\"cat"); put_u64(b, 10000 + below(r, 90000)); puts_(b, "\",");
    key(b, "name"); str_value(b, r, 6 + below(r, 14));
    putc_(b, '}');
  }
  puts_(b, "],");
  key(b, "customerReviewCount"); put_u64(b, below(r, 4000)); putc_(b, ',');
  key(b, "customerReviewAverage"); put_fixed(b, 1.0 + 4.0 * next_unit(r), 1); putc_(b, ',');
  key(b, "freeShipping"); puts_(b, below(r, 2) ? "true," : "false,");
  key(b, "inStoreAvailability"); puts_(b, "true,");
  key(b, "onlineAvailability"); puts_(b, "true,");
  key(b, "manufacturer"); str_value(b, r, 6 + below(r, 10)); putc_(b, ',');
  key(b, "modelNumber"); str_value(b, r, 10); putc_(b, ',');
  key(b, "image"); str_value(b, r, 70); putc_(b, ',');
  key(b, "thumbnailImage"); str_value(b, r, 70); putc_(b, ',');
  key(b, "shortDescription"); str_value(b, r, 40 + below(r, 80)); putc_(b, ',');
  key(b, "longDescription"); str_value(b, r, desc_len); putc_(b, ',');
  key(b, "class"); str_value(b, r, 12); putc_(b, ',');
  key(b, "subclass"); str_value(b, r, 12); putc_(b, ',');
  key(b, "department"); str_value(b, r, 10); putc_(b, ',');
  key(b, "offers"); putc_(b, '[');
  const uint32_t offers = below(r, 3);
  for (uint32_t i = 0; i < offers; ++i) {
    if (i) putc_(b, ',');
    putc_(b, '{');
    key(b, "id"); put_u64(b, below(r, 100000)); putc_(b, ',');
    key(b, "text"); str_value(b, r, 20 + below(r, 30)); putc_(b, ',');
    key(b, "type"); puts_(b, "[\"deal\",\"instore\"],");
    key(b, "startDate"); str_value(b, r, 10);
    putc_(b, '}');
  }
  puts_(b, "],");
  key(b, "shipping"); putc_(b, '{');
  key(b, "ground"); put_fixed(b, 20.0 * next_unit(r), 2); putc_(b, ',');
  key(b, "nextBusinessDay"); put_fixed(b, 40.0 * next_unit(r), 2);
  puts_(b, "}}");
}

/* One top-level array of product records, one element per line:
 * "[\n" elem ",\n" elem ... "\n]\n".  Returns the bytes written. */
uint64_t gdg_products(uint64_t seed, uint64_t target_bytes, uint8_t *out, uint64_t cap) {
  rng_t r = {seed * 0x9E3779B97F4A7C15ull + 7};
  buf_t b = {out, 0, cap, 0};
  puts_(&b, "[\n");
  uint64_t sku = 0;
  const uint64_t tail = 3; /* "\n]\n" */
  while (b.len + tail < target_bytes) {
    const uint32_t size = lognormal_size(&r, 2048.0, 0.5);
    const uint32_t desc = size > 1100u ? size - 1000u : 100u;
    const uint64_t before = b.len;
    if (sku) puts_(&b, ",\n");
    product(&b, &r, desc, ++sku);
    if (b.overflow || b.len + tail > cap) {
      b.len = before;
      b.overflow = 0;
      break;
    }
  }
  puts_(&b, "\n]\n");
  return b.len;
}
