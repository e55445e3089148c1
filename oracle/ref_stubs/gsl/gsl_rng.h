/* Project-written stand-in for the GNU Scientific Library RNG header, used only
 * to compile the reference CPU engine as a test oracle. GSL is not installed in
 * this image. The reference (simulation engine/src/Replica.cpp:265-290,
 * main.cpp:1156) only needs an mt19937 generator with uniform draws; its seeds
 * come from time(NULL), so its streams are never reproducible anyway.
 *
 * The generator is the published MT19937 of Matsumoto & Nishimura (1998),
 * written out here because the reference's `#define lambda` (definitions.h:35)
 * breaks <random>. This file is test infrastructure: nothing in the product
 * links it. */
#ifndef REMC_ORACLE_STUB_GSL_RNG_H
#define REMC_ORACLE_STUB_GSL_RNG_H

#include <stdint.h>

struct gsl_rng_type { int id; };
struct gsl_rng {
  uint32_t mt[624];
  int index;
  /* fed mode (test harness only): uniforms are served from this queue
   * instead of MT19937, so the reference's own MCSearch can be driven by a
   * counter-based stream shared with the GPU engine. */
  int fed;
  int feed_head;
  int feed_count;
  int feed_underflow;
  double feed[16];
};

static const gsl_rng_type remc_stub_mt19937_type = {19937};
static const gsl_rng_type* gsl_rng_mt19937 = &remc_stub_mt19937_type;

static inline void gsl_rng_set(gsl_rng* r, unsigned long seed) {
  r->mt[0] = (uint32_t)seed;
  for (int i = 1; i < 624; ++i)
    r->mt[i] = 1812433253u * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (uint32_t)i;
  r->index = 624;
}
static inline gsl_rng* gsl_rng_alloc(const gsl_rng_type*) {
  gsl_rng* r = new gsl_rng();
  r->fed = 0;
  r->feed_head = 0;
  r->feed_count = 0;
  r->feed_underflow = 0;
  gsl_rng_set(r, 5489u);
  return r;
}
static inline void gsl_rng_free(gsl_rng* r) { delete r; }
static inline uint32_t remc_stub_mt_next(gsl_rng* r) {
  if (r->index >= 624) {
    for (int i = 0; i < 624; ++i) {
      uint32_t y = (r->mt[i] & 0x80000000u) | (r->mt[(i + 1) % 624] & 0x7fffffffu);
      uint32_t v = r->mt[(i + 397) % 624] ^ (y >> 1);
      if (y & 1u) v ^= 0x9908b0dfu;
      r->mt[i] = v;
    }
    r->index = 0;
  }
  uint32_t y = r->mt[r->index++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}
static inline unsigned long gsl_rng_get(gsl_rng* r) { return (unsigned long)remc_stub_mt_next(r); }
static inline unsigned long gsl_rng_max(const gsl_rng*) { return 0xffffffffUL; }
static inline unsigned long gsl_rng_min(const gsl_rng*) { return 0UL; }
/* uniform on [0,1): 32-bit draw scaled by 2^-32, or the next fed value */
static inline double gsl_rng_uniform(gsl_rng* r) {
  if (r->fed) {
    if (r->feed_count <= 0) { r->feed_underflow++; return 0.5; }
    double u = r->feed[r->feed_head];
    r->feed_head = (r->feed_head + 1) & 15;
    r->feed_count--;
    return u;
  }
  return (double)remc_stub_mt_next(r) / 4294967296.0;
}
static inline void remc_stub_feed(gsl_rng* r, double u) {
  r->fed = 1;
  if (r->feed_count >= 16) return;
  r->feed[(r->feed_head + r->feed_count) & 15] = u;
  r->feed_count++;
}
static inline void remc_stub_feed_clear(gsl_rng* r) {
  r->feed_head = 0;
  r->feed_count = 0;
}
static inline double gsl_rng_uniform_pos(gsl_rng* r) {
  double u;
  do { u = gsl_rng_uniform(r); } while (u == 0.0);
  return u;
}
static inline unsigned long gsl_rng_uniform_int(gsl_rng* r, unsigned long n) {
  return (unsigned long)(gsl_rng_uniform(r) * (double)n);
}

#endif
