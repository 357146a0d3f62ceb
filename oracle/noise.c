/* Plain-C restatement of the reference's sequential noise source.
 *
 * TEST INFRASTRUCTURE ONLY: the checker uses it to produce the exact complex noise grids
 * that AVOInversion::simulate draws, so that realisations can be compared value by value
 * ("parity mode").  The product path never links it.
 *
 *   RandomGen::unif01   libs/lib/random.cpp:113-119, constants libs/lib/random.h:12-15
 *                       seed <- 69069*seed + 1 (mod 2^32), u = seed * 2^-32
 *   RandomGen::rnorm01  libs/lib/random.cpp:38-94 (Marsaglia-Bray, Ripley p. 84)
 *   RandomGen::g        libs/lib/random.cpp:97-110
 *   FFTGrid::fillInComplexNoise   src/fftgrid.cpp:997-1055, including its
 *                       flat-index parity test on the x = cnxp-1 plane (:1006)
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

static double unif01(uint32_t* s) {
  *s = 69069u * *s + 1u;
  return (double)(*s) * ((1.0 / (double)(256 * 256 * 256 * 64)) / 4.0);
}

static double gfun(double x) {
  double a = 17.49731196, b = 2.36785163, c = 2.15787544;
  double ax = fabs(x);
  double r = a * exp(-x * x / 2.0);
  if (ax < 1.0) r -= 2.0 * b * (3.0 - x * x) + c * (1.5 - ax);
  else if (ax < 1.5) r -= b * (3.0 - ax) * (3.0 - ax) + c * (1.5 - ax);
  else r -= b * (3.0 - ax) * (3.0 - ax);
  return r;
}

double oracle_rnorm01(uint32_t* s) {
  double u = unif01(s), u1, u2, u3, x, v1, v2, w, c, ss, t;
  if (u < 0.8638) {
    u1 = unif01(s); u2 = unif01(s); u3 = unif01(s);
    x = 2.0 * (u1 + u2 + u3) - 3.0;
  } else if (u < 0.9745) {
    u1 = unif01(s); u2 = unif01(s);
    x = 1.5 * (u1 + u2 - 1.0);
  } else if (u < 0.9973002039) {
    do {
      u1 = unif01(s); u2 = unif01(s);
      x = 6.0 * u1 - 3.0;
    } while (0.358 * u2 > gfun(x));
  } else {
    do {
      do {
        u1 = unif01(s); u2 = unif01(s);
        v1 = 2.0 * u1 - 1.0; v2 = 2.0 * u2 - 1.0;
        w = v1 * v1 + v2 * v2;
      } while (w >= 1.0);
      c = sqrt((9.0 - 2.0 * log(w)) / w);
      ss = c * v1; t = c * v2;
    } while (fabs(ss) <= 3.0 && fabs(t) <= 3.0);
    x = (fabs(ss) > 3.0) ? ss : t;
  }
  return x;
}

/* One complex grid (cnxp*nyp*nzp interleaved re/im floats), state advanced in *s. */
void oracle_fill_complex_noise(uint32_t* s, float* out, int nxp, int nyp, int nzp) {
  size_t cnxp = (size_t)(nxp / 2 + 1);
  size_t csize = cnxp * (size_t)nyp * (size_t)nzp;
  float sd = (float)(1.0 / sqrt(2.0));
  for (size_t i = 0; i < csize; i++) {
    size_t xs = i % cnxp;
    if (xs == 0 || (xs == cnxp - 1 && (i % 2) == 1)) {
      size_t jk = (i - xs) / cnxp;
      size_t j = jk % (size_t)nyp, k = jk / (size_t)nyp;
      size_t jc = j == 0 ? 0 : (size_t)nyp - j;
      size_t kc = k == 0 ? 0 : (size_t)nzp - k;
      size_t jkc = jc + kc * (size_t)nyp;
      if (jkc == jk) {
        out[2 * i] = (float)oracle_rnorm01(s);
        out[2 * i + 1] = 0.0f;
      } else if (jkc > jk) {
        out[2 * i] = (float)(sd * oracle_rnorm01(s));
        out[2 * i + 1] = (float)(sd * oracle_rnorm01(s));
      } else {
        size_t cc = jkc * cnxp + xs;
        out[2 * i] = out[2 * cc];
        out[2 * i + 1] = -out[2 * cc + 1];
      }
    } else {
      out[2 * i] = (float)(sd * oracle_rnorm01(s));
      out[2 * i + 1] = (float)(sd * oracle_rnorm01(s));
    }
  }
}

/* The noise of nsim realisations in simulate's draw order (seed0, seed1, seed2 per
 * realisation, src/avoinversion.cpp:1405-1407) starting from RandomGen(seed). */
void oracle_sim_noise(uint32_t seed, int nsim, int nxp, int nyp, int nzp, float* out) {
  uint32_t s = seed;
  size_t csize = (size_t)(nxp / 2 + 1) * (size_t)nyp * (size_t)nzp;
  for (int g = 0; g < 3 * nsim; g++) oracle_fill_complex_noise(&s, out + (size_t)g * 2 * csize, nxp, nyp, nzp);
}
