// Samplers of the Poisson-system-with-stochastic-rates step (the reference's
// default ``psr`` implementation, model_builder/C/templates/core_template.c:
// 105-209): binomial and multinomial splits of a compartment, Poisson
// arrivals, Gamma white noise.  The reference draws them with GSL
// (gsl_ran_binomial, gsl_ran_poisson, gsl_ran_gamma on mt19937); here they
// are exact samplers from published methods, fed by a counter-based Philox
// stream so that the GPU and the oracle draw the same numbers:
//
// * binomial: inversion of the CDF when n·min(p, 1-p) < 14, otherwise BTRD,
//   the transformed rejection with decomposition of W. Hörmann, "The
//   generation of binomial random variates", J. Statist. Comput. Simul. 46
//   (1993);
// * Poisson: inversion when mu < 10, otherwise PTRS, the transformed
//   rejection with squeeze of W. Hörmann, "The transformed rejection method
//   for generating Poisson random variables", Insurance: Mathematics and
//   Economics 12 (1993);
// * Gamma: G. Marsaglia and W. W. Tsang, "A simple method for generating
//   gamma variables", ACM TOMS 26 (2000), with the boost U^(1/a) for a < 1;
// * multinomial: sequential conditional binomials (plom_ran_multinomial,
//   model_builder/C/core/prediction_util.c:327-345).
//
// FP64 particle states (the parity modes, and the oracle) draw in double;
// FP32 states draw with the single-precision versions at the end of this
// file, which keep double where magnitudes cancel.
#pragma once

#include "plom_rt.h"

// The samplers are real calls on the device (one copy of their code for the
// many call sites of a step): inlined, the step's code overflows the
// instruction cache.
#if defined(__CUDACC__)
#ifndef PLOM_PSR_INLINE
#define PLOM_SAMPLER __host__ __device__ __noinline__
#else
#define PLOM_SAMPLER PLOM_HD
#endif
#else
#define PLOM_SAMPLER inline
#endif

namespace plomrt {

enum { STREAM_PSR = 4 };

// double-precision elementary functions of the samplers, called rather than
// inlined at every use (same values; less code)
PLOM_SAMPLER double s_log(double x) { return log(x); }
PLOM_SAMPLER double s_exp(double x) { return exp(x); }
PLOM_SAMPLER double s_pow(double x, double y) { return pow(x, y); }
PLOM_SAMPLER double s_lgamma(double x) { return lgamma(x); }
PLOM_SAMPLER double s_cos(double x) { return cos(x); }

// two 53-bit uniforms of Philox block (j, n, group, STREAM_PSR + 16 block)
PLOM_SAMPLER void psr_uniform_pair(PhiloxKey key, uint32_t j, uint32_t n, uint32_t group, uint32_t block, double* a,
                                   double* b) {
  const U4 c = {j, n, group, (uint32_t)STREAM_PSR + (block << 4)};
  const U4 r = philox4x32_10(c, key.k0, key.k1);
  *a = u01d(r.x, r.y);
  *b = u01d(r.z, r.w);
}

// Uniforms of one (particle, interval, substep, cac) group: Philox counter
// (x = particle slot, y = interval, z = substep * (N_CAC + 1) + cac,
// w = STREAM_PSR + 16 * block); two 53-bit uniforms per block.
struct UniformStream {
  PhiloxKey key;
  uint32_t j, n, group;
  uint32_t block;
  double cache;
  bool has;
  PLOM_HD void init(PhiloxKey k, uint32_t j_, uint32_t n_, uint32_t group_) {
    key = k;
    j = j_;
    n = n_;
    group = group_;
    block = 0;
    has = false;
    cache = 0.0;
  }
  // uniform in (0, 1)
  PLOM_HD double next() {
    if (has) {
      has = false;
      return cache;
    }
    double first;
    psr_uniform_pair(key, j, n, group, block, &first, &cache);
    ++block;
    has = true;
    return first;
  }
  PLOM_HD double normal() {
    const double u1 = next(), u2 = next();
    return sqrt(-2.0 * s_log(u1)) * s_cos(6.283185307179586 * u2);
  }
};

// log k! - Stirling's approximation of it (the correction term of BTRD)
PLOM_HD double stirling_correction(double k) {
  if (k < 10.0) return s_lgamma(k + 1.0) - ((k + 0.5) * s_log(k + 1.0) - (k + 1.0) + 0.9189385332046728);
  const double r = 1.0 / (k + 1.0), r2 = r * r;
  return (1.0 / 12.0 - (1.0 / 360.0 - (1.0 / 1260.0) * r2) * r2) * r;
}

// bound on rejection rounds: far beyond any realistic count (the expected
// number is below 2); a sampler that reaches it returns its mode
constexpr int kMaxRejection = 1000;

PLOM_HD double binomial_inversion(UniformStream& rs, double n, double p) {
  const double q = 1.0 - p;
  const double s = p / q, a = (n + 1.0) * s;
  const double r0 = s_pow(q, n);
  for (int round = 0; round < kMaxRejection; ++round) {
    double u = rs.next(), r = r0, x = 0.0;
    while (u > r) {
      u -= r;
      x += 1.0;
      if (x > n) break;
      r *= (a / x - s);
    }
    if (x <= n) return x;
  }
  return floor(n * p);
}

PLOM_HD double binomial_btrd(UniformStream& rs, double n, double p) {
  const double q = 1.0 - p;
  const double spq = sqrt(n * p * q);
  const double b = 1.15 + 2.53 * spq;
  const double a = -0.0873 + 0.0248 * b + 0.01 * p;
  const double c = n * p + 0.5;
  const double vr = 0.92 - 4.2 / b;
  const double alpha = (2.83 + 5.1 / b) * spq;
  const double m = floor((n + 1.0) * p);
  const double r = p / q, nr = (n + 1.0) * r, npq = n * p * q;
  for (int round = 0; round < kMaxRejection; ++round) {
    double v = rs.next();
    double u;
    if (v <= 0.86 * vr) {
      u = v / vr - 0.43;
      return floor((2.0 * a / (0.5 - fabs(u)) + b) * u + c);
    }
    if (v >= vr) {
      u = rs.next() - 0.5;
    } else {
      u = v / vr - 0.93;
      u = ((u > 0.0) ? 0.5 : -0.5) - u;
      v = rs.next() * vr;
    }
    const double us = 0.5 - fabs(u);
    const double k = floor((2.0 * a / us + b) * u + c);
    if (k < 0.0 || k > n) continue;
    v = v * alpha / (a / (us * us) + b);
    const double km = fabs(k - m);
    if (km <= 15.0) {
      // recursive evaluation of f(k) / f(m)
      double f = 1.0;
      if (m < k) {
        for (double i = m + 1.0; i <= k; i += 1.0) f *= (nr / i - r);
      } else if (m > k) {
        for (double i = k + 1.0; i <= m; i += 1.0) v *= (nr / i - r);
      }
      if (v <= f) return k;
      continue;
    }
    // squeeze
    v = s_log(v);
    const double rho = (km / npq) * (((km / 3.0 + 0.625) * km + 1.0 / 6.0) / npq + 0.5);
    const double t = -km * km / (2.0 * npq);
    if (v < t - rho) return k;
    if (v > t + rho) continue;
    const double nm = n - m + 1.0;
    const double h = (m + 0.5) * s_log((m + 1.0) / (r * nm)) + stirling_correction(m) + stirling_correction(n - m);
    const double nk = n - k + 1.0;
    if (v <= h + (n + 1.0) * s_log(nm / nk) + (k + 0.5) * s_log(nk * r / (k + 1.0)) - stirling_correction(k) -
                 stirling_correction(n - k))
      return k;
  }
  return m;
}

// Binomial(n, p), n a non-negative integer held in a double
PLOM_SAMPLER double binomial(UniformStream& rs, double n, double p) {
  if (n <= 0.0 || !(p > 0.0)) return 0.0;
  if (p >= 1.0) return n;
  const bool flip = p > 0.5;  // sample the smaller tail
  const double pp = flip ? 1.0 - p : p;
  const double x = (n * pp < 14.0) ? binomial_inversion(rs, n, pp) : binomial_btrd(rs, n, pp);
  return flip ? n - x : x;
}

PLOM_SAMPLER double poisson(UniformStream& rs, double mu) {
  if (!(mu > 0.0)) return 0.0;
  if (mu < 10.0) {
    for (int round = 0; round < kMaxRejection; ++round) {
      double u = rs.next(), p = s_exp(-mu), x = 0.0;
      while (u > p) {
        u -= p;
        x += 1.0;
        p *= mu / x;
        if (x > 1000.0) break;
      }
      if (x <= 1000.0) return x;
    }
    return floor(mu);
  }
  const double smu = sqrt(mu);
  const double b = 0.931 + 2.53 * smu;
  const double a = -0.059 + 0.02483 * b;
  const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
  const double vr = 0.9277 - 3.6224 / (b - 2.0);
  const double lmu = s_log(mu);
  for (int round = 0; round < kMaxRejection; ++round) {
    const double u = rs.next() - 0.5;
    const double v = rs.next();
    const double us = 0.5 - fabs(u);
    const double k = floor((2.0 * a / us + b) * u + mu + 0.43);
    if (us >= 0.07 && v <= vr) return k;
    if (k < 0.0 || (us < 0.013 && v > us)) continue;
    if (s_log(v) + s_log(inv_alpha) - s_log(a / (us * us) + b) <= -mu + k * lmu - s_lgamma(k + 1.0)) return k;
  }
  return floor(mu);
}

// Gamma with shape a and scale theta
PLOM_SAMPLER double gamma(UniformStream& rs, double a, double theta) {
  if (!(a > 0.0) || !(theta > 0.0)) return 0.0;
  double boost = 1.0;
  if (a < 1.0) {
    boost = s_pow(rs.next(), 1.0 / a);
    a += 1.0;
  }
  const double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
  for (int round = 0; round < kMaxRejection; ++round) {
    const double z = rs.normal();
    double v = 1.0 + c * z;
    if (v <= 0.0) continue;
    v = v * v * v;
    const double u = rs.next();
    if (u < 1.0 - 0.0331 * z * z * z * z) return d * v * theta * boost;
    if (s_log(u) < 0.5 * z * z + d * (1.0 - v + s_log(v))) return d * v * theta * boost;
  }
  return d * theta * boost;
}

// plom_ran_multinomial: K categories with probabilities p summing to one,
// N trials; out[k] = counts.  The last category takes the remaining trials:
// its conditional probability p[K-1] / (1 - sum of the others) is one in
// exact arithmetic, and deciding it in floating point would make the number
// of uniforms drawn (and so every later draw of the stream) depend on the
// last bits of the probabilities.
template <int K>
PLOM_HD void multinomial(UniformStream& rs, double N, const double (&p)[K], double (&out)[K]) {
  double sum_p = 0.0, sum_n = 0.0;
  for (int k = 0; k < K - 1; ++k) {
    out[k] = (p[k] > 0.0) ? binomial(rs, N - sum_n, p[k] / (1.0 - sum_p)) : 0.0;
    sum_p += p[k];
    sum_n += out[k];
  }
  out[K - 1] = (p[K - 1] > 0.0) ? N - sum_n : 0.0;
}

// ---------------------------------------------------------------- single precision
// The same samplers for FP32 particle states, in float where the magnitudes
// allow it: four 24-bit uniforms per Philox block instead of two 53-bit ones,
// float elementary functions.  Three quantities keep double: the location
// n p + 1/2 (or mu + 0.43) added last when a count is formed, the mode of
// BTRD, and the final acceptance tests of BTRD and PTRS, whose terms are of
// the order of the count (k log mu, log k!) and cancel to O(1).  Counts are
// exact in float below 2^24, the range of an FP32 state's integers.
// float elementary functions inline (short; as calls the psr step of SEIR
// 20x2 took 19.5 against 16.8 ms per interval), the samplers still calls
PLOM_HD float s_log(float x) { return logf(x); }
PLOM_HD float s_exp(float x) { return expf(x); }
PLOM_HD float s_pow(float x, float y) { return powf(x, y); }
PLOM_HD float s_log1p(float x) { return log1pf(x); }

// Philox block (j, n, group, STREAM_PSR + 16 block) as four uniforms in (0, 1)
PLOM_SAMPLER void psr_uniform_quad(PhiloxKey key, uint32_t j, uint32_t n, uint32_t group, uint32_t block, float* u) {
  const U4 c = {j, n, group, (uint32_t)STREAM_PSR + (block << 4)};
  const U4 r = philox4x32_10(c, key.k0, key.k1);
  const float s = 1.0f / 16777216.0f;
  u[0] = ((float)(r.x >> 8) + 0.5f) * s;
  u[1] = ((float)(r.y >> 8) + 0.5f) * s;
  u[2] = ((float)(r.z >> 8) + 0.5f) * s;
  u[3] = ((float)(r.w >> 8) + 0.5f) * s;
}

struct UniformStreamF {
  PhiloxKey key;
  uint32_t j, n, group;
  uint32_t block;
  float cache[4];
  int used;  // uniforms of the cached block already returned (4: none left)
  PLOM_HD void init(PhiloxKey k, uint32_t j_, uint32_t n_, uint32_t group_) {
    key = k;
    j = j_;
    n = n_;
    group = group_;
    block = 0;
    used = 4;
  }
  PLOM_HD float next() {
    if (used == 4) {
      psr_uniform_quad(key, j, n, group, block, cache);
      ++block;
      used = 0;
    }
    return cache[used++];
  }
  // Box-Muller with the angle in [-pi, pi): the special-function-unit cosine
  // of the fast-math build is accurate on that range only; cos(a - pi) =
  // -cos(a) flips the sign of the draw, not its distribution
  PLOM_HD float normal() {
    const float u1 = next(), u2 = next();
    return sqrtf(-2.0f * s_log(u1)) * cosf(6.2831853071795865f * (u2 - 0.5f));
  }
};

// stream type of a particle precision
template <class T> struct PsrStream { typedef UniformStream type; };
template <> struct PsrStream<float> { typedef UniformStreamF type; };

// Inversion for n p < 40 (the double samplers switch to BTRD at 14; in
// float the inversion loop is the cheaper of the two up to a mean of about
// 60: SEIR 20x2 psr 16.7 / 14.7 / 13.7 / 13.2 ms per interval with the switch
// at 14 / 30 / 40 / 60, and q^n = (1 - p)^n stays a normal float, above
// 2^-80, below 40); likewise Poisson counts below a mean of 40 (PTRS above;
// 13.7 / 12.8 / 12.4 ms with the switch at 10 / 20 / 40).  The float partial sums of the probabilities may stop
// short of a uniform near 1; the search therefore ends at x = 200 (the
// probability of more is below 1e-40 for a mean below 40) and the round
// redraws, instead of walking up to n through probabilities that underflow.
constexpr float kInversionMaxF = 200.0f;
constexpr float kInversionMeanF = 40.0f;

PLOM_HD float binomial_inversion(UniformStreamF& rs, float n, float p) {
  const float q = 1.0f - p;
  const float s = p / q, a = (n + 1.0f) * s;
  const float r0 = s_exp(n * s_log1p(-p));  // q^n, accurate for small p
  const float xmax = fminf(n, kInversionMaxF);
  for (int round = 0; round < kMaxRejection; ++round) {
    float u = rs.next(), r = r0, x = 0.0f;
    while (u > r) {
      u -= r;
      x += 1.0f;
      if (x > xmax) break;
      r *= (a / x - s);
    }
    if (x <= xmax) return x;
  }
  return floorf(n * p);
}

// the last BTRD test, log f(k) / f(m) against the scaled hat value log v
PLOM_SAMPLER bool btrd_accept(double n, double m, double k, double r, double v) {
  const double nm = n - m + 1.0;
  const double h = (m + 0.5) * s_log((m + 1.0) / (r * nm)) + stirling_correction(m) + stirling_correction(n - m);
  const double nk = n - k + 1.0;
  return v <= h + (n + 1.0) * s_log(nm / nk) + (k + 0.5) * s_log(nk * r / (k + 1.0)) - stirling_correction(k) -
                  stirling_correction(n - k);
}

PLOM_HD float binomial_btrd(UniformStreamF& rs, float n, float p) {
  const float q = 1.0f - p;
  const float spq = sqrtf(n * p * q);
  const float b = 1.15f + 2.53f * spq;
  const float a = -0.0873f + 0.0248f * b + 0.01f * p;
  const double c = (double)n * (double)p + 0.5;
  const float vr = 0.92f - 4.2f / b;
  const float alpha = (2.83f + 5.1f / b) * spq;
  const double md = floor(((double)n + 1.0) * (double)p);
  const float m = (float)md;
  const float r = p / q, nr = (n + 1.0f) * r, npq = n * p * q;
  for (int round = 0; round < kMaxRejection; ++round) {
    float v = rs.next();
    float u;
    if (v <= 0.86f * vr) {
      u = v / vr - 0.43f;
      return (float)floor((double)((2.0f * a / (0.5f - fabsf(u)) + b) * u) + c);
    }
    if (v >= vr) {
      u = rs.next() - 0.5f;
    } else {
      u = v / vr - 0.93f;
      u = ((u > 0.0f) ? 0.5f : -0.5f) - u;
      v = rs.next() * vr;
    }
    const float us = 0.5f - fabsf(u);
    const float k = (float)floor((double)((2.0f * a / us + b) * u) + c);
    if (k < 0.0f || k > n) continue;
    v = v * alpha / (a / (us * us) + b);
    const float km = fabsf(k - m);
    if (km <= 15.0f) {
      // integer steps: a float counter would stop moving above 2^24
      const int steps = (int)km;
      float f = 1.0f;
      if (m < k) {
        for (int d = 1; d <= steps; ++d) f *= (nr / (m + (float)d) - r);
      } else if (m > k) {
        for (int d = 1; d <= steps; ++d) v *= (nr / (k + (float)d) - r);
      }
      if (v <= f) return k;
      continue;
    }
    v = s_log(v);
    const float rho = (km / npq) * (((km / 3.0f + 0.625f) * km + 1.0f / 6.0f) / npq + 0.5f);
    const float t = -km * km / (2.0f * npq);
    if (v < t - rho) return k;
    if (v > t + rho) continue;
    if (btrd_accept((double)n, md, (double)k, (double)p / (double)q, (double)v)) return k;
  }
  return m;
}

PLOM_SAMPLER float binomial(UniformStreamF& rs, float n, float p) {
  if (n <= 0.0f || !(p > 0.0f)) return 0.0f;
  if (p >= 1.0f) return n;
  const bool flip = p > 0.5f;
  const float pp = flip ? 1.0f - p : p;
  const float x = (n * pp < kInversionMeanF) ? binomial_inversion(rs, n, pp) : binomial_btrd(rs, n, pp);
  return flip ? n - x : x;
}

// the last PTRS test
PLOM_SAMPLER bool ptrs_accept(double mu, double k, double v, double us, double a, double b, double inv_alpha) {
  return s_log(v) + s_log(inv_alpha) - s_log(a / (us * us) + b) <= -mu + k * s_log(mu) - s_lgamma(k + 1.0);
}

PLOM_SAMPLER float poisson(UniformStreamF& rs, float mu) {
  if (!(mu > 0.0f)) return 0.0f;
  if (mu < kInversionMeanF) {  // e^-mu stays a normal float; PTRS above
    for (int round = 0; round < kMaxRejection; ++round) {
      float u = rs.next(), p = s_exp(-mu), x = 0.0f;
      while (u > p) {
        u -= p;
        x += 1.0f;
        p *= mu / x;
        if (x > kInversionMaxF) break;
      }
      if (x <= kInversionMaxF) return x;
    }
    return floorf(mu);
  }
  const float smu = sqrtf(mu);
  const float b = 0.931f + 2.53f * smu;
  const float a = -0.059f + 0.02483f * b;
  const float inv_alpha = 1.1239f + 1.1328f / (b - 3.4f);
  const float vr = 0.9277f - 3.6224f / (b - 2.0f);
  const double loc = (double)mu + 0.43;
  for (int round = 0; round < kMaxRejection; ++round) {
    const float u = rs.next() - 0.5f;
    const float v = rs.next();
    const float us = 0.5f - fabsf(u);
    const float k = (float)floor((double)((2.0f * a / us + b) * u) + loc);
    if (us >= 0.07f && v <= vr) return k;
    if (k < 0.0f || (us < 0.013f && v > us)) continue;
    if (ptrs_accept((double)mu, (double)k, (double)v, (double)us, (double)a, (double)b, (double)inv_alpha)) return k;
  }
  return floorf(mu);
}

PLOM_SAMPLER float gamma(UniformStreamF& rs, float a, float theta) {
  if (!(a > 0.0f) || !(theta > 0.0f)) return 0.0f;
  float boost = 1.0f;
  if (a < 1.0f) {
    boost = s_pow(rs.next(), 1.0f / a);
    a += 1.0f;
  }
  const float d = a - 1.0f / 3.0f, c = 1.0f / sqrtf(9.0f * d);
  for (int round = 0; round < kMaxRejection; ++round) {
    const float z = rs.normal();
    float v = 1.0f + c * z;
    if (v <= 0.0f) continue;
    v = v * v * v;
    const float u = rs.next();
    if (u < 1.0f - 0.0331f * z * z * z * z) return d * v * theta * boost;
    if (s_log(u) < 0.5f * z * z + d * (1.0f - v + s_log(v))) return d * v * theta * boost;
  }
  return d * theta * boost;
}

template <int K>
PLOM_HD void multinomial(UniformStreamF& rs, float N, const float (&p)[K], float (&out)[K]) {
  float sum_p = 0.0f, sum_n = 0.0f;
  for (int k = 0; k < K - 1; ++k) {
    out[k] = (p[k] > 0.0f) ? binomial(rs, N - sum_n, p[k] / (1.0f - sum_p)) : 0.0f;
    sum_p += p[k];
    sum_n += out[k];
  }
  out[K - 1] = (p[K - 1] > 0.0f) ? N - sum_n : 0.0f;
}

}  // namespace plomrt
