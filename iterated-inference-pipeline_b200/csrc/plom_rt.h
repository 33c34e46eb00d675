// Shared runtime for generated plom models: compiled into the sm_100a
// kernels and (as plain C++) into the CPU oracle.
//
//  * special functions of the rate language (model_builder/C/core/special_functions.c:48-75);
//  * parameter back-transforms (model_builder/C/core/transform.c:23-111, 462-481);
//  * the discretised-normal observation density and its sanitisation
//    (model_builder/C/templates/core_template.c:342-367,
//     model_builder/C/core/likelihood.c:77-92);
//  * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
//    easy as 1, 2, 3", SC'11) and the Box-Muller transform;
//  * the exact closed form of the reference's systematic-resampling points
//    ``ran += 1/J`` (model_builder/C/core/smc.c:97-111).
#pragma once

#include <stdint.h>
#include <math.h>
#include <string.h>

#if defined(__CUDACC__)
#define PLOM_HD __host__ __device__ __forceinline__
#else
#define PLOM_HD inline
#endif

// Loop unrolling: ``PLOM_UNROLL`` fully unrolls short fixed loops; the loop
// over compartment-age classes is unrolled when the particle state lives in
// registers (small models) and kept rolled when it lives in shared memory.
// ``PLOM_PRAGMA_GROUP`` covers the cacs of one draw group (unrolled unless
// PLOM_GROUP_ROLLED is defined, which trades registers / code size for
// indexed draws).
#if defined(__CUDACC__)
#define PLOM_UNROLL _Pragma("unroll")
#if defined(PLOM_SMEM_STATE) && PLOM_SMEM_STATE
#define PLOM_PRAGMA_CAC _Pragma("unroll 1")
#else
#define PLOM_PRAGMA_CAC _Pragma("unroll")
#endif
#if defined(PLOM_GROUP_ROLLED)
#define PLOM_PRAGMA_GROUP _Pragma("unroll 1")
#else
#define PLOM_PRAGMA_GROUP _Pragma("unroll")
#endif
#else
#define PLOM_UNROLL
#define PLOM_PRAGMA_CAC
#define PLOM_PRAGMA_GROUP
#endif

namespace plomrt {

template <class T>
struct V4 {
  T a, b, c, d;
};

// ---------------------------------------------------------------- special functions
template <class T> PLOM_HD T heaviside_(T x) { return (x < T(0)) ? T(0) : T(1); }
template <class T> PLOM_HD T ramp_(T x) { return (x >= T(0)) ? x : T(0); }
// piecewise linear: 0 below 0, x on [0, d), d above (the reference's body
// returns an undeclared ``t`` in the middle branch; its comment states x)
template <class T> PLOM_HD T slowstep_(T x, T d) { return x >= T(0) ? (x >= d ? d : x) : T(0); }

// ---------------------------------------------------------------- transforms
enum { FINV_ID = 0, FINV_EXP = 1, FINV_LOGIT = 2, FINV_LOGIT_AB = 3 };
enum { SCALE_ID = 0, SCALE_POW10 = 1, SCALE_POW10_NEG = 2 };

// One group of one parameter: how a transformed value maps to the natural
// scale in data units (back_transform_x, transform.c:462-481).
struct BackTransform {
  int f_inv;
  int scale;
  int is_duration;
  int pad;
  double a, b;        // min, max of the group (logit_ab bounds)
  double multiplier;  // unit conversion to data units
};

template <class T>
PLOM_HD T back_transform(T x, const BackTransform& r) {
  T v;
  const T a = T(r.a), b = T(r.b);
  switch (r.f_inv) {
    case FINV_EXP: v = exp(x); break;
    case FINV_LOGIT: v = (x > T(0)) ? T(1) / (T(1) + exp(-x)) : exp(x) / (T(1) + exp(x)); break;
    case FINV_LOGIT_AB:
      if (a == b) v = x;
      else if (x < T(0)) v = (b * exp(x) + a) / (T(1) + exp(x));
      else v = (b + a * exp(-x)) / (T(1) + exp(-x));
      break;
    default: v = x;
  }
  if (r.scale == SCALE_POW10) v = pow(T(10), v);
  else if (r.scale == SCALE_POW10_NEG) v = pow(T(10), -v);
  v *= T(r.multiplier);
  if (r.is_duration) v = T(1) / (T(0.00001) + v);
  return v;
}

// ---------------------------------------------------------------- observation density
// Standard normal CDF; the same expression on both sides of every parity check.
PLOM_HD double std_normal_cdf(double z) { return 0.5 * erfc(-z * 0.70710678118654752440); }

// Discretised normal likelihood of an integer count y given mean mu and variance var,
// clamped to like_min (core_template.c:357-366 + likelihood.c:77-92).
PLOM_HD double disc_normal_like(double y, double mu, double var, double like_min) {
  const double sd = sqrt(var);
  double like;
  if (y > 0.0) {
    like = std_normal_cdf((y + 0.5 - mu) / sd) - std_normal_cdf((y - 0.5 - mu) / sd);
  } else {
    like = std_normal_cdf((y + 0.5 - mu) / sd);
  }
  if (isinf(like) || isnan(like) || like < 0.0) return like_min;
  return (like <= like_min) ? like_min : like;
}

// Log of one series' density, counting the series whose density sits on the
// LIKE_MIN floor.
PLOM_HD double log_like_term(double y, double mu, double var, double like_min, int* floor_hits) {
  const double l = disc_normal_like(y, mu, var, like_min);
  if (l == like_min) ++*floor_hits;
  return log(l);
}

// The same term for FP32 particle states, in single precision.  The
// differences y -/+ 1/2 - mu are taken in double (counts and means reach
// 1e7, whose float spacing would shift the bounds), the rest in float
// arranged so that no difference of nearly equal floats decides the value:
// * 1/sd <= 1/20: the interval is narrow, and the probability is the density
//   at its midpoint m times its width d with the next two terms of the
//   expansion of Phi(m + d/2) - Phi(m - d/2), phi(m) d (1 + (m^2 - 1) d^2 / 24
//   + (m^4 - 6 m^2 + 3) d^4 / 1920), whose first omitted term is
//   He6(m) d^6 / 161280 relative (He6 the sixth Hermite polynomial; below
//   3e-8 wherever the density is above LIKE_MIN = 1e-17, |m| < 8.4);
// * otherwise: upper tails by erfc when the interval lies above the mean,
//   lower tails when below, and 1 minus both tails when it straddles it.
// Clamping, the floor count and the log are those of the double version;
// the sum over series stays double.
PLOM_HD double log_like_term_f(double y, double mu, double var, double like_min, int* floor_hits) {
  const float k = 0.70710678118654752f;  // 1/sqrt(2)
  const float inv = 1.0f / sqrtf((float)var);
  float like;
  if (y > 0.0) {
    const float lo = (float)(y - 0.5 - mu) * inv, hi = (float)(y + 0.5 - mu) * inv;
    if (inv <= 0.05f) {
      const float m = 0.5f * (lo + hi), m2 = m * m, d2 = inv * inv;
      like = 0.39894228040143268f * expf(-0.5f * m2) * inv *
             (1.0f + (m2 - 1.0f) * d2 * (1.0f / 24.0f) + ((m2 - 6.0f) * m2 + 3.0f) * (d2 * d2) * (1.0f / 1920.0f));
    } else if (lo >= 0.0f) {
      like = 0.5f * (erfcf(lo * k) - erfcf(hi * k));
    } else if (hi <= 0.0f) {
      like = 0.5f * (erfcf(-hi * k) - erfcf(-lo * k));
    } else {
      like = 1.0f - 0.5f * (erfcf(hi * k) + erfcf(-lo * k));
    }
  } else {
    like = 0.5f * erfcf(-(float)(y + 0.5 - mu) * inv * k);
  }
  if (!(like > (float)like_min) || isinf(like)) {
    ++*floor_hits;
    return log(like_min);
  }
  return (double)logf(like);
}

// the term of a particle precision: FP64 states (the parity modes) keep the
// double version
template <class T>
PLOM_HD double log_like_term_p(double y, double mu, double var, double like_min, int* floor_hits) {
  if constexpr (sizeof(T) == sizeof(float)) return log_like_term_f(y, mu, var, like_min, floor_hits);
  else return log_like_term(y, mu, var, like_min, floor_hits);
}

// A particle's log-weight.  The reference fails a particle when
// exp(loglik) <= LIKE_MIN^N_TS (smc.c:44); since every density is at least
// LIKE_MIN, that holds in exact arithmetic exactly when all N_TS series are on
// the floor, a case the rounding of exp / pow would otherwise decide one way
// or the other.  Such a particle gets -inf (weight 0, a failure); integer
// (psr) counts meet the case often.
PLOM_HD double finish_loglik(double ll, int floor_hits, int n_ts) { return floor_hits >= n_ts ? -INFINITY : ll; }

// ---------------------------------------------------------------- Philox4x32-10
struct U4 { uint32_t x, y, z, w; };

PLOM_HD uint32_t mulhilo32(uint32_t a, uint32_t b, uint32_t* hi) {
#if defined(__CUDA_ARCH__) && !defined(PLOM_PHILOX_WIDE)
  *hi = __umulhi(a, b);
  return a * b;
#else
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  return (uint32_t)p;
#endif
}

// rounds unrolled per loop iteration (code size against loop overhead)
#ifndef PLOM_PHILOX_UNROLL
#define PLOM_PHILOX_UNROLL 10
#endif
#define PLOM_STR_(x) #x
#define PLOM_PRAGMA_UNROLL_N(n) _Pragma(PLOM_STR_(unroll n))

PLOM_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  PLOM_PRAGMA_UNROLL_N(PLOM_PHILOX_UNROLL)
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, hi1;
    const uint32_t lo0 = mulhilo32(M0, c.x, &hi0);
    const uint32_t lo1 = mulhilo32(M1, c.z, &hi1);
    U4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// uniform in (0, 1) with 23-bit resolution (Box-Muller angle): the high 23 bits
// as the mantissa of a float in [1, 2), minus 1 - 2^-24 (exact by Sterbenz), i.e.
// (k + 1/2) 2^-23; integer and logic instructions instead of a conversion on the
// special-function pipe
PLOM_HD float u01f(uint32_t u) {
  const uint32_t b = 0x3f800000u | (u >> 9);
  float f;
  memcpy(&f, &b, sizeof f);
  return f - 0.99999994039535522f;
}
// uniform in (0, 1] from all 32 bits, fine near 0 (Box-Muller radius: tails to 6.7 sd)
PLOM_HD float u01f_radius(uint32_t u) { return (float)u * 2.3283064365386963e-10f + 1.1641532182693481e-10f; }
// uniform in (0, 1) from 64 bits with 53-bit resolution
PLOM_HD double u01d(uint32_t lo, uint32_t hi) {
  const uint64_t v = (((uint64_t)hi << 32) | lo) >> 11;
  return ((double)v + 0.5) * (1.0 / 9007199254740992.0);
}
// uniform in [0, 1) with 53-bit resolution (the contract of gsl_rng_uniform)
PLOM_HD double u01d_closed0(uint32_t lo, uint32_t hi) {
  const uint64_t v = (((uint64_t)hi << 32) | lo) >> 11;
  return (double)v * (1.0 / 9007199254740992.0);
}

// Box-Muller: two normals from two uniforms in (0, 1)
PLOM_HD void box_muller_d(double u1, double u2, double* z0, double* z1) {
  const double r = sqrt(-2.0 * log(u1));
  const double th = 6.283185307179586 * u2;
  *z0 = r * cos(th);
  *z1 = r * sin(th);
}

PLOM_HD void box_muller_f(float u1, float u2, float* z0, float* z1) {
#if defined(__CUDA_ARCH__)
  const float r = sqrtf(-2.0f * __logf(u1));
  float s, c;
  __sincosf(6.2831853071795865f * (u2 - 0.5f), &s, &c);
#else
  const float r = sqrtf(-2.0f * logf(u1));
  const float th = 6.2831853071795865f * (u2 - 0.5f);
  const float s = sinf(th), c = cosf(th);
#endif
  *z0 = r * c;
  *z1 = r * s;
}

// Philox counter layout of one particle's draws:
//   (x = particle slot, y = observation index, z = draw block, w = stream tag)
// with key = (seed low ^ filter * golden, seed high).  Draw blocks of one
// substep: (substep * (N_CAC + 1) + cac) * blocks + b; slot cac = N_CAC holds
// the drift draws.
enum { STREAM_PROCESS = 0, STREAM_RESAMPLE = 1, STREAM_MUTATE = 2, STREAM_INIT = 3 };

struct PhiloxKey {
  uint32_t k0, k1;
};

PLOM_HD PhiloxKey make_key(uint64_t seed, uint32_t filter) {
  PhiloxKey k;
  k.k0 = (uint32_t)seed ^ (filter * 0x9E3779B9u);
  k.k1 = (uint32_t)(seed >> 32);
  return k;
}

// Normals of precision T for one (particle, observation, substep, cac) group.
template <class T> struct NormalGen;

template <> struct NormalGen<float> {
  // 4 normals per Philox block
  template <int N>
  PLOM_HD static void fill(PhiloxKey k, uint32_t j, uint32_t n, uint32_t blk0, float* out,
                           uint32_t tag = STREAM_PROCESS) {
#pragma unroll
    for (int b = 0; b < (N + 3) / 4; ++b) {
      U4 c = {j, n, blk0 + (uint32_t)b, tag};
      const U4 r = philox4x32_10(c, k.k0, k.k1);
      float z0, z1, z2, z3;
      box_muller_f(u01f_radius(r.x), u01f(r.y), &z0, &z1);
      box_muller_f(u01f_radius(r.z), u01f(r.w), &z2, &z3);
      if (4 * b + 0 < N) out[4 * b + 0] = z0;
      if (4 * b + 1 < N) out[4 * b + 1] = z1;
      if (4 * b + 2 < N) out[4 * b + 2] = z2;
      if (4 * b + 3 < N) out[4 * b + 3] = z3;
    }
  }
  static constexpr PLOM_HD int per_block() { return 4; }
};

template <> struct NormalGen<double> {
  // the two normals of one Philox block (53-bit uniforms)
  PLOM_HD static void block(PhiloxKey k, uint32_t j, uint32_t n, uint32_t blk, uint32_t tag, double* z0,
                            double* z1) {
    U4 c = {j, n, blk, tag};
    const U4 r = philox4x32_10(c, k.k0, k.k1);
    box_muller_d(u01d(r.x, r.y), u01d(r.z, r.w), z0, z1);
  }
  // 2 normals per Philox block
  template <int N>
  PLOM_HD static void fill(PhiloxKey k, uint32_t j, uint32_t n, uint32_t blk0, double* out,
                           uint32_t tag = STREAM_PROCESS) {
#pragma unroll
    for (int b = 0; b < (N + 1) / 2; ++b) {
      double z0, z1;
      block(k, j, n, blk0 + (uint32_t)b, tag, &z0, &z1);
      if (2 * b + 0 < N) out[2 * b + 0] = z0;
      if (2 * b + 1 < N) out[2 * b + 1] = z1;
    }
  }
  static constexpr PLOM_HD int per_block() { return 2; }
};

// Uniform in [0, 1) for the systematic resampling of observation n of a filter.
PLOM_HD double resample_uniform(PhiloxKey k, uint32_t n) {
  U4 c = {0u, n, 0u, (uint32_t)STREAM_RESAMPLE};
  const U4 r = philox4x32_10(c, k.k0, k.k1);
  return u01d_closed0(r.x, r.y);
}

// ---------------------------------------------------------------- systematic points
// The reference walks the points with ``ran = U; ... ran += inc;`` in double
// (smc.c:100-111), so point j is U followed by j rounded additions, not
// U + j*inc.  Inside one binade [2^e, 2^(e+1)) every rounded addition of the
// same increment moves a grid point by the same amount, except that a tie
// (inc half-way between grid points) can alter the first step after entering
// the binade; from the first point after the entry point on, the step is
// constant.  The table below stores, for each run of points, the index of its
// first point, its first value and the constant step, so that every point
// is recovered exactly (x0 + m*s is exact: both terms and the sum are grid
// multiples below 2^(e+1)).
struct SysSeg {
  int32_t j0;   // first point index of the run
  int32_t pad;
  double x0;    // value of point j0
  double step;  // exact step inside the run (0 for single points)
};

enum { SYS_MAX_SEG = 192 };

PLOM_HD int binade_hi_is_above(double x, double hi) { return x >= hi; }

PLOM_HD double binade_top(double x) {
  // smallest power of two strictly greater than x (x > 0, finite)
  int e;
  frexp(x, &e);  // x = f * 2^e, f in [0.5, 1)
  return ldexp(1.0, e);
}

// Builds the run table for J points starting at U with increment inc.
// Returns the number of runs, or -1 if the table is too small.
PLOM_HD int systematic_table(double U, double inc, int J, SysSeg* seg, int max_seg) {
  int ns = 0;
  int j = 0;
  double x = U;
  while (j < J) {
    if (ns + 2 > max_seg) return -1;
    if (!(x > 0.0)) {  // U == 0: a single point, then continue from inc
      seg[ns].j0 = j; seg[ns].x0 = x; seg[ns].step = 0.0; ++ns;
      ++j;
      x = x + inc;
      continue;
    }
    const double hi = binade_top(x);
    const double x1 = x + inc;
    seg[ns].j0 = j; seg[ns].x0 = x; seg[ns].step = 0.0; ++ns;  // entry point alone
    ++j;
    if (j >= J) break;
    if (x1 >= hi) { x = x1; continue; }
    const double x2 = x1 + inc;
    if (x2 >= hi) {
      seg[ns].j0 = j; seg[ns].x0 = x1; seg[ns].step = 0.0; ++ns;
      ++j;
      x = x2;
      continue;
    }
    const double s = x2 - x1;  // exact
    // number of points x1 + m*s < hi, m >= 0
    double q = (hi - x1) / s;
    long long M = (long long)q;
    if (M < 1) M = 1;
    while ((double)x1 + (double)M * s < hi) ++M;
    while (M > 1 && !((double)x1 + (double)(M - 1) * s < hi)) --M;
    if ((long long)j + M > (long long)J) M = J - j;
    seg[ns].j0 = j; seg[ns].x0 = x1; seg[ns].step = s; ++ns;
    j += (int)M;
    const double last = x1 + (double)(M - 1) * s;
    x = last + inc;
  }
  return ns;
}

PLOM_HD double systematic_point(const SysSeg* seg, int ns, int j) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {  // last run with j0 <= j
    const int mid = (lo + hi + 1) >> 1;
    if (seg[mid].j0 <= j) lo = mid; else hi = mid - 1;
  }
  return seg[lo].x0 + (double)(j - seg[lo].j0) * seg[lo].step;
}

// ---------------------------------------------------------------- incidence sums
// The incidence terms of one substep, summed per unique incidence series in
// cac order before they are added to the state (the order the sum of every
// implementation keeps).  In registers a series index known only at run time
// reaches its register through an unrolled compare chain.
template <class T, int N>
struct RegIncAcc {
  T v[N > 0 ? N : 1];
  PLOM_HD RegIncAcc() {}
  template <class X>
  PLOM_HD explicit RegIncAcc(X&) {}
  PLOM_HD void zero() {
    PLOM_UNROLL
    for (int w = 0; w < N; ++w) v[w] = T(0);
  }
  PLOM_HD void add(int w, T d) {
    PLOM_UNROLL
    for (int ww = 0; ww < N; ++ww)
      if (ww == w) v[ww] += d;
  }
  PLOM_HD T get(int w) const { return v[w]; }
};

// Priors of the natural-scale parameters (normal_prior, pseudo_unif_prior,
// model_builder/C/core/metropolis_hastings_prior.c:95-133; the flat prior is
// gsl_ran_flat_pdf): kind 0 flat on [lo, hi), 1 normal, 2 pseudo-uniform.
PLOM_HD double prior_density(int kind, double x, double lo, double hi) {
  if (kind == 1) {
    const double mean = (hi + lo) / 2.0, sd = (hi - lo) / 4.0;
    const double z = (x - mean) / sd;
    return exp(-0.5 * z * z) / (2.5066282746310002 * sd);
  }
  if (kind == 2) {
    const double delta = 0.01 * (hi - lo);
    const double alpha = 1.0 / (hi - lo - 2.0 / 3.0 * delta);
    const double a = -alpha / (delta * delta);
    const double b = -2.0 * (lo + delta) * a;
    const double c = alpha + a * (lo + delta) * (lo + delta);
    if (x <= lo || x >= hi) return 0.0;
    if (x < lo + delta) return a * x * x + b * x + c;
    if (x < hi - delta) return alpha;
    const double y = x - (hi - lo - 2.0 * delta);
    return a * y * y + b * y + c;
  }
  return (x >= lo && x < hi) ? 1.0 / (hi - lo) : 0.0;
}

// log of a density floored at like_min (sanitize_likelihood, likelihood.c:77-92)
PLOM_HD double log_sanitized(double p, double like_min) {
  if (isnan(p) || isinf(p) || p < 0.0) return log(like_min);
  return log(p <= like_min ? like_min : p);
}

// Accumulator of a particle store X; a store in shared memory may give the
// sums words of their own there (one indexed load / add / store per term).
template <class X, class T, int N>
struct IncAccFor {
  typedef RegIncAcc<T, N> type;
};

}  // namespace plomrt

template <class T> PLOM_HD T plom_heaviside(T x) { return plomrt::heaviside_<T>(x); }
template <class T> PLOM_HD T plom_ramp(T x) { return plomrt::ramp_<T>(x); }
template <class T> PLOM_HD T plom_slowstep(T x, T d) { return plomrt::slowstep_<T>(x, d); }
