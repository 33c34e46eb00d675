// Generated by plomgpu.emit for model "sir".  Do not edit.
#pragma once
#include "plom_rt.h"
#include "psr_samplers.h"
namespace plomgen {
// incidence links of each cac (obs * 1024 + word, -1 after its last), read with a run-time
// cac: from constant memory on the device
#if defined(__CUDACC__)
__constant__ int kIncLinkDev[1] = {0};
#endif
static const int kIncLinkHost[1] = {0};
struct Model {
  static constexpr const char* NAME = "sir";
  static constexpr int N_PAR_SV = 3, N_C = 1, N_AC = 1, N_CAC = 1;
  static constexpr int N_TS = 1, N_TS_INC_UNIQUE = 1, N_OBS_INC = 1, N_OBS_PREV = 0;
  static constexpr int N_DRIFT = 0;  // drifted parameters, N_CAC words each
  static constexpr int OFF_DRIFT = N_PAR_SV*N_CAC, OFF_INC = OFF_DRIFT + N_DRIFT*N_CAC;
  static constexpr int S = OFF_INC + N_TS_INC_UNIQUE;  // words per particle
  static constexpr int N_PAR_PROC = 5, N_PAR_OBS = 2, N_COV_CAC = 1, N_COV_TS = 1;
  static constexpr int N_REAC = 6, N_WN = 1;
  static constexpr bool COUPLED = false;
  static constexpr bool POP_SIZE_EQ_SUM_SV = true;
  static constexpr int COV_N = 0;  // index of N among cac covariates, -1 if none
  // normals drawn per cac and substep for a noise variant (bit0 no dem, bit1 no env)
  static constexpr PLOM_HD int draws_per_cac(int v) { return ((v & 1) ? 0 : N_REAC) + ((v & 2) ? 0 : N_WN); }
  static constexpr int N_INC_LINKS = 1;
  static constexpr int INC_PER_CAC = 1;
  PLOM_HD static int inc_link(int cac, int k) {
#if defined(__CUDA_ARCH__)
    return kIncLinkDev[cac * INC_PER_CAC + k];
#else
    return kIncLinkHost[cac * INC_PER_CAC + k];
#endif
  }
  template <class T>
  struct Pre {
    int unused;
  };
  template <int V, bool DRIFT, class T, class X, class E, class IA>
  PLOM_HD static void cac_body(X& x, const int cac, const T* nz, const T t, const T dt, const E& e,
                               IA& inc_acc, const Pre<T>& pre) {
    (void)t; (void)nz; (void)pre;
    const T xo_S = x[0*N_CAC+cac];
    const T xo_I = x[1*N_CAC+cac];
    const T xo_R = x[2*N_CAC+cac];
    const T r0 = e.par(3, cac)*(xo_I + xo_R + xo_S);
    const T r1 = xo_I*e.par(0, cac)*e.par(1, cac)/(xo_I + xo_R + xo_S);
    const T r2 = e.par(1, cac);
    const T r3 = e.par(4, cac);
    const T sqdt = sqrt(dt);
    (void)sqdt;
    int q = 0; (void)q;
    const T dem_0 = (V & 1) ? T(0) : sqdt*nz[q++];
    const T dem_1 = (V & 1) ? T(0) : sqdt*nz[q++];
    const T dem_2 = (V & 1) ? T(0) : sqdt*nz[q++];
    const T dem_3 = (V & 1) ? T(0) : sqdt*nz[q++];
    const T dem_4 = (V & 1) ? T(0) : sqdt*nz[q++];
    const T dem_5 = (V & 1) ? T(0) : sqdt*nz[q++];
    const T wn_0 = (V & 2) ? T(0) : sqdt*nz[q++];
    T incterm_0;
    switch (V) {
      case 0: incterm_0 = (+ (r2*xo_I))*dt + sqrt(r2*xo_I)*dem_2; break;
      case 1: incterm_0 = (+ (r2*xo_I))*dt; break;
      case 2: incterm_0 = (+ (r2*xo_I))*dt + sqrt(r2*xo_I)*dem_2; break;
      case 3: incterm_0 = (+ (r2*xo_I))*dt; break;
    }
    T f_S;
    switch (V) {
      case 0: f_S = xo_S + (- (r1*xo_S) - (r3*xo_S) + (r0))*dt - sqrt(r1*xo_S)*dem_1 - sqrt(r3*xo_S)*dem_3 + sqrt(r0)*dem_0 - (r1*xo_S)*e.par(2, cac)*wn_0; break;
      case 1: f_S = xo_S + (- (r1*xo_S) - (r3*xo_S) + (r0))*dt - (r1*xo_S)*e.par(2, cac)*wn_0; break;
      case 2: f_S = xo_S + (- (r1*xo_S) - (r3*xo_S) + (r0))*dt - sqrt(r1*xo_S)*dem_1 - sqrt(r3*xo_S)*dem_3 + sqrt(r0)*dem_0; break;
      case 3: f_S = xo_S + (- (r1*xo_S) - (r3*xo_S) + (r0))*dt; break;
    }
    T f_I;
    switch (V) {
      case 0: f_I = xo_I + (- (r2*xo_I) - (r3*xo_I) + (r1*xo_S))*dt - sqrt(r2*xo_I)*dem_2 - sqrt(r3*xo_I)*dem_4 + sqrt(r1*xo_S)*dem_1 + (r1*xo_S)*e.par(2, cac)*wn_0; break;
      case 1: f_I = xo_I + (- (r2*xo_I) - (r3*xo_I) + (r1*xo_S))*dt + (r1*xo_S)*e.par(2, cac)*wn_0; break;
      case 2: f_I = xo_I + (- (r2*xo_I) - (r3*xo_I) + (r1*xo_S))*dt - sqrt(r2*xo_I)*dem_2 - sqrt(r3*xo_I)*dem_4 + sqrt(r1*xo_S)*dem_1; break;
      case 3: f_I = xo_I + (- (r2*xo_I) - (r3*xo_I) + (r1*xo_S))*dt; break;
    }
    T f_R;
    switch (V) {
      case 0: f_R = xo_R + (- (r3*xo_R) + (r2*xo_I))*dt - sqrt(r3*xo_R)*dem_5 + sqrt(r2*xo_I)*dem_2; break;
      case 1: f_R = xo_R + (- (r3*xo_R) + (r2*xo_I))*dt; break;
      case 2: f_R = xo_R + (- (r3*xo_R) + (r2*xo_I))*dt - sqrt(r3*xo_R)*dem_5 + sqrt(r2*xo_I)*dem_2; break;
      case 3: f_R = xo_R + (- (r3*xo_R) + (r2*xo_I))*dt; break;
    }
    PLOM_UNROLL
    for (int k = 0; k < INC_PER_CAC; ++k) {
      const int l = inc_link(cac, k);
      if (l < 0) break;
      const int o = l >> 10, w = l & 1023;
      if (o == 0) inc_acc.add(w, incterm_0);
    }
    x[0*N_CAC+cac] = (f_S < T(0)) ? T(0) : f_S;
    x[1*N_CAC+cac] = (f_I < T(0)) ? T(0) : f_I;
    x[2*N_CAC+cac] = (f_R < T(0)) ? T(0) : f_R;
  }
  // cacs drawn together so that whole draw blocks are used (PER_BLOCK normals per block);
  // for generators of more than 2 normals per block (FP32) PLOM_MAX_DRAW_GROUP caps the
  // group, leaving part of the last block of a group unused (SEIR 20x2: 4 cacs = 9 whole
  // blocks measured 10 % faster than 1 cac = 3 blocks with 3 of their 12 normals unused)
  // without draws (Euler skeleton) a group of 4 cacs only sets the unrolling of the cac loop
  static constexpr PLOM_HD int draw_group(int nw, int per_block) {
    if (nw == 0) return N_CAC >= 4 ? 4 : 1;
    int g = 1;
    while (nw > 0 && (g * nw) % per_block != 0 && g < per_block) ++g;
    g = (nw > 0 && (g * nw) % per_block == 0 && g <= N_CAC) ? g : 1;
#if defined(PLOM_MAX_DRAW_GROUP)
    if (per_block > 2 && g > PLOM_MAX_DRAW_GROUP) g = PLOM_MAX_DRAW_GROUP;
#endif
    return g;
  }
  template <int V, bool DRIFT, class T, class X, class E, class D>
  PLOM_HD static void step(X& x, const T t, const T dt, const E& e, D& draws) {
    constexpr int NW = draws_per_cac(V);
    constexpr int G = draw_group(NW, D::PER_BLOCK);
    constexpr int NMAIN = N_CAC - (N_CAC % G);
    typename plomrt::IncAccFor<X, T, N_TS_INC_UNIQUE>::type inc_acc(x);
    inc_acc.zero();
    Pre<T> pre;
    pre.unused = 0;
    PLOM_PRAGMA_CAC
    for (int cac0 = 0; cac0 < NMAIN; cac0 += G) {
      T nz[NW * G > 0 ? NW * G : 1];
      draws.template normals<NW * G>(cac0, nz);
      PLOM_PRAGMA_GROUP
      for (int g = 0; g < G; ++g) cac_body<V, DRIFT, T>(x, cac0 + g, nz + g * NW, t, dt, e, inc_acc, pre);
    }
    PLOM_UNROLL
    for (int cac = NMAIN; cac < N_CAC; ++cac) {
      T nz[NW > 0 ? NW : 1];
      draws.template normals<NW>(cac, nz);
      cac_body<V, DRIFT, T>(x, cac, nz, t, dt, e, inc_acc, pre);
    }
    PLOM_UNROLL
    for (int w = 0; w < N_TS_INC_UNIQUE; ++w) {
      const T f = x[OFF_INC+w] + inc_acc.get(w);
      x[OFF_INC+w] = (f < T(0)) ? T(0) : f;
    }
    if (DRIFT) {
      // Brownian walk of the drifted parameters (model_builder/C/core/drift.c:27-41)
      PLOM_UNROLL
      for (int i = 0; i < N_DRIFT; ++i) {
        const int ng = e.drift_ngroups(i);
        PLOM_UNROLL
        for (int g = 0; g < N_CAC; ++g) {
          if (g < ng) x[OFF_DRIFT+i*N_CAC+g] += e.drift_vol(i, g)*sqrt(dt)*draws.drift_normal(i, g);
        }
      }
    }
  }
  template <int V, bool DRIFT, class T, class X, class E, class D, class TM>
  PLOM_HD static void step_team(X& x, const T t, const T dt, const E& e, D& draws, const TM& tm, Pre<T>& pre) {
    constexpr int NW = draws_per_cac(V);
    constexpr int G = draw_group(NW, D::PER_BLOCK);
    constexpr int NG = N_CAC / G;
    constexpr int NMAIN = NG * G;
    plomrt::RegIncAcc<T, N_TS_INC_UNIQUE> inc_acc;
    inc_acc.zero();
    PLOM_PRAGMA_CAC
    for (int gi = tm.rank; gi < NG; gi += TM::TP) {
      const int cac0 = gi * G;
      T nz[NW * G > 0 ? NW * G : 1];
      draws.template normals<NW * G>(cac0, nz);
      PLOM_UNROLL
      for (int g = 0; g < G; ++g) cac_body<V, DRIFT, T>(x, cac0 + g, nz + g * NW, t, dt, e, inc_acc, pre);
    }
    for (int cac = NMAIN + tm.rank; cac < N_CAC; cac += TM::TP) {
      T nz[NW > 0 ? NW : 1];
      draws.template normals<NW>(cac, nz);
      cac_body<V, DRIFT, T>(x, cac, nz, t, dt, e, inc_acc, pre);
    }
    PLOM_UNROLL
    for (int w = 0; w < N_TS_INC_UNIQUE; ++w) inc_acc.v[w] = tm.sum(inc_acc.v[w]);
    tm.sync();
    if (tm.rank == 0) {
      PLOM_UNROLL
      for (int w = 0; w < N_TS_INC_UNIQUE; ++w) {
        const T f = x[OFF_INC+w] + inc_acc.v[w];
        x[OFF_INC+w] = (f < T(0)) ? T(0) : f;
      }
    }
    if (DRIFT) {
      for (int i = 0; i < N_DRIFT; ++i) {
        const int ng = e.drift_ngroups(i);
        for (int g = tm.rank; g < ng; g += TM::TP)
          x[OFF_DRIFT+i*N_CAC+g] += e.drift_vol(i, g)*sqrt(dt)*draws.drift_normal(i, g);
      }
    }
    tm.sync();
  }
  template <class T, class X, class F, class E>
  PLOM_HD static void deriv(const X& x, F& f, const T t, const E& e) {
    (void)t;
    T inc_acc[N_TS_INC_UNIQUE > 0 ? N_TS_INC_UNIQUE : 1];
    for (int w = 0; w < N_TS_INC_UNIQUE; ++w) inc_acc[w] = T(0);
    Pre<T> pre;
    pre.unused = 0;
    for (int cac = 0; cac < N_CAC; ++cac) {
      const T xo_S = x[0*N_CAC+cac];
      const T xo_I = x[1*N_CAC+cac];
      const T xo_R = x[2*N_CAC+cac];
      const T r0 = e.par(3, cac)*(xo_I + xo_R + xo_S);
      const T r1 = xo_I*e.par(0, cac)*e.par(1, cac)/(xo_I + xo_R + xo_S);
      const T r2 = e.par(1, cac);
      const T r3 = e.par(4, cac);
      const T incterm_0 = + (r2*xo_I);
      f[0*N_CAC+cac] = - (r1*xo_S) - (r3*xo_S) + (r0);
      f[1*N_CAC+cac] = - (r2*xo_I) - (r3*xo_I) + (r1*xo_S);
      f[2*N_CAC+cac] = - (r3*xo_R) + (r2*xo_I);
      for (int k = 0; k < INC_PER_CAC; ++k) {
        const int l = inc_link(cac, k);
        if (l < 0) break;
        const int o = l >> 10, w = l & 1023;
        if (o == 0) inc_acc[w] += incterm_0;
      }
    }
    for (int w = OFF_DRIFT; w < OFF_INC; ++w) f[w] = T(0);
    for (int w = 0; w < N_TS_INC_UNIQUE; ++w) f[OFF_INC+w] = inc_acc[w];
  }
  template <bool DRIFT, bool NOENV, class T, class X, class E, class IA>
  PLOM_HD static void psr_cac(X& x, const int cac, const T t, const T dt, const E& e,
                              typename plomrt::PsrStream<T>::type& rs, IA& inc_acc, const Pre<T>& pre) {
    (void)t; (void)pre;
    const T ddt = dt;
    const T xo_S = x[0*N_CAC+cac];
    const T xo_I = x[1*N_CAC+cac];
    const T xo_R = x[2*N_CAC+cac];
    T wn_0 = T(1);
    if (!NOENV) {
      const T sd = (T)(e.par(2, cac));
      wn_0 = plomrt::gamma(rs, ddt / (sd * sd), sd * sd) / ddt;
    }
    const T r0 = e.par(3, cac)*(xo_I + xo_R + xo_S);
    const T r1 = xo_I*e.par(0, cac)*e.par(1, cac)/(xo_I + xo_R + xo_S);
    const T r2 = e.par(1, cac);
    const T r3 = e.par(4, cac);
    T inc_S[3];
    {
      const T h0 = r1*wn_0 * ddt;
      const T h1 = r3 * ddt;
      const T sum = h0 + h1;
      T p[3];
      if (sum > T(0)) {
        const T ome = T(1) - plomrt::s_exp(-sum);
        p[0] = ome * (h0 / sum);
        p[1] = ome * (h1 / sum);
        p[2] = T(1) - p[0] - p[1];
      } else {
        p[0] = T(0);
        p[1] = T(0);
        p[2] = T(1);
      }
      const T xs = xo_S;
      plomrt::multinomial<3>(rs, xs > T(0) ? floor(xs) : T(0), p, inc_S);
    }
    T inc_I[3];
    {
      const T h0 = r2 * ddt;
      const T h1 = r3 * ddt;
      const T sum = h0 + h1;
      T p[3];
      if (sum > T(0)) {
        const T ome = T(1) - plomrt::s_exp(-sum);
        p[0] = ome * (h0 / sum);
        p[1] = ome * (h1 / sum);
        p[2] = T(1) - p[0] - p[1];
      } else {
        p[0] = T(0);
        p[1] = T(0);
        p[2] = T(1);
      }
      const T xs = xo_I;
      plomrt::multinomial<3>(rs, xs > T(0) ? floor(xs) : T(0), p, inc_I);
    }
    T inc_R[2];
    {
      const T h0 = r3 * ddt;
      const T sum = h0;
      T p[2];
      if (sum > T(0)) {
        const T ome = T(1) - plomrt::s_exp(-sum);
        p[0] = ome * (h0 / sum);
        p[1] = T(1) - p[0];
      } else {
        p[0] = T(0);
        p[1] = T(1);
      }
      const T xs = xo_R;
      plomrt::multinomial<2>(rs, xs > T(0) ? floor(xs) : T(0), p, inc_R);
    }
    T inc_U[1];
    inc_U[0] = plomrt::poisson(rs, r0 * ddt);
    x[0*N_CAC+cac] = (T)(inc_S[2] + inc_U[0]);
    x[1*N_CAC+cac] = (T)(inc_I[2] + inc_S[0]);
    x[2*N_CAC+cac] = (T)(inc_R[1] + inc_I[0]);
    for (int k = 0; k < INC_PER_CAC; ++k) {
      const int l = inc_link(cac, k);
      if (l < 0) break;
      const int o = l >> 10, w = l & 1023;
      if (o == 0) inc_acc.add(w, inc_I[0]);
    }
  }
  template <bool DRIFT, bool NOENV, class T, class X, class E, class D>
  PLOM_HD static void step_psr(X& x, const T t, const T dt, const E& e, const plomrt::PhiloxKey key,
                               const uint32_t j, const uint32_t n, const uint32_t sub, D& draws) {
    typename plomrt::IncAccFor<X, T, N_TS_INC_UNIQUE>::type inc_acc(x);
    inc_acc.zero();
    Pre<T> pre;
    pre.unused = 0;
    for (int cac = 0; cac < N_CAC; ++cac) {
      typename plomrt::PsrStream<T>::type rs;
      rs.init(key, j, n, sub * (uint32_t)(N_CAC + 1) + (uint32_t)cac);
      psr_cac<DRIFT, NOENV, T>(x, cac, t, dt, e, rs, inc_acc, pre);
    }
    PLOM_UNROLL
    for (int w = 0; w < N_TS_INC_UNIQUE; ++w) x[OFF_INC+w] = x[OFF_INC+w] + inc_acc.get(w);
    if (DRIFT) {
      // Brownian walk of the drifted parameters (model_builder/C/core/drift.c:27-41)
      for (int i = 0; i < N_DRIFT; ++i) {
        const int ng = e.drift_ngroups(i);
        for (int g = 0; g < ng; ++g)
          x[OFF_DRIFT+i*N_CAC+g] += e.drift_vol(i, g)*sqrt(dt)*draws.drift_normal(i, g);
      }
    }
  }
  template <class T, class X>
  PLOM_HD static void proj2obs(const X& x, double* obs) {
    obs[0] = (double)x[OFF_INC+0];
  }
  // observation model, evaluated in double (Ccoder.print_like)
  template <class E>
  PLOM_HD static double obs_mean(const double x, const int ts, const double t, const E& e) {
    typedef double T; (void)x; (void)ts; (void)t; (void)e;
    return e.cov_ts(0, ts)*e.par_ts(0, ts)*x;
  }
  template <class E>
  PLOM_HD static double obs_var(const double x, const int ts, const double t, const E& e) {
    typedef double T; (void)x; (void)ts; (void)t; (void)e;
    return (e.par_ts(1, ts)*e.par_ts(1, ts))*(e.cov_ts(0, ts)*e.cov_ts(0, ts))*(e.par_ts(0, ts)*e.par_ts(0, ts))*(x*x) + e.cov_ts(0, ts)*e.par_ts(0, ts)*x*(T(1.0) - e.par_ts(0, ts));
  }
};
}  // namespace plomgen
