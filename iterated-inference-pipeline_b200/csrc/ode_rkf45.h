// Deterministic skeleton of a model integrated with an embedded
// Runge-Kutta-Fehlberg 4(5) pair and the standard step-size control, the
// method of the reference's ``ode`` implementation (gsl_odeiv2_step_rkf45 +
// gsl_odeiv2_control_y_new(eps_abs, eps_rel) driven by
// gsl_odeiv2_evolve_apply, model_builder/C/core/build.c:1034-1037 and
// model_builder/C/core/prediction_util.c:176-193).
//
// * Tableau: Fehlberg's 1969 coefficients; the fifth-order solution is
//   propagated and its difference with the fourth-order one is the error
//   estimate.
// * Control (the documented "standard" rule with a_y = 1, a_dydt = 0):
//   D_i = eps_abs + eps_rel |y_i|, r = max_i |err_i| / D_i.  r > 1.1: the step
//   is retried with h * max(0.2, 0.9 r^(-1/5)); r < 0.5: the next step is
//   h * min(5, max(1, 0.9 r^(-1/6))); otherwise h is kept.
// * Each observation interval starts again from the initial step DT (the
//   reference's step size is a local of f_prediction_ode); the last step is
//   shortened to end on t1.
// Covariates are evaluated at every stage time from their interpolants
// (gsl_spline_eval inside step_ode).  Shared by the GPU engine and the oracle.
#pragma once

#include "plom_rt.h"

namespace plomrt {

// Interpolants of the per-cac covariates, restating the host's Spline:
// kind 0 constant, 1 linear, 2 natural cubic (second derivatives m2); the end
// values are kept outside the knots.
struct CovSplines {
  const int* meta;   // [n][3]: kind, number of knots, offset into x / y / m2
  const double* x;
  const double* y;
  const double* m2;
  PLOM_HD double eval(int idx, double t) const {
    const int kind = meta[3 * idx], n = meta[3 * idx + 1], off = meta[3 * idx + 2];
    const double* xs = x + off;
    const double* ys = y + off;
    if (kind == 0 || n == 1) return ys[0];
    if (t <= xs[0]) return ys[0];
    if (t >= xs[n - 1]) return ys[n - 1];
    int lo = 0, hi = n - 1;  // xs[lo] <= t < xs[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (xs[mid] <= t) lo = mid; else hi = mid;
    }
    const double h = xs[lo + 1] - xs[lo];
    const double a = (xs[lo + 1] - t) / h, b = (t - xs[lo]) / h;
    if (kind == 1) return a * ys[lo] + b * ys[lo + 1];
    const double* ms = m2 + off;
    return a * ys[lo] + b * ys[lo + 1] + ((a * a * a - a) * ms[lo] + (b * b * b - b) * ms[lo + 1]) * h * h / 6.0;
  }
};

enum { ODE_OK = 0, ODE_STEP_UNDERFLOW = 1, ODE_TOO_MANY_STEPS = 2 };

template <class T>
struct ArrayView {
  const T* p;
  PLOM_HD T operator[](int w) const { return p[w]; }
};

// Integrates y (the model's S state words) from t0 to t1.  Env exposes a
// writable covariate buffer covl_ ([N_COV_CAC][N_CAC]) that its cov() reads;
// work holds 8 * S values.  Returns ODE_OK or an error code; *n_steps counts
// the attempted steps.
template <class Model, class T, class Env>
PLOM_HD int rkf45_interval(T* y, double t0, double t1, double h_init, double eps_abs, double eps_rel, Env& e,
                           const CovSplines& cs, T* work, int max_steps, int* n_steps) {
  constexpr int S = Model::S;
  constexpr int NCOV = Model::N_COV_CAC * Model::N_CAC;
  T* k1 = work;
  T* k2 = k1 + S;
  T* k3 = k2 + S;
  T* k4 = k3 + S;
  T* k5 = k4 + S;
  T* k6 = k5 + S;
  T* yt = k6 + S;
  T* y5 = yt + S;
  auto rhs = [&](const T* yy, T* f, double ts) {
    for (int i = 0; i < NCOV; ++i) e.covl_[i] = (T)cs.eval(i, ts);
    const ArrayView<T> v{yy};
    Model::template deriv<T>(v, f, (T)ts, e);
  };
  // Fehlberg (1969)
  const double c2 = 1.0 / 4, c3 = 3.0 / 8, c4 = 12.0 / 13, c5 = 1.0, c6 = 1.0 / 2;
  const double a21 = 1.0 / 4;
  const double a31 = 3.0 / 32, a32 = 9.0 / 32;
  const double a41 = 1932.0 / 2197, a42 = -7200.0 / 2197, a43 = 7296.0 / 2197;
  const double a51 = 439.0 / 216, a52 = -8.0, a53 = 3680.0 / 513, a54 = -845.0 / 4104;
  const double a61 = -8.0 / 27, a62 = 2.0, a63 = -3544.0 / 2565, a64 = 1859.0 / 4104, a65 = -11.0 / 40;
  const double b1 = 16.0 / 135, b3 = 6656.0 / 12825, b4 = 28561.0 / 56430, b5 = -9.0 / 50, b6 = 2.0 / 55;
  const double e1 = 1.0 / 360, e3 = -128.0 / 4275, e4 = -2197.0 / 75240, e5 = 1.0 / 50, e6 = 2.0 / 55;
  double t = t0, h = h_init;
  int steps = 0;
  while (t < t1) {
    double h0 = h;
    if (h0 > t1 - t) h0 = t1 - t;
    for (;;) {
      if (++steps > max_steps) {
        *n_steps = steps;
        return ODE_TOO_MANY_STEPS;
      }
      if (!(h0 > 0.0) || t + h0 == t) {
        *n_steps = steps;
        return ODE_STEP_UNDERFLOW;
      }
      const T H = (T)h0;
      rhs(y, k1, t);
      for (int i = 0; i < S; ++i) yt[i] = y[i] + H * (T)a21 * k1[i];
      rhs(yt, k2, t + c2 * h0);
      for (int i = 0; i < S; ++i) yt[i] = y[i] + H * ((T)a31 * k1[i] + (T)a32 * k2[i]);
      rhs(yt, k3, t + c3 * h0);
      for (int i = 0; i < S; ++i) yt[i] = y[i] + H * ((T)a41 * k1[i] + (T)a42 * k2[i] + (T)a43 * k3[i]);
      rhs(yt, k4, t + c4 * h0);
      for (int i = 0; i < S; ++i)
        yt[i] = y[i] + H * ((T)a51 * k1[i] + (T)a52 * k2[i] + (T)a53 * k3[i] + (T)a54 * k4[i]);
      rhs(yt, k5, t + c5 * h0);
      for (int i = 0; i < S; ++i)
        yt[i] = y[i] + H * ((T)a61 * k1[i] + (T)a62 * k2[i] + (T)a63 * k3[i] + (T)a64 * k4[i] + (T)a65 * k5[i]);
      rhs(yt, k6, t + c6 * h0);
      double rmax = 0.0;
      bool bad = false;
      for (int i = 0; i < S; ++i) {
        y5[i] = y[i] + H * ((T)b1 * k1[i] + (T)b3 * k3[i] + (T)b4 * k4[i] + (T)b5 * k5[i] + (T)b6 * k6[i]);
        const double err =
            (double)(H * ((T)e1 * k1[i] + (T)e3 * k3[i] + (T)e4 * k4[i] + (T)e5 * k5[i] + (T)e6 * k6[i]));
        const double D = eps_abs + eps_rel * fabs((double)y5[i]);
        const double r = fabs(err) / D;
        if (r != r) bad = true;
        else if (r > rmax) rmax = r;
      }
      if (bad) rmax = 1e300;  // a NaN error estimate is a failed step
      if (rmax > 1.1) {
        double f = 0.9 / pow(rmax, 1.0 / 5.0);
        if (f < 0.2) f = 0.2;
        h0 *= f;
        continue;  // retry the step from t with the smaller h
      }
      for (int i = 0; i < S; ++i) y[i] = y5[i];
      const bool final_step = (t + h0 >= t1);
      t = final_step ? t1 : t + h0;
      h = h0;
      if (rmax < 0.5) {
        double f = (rmax > 0.0) ? 0.9 / pow(rmax, 1.0 / 6.0) : 5.0;
        if (f > 5.0) f = 5.0;
        if (f < 1.0) f = 1.0;
        h = h0 * f;
      }
      break;
    }
  }
  *n_steps = steps;
  return ODE_OK;
}

}  // namespace plomrt
