// Host drivers above the device pair sums: profile fitting (crabSAXS
// src/fit.rs:84-454), maximum-entropy reweighting (src/reweight.rs:84-374) and
// ensemble population fitting (src/ensemble.rs:127-465).  These loops work on
// vectors of length Nq (or K x Nq) and stay in f64 on the host; the
// O(N²·Nq) basis evaluation underneath runs on the device.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>

#include "engine.hpp"
#include "ops.hpp"

namespace crab {
namespace {

// fit.rs:84-91
std::vector<size_t> sampled_indices(size_t length, size_t stride) {
  const size_t st = length < 64 ? 1 : std::max<size_t>(stride, 1);
  std::vector<size_t> idx;
  for (size_t i = 0; i < length; i += st) idx.push_back(i);
  if (idx.empty() || idx.back() != length - 1) idx.push_back(length - 1);
  return idx;
}

// fit.rs:93-123
std::vector<double> cubic_hermite(const std::vector<double>& x, const double* y, const double* t, int64_t nt) {
  std::vector<double> out(nt);
  const size_t n = x.size();
  if (n == 1) {
    std::fill(out.begin(), out.end(), y[0]);
    return out;
  }
  std::vector<double> sl(n);
  const size_t last = n - 1;
  sl[0] = (y[1] - y[0]) / (x[1] - x[0]);
  sl[last] = (y[last] - y[last - 1]) / (x[last] - x[last - 1]);
  for (size_t i = 1; i < last; ++i) sl[i] = (y[i + 1] - y[i - 1]) / (x[i + 1] - x[i - 1]);
  size_t seg = 0;
  for (int64_t k = 0; k < nt; ++k) {
    while (seg + 1 < last && t[k] > x[seg + 1]) ++seg;
    const double h = x[seg + 1] - x[seg];
    const double u = std::fmin(std::fmax((t[k] - x[seg]) / h, 0.0), 1.0);
    const double u2 = u * u, u3 = u2 * u;
    out[k] = (2.0 * u3 - 3.0 * u2 + 1.0) * y[seg] + (u3 - 2.0 * u2 + u) * h * sl[seg] +
             (-2.0 * u3 + 3.0 * u2) * y[seg + 1] + (u3 - u2) * h * sl[seg + 1];
  }
  return out;
}

struct Data {
  const double* q;
  const double* y;
  const double* sigma;
  int64_t n;
};

// fit.rs:137-244 (scale and background solved in closed form)
void solve_scale_background(const double* th, const Data& d, int scale_mode, double scale_value, int bg_mode,
                            double bg_value, double* so, double* bo, double* chi_out) {
  double scale, bg;
  if (scale_mode == CRAB_SCALE_FIT) {
    double sw = 0, sx = 0, sy = 0, sxx = 0, sxy = 0;
    for (int64_t i = 0; i < d.n; ++i) {
      const double x = th[i], w = 1.0 / (d.sigma[i] * d.sigma[i]);
      sw += w;
      sx += w * x;
      sy += w * d.y[i];
      sxx += w * x * x;
      sxy += w * x * d.y[i];
    }
    if (bg_mode == CRAB_BG_FIT) {
      const double det = sxx * sw - sx * sx;
      scale = std::fmax(std::fabs(det) > 1e-20 ? (sxy * sw - sx * sy) / det : 0.0, 0.0);
      bg = sw > 0.0 ? (sy - scale * sx) / sw : 0.0;
    } else if (bg_mode == CRAB_BG_FIXED_ZERO) {
      scale = std::fmax(sxx > 0.0 ? sxy / sxx : 0.0, 0.0);
      bg = 0.0;
    } else {
      scale = std::fmax(sxx > 0.0 ? (sxy - bg_value * sx) / sxx : 0.0, 0.0);
      bg = bg_value;
    }
  } else {
    scale = std::fmax(scale_value, 0.0);
    if (bg_mode == CRAB_BG_FIT) {
      double weighted = 0, weight = 0;
      for (int64_t i = 0; i < d.n; ++i) {
        const double w = 1.0 / (d.sigma[i] * d.sigma[i]);
        weighted += w * (d.y[i] - scale * th[i]);
        weight += w;
      }
      bg = weight > 0.0 ? weighted / weight : 0.0;
    } else if (bg_mode == CRAB_BG_FIXED_ZERO) bg = 0.0;
    else bg = bg_value;
  }
  const double dof = (double)std::max<int64_t>(d.n - 1, 1);
  double chi = 0.0;
  for (int64_t i = 0; i < d.n; ++i) {
    const double r = (scale * th[i] + bg - d.y[i]) / d.sigma[i];
    chi += r * r;
  }
  *so = scale;
  *bo = bg;
  *chi_out = chi / dof;
}

struct Objective {
  const std::vector<double>* basis;  // [6][n]
  Data d;
  double c1_lo, c1_hi, c2_lo, c2_hi;
  int scale_mode, bg_mode;
  double scale_value, bg_value;
  mutable std::vector<double> curve;

  // fit.rs:256-273 (penalised outside the box)
  double cost(double c1, double c2) const {
    if (!(c1 >= c1_lo && c1 <= c1_hi) || !(c2 >= c2_lo && c2 <= c2_hi)) {
      const double d1 = std::fmax(c1_lo - c1, 0.0) + std::fmax(c1 - c1_hi, 0.0);
      const double d2 = std::fmax(c2_lo - c2, 0.0) + std::fmax(c2 - c2_hi, 0.0);
      return 1e20 + 1e20 * (d1 * d1 + d2 * d2);
    }
    curve.resize(d.n);
    combine_basis(d.q, d.n, basis->data(), c1, c2, curve.data());
    double s, b, chi;
    solve_scale_background(curve.data(), d, scale_mode, scale_value, bg_mode, bg_value, &s, &b, &chi);
    return chi;
  }

  // Gradient of the profiled objective with respect to (c1, c2): the
  // derivative through I(q) at the optimal (scale, background).
  double cost_grad(double c1, double c2, double* g) const {
    curve.resize(d.n);
    combine_basis(d.q, d.n, basis->data(), c1, c2, curve.data());
    double s, b, chi;
    solve_scale_background(curve.data(), d, scale_mode, scale_value, bg_mode, bg_value, &s, &b, &chi);
    const double dof = (double)std::max<int64_t>(d.n - 1, 1);
    const double* B = basis->data();
    const int64_t n = d.n;
    g[0] = g[1] = 0.0;
    for (int64_t k = 0; k < n; ++k) {
      if (curve[k] <= 0.0) continue;  // clamped at zero
      const double qq = d.q[k];
      const double G = excluded_volume_scale(qq, c1);
      const double dG = G * (3.0 / c1 - 2.0 * c1 * (1.62 * 1.62) * qq * qq / 4.0);
      const double dIdG = 2.0 * G * B[n + k] - 2.0 * B[3 * n + k] - 2.0 * c2 * B[5 * n + k];
      const double dIdc2 = 2.0 * c2 * B[2 * n + k] + 2.0 * B[4 * n + k] - 2.0 * G * B[5 * n + k];
      const double w = 2.0 * s * (s * curve[k] + b - d.y[k]) / (d.sigma[k] * d.sigma[k]) / dof;
      g[0] += w * dIdG * dG;
      g[1] += w * dIdc2;
    }
    return chi;
  }
};

// Nelder–Mead over (c1, c2) following argmin 0.10's NelderMead: reflection
// 1, expansion 2, contraction 0.5, shrink 0.5; stops when the standard
// deviation of the vertex costs falls below sd_tolerance (fit.rs:401-418).
struct NMResult {
  double c1, c2;
  int iterations;
  bool converged;
};
NMResult nelder_mead(const Objective& f, double c1, double c2, double step1, double step2, int max_iter,
                     double sd_tol) {
  auto offset = [](double v, double step, double hi) { return v + step <= hi ? v + step : v - step; };
  struct V {
    double x[2];
    double c;
  };
  std::vector<V> s(3);
  s[0] = {{c1, c2}, 0};
  s[1] = {{offset(c1, step1, f.c1_hi), c2}, 0};
  s[2] = {{c1, offset(c2, step2, f.c2_hi)}, 0};
  for (auto& v : s) v.c = f.cost(v.x[0], v.x[1]);
  auto sort = [&]() { std::stable_sort(s.begin(), s.end(), [](const V& a, const V& b) { return a.c < b.c; }); };
  sort();
  int it = 0;
  bool converged = false;
  for (; it < max_iter; ++it) {
    const double mean = (s[0].c + s[1].c + s[2].c) / 3.0;
    double var = 0.0;
    for (auto& v : s) var += (v.c - mean) * (v.c - mean);
    if (std::sqrt(var / 2.0) < sd_tol) {
      converged = true;
      break;
    }
    double x0[2];
    for (int d = 0; d < 2; ++d) x0[d] = (s[0].x[d] + s[1].x[d]) / 2.0;
    V xr;
    for (int d = 0; d < 2; ++d) xr.x[d] = x0[d] + 1.0 * (x0[d] - s[2].x[d]);
    xr.c = f.cost(xr.x[0], xr.x[1]);
    if (xr.c < s[1].c && xr.c >= s[0].c) {
      s[2] = xr;
    } else if (xr.c < s[0].c) {
      V xe;
      for (int d = 0; d < 2; ++d) xe.x[d] = x0[d] + 2.0 * (xr.x[d] - x0[d]);
      xe.c = f.cost(xe.x[0], xe.x[1]);
      s[2] = xe.c < xr.c ? xe : xr;
    } else {
      V xc;
      for (int d = 0; d < 2; ++d) xc.x[d] = x0[d] + 0.5 * (s[2].x[d] - x0[d]);
      xc.c = f.cost(xc.x[0], xc.x[1]);
      if (xc.c < s[2].c) s[2] = xc;
      else
        for (int v = 1; v < 3; ++v) {
          for (int d = 0; d < 2; ++d) s[v].x[d] = s[0].x[d] + 0.5 * (s[v].x[d] - s[0].x[d]);
          s[v].c = f.cost(s[v].x[0], s[v].x[1]);
        }
    }
    sort();
  }
  return {s[0].x[0], s[0].x[1], it, converged};
}

// Projected L-BFGS over the (c1, c2) box with Armijo backtracking on the
// analytic gradient.
NMResult lbfgs_box(const Objective& f, double c1, double c2, int max_iter) {
  const int m = 5;
  double x[2] = {c1, c2}, g[2];
  double fx = f.cost_grad(x[0], x[1], g);
  std::vector<std::array<double, 2>> S, Y;
  auto project = [&](double* v) {
    v[0] = std::fmin(std::fmax(v[0], f.c1_lo), f.c1_hi);
    v[1] = std::fmin(std::fmax(v[1], f.c2_lo), f.c2_hi);
  };
  int it = 0;
  bool converged = false;
  for (; it < max_iter; ++it) {
    // projected-gradient stationarity
    double pg[2] = {x[0] - g[0], x[1] - g[1]};
    project(pg);
    const double pgn = std::fabs(pg[0] - x[0]) + std::fabs(pg[1] - x[1]);
    if (pgn < 1e-10 * (1.0 + std::fabs(fx))) {
      converged = true;
      break;
    }
    // two-loop recursion
    double d[2] = {-g[0], -g[1]};
    std::vector<double> alpha(S.size());
    for (int i = (int)S.size() - 1; i >= 0; --i) {
      const double rho = 1.0 / (S[i][0] * Y[i][0] + S[i][1] * Y[i][1]);
      alpha[i] = rho * (S[i][0] * d[0] + S[i][1] * d[1]);
      d[0] -= alpha[i] * Y[i][0];
      d[1] -= alpha[i] * Y[i][1];
    }
    if (!S.empty()) {
      const auto& s = S.back();
      const auto& y = Y.back();
      const double gamma = (s[0] * y[0] + s[1] * y[1]) / (y[0] * y[0] + y[1] * y[1]);
      d[0] *= gamma;
      d[1] *= gamma;
    } else {
      const double gn = std::sqrt(g[0] * g[0] + g[1] * g[1]);
      const double scale = gn > 0 ? 0.01 / gn : 0.0;
      d[0] *= scale;
      d[1] *= scale;
    }
    for (size_t i = 0; i < S.size(); ++i) {
      const double rho = 1.0 / (S[i][0] * Y[i][0] + S[i][1] * Y[i][1]);
      const double beta = rho * (Y[i][0] * d[0] + Y[i][1] * d[1]);
      d[0] += (alpha[i] - beta) * S[i][0];
      d[1] += (alpha[i] - beta) * S[i][1];
    }
    if (d[0] * g[0] + d[1] * g[1] >= 0.0) {  // not a descent direction: restart
      S.clear();
      Y.clear();
      d[0] = -g[0];
      d[1] = -g[1];
      const double gn = std::sqrt(g[0] * g[0] + g[1] * g[1]);
      if (gn > 0) { d[0] *= 0.01 / gn; d[1] *= 0.01 / gn; }
    }
    double step = 1.0, xn[2], gn2[2], fn = fx;
    bool accepted = false;
    for (int ls = 0; ls < 40; ++ls) {
      xn[0] = x[0] + step * d[0];
      xn[1] = x[1] + step * d[1];
      project(xn);
      fn = f.cost_grad(xn[0], xn[1], gn2);
      const double dec = g[0] * (xn[0] - x[0]) + g[1] * (xn[1] - x[1]);
      if (fn <= fx + 1e-4 * dec) {
        accepted = true;
        break;
      }
      step *= 0.5;
    }
    if (!accepted) {
      converged = true;
      break;
    }
    std::array<double, 2> sv = {xn[0] - x[0], xn[1] - x[1]}, yv = {gn2[0] - g[0], gn2[1] - g[1]};
    if (sv[0] * yv[0] + sv[1] * yv[1] > 1e-300) {
      S.push_back(sv);
      Y.push_back(yv);
      if ((int)S.size() > m) {
        S.erase(S.begin());
        Y.erase(Y.begin());
      }
    }
    const double df = std::fabs(fx - fn);
    x[0] = xn[0];
    x[1] = xn[1];
    g[0] = gn2[0];
    g[1] = gn2[1];
    fx = fn;
    if (df <= 1e-14 * (1.0 + std::fabs(fx))) {
      converged = true;
      ++it;
      break;
    }
  }
  return {x[0], x[1], it, converged};
}

void validate_fit(const crab_struct* st, const double* q, const double* y, const double* sigma, int64_t nq,
                  const crab_fit_options& o) {
  bool bad = nq <= 0 || st->n == 0;
  for (int64_t k = 0; k < nq && !bad; ++k) {
    if (!std::isfinite(q[k]) || q[k] < 0.0 || (k > 0 && q[k] < q[k - 1])) bad = true;
    if (!std::isfinite(y[k])) bad = true;
    if (!std::isfinite(sigma[k]) || sigma[k] <= 0.0) bad = true;
  }
  if (bad)
    throw Error(CRAB_EINVAL,
                "fit requires a non-empty structure and equal-length finite q, intensity, and positive-sigma arrays on "
                "a non-decreasing q grid");
  if (o.q_sampling_stride <= 0 || o.max_iterations <= 0 || !std::isfinite(o.c1_lo) || !std::isfinite(o.c1_hi) ||
      o.c1_lo <= 0.0 || o.c1_lo >= o.c1_hi || !std::isfinite(o.c2_lo) || !std::isfinite(o.c2_hi) ||
      o.c2_lo >= o.c2_hi || (o.scale_mode == CRAB_SCALE_FIXED && (!std::isfinite(o.scale_value) || o.scale_value < 0.0)) ||
      (o.bg_mode == CRAB_BG_FIXED && !std::isfinite(o.bg_value)))
    throw Error(CRAB_EINVAL, "fit bounds, iteration limit, and q sampling stride are invalid");
}

// Six-term basis for a fit on the given q values with the method rule of
// fit.rs:352-377.
void fit_basis(crab_ctx* ctx, const crab_struct* st, const std::vector<double>& q, const crab_fit_options& o,
               int l_max, double* out6) {
  int method = o.method;
  if (method == CRAB_METHOD_AUTO) {
    if (o.solvent.hydration_model != CRAB_HYD_ANALYTIC) method = CRAB_METHOD_MULTIPOLE;
    else if (st->n < 500) method = CRAB_METHOD_DEBYE;
    else method = CRAB_METHOD_MULTIPOLE;
  }
  if (method == CRAB_METHOD_DEBYE)
    debye_basis(ctx, st, q.data(), (int64_t)q.size(), o.solvent, o.implicit_hydrogen != 0, out6, false);
  else
    multipole_solvent_basis_impl(ctx, st, q.data(), (int64_t)q.size(), l_max, o.solvent, o.implicit_hydrogen != 0,
                                 CRAB_PREC_TF32_SPLIT, out6);
}

// ---------------------------------------------------------------- ensemble helpers (ensemble.rs)

void mix_curves(const std::vector<const double*>& curves, const double* w, int64_t nq, double* out) {
  for (int64_t p = 0; p < nq; ++p) {
    double s = 0.0;
    for (size_t k = 0; k < curves.size(); ++k) s += curves[k][p] * w[k];
    out[p] = s;
  }
}

}  // namespace

}  // namespace crab

using namespace crab;

extern "C" {

int crab_fit(crab_ctx* ctx, crab_struct* st, const double* q, const double* intensity, const double* sigma, int64_t nq,
             const crab_fit_options* opt, double init_c1, double init_c2, crab_fit_result* result, double* fitted) {
  if (!ctx || !st || !opt || !result || (nq > 0 && (!q || !intensity || !sigma))) return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    const crab_fit_options& o = *opt;
    validate_fit(st, q, intensity, sigma, nq, o);
    validate_solvent(o.solvent);
    double c[3], rmax;
    centre_and_rmax(st, c, &rmax);
    double qmax = 0.0;
    for (int64_t k = 0; k < nq; ++k) qmax = std::fmax(qmax, q[k]);
    const int l_max = (int)std::min(64L, std::max(8L, (long)std::ceil(qmax * rmax) + 8));
    const std::vector<size_t> idx = sampled_indices((size_t)nq, (size_t)o.q_sampling_stride);
    std::vector<double> sq;
    for (size_t i : idx) sq.push_back(q[i]);
    sq.erase(std::unique(sq.begin(), sq.end()), sq.end());
    std::vector<double> sampled(6 * sq.size());
    fit_basis(ctx, st, sq, o, l_max, sampled.data());
    std::vector<double> basis(6 * nq);
    if ((int64_t)sq.size() == nq) basis = sampled;
    else
      for (int c6 = 0; c6 < 6; ++c6) {
        std::vector<double> v = cubic_hermite(sq, sampled.data() + c6 * sq.size(), q, nq);
        std::copy(v.begin(), v.end(), basis.begin() + c6 * nq);
      }
    Objective f{&basis, {q, intensity, sigma, nq}, o.c1_lo, o.c1_hi, o.c2_lo, o.c2_hi,
                o.scale_mode, o.bg_mode, o.scale_value, o.bg_value, {}};
    const double ic1 = std::fmin(std::fmax(init_c1, o.c1_lo), o.c1_hi);
    const double ic2 = std::fmin(std::fmax(init_c2, o.c2_lo), o.c2_hi);
    NMResult r = (o.optimizer == 1)
                     ? lbfgs_box(f, ic1, ic2, o.max_iterations)
                     : nelder_mead(f, ic1, ic2, (o.c1_hi - o.c1_lo) * 0.1, (o.c2_hi - o.c2_lo) * 0.1, o.max_iterations,
                                   1e-8);
    const double c1 = std::fmin(std::fmax(r.c1, o.c1_lo), o.c1_hi);
    const double c2 = std::fmin(std::fmax(r.c2, o.c2_lo), o.c2_hi);
    std::vector<double> raw(nq);
    combine_basis(q, nq, basis.data(), c1, c2, raw.data());
    double s, b, chi;
    solve_scale_background(raw.data(), f.d, o.scale_mode, o.scale_value, o.bg_mode, o.bg_value, &s, &b, &chi);
    if (!std::isfinite(chi)) throw Error(CRAB_ENOTCONV, "objective was not finite");
    result->scale = s;
    result->background = b;
    result->c1 = c1;
    result->c2 = c2;
    result->chi2 = chi;
    result->iterations = r.iterations;
    result->converged = r.converged ? 1 : 0;
    if (fitted)
      for (int64_t k = 0; k < nq; ++k) fitted[k] = s * raw[k] + b;
  });
}

// reweight.rs:84-154
int crab_reweight_curves(const double* curves, int32_t K, const double* q, const double* y, const double* sigma,
                         int64_t nq, const double* prior_in, const crab_reweight_options* opt, double* weights_out,
                         crab_reweight_result* res) {
  (void)q;
  if (!curves || !y || !sigma || !opt || !weights_out || !res || K <= 0 || nq <= 0) return CRAB_EINVAL;
  const crab_reweight_options& o = *opt;
  if (!std::isfinite(o.kl_strength) || o.kl_strength < 0.0 || o.max_iterations <= 0 || !std::isfinite(o.step_size) ||
      o.step_size <= 0.0 || !std::isfinite(o.tolerance) || o.tolerance <= 0.0 || !std::isfinite(o.min_weight) ||
      o.min_weight < 0.0 || o.min_weight * (double)K >= 1.0)
    return CRAB_EINVAL;
  for (int64_t i = 0; i < (int64_t)K * nq; ++i)
    if (!std::isfinite(curves[i])) return CRAB_EINVAL;
  std::vector<double> prior(K, 1.0);
  if (prior_in) {
    for (int k = 0; k < K; ++k) {
      if (!std::isfinite(prior_in[k]) || prior_in[k] <= 0.0) return CRAB_EINVAL;
      prior[k] = prior_in[k];
    }
  }
  double psum = 0.0;
  for (double v : prior) psum += v;
  if (!std::isfinite(psum) || psum <= 0.0) return CRAB_EINVAL;
  for (double& v : prior) v /= psum;
  auto apply_floor = [&](std::vector<double> w) {
    double sum = 0.0;
    for (double v : w) sum += v;
    sum = std::fmax(sum, 1e-300);
    if (o.min_weight <= 0.0) {
      for (double& v : w) v /= sum;
      return w;
    }
    const double residual = 1.0 - o.min_weight * (double)w.size();
    for (double& v : w) v = o.min_weight + residual * v / sum;
    return w;
  };
  auto kl = [&](const std::vector<double>& w) {
    double s = 0.0;
    for (int k = 0; k < K; ++k) s += w[k] * std::log(w[k] / prior[k]);
    return s;
  };
  std::vector<const double*> cv(K);
  for (int k = 0; k < K; ++k) cv[k] = curves + (size_t)k * nq;
  Data d{q, y, sigma, nq};
  // reweight.rs:236-301 closed-form scale/background for every mode pair
  auto fit = [&](const std::vector<double>& w, std::vector<double>& mix, double* s, double* b, double* chi) {
    mix_curves(cv, w.data(), nq, mix.data());
    double sw = 0, sx = 0, sy = 0, sxx = 0, sxy = 0;
    for (int64_t i = 0; i < nq; ++i) {
      const double ww = 1.0 / (sigma[i] * sigma[i]);
      sw += ww;
      sx += ww * mix[i];
      sy += ww * y[i];
      sxx += ww * mix[i] * mix[i];
      sxy += ww * mix[i] * y[i];
    }
    auto fscale = [&](double bb) { return sxx > 0.0 ? std::fmax((sxy - bb * sx) / sxx, 0.0) : 0.0; };
    auto fbg = [&](double ss) { return sw > 0.0 ? (sy - ss * sx) / sw : 0.0; };
    if (o.scale_mode == CRAB_SCALE_FIXED) {
      *s = std::fmax(o.scale_value, 0.0);
      *b = o.bg_mode == CRAB_BG_FIXED ? o.bg_value : o.bg_mode == CRAB_BG_FIXED_ZERO ? 0.0 : fbg(*s);
    } else if (o.bg_mode == CRAB_BG_FIXED) {
      *s = fscale(o.bg_value);
      *b = o.bg_value;
    } else if (o.bg_mode == CRAB_BG_FIXED_ZERO) {
      *s = fscale(0.0);
      *b = 0.0;
    } else {
      const double det = sxx * sw - sx * sx;
      *s = std::fabs(det) > 1e-20 ? std::fmax((sxy * sw - sx * sy) / det, 0.0) : 0.0;
      *b = fbg(*s);
    }
    double c = 0.0;
    for (int64_t i = 0; i < nq; ++i) {
      const double r = (*s * mix[i] + *b - y[i]) / sigma[i];
      c += r * r;
    }
    *chi = c / (double)std::max<int64_t>(nq - 1, 1);
  };
  std::vector<double> w = apply_floor(prior), mix(nq), grad(K);
  int iterations = 0, converged = 0;
  const double dof = (double)std::max<int64_t>(nq - 1, 1);
  for (int it = 0; it < o.max_iterations; ++it) {
    iterations = it + 1;
    double s, b, chi;
    fit(w, mix, &s, &b, &chi);
    for (int k = 0; k < K; ++k) {
      double dg = 0.0;
      for (int64_t i = 0; i < nq; ++i) {
        const double fitted = s * mix[i] + b;
        dg += 2.0 * (fitted - y[i]) * s * cv[k][i] / (sigma[i] * sigma[i]) / dof;
      }
      grad[k] = dg + o.kl_strength * (std::log(w[k] / prior[k]) + 1.0);
    }
    double gmax = 0.0;
    for (double g : grad) gmax = std::fmax(gmax, std::fabs(g));
    double step = o.step_size / std::fmax(gmax, 1e-12);
    const double objective = chi + o.kl_strength * kl(w);
    std::vector<double> accepted;
    for (int h = 0; h < 14; ++h) {
      std::vector<double> lw(K), pr(K);
      double mx = -INFINITY;
      for (int k = 0; k < K; ++k) {
        lw[k] = std::log(std::fmax(w[k], 1e-300)) - step * grad[k];
        mx = std::fmax(mx, lw[k]);
      }
      double sum = 0.0;
      for (int k = 0; k < K; ++k) pr[k] = std::exp(lw[k] - mx);
      for (int k = 0; k < K; ++k) sum += pr[k];
      sum = std::fmax(sum, 1e-300);
      for (double& v : pr) v /= sum;
      pr = apply_floor(pr);
      double s2, b2, chi2;
      std::vector<double> mix2(nq);
      fit(pr, mix2, &s2, &b2, &chi2);
      if (chi2 + o.kl_strength * kl(pr) <= objective + 1e-12) {
        accepted = pr;
        break;
      }
      step *= 0.5;
    }
    if (accepted.empty()) break;
    double delta = 0.0;
    for (int k = 0; k < K; ++k) delta += std::fabs(accepted[k] - w[k]);
    w = accepted;
    if (delta <= o.tolerance) {
      converged = 1;
      break;
    }
  }
  double s, b, chi;
  fit(w, mix, &s, &b, &chi);
  std::copy(w.begin(), w.end(), weights_out);
  double ess = 0.0;
  for (double v : w) ess += v * v;
  res->scale = s;
  res->background = b;
  res->reduced_chi2 = chi;
  res->chi2 = chi * dof;
  res->kl_divergence = kl(w);
  res->effective_sample_size = 1.0 / ess;
  res->iterations = iterations;
  res->converged = converged;
  (void)d;
  return CRAB_OK;
}

}  // extern "C"
