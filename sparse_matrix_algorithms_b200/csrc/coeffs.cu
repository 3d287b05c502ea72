// Chebyshev filter coefficients (host).  O(K) work, or O(K*nsamp) for the smooth
// window; none of it is on the device.
#include <algorithm>
#include <cmath>

#include "sma_internal.h"

namespace sma {

static const double kPi = 3.14159265358979323846;

// jackson_kernel(K), chebyshev_subspace_iteration.jl:376-387:
//   g_k = sin((k+1)a)/((K+2) sin a) + (1 - (k+1)/(K+2)) cos(k a),  a = pi/(K+2)
std::vector<double> jackson_kernel(int64_t K) {
  if (K <= 0) return {1.0};
  std::vector<double> g(K + 1);
  const double a = kPi / (double)(K + 2);
  const double sa = std::sin(a);
  for (int64_t k = 0; k <= K; ++k)
    g[k] = std::sin((double)(k + 1) * a) / ((double)(K + 2) * sa) +
           (1.0 - (double)(k + 1) / (double)(K + 2)) * std::cos((double)k * a);
  return g;
}

static void damp(std::vector<double> &c, int64_t K, bool jackson) {
  if (!jackson) return;
  const std::vector<double> g = jackson_kernel(K);
  for (int64_t k = 0; k <= K; ++k) c[k] *= g[k];
}

// cheb_delta_coeffs, chebyshev_subspace_iteration.jl:400-414:
//   c_0 = 1/pi, c_k = 2 cos(k theta)/pi, theta = acos(clamp(sigma_hat, -1, 1))
std::vector<double> cheb_delta_coeffs(double sh, int64_t K, bool jackson) {
  std::vector<double> c(K + 1, 0.0);
  const double th = std::acos(std::min(std::max(sh, -1.0), 1.0));
  c[0] = 1.0 / kPi;
  for (int64_t k = 1; k <= K; ++k) c[k] = 2.0 * std::cos((double)k * th) / kPi;
  damp(c, K, jackson);
  return c;
}

// cheb_window_coeffs, chebyshev_subspace_iteration.jl:430-447: indicator of [a, b]:
//   c_0 = (beta - alpha)/pi, c_k = 2 (sin(k beta) - sin(k alpha))/(k pi),
//   alpha = acos(b), beta = acos(a) after clamping to [-1, 1] and ordering.
std::vector<double> cheb_window_coeffs(double a, double b, int64_t K, bool jackson) {
  double aa = std::max(-1.0, std::min(1.0, a));
  double bb = std::max(-1.0, std::min(1.0, b));
  if (aa > bb) std::swap(aa, bb);
  const double al = std::acos(bb), be = std::acos(aa);
  std::vector<double> c(K + 1, 0.0);
  c[0] = (be - al) / kPi;
  for (int64_t k = 1; k <= K; ++k)
    c[k] = 2.0 * (std::sin((double)k * be) - std::sin((double)k * al)) / ((double)k * kPi);
  damp(c, K, jackson);
  return c;
}

// cheb_smooth_window_coeffs, chebyshev_subspace_iteration.jl:465-489: the window
// f(x) = 1/2(1+tanh((x-a)/delta)) * 1/2(1-tanh((x-b)/delta)) projected on T_k by the
// trapezoid rule in theta on nsamp equispaced nodes of [0, pi].
std::vector<double> cheb_smooth_window_coeffs(double a, double b, int64_t K, bool jackson,
                                              int64_t nsamp, double delta) {
  double aa = std::max(-1.0, std::min(1.0, a));
  double bb = std::max(-1.0, std::min(1.0, b));
  if (aa > bb) std::swap(aa, bb);
  require(nsamp >= 2, SMA_ERR_ARG, "nsamp must be at least 2");
  std::vector<double> c(K + 1, 0.0);
  const double w = kPi / (double)(nsamp - 1);
  std::vector<double> f(nsamp), th(nsamp);
  for (int64_t i = 0; i < nsamp; ++i) {
    th[i] = (double)i * w;
    const double xi = std::cos(th[i]);
    const double fi = 0.5 * (1.0 + std::tanh((xi - aa) / delta)) * 0.5 *
                      (1.0 - std::tanh((xi - bb) / delta));
    const double wt = (i == 0 || i == nsamp - 1) ? 0.5 : 1.0;
    f[i] = wt * fi;
  }
  for (int64_t k = 0; k <= K; ++k) {
    double s = 0.0;
    for (int64_t i = 0; i < nsamp; ++i) s += f[i] * std::cos((double)k * th[i]);
    c[k] = (k == 0 ? 1.0 / kPi : 2.0 / kPi) * w * s;
  }
  damp(c, K, jackson);
  return c;
}

// _build_coeffs, polfed.jl:404-414
std::vector<double> build_coeffs(int64_t degree, double smin, double smax, double sigma,
                                 double emin, double emax, int64_t window_type, bool jackson) {
  require(degree >= 0, SMA_ERR_ARG, "degree must be nonnegative");
  const double c = 0.5 * (smin + smax), d = 0.5 * (smax - smin);
  const double sh = (sigma - c) / d, a = (emin - c) / d, b = (emax - c) / d;
  switch (window_type) {
    case SMA_WINDOW_STEP: return cheb_window_coeffs(a, b, degree, jackson);
    case SMA_WINDOW_DELTA: return cheb_delta_coeffs(sh, degree, jackson);
    case SMA_WINDOW_SMOOTH: return cheb_smooth_window_coeffs(a, b, degree, jackson, 4096, 0.02);
    default:
      throw Error(SMA_ERR_WINDOW, "Unknown window type: " + std::to_string(window_type));
  }
}

}  // namespace sma
