// Complex Kaiser-Bessel interpolation coefficients and deapodization (FP64, host).
//
// The reference takes both from torchkbnufft 1.5.2 (calc_tensor_spmatrix at
// src/export_torchkbnufft_gpu_case.py:537-567, KbNufft.scaling_coef at
// experiments/data_prep/export_real_runtime_inputs.py:97-101), which is not vendored.
// This is the published gridding NUFFT with the reference's own KB kernel and Beatty
// beta (src/nufft_layout_oracle.py:152-156, :168-169):
//   phi(d)   = I0(beta*sqrt(1-(2d/J)^2)) / I0(beta) for |d| < J/2, else 0
//   support  J points per axis from floor(u - J/2) + 1, u = k*G (grid units)
//   phase    exp(2*pi*i*q*c/G), c = N/2: the image sits at [0,N) of the padded grid
//   deapod   1/(Phi(t0/G) Phi(t1/G)), Phi(xi) = J*sinh(z)/z/I0(beta), z^2 = beta^2-(pi*J*xi)^2
#include <algorithm>
#include <atomic>
#include <cmath>
#include <numeric>
#include <thread>
#include <vector>

#include "kb.hpp"

namespace tsn {

double bessel_i0(double x) {
  // power series sum_k ((x/2)^2)^k / (k!)^2, converges for all x; exact to ~1 ulp for |x| < 40
  const double q = 0.25 * x * x;
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 500; ++k) {
    term *= q / (static_cast<double>(k) * k);
    sum += term;
    if (term < sum * 1e-18) break;
  }
  return sum;
}

double beatty_beta(int width, double oversampling) {
  const double term = std::pow(width / oversampling * (oversampling - 0.5), 2) - 0.8;
  return M_PI * std::sqrt(std::max(term, 0.01));
}

double kb_weight(double d, int width, double beta, double i0_beta) {
  const double s = 2.0 * d / width;
  if (std::fabs(s) >= 1.0) return 0.0;
  return bessel_i0(beta * std::sqrt(std::max(0.0, 1.0 - s * s))) / i0_beta;
}

double kb_fourier(double xi, int width, double beta, double i0_beta) {
  const double z2 = beta * beta - std::pow(M_PI * width * xi, 2);
  const double z = std::sqrt(std::fabs(z2));
  double r;
  if (z == 0.0) r = 1.0;
  else if (z2 >= 0.0) r = std::sinh(z) / z;
  else r = std::sin(z) / z;
  return width * r / i0_beta;
}

std::vector<double> deapodization(int im_size, int grid_size, int width) {
  const double beta = beatty_beta(width, static_cast<double>(grid_size) / im_size);
  const double i0b = bessel_i0(beta);
  std::vector<double> inv(im_size);
  for (int i = 0; i < im_size; ++i)
    inv[i] = 1.0 / kb_fourier(static_cast<double>(i - im_size / 2) / grid_size, width, beta, i0b);
  std::vector<double> out(static_cast<size_t>(im_size) * im_size);
  for (int a = 0; a < im_size; ++a)
    for (int b = 0; b < im_size; ++b) out[static_cast<size_t>(a) * im_size + b] = inv[a] * inv[b];
  return out;
}

static void exact_phase(int64_t k, int64_t g, double* c, double* s) {
  k %= g;
  if (k < 0) k += g;
  if ((4 * k) % g == 0) {
    static const double cs[4] = {1.0, 0.0, -1.0, 0.0};
    static const double sn[4] = {0.0, 1.0, 0.0, -1.0};
    const int q = static_cast<int>((4 * k) / g) & 3;
    *c = cs[q];
    *s = sn[q];
    return;
  }
  const double a = 2.0 * M_PI * static_cast<double>(k) / static_cast<double>(g);
  *c = std::cos(a);
  *s = std::sin(a);
}

KbCsr kb_interpolation_csr(const float* traj, int64_t m, int im_size, int grid_size, int width) {
  if (m < 0 || im_size <= 0 || grid_size < im_size || width <= 0 || width > grid_size)
    fail(TSN_ERR_ARG, "invalid KB interpolation shape");
  const double beta = beatty_beta(width, static_cast<double>(grid_size) / im_size);
  const double i0b = bessel_i0(beta);
  const int64_t c = im_size / 2;
  KbCsr out;
  out.row_ptr.assign(static_cast<size_t>(m) + 1, 0);
  out.cols.reserve(static_cast<size_t>(m) * width * width);
  out.re.reserve(out.cols.capacity());
  out.im.reserve(out.cols.capacity());
  std::vector<int64_t> q0(width), q1(width), cols(width * width);
  std::vector<double> w0(width), w1(width), w2(width * width), re(width * width), im(width * width);
  std::vector<int> idx(width * width);
  for (int64_t r = 0; r < m; ++r) {
    const double u0 = static_cast<double>(traj[2 * r]) * grid_size;
    const double u1 = static_cast<double>(traj[2 * r + 1]) * grid_size;
    if (!std::isfinite(u0) || !std::isfinite(u1)) fail(TSN_ERR_NONFINITE, "trajectory contains non-finite coordinates");
    const int64_t s0 = static_cast<int64_t>(std::floor(u0 - width / 2.0)) + 1;
    const int64_t s1 = static_cast<int64_t>(std::floor(u1 - width / 2.0)) + 1;
    for (int j = 0; j < width; ++j) {
      q0[j] = s0 + j;
      q1[j] = s1 + j;
      w0[j] = kb_weight(u0 - static_cast<double>(q0[j]), width, beta, i0b);
      w1[j] = kb_weight(u1 - static_cast<double>(q1[j]), width, beta, i0b);
    }
    for (int a = 0; a < width; ++a)
      for (int b = 0; b < width; ++b) {
        const int e = a * width + b;
        double cp, sp;
        exact_phase(q0[a] * c + q1[b] * c, grid_size, &cp, &sp);
        w2[e] = w0[a] * w1[b];
        re[e] = w2[e] * cp;
        im[e] = w2[e] * sp;
        const int64_t m0 = ((q0[a] % grid_size) + grid_size) % grid_size;
        const int64_t m1 = ((q1[b] % grid_size) + grid_size) % grid_size;
        cols[e] = m0 * grid_size + m1;
      }
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return cols[x] < cols[y]; });
    for (int e : idx) {
      if (w2[e] == 0.0) continue;
      out.cols.push_back(cols[e]);
      out.re.push_back(re[e]);
      out.im.push_back(im[e]);
    }
    out.row_ptr[r + 1] = static_cast<int64_t>(out.cols.size());
  }
  return out;
}


std::vector<double> deapodization3(int im_size, int grid_size, int width) {
  const double beta = beatty_beta(width, static_cast<double>(grid_size) / im_size);
  const double i0b = bessel_i0(beta);
  std::vector<double> inv(im_size);
  for (int i = 0; i < im_size; ++i)
    inv[i] = 1.0 / kb_fourier(static_cast<double>(i - im_size / 2) / grid_size, width, beta, i0b);
  const size_t n = static_cast<size_t>(im_size);
  std::vector<double> out(n * n * n);
  for (size_t a = 0; a < n; ++a)
    for (size_t b = 0; b < n; ++b)
      for (size_t c = 0; c < n; ++c) out[(a * n + b) * n + c] = (inv[a] * inv[b]) * inv[c];
  return out;
}

namespace {

// Support start, weights and wrapped cell index of one sample along one axis.
struct Axis {
  int64_t cell[16];
  double w[16];
};

inline void axis_weights(double u, int width, int64_t g, double beta, double i0b, Axis& a) {
  const int64_t s = static_cast<int64_t>(std::floor(u - width / 2.0)) + 1;
  for (int j = 0; j < width; ++j) {
    const int64_t q = s + j;
    a.w[j] = kb_weight(u - static_cast<double>(q), width, beta, i0b);
    a.cell[j] = ((q % g) + g) % g;
  }
}

template <class F>
void parallel_rows(int64_t n, int threads, F&& body) {
  threads = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(threads, n / 4096 + 1)));
  std::atomic<int64_t> next{0};
  auto work = [&]() {
    for (;;) {
      const int64_t lo = next.fetch_add(4096);
      if (lo >= n) break;
      const int64_t hi = std::min(n, lo + 4096);
      for (int64_t r = lo; r < hi; ++r) body(r);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}

}  // namespace

KbCsr kb_weights_csr3(const float* traj, int64_t m, int im_size, int grid_size, int width, int threads) {
  if (m < 0 || im_size <= 0 || grid_size < im_size || width <= 0 || width > 16 || width > grid_size)
    fail(TSN_ERR_ARG, "invalid 3D KB interpolation shape");
  const double beta = beatty_beta(width, static_cast<double>(grid_size) / im_size);
  const double i0b = bessel_i0(beta);
  const int64_t g = grid_size;
  for (int64_t i = 0; i < 3 * m; ++i)
    if (!std::isfinite(traj[i])) fail(TSN_ERR_NONFINITE, "trajectory contains non-finite coordinates");
  if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  KbCsr out;
  resize_huge(out.row_ptr, static_cast<size_t>(m) + 1);
  out.row_ptr[0] = 0;
  auto axes = [&](int64_t r, Axis (&ax)[3]) {
    for (int d = 0; d < 3; ++d) axis_weights(static_cast<double>(traj[3 * r + d]) * grid_size, width, g, beta, i0b, ax[d]);
  };
  // pass 1: nonzero count per row
  parallel_rows(m, threads, [&](int64_t r) {
    Axis ax[3];
    axes(r, ax);
    int64_t n[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d)
      for (int j = 0; j < width; ++j) n[d] += ax[d].w[j] != 0.0;
    out.row_ptr[r + 1] = n[0] * n[1] * n[2];
  });
  for (int64_t r = 0; r < m; ++r) out.row_ptr[r + 1] += out.row_ptr[r];
  resize_huge(out.cols, static_cast<size_t>(out.row_ptr[m]));
  resize_huge(out.re, out.cols.size());
  // pass 2: entries, sorted by cell
  parallel_rows(m, threads, [&](int64_t r) {
    Axis ax[3];
    axes(r, ax);
    std::vector<std::pair<int64_t, double>> e;
    e.reserve(static_cast<size_t>(width) * width * width);
    for (int a = 0; a < width; ++a) {
      if (ax[0].w[a] == 0.0) continue;
      for (int b = 0; b < width; ++b) {
        if (ax[1].w[b] == 0.0) continue;
        const double wab = ax[0].w[a] * ax[1].w[b];
        for (int c = 0; c < width; ++c) {
          if (ax[2].w[c] == 0.0) continue;
          e.emplace_back((ax[0].cell[a] * g + ax[1].cell[b]) * g + ax[2].cell[c], wab * ax[2].w[c]);
        }
      }
    }
    std::sort(e.begin(), e.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    int64_t at = out.row_ptr[r];
    for (const auto& kv : e) {
      out.cols[at] = kv.first;
      out.re[at] = kv.second;
      ++at;
    }
  });
  return out;
}

}  // namespace tsn
