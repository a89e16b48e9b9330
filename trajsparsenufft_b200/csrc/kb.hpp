// Complex KB interpolation coefficients and deapodization (see kb.cpp).
#pragma once

#include <cstdint>
#include <vector>

#include "common.hpp"

namespace tsn {

struct KbCsr {
  std::vector<int64_t> row_ptr, cols;
  std::vector<double> re, im;
};

double bessel_i0(double x);
double beatty_beta(int width, double oversampling);
double kb_weight(double d, int width, double beta, double i0_beta);
double kb_fourier(double xi, int width, double beta, double i0_beta);
std::vector<double> deapodization(int im_size, int grid_size, int width);
KbCsr kb_interpolation_csr(const float* traj, int64_t m, int im_size, int grid_size, int width);
// 3D real KB weights (the centred-image layout: the phase exp(2 pi i q.c/G) becomes the FFT
// shift), CSR over samples, cells (q0 G + q1) G + q2 (q_d from trajectory column d), columns
// sorted, exact zeros dropped; weight = (phi0 * phi1) * phi2.  `im` stays empty.
KbCsr kb_weights_csr3(const float* traj, int64_t m, int im_size, int grid_size, int width, int threads);
// [N][N][N] deapodization 1/(Phi(t0/G) Phi(t1/G) Phi(t2/G)), product in the same order.
std::vector<double> deapodization3(int im_size, int grid_size, int width);

}  // namespace tsn
