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

}  // namespace tsn
