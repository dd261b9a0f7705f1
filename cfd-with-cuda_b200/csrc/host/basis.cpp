// Gauss points and hex27 / hex8 shape functions at the Gauss points
// (setupGQ and calcShape, blascoCodinaHuerta.cpp:2166-2488), tabulated for
// the device.  NGP 1 and 8 follow the reference (8-point rule ordered with xi
// fastest; the 1-point weight 4.0 is kept as the reference sets it,
// blascoCodinaHuerta.cpp:2179).  NGP 27 -- an empty TODO in the reference
// (blascoCodinaHuerta.cpp:2197-2201) -- is the 3x3x3 Gauss-Legendre rule
// (points 0, +-sqrt(3/5), weights 8/9, 5/9) in the same xi-fastest order.
#include <cmath>
#include <cstring>

#include "../cuda/common.cuh"
#include "problem.h"

namespace cfd {

namespace {
// 1D quadratic Lagrange factors on the nodes -1, 0, +1 and their derivatives.
double lq(int a, double x) { return a == 0 ? 0.5 * (x * x - x) : (a == 1 ? 1.0 - x * x : 0.5 * (x * x + x)); }
double dlq(int a, double x) { return a == 0 ? 0.5 * (2 * x - 1) : (a == 1 ? -2 * x : 0.5 * (2 * x + 1)); }
}  // namespace

int make_basis(int ngp, Basis& B) {
  std::memset(&B, 0, sizeof(B));
  B.ngp = ngp;
  double pts[kMaxNGP][3];
  if (ngp == 1) {
    pts[0][0] = pts[0][1] = pts[0][2] = 0.0;
    B.w[0] = 4.0;
  } else if (ngp == 8) {
    const double g = std::sqrt(1. / 3);
    for (int k = 0; k < 8; k++) {
      pts[k][0] = (k & 1) ? g : -g;
      pts[k][1] = (k & 2) ? g : -g;
      pts[k][2] = (k & 4) ? g : -g;
      B.w[k] = 1.0;
    }
  } else if (ngp == 27) {
    const double p[3] = {-std::sqrt(0.6), 0.0, std::sqrt(0.6)};
    const double w[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    for (int c = 0; c < 3; c++)
      for (int b = 0; b < 3; b++)
        for (int a = 0; a < 3; a++) {
          int k = a + 3 * b + 9 * c;
          pts[k][0] = p[a];
          pts[k][1] = p[b];
          pts[k][2] = p[c];
          B.w[k] = w[a] * w[b] * w[c];
        }
  } else {
    return -1;
  }
  for (int k = 0; k < ngp; k++) {
    const double x = pts[k][0], y = pts[k][1], z = pts[k][2];
    for (int j = 0; j < 27; j++) {
      const int a = kNode27[j][0], b = kNode27[j][1], c = kNode27[j][2];
      B.Sv[k][j] = lq(a, x) * lq(b, y) * lq(c, z);
      B.dSv[0][k][j] = dlq(a, x) * lq(b, y) * lq(c, z);
      B.dSv[1][k][j] = lq(a, x) * dlq(b, y) * lq(c, z);
      B.dSv[2][k][j] = lq(a, x) * lq(b, y) * dlq(c, z);
    }
    for (int m = 0; m < 8; m++) {
      const double sx = kNode27[m][0] ? 1.0 : -1.0, sy = kNode27[m][1] ? 1.0 : -1.0,
                   sz = kNode27[m][2] ? 1.0 : -1.0;
      const double fx = 1 + sx * x, fy = 1 + sy * y, fz = 1 + sz * z;
      B.Sp[k][m] = 0.125 * fx * fy * fz;
      B.dSp[0][k][m] = 0.125 * sx * fy * fz;
      B.dSp[1][k][m] = 0.125 * fx * sy * fz;
      B.dSp[2][k][m] = 0.125 * fx * fy * sz;
    }
  }
  return 0;
}

}  // namespace cfd
