// Coarse space of the two-level pressure preconditioners (see coarse.h).
#include "coarse.h"

#include <algorithm>
#include <cmath>
#include <cstdint>

namespace cfd {

namespace {

// Hat functions along one axis: voxel x lies in coarse cell i0[x] with
// weights (1 - f[x]) on node i0 and f[x] on node i0 + 1.
struct Axis {
  std::vector<int> i0;
  std::vector<double> f;
};

Axis make_axis(int n, int nc, double h) {
  Axis a;
  a.i0.resize(n);
  a.f.resize(n);
  for (int x = 0; x < n; x++) {
    if (nc < 2) {
      a.i0[x] = 0;
      a.f[x] = 0.0;
      continue;
    }
    const double t = x / h;
    int i = (int)std::floor(t);
    i = std::min(std::max(i, 0), nc - 2);
    a.i0[x] = i;
    a.f[x] = std::min(std::max(t - i, 0.0), 1.0);
  }
  return a;
}

// In-place lower Cholesky of the row-major n x n matrix A (upper triangle
// ignored); false if A is not numerically positive definite.
bool cholesky(std::vector<double>& A, int n) {
  constexpr int NB = 96;
  double* a = A.data();
  bool ok = true;
  for (int k0 = 0; k0 < n && ok; k0 += NB) {
    const int k1 = std::min(n, k0 + NB);
    for (int j = k0; j < k1 && ok; j++) {
      double* rj = a + (size_t)j * n;
      double d = rj[j];
      for (int k = k0; k < j; k++) d -= rj[k] * rj[k];
      if (!(d > 0.0) || !std::isfinite(d)) {
        ok = false;
        break;
      }
      rj[j] = std::sqrt(d);
      for (int i = j + 1; i < k1; i++) {
        double* ri = a + (size_t)i * n;
        double s = ri[j];
#pragma omp simd reduction(- : s)
        for (int k = k0; k < j; k++) s -= ri[k] * rj[k];
        ri[j] = s / rj[j];
      }
    }
    if (!ok) break;
#pragma omp parallel for schedule(static)
    for (int i = k1; i < n; i++) {
      double* ri = a + (size_t)i * n;
      for (int j = k0; j < k1; j++) {
        const double* rj = a + (size_t)j * n;
        double s = ri[j];
#pragma omp simd reduction(- : s)
        for (int k = k0; k < j; k++) s -= ri[k] * rj[k];
        ri[j] = s / rj[j];
      }
    }
    // trailing update A[i][j] -= sum_k A[i][k] A[j][k] (k in the panel,
    // k1 <= j <= i) in 4 x 4 tiles: 16 dot products share the loads of 8
    // panel rows
    const int nbk = k1 - k0;
    const int ntile = (n - k1 + 3) / 4;
#pragma omp parallel for schedule(dynamic, 2)
    for (int ti = 0; ti < ntile; ti++) {
      const int i0 = k1 + 4 * ti;
      const int ni = std::min(4, n - i0);
      for (int j0 = k1; j0 < i0 + ni; j0 += 4) {
        const int nj = std::min(4, n - j0);
        double s[4][4] = {};
        if (ni == 4 && nj == 4) {
          const double *p0 = a + (size_t)i0 * n + k0, *p1 = p0 + n, *p2 = p1 + n, *p3 = p2 + n;
          const double *q0 = a + (size_t)j0 * n + k0, *q1 = q0 + n, *q2 = q1 + n, *q3 = q2 + n;
          double s00 = 0, s01 = 0, s02 = 0, s03 = 0, s10 = 0, s11 = 0, s12 = 0, s13 = 0;
          double s20 = 0, s21 = 0, s22 = 0, s23 = 0, s30 = 0, s31 = 0, s32 = 0, s33 = 0;
#pragma omp simd reduction(+ : s00, s01, s02, s03, s10, s11, s12, s13, s20, s21, s22, s23, s30, s31, s32, s33)
          for (int k = 0; k < nbk; k++) {
            const double x0 = p0[k], x1 = p1[k], x2 = p2[k], x3 = p3[k];
            const double y0 = q0[k], y1 = q1[k], y2 = q2[k], y3 = q3[k];
            s00 += x0 * y0; s01 += x0 * y1; s02 += x0 * y2; s03 += x0 * y3;
            s10 += x1 * y0; s11 += x1 * y1; s12 += x1 * y2; s13 += x1 * y3;
            s20 += x2 * y0; s21 += x2 * y1; s22 += x2 * y2; s23 += x2 * y3;
            s30 += x3 * y0; s31 += x3 * y1; s32 += x3 * y2; s33 += x3 * y3;
          }
          const double t[4][4] = {{s00, s01, s02, s03}, {s10, s11, s12, s13}, {s20, s21, s22, s23},
                                  {s30, s31, s32, s33}};
          for (int u = 0; u < 4; u++)
            for (int v = 0; v < 4; v++) s[u][v] = t[u][v];
        } else {
          for (int u = 0; u < ni; u++)
            for (int v = 0; v < nj; v++) {
              const double* pi = a + (size_t)(i0 + u) * n + k0;
              const double* pj = a + (size_t)(j0 + v) * n + k0;
              double acc = 0.0;
              for (int k = 0; k < nbk; k++) acc += pi[k] * pj[k];
              s[u][v] = acc;
            }
        }
        for (int u = 0; u < ni; u++)
          for (int v = 0; v < nj && j0 + v <= i0 + u; v++) a[(size_t)(i0 + u) * n + j0 + v] -= s[u][v];
      }
    }
  }
  return ok;
}

// From the Cholesky factor L (lower triangle of A): inv = (L L^T)^-1 =
// L^-T L^-1.  U = L^-T is formed row by row in the upper triangle of A (the
// diagonal of L kept aside), then inv[a][b] = sum_{i >= max(a,b)} U[a][i] U[b][i].
//
// Both phases are memory-bound dot products over long rows.  A task owns a
// tile of consecutive rows (of U in the first phase, of the result in the
// second) and walks the streamed rows once for the whole tile, so each
// streamed row is read once per tile instead of once per row; every dot
// product is the same loop as row by row, so the result does not depend on
// the tiling.
void cholesky_inverse(std::vector<double>& A, int n, std::vector<double>& inv) {
  constexpr int kTileU = 16, kTileInv = 32;
  double* a = A.data();
  std::vector<double> ld(n), ud(n);
  for (int i = 0; i < n; i++) {
    ld[i] = a[(size_t)i * n + i];
    ud[i] = 1.0 / ld[i];
  }
  // U[j][i] = (delta_ij - sum_{k=j}^{i-1} L[i][k] U[j][k]) / L[i][i], i >= j
#pragma omp parallel for schedule(dynamic, 1)
  for (int j0 = 0; j0 < n; j0 += kTileU) {
    const int j1 = std::min(n, j0 + kTileU);
    for (int i = j0 + 1; i < n; i++) {
      const double* li = a + (size_t)i * n;
      const int je = std::min(j1, i);
      for (int j = j0; j < je; j++) {
        double* uj = a + (size_t)j * n;  // U[j][i] stored at A[j][i] (i > j)
        double s = li[j] * ud[j];
#pragma omp simd reduction(+ : s)
        for (int k = j + 1; k < i; k++) s += li[k] * uj[k];
        uj[i] = -s / ld[i];
      }
    }
  }
  inv.assign((size_t)n * n, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int r0 = 0; r0 < n; r0 += kTileInv) {
    const int r1 = std::min(n, r0 + kTileInv);
    for (int c = r0; c < n; c++) {
      const double* uc = a + (size_t)c * n;
      const int re = std::min(r1, c + 1);
      for (int r = r0; r < re; r++) {
        const double* ur = a + (size_t)r * n;
        // i = c contributes U[r][c] U[c][c]; i > c both off-diagonal
        double s = (c == r ? ud[r] : ur[c]) * ud[c];
#pragma omp simd reduction(+ : s)
        for (int i = c + 1; i < n; i++) s += ur[i] * uc[i];
        inv[(size_t)r * n + c] = s;
        inv[(size_t)c * n + r] = s;
      }
    }
  }
}

}  // namespace

void coarse_lattice(const int fd[3], int max_nodes, int cd[3], double h[3], double spacing) {
  double s = spacing > 1.0 ? spacing : 4.0;
  for (;;) {
    long long total = 1;
    for (int a = 0; a < 3; a++) {
      if (fd[a] < 2) {
        cd[a] = 1;
        h[a] = 1.0;
      } else {
        cd[a] = (int)std::ceil((fd[a] - 1) / s - 1e-9) + 1;
        cd[a] = std::max(2, std::min(cd[a], fd[a]));
        h[a] = (fd[a] - 1) / (double)(cd[a] - 1);
      }
      total *= cd[a];
    }
    if (total <= max_nodes) return;
    s *= 1.25;
  }
}

int coarse_build(const int fd[3], int max_nodes, const std::vector<int>& vox_of_p, const std::vector<int>& rp,
                 const std::vector<int>& col, const std::vector<double>& val, CoarseSpace& cs, std::string& err,
                 bool with_w, bool factor, double spacing) {
  for (int a = 0; a < 3; a++) cs.fd[a] = fd[a];
  coarse_lattice(fd, max_nodes, cs.cd, cs.h, spacing);
  const int nc = cs.cd[0] * cs.cd[1] * cs.cd[2];
  cs.nc = nc;
  const Axis ax = make_axis(fd[0], cs.cd[0], cs.h[0]), ay = make_axis(fd[1], cs.cd[1], cs.h[1]),
             az = make_axis(fd[2], cs.cd[2], cs.h[2]);
  const int np = (int)rp.size() - 1;
  auto voxel = [&](int p, int& x, int& y, int& z) {
    const int v = vox_of_p.empty() ? p : vox_of_p[p];
    x = v % fd[0];
    y = (v / fd[0]) % fd[1];
    z = v / (fd[0] * fd[1]);
  };
  // W = Z P, row by row: the coarse nodes a row reaches form a small box,
  // accumulated densely; rows are independent.  Both products below use
  // explicit fused multiply-adds, so the device build (galerkin.cu) can
  // take the same sums in the same order.
  std::vector<int> lo(3 * (size_t)np), bx(3 * (size_t)np);
  size_t wmax = 1;
#pragma omp parallel for reduction(max : wmax)
  for (int p = 0; p < np; p++) {
    int mn[3] = {1 << 30, 1 << 30, 1 << 30}, mx[3] = {-1, -1, -1};
    for (int k = rp[p]; k < rp[p + 1]; k++) {
      int q[3];
      voxel(col[k], q[0], q[1], q[2]);
      const int i[3] = {ax.i0[q[0]], ay.i0[q[1]], az.i0[q[2]]};
      for (int a = 0; a < 3; a++) {
        mn[a] = std::min(mn[a], i[a]);
        mx[a] = std::max(mx[a], std::min(i[a] + 1, cs.cd[a] - 1));
      }
    }
    size_t sz = 1;
    for (int a = 0; a < 3; a++) {
      if (mx[a] < mn[a]) mx[a] = mn[a] = 0;
      lo[3 * (size_t)p + a] = mn[a];
      bx[3 * (size_t)p + a] = mx[a] - mn[a] + 1;
      sz *= (size_t)(mx[a] - mn[a] + 1);
    }
    wmax = std::max(wmax, sz);
  }
  std::vector<double> W((size_t)np * wmax, 0.0);
#pragma omp parallel for schedule(static)
  for (int p = 0; p < np; p++) {
    const int* l = &lo[3 * (size_t)p];
    const int* b = &bx[3 * (size_t)p];
    double* w = &W[(size_t)p * wmax];
    for (int k = rp[p]; k < rp[p + 1]; k++) {
      int q[3];
      voxel(col[k], q[0], q[1], q[2]);
      const int ix = ax.i0[q[0]], iy = ay.i0[q[1]], iz = az.i0[q[2]];
      const double fx = ax.f[q[0]], fy = ay.f[q[1]], fz = az.f[q[2]];
      for (int c = 0; c < 8; c++) {
        const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
        if ((dx && cs.cd[0] < 2) || (dy && cs.cd[1] < 2) || (dz && cs.cd[2] < 2)) continue;
        const double wt = (dx ? fx : 1 - fx) * (dy ? fy : 1 - fy) * (dz ? fz : 1 - fz);
        if (wt == 0.0) continue;
        const int jx = ix + dx - l[0], jy = iy + dy - l[1], jz = iz + dz - l[2];
        double& acc = w[jx + b[0] * (jy + b[1] * jz)];
        acc = std::fma(val[k], wt, acc);
      }
    }
  }
  cs.w_ok = false;
  cs.wlo.clear();
  cs.w27.clear();
  if (with_w) {
    int widest = 0;
    for (size_t k = 0; k < bx.size(); k++) widest = std::max(widest, bx[k]);
    if (widest <= 3) {
      cs.w_ok = true;
      cs.wlo.resize(np);
      cs.w27.assign(27 * (size_t)np, 0.0);
#pragma omp parallel for schedule(static)
      for (int p = 0; p < np; p++) {
        const int* l = &lo[3 * (size_t)p];
        const int* b = &bx[3 * (size_t)p];
        const double* w = &W[(size_t)p * wmax];
        cs.wlo[p] = l[0] + cs.cd[0] * (l[1] + cs.cd[1] * l[2]);
        for (int jz = 0; jz < b[2]; jz++)
          for (int jy = 0; jy < b[1]; jy++)
            for (int jx = 0; jx < b[0]; jx++)
              cs.w27[27 * (size_t)p + jx + 3 * jy + 9 * jz] = w[jx + b[0] * (jy + b[1] * jz)];
      }
    }
  }
  // Zc = P^T W, dense; each row of P has 8 coarse nodes
  std::vector<double> Zc((size_t)nc * nc, 0.0);
  for (int p = 0; p < np; p++) {
    int x, y, z;
    voxel(p, x, y, z);
    const int ix = ax.i0[x], iy = ay.i0[y], iz = az.i0[z];
    const double fx = ax.f[x], fy = ay.f[y], fz = az.f[z];
    const int* l = &lo[3 * (size_t)p];
    const int* b = &bx[3 * (size_t)p];
    const double* w = &W[(size_t)p * wmax];
    for (int c = 0; c < 8; c++) {
      const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
      if ((dx && cs.cd[0] < 2) || (dy && cs.cd[1] < 2) || (dz && cs.cd[2] < 2)) continue;
      const double wt = (dx ? fx : 1 - fx) * (dy ? fy : 1 - fy) * (dz ? fz : 1 - fz);
      if (wt == 0.0) continue;
      const int i = (ix + dx) + cs.cd[0] * ((iy + dy) + cs.cd[1] * (iz + dz));
      double* zi = &Zc[(size_t)i * nc];
      for (int jz = 0; jz < b[2]; jz++)
        for (int jy = 0; jy < b[1]; jy++)
          for (int jx = 0; jx < b[0]; jx++) {
            const double v = w[jx + b[0] * (jy + b[1] * jz)];
            if (v == 0.0) continue;
            double& acc = zi[(l[0] + jx) + cs.cd[0] * ((l[1] + jy) + cs.cd[1] * (l[2] + jz))];
            acc = std::fma(wt, v, acc);
          }
    }
  }
  W.clear();
  W.shrink_to_fit();
  // symmetrise the rounding of the two accumulation orders
  for (int i = 0; i < nc; i++)
    for (int j = 0; j < i; j++) {
      const double s = 0.5 * (Zc[(size_t)i * nc + j] + Zc[(size_t)j * nc + i]);
      Zc[(size_t)i * nc + j] = Zc[(size_t)j * nc + i] = s;
    }
  if (!factor) {
    cs.inv.swap(Zc);
    return 0;
  }
  if (!cholesky(Zc, nc)) {
    err = "coarse matrix P^T Z P is not positive definite";
    return -1;
  }
  cholesky_inverse(Zc, nc, cs.inv);
  return 0;
}

}  // namespace cfd
