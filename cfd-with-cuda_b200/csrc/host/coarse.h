// Coarse space of the two-level pressure preconditioners: trilinear hat
// functions on a coarse lattice laid over the structured grid of pressure
// nodes (voxel grid), the Galerkin coarse matrix Zc = P^T Z P and its dense
// inverse.  The preconditioner adds P Zc^-1 P^T r to the Jacobi step D^-1 r,
// so the lowest (mesh-wide) pressure modes, which Jacobi-PCG resolves one
// Krylov step at a time, are solved exactly on the coarse lattice.
#pragma once
#include <string>
#include <vector>

namespace cfd {

struct CoarseSpace {
  int fd[3] = {0, 0, 0};      // voxel grid (pressure nodes per axis)
  int cd[3] = {0, 0, 0};      // coarse nodes per axis
  double h[3] = {1, 1, 1};    // coarse spacing in voxels: (fd - 1) / (cd - 1)
  int nc = 0;                 // cd[0] cd[1] cd[2]
  std::vector<double> inv;    // nc x nc inverse of Zc (symmetric, row-major)
  // W = Z P row by row (with_w): row p couples to the coarse nodes of a box
  // of at most 3 per axis with origin wlo[p] (a coarse node index); w27
  // holds its 27 coefficients, tap dx + 3 dy + 9 dz (zero outside the box).
  // w_ok is false when some row's box is wider.
  bool w_ok = false;
  std::vector<int> wlo;
  std::vector<double> w27;
};

// Coarse lattice for a voxel grid: spacing `spacing` voxels (default 4)
// where the axis allows, widened until the lattice has at most max_nodes
// nodes.
void coarse_lattice(const int fd[3], int max_nodes, int cd[3], double h[3], double spacing = 4.0);

// Builds Zc = P^T Z P from Z in CSR (pressure-node numbering) and inverts it
// (Cholesky, FP64); with_w also keeps W = Z P in 27-tap boxes.  vox_of_p
// maps a pressure node to its voxel (empty: identity).  Returns 0, or -1 with
// err set when Zc is not positive definite.
// factor = false: cs.inv receives Zc itself (dense, symmetric, row-major),
// to be factored and inverted elsewhere (on the device).
int coarse_build(const int fd[3], int max_nodes, const std::vector<int>& vox_of_p, const std::vector<int>& rp,
                 const std::vector<int>& col, const std::vector<double>& val, CoarseSpace& cs, std::string& err,
                 bool with_w = false, bool factor = true, double spacing = 4.0);

}  // namespace cfd
