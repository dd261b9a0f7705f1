// Host-side problem description: the deck as read, the generated hex27 node
// numbering and every CSR pattern the device operators need.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace cfd {

struct HostProblem {
  // header, blascoCodinaHuerta.cpp:545-562
  int eType = 1, NE = 0, NCN = 0, NENv = 27, NENp = 8, NGP = 8;
  double alpha = 0, dt = 0, t_ini = 0, t_final = 0;
  int maxIter = 1;
  double tolerance = 0, convergence = 0;
  int isRestart = 0;
  double density = 1, viscosity = 1, fx = 0, fy = 0;

  int NN = 0, NNp = 0;
  std::vector<double> coord;   // NN x 3 after preprocessing (NCN x 3 as read)
  std::vector<int> ltog;       // NE x 27 (first 8 read from the deck)
  int nBC = 0;
  std::vector<double> bcstr;   // nBC x 3
  std::vector<int> velfaces;   // nVelFaces x 3 (element, face, bc), 0-based
  std::vector<int> outfaces;   // nOutFaces x 3, 0-based (natural BC; unused)
  int zeroP = -1;
  double mon[3] = {0, 0, 0};
  int monPoint = 0;

  // Dirichlet nodes, ascending, with their BC id (blascoCodinaHuerta.cpp:1543-1565)
  std::vector<int> bcnode, bcid;

  // CSR patterns (rows sorted ascending)
  std::vector<int> k_rp, k_col;           // NN x NN block shared by M, K, A
  std::vector<int> g_rp, g_col;           // NN x NNp (G1, G2, G3)
  std::vector<int> gt_rp, gt_col, gt_pos; // NNp x NN; gt_pos = index of (v,p) in G
  std::vector<int> z_rp, z_col;           // NNp x NNp
  int maxZrow = 0, maxKrow = 0, maxGrow = 0, maxGtrow = 0;
  // stored entries of K, G (= G^T) and Z, whichever side built the patterns
  long long nnzK = 0, nnzG = 0, nnzZ = 0;
};

// readInputFile semantics (blascoCodinaHuerta.cpp:528-725).  Returns 0 or a
// negative cfd_status; err receives a message.
int read_inp(const std::string& path, HostProblem& P, std::string& err);

// Fills NN, coord, ltog (mid nodes), bcnode/bcid, monPoint and, with
// patterns, every CSR pattern (the solver builds them on the device
// instead and calls build_patterns only as a fallback).
int preprocess(HostProblem& P, std::string& err, bool patterns = true);
// The CSR patterns of K, G, G^T (with gt_pos) and Z from ltog.
int build_patterns(HostProblem& P, std::string& err);

// Conflict-free greedy colouring of the elements over their corner nodes
// (elements that share a node get different colours): order lists the
// elements colour by colour (ascending element id inside a colour), colour c
// owns order[off[c] .. off[c+1]).  The reference colours elements for the
// same purpose, serialising its scatters (setupMeshColoring,
// blascoCodinaHuerta.cpp:853-947).  Returns 0, or -1 beyond 64 colours.
int color_elements(const HostProblem& P, std::vector<int>& order, std::vector<int>& off);

// Edge corner pairs, face corner quads and face mid-node lists of a hex27
// element (blascoCodinaHuerta.cpp:1005-1054, 1143-1180, 1485-1528).
extern const int kEdge[12][2];
extern const int kFace[6][4];
extern const int kFaceMid[6][5];
extern const int kNode27[27][3];
extern const int kSubBrick[8][8];

}  // namespace cfd
