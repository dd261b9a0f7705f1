// ============================================================================
//  fs_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle; never the product)
//
//  CPU FP64 restatement of the fractional-step (Blasco-Codina-Huerta 1998)
//  hex27-velocity / hex8-pressure Navier-Stokes solver of the reference,
//  fractionalStep/Cpp/blascoCodinaHuerta.cpp (cited below as BCH.cpp:<line>),
//  and of its GPU twin fractionalStep/Cpp/CUDAcodes.cu (CU.cu:<line>).
//
//  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
//  this library, and only as the checker.  The product (libcfdfs.so) never
//  links, calls or falls back to it.
//
//  Third-party arithmetic the reference delegates and how it is restated:
//    * MKL mkl_dcsrmv / cuSPARSE csrmv      -> plain CSR row loops (same math).
//    * CSparse cs_multiply (Z = G^T D G)    -> explicit accumulation in the
//      column-scatter order of CSparse's published cs_multiply (Davis 2006).
//    * MKL dcg / cusp::krylov::cg + Jacobi  -> own Jacobi-PCG with the stopping
//      rule ||r||_2 <= rtol*||b||_2 and a selectable initial guess (0 = the MKL
//      call site BCH.cpp:4002-4004, warm = the CUSP call site CU.cu:268,430).
//      MKL dcg tests squared norms, so the reference's dpar[0] = 1e-12
//      (BCH.cpp:4018) is rtol = 1e-6 here.
//  Parity with the reference is PINNED: the reference's own CPU solver,
//  compiled unmodified against the MKL/CSparse stand-ins of oracle/refshim
//  (oracle/_ref/fs_ref), produced the fixtures tests/golden/ref_*.npz, and
//  this oracle reproduces them (final fields to 1e-9, every pressure solve's
//  CG iteration count and every monitor row exactly, the node numbering bit
//  for bit; tests/test_ref_parity.py).  Known-answer tests derived from the
//  mathematics (partition of unity, element volumes, K*1=0, Z symmetric
//  positive definite, nnz formulas) check it as well.
//
//  Floating-point contraction is disabled at build time (-ffp-contract=off).
//  Reductions use a fixed chunking so results do not depend on thread count.
// ============================================================================
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kChunks = 64;  // fixed reduction chunking (deterministic sums)

template <class F>
double det_sum(long n, F f) {
  double part[kChunks];
#pragma omp parallel for schedule(static)
  for (int c = 0; c < kChunks; ++c) {
    long b = n * c / kChunks, e = n * (c + 1) / kChunks;
    double s = 0.0;
    for (long i = b; i < e; ++i) s += f(i);
    part[c] = s;
  }
  double s = 0.0;
  for (int c = 0; c < kChunks; ++c) s += part[c];
  return s;
}

struct CgStats {
  int its = 0;
  double relres = 0.0;
  int status = 0;  // 0 converged, 1 max iterations, 2 non-finite
};

struct Oracle {
  // ---- header fields, BCH.cpp:147-172, read at BCH.cpp:545-562 ----
  int eType = 1, NE = 0, NCN = 0, NENv = 27, NENp = 8, NGP = 8;
  double alpha = 0, dt = 0, t_ini = 0, t_final = 0;
  int maxIter = 1;
  double tolerance = 0, convergenceCriteria = 0;
  int isRestart = 0;
  double density = 1, viscosity = 1, fx = 0, fy = 0;
  int NN = 0, NNp = 0, NEC = 8, NEF = 6, NEE = 12;
  std::string basename;

  std::vector<double> coord;   // (NE*NENv) x 3 while generating, NN x 3 after
  std::vector<int> LtoGnode;   // NE x NENv
  int nBC = 0;
  std::vector<double> BCtype, BCstr;           // nBC, nBC x 3
  int BCnVelFaces = 0, BCnOutFaces = 0;
  std::vector<int> BCvelFaces, BCoutFaces;     // n x 3 (0-based)
  int zeroPressureNode = -1;
  double monPointCoord[3] = {0, 0, 0};
  int monPoint = 0;
  std::vector<int> BCvelNodes;  // BCnVelNodes x 2 (node, bc), sorted by node
  int BCnVelNodes = 0;

  // adjacency, BCH.cpp:732-947
  std::vector<int> elemsOfPresNodes, NelemOfPresNodes;  // NNp x 10
  std::vector<int> elemNeighbors, NelemNeighbors;       // NE x 26
  std::vector<int> meshColors, NmeshColors, elementsOfColor;
  int nActiveColors = 0;
  std::vector<int> elemsOfVelNodes, NelemOfVelNodes;    // NN x 10

  // sparse patterns, BCH.cpp:1675-2159
  std::vector<int> Mrow, Mcol, MrowStarts;  // one NN x NN block (M, K, A)
  std::vector<double> Mval, Kval;
  std::vector<int> Grow, Gcol, GrowStarts;  // NN x NNp (G1, G2, G3)
  std::vector<double> G1, G2, G3;
  std::vector<int> sparseMapM, sparseMapG;  // NE x 27 x 27, NE x 27 x 8

  // Z (sorted CSR) and its diagonal positions
  std::vector<int> ZrowStarts, Zcol;
  std::vector<double> Zval, Zdiag;

  // basis, BCH.cpp:2166-2711
  std::vector<double> GQpoint, GQweight;  // NGP x 3, NGP
  std::vector<double> Sv, dSv, Sp, dSp;   // Sv[k][i]; dSv[d][i][k]; Sp[k][m]; dSp[d][m][k]
  std::vector<double> detJacob, gDSv;     // NE x NGP ; NE x NGP x NENv x 3

  // state, BCH.cpp:261-289
  std::vector<double> Un, Unp1, Unp1_prev, UnpHalf, UnpHalf_prev, Acc, Acc_prev;
  std::vector<double> Pn, Pnp1, Pnp1_prev, Pdot;
  std::vector<double> Md, MdOrig, MdInv, MdOrigInv, KtimesAcc_prev;
  std::vector<double> R1, R2, R3;
  int timeN = 0;
  double timeT = 0;
  double maxAcc = 0;
  double lastNorm1 = 0, lastNorm2 = 0;

  // solver controls (not in the reference input deck)
  double cg_rtol = 1e-8;
  int cg_maxit = 1000;
  int cg_warm = 0;
  int print_monitor = 0;
  CgStats last_cg;
  long cg_total_its = 0;
  int last_iters = 0;
  // Run logs for comparison with the reference's screen output: CG
  // iterations of every pressure solve ("MKL_CG converged after N
  // iterations.", BCH.cpp:4032) and one monitor row per time step
  // (timeN, iter, timeT, u, v, w, p, maxAcc; BCH.cpp:3091-3093).
  std::vector<int> cg_log;
  std::vector<double> mon_log;

  // ------------------------------------------------------------------------
  // readInputFile, BCH.cpp:528-725.  Same token semantics: every header value
  // follows the first ':' on its line; 1-based ids become 0-based.
  // ------------------------------------------------------------------------
  int readInputFile(const std::string& path) {
    std::ifstream in(path.c_str());
    if (!in) return -1;
    std::string dummy;
    int intDummy;
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    auto hdr = [&](auto& v) {
      in.ignore(256, ':');
      in >> v;
      in.ignore(256, '\n');
    };
    hdr(eType); hdr(NE); hdr(NCN); hdr(NENv); hdr(NENp); hdr(NGP);
    hdr(alpha); hdr(dt); hdr(t_ini); hdr(t_final); hdr(maxIter);
    hdr(tolerance); hdr(convergenceCriteria); hdr(isRestart);
    hdr(density); hdr(viscosity); hdr(fx); hdr(fy);
    if (!in || NE <= 0 || NCN <= 0 || NENv != 27 || NENp != 8 || eType != 1) return -2;

    coord.assign((size_t)NE * NENv * 3, 0.0);
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    for (int i = 0; i < NCN; i++) {
      in >> intDummy >> coord[3 * i] >> coord[3 * i + 1] >> coord[3 * i + 2];
      in.ignore(256, '\n');
    }
    NEC = 8; NEF = 6; NEE = 12;
    LtoGnode.assign((size_t)NE * NENv, -1);
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    for (int e = 0; e < NE; e++) {
      in >> intDummy;
      for (int i = 0; i < NEC; i++) {
        int v;
        in >> v;
        LtoGnode[(size_t)e * NENv + i] = v - 1;
      }
      in.ignore(256, '\n');
    }
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    in.ignore(256, ':');
    in >> nBC;
    in.ignore(256, '\n');
    BCtype.assign(nBC, 0.0);
    BCstr.assign((size_t)nBC * 3, 0.0);
    for (int i = 0; i < nBC; i++) {
      in.ignore(256, ':');
      in >> BCtype[i];
      in >> BCstr[3 * i + 0];
      in >> dummy;
      in >> BCstr[3 * i + 1];
      in >> dummy;
      in >> BCstr[3 * i + 2];
      in.ignore(256, '\n');
    }
    in.ignore(256, '\n');
    in.ignore(256, ':');
    in >> BCnVelFaces;
    in.ignore(256, '\n');
    in.ignore(256, ':');
    in >> BCnOutFaces;
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    BCvelFaces.assign((size_t)BCnVelFaces * 3, 0);
    for (int i = 0; i < BCnVelFaces; i++) {
      in >> BCvelFaces[3 * i] >> BCvelFaces[3 * i + 1] >> BCvelFaces[3 * i + 2];
      for (int j = 0; j < 3; j++) BCvelFaces[3 * i + j] -= 1;
      in.ignore(256, '\n');
    }
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    BCoutFaces.assign((size_t)BCnOutFaces * 3, 0);
    for (int i = 0; i < BCnOutFaces; i++) {
      in >> BCoutFaces[3 * i] >> BCoutFaces[3 * i + 1] >> BCoutFaces[3 * i + 2];
      for (int j = 0; j < 3; j++) BCoutFaces[3 * i + j] -= 1;
      in.ignore(256, '\n');
    }
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    in >> zeroPressureNode;
    zeroPressureNode -= 1;
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    in >> monPointCoord[0] >> monPointCoord[1] >> monPointCoord[2];
    if (in.fail()) return -3;
    NNp = (NENp == 1) ? NE : NCN;  // BCH.cpp:718-723
    return 0;
  }

  int& L(int e, int i) { return LtoGnode[(size_t)e * NENv + i]; }

  // findElemsOfPresNodes, BCH.cpp:732-783 (fixed width 10)
  void findElemsOfPresNodes() {
    elemsOfPresNodes.assign((size_t)NNp * 10, -1);
    NelemOfPresNodes.assign(NNp, 0);
    for (int e = 0; e < NE; e++)
      for (int i = 0; i < NENp; i++) {
        int node = L(e, i);
        elemsOfPresNodes[(size_t)node * 10 + NelemOfPresNodes[node]] = e;
        NelemOfPresNodes[node]++;
      }
  }

  // findElemNeighbors, BCH.cpp:790-846 (elements sharing a corner, width 26)
  void findElemNeighbors() {
    elemNeighbors.assign((size_t)NE * 26, -1);
    NelemNeighbors.assign(NE, 0);
    for (int e = 0; e < NE; e++) {
      int* nb = &elemNeighbors[(size_t)e * 26];
      for (int i = 0; i < NEC; i++) {
        int node = L(e, i);
        for (int j = 0; j < NelemOfPresNodes[node]; j++) {
          int elem = elemsOfPresNodes[(size_t)node * 10 + j];
          if (elem == e) continue;
          bool inList = false;
          for (int k = 0; k < NelemNeighbors[e]; k++)
            if (nb[k] == elem) { inList = true; break; }
          if (!inList) nb[NelemNeighbors[e]++] = elem;
        }
      }
    }
  }

  // setupMeshColoring, BCH.cpp:853-947.  The greedy loop is kept as written,
  // including its restart quirk (after a clash the scan resumes at neighbour 1,
  // BCH.cpp:880-886).
  void setupMeshColoring() {
    const int LARGE = 30;
    meshColors.assign(NE, -1);
    NmeshColors.assign(LARGE, 0);
    elementsOfColor.assign(NE, 0);
    for (int e = 0; e < NE; e++) {
      int candidate = 0;
      for (int i = 0; i < NelemNeighbors[e]; i++) {
        int elem = elemNeighbors[(size_t)e * 26 + i];
        if (candidate == meshColors[elem]) {
          candidate++;
          i = 0;
        }
      }
      meshColors[e] = candidate;
      NmeshColors[candidate]++;
    }
    int count = 0;
    nActiveColors = 0;
    for (int c = 0; c < LARGE; c++) {
      if (NmeshColors[c] > 0) {
        nActiveColors++;
        for (int e = 0; e < NE; e++)
          if (meshColors[e] == c) elementsOfColor[count++] = e;
      }
    }
  }

  // Corner pairs of the 12 edges and corner quads of the 6 faces
  // (BCH.cpp:1005-1054 and 1143-1180).
  static constexpr int kEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 5},
                                       {2, 6}, {3, 7}, {4, 5}, {5, 6}, {6, 7}, {7, 4}};
  static constexpr int kFace[6][4] = {{0, 1, 2, 3}, {0, 1, 4, 5}, {1, 2, 5, 6},
                                      {2, 3, 6, 7}, {0, 3, 4, 7}, {4, 5, 6, 7}};
  // Non-corner nodes of each face, BCH.cpp:1485-1528.
  static constexpr int kFaceMid[6][5] = {{8, 9, 10, 11, 20},  {8, 12, 13, 16, 21},
                                         {9, 13, 14, 17, 22}, {10, 14, 15, 18, 23},
                                         {11, 12, 15, 19, 24}, {16, 17, 18, 19, 25}};

  // setupNonCornerNodes, BCH.cpp:954-1320.  New mid-edge and mid-face nodes
  // are numbered in element-then-edge (face) order; a candidate is matched
  // against the already numbered mid-nodes of the neighbouring elements by
  // coordinates (|dx|,|dy|,|dz| < 1e-10).  Centre nodes come last.
  void setupNonCornerNodes() {
    const double SMALL = 1e-10;
    int nodeCount = NCN;
    std::vector<int> neighborMN;
    neighborMN.reserve(26 * 12);
    for (int e = 0; e < NE; e++) {
      neighborMN.clear();
      for (int e2 = 0; e2 < NelemNeighbors[e]; e2++) {
        int ne = elemNeighbors[(size_t)e * 26 + e2];
        for (int i = NEC; i < NEC + NEE; i++)
          if (L(ne, i) != -1) neighborMN.push_back(L(ne, i));
      }
      for (int ed = 0; ed < NEE; ed++) {
        int n1 = L(e, kEdge[ed][0]), n2 = L(e, kEdge[ed][1]);
        double m[3];
        for (int d = 0; d < 3; d++) m[d] = 0.5 * (coord[3 * (size_t)n1 + d] + coord[3 * (size_t)n2 + d]);
        bool found = false;
        for (int c : neighborMN) {
          if (std::fabs(m[0] - coord[3 * (size_t)c]) < SMALL &&
              std::fabs(m[1] - coord[3 * (size_t)c + 1]) < SMALL &&
              std::fabs(m[2] - coord[3 * (size_t)c + 2]) < SMALL) {
            L(e, ed + NEC) = c;
            found = true;
            break;
          }
        }
        if (!found) {
          L(e, ed + NEC) = nodeCount;
          for (int d = 0; d < 3; d++) coord[3 * (size_t)nodeCount + d] = m[d];
          nodeCount++;
        }
      }
    }
    for (int e = 0; e < NE; e++) {
      neighborMN.clear();
      for (int e2 = 0; e2 < NelemNeighbors[e]; e2++) {
        int ne = elemNeighbors[(size_t)e * 26 + e2];
        for (int i = NEC + NEE; i < NENv; i++)
          if (L(ne, i) != -1) neighborMN.push_back(L(ne, i));
      }
      for (int f = 0; f < NEF; f++) {
        int n[4];
        for (int j = 0; j < 4; j++) n[j] = L(e, kFace[f][j]);
        double m[3];
        for (int d = 0; d < 3; d++)
          m[d] = 0.25 * (coord[3 * (size_t)n[0] + d] + coord[3 * (size_t)n[1] + d] +
                         coord[3 * (size_t)n[2] + d] + coord[3 * (size_t)n[3] + d]);
        bool found = false;
        for (int c : neighborMN) {
          if (std::fabs(m[0] - coord[3 * (size_t)c]) < SMALL &&
              std::fabs(m[1] - coord[3 * (size_t)c + 1]) < SMALL &&
              std::fabs(m[2] - coord[3 * (size_t)c + 2]) < SMALL) {
            L(e, f + NEC + NEE) = c;
            found = true;
            break;
          }
        }
        if (!found) {
          L(e, f + NEC + NEE) = nodeCount;
          for (int d = 0; d < 3; d++) coord[3 * (size_t)nodeCount + d] = m[d];
          nodeCount++;
        }
      }
    }
    for (int e = 0; e < NE; e++) {
      double m[3];
      for (int d = 0; d < 3; d++) {
        double s = coord[3 * (size_t)L(e, 0) + d];
        for (int j = 1; j < 8; j++) s = s + coord[3 * (size_t)L(e, j) + d];
        m[d] = 0.125 * s;
      }
      L(e, NEC + NEE + NEF) = nodeCount;
      for (int d = 0; d < 3; d++) coord[3 * (size_t)nodeCount + d] = m[d];
      nodeCount++;
    }
    NN = nodeCount;
    coord.resize((size_t)NN * 3);
    coord.shrink_to_fit();
  }

  // Velocity dof of local index i (0..3*NENv-1) of element e: component
  // blocks [u | v | w], BCH.cpp:1348-1368.
  int LtoGvel(int e, int i) const {
    int comp = i / NENv, loc = i % NENv;
    return comp * NN + LtoGnode[(size_t)e * NENv + loc];
  }

  // determineVelBCnodes, BCH.cpp:1410-1580 (later faces overwrite earlier).
  void determineVelBCnodes() {
    std::vector<double> velBCinfo(NN, -1.0);
    for (int i = 0; i < BCnVelFaces; i++) {
      int e = BCvelFaces[3 * i], f = BCvelFaces[3 * i + 1], which = BCvelFaces[3 * i + 2];
      for (int j = 0; j < 4; j++) velBCinfo[L(e, kFace[f][j])] = which;
      for (int j = 0; j < 5; j++) velBCinfo[L(e, kFaceMid[f][j])] = which;
    }
    BCvelNodes.clear();
    for (int i = 0; i < NN; i++)
      if (velBCinfo[i] != -1) {
        BCvelNodes.push_back(i);
        BCvelNodes.push_back(int(velBCinfo[i]));
      }
    BCnVelNodes = (int)BCvelNodes.size() / 2;
  }

  // findElemsOfVelNodes, BCH.cpp:1587-1637
  void findElemsOfVelNodes() {
    elemsOfVelNodes.assign((size_t)NN * 10, -1);
    NelemOfVelNodes.assign(NN, 0);
    for (int e = 0; e < NE; e++)
      for (int i = 0; i < NENv; i++) {
        int node = L(e, i);
        elemsOfVelNodes[(size_t)node * 10 + NelemOfVelNodes[node]] = e;
        NelemOfVelNodes[node]++;
      }
  }

  // findMonitorPoint, BCH.cpp:1644-1668 (first minimum among corner nodes)
  void findMonitorPoint() {
    double distance = 1e6;
    for (int i = 0; i < NCN; i++) {
      double dx = coord[3 * (size_t)i] - monPointCoord[0];
      double dy = coord[3 * (size_t)i + 1] - monPointCoord[1];
      double dz = coord[3 * (size_t)i + 2] - monPointCoord[2];
      if (std::sqrt(dx * dx + dy * dy + dz * dz) < distance) {
        distance = std::sqrt(dx * dx + dy * dy + dz * dz);
        monPoint = i;
      }
    }
  }

  // setupSparseM, BCH.cpp:1675-1921: CSR of one NN x NN block (sorted
  // columns) and sparseMapM[e][i][j] by linear search in the row.
  void setupSparseM() {
    MrowStarts.assign(NN + 1, 0);
    std::vector<std::vector<int>> rows(NN);
#pragma omp parallel
    {
      std::vector<char> isColNZ(NN, 0);
#pragma omp for schedule(static)
      for (int r = 0; r < NN; r++) {
        std::vector<int>& cols = rows[r];
        for (int i = 0; i < NelemOfVelNodes[r]; i++) {
          int e = elemsOfVelNodes[(size_t)r * 10 + i];
          for (int j = 0; j < NENv; j++) {
            int c = L(e, j);
            if (!isColNZ[c]) { isColNZ[c] = 1; cols.push_back(c); }
          }
        }
        for (int c : cols) isColNZ[c] = 0;
        std::sort(cols.begin(), cols.end());
      }
    }
    for (int r = 0; r < NN; r++) MrowStarts[r + 1] = MrowStarts[r] + (int)rows[r].size();
    long nnz = MrowStarts[NN];
    Mcol.resize(nnz);
    Mrow.resize(nnz);
    for (int r = 0; r < NN; r++) {
      std::copy(rows[r].begin(), rows[r].end(), Mcol.begin() + MrowStarts[r]);
      std::fill(Mrow.begin() + MrowStarts[r], Mrow.begin() + MrowStarts[r + 1], r);
      std::vector<int>().swap(rows[r]);
    }
    sparseMapM.assign((size_t)NE * NENv * NENv, 0);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < NE; e++)
      for (int i = 0; i < NENv; i++) {
        int r = L(e, i);
        const int* col = &Mcol[MrowStarts[r]];
        int n = MrowStarts[r + 1] - MrowStarts[r];
        for (int j = 0; j < NENv; j++) {
          int jj = L(e, j), c;
          for (c = 0; c < n; c++)
            if (col[c] == jj) break;
          sparseMapM[((size_t)e * NENv + i) * NENv + j] = c + MrowStarts[r];
        }
      }
  }

  // setupSparseG, BCH.cpp:1928-2159: CSR of NN x NNp and sparseMapG.
  void setupSparseG() {
    GrowStarts.assign(NN + 1, 0);
    std::vector<std::vector<int>> rows(NN);
#pragma omp parallel
    {
      std::vector<char> isColNZ(NNp, 0);
#pragma omp for schedule(static)
      for (int r = 0; r < NN; r++) {
        std::vector<int>& cols = rows[r];
        for (int i = 0; i < NelemOfVelNodes[r]; i++) {
          int e = elemsOfVelNodes[(size_t)r * 10 + i];
          for (int j = 0; j < NENp; j++) {
            int c = L(e, j);
            if (!isColNZ[c]) { isColNZ[c] = 1; cols.push_back(c); }
          }
        }
        for (int c : cols) isColNZ[c] = 0;
        std::sort(cols.begin(), cols.end());
      }
    }
    for (int r = 0; r < NN; r++) GrowStarts[r + 1] = GrowStarts[r] + (int)rows[r].size();
    long nnz = GrowStarts[NN];
    Gcol.resize(nnz);
    Grow.resize(nnz);
    for (int r = 0; r < NN; r++) {
      std::copy(rows[r].begin(), rows[r].end(), Gcol.begin() + GrowStarts[r]);
      std::fill(Grow.begin() + GrowStarts[r], Grow.begin() + GrowStarts[r + 1], r);
    }
    sparseMapG.assign((size_t)NE * NENv * NENp, 0);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < NE; e++)
      for (int i = 0; i < NENv; i++) {
        int r = L(e, i);
        const int* col = &Gcol[GrowStarts[r]];
        int n = GrowStarts[r + 1] - GrowStarts[r];
        for (int j = 0; j < NENp; j++) {
          int jj = L(e, j), c;
          for (c = 0; c < n; c++)
            if (col[c] == jj) break;
          sparseMapG[((size_t)e * NENv + i) * NENp + j] = c + GrowStarts[r];
        }
      }
  }

  // setupGQ, BCH.cpp:2166-2208.  NGP 1 and 8 as in the reference (the
  // 8-point rule orders xi fastest).  NGP 27 is an empty TODO in the
  // reference (BCH.cpp:2197-2201); the oracle adds the 3x3x3 Gauss-Legendre
  // rule in the same xi-fastest ordering.
  int setupGQ() {
    GQpoint.assign((size_t)NGP * 3, 0.0);
    GQweight.assign(NGP, 0.0);
    if (NGP == 1) {
      GQweight[0] = 4.0;  // as BCH.cpp:2179
    } else if (NGP == 8) {
      double g = std::sqrt(1. / 3);
      for (int k = 0; k < 8; k++) {
        GQpoint[3 * k + 0] = (k & 1) ? g : -g;
        GQpoint[3 * k + 1] = (k & 2) ? g : -g;
        GQpoint[3 * k + 2] = (k & 4) ? g : -g;
        GQweight[k] = 1.0;
      }
    } else if (NGP == 27) {
      const double p[3] = {-std::sqrt(0.6), 0.0, std::sqrt(0.6)};
      const double w[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
      for (int c = 0; c < 3; c++)
        for (int b = 0; b < 3; b++)
          for (int a = 0; a < 3; a++) {
            int k = a + 3 * b + 9 * c;
            GQpoint[3 * k + 0] = p[a];
            GQpoint[3 * k + 1] = p[b];
            GQpoint[3 * k + 2] = p[c];
            GQweight[k] = w[a] * w[b] * w[c];
          }
    } else {
      return -1;
    }
    return 0;
  }

  // 1D quadratic Lagrange factors on nodes -1, 0, +1 (index 0, 1, 2) and
  // their derivatives; hex27 functions are products of three of them.
  static double q1(int a, double x) {
    return a == 0 ? 0.5 * (x * x - x) : (a == 1 ? 1.0 - x * x : 0.5 * (x * x + x));
  }
  static double dq1(int a, double x) {
    return a == 0 ? 0.5 * (2 * x - 1) : (a == 1 ? -2 * x : 0.5 * (2 * x + 1));
  }
  // (xi, eta, zeta) position index of each hex27 local node, in the
  // reference's local numbering (corners 0-7, mid-edges 8-19, mid-faces
  // 20-25, centre 26), BCH.cpp:2312-2343.
  static constexpr int kNode27[27][3] = {
      {0, 0, 0}, {2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {0, 0, 2}, {2, 0, 2}, {2, 2, 2},
      {0, 2, 2}, {1, 0, 0}, {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 1},
      {2, 2, 1}, {0, 2, 1}, {1, 0, 2}, {2, 1, 2}, {1, 2, 2}, {0, 1, 2}, {1, 1, 0},
      {1, 0, 1}, {2, 1, 1}, {1, 2, 1}, {0, 1, 1}, {1, 1, 2}, {1, 1, 1}};

  // calcShape, BCH.cpp:2215-2488: hex8 Sp, dSp and hex27 Sv, dSv at the GPs.
  void calcShape() {
    Sv.assign((size_t)NGP * NENv, 0.0);
    Sp.assign((size_t)NGP * NENp, 0.0);
    dSv.assign((size_t)3 * NENv * NGP, 0.0);
    dSp.assign((size_t)3 * NENp * NGP, 0.0);
    for (int k = 0; k < NGP; k++) {
      double x[3] = {GQpoint[3 * k], GQpoint[3 * k + 1], GQpoint[3 * k + 2]};
      for (int m = 0; m < 8; m++) {
        double s[3];
        for (int d = 0; d < 3; d++) s[d] = (kNode27[m][d] == 0) ? -1.0 : 1.0;
        double f[3], df[3];
        for (int d = 0; d < 3; d++) { f[d] = 1 + s[d] * x[d]; df[d] = s[d]; }
        Sp[(size_t)k * 8 + m] = 0.125 * f[0] * f[1] * f[2];
        dSp[((size_t)0 * 8 + m) * NGP + k] = 0.125 * df[0] * f[1] * f[2];
        dSp[((size_t)1 * 8 + m) * NGP + k] = 0.125 * f[0] * df[1] * f[2];
        dSp[((size_t)2 * 8 + m) * NGP + k] = 0.125 * f[0] * f[1] * df[2];
      }
      for (int i = 0; i < 27; i++) {
        int a = kNode27[i][0], b = kNode27[i][1], c = kNode27[i][2];
        Sv[(size_t)k * 27 + i] = q1(a, x[0]) * q1(b, x[1]) * q1(c, x[2]);
        dSv[((size_t)0 * 27 + i) * NGP + k] = dq1(a, x[0]) * q1(b, x[1]) * q1(c, x[2]);
        dSv[((size_t)1 * 27 + i) * NGP + k] = q1(a, x[0]) * dq1(b, x[1]) * q1(c, x[2]);
        dSv[((size_t)2 * 27 + i) * NGP + k] = q1(a, x[0]) * q1(b, x[1]) * dq1(c, x[2]);
      }
    }
  }

  // calcJacob, BCH.cpp:2495-2711: J from the 8 corner nodes (trilinear map
  // even for hex27), adjugate inverse, detJ, global derivatives gDSv.
  void calcJacob() {
    detJacob.assign((size_t)NE * NGP, 0.0);
    gDSv.assign((size_t)NE * NGP * NENv * 3, 0.0);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < NE; e++) {
      double X[8][3];
      for (int i = 0; i < 8; i++)
        for (int d = 0; d < 3; d++) X[i][d] = coord[3 * (size_t)L(e, i) + d];
      for (int k = 0; k < NGP; k++) {
        double J[3][3], iJ[3][3];
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) {
            double s = 0;
            for (int m = 0; m < 8; m++) s = s + dSp[((size_t)i * 8 + m) * NGP + k] * X[m][j];
            J[i][j] = s;
          }
        iJ[0][0] = J[1][1] * J[2][2] - J[2][1] * J[1][2];
        iJ[0][1] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]);
        iJ[0][2] = J[0][1] * J[1][2] - J[1][1] * J[0][2];
        iJ[1][0] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]);
        iJ[1][1] = J[2][2] * J[0][0] - J[2][0] * J[0][2];
        iJ[1][2] = -(J[1][2] * J[0][0] - J[1][0] * J[0][2]);
        iJ[2][0] = J[1][0] * J[2][1] - J[2][0] * J[1][1];
        iJ[2][1] = -(J[2][1] * J[0][0] - J[2][0] * J[0][1]);
        iJ[2][2] = J[1][1] * J[0][0] - J[1][0] * J[0][1];
        double det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) +
                     J[0][1] * (J[1][2] * J[2][0] - J[1][0] * J[2][2]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        detJacob[(size_t)e * NGP + k] = det;
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) iJ[i][j] = iJ[i][j] / det;
        for (int j = 0; j < NENv; j++)
          for (int i = 0; i < 3; i++) {
            double s = 0;
            for (int m = 0; m < 3; m++) s = s + iJ[i][m] * dSv[((size_t)m * 27 + j) * NGP + k];
            gDSv[(((size_t)e * NGP + k) * NENv + j) * 3 + i] = s;
          }
      }
    }
  }

  // initializeAndAllocate + applyBC_initial, BCH.cpp:2718-2808, 4062-4110
  void initializeAndAllocate() {
    size_t n3 = (size_t)3 * NN;
    for (auto* v : {&Un, &Unp1, &Unp1_prev, &UnpHalf, &UnpHalf_prev, &Acc, &Acc_prev, &Md, &MdOrig,
                    &MdInv, &MdOrigInv, &KtimesAcc_prev, &R1, &R3})
      v->assign(n3, 0.0);
    for (auto* v : {&Pn, &Pnp1, &Pnp1_prev, &Pdot, &R2}) v->assign(NNp, 0.0);
    for (int i = 0; i < BCnVelNodes; i++) {
      int node = BCvelNodes[2 * i], which = BCvelNodes[2 * i + 1];
      Un[node] = BCstr[3 * which + 0];
      Un[node + NN] = BCstr[3 * which + 1];
      Un[node + 2 * (size_t)NN] = BCstr[3 * which + 2];
    }
    timeN = 0;
    timeT = t_ini;
  }

  // step0, BCH.cpp:3127-3315: element Me, Ke, Ge assembled through the slot
  // maps; Md = row sums of M; MdOrig(Inv); Md = 1 at Dirichlet nodes; Z.
  void step0() {
    long nnzM = MrowStarts[NN], nnzG = GrowStarts[NN];
    Mval.assign(nnzM, 0.0);
    Kval.assign(nnzM, 0.0);
    G1.assign(nnzG, 0.0);
    G2.assign(nnzG, 0.0);
    G3.assign(nnzG, 0.0);
    const double inverseDensity = 1.0 / density;
    // Element matrices are computed in parallel and scattered in element
    // order, which reproduces the reference's sequential summation order.
    const int B = 4096;
    std::vector<double> Me((size_t)B * 729), Ke((size_t)B * 729), Ge((size_t)B * 3 * 216);
    for (int e0 = 0; e0 < NE; e0 += B) {
      int e1 = std::min(NE, e0 + B);
#pragma omp parallel for schedule(static)
      for (int e = e0; e < e1; e++) {
        double* me = &Me[(size_t)(e - e0) * 729];
        double* ke = &Ke[(size_t)(e - e0) * 729];
        double* ge = &Ge[(size_t)(e - e0) * 648];
        std::fill(me, me + 729, 0.0);
        std::fill(ke, ke + 729, 0.0);
        std::fill(ge, ge + 648, 0.0);
        for (int k = 0; k < NGP; k++) {
          double GQfactor = detJacob[(size_t)e * NGP + k] * GQweight[k];
          const double* gd = &gDSv[(((size_t)e * NGP + k) * NENv) * 3];
          const double* sv = &Sv[(size_t)k * 27];
          for (int i = 0; i < 27; i++)
            for (int j = 0; j < 27; j++) {
              me[i * 27 + j] = me[i * 27 + j] + sv[i] * sv[j] * GQfactor;
              ke[i * 27 + j] = ke[i * 27 + j] +
                               viscosity * (gd[3 * i] * gd[3 * j] + gd[3 * i + 1] * gd[3 * j + 1] +
                                            gd[3 * i + 2] * gd[3 * j + 2]) * GQfactor;
            }
          for (int i = 0; i < 27; i++)
            for (int j = 0; j < 8; j++) {
              double spj = Sp[(size_t)k * 8 + j];
              ge[0 * 216 + i * 8 + j] = ge[0 * 216 + i * 8 + j] - inverseDensity * spj * gd[3 * i + 0] * GQfactor;
              ge[1 * 216 + i * 8 + j] = ge[1 * 216 + i * 8 + j] - inverseDensity * spj * gd[3 * i + 1] * GQfactor;
              ge[2 * 216 + i * 8 + j] = ge[2 * 216 + i * 8 + j] - inverseDensity * spj * gd[3 * i + 2] * GQfactor;
            }
        }
      }
      for (int e = e0; e < e1; e++) {
        const double* me = &Me[(size_t)(e - e0) * 729];
        const double* ke = &Ke[(size_t)(e - e0) * 729];
        const double* ge = &Ge[(size_t)(e - e0) * 648];
        const int* mapM = &sparseMapM[(size_t)e * 729];
        const int* mapG = &sparseMapG[(size_t)e * 216];
        for (int t = 0; t < 729; t++) {
          Mval[mapM[t]] += me[t];
          Kval[mapM[t]] += ke[t];
        }
        for (int t = 0; t < 216; t++) {
          G1[mapG[t]] += ge[t];
          G2[mapG[t]] += ge[216 + t];
          G3[mapG[t]] += ge[432 + t];
        }
      }
    }
    for (long i = 0; i < nnzM; i++) Md[Mrow[i]] += Mval[i];
    for (int i = 0; i < NN; i++) {
      Md[i + NN] = Md[i];
      Md[i + 2 * (size_t)NN] = Md[i];
    }
    std::vector<double>().swap(Mval);
    for (size_t i = 0; i < (size_t)3 * NN; i++) {
      MdOrig[i] = Md[i];
      MdOrigInv[i] = 1.0 / MdOrig[i];
    }
    applyBC_Step1_Md();
    for (size_t i = 0; i < (size_t)3 * NN; i++) MdInv[i] = 1.0 / Md[i];
    calculateZ();
  }

  // calculateZ, BCH.cpp:3322-3479 (+ applyBC_Step2(1), BCH.cpp:4171-4180):
  // Z = sum_d G_d^T diag(MdOrigInv) G_d, summed per component in ascending
  // velocity-row order (the column scatter of cs_multiply), then
  // Z = (Z1 + Z2) + Z3; Z[p][p] *= 1000 for p = zeroPressureNode > 0.
  void calculateZ() {
    // transpose pattern of G: for each pressure node p, the velocity rows v
    // (ascending) and the position of (v,p) in G.
    std::vector<int> tStart(NNp + 1, 0), tRow, tPos;
    long nnzG = GrowStarts[NN];
    for (long i = 0; i < nnzG; i++) tStart[Gcol[i] + 1]++;
    for (int p = 0; p < NNp; p++) tStart[p + 1] += tStart[p];
    tRow.resize(nnzG);
    tPos.resize(nnzG);
    {
      std::vector<int> fill(tStart.begin(), tStart.end() - 1);
      for (int v = 0; v < NN; v++)
        for (int i = GrowStarts[v]; i < GrowStarts[v + 1]; i++) {
          int p = Gcol[i];
          tRow[fill[p]] = v;
          tPos[fill[p]] = i;
          fill[p]++;
        }
    }
    // Z pattern: row p = union of G-row columns over v in column p of G.
    ZrowStarts.assign(NNp + 1, 0);
    std::vector<std::vector<int>> zc(NNp);
#pragma omp parallel
    {
      std::vector<char> mark(NNp, 0);
#pragma omp for schedule(static)
      for (int p = 0; p < NNp; p++) {
        auto& cols = zc[p];
        for (int t = tStart[p]; t < tStart[p + 1]; t++) {
          int v = tRow[t];
          for (int i = GrowStarts[v]; i < GrowStarts[v + 1]; i++) {
            int q = Gcol[i];
            if (!mark[q]) { mark[q] = 1; cols.push_back(q); }
          }
        }
        for (int q : cols) mark[q] = 0;
        std::sort(cols.begin(), cols.end());
      }
    }
    for (int p = 0; p < NNp; p++) ZrowStarts[p + 1] = ZrowStarts[p] + (int)zc[p].size();
    long nnzZ = ZrowStarts[NNp];
    Zcol.resize(nnzZ);
    Zval.assign(nnzZ, 0.0);
    for (int p = 0; p < NNp; p++) std::copy(zc[p].begin(), zc[p].end(), Zcol.begin() + ZrowStarts[p]);
    std::vector<std::vector<int>>().swap(zc);
    // Values.  Row r of the sorted CSR holds Z[r][c], which cs_multiply
    // forms in column c as  sum over v ascending of (G_d[v][c]*Minv[v]) *
    // G_d[v][r];  the v with both G[v][r] and G[v][c] nonzero are exactly
    // column r of G, taken here in ascending order.
#pragma omp parallel
    {
      std::vector<double> acc1(NNp, 0.0), acc2(NNp, 0.0), acc3(NNp, 0.0);
#pragma omp for schedule(dynamic, 64)
      for (int r = 0; r < NNp; r++) {
        for (int t = tStart[r]; t < tStart[r + 1]; t++) {
          int v = tRow[t], ir = tPos[t];
          double minv = MdOrigInv[v];
          double g1r = G1[ir], g2r = G2[ir], g3r = G3[ir];
          for (int i = GrowStarts[v]; i < GrowStarts[v + 1]; i++) {
            int c = Gcol[i];
            acc1[c] += (G1[i] * minv) * g1r;
            acc2[c] += (G2[i] * minv) * g2r;
            acc3[c] += (G3[i] * minv) * g3r;
          }
        }
        for (int j = ZrowStarts[r]; j < ZrowStarts[r + 1]; j++) {
          int c = Zcol[j];
          Zval[j] = (acc1[c] + acc2[c]) + acc3[c];
          acc1[c] = acc2[c] = acc3[c] = 0.0;
        }
      }
    }
    int node = zeroPressureNode;
    if (node > 0) {
      for (int j = ZrowStarts[node]; j < ZrowStarts[node + 1]; j++)
        if (Zcol[j] == node) { Zval[j] *= 1000.0; break; }
    }
    Zdiag.assign(NNp, 0.0);
    for (int p = 0; p < NNp; p++)
      for (int j = ZrowStarts[p]; j < ZrowStarts[p + 1]; j++)
        if (Zcol[j] == p) Zdiag[p] = Zval[j];
  }

  // applyBC_Step1(1), BCH.cpp:4129-4135
  void applyBC_Step1_Md() {
    for (int i = 0; i < BCnVelNodes; i++) {
      int node = BCvelNodes[2 * i];
      Md[node] = 1.0;
      Md[node + NN] = 1.0;
      Md[node + 2 * (size_t)NN] = 1.0;
    }
  }

  // y[r] (+)= alpha * sum_j A[r][j] x[j], mkl_dcsrmv with transa='n'.
  static void csrmv(int m, const int* rs, const int* col, const double* val, const double* x,
                    double alpha, double beta, double* y) {
#pragma omp parallel for schedule(static)
    for (int r = 0; r < m; r++) {
      double s = 0;
      for (int j = rs[r]; j < rs[r + 1]; j++) s += val[j] * x[col[j]];
      y[r] = (beta == 0.0 ? 0.0 : beta * y[r]) + alpha * s;
    }
  }

  // calculateMatrixA, BCH.cpp:3520-3685: R11..R13 = -sum_e Ae(Un)*UnpHalf_prev
  // with Ae[i][j] = sum_k (u0_k . gDSv[k][j]) Sv[k][i] detJ w.  Element vectors
  // are computed in parallel and scattered in colour order (the order in
  // which the reference's coloured loop accumulates).
  void calculateMatrixA(std::vector<double>& R) {
    std::fill(R.begin(), R.end(), 0.0);
    const int B = 8192;
    std::vector<double> Re((size_t)B * 81);
    for (int o0 = 0; o0 < NE; o0 += B) {
      int o1 = std::min(NE, o0 + B);
#pragma omp parallel for schedule(static)
      for (int o = o0; o < o1; o++) {
        int e = elementsOfColor[o];
        double u0n[27], v0n[27], w0n[27], up[27], vp[27], wp[27];
        double Ae[27][27];
        for (int i = 0; i < 27; i++) {
          int g = L(e, i);
          u0n[i] = Un[g];
          up[i] = UnpHalf_prev[g];
          v0n[i] = Un[g + NN];
          vp[i] = UnpHalf_prev[g + NN];
          w0n[i] = Un[g + 2 * (size_t)NN];
          wp[i] = UnpHalf_prev[g + 2 * (size_t)NN];
        }
        for (int i = 0; i < 27; i++)
          for (int j = 0; j < 27; j++) Ae[i][j] = 0.0;
        for (int k = 0; k < NGP; k++) {
          double GQfactor = detJacob[(size_t)e * NGP + k] * GQweight[k];
          const double* sv = &Sv[(size_t)k * 27];
          double u0 = 0, v0 = 0, w0 = 0;
          for (int i = 0; i < 27; i++) {
            u0 = u0 + sv[i] * u0n[i];
            v0 = v0 + sv[i] * v0n[i];
            w0 = w0 + sv[i] * w0n[i];
          }
          const double* gd = &gDSv[(((size_t)e * NGP + k) * NENv) * 3];
          for (int i = 0; i < 27; i++)
            for (int j = 0; j < 27; j++)
              Ae[i][j] = Ae[i][j] + (u0 * gd[3 * j] + v0 * gd[3 * j + 1] + w0 * gd[3 * j + 2]) * sv[i] * GQfactor;
        }
        double* re = &Re[(size_t)(o - o0) * 81];
        for (int i = 0; i < 27; i++) {
          double a = 0, b = 0, c = 0;
          for (int j = 0; j < 27; j++) {
            a += Ae[i][j] * up[j];
            b += Ae[i][j] * vp[j];
            c += Ae[i][j] * wp[j];
          }
          re[i] = a;
          re[27 + i] = b;
          re[54 + i] = c;
        }
      }
      for (int o = o0; o < o1; o++) {
        int e = elementsOfColor[o];
        const double* re = &Re[(size_t)(o - o0) * 81];
        for (int i = 0; i < 27; i++) {
          int g = L(e, i);
          R[g] -= re[i];
          R[g + NN] -= re[27 + i];
          R[g + 2 * (size_t)NN] -= re[54 + i];
        }
      }
    }
  }

  // step1, BCH.cpp:3692-3801
  void step1(int /*iter*/) {
    calculateMatrixA(R1);
    int m = NN;
    for (int d = 0; d < 3; d++)
      csrmv(m, MrowStarts.data(), Mcol.data(), Kval.data(), &UnpHalf_prev[(size_t)d * NN], -1.0, 1.0,
            &R1[(size_t)d * NN]);
    const std::vector<double>* Gd[3] = {&G1, &G2, &G3};
    for (int d = 0; d < 3; d++)
      csrmv(m, GrowStarts.data(), Gcol.data(), Gd[d]->data(), Pn.data(), -1.0, 1.0, &R1[(size_t)d * NN]);
    for (int i = 0; i < BCnVelNodes; i++) {  // applyBC_Step1(2), BCH.cpp:4137-4146
      int node = BCvelNodes[2 * i];
      R1[node] = 0.0;
      R1[node + NN] = 0.0;
      R1[node + 2 * (size_t)NN] = 0.0;
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < 3L * NN; i++) UnpHalf[i] = Un[i] + dt * R1[i] * MdInv[i];
  }

  // step2, BCH.cpp:3808-3905: R2 = G^T (UnpHalf/dt^2 - [iter>1] MdOrigInv K Acc_prev)
  void step2(int iter) {
    std::vector<double> dummy((size_t)3 * NN);
    double oneOverdt2 = 1.0000000000000000 / (dt * dt);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < 3L * NN; i++) {
      double v = oneOverdt2 * UnpHalf[i];
      if (iter != 1) v = v - MdOrigInv[i] * KtimesAcc_prev[i];
      dummy[i] = v;
    }
    // G^T x as three transposed products accumulated in order d = 1, 2, 3.
    std::fill(R2.begin(), R2.end(), 0.0);
    const std::vector<double>* Gd[3] = {&G1, &G2, &G3};
    for (int d = 0; d < 3; d++) {
      std::vector<double> t(NNp, 0.0);
      const double* x = &dummy[(size_t)d * NN];
      const double* g = Gd[d]->data();
      for (int v = 0; v < NN; v++)
        for (int i = GrowStarts[v]; i < GrowStarts[v + 1]; i++) t[Gcol[i]] += g[i] * x[v];
      for (int p = 0; p < NNp; p++) R2[p] += t[p];
    }
    if (zeroPressureNode > 0) R2[zeroPressureNode] = 0.0;  // applyBC_Step2(2)
    cg_solve(R2.data(), Pdot.data());
    for (int i = 0; i < NNp; i++) Pnp1[i] = Pn[i] + dt * Pdot[i];
  }

  // Jacobi-PCG on Z (stands in for MKL dcg with ipar[10]=1, BCH.cpp:3981-4055,
  // and cusp::krylov::cg with precond::diagonal, CU.cu:418-451).
  CgStats cg_solve(const double* b, double* x) {
    CgStats st;
    int n = NNp;
    std::vector<double> r(n), z(n), p(n), q(n);
    if (!cg_warm) std::fill(x, x + n, 0.0);
    const int* rs = ZrowStarts.data();
    const int* col = Zcol.data();
    const double* val = Zval.data();
    csrmv(n, rs, col, val, x, 1.0, 0.0, q.data());
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      r[i] = b[i] - q[i];
      z[i] = r[i] / Zdiag[i];
      p[i] = z[i];
    }
    double bnorm = std::sqrt(det_sum(n, [&](long i) { return b[i] * b[i]; }));
    double rz = det_sum(n, [&](long i) { return r[i] * z[i]; });
    double rn = std::sqrt(det_sum(n, [&](long i) { return r[i] * r[i]; }));
    if (!std::isfinite(bnorm) || !std::isfinite(rn)) {
      st.status = 2;
      last_cg = st;
      return st;
    }
    if (bnorm == 0.0) {
      std::fill(x, x + n, 0.0);
      st.relres = 0;
      last_cg = st;
      cg_log.push_back(0);
      return st;
    }
    double tol = cg_rtol * bnorm;
    int it = 0;
    st.status = 1;
    if (rn <= tol) st.status = 0;
    while (st.status != 0 && it < cg_maxit) {
      csrmv(n, rs, col, val, p.data(), 1.0, 0.0, q.data());
      double pq = det_sum(n, [&](long i) { return p[i] * q[i]; });
      double a = rz / pq;
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) {
        x[i] += a * p[i];
        r[i] -= a * q[i];
        z[i] = r[i] / Zdiag[i];
      }
      it++;
      double rr = det_sum(n, [&](long i) { return r[i] * r[i]; });
      double rzn = det_sum(n, [&](long i) { return r[i] * z[i]; });
      rn = std::sqrt(rr);
      if (!std::isfinite(rn)) { st.status = 2; break; }
      if (rn <= tol) { st.status = 0; break; }
      double beta = rzn / rz;
      rz = rzn;
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    }
    st.its = it;
    st.relres = rn / bnorm;
    last_cg = st;
    cg_total_its += it;
    cg_log.push_back(it);
    return st;
  }

  // step3, BCH.cpp:3912-3974
  void step3(int iter) {
    const std::vector<double>* Gd[3] = {&G1, &G2, &G3};
    for (int d = 0; d < 3; d++)
      csrmv(NN, GrowStarts.data(), Gcol.data(), Gd[d]->data(), Pdot.data(), -dt, 0.0, &R3[(size_t)d * NN]);
    if (iter != 1) {
#pragma omp parallel for schedule(static)
      for (long i = 0; i < 3L * NN; i++) R3[i] = R3[i] - dt * KtimesAcc_prev[i];
    }
    for (int i = 0; i < BCnVelNodes; i++) {  // applyBC_Step3, BCH.cpp:4192-4207
      int node = BCvelNodes[2 * i];
      R3[node] = 0.0;
      R3[node + NN] = 0.0;
      R3[node + 2 * (size_t)NN] = 0.0;
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < 3L * NN; i++) {
      Acc[i] = R3[i] * MdInv[i];
      Unp1[i] = UnpHalf[i] + dt * Acc[i];
    }
  }

  // Sub-iteration convergence test, BCH.cpp:2936-2961.
  bool checkIter() {
    long n3 = 3L * NN;
    double s1 = det_sum(n3, [&](long i) { return Unp1[i] * Unp1[i]; });
    double s2 = det_sum(n3, [&](long i) { double d = Unp1[i] - Unp1_prev[i]; return d * d; });
    double norm1 = std::sqrt(s2) / std::sqrt(s1);
    s1 = det_sum(NNp, [&](long i) { return Pnp1[i] * Pnp1[i]; });
    s2 = det_sum(NNp, [&](long i) { double d = Pnp1[i] - Pnp1_prev[i]; return d * d; });
    double norm2 = std::sqrt(s2) / std::sqrt(s1);
    lastNorm1 = norm1;
    lastNorm2 = norm2;
    return norm1 < tolerance && norm2 < tolerance;
  }

  // Rotation + KtimesAcc_prev = K * Acc_prev, BCH.cpp:2964-3033.
  void rotateAndKAcc() {
    UnpHalf_prev = UnpHalf;
    Unp1_prev = Unp1;
    Acc_prev = Acc;
    Pnp1_prev = Pnp1;
    for (int d = 0; d < 3; d++)
      csrmv(NN, MrowStarts.data(), Mcol.data(), Kval.data(), &Acc_prev[(size_t)d * NN], 1.0, 0.0,
            &KtimesAcc_prev[(size_t)d * NN]);
  }

  // Start of a time step, BCH.cpp:2860-2881 (Unp1_prev is NOT reset, as in
  // the C++ code; BCH.cpp:2874 is commented out).
  void beginStep() {
    timeN = timeN + 1;
    timeT = timeT + dt;
    UnpHalf_prev = Un;
    std::fill(Acc_prev.begin(), Acc_prev.end(), 0.0);
    Pnp1_prev = Pn;
  }

  // Steady-state test and Un <- Unp1, Pn <- Pnp1, BCH.cpp:3048-3081.
  // maxAcc = max |Unp1 - Un| / dt (CPU semantics; the GPU build omits /dt).
  bool endStep() {
    double oneOverdt = 1.0000000000000000 / dt;
    double m = 0.0;
    for (long i = 0; i < 3L * NN; i++) {
      double a = std::fabs((Unp1[i] - Un[i]) * oneOverdt);
      if (a > m) m = a;
    }
    maxAcc = m;
    bool steady = !(maxAcc > convergenceCriteria);
    Un = Unp1;
    Pn = Pnp1;
    return steady;
  }

  // One full time step of timeLoop, BCH.cpp:2859-3094.  Returns 1 when the
  // steady-state test fired.
  int timeStep() {
    beginStep();
    int iter;
    for (iter = 1; iter <= maxIter; iter++) {
      step1(iter);
      step2(iter);
      step3(iter);
      if (checkIter()) break;
      rotateAndKAcc();
    }
    last_iters = iter;
    bool steady = endStep();
    const double row[8] = {(double)timeN, (double)iter, timeT, Un[monPoint], Un[NN + monPoint],
                           Un[2 * (size_t)NN + monPoint], Pn[monPoint], maxAcc};
    mon_log.insert(mon_log.end(), row, row + 8);
    if (print_monitor)
      printf("%6d  %6d  %10.5f  %12.5f  %12.5f  %12.5f  %12.5f %12.5f %12.5f\n", timeN, iter, timeT,
             Un[monPoint], Un[NN + monPoint], Un[2 * (size_t)NN + monPoint], Pn[monPoint], 0.0, maxAcc);
    return steady ? 1 : 0;
  }

  // createTecplot, BCH.cpp:4249-4482: 8 sub-bricks per hex27; mid-node
  // pressures averaged from corners in element order.
  int createTecplot(const std::string& path, const std::string& title) {
    std::ofstream out(path.c_str());
    if (!out) return -1;
    out << "TITLE = " << title << std::endl;
    out << "VARIABLES = x,  y,  z,  u, v, w, p" << std::endl;
    out << "ZONE N=" << NN << ", E=" << 8 * NE << ", F=FEPOINT, ET=BRICK" << std::endl;
    std::vector<double> pNode(NN, 0.0);
    for (int i = 0; i < NNp; i++) pNode[i] = Pn[i];
    for (int e = 0; e < NE; e++) {
      for (int ed = 0; ed < NEE; ed++)
        pNode[L(e, ed + NEC)] = 0.5 * (pNode[L(e, kEdge[ed][0])] + pNode[L(e, kEdge[ed][1])]);
      for (int f = 0; f < NEF; f++)
        pNode[L(e, f + NEC + NEE)] = 0.25 * (pNode[L(e, kFace[f][0])] + pNode[L(e, kFace[f][1])] +
                                             pNode[L(e, kFace[f][2])] + pNode[L(e, kFace[f][3])]);
      pNode[L(e, 26)] = 0.125 * (pNode[L(e, 0)] + pNode[L(e, 1)] + pNode[L(e, 2)] + pNode[L(e, 3)] +
                                 pNode[L(e, 4)] + pNode[L(e, 5)] + pNode[L(e, 6)] + pNode[L(e, 7)]);
    }
    for (int i = 0; i < NN; i++) {
      out.precision(11);
      out << std::scientific << coord[3 * (size_t)i] << " " << coord[3 * (size_t)i + 1] << " "
          << coord[3 * (size_t)i + 2] << " " << Un[i] << " " << Un[i + NN] << " " << Un[i + 2 * (size_t)NN]
          << " " << pNode[i] << std::endl;
    }
    static const int sub[8][8] = {{0, 8, 20, 11, 12, 21, 26, 24},  {8, 1, 9, 20, 21, 13, 22, 26},
                                  {11, 20, 10, 3, 24, 26, 23, 15}, {20, 9, 2, 10, 26, 22, 14, 23},
                                  {12, 21, 26, 24, 4, 16, 25, 19}, {21, 13, 22, 26, 16, 5, 17, 25},
                                  {24, 26, 23, 15, 19, 25, 18, 7}, {26, 22, 14, 23, 25, 17, 6, 18}};
    for (int e = 0; e < NE; e++)
      for (int s = 0; s < 8; s++) {
        for (int j = 0; j < 8; j++) {
          out << L(e, sub[s][j]) + 1;
          out << (j < 7 ? " " : "");
        }
        out << std::endl;
      }
    return 0;
  }

  // readRestartFile, BCH.cpp:4214-4242 (three header lines; pressure from the
  // first NCN rows only).
  int readRestartFile(const std::string& path) {
    std::ifstream in(path.c_str());
    if (!in) return -1;
    double d1, d2, d3, d4;
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    in.ignore(256, '\n');
    for (int i = 0; i < NCN; i++) {
      in >> d1 >> d2 >> d3 >> Un[i] >> Un[NN + i] >> Un[2 * (size_t)NN + i] >> Pn[i];
      in.ignore(256, '\n');
    }
    for (int i = NCN; i < NN; i++) {
      in >> d1 >> d2 >> d3 >> Un[i] >> Un[NN + i] >> Un[2 * (size_t)NN + i] >> d4;
      in.ignore(256, '\n');
    }
    return in.fail() ? -2 : 0;
  }

  // main() order of the preprocessing stages, BCH.cpp:412-506.
  int setup(const std::string& path, int ngp_override) {
    int rc = readInputFile(path);
    if (rc) return rc;
    if (ngp_override > 0) NGP = ngp_override;
    findElemsOfPresNodes();
    findElemNeighbors();
    setupMeshColoring();
    setupNonCornerNodes();
    determineVelBCnodes();
    findElemsOfVelNodes();
    findMonitorPoint();
    setupSparseM();
    setupSparseG();
    if (setupGQ()) return -4;
    calcShape();
    calcJacob();
    initializeAndAllocate();
    return 0;
  }
};

constexpr int Oracle::kEdge[12][2];
constexpr int Oracle::kFace[6][4];
constexpr int Oracle::kFaceMid[6][5];
constexpr int Oracle::kNode27[27][3];

}  // namespace

// ============================================================================
//  C interface used by the tests and by the CPU-baseline timer.
// ============================================================================
extern "C" {

void* orc_create(const char* inp_path, int ngp_override, int nthreads, int* rc) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  Oracle* o = new Oracle();
  int r = o->setup(inp_path, ngp_override);
  if (rc) *rc = r;
  if (r) {
    delete o;
    return nullptr;
  }
  return o;
}

void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }

int orc_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// sizes: NE NCN NN NNp nnzK nnzG nnzZ BCnVelNodes monPoint zeroPressureNode NGP maxIter nActiveColors
void orc_sizes(void* h, long* out) {
  Oracle* o = static_cast<Oracle*>(h);
  out[0] = o->NE; out[1] = o->NCN; out[2] = o->NN; out[3] = o->NNp;
  out[4] = o->MrowStarts.empty() ? 0 : o->MrowStarts[o->NN];
  out[5] = o->GrowStarts.empty() ? 0 : o->GrowStarts[o->NN];
  out[6] = o->ZrowStarts.empty() ? 0 : o->ZrowStarts[o->NNp];
  out[7] = o->BCnVelNodes; out[8] = o->monPoint; out[9] = o->zeroPressureNode;
  out[10] = o->NGP; out[11] = o->maxIter; out[12] = o->nActiveColors;
}

// params: dt t_ini t_final tolerance converge density viscosity
void orc_params(void* h, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  out[0] = o->dt; out[1] = o->t_ini; out[2] = o->t_final; out[3] = o->tolerance;
  out[4] = o->convergenceCriteria; out[5] = o->density; out[6] = o->viscosity;
}

void orc_set_cg(void* h, double rtol, int maxit, int warm) {
  Oracle* o = static_cast<Oracle*>(h);
  o->cg_rtol = rtol;
  o->cg_maxit = maxit;
  o->cg_warm = warm;
}

void orc_set_print(void* h, int on) { static_cast<Oracle*>(h)->print_monitor = on; }
void orc_set_maxiter(void* h, int m) { static_cast<Oracle*>(h)->maxIter = m; }

void orc_get_ltog(void* h, int* out) {
  Oracle* o = static_cast<Oracle*>(h);
  std::copy(o->LtoGnode.begin(), o->LtoGnode.end(), out);
}
void orc_get_coord(void* h, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  std::copy(o->coord.begin(), o->coord.end(), out);
}
void orc_get_bcnodes(void* h, int* out) {
  Oracle* o = static_cast<Oracle*>(h);
  std::copy(o->BCvelNodes.begin(), o->BCvelNodes.end(), out);
}
void orc_get_colors(void* h, int* out) {
  Oracle* o = static_cast<Oracle*>(h);
  std::copy(o->meshColors.begin(), o->meshColors.end(), out);
}
void orc_get_basis(void* h, double* gqp, double* gqw, double* sv, double* dsv, double* sp, double* dsp) {
  Oracle* o = static_cast<Oracle*>(h);
  std::copy(o->GQpoint.begin(), o->GQpoint.end(), gqp);
  std::copy(o->GQweight.begin(), o->GQweight.end(), gqw);
  std::copy(o->Sv.begin(), o->Sv.end(), sv);
  std::copy(o->dSv.begin(), o->dSv.end(), dsv);
  std::copy(o->Sp.begin(), o->Sp.end(), sp);
  std::copy(o->dSp.begin(), o->dSp.end(), dsp);
}
void orc_get_detj(void* h, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  std::copy(o->detJacob.begin(), o->detJacob.end(), out);
}
void orc_get_slotmaps(void* h, int* mapM, int* mapG) {
  Oracle* o = static_cast<Oracle*>(h);
  if (mapM) std::copy(o->sparseMapM.begin(), o->sparseMapM.end(), mapM);
  if (mapG) std::copy(o->sparseMapG.begin(), o->sparseMapG.end(), mapG);
}

void orc_step0(void* h) { static_cast<Oracle*>(h)->step0(); }

// which: 0 = K pattern (rowStarts NN+1, col nnzK); 1 = G pattern; 2 = Z pattern
void orc_get_pattern(void* h, int which, int* rowstarts, int* col) {
  Oracle* o = static_cast<Oracle*>(h);
  const std::vector<int>& rs = which == 0 ? o->MrowStarts : which == 1 ? o->GrowStarts : o->ZrowStarts;
  const std::vector<int>& c = which == 0 ? o->Mcol : which == 1 ? o->Gcol : o->Zcol;
  std::copy(rs.begin(), rs.end(), rowstarts);
  std::copy(c.begin(), c.end(), col);
}
// which: 0 K, 1 G1, 2 G2, 3 G3, 4 Z
void orc_get_values(void* h, int which, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  const std::vector<double>* v[5] = {&o->Kval, &o->G1, &o->G2, &o->G3, &o->Zval};
  std::copy(v[which]->begin(), v[which]->end(), out);
}

static std::vector<double>* vec_by_id(Oracle* o, int id) {
  switch (id) {
    case 0: return &o->Un;
    case 1: return &o->Unp1;
    case 2: return &o->Unp1_prev;
    case 3: return &o->UnpHalf;
    case 4: return &o->UnpHalf_prev;
    case 5: return &o->Acc;
    case 6: return &o->Acc_prev;
    case 7: return &o->Pn;
    case 8: return &o->Pnp1;
    case 9: return &o->Pnp1_prev;
    case 10: return &o->Pdot;
    case 11: return &o->Md;
    case 12: return &o->MdOrig;
    case 13: return &o->MdInv;
    case 14: return &o->MdOrigInv;
    case 15: return &o->KtimesAcc_prev;
    case 16: return &o->R1;
    case 17: return &o->R2;
    case 18: return &o->R3;
  }
  return nullptr;
}
long orc_get_vec(void* h, int id, double* out) {
  std::vector<double>* v = vec_by_id(static_cast<Oracle*>(h), id);
  if (!v) return -1;
  if (out) std::copy(v->begin(), v->end(), out);
  return (long)v->size();
}
long orc_set_vec(void* h, int id, const double* in) {
  std::vector<double>* v = vec_by_id(static_cast<Oracle*>(h), id);
  if (!v) return -1;
  std::copy(in, in + v->size(), v->begin());
  return (long)v->size();
}

// Stage-level entry points mirroring the timeLoop call sequence.
void orc_begin_step(void* h) { static_cast<Oracle*>(h)->beginStep(); }
void orc_convect(void* h, double* R) {
  Oracle* o = static_cast<Oracle*>(h);
  std::vector<double> tmp((size_t)3 * o->NN);
  o->calculateMatrixA(tmp);
  std::copy(tmp.begin(), tmp.end(), R);
}
void orc_step1(void* h, int iter) { static_cast<Oracle*>(h)->step1(iter); }
void orc_step2(void* h, int iter, double* cgstats) {
  Oracle* o = static_cast<Oracle*>(h);
  o->step2(iter);
  if (cgstats) {
    cgstats[0] = o->last_cg.its;
    cgstats[1] = o->last_cg.relres;
    cgstats[2] = o->last_cg.status;
  }
}
void orc_step3(void* h, int iter) { static_cast<Oracle*>(h)->step3(iter); }
int orc_check_iter(void* h, double* norms) {
  Oracle* o = static_cast<Oracle*>(h);
  int c = o->checkIter() ? 1 : 0;
  if (norms) { norms[0] = o->lastNorm1; norms[1] = o->lastNorm2; }
  return c;
}
void orc_rotate(void* h) { static_cast<Oracle*>(h)->rotateAndKAcc(); }
int orc_end_step(void* h, double* maxAcc) {
  Oracle* o = static_cast<Oracle*>(h);
  int s = o->endStep() ? 1 : 0;
  if (maxAcc) *maxAcc = o->maxAcc;
  return s;
}

// Standalone CG on the oracle's Z: x (in: initial guess when warm) -> solution.
void orc_cg(void* h, const double* b, double* x, double* stats) {
  Oracle* o = static_cast<Oracle*>(h);
  CgStats st = o->cg_solve(b, x);
  if (stats) { stats[0] = st.its; stats[1] = st.relres; stats[2] = st.status; }
}

// Runs nsteps time steps (nsteps < 0: the reference's while (timeT < t_final)
// loop).  info: steps run, total CG iterations, total sub-iterations, steady flag,
// last maxAcc.
int orc_run(void* h, int nsteps, double* info) {
  Oracle* o = static_cast<Oracle*>(h);
  int steps = 0, steady = 0;
  long subits = 0;
  o->cg_total_its = 0;
  while (nsteps < 0 ? (o->timeT < o->t_final) : (steps < nsteps)) {
    steady = o->timeStep();
    steps++;
    subits += std::min(o->last_iters, o->maxIter);
    if (steady) break;
  }
  if (info) {
    info[0] = steps; info[1] = (double)o->cg_total_its; info[2] = (double)subits;
    info[3] = steady; info[4] = o->maxAcc;
  }
  return steps;
}

// Sizes of the run logs (out[0] pressure solves, out[1] time steps) and,
// when the arrays are non-NULL, their contents; clear != 0 empties them.
void orc_logs(void* h, long* sizes, int* cg, double* mon, int clear) {
  Oracle* o = static_cast<Oracle*>(h);
  if (sizes) { sizes[0] = (long)o->cg_log.size(); sizes[1] = (long)(o->mon_log.size() / 8); }
  if (cg) std::copy(o->cg_log.begin(), o->cg_log.end(), cg);
  if (mon) std::copy(o->mon_log.begin(), o->mon_log.end(), mon);
  if (clear) { o->cg_log.clear(); o->mon_log.clear(); }
}

int orc_time(void* h, int* timeN, double* timeT) {
  Oracle* o = static_cast<Oracle*>(h);
  if (timeN) *timeN = o->timeN;
  if (timeT) *timeT = o->timeT;
  return 0;
}

int orc_write_tecplot(void* h, const char* path, const char* title) {
  return static_cast<Oracle*>(h)->createTecplot(path, title);
}
int orc_read_restart(void* h, const char* path) { return static_cast<Oracle*>(h)->readRestartFile(path); }

}  // extern "C"
