// Tecplot output and restart input in the reference's text layout
// (createTecplot, blascoCodinaHuerta.cpp:4249-4482; readRestartFile,
// blascoCodinaHuerta.cpp:4214-4242).
//
// Output: "TITLE = <title>", the variable line, "ZONE N=<NN>, E=<8NE>,
// F=FEPOINT, ET=BRICK", NN rows "x y z u v w p" in %.11e, then 8 linear
// sub-bricks per hex27 element (1-based).  Pressure at mid-edge, mid-face
// and centre nodes is the average of the element's corner values, written
// in element order so a node shared by several elements keeps the value of
// the last one, as in the reference.
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "../../../include/cfdfs.h"
#include "problem.h"

namespace cfd {

int write_tecplot(const HostProblem& P, const double* U, const double* Pn, const std::string& path,
                  const std::string& title) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return CFD_E_IO;
  std::vector<char> buf(1 << 22);
  std::setvbuf(f, buf.data(), _IOFBF, buf.size());
  const int NN = P.NN, NE = P.NE;
  std::fprintf(f, "TITLE = %s\n", title.c_str());
  std::fprintf(f, "VARIABLES = x,  y,  z,  u, v, w, p\n");
  std::fprintf(f, "ZONE N=%d, E=%d, F=FEPOINT, ET=BRICK\n", NN, 8 * NE);
  std::vector<double> p(NN, 0.0);
  for (int i = 0; i < P.NNp; i++) p[i] = Pn[i];
  for (int e = 0; e < NE; e++) {
    const int* L = &P.ltog[(size_t)e * 27];
    for (int ed = 0; ed < 12; ed++) p[L[8 + ed]] = 0.5 * (p[L[kEdge[ed][0]]] + p[L[kEdge[ed][1]]]);
    for (int fc = 0; fc < 6; fc++)
      p[L[20 + fc]] = 0.25 * (p[L[kFace[fc][0]]] + p[L[kFace[fc][1]]] + p[L[kFace[fc][2]]] + p[L[kFace[fc][3]]]);
    p[L[26]] = 0.125 * (p[L[0]] + p[L[1]] + p[L[2]] + p[L[3]] + p[L[4]] + p[L[5]] + p[L[6]] + p[L[7]]);
  }
  for (int i = 0; i < NN; i++)
    std::fprintf(f, "%.11e %.11e %.11e %.11e %.11e %.11e %.11e\n", P.coord[3 * (size_t)i], P.coord[3 * (size_t)i + 1],
                 P.coord[3 * (size_t)i + 2], U[i], U[(size_t)NN + i], U[2 * (size_t)NN + i], p[i]);
  for (int e = 0; e < NE; e++) {
    const int* L = &P.ltog[(size_t)e * 27];
    for (int s = 0; s < 8; s++)
      std::fprintf(f, "%d %d %d %d %d %d %d %d\n", L[kSubBrick[s][0]] + 1, L[kSubBrick[s][1]] + 1,
                   L[kSubBrick[s][2]] + 1, L[kSubBrick[s][3]] + 1, L[kSubBrick[s][4]] + 1, L[kSubBrick[s][5]] + 1,
                   L[kSubBrick[s][6]] + 1, L[kSubBrick[s][7]] + 1);
  }
  int rc = std::ferror(f) ? CFD_E_IO : CFD_OK;
  std::fclose(f);
  return rc;
}

int read_restart(const HostProblem& P, const std::string& path, double* U, double* Pn) {
  std::ifstream in(path.c_str());
  if (!in) return CFD_E_IO;
  const int NN = P.NN;
  double d1, d2, d3, d4;
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  for (int i = 0; i < P.NCN; i++) {
    in >> d1 >> d2 >> d3 >> U[i] >> U[(size_t)NN + i] >> U[2 * (size_t)NN + i] >> Pn[i];
    in.ignore(256, '\n');
  }
  for (int i = P.NCN; i < NN; i++) {
    in >> d1 >> d2 >> d3 >> U[i] >> U[(size_t)NN + i] >> U[2 * (size_t)NN + i] >> d4;
    in.ignore(256, '\n');
  }
  return in.fail() ? CFD_E_BADINPUT : CFD_OK;
}

}  // namespace cfd
