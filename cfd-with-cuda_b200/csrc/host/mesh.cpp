// Deck reader and mesh preprocessing on the host (C++, OpenMP).
//
// Reference behaviour followed:
//   readInputFile        blascoCodinaHuerta.cpp:528-725
//   setupNonCornerNodes  blascoCodinaHuerta.cpp:954-1320
//   determineVelBCnodes  blascoCodinaHuerta.cpp:1410-1580
//   findMonitorPoint     blascoCodinaHuerta.cpp:1644-1668
//   setupSparseM / G     blascoCodinaHuerta.cpp:1675-2159
//
// The reference finds shared mid-edge / mid-face nodes by comparing
// coordinates against the neighbours' mid-nodes.  On a conforming mesh two
// elements share a mid-edge (mid-face) node exactly when they share the
// edge's two (the face's four) corner nodes, so the same numbering -- new
// nodes in order of first appearance in the element-then-edge (face) loop --
// is produced here by sorting topological keys, in O(NE log NE).  The
// element->slot maps of the reference (sparseMapM/G) are not built: device
// kernels find CSR slots by binary search in the sorted rows.
#include <algorithm>
#include <charconv>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <utility>

#include "../../../include/cfdfs.h"
#include "problem.h"

namespace cfd {

const int kEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 5},
                          {2, 6}, {3, 7}, {4, 5}, {5, 6}, {6, 7}, {7, 4}};
const int kFace[6][4] = {{0, 1, 2, 3}, {0, 1, 4, 5}, {1, 2, 5, 6},
                         {2, 3, 6, 7}, {0, 3, 4, 7}, {4, 5, 6, 7}};
const int kFaceMid[6][5] = {{8, 9, 10, 11, 20},  {8, 12, 13, 16, 21},  {9, 13, 14, 17, 22},
                            {10, 14, 15, 18, 23}, {11, 12, 15, 19, 24}, {16, 17, 18, 19, 25}};
// (xi, eta, zeta) position (0: -1, 1: 0, 2: +1) of each local hex27 node.
const int kNode27[27][3] = {{0, 0, 0}, {2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {0, 0, 2}, {2, 0, 2}, {2, 2, 2},
                            {0, 2, 2}, {1, 0, 0}, {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 1},
                            {2, 2, 1}, {0, 2, 1}, {1, 0, 2}, {2, 1, 2}, {1, 2, 2}, {0, 1, 2}, {1, 1, 0},
                            {1, 0, 1}, {2, 1, 1}, {1, 2, 1}, {0, 1, 1}, {1, 1, 2}, {1, 1, 1}};
// Eight linear sub-bricks of a hex27 element used by the Tecplot writer
// (blascoCodinaHuerta.cpp:4453-4470).
const int kSubBrick[8][8] = {{0, 8, 20, 11, 12, 21, 26, 24},  {8, 1, 9, 20, 21, 13, 22, 26},
                             {11, 20, 10, 3, 24, 26, 23, 15}, {20, 9, 2, 10, 26, 22, 14, 23},
                             {12, 21, 26, 24, 4, 16, 25, 19}, {21, 13, 22, 26, 16, 5, 17, 25},
                             {24, 26, 23, 15, 19, 25, 18, 7}, {26, 22, 14, 23, 25, 17, 6, 18}};

namespace {

// Token scanner reproducing the std::istream operations the reference uses:
// ignore(256, delim), >> int, >> double, >> std::string.  A failed
// extraction sets the fail flag and every later extraction fails too.
class Scanner {
 public:
  explicit Scanner(std::string text) : s_(std::move(text)), i_(0), fail_(false) {}
  void ignore(int n, char delim) {
    for (int k = 0; k < n && i_ < s_.size(); k++)
      if (s_[i_++] == delim) return;
  }
  void skip_ws() {
    while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r' ||
                              s_[i_] == '\v' || s_[i_] == '\f'))
      i_++;
  }
  // The numbers are read by std::from_chars (correctly rounded, as glibc's
  // strtod), which is several times faster on a 64^3 deck; it accepts no
  // leading '+' and no hexadecimal form, so those, and values out of range,
  // go to strtol / strtod as before.
  bool get(int& v) {
    if (fail_) return false;
    skip_ws();
    const char* b = s_.c_str() + i_;
    const char* end = s_.c_str() + s_.size();
    long x = 0;
    const auto r = std::from_chars(b, end, x, 10);
    if (r.ec == std::errc() && r.ptr != b) {
      i_ += (size_t)(r.ptr - b);
      v = (int)x;
      return true;
    }
    char* e = nullptr;
    x = std::strtol(b, &e, 10);
    if (e == b) { fail_ = true; return false; }
    i_ += (size_t)(e - b);
    v = (int)x;
    return true;
  }
  bool get(double& v) {
    if (fail_) return false;
    skip_ws();
    const char* b = s_.c_str() + i_;
    const char* end = s_.c_str() + s_.size();
    double x = 0.0;
    const auto r = std::from_chars(b, end, x, std::chars_format::general);
    // "0x..." parses as 0 here and as a hexadecimal value in strtod
    const bool hex = r.ptr < end && (*r.ptr == 'x' || *r.ptr == 'X');
    if (r.ec == std::errc() && r.ptr != b && !hex) {
      i_ += (size_t)(r.ptr - b);
      v = x;
      return true;
    }
    char* e = nullptr;
    x = std::strtod(b, &e);
    if (e == b) { fail_ = true; return false; }
    i_ += (size_t)(e - b);
    v = x;
    return true;
  }
  bool word() {
    if (fail_) return false;
    skip_ws();
    size_t b = i_;
    while (i_ < s_.size() && !std::isspace((unsigned char)s_[i_])) i_++;
    if (i_ == b) { fail_ = true; return false; }
    return true;
  }
  bool failed() const { return fail_; }

 private:
  std::string s_;
  size_t i_;
  bool fail_;
};

}  // namespace

int read_inp(const std::string& path, HostProblem& P, std::string& err) {
  std::ifstream f(path.c_str(), std::ios::binary);
  if (!f) {
    err = "cannot open deck " + path;
    return CFD_E_IO;
  }
  std::string text;
  f.seekg(0, std::ios::end);
  const std::streamoff size = f.tellg();
  f.seekg(0, std::ios::beg);
  if (size < 0) {
    err = "cannot read deck " + path;
    return CFD_E_IO;
  }
  text.resize((size_t)size);
  if (size > 0 && !f.read(&text[0], size)) {
    err = "cannot read deck " + path;
    return CFD_E_IO;
  }
  Scanner in(std::move(text));
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  auto hdr = [&](auto& v) {
    in.ignore(256, ':');
    in.get(v);
    in.ignore(256, '\n');
  };
  hdr(P.eType); hdr(P.NE); hdr(P.NCN); hdr(P.NENv); hdr(P.NENp); hdr(P.NGP);
  hdr(P.alpha); hdr(P.dt); hdr(P.t_ini); hdr(P.t_final); hdr(P.maxIter);
  hdr(P.tolerance); hdr(P.convergence); hdr(P.isRestart);
  hdr(P.density); hdr(P.viscosity); hdr(P.fx); hdr(P.fy);
  if (in.failed()) {
    err = "malformed header";
    return CFD_E_BADINPUT;
  }
  if (P.eType != 1 || P.NENv != 27 || P.NENp != 8) {
    err = "only hexahedral hex27/hex8 decks (eType 1, NENv 27, NENp 8) are supported";
    return CFD_E_BADINPUT;
  }
  if (P.NE <= 0 || P.NCN <= 0 || (long)P.NE * 27 > 2000000000L) {
    err = "bad NE/NCN";
    return CFD_E_BADINPUT;
  }
  if (P.NGP != 1 && P.NGP != 8 && P.NGP != 27) {
    err = "NGP must be 1, 8 or 27";
    return CFD_E_BADINPUT;
  }
  if (!(P.dt > 0) || P.maxIter < 1) {
    err = "dt must be > 0 and maxIter >= 1";
    return CFD_E_BADINPUT;
  }
  P.coord.assign((size_t)P.NCN * 3, 0.0);
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  for (int i = 0; i < P.NCN; i++) {
    int id;
    in.get(id);
    in.get(P.coord[3 * (size_t)i]);
    in.get(P.coord[3 * (size_t)i + 1]);
    in.get(P.coord[3 * (size_t)i + 2]);
    in.ignore(256, '\n');
  }
  P.ltog.assign((size_t)P.NE * 27, -1);
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  for (int e = 0; e < P.NE; e++) {
    int id;
    in.get(id);
    for (int i = 0; i < 8; i++) {
      int v = 0;
      in.get(v);
      P.ltog[(size_t)e * 27 + i] = v - 1;
    }
    in.ignore(256, '\n');
  }
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  in.ignore(256, ':');
  in.get(P.nBC);
  in.ignore(256, '\n');
  if (in.failed() || P.nBC < 0 || P.nBC > 1000000) {
    err = "malformed node/element/BC section";
    return CFD_E_BADINPUT;
  }
  P.bcstr.assign((size_t)P.nBC * 3, 0.0);
  for (int i = 0; i < P.nBC; i++) {
    double type;
    in.ignore(256, ':');
    in.get(type);
    in.get(P.bcstr[3 * (size_t)i]);
    in.word();
    in.get(P.bcstr[3 * (size_t)i + 1]);
    in.word();
    in.get(P.bcstr[3 * (size_t)i + 2]);
    in.ignore(256, '\n');
  }
  int nVel = 0, nOut = 0;
  in.ignore(256, '\n');
  in.ignore(256, ':');
  in.get(nVel);
  in.ignore(256, '\n');
  in.ignore(256, ':');
  in.get(nOut);
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  if (in.failed() || nVel < 0 || nOut < 0) {
    err = "malformed face counts";
    return CFD_E_BADINPUT;
  }
  P.velfaces.assign((size_t)nVel * 3, 0);
  for (int i = 0; i < nVel; i++) {
    for (int j = 0; j < 3; j++) {
      in.get(P.velfaces[3 * (size_t)i + j]);
      P.velfaces[3 * (size_t)i + j] -= 1;
    }
    in.ignore(256, '\n');
  }
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  P.outfaces.assign((size_t)nOut * 3, 0);
  for (int i = 0; i < nOut; i++) {
    for (int j = 0; j < 3; j++) {
      in.get(P.outfaces[3 * (size_t)i + j]);
      P.outfaces[3 * (size_t)i + j] -= 1;
    }
    in.ignore(256, '\n');
  }
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  in.get(P.zeroP);
  P.zeroP -= 1;
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  in.ignore(256, '\n');
  in.get(P.mon[0]);
  in.get(P.mon[1]);
  in.get(P.mon[2]);
  if (in.failed()) {
    err = "deck ended early or holds a malformed value";
    return CFD_E_BADINPUT;
  }
  for (int e = 0; e < P.NE; e++)
    for (int i = 0; i < 8; i++) {
      int v = P.ltog[(size_t)e * 27 + i];
      if (v < 0 || v >= P.NCN) {
        err = "element corner out of range";
        return CFD_E_BADINPUT;
      }
    }
  for (int i = 0; i < nVel; i++) {
    int e = P.velfaces[3 * (size_t)i], f = P.velfaces[3 * (size_t)i + 1], b = P.velfaces[3 * (size_t)i + 2];
    if (e < 0 || e >= P.NE || f < 0 || f > 5 || b < 0 || b >= P.nBC) {
      err = "velocity BC face out of range";
      return CFD_E_BADINPUT;
    }
  }
  if (P.zeroP >= P.NCN) {
    err = "zero-pressure node out of range";
    return CFD_E_BADINPUT;
  }
  P.NNp = P.NCN;  // blascoCodinaHuerta.cpp:718-723 (NENp = 8)
  return CFD_OK;
}

namespace {

struct Key2 {
  uint64_t a, b;
  bool operator<(const Key2& o) const { return a < o.a || (a == o.a && b < o.b); }
  bool operator==(const Key2& o) const { return a == o.a && b == o.b; }
};

// Numbers the distinct keys in order of first appearance (appearance index =
// position in keys[]) starting at base; out[i] = number of keys[i].  Every
// key starts with its smallest corner id (the high word of a), which buckets
// it: a CSR over the ncorner corner nodes, sized by counting, holds the keys
// met so far per corner, and one pass in index order looks each key up among
// its corner's few distinct keys (an edge or face of a hex mesh has at most
// a dozen per corner), numbering it when it is new.
inline uint32_t first_corner(uint64_t k) { return (uint32_t)(k >> 32); }
inline uint32_t first_corner(const Key2& k) { return (uint32_t)(k.a >> 32); }
template <class K>
int number_by_first_appearance(const std::vector<K>& keys, int ncorner, int base, std::vector<int>& out) {
  const size_t n = keys.size();
  std::vector<int> off((size_t)ncorner + 1, 0);
  for (size_t i = 0; i < n; i++) off[first_corner(keys[i]) + 1]++;
  for (int c = 0; c < ncorner; c++) off[c + 1] += off[c];
  std::vector<K> bkey(n);
  std::vector<int> bnum(n), fill((size_t)ncorner, 0);
  out.resize(n);
  int count = 0;
  for (size_t i = 0; i < n; i++) {
    const K& k = keys[i];
    const uint32_t c = first_corner(k);
    const int s = off[c], f = fill[c];
    int t = 0;
    while (t < f && !(bkey[s + t] == k)) t++;
    if (t == f) {
      bkey[s + f] = k;
      bnum[s + f] = base + count++;
      fill[c] = f + 1;
    }
    out[i] = bnum[s + t];
  }
  return count;
}

// Row r: the distinct nodes j in [first, first + count) of the elements
// around r (in incidence order), written to out when it is not null;
// returns how many.  stamp (ncols entries) must not hold r on entry.
inline int gather_row(int r, const std::vector<int>& inc_rp, const std::vector<int>& inc_el, const std::vector<int>& ltog,
                      int first, int count, std::vector<int>& stamp, int* out) {
  int k = 0;
  for (int t = inc_rp[r]; t < inc_rp[r + 1]; t++) {
    const int* L = &ltog[(size_t)inc_el[t] * 27];
    for (int j = first; j < first + count; j++) {
      const int v = L[j];
      if (stamp[v] != r) {
        stamp[v] = r;
        if (out) out[k] = v;
        k++;
      }
    }
  }
  return k;
}

// CSR of the union, per row, of the node sets of the elements around it:
// one pass counts the row lengths, a second fills the rows in place and
// sorts them.
void build_pattern(int nrows, const std::vector<int>& inc_rp, const std::vector<int>& inc_el,
                   const std::vector<int>& ltog, int first, int count, int ncols, std::vector<int>& rp,
                   std::vector<int>& col, int& maxrow) {
  std::vector<int> len(nrows, 0);
#pragma omp parallel
  {
    std::vector<int> stamp(ncols, -1);
#pragma omp for schedule(dynamic, 1024)
    for (int r = 0; r < nrows; r++) len[r] = gather_row(r, inc_rp, inc_el, ltog, first, count, stamp, nullptr);
  }
  rp.assign(nrows + 1, 0);
  maxrow = 0;
  for (int r = 0; r < nrows; r++) {
    rp[r + 1] = rp[r] + len[r];
    maxrow = std::max(maxrow, len[r]);
  }
  col.resize(rp[nrows]);
#pragma omp parallel
  {
    std::vector<int> stamp(ncols, -1);
#pragma omp for schedule(dynamic, 1024)
    for (int r = 0; r < nrows; r++) {
      int* c = col.data() + rp[r];
      gather_row(r, inc_rp, inc_el, ltog, first, count, stamp, c);
      std::sort(c, c + len[r]);
    }
  }
}

}  // namespace

int preprocess(HostProblem& P, std::string& err, bool patterns) {
  const int NE = P.NE, NCN = P.NCN;
  // ---- mid-edge nodes (first appearance in element-then-edge order) ----
  std::vector<uint64_t> ekeys((size_t)NE * 12);
  for (int e = 0; e < NE; e++)
    for (int ed = 0; ed < 12; ed++) {
      uint32_t a = P.ltog[(size_t)e * 27 + kEdge[ed][0]], b = P.ltog[(size_t)e * 27 + kEdge[ed][1]];
      if (a > b) std::swap(a, b);
      ekeys[(size_t)e * 12 + ed] = ((uint64_t)a << 32) | b;
    }
  std::vector<int> enum_;
  int nEdge = number_by_first_appearance(ekeys, NCN, NCN, enum_);
  std::vector<uint64_t>().swap(ekeys);
  // ---- mid-face nodes ----
  std::vector<Key2> fkeys((size_t)NE * 6);
  for (int e = 0; e < NE; e++)
    for (int f = 0; f < 6; f++) {
      uint32_t c[4];
      for (int j = 0; j < 4; j++) c[j] = P.ltog[(size_t)e * 27 + kFace[f][j]];
      std::sort(c, c + 4);
      fkeys[(size_t)e * 6 + f] = Key2{((uint64_t)c[0] << 32) | c[1], ((uint64_t)c[2] << 32) | c[3]};
    }
  std::vector<int> fnum;
  int nFace = number_by_first_appearance(fkeys, NCN, NCN + nEdge, fnum);
  std::vector<Key2>().swap(fkeys);
  P.NN = NCN + nEdge + nFace + NE;
  std::vector<double> coord((size_t)P.NN * 3, 0.0);
  std::copy(P.coord.begin(), P.coord.begin() + (size_t)NCN * 3, coord.begin());
  std::vector<char> made((size_t)P.NN, 0);
  for (int e = 0; e < NE; e++) {
    int* L = &P.ltog[(size_t)e * 27];
    for (int ed = 0; ed < 12; ed++) {
      int n = enum_[(size_t)e * 12 + ed];
      L[8 + ed] = n;
      if (!made[n]) {  // coordinates from the creating element, as the reference
        made[n] = 1;
        int n1 = L[kEdge[ed][0]], n2 = L[kEdge[ed][1]];
        for (int d = 0; d < 3; d++) coord[3 * (size_t)n + d] = 0.5 * (coord[3 * (size_t)n1 + d] + coord[3 * (size_t)n2 + d]);
      }
    }
  }
  for (int e = 0; e < NE; e++) {
    int* L = &P.ltog[(size_t)e * 27];
    for (int f = 0; f < 6; f++) {
      int n = fnum[(size_t)e * 6 + f];
      L[20 + f] = n;
      if (!made[n]) {
        made[n] = 1;
        const int* c = kFace[f];
        for (int d = 0; d < 3; d++)
          coord[3 * (size_t)n + d] = 0.25 * (coord[3 * (size_t)L[c[0]] + d] + coord[3 * (size_t)L[c[1]] + d] +
                                             coord[3 * (size_t)L[c[2]] + d] + coord[3 * (size_t)L[c[3]] + d]);
      }
    }
  }
  for (int e = 0; e < NE; e++) {
    int* L = &P.ltog[(size_t)e * 27];
    int n = NCN + nEdge + nFace + e;
    L[26] = n;
    for (int d = 0; d < 3; d++) {
      double s = coord[3 * (size_t)L[0] + d];
      for (int j = 1; j < 8; j++) s = s + coord[3 * (size_t)L[j] + d];
      coord[3 * (size_t)n + d] = 0.125 * s;
    }
  }
  P.coord.swap(coord);
  // ---- velocity-BC nodes: later faces overwrite earlier ----
  {
    std::vector<int> info(P.NN, -1);
    size_t nv = P.velfaces.size() / 3;
    for (size_t i = 0; i < nv; i++) {
      int e = P.velfaces[3 * i], f = P.velfaces[3 * i + 1], b = P.velfaces[3 * i + 2];
      const int* L = &P.ltog[(size_t)e * 27];
      for (int j = 0; j < 4; j++) info[L[kFace[f][j]]] = b;
      for (int j = 0; j < 5; j++) info[L[kFaceMid[f][j]]] = b;
    }
    P.bcnode.clear();
    P.bcid.clear();
    for (int i = 0; i < P.NN; i++)
      if (info[i] != -1) {
        P.bcnode.push_back(i);
        P.bcid.push_back(info[i]);
      }
  }
  // ---- monitor node (first minimum over corner nodes) ----
  {
    double best = 1e6;
    P.monPoint = 0;
    for (int i = 0; i < NCN; i++) {
      double dx = P.coord[3 * (size_t)i] - P.mon[0], dy = P.coord[3 * (size_t)i + 1] - P.mon[1],
             dz = P.coord[3 * (size_t)i + 2] - P.mon[2];
      double d = std::sqrt(dx * dx + dy * dy + dz * dz);
      if (d < best) {
        best = d;
        P.monPoint = i;
      }
    }
  }
  return patterns ? build_patterns(P, err) : CFD_OK;
}

int build_patterns(HostProblem& P, std::string& err) {
  const int NE = P.NE;
  // ---- node -> element incidence ----
  std::vector<int> inc_rp(P.NN + 1, 0), inc_el((size_t)NE * 27);
  for (size_t t = 0; t < P.ltog.size(); t++) inc_rp[P.ltog[t] + 1]++;
  for (int i = 0; i < P.NN; i++) inc_rp[i + 1] += inc_rp[i];
  {
    std::vector<int> fill(inc_rp.begin(), inc_rp.end() - 1);
    for (int e = 0; e < NE; e++)
      for (int j = 0; j < 27; j++) inc_el[fill[P.ltog[(size_t)e * 27 + j]]++] = e;
  }
  // ---- patterns ----
  build_pattern(P.NN, inc_rp, inc_el, P.ltog, 0, 27, P.NN, P.k_rp, P.k_col, P.maxKrow);
  build_pattern(P.NN, inc_rp, inc_el, P.ltog, 0, 8, P.NNp, P.g_rp, P.g_col, P.maxGrow);
  // G^T (rows p, columns v ascending): (v, p) is in G exactly when v and the
  // corner node p share an element, so row p is the union of the 27 nodes
  // of the elements around p (pressure nodes are the corner nodes 0..NCN-1);
  // gt_pos = index of (v, p) in the sorted G row v
  build_pattern(P.NNp, inc_rp, inc_el, P.ltog, 0, 27, P.NN, P.gt_rp, P.gt_col, P.maxGtrow);
  if (P.gt_col.size() != P.g_col.size()) {
    err = "inconsistent G and G^T patterns";
    return CFD_E_BADINPUT;
  }
  P.gt_pos.resize(P.gt_col.size());
#pragma omp parallel for schedule(dynamic, 1024)
  for (int p = 0; p < P.NNp; p++)
    for (int t = P.gt_rp[p]; t < P.gt_rp[p + 1]; t++) {
      const int v = P.gt_col[t];
      const int* b = P.g_col.data() + P.g_rp[v];
      const int* e = P.g_col.data() + P.g_rp[v + 1];
      P.gt_pos[t] = (int)(std::lower_bound(b, e, p) - P.g_col.data());
    }
  // Z pattern: row p = union of G-row columns over the velocity nodes in
  // G^T row p (counted, then filled in place and sorted)
  {
    auto zrow = [&](int p, std::vector<int>& stamp, int* out) {
      int k = 0;
      for (int t = P.gt_rp[p]; t < P.gt_rp[p + 1]; t++) {
        const int v = P.gt_col[t];
        for (int i = P.g_rp[v]; i < P.g_rp[v + 1]; i++) {
          const int q = P.g_col[i];
          if (stamp[q] != p) {
            stamp[q] = p;
            if (out) out[k] = q;
            k++;
          }
        }
      }
      return k;
    };
    std::vector<int> len(P.NNp, 0);
#pragma omp parallel
    {
      std::vector<int> stamp(P.NNp, -1);
#pragma omp for schedule(dynamic, 256)
      for (int p = 0; p < P.NNp; p++) len[p] = zrow(p, stamp, nullptr);
    }
    P.z_rp.assign(P.NNp + 1, 0);
    P.maxZrow = 0;
    for (int p = 0; p < P.NNp; p++) {
      P.z_rp[p + 1] = P.z_rp[p] + len[p];
      P.maxZrow = std::max(P.maxZrow, len[p]);
    }
    P.z_col.resize(P.z_rp[P.NNp]);
#pragma omp parallel
    {
      std::vector<int> stamp(P.NNp, -1);
#pragma omp for schedule(dynamic, 256)
      for (int p = 0; p < P.NNp; p++) {
        int* c = P.z_col.data() + P.z_rp[p];
        zrow(p, stamp, c);
        std::sort(c, c + len[p]);
      }
    }
  }
  if ((long long)P.k_rp[P.NN] >= (1LL << 31) - 1) {
    err = "K has more than 2^31 non-zeros";
    return CFD_E_BADINPUT;
  }
  P.nnzK = (long long)P.k_col.size();
  P.nnzG = (long long)P.g_col.size();
  P.nnzZ = (long long)P.z_col.size();
  return CFD_OK;
}

int color_elements(const HostProblem& P, std::vector<int>& order, std::vector<int>& off) {
  const int NE = P.NE;
  std::vector<uint64_t> used((size_t)P.NCN, 0);  // colours of the elements touching each corner node
  std::vector<int> color(NE);
  int ncol = 0;
  for (int e = 0; e < NE; e++) {
    uint64_t m = 0;
    for (int c = 0; c < 8; c++) m |= used[P.ltog[(size_t)e * 27 + c]];
    if (~m == 0) return -1;
    int k = 0;
    while (m & (1ull << k)) k++;
    color[e] = k;
    ncol = std::max(ncol, k + 1);
    for (int c = 0; c < 8; c++) used[P.ltog[(size_t)e * 27 + c]] |= 1ull << k;
  }
  off.assign(ncol + 1, 0);
  for (int e = 0; e < NE; e++) off[color[e] + 1]++;
  for (int c = 0; c < ncol; c++) off[c + 1] += off[c];
  order.assign(NE, 0);
  std::vector<int> pos(off.begin(), off.end() - 1);
  for (int e = 0; e < NE; e++) order[pos[color[e]]++] = e;
  return 0;
}

}  // namespace cfd
