// Host-only part of the C ABI: deck reading and mesh preprocessing without
// a device (cfdh_*), used to inspect numbering and patterns.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/cfdfs.h"
#include "coarse.h"
#include "problem.h"

namespace cfd {
int write_tecplot(const HostProblem& P, const double* U, const double* Pn, const std::string& path,
                  const std::string& title);
}

struct cfd_host {
  cfd::HostProblem P;
};

extern "C" {

int cfdh_load(cfd_host** out, const char* path, char* errbuf, int errlen) {
  if (!out || !path) return CFD_E_BADARG;
  *out = nullptr;
  cfd_host* h = new cfd_host();
  std::string err;
  int rc = cfd::read_inp(path, h->P, err);
  if (!rc) rc = cfd::preprocess(h->P, err);
  if (rc) {
    if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", err.c_str());
    delete h;
    return rc;
  }
  *out = h;
  return CFD_OK;
}

void cfdh_free(cfd_host* h) { delete h; }

int cfdh_sizes(const cfd_host* h, long long* o) {
  if (!h || !o) return CFD_E_BADARG;
  const cfd::HostProblem& P = h->P;
  o[0] = P.NE; o[1] = P.NCN; o[2] = P.NN; o[3] = P.NNp;
  o[4] = (long long)P.k_col.size(); o[5] = (long long)P.g_col.size(); o[6] = (long long)P.z_col.size();
  o[7] = (long long)P.bcnode.size(); o[8] = P.monPoint; o[9] = P.zeroP; o[10] = P.NGP; o[11] = P.maxIter;
  return CFD_OK;
}

int cfdh_get_ltog(const cfd_host* h, int* out) {
  if (!h || !out) return CFD_E_BADARG;
  std::copy(h->P.ltog.begin(), h->P.ltog.end(), out);
  return CFD_OK;
}

int cfdh_get_coord(const cfd_host* h, double* out) {
  if (!h || !out) return CFD_E_BADARG;
  std::copy(h->P.coord.begin(), h->P.coord.end(), out);
  return CFD_OK;
}

int cfdh_get_bcnodes(const cfd_host* h, int* out) {
  if (!h || !out) return CFD_E_BADARG;
  for (size_t i = 0; i < h->P.bcnode.size(); i++) {
    out[2 * i] = h->P.bcnode[i];
    out[2 * i + 1] = h->P.bcid[i];
  }
  return CFD_OK;
}

int cfdh_get_pattern(const cfd_host* h, int which, int* rowptr, int* col) {
  if (!h) return CFD_E_BADARG;
  const cfd::HostProblem& P = h->P;
  const std::vector<int>* rp[4] = {&P.k_rp, &P.g_rp, &P.gt_rp, &P.z_rp};
  const std::vector<int>* cl[4] = {&P.k_col, &P.g_col, &P.gt_col, &P.z_col};
  if (which < 0 || which > 3) return CFD_E_BADARG;
  if (rowptr) std::copy(rp[which]->begin(), rp[which]->end(), rowptr);
  if (col) std::copy(cl[which]->begin(), cl[which]->end(), col);
  return CFD_OK;
}

int cfdh_element_colors(const cfd_host* h, int* order, int* off) {
  if (!h) return CFD_E_BADARG;
  std::vector<int> o, f;
  if (cfd::color_elements(h->P, o, f)) return -1;
  if (order) std::copy(o.begin(), o.end(), order);
  if (off) std::copy(f.begin(), f.end(), off);
  return (int)f.size() - 1;
}

int cfdh_write_tecplot(const cfd_host* h, const double* U, const double* Pv, const char* path, const char* title) {
  if (!h || !U || !Pv || !path) return CFD_E_BADARG;
  return cfd::write_tecplot(h->P, U, Pv, path, title ? title : "");
}

int cfdh_coarse_inverse(const int dims[3], const int* rowptr, const int* col, const double* val, int* cd,
                        double* inv) {
  if (!dims || !rowptr || !col || !val || !cd) return CFD_E_BADARG;
  const long long n = (long long)dims[0] * dims[1] * dims[2];
  if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || n > (1LL << 30)) return CFD_E_BADARG;
  const int kMaxNodes = 6000;
  if (!inv) {
    double h[3];
    cfd::coarse_lattice(dims, kMaxNodes, cd, h);
    return CFD_OK;
  }
  std::vector<int> rp(rowptr, rowptr + n + 1);
  std::vector<int> cl(col, col + rp[n]);
  std::vector<double> vl(val, val + rp[n]);
  cfd::CoarseSpace cs;
  std::string err;
  if (cfd::coarse_build(dims, kMaxNodes, std::vector<int>(), rp, cl, vl, cs, err)) return CFD_E_NONFINITE;
  for (int a = 0; a < 3; a++) cd[a] = cs.cd[a];
  std::copy(cs.inv.begin(), cs.inv.end(), inv);
  return CFD_OK;
}

int cfdh_coarse_matrix(const int dims[3], const int* rowptr, const int* col, const double* val, double spacing,
                       int* cd, double* zc) {
  if (!dims || !rowptr || !col || !val || !cd) return CFD_E_BADARG;
  const long long n = (long long)dims[0] * dims[1] * dims[2];
  if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || n > (1LL << 30)) return CFD_E_BADARG;
  const int kMaxNodes = 6000;
  if (!zc) {
    double h[3];
    cfd::coarse_lattice(dims, kMaxNodes, cd, h, spacing);
    return CFD_OK;
  }
  std::vector<int> rp(rowptr, rowptr + n + 1);
  std::vector<int> cl(col, col + rp[n]);
  std::vector<double> vl(val, val + rp[n]);
  cfd::CoarseSpace cs;
  std::string err;
  if (cfd::coarse_build(dims, kMaxNodes, std::vector<int>(), rp, cl, vl, cs, err, false, false, spacing))
    return CFD_E_NONFINITE;
  for (int a = 0; a < 3; a++) cd[a] = cs.cd[a];
  std::copy(cs.inv.begin(), cs.inv.end(), zc);
  return CFD_OK;
}

}  // extern "C"
