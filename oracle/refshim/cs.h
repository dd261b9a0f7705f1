/* Stand-in for Timothy Davis' CSparse header cs.h (test infrastructure
 * only), for the calls of the reference's Z build
 * (blascoCodinaHuerta.cpp:3349-3477).  The reference assigns int arrays to
 * the i and p members (blascoCodinaHuerta.cpp:3350-3351), which fixes the
 * index type to int, as in CSparse 2.x.
 * A cs is a triplet matrix when nz >= 0 (p holds column indices, nz
 * entries) and a compressed-column matrix when nz == -1 (p holds n+1
 * column pointers). */
#ifndef REFSHIM_CS_H
#define REFSHIM_CS_H
#ifdef __cplusplus
extern "C" {
#endif
typedef int csi;
typedef struct cs_sparse {
  int nzmax;  /* capacity of i and x */
  int m;      /* rows */
  int n;      /* columns */
  int* p;     /* column pointers (n+1) or column indices (triplet) */
  int* i;     /* row indices */
  double* x;  /* values, or NULL for a pattern */
  int nz;     /* entries of a triplet matrix, -1 when compressed */
} cs;
cs* cs_spalloc(int m, int n, int nzmax, int values, int triplet);
cs* cs_spfree(cs* A);
cs* cs_compress(const cs* T);
cs* cs_transpose(const cs* A, int values);
cs* cs_multiply(const cs* A, const cs* B);
int cs_print(const cs* A, int brief);
#ifdef __cplusplus
}
#endif
#endif
