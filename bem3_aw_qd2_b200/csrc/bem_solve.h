// Device view of the whole boundary-value problem, used by bem_solve.cu.
#pragma once
#include <cuda_runtime.h>

struct bem_sys_dev {
  int n;                  // global unknowns 2 NN
  int NN;                 // element nodes
  int MN;                 // media
  const int *dom_ne;      // [MN+1] elements per domain (device)
  const int *dom_off;     // [MN+1] offset of each domain in sid (device)
  int dom_ne_h[8];        // host copies for launch sizes (MN+1 <= 8)
  const int *sid;         // concatenated signed element ids
  const int *rowidx;      // [4 * sum(dom_ne)] global row of (domain, element, node), -1 if absent
  const int *npe;         // [Ne] nodes per element (3 or 4)
  const int *eni;         // [Ne][4] element node ids
  const int *md;          // [Ne] main domain
  const double *hk2;      // [Ne] complex k2(main)/k2(sub)
  const double *Pi, *dPi; // [Ne][4] complex incident potential and its normal derivative
  const double *p_inc;    // [Ne][4] complex incident pressure at the element nodes
  const double *v_inc;    // [Ne][4][3] complex incident particle velocity
  const double *cr, *ren, *wen;
  const double *rho0;     // [MN+1] (device)
  const double *k2;       // [MN+1] complex (device)
  double zt44[4], et44[4];
};

extern "C" {
// A == NULL: the right-hand side b only
int bem_launch_gather(const bem_sys_dev *S, int d, const double *G, const double *H, double *A, double *b, cudaStream_t st);
int bem_launch_store(const bem_sys_dev *S, int d, const double *X, double *P, double *dP, cudaStream_t st);
int bem_launch_pv(const bem_sys_dev *S, int d, const double *dG, const double *dH, const double *dF, const double *P,
                  const double *dP, double *pv, double *tpv, cudaStream_t st);
// interior domain d, rows p0 .. p0 + np - 1, with dG, dH holding only those rows
int bem_launch_pv_rows(const bem_sys_dev *S, int d, const double *dG, const double *dH, const double *dF,
                       const double *P, const double *dP, double *pv, double *tpv, int p0, int np, cudaStream_t st);
int bem_launch_dpv_rhs(int Nd, const double *H, const double *pv, double *B, cudaStream_t st);
int bem_launch_dpv_store(int Nd, const double *B, double *dpv, cudaStream_t st);
// domains with triangles: dpv system without the padding rows / columns
int bem_launch_compress(const double *G, int N, const int *inv, int nn, double *Gc, cudaStream_t st);
int bem_launch_rows(const double *src, double *dst, int N, const int *inv, int nn, int nrhs, int to_full, cudaStream_t st);
// ctr / cbd / pw: triangle centres (see k_force0); NULL when domain 0 has no triangles
int bem_launch_force0(const bem_sys_dev *S, const double *P0, const double *pv0, const double *rc, double c0, double rho0,
                      const int *ctr, const double *cbd, const double *pw, double *out, cudaStream_t st);
}
