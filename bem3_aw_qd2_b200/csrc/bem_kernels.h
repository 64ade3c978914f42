// Device-side views and launcher prototypes shared by the .cu files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "bem_types.h"

// One domain's element list and the element tables it indexes (device pointers).
struct bem_dom_dev {
  int ne;                       // elements bordering the domain
  const int *sid;               // signed element ids (1-based, sign = orientation)
  const double *cr, *cw, *ren;  // element tables, see bem_types.h
  const double *wen;            // normal vectors at the collocation nodes (field rule 0)
  const uint8_t *plane;         // 1 if the element is plane (bil_check_plane)
  const int *npe;               // nodes per element: 4 bilinear quad, 3 linear triangle
  int has_tri;                  // any triangle among the domain's elements
  int far_rule;                 // periodic domain: shorter rules for regular pairs far from every lattice image (k_q0_far)
  int near_cap;                 // near-singular sources one collocation node can hold (<= 256):
                                // the stride of bem_scratch.near_s / nearF
};

// Scratch used by one domain assembly (sized for N = 4 ne rows).
struct bem_scratch {
  double *rowF;     // [N][3] geometric F, dF/dtz, dF/dte summed over regular sources
  int *near_s;      // [N][near_cap] near-singular source indices, sorted
  int *near_n;      // [N]
  double *nearF;    // [N][near_cap][3]
  double *selfF;    // [N][3]
  uint8_t *flag;    // [N][ne] 0 regular, 1 near-singular, 2 self, 3 + t regular on shorter-rule tier t
  unsigned *plist;  // [pcap] periodic-domain pair lists p * ne + s: regular, then tier 0, 1, ... (optional)
  unsigned *pcount; // [16] list lengths, then the fill counters
  unsigned long long pcap;
  unsigned *status; // BEM_ST_* bits
  unsigned long long *terms;  // [6] lattice terms of regular / near / self pairs, then point counts
};

extern "C" {
// the periodic domain of nb problems that differ only in the Bloch wave
// vector, each kernel launched once for all (bem_assemble.cu)
int bem_launch_assemble_batch(const bem_dom_dev *D, const bem_qp *q, int nb, const bem_qp *qps, double *const *Gh,
                              double *const *Hh, bem_scratch *S, double *dF, cudaStream_t st);
int bem_set_constants(const double *xl, const double *wl, const double *xh, const double *wh);
int bem_launch_faddeeva(const double *z, int n, double *w, cudaStream_t st);
// table of w(x + i y), y in [0, 8), for the Ewald real-space terms (bem_qp.wt)
// the real-space term table of the problem with wave number k and Ewald parameter ve
int bem_launch_wtab(double k, double ve, double *out, cudaStream_t st);
// the evanescent spectral order table of q (window and interval count set in q,
// out: st_n1cnt x st_n2cnt x st_nint x BEM_ST_DEG (P, M) pairs)
int bem_launch_stab(const bem_qp *q, double *out, cudaStream_t st);
int bem_launch_qpgf(const bem_qp *q, const double *r, int n, double *G, double *dG, int *ret, cudaStream_t st);
int bem_launch_field(const bem_dom_dev *D, const bem_qp *q, int periodic, int grad, double k, int type, int npts,
                     const double *pts, const double *P, const double *dP, const double *pv, const double *dpv,
                     double *out, unsigned *status, cudaStream_t st);
int bem_launch_bdval(const bem_dom_dev *D, const bem_qp *q, int periodic, double k, int type, int ntgt, const int *tgt_t,
                     const double *tgt_ze,
                     const double *P, const double *dP, const double *pv, const double *dpv, double *out,
                     unsigned *status, cudaStream_t st);
int bem_launch_force_bd(const bem_dom_dev *D, int ntgt, const int *tgt_t, const double *tgt_ze, const double *wts,
                        const double *bdv, const double *pw, double k2r, double k2i, const double *rc, double c0,
                        double rho0, double *out, cudaStream_t st);
int bem_launch_classify(const bem_dom_dev *D, const bem_qp *q, int periodic, bem_scratch *S, cudaStream_t st);
// free-space derivative rows dG, dH of rows p0 .. p0 + np - 1 only (row 2 (p - p0))
int bem_launch_fs_deriv(const bem_dom_dev *D, double k, bem_scratch *S, int p0, int np, double *dG, double *dH,
                        cudaStream_t st);
int bem_time_regular(const bem_dom_dev *D, const bem_qp *q, bem_scratch *S, double *G, double *H, double frac,
                     int nchunk, cudaStream_t st, float *ms);
int bem_launch_assemble(const bem_dom_dev *D, const bem_qp *q, int periodic, int exterior, double k, bem_scratch *S,
                        double *G, double *H, double *dG, double *dH, double *dF, cudaStream_t st, cudaEvent_t *ev);
}

// host-side copies of the table sizes
#define BEM_GLN_H 12
#define BEM_GHN_H 64
#define BEM_MAXNEAR_H 256      // near-singular table of a context (bodies a millimetre apart need ~90)
#define BEM_MAXNEAR_STATIC 64  // near-singular table of the allocation-free entry point
