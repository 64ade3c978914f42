// C ABI (include/bemgpu.h): device buffers, problem upload, the assembly /
// solve sequence and the dense factorisations (bem_lu.cu, bem_mixed.cu).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <thread>
#include <unordered_map>
#include <vector>
#include "../../include/bemgpu.h"
#include "bem_kernels.h"
#include "bem_solve.h"
#include "bem_lattice.h"
#include "bem_mixed.h"
#include "bem_lu.h"
#include "bem_count.h"
#include <atomic>

#define BEMGPU_MAXDOM 8

struct bemgpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  char err[512] = {0};
  // problem
  bool loaded = false;
  // bytes allocated behind each device-pointer field that a problem load sizes:
  // a new load reuses an allocation that is large enough instead of freeing
  // and allocating again (cudaFree waits for the device)
  std::unordered_map<const void *, size_t> cap;
  int Ne = 0, NN = 0, MN = 0, n = 0;
  bem_qp qp;
  std::vector<int> dom_ne, dom_off, dom_tri;
  std::vector<double> k0, c0, rho0, k2;
  // device problem data
  double *cr = nullptr, *cw = nullptr, *ren = nullptr, *wen = nullptr;
  uint8_t *plane = nullptr;
  int *sid = nullptr, *rowidx = nullptr, *npe = nullptr, *eni = nullptr, *md = nullptr, *dom_ne_d = nullptr, *dom_off_d = nullptr;
  double *hk2 = nullptr, *Pi = nullptr, *dPi = nullptr, *p_inc = nullptr, *v_inc = nullptr, *rho0_d = nullptr, *k2_d = nullptr;
  // per-domain matrices and boundary values
  double *G[BEMGPU_MAXDOM] = {}, *H[BEMGPU_MAXDOM] = {}, *dG[BEMGPU_MAXDOM] = {}, *dH[BEMGPU_MAXDOM] = {}, *dF[BEMGPU_MAXDOM] = {};
  double *P[BEMGPU_MAXDOM] = {}, *dP[BEMGPU_MAXDOM] = {}, *pv[BEMGPU_MAXDOM] = {}, *dpv[BEMGPU_MAXDOM] = {};
  bem_scratch scr = {};   // periodic domain (context stream)
  bem_scratch scr1 = {};  // domains 1.. (side stream, beside the periodic domain)
  // solve work
  double *A = nullptr, *b = nullptr, *tpv = nullptr, *B3 = nullptr;
  double *fout = nullptr, *rc_d = nullptr;
  double *wtab = nullptr;  // real-space term table of the Ewald sums (A, B at eta_run)
  double *stab = nullptr;  // evanescent spectral order table (at eta_run)
  double zspan = 0.0;      // height of the mesh (z extent of all elements)
  double pw[16] = {};      // incident plane wave (bemgpu_problem.pw)
  int far_rule = 1;        // shorter rules for regular pairs of the periodic domain (bemgpu_set_far_rule)
  double eta_scale = 0.0;  // Ewald parameter off the lattice plane = eta0 x eta_scale; 0: by rule per problem
  double *pw_d = nullptr;
  // 9-point targets on the domain-0 elements for the type-1 force
  int ntgt = 0;
  int *tgt_t = nullptr;
  double *tgt_ze = nullptr, *tgt_w = nullptr, *bdv = nullptr;
  // centres of the domain-0 triangles for the 4-point force rule
  int nctr = 0;
  int *ctr_t = nullptr, *ctr_idx = nullptr;
  double *ctr_ze = nullptr, *ctr_bdv = nullptr;
  // staging buffers of the point evaluators (grown on demand, kept until destroy)
  size_t pt_cap = 0;
  double *pt_in = nullptr, *pt_out = nullptr;
  int *pt_t = nullptr;
  unsigned *status = nullptr;
  unsigned long long *terms = nullptr;
  bem_sys_dev sys;
  // optional per-phase timing: 6 events per domain (0, 1), then 5 for the solve
  bool prof = false;
  cudaEvent_t ev[17] = {};
  // precision of the dense solves: 0 FP64 LU; BEM_MIXED_* complex FP32 LU + FP64 refinement
  int precision = 0;
  bem_mixed mxs[BEMGPU_MAXDOM + 1];  // FP32 factors per dense system (0 global, 1 + d dpv of domain d)
  int refine = 0;  // refinement of the mixed solves: 0 IR then GMRES-IR, 1 IR only, 2 GMRES-IR only
  bool mx_ready[BEMGPU_MAXDOM + 1] = {};
  // FP64 factors: the global system in A, domain d's dpv system in Wd[d]; the
  // row pivoting and the scratch of each in lus[slot] (0 global, 1 + d dpv)
  double *Wd[BEMGPU_MAXDOM] = {};
  bem_lu lus[BEMGPU_MAXDOM + 1];
  bool lu_ready[BEMGPU_MAXDOM + 1] = {};
  // domains with triangles: the dpv system without padding (compact -> full index, size, matrix)
  int *cinv[BEMGPU_MAXDOM] = {};
  int cn[BEMGPU_MAXDOM] = {};
  double *Gc[BEMGPU_MAXDOM] = {};
  double *B3c = nullptr;
  bool fac_fp64[BEMGPU_MAXDOM + 1] = {};
  bool factored = false;  // factors of the current matrices are held (bemgpu_solve_rhs may run)
  double *b0 = nullptr, *B3s = nullptr;  // saved right-hand sides (FP64 fallback)
  // side lane: the dpv factorisations run there, overlapping the global system
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int st_n = 0, st_iters[BEMGPU_MAXDOM + 1] = {}, st_fallback[BEMGPU_MAXDOM + 1] = {}, st_gmres[BEMGPU_MAXDOM + 1] = {};
  double st_corr[BEMGPU_MAXDOM + 1] = {};
  // Free-space (interior) domains: their matrices depend on the mesh, the
  // media and the frequency only, not on the in-plane Bloch wave vector or the
  // incident field.  int_data is what defines them for the loaded problem;
  // int_valid: G, H, dG, dH, dF of domains >= 1 hold that problem's matrices;
  // int_factored[d]: domain d's dpv factors are those of these matrices in the
  // current precision; int_reuse: this load found the same data, so assembly
  // and dpv factorisation of the interior domains are skipped.
  std::vector<unsigned char> int_data;
  bool int_valid = false, int_reuse = false;
  bool int_reuse_on = true;  // bemgpu_set_interior_reuse
  // interior derivative rows dG, dH: kept (default) or recomputed a block of
  // rows at a time in the particle-velocity step (bemgpu_set_interior_derivatives;
  // dgh_keep_req takes effect at the next load)
  bool dgh_keep = true, dgh_keep_req = true;
  double *dGc = nullptr, *dHc = nullptr;  // one block of recomputed rows
  int dgh_rows = 0;                       // rows a block holds
  int dgh_rows_req = 0;                   // asked for (0: 256 MiB of each)
  bool int_factored[BEMGPU_MAXDOM] = {};
  long long int_reused_loads = 0;
  // batch of Bloch vectors (bemgpu_batch_load): instance b's Ewald parameters,
  // periodic-domain G and H and incident data; instance 0's G, H and spectral
  // table are the context's own, the others' are owned here.  G[0], H[0] and
  // qp point at the selected instance (bemgpu_batch_select).
  struct batch_inst {
    bem_qp qp;
    double *G = nullptr, *H = nullptr, *stab = nullptr;
    std::vector<double> Pi, dPi, p_inc, v_inc;
    double pw[16];
  };
  std::vector<batch_inst> bat;
  int bat_cur = -1;
  // instance buffers kept between batches (G, H, spectral table; bytes each)
  struct batch_bufs { double *G = nullptr, *H = nullptr, *stab = nullptr; size_t gh = 0, st = 0; };
  std::vector<batch_bufs> bat_pool;
};


static int fail(bemgpu_ctx *c, const char *what, cudaError_t e) {
  if (c) snprintf(c->err, sizeof(c->err), "%s: %s", what, cudaGetErrorString(e));
  return -1;
}
#define CK(call, what)                           \
  do {                                           \
    cudaError_t _e = (call);                     \
    if (_e != cudaSuccess) return fail(c, what, _e); \
  } while (0)

template <class T>
static cudaError_t dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  return cudaMalloc((void **)p, count * sizeof(T));
}
template <class T>
static void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}
// a problem-sized field of the context: reuses its allocation when it is large enough
template <class T>
static cudaError_t falloc(bemgpu_ctx *c, T **p, size_t count) {
  const size_t bytes = (count ? count : 1) * sizeof(T);
  auto it = c->cap.find((const void *)p);
  if (*p && it != c->cap.end() && it->second >= bytes) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  c->cap.erase((const void *)p);
  const cudaError_t e = cudaMalloc((void **)p, bytes);
  if (e == cudaSuccess) c->cap[(const void *)p] = bytes;
  return e;
}

// Gauss-Legendre tables and Faddeeva constants are uploaded once per device.
static int g_const_dev = -1;

// back to a single problem: instance 0 selected again (its G, H and
// parameters are the context's own buffers), the others' buffers freed
static void batch_clear(bemgpu_ctx *c) {
  if (c->bat.empty()) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->G[0] = c->bat[0].G;
  c->H[0] = c->bat[0].H;
  c->qp = c->bat[0].qp;
  // instance b >= 1's buffers stay in bat_pool[b - 1] for the next batch
  c->bat.clear();
  c->bat_cur = -1;
}

// release: give every problem buffer back (unload, destroy); otherwise a new
// load follows and reuses the allocations that are large enough (falloc)
static void free_problem(bemgpu_ctx *c, bool release) {
  batch_clear(c);
  if (release) {
    for (auto &p : c->bat_pool) { dfree(p.G); dfree(p.H); dfree(p.stab); }
    c->bat_pool.clear();
    dfree(c->cr); dfree(c->cw); dfree(c->ren); dfree(c->wen); dfree(c->plane);
    dfree(c->sid); dfree(c->rowidx); dfree(c->npe); dfree(c->eni); dfree(c->md); dfree(c->dom_ne_d); dfree(c->dom_off_d);
    dfree(c->hk2); dfree(c->Pi); dfree(c->dPi); dfree(c->p_inc); dfree(c->v_inc); dfree(c->rho0_d); dfree(c->k2_d);
    for (int d = 0; d < BEMGPU_MAXDOM; ++d) {
      dfree(c->G[d]); dfree(c->H[d]); dfree(c->dG[d]); dfree(c->dH[d]); dfree(c->dF[d]);
      c->cap.erase((const void *)&c->dG[d]);
      c->cap.erase((const void *)&c->dH[d]);
      dfree(c->P[d]); dfree(c->dP[d]); dfree(c->pv[d]); dfree(c->dpv[d]);
    }
    for (bem_scratch *S : {&c->scr, &c->scr1}) {
      dfree(S->rowF); dfree(S->near_s); dfree(S->near_n); dfree(S->nearF); dfree(S->selfF); dfree(S->flag);
    }
    dfree(c->scr.plist); dfree(c->scr.pcount);
    dfree(c->A); dfree(c->b); dfree(c->tpv); dfree(c->B3); dfree(c->wtab); dfree(c->stab); dfree(c->b0); dfree(c->B3s);
    for (int d = 0; d < BEMGPU_MAXDOM; ++d) { dfree(c->Wd[d]); dfree(c->cinv[d]); dfree(c->Gc[d]); }
    dfree(c->B3c);
    dfree(c->dGc); dfree(c->dHc);
    dfree(c->pw_d); dfree(c->tgt_t); dfree(c->tgt_ze); dfree(c->tgt_w); dfree(c->bdv);
    dfree(c->ctr_t); dfree(c->ctr_idx); dfree(c->ctr_ze); dfree(c->ctr_bdv);
    c->cap.clear();
    c->int_valid = false;  // the interior matrices went with the buffers
    c->int_data.clear();
    for (int d = 0; d < BEMGPU_MAXDOM; ++d) c->int_factored[d] = false;
  }
  for (int d = 0; d < BEMGPU_MAXDOM; ++d) c->cn[d] = 0;
  c->factored = false;
  c->nctr = 0;
  c->ntgt = 0;
  c->loaded = false;
}

extern "C" int bemgpu_create(int device, void *stream, bemgpu_ctx **out) {
  *out = nullptr;
  bemgpu_ctx *c = new bemgpu_ctx();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { delete c; return -1; }
  if (stream) {
    c->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return -1; }
    c->own_stream = true;
  }
  if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    delete c;
    return -1;
  }
  for (int i = 0; i <= BEMGPU_MAXDOM; ++i) {
    if (bem_lu_init(&c->lus[i], device) != 0) {
      for (int j = 0; j < i; ++j) bem_lu_free(&c->lus[j]);
      delete c;
      return -1;
    }
    c->lu_ready[i] = true;
  }
  if (dalloc(&c->status, 1) != cudaSuccess || dalloc(&c->fout, 8) != cudaSuccess ||
      dalloc(&c->rc_d, 4) != cudaSuccess || dalloc(&c->terms, 6) != cudaSuccess) {
    delete c;
    return -1;
  }
  for (int i = 0; i < 17; ++i)
    if (cudaEventCreate(&c->ev[i]) != cudaSuccess) { delete c; return -1; }
  cudaMemset(c->status, 0, sizeof(unsigned));
  cudaMemset(c->terms, 0, 6 * sizeof(unsigned long long));
  *out = c;
  return 0;
}

extern "C" void bemgpu_destroy(bemgpu_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_problem(c, true);
  dfree(c->status); dfree(c->fout); dfree(c->rc_d); dfree(c->terms);
  dfree(c->pt_in); dfree(c->pt_out); dfree(c->pt_t);
  for (int i = 0; i <= BEMGPU_MAXDOM; ++i)
    if (c->mx_ready[i]) { bem_mixed_free(&c->mxs[i]); c->mx_ready[i] = false; }
  for (int i = 0; i <= BEMGPU_MAXDOM; ++i)
    if (c->lu_ready[i]) { bem_lu_free(&c->lus[i]); c->lu_ready[i] = false; }
  for (int i = 0; i < 17; ++i)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  if (c->side) { cudaStreamSynchronize(c->side); cudaStreamDestroy(c->side); }
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" const char *bemgpu_error(const bemgpu_ctx *c) { return c ? c->err : "no context"; }

extern "C" unsigned bemgpu_status(bemgpu_ctx *c) {
  unsigned s = 0;
  cudaMemcpyAsync(&s, c->status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream);
  cudaStreamSynchronize(c->stream);
  return s;
}

extern "C" int bemgpu_sync(bemgpu_ctx *c) {
  CK(cudaStreamSynchronize(c->stream), "sync");
  return 0;
}


// Gauss-Legendre nodes and weights on [-1,1] by Newton iteration on the
// three-term Legendre recurrence (the rule the reference tabulates with
// gauleg, com_src/gauleg.c).
static void gl_rule(int n, double *x, double *w) {
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = 0.0;
      for (int j = 1; j <= n; ++j) {
        const double p2 = p1;
        p1 = p0;
        p0 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j;
      }
      dp = n * (z * p0 - p1) / (z * z - 1.0);
      const double dz = p0 / dp;
      z -= dz;
      if (fabs(dz) <= 3e-16) break;
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
}

static int ensure_constants(bemgpu_ctx *c, const double *xl, const double *wl, const double *xh, const double *wh) {
  double bxl[BEM_GLN_H], bwl[BEM_GLN_H], bxh[BEM_GHN_H], bwh[BEM_GHN_H];
  if (!xl) { gl_rule(BEM_GLN_H, bxl, bwl); xl = bxl; wl = bwl; }
  if (!xh) { gl_rule(BEM_GHN_H, bxh, bwh); xh = bxh; wh = bwh; }
  if (bem_set_constants(xl, wl, xh, wh) != 0) {
    if (c) snprintf(c->err, sizeof(c->err), "constant upload failed");
    return -1;
  }
  g_const_dev = c ? c->device : 0;
  return 0;
}

template <class T>
static int upload(bemgpu_ctx *c, T **dst, const T *src, size_t count, const char *what) {
  CK(falloc(c, dst, count), what);
  if (src && count) CK(cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice, c->stream), what);
  return 0;
}

// Window of the spectral order table for q: n1 within BEM_ST_W of nc1, n2
// within BEM_ST_W of every such row's centre, d = z / (2 eta_run) within
// +-zspan / (2 eta_run).  Returns the table's doubles (0: no table, when
// it would exceed 64 MB).
static size_t stab_window(bem_qp *q, double zspan) {
  q->st = nullptr;
  q->st_n1lo = q->nc1 - BEM_ST_W;
  q->st_n1cnt = 2 * BEM_ST_W + 1;
  int lo = 0, hi = 0;
  for (int i = 0; i < q->st_n1cnt; ++i) {
    const int n1 = q->st_n1lo + i;
    const int nc = (int)round(-((-q->kx + n1 * q->g1x) * q->g2x + (-q->ky + n1 * q->g1y) * q->g2y) / q->g2sq);
    if (i == 0 || nc < lo) lo = nc;
    if (i == 0 || nc > hi) hi = nc;
  }
  q->st_n2lo = lo - BEM_ST_W;
  q->st_n2cnt = hi - lo + 2 * BEM_ST_W + 1;
  q->st_nint = 2 * ((int)ceil(zspan / (2.0 * q->eta_run) / BEM_ST_H) + 1);  // d in [-D, D)
  const size_t cnt = (size_t)q->st_n1cnt * q->st_n2cnt * q->st_nint * BEM_ST_DEG * 2;
  if (cnt > ((size_t)64 << 20) / sizeof(double)) {
    q->st_n1cnt = q->st_n2cnt = q->st_nint = 0;
    return 0;
  }
  return cnt;
}

// The Ewald parameter by rule: k^2 eta^2 just below the reference's cap
// EW_EXPM = 3 (d3_qpgf_d2.h:26, 1684-1697), so that no point needs its own
// capped parameter (such points miss the per-problem term tables) and the
// split leans as far to the cheaper spectral side as the cap allows; clamped
// to [0.5, 1.3] x eta0.  Results agree with any other scale to round-off.
static double ewald_rule_scale(const bem_qp &q) {
  const double s = 0.98 * sqrt(3.0) / (q.k * q.eta0);
  return s < 0.5 ? 0.5 : (s > 1.3 ? 1.3 : s);
}

// (re)build the context's evanescent order table for its eta_run
static int build_stab(bemgpu_ctx *c) {
  const size_t cnt = stab_window(&c->qp, c->zspan);
  if (!cnt) return 0;
  CK(falloc(c, &c->stab, cnt), "spectral table");
  if (bem_launch_stab(&c->qp, c->stab, c->stream) != 0) return fail(c, "spectral table", cudaGetLastError());
  c->qp.st = c->stab;
  return 0;
}

extern "C" int bemgpu_load(bemgpu_ctx *c, const bemgpu_problem *pr) {
  CK(cudaSetDevice(c->device), "set device");
  // the previous problem's work ends before its buffers are reused
  if (c->stream) CK(cudaStreamSynchronize(c->stream), "load");
  if (c->side) CK(cudaStreamSynchronize(c->side), "load");
  free_problem(c, false);
  if (pr->MN + 1 > BEMGPU_MAXDOM) { snprintf(c->err, sizeof(c->err), "at most %d domains", BEMGPU_MAXDOM); return -2; }
  if (pr->ps != 1) { snprintf(c->err, sizeof(c->err), "only the quasi-periodic problem (ps=1) is implemented"); return -2; }
  for (int e = 0; e < pr->Ne; ++e)
    if (pr->npe[e] != 4 && pr->npe[e] != 3) { snprintf(c->err, sizeof(c->err), "element %d: %d nodes (3 or 4 expected)", e + 1, pr->npe[e]); return -2; }
  if (ensure_constants(c, pr->xl, pr->wl, pr->xh, pr->wh) != 0) return -1;
  {
    // what the interior domains' matrices depend on: the element tables, the
    // domain lists and the interior wave numbers (quadrature rules are fixed)
    std::vector<unsigned char> idata;
    auto put = [&idata](const void *p, size_t bytes) {
      const unsigned char *b = (const unsigned char *)p;
      idata.insert(idata.end(), b, b + bytes);
    };
    const size_t ne = pr->Ne;
    int tot = 0;
    for (int d = 0; d <= pr->MN; ++d) tot += pr->dom_ne[d];
    put(&pr->Ne, sizeof(int)); put(&pr->MN, sizeof(int));
    put(pr->dom_ne, sizeof(int) * (pr->MN + 1)); put(pr->sid, sizeof(int) * (size_t)tot);
    put(pr->cr, sizeof(double) * 12 * ne); put(pr->cw, sizeof(double) * 9 * ne);
    put(pr->ren, sizeof(double) * 12 * ne); put(pr->wen, sizeof(double) * 12 * ne);
    put(pr->npe, sizeof(int) * ne); put(pr->plane, ne);
    put(pr->k0 + 1, sizeof(double) * pr->MN);
    c->int_reuse = c->int_reuse_on && pr->MN >= 1 && c->int_valid && idata == c->int_data;
    if (!c->int_reuse) {
      c->int_valid = false;
      for (int d = 0; d < BEMGPU_MAXDOM; ++d) c->int_factored[d] = false;
      c->int_data.swap(idata);
    } else {
      ++c->int_reused_loads;
    }
  }
  c->Ne = pr->Ne; c->NN = pr->NN; c->MN = pr->MN; c->n = 2 * pr->NN;
  bem_qp_prepare(pr->qp, &c->qp);
  CK(falloc(c, &c->wtab, BEM_WT_SIZE), "w table");
  c->qp.eta_run = c->qp.eta0 * (c->eta_scale > 0.0 ? c->eta_scale : ewald_rule_scale(c->qp));
  if (bem_launch_wtab(c->qp.k, c->qp.eta_run, c->wtab, c->stream) != 0) return fail(c, "w table", cudaGetLastError());
  c->qp.wt = c->wtab;
  c->qp.wt_h = BEM_WT_H;
  c->qp.wt_n = BEM_WT_N;
  {  // z extent of the mesh: every element within cr0 -+ (|cr1| + |cr2| + |cr3|)
    double zlo = 0.0, zhi = 0.0;
    for (int e = 0; e < pr->Ne; ++e) {
      const double *z = pr->cr + (size_t)e * 12 + 8;
      const double hw = fabs(z[1]) + fabs(z[2]) + fabs(z[3]);
      if (e == 0 || z[0] - hw < zlo) zlo = z[0] - hw;
      if (e == 0 || z[0] + hw > zhi) zhi = z[0] + hw;
    }
    c->zspan = zhi - zlo;
  }
  if (build_stab(c)) return -1;
  memcpy(c->pw, pr->pw, sizeof(c->pw));
  if (upload(c, &c->pw_d, c->pw, 16, "pw")) return -1;
  const int nd = pr->MN + 1;
  c->dom_ne.assign(pr->dom_ne, pr->dom_ne + nd);
  c->dom_off.assign(nd, 0);
  int tot = 0;
  for (int d = 0; d < nd; ++d) { c->dom_off[d] = tot; tot += c->dom_ne[d]; }
  c->dom_tri.assign(nd, 0);
  for (int d = 0; d < nd; ++d)
    for (int s2 = 0; s2 < c->dom_ne[d]; ++s2)
      if (pr->npe[abs(pr->sid[c->dom_off[d] + s2]) - 1] == 3) c->dom_tri[d] = 1;
  c->k0.assign(pr->k0, pr->k0 + nd);
  c->c0.assign(pr->c0, pr->c0 + nd);
  c->rho0.assign(pr->rho0, pr->rho0 + nd);
  c->k2.assign(pr->k2, pr->k2 + 2 * nd);
  // global row of each (domain, element, node): the reference's row order
  // (create_matrix_csr_dac writes rows domain by domain, element by element)
  std::vector<int> rowidx(4 * (size_t)tot, -1);
  int row = 0;
  for (int d = 0; d < nd; ++d)
    for (int s = 0; s < c->dom_ne[d]; ++s) {
      const int asd = abs(pr->sid[c->dom_off[d] + s]) - 1;
      for (int l = 0; l < pr->npe[asd]; ++l) rowidx[4 * (size_t)(c->dom_off[d] + s) + l] = row++;
    }
  if (row != c->n) { snprintf(c->err, sizeof(c->err), "row count %d != 2 NN = %d", row, c->n); return -2; }
  std::vector<double> hk2(2 * (size_t)pr->Ne);
  for (int e = 0; e < pr->Ne; ++e) {
    const double *km = pr->k2 + 2 * pr->md[e], *ks = pr->k2 + 2 * pr->sd[e];
    const double den = ks[0] * ks[0] + ks[1] * ks[1];
    hk2[2 * e] = (km[0] * ks[0] + km[1] * ks[1]) / den;
    hk2[2 * e + 1] = (km[1] * ks[0] - km[0] * ks[1]) / den;
  }
  const size_t Ne = pr->Ne;
  if (upload(c, &c->cr, pr->cr, Ne * 12, "cr") || upload(c, &c->cw, pr->cw, Ne * 9, "cw") ||
      upload(c, &c->ren, pr->ren, Ne * 12, "ren") || upload(c, &c->wen, pr->wen, Ne * 12, "wen") ||
      upload(c, &c->plane, pr->plane, Ne, "plane") || upload(c, &c->sid, pr->sid, (size_t)tot, "sid") ||
      upload(c, &c->rowidx, rowidx.data(), rowidx.size(), "rowidx") || upload(c, &c->npe, pr->npe, Ne, "npe") ||
      upload(c, &c->eni, pr->eni, Ne * 4, "eni") || upload(c, &c->md, pr->md, Ne, "md") ||
      upload(c, &c->dom_ne_d, c->dom_ne.data(), (size_t)nd, "dom_ne") || upload(c, &c->dom_off_d, c->dom_off.data(), (size_t)nd, "dom_off") ||
      upload(c, &c->hk2, hk2.data(), hk2.size(), "hk2") || upload(c, &c->Pi, pr->Pi, Ne * 8, "Pi") ||
      upload(c, &c->dPi, pr->dPi, Ne * 8, "dPi") || upload(c, &c->p_inc, pr->p_inc, Ne * 8, "p_inc") ||
      upload(c, &c->v_inc, pr->v_inc, Ne * 24, "v_inc") || upload(c, &c->rho0_d, pr->rho0, (size_t)nd, "rho0") ||
      upload(c, &c->k2_d, pr->k2, 2 * (size_t)nd, "k2"))
    return -1;
  // per-domain outputs
  int maxN = 0;
  for (int d = 0; d < nd; ++d) {
    const size_t N = 4 * (size_t)c->dom_ne[d];
    if ((int)N > maxN) maxN = (int)N;
    CK(falloc(c, &c->G[d], 2 * N * N), "G");
    CK(falloc(c, &c->H[d], 2 * N * N), "H");
    if (d > 0 && c->dgh_keep_req) {
      CK(falloc(c, &c->dG[d], 4 * N * N), "dG");
      CK(falloc(c, &c->dH[d], 4 * N * N), "dH");
    } else if (d > 0) {
      // recomputed per block of rows: the full-size rows are not kept
      dfree(c->dG[d]);
      dfree(c->dH[d]);
      c->cap.erase((const void *)&c->dG[d]);
      c->cap.erase((const void *)&c->dH[d]);
    }
    CK(falloc(c, &c->dF[d], 3 * N), "dF");
    CK(falloc(c, &c->P[d], 2 * N), "P");
    CK(falloc(c, &c->dP[d], 2 * N), "dP");
    CK(falloc(c, &c->pv[d], 6 * N), "pv");
    CK(falloc(c, &c->dpv[d], 6 * N), "dpv");
    CK(cudaMemsetAsync(c->pv[d], 0, 6 * N * sizeof(double), c->stream), "pv");
  }
  // scratch of the periodic domain and, apart, of the free-space domains (they
  // are assembled on the side stream while the periodic domain is)
  for (int g = 0; g < 2; ++g) {
    bem_scratch &S = g == 0 ? c->scr : c->scr1;
    size_t sN = 0, sNe = 0;
    for (int d = g; d < (g == 0 ? 1 : nd); ++d) {
      sN = 4 * (size_t)c->dom_ne[d] > sN ? 4 * (size_t)c->dom_ne[d] : sN;
      sNe = (size_t)c->dom_ne[d] > sNe ? (size_t)c->dom_ne[d] : sNe;
    }
    CK(falloc(c, &S.rowF, 3 * sN), "rowF");
    CK(falloc(c, &S.near_s, sN * BEM_MAXNEAR_H), "near_s");
    CK(falloc(c, &S.near_n, sN), "near_n");
    CK(falloc(c, &S.nearF, sN * BEM_MAXNEAR_H * 3), "nearF");
    CK(falloc(c, &S.selfF, 3 * sN), "selfF");
    CK(falloc(c, &S.flag, sN * sNe), "flag");
    S.status = c->status;
    S.terms = c->terms;
  }
  // pair lists of the periodic domain (32-bit entries: up to 2^32 pairs)
  const size_t npair = (size_t)4 * c->dom_ne[0] * c->dom_ne[0];
  if (npair > 0 && npair <= 0xffffffffull) {
    CK(falloc(c, &c->scr.plist, npair), "pair lists");
    CK(falloc(c, &c->scr.pcount, 16), "pair lists");
    c->scr.pcap = npair;
  } else {
    c->scr.pcap = 0;
  }
  CK(cudaMemsetAsync(c->terms, 0, 6 * sizeof(unsigned long long), c->stream), "counters");
  const size_t n = c->n;
  CK(falloc(c, &c->A, 2 * n * n), "A");
  CK(falloc(c, &c->b, 2 * n), "b");
  CK(falloc(c, &c->tpv, 6 * (size_t)c->NN), "tpv");
  for (int d = 0; d < nd; ++d) {
    const size_t N = 4 * (size_t)c->dom_ne[d];
    CK(falloc(c, &c->Wd[d], 2 * N * N), "dpv factors");
    c->cn[d] = (int)N;
    if (c->dom_tri[d]) {
      std::vector<int> inv;
      for (int s2 = 0; s2 < c->dom_ne[d]; ++s2) {
        const int npe = pr->npe[abs(pr->sid[c->dom_off[d] + s2]) - 1];
        for (int l = 0; l < npe; ++l) inv.push_back(4 * s2 + l);
      }
      c->cn[d] = (int)inv.size();
      if (upload(c, &c->cinv[d], inv.data(), inv.size(), "dpv index")) return -1;
      CK(falloc(c, &c->Gc[d], 2 * inv.size() * inv.size()), "dpv matrix");
      CK(falloc(c, &c->B3c, 6 * (size_t)maxN), "dpv rhs");
    }
  }
  CK(falloc(c, &c->B3, 6 * (size_t)maxN), "B3");
  c->dgh_keep = c->dgh_keep_req;
  if (!c->dgh_keep && nd > 1) {
    // a block of recomputed derivative rows: 256 MiB for each of dG, dH (at
    // least 32 rows), rows a multiple of 4 (one element's nodes)
    int maxNi = 0;
    for (int d = 1; d < nd; ++d) maxNi = 4 * c->dom_ne[d] > maxNi ? 4 * c->dom_ne[d] : maxNi;
    size_t rows = ((size_t)256 << 20) / (64 * (size_t)(maxNi ? maxNi : 1));
    rows = rows < 32 ? 32 : rows;
    if (c->dgh_rows_req > 0) rows = (size_t)c->dgh_rows_req;
    rows = rows > (size_t)maxNi ? (size_t)maxNi : rows;
    rows -= rows % 4;
    c->dgh_rows = (int)(rows ? rows : 4);
    CK(falloc(c, &c->dGc, 4 * (size_t)c->dgh_rows * maxNi), "dG rows");
    CK(falloc(c, &c->dHc, 4 * (size_t)c->dgh_rows * maxNi), "dH rows");
  }
  CK(cudaMemsetAsync(c->status, 0, sizeof(unsigned), c->stream), "status");
  // device view of the system
  bem_sys_dev &S = c->sys;
  memset(&S, 0, sizeof(S));
  S.n = c->n; S.NN = c->NN; S.MN = c->MN;
  S.dom_ne = c->dom_ne_d; S.dom_off = c->dom_off_d;
  for (int d = 0; d < nd; ++d) S.dom_ne_h[d] = c->dom_ne[d];
  S.sid = c->sid; S.rowidx = c->rowidx; S.npe = c->npe; S.eni = c->eni; S.md = c->md; S.hk2 = c->hk2;
  S.Pi = c->Pi; S.dPi = c->dPi; S.p_inc = c->p_inc; S.v_inc = c->v_inc;
  S.cr = c->cr; S.ren = c->ren; S.wen = c->wen; S.rho0 = c->rho0_d; S.k2 = c->k2_d;
  const double a = 0.5773502691896257645091;
  const double zt[4] = {-a, a, a, -a}, et[4] = {-a, -a, a, a};
  for (int i = 0; i < 4; ++i) { S.zt44[i] = zt[i]; S.et44[i] = et[i]; }
  c->loaded = true;
  return 0;
}

extern "C" int bemgpu_set_far_rule(bemgpu_ctx *c, int on) {
  c->far_rule = on ? 1 : 0;
  c->factored = false;
  return 0;
}

extern "C" int bemgpu_rule_pairs(bemgpu_ctx *c, unsigned long long counts[6]) {
  if (!c || !counts) return -2;
  if (!c->scr.pcount || c->scr.pcap == 0) return -2;
  unsigned n[6];
  if (cudaMemcpyAsync(n, c->scr.pcount, sizeof(n), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return fail(c, "rule_pairs", cudaGetLastError());
  for (int i = 0; i < 6; ++i) counts[i] = n[i];
  return 0;
}

extern "C" int bemgpu_set_ewald_scale(bemgpu_ctx *c, double scale) {
  if (!c->bat.empty()) { snprintf(c->err, sizeof(c->err), "a batch is loaded (load a single problem first)"); return -2; }
  if (scale != BEMGPU_EWALD_RULE && !(scale >= 0.25 && scale <= 4.0)) {
    snprintf(c->err, sizeof(c->err), "Ewald scale %g outside [0.25, 4]", scale);
    return -2;
  }
  c->eta_scale = scale;  // 0 (the rule) is applied to every problem loaded from now on
  c->factored = false;
  if (!c->loaded) return 0;
  c->qp.eta_run = c->qp.eta0 * (scale > 0.0 ? scale : ewald_rule_scale(c->qp));
  if (bem_launch_wtab(c->qp.k, c->qp.eta_run, c->wtab, c->stream) != 0) return fail(c, "w table", cudaGetLastError());
  return build_stab(c);
}

static bem_dom_dev dom_view(bemgpu_ctx *c, int d);

// Ewald-parameter autotuner: time the periodic regular-pair kernel on a
// sample of the pairs for the rule's scale and three neighbours (larger
// factors meet the per-point cap and lose the tabulated terms) and keep the
// fastest.
extern "C" int bemgpu_autotune(bemgpu_ctx *c, double *best_scale) {
  if (!c->bat.empty()) { snprintf(c->err, sizeof(c->err), "a batch is loaded (load a single problem first)"); return -2; }
  if (!c->loaded) { snprintf(c->err, sizeof(c->err), "no problem loaded"); return -2; }
  bem_dom_dev D = dom_view(c, 0);
  if (bem_launch_classify(&D, &c->qp, 1, &c->scr, c->stream)) return fail(c, "autotune", cudaGetLastError());
  double *tab = nullptr, *stab = nullptr;
  CK(dalloc(&tab, BEM_WT_SIZE), "autotune");
  // the rule's scale and its neighbours
  const double r0 = ewald_rule_scale(c->qp);
  const double cand[4] = {r0, 0.9 * r0, 0.8 * r0, r0 < 1.0 ? 1.0 : 1.1 * r0};
  double best = r0;
  float tbest = 1e30f;
  int rc = 0;
  for (int i = 0; i < 4 && !rc; ++i) {
    bem_qp q = c->qp;
    q.eta_run = q.eta0 * cand[i];
    q.wt = tab;
    if (bem_launch_wtab(q.k, q.eta_run, tab, c->stream)) { rc = fail(c, "autotune", cudaGetLastError()); break; }
    // the candidate's own evanescent order table, as the assembly would use it
    dfree(stab);
    stab = nullptr;
    const size_t scnt = stab_window(&q, c->zspan);
    if (scnt) {
      if (dalloc(&stab, scnt) != cudaSuccess || bem_launch_stab(&q, stab, c->stream)) {
        rc = fail(c, "autotune", cudaGetLastError());
        break;
      }
      q.st = stab;
    }
    float t = 0.f, tmin = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {
      if (bem_time_regular(&D, &q, &c->scr, c->G[0], c->H[0], 0.125, 4, c->stream, &t)) {
        rc = fail(c, "autotune", cudaGetLastError());
        break;
      }
      tmin = t < tmin ? t : tmin;
    }
    if (tmin < tbest) { tbest = tmin; best = cand[i]; }
  }
  cudaStreamSynchronize(c->stream);
  cudaFree(tab);
  dfree(stab);
  if (rc) return rc;
  if (best_scale) *best_scale = best;
  return bemgpu_set_ewald_scale(c, best);
}

extern "C" int bemgpu_unload(bemgpu_ctx *c) {
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->side) cudaStreamSynchronize(c->side);
  free_problem(c, true);
  return 0;
}

static bem_dom_dev dom_view(bemgpu_ctx *c, int d);

extern "C" int bemgpu_assemble(bemgpu_ctx *c) {
  c->factored = false;
  if (!c->loaded) { snprintf(c->err, sizeof(c->err), "no problem loaded"); return -2; }
  // the free-space domains on the side stream, beside the periodic domain
  if (c->MN >= 1) {
    CK(cudaEventRecord(c->ev_fork, c->stream), "assembly fork");
    CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0), "assembly fork");
  }
  // interior matrices of the same mesh, media and frequency are kept (int_reuse)
  const bool skip_interior = c->int_reuse && c->int_valid;
  for (int d = 0; d <= c->MN; ++d) {
    cudaEvent_t *ev = c->prof && d < 2 ? c->ev + 6 * d : nullptr;
    if (d > 0 && skip_interior) {
      if (ev)
        for (int i = 0; i < 6; ++i) CK(cudaEventRecord(ev[i], c->side), "phase events");
      continue;
    }
    bem_dom_dev D = dom_view(c, d);
    const int periodic = d == 0;
    if (bem_launch_assemble(&D, &c->qp, periodic, d == 0, c->k0[d], d == 0 ? &c->scr : &c->scr1, c->G[d], c->H[d],
                            c->dG[d], c->dH[d], c->dF[d], d == 0 ? c->stream : c->side, ev) != 0)
      return fail(c, "assembly launch", cudaGetLastError());
  }
  if (c->MN >= 1) {
    CK(cudaEventRecord(c->ev_join, c->side), "assembly join");
    CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0), "assembly join");
  }
  c->int_valid = c->MN >= 1;
  return 0;
}

// ---------------------------------------------------------------- batches of Bloch vectors
// Problems on one body, media, lattice and frequency that differ only in the
// incidence (in-plane Bloch wave vector and incident field): the free-space
// domains and the periodic domain's classification are the same for all of
// them, so one batch assembles the interior domains once and the periodic
// domain of every instance with each kernel launched once
// (bem_launch_assemble_batch).
static bool same_body(const bemgpu_problem *a, const bemgpu_problem *b) {
  if (a->Ne != b->Ne || a->NN != b->NN || a->MN != b->MN || a->ps != b->ps) return false;
  const size_t ne = a->Ne, nd = a->MN + 1;
  size_t tot = 0;
  for (size_t d = 0; d < nd; ++d) {
    if (a->dom_ne[d] != b->dom_ne[d]) return false;
    tot += a->dom_ne[d];
  }
  if (a->qp[0] != b->qp[0]) return false;                       // k
  for (int i = 4; i < 8; ++i) if (a->qp[i] != b->qp[i]) return false;  // lattice
  return !memcmp(a->sid, b->sid, tot * sizeof(int)) && !memcmp(a->cr, b->cr, ne * 12 * sizeof(double)) &&
         !memcmp(a->cw, b->cw, ne * 9 * sizeof(double)) && !memcmp(a->ren, b->ren, ne * 12 * sizeof(double)) &&
         !memcmp(a->wen, b->wen, ne * 12 * sizeof(double)) && !memcmp(a->npe, b->npe, ne * sizeof(int)) &&
         !memcmp(a->eni, b->eni, ne * 4 * sizeof(int)) && !memcmp(a->plane, b->plane, ne) &&
         !memcmp(a->md, b->md, ne * sizeof(int)) && !memcmp(a->sd, b->sd, ne * sizeof(int)) &&
         !memcmp(a->k0, b->k0, nd * sizeof(double)) && !memcmp(a->k2, b->k2, 2 * nd * sizeof(double)) &&
         !memcmp(a->rho0, b->rho0, nd * sizeof(double)) && !memcmp(a->c0, b->c0, nd * sizeof(double));
}

extern "C" int bemgpu_batch_load(bemgpu_ctx *c, int nb, const bemgpu_problem *const *probs) {
  if (nb < 1 || !probs) { snprintf(c->err, sizeof(c->err), "batch of %d problems", nb); return -2; }
  for (int b = 1; b < nb; ++b)
    if (!same_body(probs[0], probs[b])) {
      snprintf(c->err, sizeof(c->err), "batch problem %d: not the same body, media, lattice and frequency", b);
      return -2;
    }
  const int rc = bemgpu_load(c, probs[0]);
  if (rc) return rc;
  if (c->dom_tri[0]) { snprintf(c->err, sizeof(c->err), "batches take quad meshes only"); return -2; }
  const size_t N = 4 * (size_t)c->dom_ne[0], ne = c->Ne;
  if (!c->scr.plist || (unsigned long long)(N * (size_t)c->dom_ne[0]) > c->scr.pcap) {
    snprintf(c->err, sizeof(c->err), "batches need the periodic domain's pair lists (at most 32768 elements)");
    return -2;
  }
  c->bat.resize(nb);
  for (int b = 0; b < nb; ++b) {
    bemgpu_ctx::batch_inst &I = c->bat[b];
    const bemgpu_problem *pr = probs[b];
    I.Pi.assign(pr->Pi, pr->Pi + ne * 8);
    I.dPi.assign(pr->dPi, pr->dPi + ne * 8);
    I.p_inc.assign(pr->p_inc, pr->p_inc + ne * 8);
    I.v_inc.assign(pr->v_inc, pr->v_inc + ne * 24);
    memcpy(I.pw, pr->pw, sizeof(I.pw));
    if (b == 0) {
      I.qp = c->qp;
      I.G = c->G[0];
      I.H = c->H[0];
      continue;
    }
    bem_qp_prepare(pr->qp, &I.qp);
    if (I.qp.eta0 != c->qp.eta0) {
      snprintf(c->err, sizeof(c->err), "batch problem %d: another Ewald parameter", b);
      batch_clear(c);
      return -2;
    }
    I.qp.eta_run = c->qp.eta_run;  // one real-space table for the batch
    I.qp.wt = c->qp.wt;
    I.qp.wt_h = c->qp.wt_h;
    I.qp.wt_n = c->qp.wt_n;
    const size_t cnt = stab_window(&I.qp, c->zspan);
    if ((int)c->bat_pool.size() < b) c->bat_pool.resize(b);
    bemgpu_ctx::batch_bufs &P = c->bat_pool[b - 1];
    cudaError_t e = cudaSuccess;
    if (P.gh < 2 * N * N) {
      dfree(P.G); dfree(P.H);
      P.gh = 0;
      e = dalloc(&P.G, 2 * N * N);
      if (e == cudaSuccess) e = dalloc(&P.H, 2 * N * N);
      if (e == cudaSuccess) P.gh = 2 * N * N;
    }
    if (e == cudaSuccess && cnt && P.st < cnt) {
      dfree(P.stab);
      P.st = 0;
      e = dalloc(&P.stab, cnt);
      if (e == cudaSuccess) P.st = cnt;
    }
    if (e == cudaSuccess && cnt && bem_launch_stab(&I.qp, P.stab, c->stream) != 0) e = cudaGetLastError();
    if (e != cudaSuccess) {
      batch_clear(c);
      return fail(c, "batch buffers", e);
    }
    I.G = P.G;
    I.H = P.H;
    I.stab = cnt ? P.stab : nullptr;
    I.qp.st = I.stab;
  }
  c->bat_cur = 0;
  return 0;
}

extern "C" int bemgpu_batch_assemble(bemgpu_ctx *c) {
  if (!c->loaded || c->bat.empty()) { snprintf(c->err, sizeof(c->err), "no batch loaded"); return -2; }
  c->factored = false;
  if (c->MN >= 1) {
    CK(cudaEventRecord(c->ev_fork, c->stream), "assembly fork");
    CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0), "assembly fork");
  }
  const bool skip_interior = c->int_reuse && c->int_valid;
  for (int d = 1; d <= c->MN && !skip_interior; ++d) {
    bem_dom_dev D = dom_view(c, d);
    if (bem_launch_assemble(&D, &c->qp, 0, 0, c->k0[d], &c->scr1, c->G[d], c->H[d], c->dG[d], c->dH[d], c->dF[d],
                            c->side, nullptr) != 0)
      return fail(c, "assembly launch", cudaGetLastError());
  }
  const int nb = (int)c->bat.size();
  std::vector<bem_qp> qps(nb);
  std::vector<double *> gs(nb), hs(nb);
  for (int b = 0; b < nb; ++b) { qps[b] = c->bat[b].qp; gs[b] = c->bat[b].G; hs[b] = c->bat[b].H; }
  bem_dom_dev D = dom_view(c, 0);
  const int r = bem_launch_assemble_batch(&D, &c->bat[0].qp, nb, qps.data(), gs.data(), hs.data(), &c->scr, c->dF[0],
                                          c->stream);
  if (r == -2) { snprintf(c->err, sizeof(c->err), "batch assembly: quad meshes with pair lists only"); return -2; }
  if (r) return fail(c, "batch assembly launch", cudaGetLastError());
  if (c->MN >= 1) {
    CK(cudaEventRecord(c->ev_join, c->side), "assembly join");
    CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0), "assembly join");
  }
  c->int_valid = c->MN >= 1;
  return 0;
}

extern "C" int bemgpu_batch_select(bemgpu_ctx *c, int b) {
  if (!c->loaded || c->bat.empty() || b < 0 || b >= (int)c->bat.size()) {
    snprintf(c->err, sizeof(c->err), "no batch instance %d", b);
    return -2;
  }
  bemgpu_ctx::batch_inst &I = c->bat[b];
  CK(cudaStreamSynchronize(c->stream), "batch select");
  c->G[0] = I.G;
  c->H[0] = I.H;
  c->qp = I.qp;
  c->bat_cur = b;
  c->factored = false;
  // the interior domains' matrices are the batch's: their dpv factors, once
  // made by a solve, serve every instance
  if (b > 0) c->int_reuse = c->int_reuse_on;
  return bemgpu_set_incident(c, I.Pi.data(), I.dPi.data(), I.p_inc.data(), I.v_inc.data(), I.pw);
}

// Dense systems M X = B with M row-major FP64 (n x n), B column-major (n x nrhs).
// slot 0 is the global system (factors in place of A), slot 1 + d the dpv
// system of domain d (M = G[d], FP64 factors in Wd[d]).  FP64: the device LU
// of bem_lu.cu (P M = L U, row pivoting).  Mixed precision: FP32 factors +
// FP64 refinement against M, which stays intact; a system with a zero FP32
// pivot, or whose refinement does not reach 1e-12, switches to FP64 factors
// (then kept for later right-hand sides).
// lane 0: the context's stream (checked at once); lane 1: the side stream
// (dpv systems, checked after the join in bemgpu_solve)
static int lu_status_check(bemgpu_ctx *c, int slot, const char *what) {
  const unsigned st = bem_lu_status(&c->lus[slot], c->stream);
  if (st == 0xffffffffu) return fail(c, what, cudaGetLastError());
  if (st & BEM_LU_ST_ZERO) {
    snprintf(c->err, sizeof(c->err), "%s: zero pivot (singular matrix)", what);
    return -3;
  }
  if (st & (BEM_LU_ST_WAIT | BEM_LU_ST_INTERNAL)) {
    snprintf(c->err, sizeof(c->err), "%s: %s", what,
             (st & BEM_LU_ST_WAIT) ? "a triangular-solve wait gave up" : "a row move out of range");
    return -1;
  }
  return 0;
}

static int dense_factor_fp64(bemgpu_ctx *c, int slot, double *M, int64_t n, const char *what, int lane = 0) {
  double *F = slot == 0 ? M : c->Wd[slot - 1];
  cudaStream_t st = lane ? c->side : c->stream;
  if (F != M) CK(cudaMemcpyAsync(F, M, 2 * n * n * sizeof(double), cudaMemcpyDeviceToDevice, st), what);
  if (bem_lu_factor_z(&c->lus[slot], F, (int)n, st)) {
    snprintf(c->err, sizeof(c->err), "%s: %s", what, c->lus[slot].err);
    return -1;
  }
  c->fac_fp64[slot] = true;
  if (lane == 0) return lu_status_check(c, slot, what);
  return 0;
}

static int dense_factor(bemgpu_ctx *c, int slot, double *M, int64_t n, const char *what, int lane = 0) {
  c->fac_fp64[slot] = false;
  if (c->precision == 0) return dense_factor_fp64(c, slot, M, n, what, lane);
  if (!c->mx_ready[slot]) {
    if (bem_mixed_init(&c->mxs[slot], c->precision, c->stream)) { snprintf(c->err, sizeof(c->err), "%s: %s", what, c->mxs[slot].err); return -1; }
    c->mx_ready[slot] = true;
  }
  c->mxs[slot].req_mode = c->precision;
  cudaStream_t st = lane ? c->side : c->stream;
  if (bem_mixed_factor(&c->mxs[slot], M, (int)n, st)) {
    snprintf(c->err, sizeof(c->err), "%s: %s", what, c->mxs[slot].err);
    return -1;
  }
  if (lane == 0 && (bem_mixed_status(&c->mxs[slot], c->stream) & 0x20u)) {
    c->st_fallback[slot] = 1;
    return dense_factor_fp64(c, slot, M, n, what);
  }
  return 0;
}

// After the side lane joined: the dpv factorisations' outcome (zero pivots).
static int check_side_factors(bemgpu_ctx *c) {
  for (int d = 0; d <= c->MN; ++d) {
    const int slot = 1 + d;
    if (c->fac_fp64[slot]) {
      char what[48];
      snprintf(what, sizeof(what), "dpv LU of domain %d", d);
      const int r = lu_status_check(c, slot, what);
      if (r) return r;
    } else if (bem_mixed_status(&c->mxs[slot], c->stream) & 0x20u) {
      c->st_fallback[slot] = 1;
      const int r = dense_factor_fp64(c, slot, c->dom_tri[d] ? c->Gc[d] : c->G[d], c->cn[d], "dpv LU");
      if (r) return r;
    }
    if (d > 0) c->int_factored[d] = true;
  }
  return 0;
}

static int dense_apply(bemgpu_ctx *c, int slot, double *M, int64_t n, int64_t nrhs, double *B, double *Bsave,
                       const char *what) {
  c->st_iters[slot] = 0;
  c->st_corr[slot] = 0.0;
  if (!c->fac_fp64[slot]) {
    CK(cudaMemcpyAsync(Bsave, B, 2 * n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), what);
    int it = 0;
    double rc = 1.0;
    if (c->refine != 2) {
      if (bem_mixed_solve(&c->mxs[slot], M, (int)n, (int)nrhs, B, 30, 4.0 * 1.1102230246251565e-16, &it, &rc,
                          c->stream)) {
        snprintf(c->err, sizeof(c->err), "%s: %s", what, c->mxs[slot].err);
        return -1;
      }
      c->st_iters[slot] = it;
      c->st_corr[slot] = rc;
      if (rc <= 1e-12) return 0;
    }
    if (c->refine != 1) {
      // GMRES-IR with the same FP32 factors as the preconditioner, from the
      // saved right-hand sides; success: relative residual <= 1e-12
      CK(cudaMemcpyAsync(B, Bsave, 2 * n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), what);
      if (bem_mixed_solve_gmres(&c->mxs[slot], M, (int)n, (int)nrhs, B, 1e-14, &it, &rc, c->stream)) {
        snprintf(c->err, sizeof(c->err), "%s: %s", what, c->mxs[slot].err);
        return -1;
      }
      c->st_iters[slot] = it;
      c->st_corr[slot] = rc;
      c->st_gmres[slot] = 1;
      if (rc <= 1e-12) return 0;
    }
    // not refined to FP64 accuracy: FP64 factors from the intact M
    c->st_fallback[slot] = 1;
    CK(cudaMemcpyAsync(B, Bsave, 2 * n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), what);
    const int r = dense_factor_fp64(c, slot, M, n, what);
    if (r) return r;
  }
  double *F = slot == 0 ? M : c->Wd[slot - 1];
  if (bem_lu_solve_z(&c->lus[slot], F, (int)n, (int)nrhs, B, c->stream)) {
    snprintf(c->err, sizeof(c->err), "%s: %s", what, c->lus[slot].err);
    return -1;
  }
  return 0;
}

extern "C" int bemgpu_set_precision(bemgpu_ctx *c, int mode) {
  if (mode < 0 || mode > BEM_MIXED_FAST) { snprintf(c->err, sizeof(c->err), "precision mode %d (0..4)", mode); return -2; }
  c->precision = mode;
  c->factored = false;  // factors of the other precision are not reused
  for (int d = 0; d < BEMGPU_MAXDOM; ++d) c->int_factored[d] = false;
  return 0;
}

extern "C" int bemgpu_get_precision(bemgpu_ctx *c) {
  if (c->precision == 0) return 0;
  return c->mx_ready[0] ? c->mxs[0].mode : c->precision;
}

extern "C" int bemgpu_solve_stats(bemgpu_ctx *c, int *iters, double *rel_corr, int *fallback, int max) {
  int k = 0;
  for (; k < c->st_n && k < max; ++k) {
    if (iters) iters[k] = c->st_iters[k];
    if (rel_corr) rel_corr[k] = c->st_corr[k];
    if (fallback) fallback[k] = c->st_fallback[k];
  }
  return k;
}

// After the global solution X (in b): surface values, particle velocity and
// dpv of every domain (tmatrix_bd_store, q_solve_pv_bv, solve_dpv_bv,
// bem3_aw_qd2_solve_bieq.c:370-750), with the dpv factors already held.
static int solve_tail(bemgpu_ctx *c) {
  for (int d = 0; d <= c->MN; ++d)
    if (bem_launch_store(&c->sys, d, c->b, c->P[d], c->dP[d], c->stream)) return fail(c, "store", cudaGetLastError());
  if (c->prof) cudaEventRecord(c->ev[14], c->stream);
  // particle velocity: interior domains first, then domain 0 from the interface condition
  CK(cudaMemsetAsync(c->tpv, 0, 6 * (size_t)c->NN * sizeof(double), c->stream), "tpv");
  for (int d = 1; d <= c->MN; ++d) {
    if (c->dgh_keep) {
      if (bem_launch_pv(&c->sys, d, c->dG[d], c->dH[d], c->dF[d], c->P[d], c->dP[d], c->pv[d], c->tpv, c->stream))
        return fail(c, "pv", cudaGetLastError());
      continue;
    }
    // derivative rows recomputed a block at a time (pair flags and near lists
    // of this domain first: the free-space scratch may hold another domain's)
    bem_dom_dev D = dom_view(c, d);
    const int N = 4 * c->dom_ne[d];
    if (bem_launch_classify(&D, &c->qp, 0, &c->scr1, c->stream)) return fail(c, "classify", cudaGetLastError());
    for (int p0 = 0; p0 < N; p0 += c->dgh_rows) {
      const int np = N - p0 < c->dgh_rows ? N - p0 : c->dgh_rows;
      if (bem_launch_fs_deriv(&D, c->k0[d], &c->scr1, p0, np, c->dGc, c->dHc, c->stream) ||
          bem_launch_pv_rows(&c->sys, d, c->dGc, c->dHc, c->dF[d], c->P[d], c->dP[d], c->pv[d], c->tpv, p0, np,
                             c->stream))
        return fail(c, "pv", cudaGetLastError());
    }
  }
  if (bem_launch_pv(&c->sys, 0, nullptr, nullptr, nullptr, nullptr, nullptr, c->pv[0], c->tpv, c->stream))
    return fail(c, "pv0", cudaGetLastError());
  if (c->prof) cudaEventRecord(c->ev[15], c->stream);
  // dpv: G_d dpv = H_d pv per domain (solve_dpv_bv)
  for (int d = 0; d <= c->MN; ++d) {
    const int64_t Nd = 4 * (int64_t)c->dom_ne[d];
    if (Nd == 0) continue;
    if (bem_launch_dpv_rhs((int)Nd, c->H[d], c->pv[d], c->B3, c->stream)) return fail(c, "dpv rhs", cudaGetLastError());
    if (c->dom_tri[d]) {
      if (bem_launch_rows(c->B3, c->B3c, (int)Nd, c->cinv[d], c->cn[d], 3, 0, c->stream)) return fail(c, "dpv", cudaGetLastError());
      const int rc = dense_apply(c, 1 + d, c->Gc[d], c->cn[d], 3, c->B3c, c->B3s, "dpv solve");
      if (rc) return rc;
      if (bem_launch_rows(c->B3c, c->B3, (int)Nd, c->cinv[d], c->cn[d], 3, 1, c->stream)) return fail(c, "dpv", cudaGetLastError());
    } else {
      const int rc = dense_apply(c, 1 + d, c->G[d], Nd, 3, c->B3, c->B3s, "dpv solve");
      if (rc) return rc;
    }
    if (bem_launch_dpv_store((int)Nd, c->B3, c->dpv[d], c->stream)) return fail(c, "dpv store", cudaGetLastError());
  }
  if (c->prof) cudaEventRecord(c->ev[16], c->stream);
  return 0;
}

// The triangular solves' waits of every FP64 system (one synchronisation).
static int check_solve_waits(bemgpu_ctx *c) {
  for (int slot = 0; slot <= c->MN + 1; ++slot)
    if (c->fac_fp64[slot]) {
      const int r = lu_status_check(c, slot, slot ? "dpv solve" : "global solve");
      if (r) return r;
    }
  return 0;
}

static int ensure_saves(bemgpu_ctx *c) {
  if (c->precision != 0) {
    CK(falloc(c, &c->b0, 2 * (size_t)c->n), "b copy");
    CK(falloc(c, &c->B3s, 6 * (size_t)c->NN), "B3 copy");
  }
  // mixed-precision state of every dense system, set up before any lane uses it
  for (int slot = 0; c->precision != 0 && slot <= c->MN + 1; ++slot)
    if (!c->mx_ready[slot]) {
      if (bem_mixed_init(&c->mxs[slot], c->precision, c->stream)) {
        snprintf(c->err, sizeof(c->err), "mixed-precision set-up: %s", c->mxs[slot].err);
        return -1;
      }
      c->mx_ready[slot] = true;
    }
  c->st_n = c->MN + 2;
  for (int i = 0; i < c->st_n; ++i) c->st_fallback[i] = c->st_gmres[i] = 0;
  return 0;
}

extern "C" int bemgpu_solve(bemgpu_ctx *c) {
  if (!c->loaded) { snprintf(c->err, sizeof(c->err), "no problem loaded"); return -2; }
  const size_t n = c->n;
  c->factored = false;
  if (ensure_saves(c)) return -1;
  if (c->prof) cudaEventRecord(c->ev[12], c->stream);
  // the dpv systems depend only on G_d: factor them on the side lane while the
  // global system is gathered, factored and solved here
  CK(cudaEventRecord(c->ev_fork, c->stream), "fork");
  CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0), "fork");
  auto side_lane = [c]() -> int {
    for (int d = 0; d <= c->MN; ++d) {
      const int64_t Nd = 4 * (int64_t)c->dom_ne[d];
      if (Nd == 0) continue;
      if (d > 0 && c->int_reuse && c->int_factored[d]) continue;  // factors of the same interior matrices held
      c->int_factored[d] = false;
      double *M = c->G[d];
      if (c->dom_tri[d]) {
        if (bem_launch_compress(c->G[d], (int)Nd, c->cinv[d], c->cn[d], c->Gc[d], c->side))
          return fail(c, "dpv", cudaGetLastError());
        M = c->Gc[d];
      }
      const int r = dense_factor(c, 1 + d, M, c->cn[d], "dpv LU", 1);
      if (r) return r;
    }
    CK(cudaEventRecord(c->ev_join, c->side), "join");
    return 0;
  };
  // A large FP64 factorisation holds the calling thread until it is done, so
  // large dpv systems are factored from a second host thread: the global LU
  // below then runs beside them instead of after them.
  int max_nd = 0;
  for (int d = 0; d <= c->MN; ++d) max_nd = 4 * c->dom_ne[d] > max_nd ? 4 * c->dom_ne[d] : max_nd;
  int side_rc = 0;
  std::thread side_thread;
  if (max_nd >= 2048) {
    side_thread = std::thread([c, &side_rc, &side_lane]() {
      if (cudaSetDevice(c->device) != cudaSuccess) { side_rc = -1; return; }
      side_rc = side_lane();
    });
  } else {
    side_rc = side_lane();
    if (side_rc) return side_rc;
  }
  struct joiner {
    std::thread &t;
    ~joiner() { if (t.joinable()) t.join(); }
  } join_side{side_thread};
  CK(cudaMemsetAsync(c->A, 0, 2 * n * n * sizeof(double), c->stream), "A clear");
  CK(cudaMemsetAsync(c->b, 0, 2 * n * sizeof(double), c->stream), "b clear");
  for (int d = 0; d <= c->MN; ++d)
    if (bem_launch_gather(&c->sys, d, c->G[d], c->H[d], c->A, c->b, c->stream)) return fail(c, "gather", cudaGetLastError());
  if (c->prof) cudaEventRecord(c->ev[13], c->stream);
  int rc = dense_factor(c, 0, c->A, (int64_t)n, "global LU");
  if (!rc) rc = dense_apply(c, 0, c->A, (int64_t)n, 1, c->b, c->b0, "global solve");
  // join the side lane before anything reads the dpv factors
  if (side_thread.joinable()) side_thread.join();
  if (!rc) rc = side_rc;
  if (rc) return rc;
  const cudaError_t je = cudaStreamWaitEvent(c->stream, c->ev_join, 0);
  if (!rc && je != cudaSuccess) rc = fail(c, "join", je);
  if (!rc) rc = check_side_factors(c);
  if (!rc) rc = solve_tail(c);
  if (!rc) rc = check_solve_waits(c);
  if (rc) return rc;
  c->factored = true;
  return 0;
}

extern "C" int bemgpu_solve_rhs(bemgpu_ctx *c) {
  if (!c->loaded || !c->factored) {
    snprintf(c->err, sizeof(c->err), "no factorisation of the current matrices (run bemgpu_solve first)");
    return -2;
  }
  if (ensure_saves(c)) return -1;
  if (c->prof) cudaEventRecord(c->ev[12], c->stream);
  CK(cudaMemsetAsync(c->b, 0, 2 * (size_t)c->n * sizeof(double), c->stream), "b clear");
  for (int d = 0; d <= c->MN; ++d)
    if (bem_launch_gather(&c->sys, d, c->G[d], c->H[d], nullptr, c->b, c->stream)) return fail(c, "rhs", cudaGetLastError());
  if (c->prof) cudaEventRecord(c->ev[13], c->stream);
  int rc = dense_apply(c, 0, c->A, (int64_t)c->n, 1, c->b, c->b0, "global solve");
  if (!rc) rc = solve_tail(c);
  if (!rc) rc = check_solve_waits(c);
  return rc;
}

extern "C" int bemgpu_set_incident(bemgpu_ctx *c, const double *Pi, const double *dPi, const double *p_inc,
                                   const double *v_inc, const double *pw) {
  if (!c->loaded) { snprintf(c->err, sizeof(c->err), "no problem loaded"); return -2; }
  const size_t Ne = c->Ne;
  CK(cudaMemcpyAsync(c->Pi, Pi, Ne * 8 * sizeof(double), cudaMemcpyHostToDevice, c->stream), "Pi");
  CK(cudaMemcpyAsync(c->dPi, dPi, Ne * 8 * sizeof(double), cudaMemcpyHostToDevice, c->stream), "dPi");
  CK(cudaMemcpyAsync(c->p_inc, p_inc, Ne * 8 * sizeof(double), cudaMemcpyHostToDevice, c->stream), "p_inc");
  CK(cudaMemcpyAsync(c->v_inc, v_inc, Ne * 24 * sizeof(double), cudaMemcpyHostToDevice, c->stream), "v_inc");
  memcpy(c->pw, pw, sizeof(c->pw));
  CK(cudaMemcpyAsync(c->pw_d, c->pw, 16 * sizeof(double), cudaMemcpyHostToDevice, c->stream), "pw");
  CK(cudaStreamSynchronize(c->stream), "incident");
  return 0;
}

extern "C" int bemgpu_set_profiling(bemgpu_ctx *c, int on) {
  c->prof = on != 0;
  return 0;
}

// phases: domain 0 classify, regular, near, self, diag; domain 1 the same;
// gather, global LU + solve, boundary values (P, dP, pv), dpv solves
extern "C" int bemgpu_phase_times(bemgpu_ctx *c, double *ms, int max) {
  if (!c->prof) return 0;
  CK(cudaStreamSynchronize(c->stream), "phase times");
  int k = 0;
  for (int d = 0; d < 2 && d <= c->MN; ++d)
    for (int i = 0; i < 5 && k < max; ++i) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, c->ev[6 * d + i], c->ev[6 * d + i + 1]) != cudaSuccess) {
        t = -1.f;            // a phase that did not run since profiling was switched on
        cudaGetLastError();  // (clear the error so that it does not surface in a later launch check)
      }
      ms[k++] = t;
    }
  for (int i = 12; i < 16 && k < max; ++i) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, c->ev[i], c->ev[i + 1]) != cudaSuccess) {
      t = -1.f;
      cudaGetLastError();
    }
    ms[k++] = t;
  }
  return k;
}

extern "C" int bemgpu_work_counters(bemgpu_ctx *c, unsigned long long *out6, int reset) {
  CK(cudaMemcpyAsync(out6, c->terms, 6 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream), "counters");
  if (reset) CK(cudaMemsetAsync(c->terms, 0, 6 * sizeof(unsigned long long), c->stream), "counters");
  CK(cudaStreamSynchronize(c->stream), "counters");
  return 0;
}

extern "C" void *bemgpu_stream(bemgpu_ctx *c) { return (void *)c->stream; }

extern "C" int bemgpu_run(bemgpu_ctx *c) {
  int r = bemgpu_assemble(c);
  if (r) return r;
  return bemgpu_solve(c);
}

extern "C" int bemgpu_get_solution(bemgpu_ctx *c, int d, double *P, double *dP, double *pv, double *dpv) {
  if (!c->loaded || d < 0 || d > c->MN) { snprintf(c->err, sizeof(c->err), "bad domain"); return -2; }
  const size_t N = 4 * (size_t)c->dom_ne[d];
  if (P) CK(cudaMemcpyAsync(P, c->P[d], 2 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "P");
  if (dP) CK(cudaMemcpyAsync(dP, c->dP[d], 2 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "dP");
  if (pv) CK(cudaMemcpyAsync(pv, c->pv[d], 6 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "pv");
  if (dpv) CK(cudaMemcpyAsync(dpv, c->dpv[d], 6 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "dpv");
  CK(cudaStreamSynchronize(c->stream), "get solution");
  return 0;
}

extern "C" int bemgpu_get_matrix(bemgpu_ctx *c, int d, int which, double *dst) {
  if (!c->loaded || d < 0 || d > c->MN) { snprintf(c->err, sizeof(c->err), "bad domain"); return -2; }
  const size_t N = 4 * (size_t)c->dom_ne[d];
  const double *src = nullptr;
  size_t cnt = 0;
  switch (which) {
    case 0: src = c->G[d]; cnt = 2 * N * N; break;
    case 1: src = c->H[d]; cnt = 2 * N * N; break;
    case 2: src = c->dG[d]; cnt = 4 * N * N; break;
    case 3: src = c->dH[d]; cnt = 4 * N * N; break;
    case 4: src = c->dF[d]; cnt = 3 * N; break;
    default: break;
  }
  if (!src) { snprintf(c->err, sizeof(c->err), "matrix %d of domain %d is not kept", which, d); return -2; }
  CK(cudaMemcpyAsync(dst, src, cnt * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "get matrix");
  CK(cudaStreamSynchronize(c->stream), "get matrix");
  return 0;
}

static int ensure_force_targets(bemgpu_ctx *c);
static int ensure_centres(bemgpu_ctx *c);
static bem_dom_dev dom_view(bemgpu_ctx *c, int d);

extern "C" int bemgpu_force(bemgpu_ctx *c, int type, const double *rc, double *F, double *N) {
  if (!c->loaded) { snprintf(c->err, sizeof(c->err), "no problem loaded"); return -2; }
  CK(cudaMemcpyAsync(c->rc_d, rc, 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream), "rc");
  if (type == 0) {
    const int *ctr = nullptr;
    if (c->dom_tri[0]) {
      // boundary values at the centres of the domain-0 triangles (lit_force_4p's 4th point)
      if (ensure_centres(c)) return -1;
      bem_dom_dev D = dom_view(c, 0);
      if (bem_launch_bdval(&D, &c->qp, 1, c->k0[0], 0, c->nctr, c->ctr_t, c->ctr_ze, c->P[0], c->dP[0], c->pv[0],
                           c->dpv[0], c->ctr_bdv, c->status, c->stream))
        return fail(c, "force", cudaGetLastError());
      ctr = c->ctr_idx;
    }
    if (bem_launch_force0(&c->sys, c->P[0], c->pv[0], c->rc_d, c->c0[0], c->rho0[0], ctr, c->ctr_bdv, c->pw_d, c->fout,
                          c->stream))
      return fail(c, "force", cudaGetLastError());
  } else {
    // boundary values at the rule points of every domain-0 element, then the stress integral
    if (ensure_force_targets(c)) return -1;
    bem_dom_dev D = dom_view(c, 0);
    if (bem_launch_bdval(&D, &c->qp, 1, c->k0[0], 1, c->ntgt, c->tgt_t, c->tgt_ze, c->P[0], c->dP[0], c->pv[0], c->dpv[0], c->bdv,
                         c->status, c->stream) ||
        bem_launch_force_bd(&D, c->ntgt, c->tgt_t, c->tgt_ze, c->tgt_w, c->bdv, c->pw_d, c->k2[0], c->k2[1], c->rc_d,
                            c->c0[0], c->rho0[0], c->fout, c->stream))
      return fail(c, "force", cudaGetLastError());
  }
  double out[6];
  CK(cudaMemcpyAsync(out, c->fout, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "force");
  CK(cudaStreamSynchronize(c->stream), "force");
  for (int i = 0; i < 3; ++i) { F[i] = out[i]; N[i] = out[3 + i]; }
  return 0;
}

static bem_dom_dev dom_view(bemgpu_ctx *c, int d) {
  bem_dom_dev D;
  D.ne = c->dom_ne[d];
  D.sid = c->sid + c->dom_off[d];
  D.cr = c->cr; D.cw = c->cw; D.ren = c->ren; D.plane = c->plane; D.wen = c->wen;
  D.npe = c->npe;
  D.has_tri = c->dom_tri[d];
  D.far_rule = c->far_rule;
  D.near_cap = BEM_MAXNEAR_H;
  return D;
}

extern "C" int bemgpu_set_solution(bemgpu_ctx *c, int d, const double *P, const double *dP, const double *pv,
                                   const double *dpv) {
  if (!c->loaded || d < 0 || d > c->MN) { snprintf(c->err, sizeof(c->err), "bad domain"); return -2; }
  const size_t N = 4 * (size_t)c->dom_ne[d];
  CK(cudaMemcpyAsync(c->P[d], P, 2 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream), "P");
  CK(cudaMemcpyAsync(c->dP[d], dP, 2 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream), "dP");
  CK(cudaMemcpyAsync(c->pv[d], pv, 6 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream), "pv");
  CK(cudaMemcpyAsync(c->dpv[d], dpv, 6 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream), "dpv");
  CK(cudaStreamSynchronize(c->stream), "set solution");
  return 0;
}

// room for n points of the point evaluators (inputs: 3 doubles + 1 int each, outputs: 18 doubles)
static int ensure_points(bemgpu_ctx *c, int n) {
  if ((size_t)n <= c->pt_cap) return 0;
  dfree(c->pt_in); dfree(c->pt_out); dfree(c->pt_t);
  c->pt_cap = 0;
  size_t cap = 256;
  while (cap < (size_t)n) cap *= 2;
  CK(dalloc(&c->pt_in, 3 * cap), "point buffers");
  CK(dalloc(&c->pt_out, 18 * cap), "point buffers");
  CK(dalloc(&c->pt_t, cap), "point buffers");
  c->pt_cap = cap;
  return 0;
}

extern "C" int bemgpu_field(bemgpu_ctx *c, int d, int type, int n, const double *r, double *out) {
  if (!c->loaded || d < 0 || d > c->MN) { snprintf(c->err, sizeof(c->err), "bad domain %d", d); return -2; }
  const int grad = !(type & BEMGPU_FIELD_POTENTIAL);
  type &= ~BEMGPU_FIELD_POTENTIAL;
  if (type < 0 || type > 3) { snprintf(c->err, sizeof(c->err), "field rule type %d not available (0..3)", type); return -2; }
  if (n <= 0) return 0;
  if (ensure_points(c, n)) return -1;
  bem_dom_dev D = dom_view(c, d);
  CK(cudaMemcpyAsync(c->pt_in, r, 3 * sizeof(double) * n, cudaMemcpyHostToDevice, c->stream), "field points");
  if (bem_launch_field(&D, &c->qp, d == 0, grad, c->k0[d], type, n, c->pt_in, c->P[d], c->dP[d], c->pv[d], c->dpv[d],
                       c->pt_out, c->status, c->stream))
    return fail(c, "field", cudaGetLastError());
  CK(cudaMemcpyAsync(out, c->pt_out, 18 * sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream), "field");
  CK(cudaStreamSynchronize(c->stream), "field");
  return 0;
}

extern "C" int bemgpu_boundary_field(bemgpu_ctx *c, int d, int type, int n, const int *t, const double *ze,
                                     double *out) {
  if (!c->loaded || d < 0 || d > c->MN) { snprintf(c->err, sizeof(c->err), "bad domain %d", d); return -2; }
  if (type < 0 || type > 3) { snprintf(c->err, sizeof(c->err), "rule type %d not available (0..3)", type); return -2; }
  if (n <= 0) return 0;
  for (int i = 0; i < n; ++i)
    if (t[i] < 0 || t[i] >= c->dom_ne[d]) {
      snprintf(c->err, sizeof(c->err), "element %d is not in domain %d (0..%d)", t[i], d, c->dom_ne[d] - 1);
      return -2;
    }
  if (ensure_points(c, n)) return -1;
  bem_dom_dev D = dom_view(c, d);
  CK(cudaMemcpyAsync(c->pt_t, t, sizeof(int) * n, cudaMemcpyHostToDevice, c->stream), "targets");
  CK(cudaMemcpyAsync(c->pt_in, ze, 2 * sizeof(double) * n, cudaMemcpyHostToDevice, c->stream), "targets");
  if (bem_launch_bdval(&D, &c->qp, d == 0, c->k0[d], type, n, c->pt_t, c->pt_in, c->P[d], c->dP[d], c->pv[d],
                       c->dpv[d], c->pt_out, c->status, c->stream))
    return fail(c, "boundary field", cudaGetLastError());
  CK(cudaMemcpyAsync(out, c->pt_out, 9 * sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream), "boundary field");
  CK(cudaStreamSynchronize(c->stream), "boundary field");
  return 0;
}

// centres of the domain-0 triangles: targets (t, 0, 0) and the element -> target map
static int ensure_centres(bemgpu_ctx *c) {
  if (c->nctr) return 0;
  const int ne = c->dom_ne[0];
  std::vector<int> sid(ne), npe(c->Ne), t, idx(ne, -1);
  CK(cudaMemcpy(sid.data(), c->sid, sizeof(int) * ne, cudaMemcpyDeviceToHost), "centres");
  CK(cudaMemcpy(npe.data(), c->npe, sizeof(int) * c->Ne, cudaMemcpyDeviceToHost), "centres");
  for (int s = 0; s < ne; ++s)
    if (npe[abs(sid[s]) - 1] == 3) { idx[s] = (int)t.size(); t.push_back(s); }
  std::vector<double> ze(2 * t.size(), 0.0);
  if (t.empty()) return 0;
  if (upload(c, &c->ctr_t, t.data(), t.size(), "centres") || upload(c, &c->ctr_idx, idx.data(), idx.size(), "centres") ||
      upload(c, &c->ctr_ze, ze.data(), ze.size(), "centres"))
    return -1;
  CK(falloc(c, &c->ctr_bdv, 9 * t.size()), "centres");
  c->nctr = (int)t.size();
  return 0;
}

// targets of the type-1 force rule: the 9 rule points of every domain-0 quad
// (bil_force_9p) and the 7 of every triangle (lit_force_7p, whose element sum
// is halved: the weight carries the 1/2)
static int ensure_force_targets(bemgpu_ctx *c) {
  if (c->ntgt) return 0;
  const int ne = c->dom_ne[0];
  const double b = 0.7745966692414833770359, w0 = 25.0 / 81.0, w1 = 40.0 / 81.0, w2 = 64.0 / 81.0;
  const double z9[9] = {-b, b, b, -b, 0.0, b, 0.0, -b, 0.0}, e9[9] = {-b, -b, b, b, -b, 0.0, b, 0.0, 0.0};
  const double w9[9] = {w0, w0, w0, w0, w1, w1, w1, w1, w2};
  const double n0 = 0.3480702390148154917985, n1 = 0.2052130961576726346557;
  const double n2 = 0.6028753385763033130539, n3 = 0.3554395089236065568357;
  const double v0 = 0.1259391805448271525957, v1 = 0.1323941527885061807376, v2 = 0.225;
  const double z7[7] = {-n0, 2.0 * n0, -n0, n1, -2.0 * n1, n1, 0.0}, e7[7] = {-n2, 0.0, n2, n3, 0.0, -n3, 0.0};
  const double w7[7] = {v0, v0, v0, v1, v1, v1, v2};
  std::vector<int> sid(ne), npe(c->Ne);
  CK(cudaMemcpy(sid.data(), c->sid, sizeof(int) * ne, cudaMemcpyDeviceToHost), "targets");
  CK(cudaMemcpy(npe.data(), c->npe, sizeof(int) * c->Ne, cudaMemcpyDeviceToHost), "targets");
  std::vector<int> t;
  std::vector<double> ze, w;
  for (int s = 0; s < ne; ++s) {
    const bool tri = npe[abs(sid[s]) - 1] == 3;
    for (int i = 0; i < (tri ? 7 : 9); ++i) {
      t.push_back(s);
      ze.push_back(tri ? z7[i] : z9[i]);
      ze.push_back(tri ? e7[i] : e9[i]);
      w.push_back(tri ? 0.5 * w7[i] : w9[i]);
    }
  }
  const int n = (int)t.size();
  if (upload(c, &c->tgt_t, t.data(), t.size(), "targets") || upload(c, &c->tgt_ze, ze.data(), ze.size(), "targets") ||
      upload(c, &c->tgt_w, w.data(), w.size(), "targets"))
    return -1;
  CK(falloc(c, &c->bdv, 9 * (size_t)n), "boundary values");
  c->ntgt = n;
  return 0;
}

// ---------------------------------------------------------------- point evaluators
extern "C" int bemgpu_faddeeva_w(const double *z, int n, double *w) {
  if (n <= 0) return 0;
  if (ensure_constants(nullptr, nullptr, nullptr, nullptr, nullptr) != 0) return -1;
  double *dz = nullptr, *dw = nullptr;
  if (cudaMalloc(&dz, 2 * sizeof(double) * n) != cudaSuccess) return -1;
  if (cudaMalloc(&dw, 2 * sizeof(double) * n) != cudaSuccess) { cudaFree(dz); return -1; }
  cudaMemcpy(dz, z, 2 * sizeof(double) * n, cudaMemcpyHostToDevice);
  int r = bem_launch_faddeeva(dz, n, dw, 0);
  if (r == 0 && cudaMemcpy(w, dw, 2 * sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess) r = -1;
  cudaFree(dz);
  cudaFree(dw);
  return r;
}

extern "C" int bemgpu_qpgf(const double *qpar, const double *r, int n, double *G, double *dG, int *ret) {
  if (n <= 0) return 0;
  if (ensure_constants(nullptr, nullptr, nullptr, nullptr, nullptr) != 0) return -1;
  bem_qp q;
  bem_qp_prepare(qpar, &q);
  double *wt = nullptr;
  if (cudaMalloc(&wt, BEM_WT_SIZE * sizeof(double)) != cudaSuccess) return -1;
  if (bem_launch_wtab(q.k, q.eta_run, wt, 0) != 0) { cudaFree(wt); return -1; }
  q.wt = wt;
  q.wt_h = BEM_WT_H;
  q.wt_n = BEM_WT_N;
  // evanescent order table reaching the points' |z|
  double zmax = 0.0;
  for (int i = 0; i < n; ++i) zmax = fabs(r[3 * i + 2]) > zmax ? fabs(r[3 * i + 2]) : zmax;
  double *stb = nullptr;
  const size_t scnt = stab_window(&q, 2.0 * zmax);
  if (scnt) {
    if (cudaMalloc(&stb, scnt * sizeof(double)) != cudaSuccess) { cudaFree(wt); return -1; }
    if (bem_launch_stab(&q, stb, 0) != 0) { cudaFree(wt); cudaFree(stb); return -1; }
    q.st = stb;
  }
  double *dr = nullptr, *dg = nullptr, *ddg = nullptr;
  int *dret = nullptr;
  int rc = -1;
  if (cudaMalloc(&dr, 3 * sizeof(double) * n) == cudaSuccess && cudaMalloc(&dg, 2 * sizeof(double) * n) == cudaSuccess &&
      cudaMalloc(&ddg, 6 * sizeof(double) * n) == cudaSuccess && cudaMalloc(&dret, sizeof(int) * n) == cudaSuccess) {
    cudaMemcpy(dr, r, 3 * sizeof(double) * n, cudaMemcpyHostToDevice);
    rc = bem_launch_qpgf(&q, dr, n, dg, ddg, dret, 0);
    if (rc == 0) {
      if (cudaMemcpy(G, dg, 2 * sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMemcpy(dG, ddg, 6 * sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMemcpy(ret, dret, sizeof(int) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = -1;
    }
  }
  cudaFree(dr); cudaFree(dg); cudaFree(ddg); cudaFree(dret); cudaFree(wt); cudaFree(stb);
  return rc;
}

extern "C" int bemgpu_zgesv(int device, int n, int nrhs, const double *A, double *B) {
  if (n <= 0 || nrhs < 1 || nrhs > 4) return -2;
  if (cudaSetDevice(device) != cudaSuccess) return -1;
  bem_lu w;
  if (bem_lu_init(&w, device)) return -1;
  cudaStream_t st = nullptr;
  double *dA = nullptr, *dB = nullptr;
  int rc = -1;
  const size_t an = 2 * (size_t)n * n * sizeof(double), bn = 2 * (size_t)n * nrhs * sizeof(double);
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess && cudaMalloc(&dA, an) == cudaSuccess &&
      cudaMalloc(&dB, bn) == cudaSuccess && cudaMemcpyAsync(dA, A, an, cudaMemcpyHostToDevice, st) == cudaSuccess &&
      cudaMemcpyAsync(dB, B, bn, cudaMemcpyHostToDevice, st) == cudaSuccess && bem_lu_factor_z(&w, dA, n, st) == 0 &&
      bem_lu_solve_z(&w, dA, n, nrhs, dB, st) == 0 &&
      cudaMemcpyAsync(B, dB, bn, cudaMemcpyDeviceToHost, st) == cudaSuccess) {
    const unsigned s = bem_lu_status(&w, st);
    rc = s == 0 ? 0 : (s & BEM_LU_ST_ZERO) ? -3 : -1;
  }
  if (st) cudaStreamSynchronize(st);
  cudaFree(dA);
  cudaFree(dB);
  bem_lu_free(&w);
  if (st) cudaStreamDestroy(st);
  return rc;
}

extern "C" long long bemgpu_interior_reuses(bemgpu_ctx *c) { return c ? c->int_reused_loads : -1; }

extern "C" int bemgpu_set_interior_derivatives(bemgpu_ctx *c, int keep, int block_rows) {
  if (!c || block_rows < 0) return -2;
  c->dgh_keep_req = keep != 0;
  c->dgh_rows_req = block_rows;
  return 0;
}

extern "C" int bemgpu_set_interior_reuse(bemgpu_ctx *c, int on) {
  if (!c) return -2;
  c->int_reuse_on = on != 0;
  if (!c->int_reuse_on) {
    // the next load assembles and factors every domain
    c->int_valid = false;
    c->int_reuse = false;
    c->int_data.clear();
  }
  return 0;
}

static std::atomic<unsigned long long> g_launches{0};
extern "C" void bem_count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
extern "C" unsigned long long bemgpu_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

extern "C" cudaError_t bem_launch_transform(int ne, const double *rv, double th, const double *tv, double *cr,
                                            double *cw, double *ren, double *wen, double *Pi, double *dPi,
                                            double *p_inc, double *v_inc, const double *pw_d, const double *k2,
                                            cudaStream_t st);

extern "C" int bemgpu_transform_mesh(bemgpu_ctx *c, const double *rv, double th, const double *tv) {
  if (!c->bat.empty()) { snprintf(c->err, sizeof(c->err), "a batch is loaded (load a single problem first)"); return -2; }
  if (!c->loaded) { snprintf(c->err, sizeof(c->err), "no problem loaded"); return -2; }
  CK(bem_launch_transform(c->Ne, rv, th, tv, c->cr, c->cw, c->ren, c->wen, c->Pi, c->dPi, c->p_inc, c->v_inc,
                          c->pw_d, c->k2.data(), c->stream),
     "mesh transform");
  // the z extent of the moved mesh sets the spectral table's window
  std::vector<double> cr(12 * (size_t)c->Ne);
  CK(cudaMemcpyAsync(cr.data(), c->cr, cr.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "mesh transform");
  CK(cudaStreamSynchronize(c->stream), "mesh transform");
  double zlo = 0.0, zhi = 0.0;
  for (int e = 0; e < c->Ne; ++e) {
    const double *z = cr.data() + (size_t)e * 12 + 8;
    const double hw = fabs(z[1]) + fabs(z[2]) + fabs(z[3]);
    if (e == 0 || z[0] - hw < zlo) zlo = z[0] - hw;
    if (e == 0 || z[0] + hw > zhi) zhi = z[0] + hw;
  }
  c->zspan = zhi - zlo;
  if (build_stab(c)) return -1;
  // every matrix and factor belongs to the old placement
  c->factored = false;
  c->int_valid = false;
  c->int_data.clear();
  for (int d = 0; d < BEMGPU_MAXDOM; ++d) c->int_factored[d] = false;
  return 0;
}

extern "C" int bemgpu_set_refinement(bemgpu_ctx *c, int method) {
  if (method < 0 || method > 2) { snprintf(c->err, sizeof(c->err), "refinement method %d (0..2)", method); return -2; }
  c->refine = method;
  return 0;
}

extern "C" int bemgpu_refinement_used(bemgpu_ctx *c, int *gmres, int max) {
  int k = 0;
  for (; k < c->st_n && k < max; ++k) gmres[k] = c->st_gmres[k];
  return k;
}
