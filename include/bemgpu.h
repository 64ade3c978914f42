/* bemgpu.h -- C ABI of the B200 boundary-element engine.
 *
 * Plain C types only (pointers, sizes, doubles as interleaved re/im pairs);
 * no CUDA or PyTorch types.  Every entry point returns 0 on success and a
 * negative code on failure; bemgpu_error() gives the message.  Device faults
 * are never used as an error channel: kernels write status bits
 * (BEMGPU_ST_*) that the host turns into an error return.
 *
 * These entry points replace the compute inside the reference's drop-in API
 * (d3qd2_src/bem3_aw_qd2.h); the host library in bem3_aw_qd2_b200/csrc/host
 * calls them from its re-implementation of that API, so the reference's
 * drivers (aw_d3qd2_bv_solver.c, example1.c) link against it unchanged.
 */
#ifndef BEMGPU_H
#define BEMGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BEMGPU_ST_QPGF_LIMIT    0x01 /* a lattice sum reached its term limit (d3_qpgf_d2.c error -1/-2) */
#define BEMGPU_ST_RAYLEIGH      0x02 /* beta_n == 0: Rayleigh anomaly (d3_qpgf_d2.c:882, 2006) */
#define BEMGPU_ST_NEAR_OVERFLOW 0x04 /* > 64 near-singular sources for one collocation node */
#define BEMGPU_ST_NONFINITE     0x08 /* non-finite coefficient */
#define BEMGPU_ST_GEOMETRY      0x10 /* negative polar radius in a singular integral */
#define BEMGPU_ST_SOLVE         0x20 /* singular matrix in an LU factorisation */

/* The boundary-value problem, in the reference's element-table form
 * (AQD2/BOUD, d3qd2_src/d3qd2_elem.h:13-65).  Element e (0-based) is the
 * reference's element id e+1.  Complex numbers are (re, im) pairs. */
typedef struct bemgpu_problem {
  int Ne;              /* elements */
  int NN;              /* element nodes, sum of nodes per element */
  int MN;              /* media; domains are 0 (host, open) .. MN; MN <= 7 */
  int ps;              /* 1: quasi-periodic host domain (the only mode implemented) */
  double qp[8];        /* QPD2: k, kx, ky, kz, d1x, d1y, d2x, d2y */
  const double *cr;    /* [Ne][3][4] element geometry constants */
  const double *cw;    /* [Ne][3][3] normal-vector constants */
  const double *ren;   /* [Ne][4][3] collocation nodes */
  const double *wen;   /* [Ne][4][3] normal (Jacobian) vectors at the nodes */
  const int *npe;      /* [Ne] nodes per element (4: bilinear quad) */
  const int *eni;      /* [Ne][4] element node ids 0..NN-1 */
  const int *md;       /* [Ne] main domain */
  const int *sd;       /* [Ne] sub domain */
  const int *dom_ne;   /* [MN+1] elements bordering each domain */
  const int *sid;      /* signed element ids (1-based) of domain 0, then 1, ... */
  const double *k0;    /* [MN+1] wave numbers */
  const double *k2;    /* [MN+1] complex i omega rho */
  const double *rho0;  /* [MN+1] densities */
  const double *c0;    /* [MN+1] sound speeds */
  const double *Pi;    /* [Ne][4] complex incident potential at the nodes (init_boundary_data) */
  const double *dPi;   /* [Ne][4] complex normal derivative of Pi */
  const double *p_inc; /* [Ne][4] complex incident pressure at the nodes */
  const double *v_inc; /* [Ne][4][3] complex incident particle velocity at the nodes */
  const double *xl, *wl; /* 12-point Gauss-Legendre nodes/weights on [-1,1] (BOUD xli/wli) */
  const double *xh, *wh; /* 64-point Gauss-Legendre nodes/weights (BOUD xhi/whi) */
  const unsigned char *plane; /* [Ne] 1 if the element is plane (bil_check_plane, d3qd2_elem.c:986) */
  double pw[16];       /* incident plane wave: amplitude (re, im), rotation R[9], translation tv[3],
                          k0, rho0 c0 (Apw, aw_pw.h:16-34; evaluated as calc_apw_pv) */
} bemgpu_problem;

typedef struct bemgpu_ctx bemgpu_ctx;

/* Context on one CUDA device; stream may be NULL (a private stream is made). */
int bemgpu_create(int device, void *stream, bemgpu_ctx **out);
void bemgpu_destroy(bemgpu_ctx *ctx);
const char *bemgpu_error(const bemgpu_ctx *ctx);
unsigned bemgpu_status(bemgpu_ctx *ctx); /* BEMGPU_ST_* bits accumulated since load */

/* Copy a problem from host memory to the device (replaces the state that
 * read_aqd2/initialize_aqd2 build, bem3_aw_qd2.c:3-109).  Device buffers of a
 * previously loaded problem that are large enough are reused (no free and
 * allocate per load); bemgpu_unload gives them back. */
int bemgpu_load(bemgpu_ctx *ctx, const bemgpu_problem *prob);

/* Ewald splitting parameter used off the lattice plane: eta0 x scale, where
 * eta0 is the reference's (d3_qpgf_d2.c:1683-1693; the per-point cap still
 * applies).  Both lattice sums converge to the reference's 1e-15 tolerance for
 * any scale, so the results agree to round-off while the split of the terms
 * between the real-space and spectral sums, and so the cost, changes.  On the
 * lattice plane (z = 0) eta0 is always used.  scale = BEMGPU_EWALD_RULE (0,
 * the default): each loaded problem's scale by rule, the largest for which
 * k^2 eta^2 stays below the cap (0.98 sqrt(3) / (k eta0), clamped to
 * [0.5, 1.3]; points past the cap would need their own parameter and miss the
 * per-problem term tables); a scale in [0.25, 4] is used for every problem
 * loaded until changed. */
#define BEMGPU_EWALD_RULE 0.0
int bemgpu_set_ewald_scale(bemgpu_ctx *ctx, double scale);

/* Quadrature of the regular pairs of the periodic domain (no counterpart in
 * the reference, which uses its 12 x 12 Gauss rule for every regular pair,
 * on each of 3 parts of a triangle): on = 1 (the default) uses a shorter
 * n x n rule (Gauss on a quad, collapsed over a whole triangle) where the
 * source element's centre is at least d circumradii R from the nearest
 * lattice image of the collocation node:
 *     n = 10 from d = 3, 9 from 3.5, 8 from 5 (all with k R <= 1),
 *     7 from 8 (k R <= 0.5), 6 from 25 (k R <= 0.2);
 *     on triangles 7 from 6 and 6 from 12 (k R <= 0.5);
 * the 10, 9, 7 and 6-point rules only on quads whose twist along the normal
 * is at most a tenth of the shorter half-side and whose half-sides are within
 * 3x (every triangle).  Each reproduces the reference's integrals to about
 * 1e-13 of the pair's largest entry with up to 4 (quads) or 12 (triangles)
 * times fewer Green's-function values; on = 0 keeps the reference's rules
 * everywhere.  Applies from the next assembly. */
int bemgpu_set_far_rule(bemgpu_ctx *ctx, int on);
/* Regular pairs of the periodic domain by rule in the last assembly:
 * counts[0] on the reference's 12 x 12 rule, counts[1 .. 5] on the 10, 9, 8,
 * 7 and 6-point rules.  Returns 0, or -2 when the assembly kept no pair
 * lists (no counts; domains of more than 32768 elements). */
int bemgpu_rule_pairs(bemgpu_ctx *ctx, unsigned long long counts[6]);

/* Autotuner of the Ewald parameter for the loaded problem: times the periodic
 * regular-pair kernel on an eighth of the pairs for the rule's scale and three
 * neighbours and sets the fastest (bemgpu_set_ewald_scale); *best_scale gets it.
 * Costs about half of one regular-pair launch. */
int bemgpu_autotune(bemgpu_ctx *ctx, double *best_scale);

/* Batches of Bloch vectors (form 2; no counterpart in the reference, which
 * assembles every problem on its own): nb problems on one body, media,
 * lattice and frequency that differ only in the incidence (in-plane Bloch
 * wave vector and incident field).  bemgpu_batch_load checks that, loads
 * probs[0] as bemgpu_load does and keeps every instance's Ewald parameters
 * (its own spectral table) and incident data, with device room for its
 * periodic-domain G and H (32 N_0^2 bytes each, kept for the next batch); quad
 * meshes of at most 32768 elements.  bemgpu_batch_assemble assembles the
 * free-space domains once and the periodic domain of all instances with each
 * kernel launched once per 8 instances (one classification and one set of
 * pair lists; the regular-pair kernels stride over the lists instance after
 * instance, the near-singular and self kernels take the instance from the
 * grid).  bemgpu_batch_select(ctx, b) makes
 * instance b the context's problem: bemgpu_solve, bemgpu_force,
 * bemgpu_get_solution, bemgpu_get_matrix and the field functions then act on
 * it (the interior domains' dpv factors made by the first solve serve every
 * instance).  Results equal those of loading and running each problem alone
 * (same kernels and order of sums).  The batch ends at the next load; the
 * Ewald scale, the autotuner and mesh transforms are refused while it is
 * loaded.  Returns 0, -2 for bad input, -1 on a CUDA error. */
int bemgpu_batch_load(bemgpu_ctx *ctx, int nb, const bemgpu_problem *const *probs);
int bemgpu_batch_assemble(bemgpu_ctx *ctx);
int bemgpu_batch_select(bemgpu_ctx *ctx, int b);

/* Interior-domain reuse (no counterpart in the reference, which assembles
 * every domain for every solve): the free-space domains' matrices (G, H, dG,
 * dH, dF of domains >= 1, create_cmatrix_domain with did >= 1,
 * bem3_aw_qd2_solve_bieq.c:133-218) and their dpv factors depend only on the
 * mesh, the media and the frequency.  bemgpu_load compares the new problem's
 * element tables, domain lists and interior wave numbers with the previous
 * load's; when they are the same (a new in-plane Bloch wave vector or
 * incident field on the same body at the same frequency) the context keeps
 * those matrices and factors and the next bemgpu_assemble / bemgpu_solve skip
 * them.  Returns the number of loads that did so. */
long long bemgpu_interior_reuses(bemgpu_ctx *ctx);
/* Interior-domain reuse on (1, the default) or off (0: every load assembles
 * and factors every domain, as the reference does). */
int bemgpu_set_interior_reuse(bemgpu_ctx *ctx, int on);

/* Interior-domain derivative rows (no counterpart in the reference, which
 * keeps them: dG, dH of create_cmatrix_domain with did >= 1,
 * bem3_aw_qd2_solve_bieq.c:133-218, used by dpdt_fcm in q_solve_pv_bv,
 * :516-530, 655-750).  keep = 1 (default): dG and dH (2N x N complex each)
 * stay on the device after the assembly.  keep = 0: they are not stored; the
 * particle-velocity step recomputes them a block of rows at a time (about
 * 256 MiB each) and contracts each block with P and dP at once.  This saves
 * 64 N^2 bytes per interior domain (38.7 GB at N = 24576) for one more
 * free-space integration per solve.  Takes effect at the next bemgpu_load;
 * bemgpu_get_matrix then has no dG, dH (which = 2, 3) to return.  block_rows
 * (keep = 0 only): rows recomputed at a time, rounded down to a multiple of 4;
 * 0 chooses the 256 MiB block.  The request server chooses keep = 0 for a
 * request that does not fit its device-memory budget otherwise. */
int bemgpu_set_interior_derivatives(bemgpu_ctx *ctx, int keep, int block_rows);

/* Kernel launches of this library in this process so far, all contexts and
 * threads (no counterpart in the reference): every launch counts one, a
 * replay of a captured factorisation counts its kernels. */
unsigned long long bemgpu_kernel_launches(void);

/* Rotation and translation of the loaded body on the device (the
 * reference's Rodrigues options of read_aqd2, bem3_aw_qd2.c:16-24, 395-422:
 * rotation about the axis rv[3] by th radians, then translation by tv[3]),
 * for requests that differ from a resident problem only in the body's
 * placement: the element constants, collocation nodes and normals are turned
 * and moved, and the incident field at the new nodes is evaluated on the
 * device (init_boundary_data, bem3_aw_qd2.c:1104-1146), so nothing is
 * uploaded again.  The lattice and the incident wave stay.  The next
 * bemgpu_run assembles and solves the moved body.  Transforms compose: each
 * applies to the current placement.  A host AQD2 the problem came from is not
 * changed. */
int bemgpu_transform_mesh(bemgpu_ctx *ctx, const double *rv, double th, const double *tv);

/* Free the loaded problem's device memory (the context stays usable). */
int bemgpu_unload(bemgpu_ctx *ctx);

/* Coefficient matrices of every domain (create_cmatrix,
 * bem3_aw_qd2_solve_bieq.c:124-218). */
int bemgpu_assemble(bemgpu_ctx *ctx);

/* Global system, LU solve, P/dP, pv, dpv (bem3_aw_qd2_solve_bieq.c:220-750). */
int bemgpu_solve(bemgpu_ctx *ctx);

/* Factorisation reuse: replace the incident field (same layouts as
 * bemgpu_problem: Pi, dPi, p_inc [Ne][4] complex, v_inc [Ne][4][3] complex,
 * pw[16]) and solve again with the factors of the last bemgpu_solve; only the
 * right-hand side changes (same mesh, media, frequency and in-plane Bloch
 * wave vector: the matrices are those of init_boundary_data's new incident
 * field, bem3_aw_qd2.c:1104-1146).  bemgpu_solve_rhs returns -2 when no
 * factorisation of the current matrices is held (after bemgpu_load,
 * bemgpu_assemble or bemgpu_set_precision). */
int bemgpu_set_incident(bemgpu_ctx *ctx, const double *Pi, const double *dPi, const double *p_inc, const double *v_inc,
                        const double *pw);
int bemgpu_solve_rhs(bemgpu_ctx *ctx);

/* solve_bieq_aqd2 (bem3_aw_qd2_solve_bieq.c:3): assemble + solve. */
int bemgpu_run(bemgpu_ctx *ctx);

/* Boundary values of domain d to host arrays: P, dP [Ne_d][4] complex,
 * pv, dpv [Ne_d][4][3] complex (SUBD, d3qd2_elem.h:13-19). */
int bemgpu_get_solution(bemgpu_ctx *ctx, int d, double *P, double *dP, double *pv, double *dpv);

/* Coefficient matrix of domain d to a host array, in the layout of the
 * reference's temporary files (bem3_aw_qd2_solve_bieq.c:176-182):
 * which 0: G [N][N] complex, 1: H, 2: dG [2N][N] complex, 3: dH, 4: dF [N][3] real. */
int bemgpu_get_matrix(bemgpu_ctx *ctx, int d, int which, double *dst);

/* Radiation force and torque about rc (force_FN_aqd2, bem3_aw_qd2_force.c:4).
 * type 0: 4-point rule on the node values (bil_force_4p); type != 0: the
 * 9-point rule with the boundary values evaluated at the rule points
 * (bil_force_9p + pv_t_bd_aqd2 with the 9-point coefficients). */
int bemgpu_force(bemgpu_ctx *ctx, int type, const double *rc, double *F, double *N);

/* Replace the boundary values of domain d (same layout as
 * bemgpu_get_solution), e.g. after reading a .dat file, so that the force and
 * field functions can run without a new solve. */
int bemgpu_set_solution(bemgpu_ctx *ctx, int d, const double *P, const double *dP, const double *pv, const double *dpv);

/* Field sums at n points r[n][3] of domain d, already reduced to the home
 * lattice cell (pv_s_dbieq_aqd2 / pv_s_bieq_aqd2 / phi_s_aqd2,
 * bem3_aw_qd2_field.c:3-297).  type: 0 4-point, 1 9-point, 2 12x12, 3 64x64
 * rule.  out[n][18] = S0 (complex) = sum(G dP - H P), S1[3] (complex) its
 * gradient with respect to r, F, dF[3], S2[3] (complex) = sum(G dpv - H pv);
 * the caller applies the normalisation 1/(1+F) (domain 0) or 1/F.
 * type | BEMGPU_FIELD_POTENTIAL: S0, S2 and F alone (S1, dF zero), with the
 * first-derivative Green's function as phi_s_aqd2 and pv_s_bieq_aqd2 use it
 * (q0_coef_rt, d3qd2_elem.c:574); without the flag the sums use the
 * second-derivative one as pv_s_dbieq_aqd2 does (q0_dcoef_rt_grad, :650). */
#define BEMGPU_FIELD_POTENTIAL 0x100
int bemgpu_field(bemgpu_ctx *ctx, int d, int type, int n, const double *r, double *out);

/* Boundary sums of domain d at parameter points ze[n][2] = (zeta, eta) of its
 * elements t[n] (0-based index into domain d's element list; the reference's
 * t - 1): out[n][9] = S0 (complex) = sum(G dP - H P), S2[3] (complex) =
 * sum(G dpv - H pv), F (pv_s_bd_aqd2, bem3_aw_qd2_field.c:394-433, with
 * q0_coef_bd for domain 0 and coef_bd for the others); the caller applies the
 * normalisation.  type as bemgpu_field; the element itself always gets the
 * singular polar rule. */
int bemgpu_boundary_field(bemgpu_ctx *ctx, int d, int type, int n, const int *t, const double *ze, double *out);

/* Precision of the dense solves (the global system and the per-domain dpv
 * systems; the reference uses FP64 PARDISO and LAPACKE_zgesv,
 * d3qd2_mkl_solver.c:18-148, bem3_aw_qd2_solve_bieq.c:533-653).  Assembly,
 * residuals and the force integral stay FP64 in every mode.
 *   0 BEMGPU_FP64      FP64 LU (default; the drop-in)
 *   1 BEMGPU_MIXED_FP32   complex FP32 LU, FP32 CUDA-core trailing updates
 *   2 BEMGPU_MIXED_TF32   complex FP32 LU, trailing updates as one TF32
 *                         product on the tensor cores (tcgen05)
 *   3 BEMGPU_MIXED_TF32X3 complex FP32 LU, trailing updates as three split
 *                         TF32 products on the tensor cores (FP32-accurate)
 *   4 BEMGPU_MIXED_FAST   a single low-precision tensor-core product: mode 2
 * Modes 1-4 refine in FP64 against the FP64 matrix until the correction is
 * below 1e-15 of the solution; a system that does not get below 1e-12 is
 * solved again in FP64 (reported by bemgpu_solve_stats).  A mode whose
 * tensor-core update this build does not have runs as mode 1;
 * bemgpu_get_precision reports the mode in effect. */
#define BEMGPU_FP64 0
#define BEMGPU_MIXED_FP32 1
#define BEMGPU_MIXED_TF32 2
#define BEMGPU_MIXED_TF32X3 3
#define BEMGPU_MIXED_FAST 4
int bemgpu_set_precision(bemgpu_ctx *ctx, int mode);
/* The mode in effect (see bemgpu_set_precision). */
int bemgpu_get_precision(bemgpu_ctx *ctx);

/* Refinement of the mixed-precision solves (no counterpart in the reference):
 *   0 (default) iterative refinement; a system it does not bring below 1e-12
 *     is solved by GMRES-IR before any FP64 fallback
 *   1 iterative refinement only
 *   2 GMRES-IR only: GMRES(20) on the system preconditioned by the FP32
 *     factors, FP64 residuals and Krylov vectors, to a relative residual of
 *     1e-14 (success: 1e-12)
 * bemgpu_refinement_used gives, per dense system of the last solve, 1 if
 * GMRES-IR ran (bemgpu_solve_stats then reports its Krylov steps and the
 * relative residual ||b - A x|| / ||b||). */
int bemgpu_set_refinement(bemgpu_ctx *ctx, int method);
int bemgpu_refinement_used(bemgpu_ctx *ctx, int *gmres, int max);

/* Refinement record of the last bemgpu_solve, one entry per dense system
 * (0: global system, 1 + d: dpv system of domain d): refinement steps, final
 * max|correction| / max|solution|, 1 if solved again in FP64.  Returns the
 * number of entries written (at most max). */
int bemgpu_solve_stats(bemgpu_ctx *ctx, int *iters, double *rel_corr, int *fallback, int max);

/* Wait for all queued work of the context. */
int bemgpu_sync(bemgpu_ctx *ctx);

/* The CUDA stream (cudaStream_t) all work of the context is queued on. */
void *bemgpu_stream(bemgpu_ctx *ctx);

/* Per-phase device timing (CUDA events on the context's stream). With
 * profiling on, bemgpu_phase_times fills up to max entries (ms) and returns
 * their number: domain 0 classify, regular, near-singular, self, diagonal;
 * domain 1 the same; gather, global LU + solve, boundary values, dpv solves. */
int bemgpu_set_profiling(bemgpu_ctx *ctx, int on);
int bemgpu_phase_times(bemgpu_ctx *ctx, double *ms, int max);

/* Work done by the periodic-domain kernels since load (or the last reset):
 * out6 = lattice terms of regular, near-singular and self pairs, then the
 * number of Green's-function points of each class. */
int bemgpu_work_counters(bemgpu_ctx *ctx, unsigned long long *out6, int reset);

/* Coefficient matrices of one domain without any device allocation.
 *
 * No counterpart in the reference (the reference has no GPU code).  This is
 * for callers that cannot allocate device memory, neither themselves nor
 * through this library: a process whose device memory belongs to another
 * allocator's fixed pool that must not be bypassed, or a caller through a
 * foreign-function interface that can hand over device buffers but has no
 * way to manage CUDA allocations.
 *
 * The caller passes device pointers for every input and output: the element
 * tables cr, cw, ren and plane (laid out as in bemgpu_problem), the domain's
 * signed element ids sid[ne], and the outputs G, H [4 ne][4 ne] complex,
 * dF [4 ne][3], and for an interior domain dG, dH [8 ne][4 ne] complex (may
 * be NULL when periodic = 1).  qp is a host array as bemgpu_problem.qp.
 * periodic = 1: the host domain 0 with the quasi-periodic Green's function
 * (H gets 1 + F on its diagonal); 0: an interior domain in free space with
 * wave number k (H gets F).  The layouts are those of bemgpu_get_matrix.
 * Every element is taken as a bilinear quad (4 nodes); meshes with linear
 * triangles go through bemgpu_load + bemgpu_assemble.  Every regular pair is
 * integrated with the reference's 12 x 12 rule (as a context after
 * bemgpu_set_far_rule(ctx, 0)) and the Ewald parameter is the reference's.
 *
 * The scratch the assembly needs lives in one fixed array inside the library
 * (about 21 MB on every GPU that loads it, kept until the process exits), so
 * a domain may have at most BEMGPU_STATIC_MAX_NE elements; more is rejected
 * with -2 and a message on stderr.  The first call on each device sets the
 * array up (finds its device address, uploads the quadrature tables); make
 * that first call before any stream capture.  Each call checks a marker in
 * device memory and repeats the set-up when the device lost it (a
 * cudaDeviceReset), and looks the array's address up again.  Every call reuses the array and
 * finds the previous call's contents in it (the status word is cleared at
 * the start of each call); calls that overlap on the GPU race on it, so the
 * caller must not run two at once.  The call returns after its work on
 * stream has finished.  Returns 0; -2 size out of range or a required
 * pointer NULL (dG, dH may be NULL only when periodic = 1); -3 device set-up
 * failed; -4 launch or copy failed; -5 a BEMGPU_ST_* status bit was set. */
#define BEMGPU_STATIC_MAX_NE 1536
int bemgpu_assemble_domain_static(const double *cr, const double *cw, const double *ren, const unsigned char *plane,
                                  const int *sid, int ne, const double *qp, int periodic, double k, double *G,
                                  double *H, double *dG, double *dH, double *dF, void *stream);

/* ---- Request server (no counterpart in the reference: there each request
 * is one solve_bieq_aqd2 + force_FN_aqd2 run).
 *
 * Continuous batching on one GPU: submitted requests queue and are admitted
 * to one of `slots` solver slots as slots and device memory free up; each
 * slot has its own CUDA stream and host worker thread, so admitted requests'
 * assemblies and solves overlap on the device.  A slot keeps its problem's
 * matrices and factors: a request whose reuse_key equals an idle slot's (the
 * caller's hash of mesh, media, lattice, frequency and in-plane Bloch wave
 * vector) is routed there and only its right-hand side is solved
 * (bemgpu_set_incident + bemgpu_solve_rhs).  Admission keeps the resident
 * problems' device bytes within hbm_budget (per problem: 16 n^2 for the
 * global matrix, 48 N_d^2 per domain and 64 N_d^2 more for interior domains,
 * 8 n^2 + 8 N_d^2 more in mixed precision, plus tables and 64 MB of solver
 * workspace), evicting idle slots' problems least recently used first; later
 * requests that fit may pass one that does not until it has waited 2 s.
 * The problem's arrays are copied on submit.  Results (radiation force and
 * torque of the given rule about rc) come back through bemgpu_server_poll in
 * completion order. */
typedef struct bemgpu_server bemgpu_server;
typedef struct bemgpu_result {
  long long id;        /* the id given to bemgpu_server_submit */
  int status;          /* 0, or the failing call's return code */
  int reused;          /* 1: solved with a resident factorisation (right-hand side only) */
  int precision;       /* precision the request ran in (a mixed request whose footprint
                          exceeds the budget runs in BEMGPU_FP64 when that fits) */
  double F[3], N[3];   /* force and torque */
  double queue_ms;     /* submit -> admitted to a slot */
  double service_ms;   /* admitted -> result */
  char error[160];
} bemgpu_result;
int bemgpu_server_create(int device, size_t hbm_budget, int slots, bemgpu_server **out);
/* 0 queued; -2 the problem needs more than the whole budget (in FP64 too) */
int bemgpu_server_submit(bemgpu_server *srv, const bemgpu_problem *prob, unsigned long long reuse_key, int precision,
                         int force_type, const double *rc, long long id);
/* Up to max finished results; waits up to timeout_ms for the first one.  Returns the count. */
int bemgpu_server_poll(bemgpu_server *srv, bemgpu_result *out, int max, int timeout_ms);
/* out8: submitted, completed, solved by reuse, running, queued, device bytes resident, peak, evictions */
int bemgpu_server_stats(bemgpu_server *srv, double *out8);
void bemgpu_server_destroy(bemgpu_server *srv);

/* Dense complex solve A X = B on the device (the FP64 factorisation and
 * solves the context uses for the global and dpv systems, bem_lu.cu),
 * replacing LAPACKE_zgesv (solve_dpv_bv, bem3_aw_qd2_solve_bieq.c:617) and
 * the dense PARDISO solve (b_mkl_solver_pardiso_d, d3qd2_mkl_solver.c:18):
 * A row-major n x n complex (host), B column-major n x nrhs complex (host,
 * nrhs <= 4), overwritten by X.  Allocates its own device buffers for the
 * call.  Returns 0; -2 bad size; -3 singular (zero pivot); -1 CUDA error. */
int bemgpu_zgesv(int device, int n, int nrhs, const double *A, double *B);

/* Faddeeva w(z) at n points (host arrays of (re, im) pairs), relative error
 * 1e-15 (Faddeeva_w, qgf2_src/Faddeeva.cc:679, called with MEPS). */
int bemgpu_faddeeva_w(const double *z, int n, double *w);

/* Quasi-periodic Green's function and gradient at n points r[n][3] (host
 * arrays): G[n] complex, dG[n][3] complex, ret[n] = lattice terms used or the
 * reference's negative error code (d3hm_qpgf_d2_v1, qgf2_src/d3_qpgf_d2.c:124). */
int bemgpu_qpgf(const double *qp, const double *r, int n, double *G, double *dG, int *ret);

#ifdef __cplusplus
}
#endif
#endif
