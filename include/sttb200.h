/* sttb200.h -- C ABI of the B200 (sm_100a) matrix-free FEM solve path.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t, returns an
 * int status (STT_OK or an STT_ERR_* code) and retains no pointer past the call, except
 * through the explicit hierarchy handle (stt_hier_*), whose device memory is a
 * caller-owned workspace.  No entry point allocates device memory.
 *
 * Conventions match the reference's tensors: nodes in C order row * (nelx + 1) + col
 * with row 0 at the top, dofs interleaved d * node + i (d = 2 plane stress, d = 1 scalar
 * heat), elements row * nelx + col with local corners BL, BR, TR, TL.  Vectors are
 * batched as rows with an explicit row stride (in elements).  Boundary conditions are a
 * per-node byte of "fixed" flags (bit i set = dof i fixed), the mask P of the reference's
 * projected operator A(v) = P(K P v).
 *
 * Reference interfaces replaced (paths inside the sttopt project):
 *   stt_q4_apply        sttopt/torch_fem.py:62-83 (matvec), :135-159 (operator)
 *   stt_q4_diag         sttopt/torch_fem.py:86-98 (matvec_diagonal), :162-181 (jacobi diag)
 *   stt_lumped_reaction sttopt/torch_fem.py:117-132
 *   stt_ke_modal        sttopt/fem.py:17-30, :98-111 (the element matrices it recognises)
 *   stt_cone_filter*    sttopt/filters.py:38-85 (density_filter, apply_density_filter),
 *                       :109-133 (heaviside_projection and its derivative)
 *   stt_hier_*          sttopt/torch_mg.py:293-400 (build_hierarchy), :257-266 (select)
 *   stt_level_apply     sttopt/torch_mg.py:239-255 (_Level.__call__), :179-193 (keff_matvec)
 *   stt_vcycle          sttopt/torch_mg.py:403-476 (VCycle.__call__)
 *   stt_grid_transfer   sttopt/torch_mg.py:75-109 (_interp_axis, _restrict_axis, _on_node_grid)
 *   stt_keff_apply      sttopt/torch_mg.py:168-193 (_scatter, keff_matvec)
 *   stt_pcg_mg          sttopt/torch_fem.py:201-343 (pcg with a multigrid preconditioner)
 *   stt_vec_*           sttopt/torch_fem.py:253-331 (the PCG vector updates, any operator)
 *   stt_element_sens    sttopt/torch_solve.py:144-152 (FemSolve.backward element terms),
 *                       sttopt/compliance.py:49-59 (_element_strain_energy)
 *   stt_stage_*         sttopt/compliance.py:137-161,198-253 with a hard stage threshold
 *   stt_stage_glue_*    sttopt/compliance.py:33-46 (time_mask), :137-161 (_gravity_load),
 *                       :164-253 (gravity_compliance, batched_whole_and_gravity_compliance)
 *   stt_lumped_reaction_adjoint  sttopt/torch_fem.py:117-132 (lumped_reaction's gradient)
 *   stt_q4_apply_dots, stt_adjoint_warm_start  sttopt/torch_solve.py:117-140 (FemSolve.backward:
 *                       the adjoint load and its warm start alpha U, alpha = (U.g)/(U.F))
 *   stt_heat_*          sttopt/virtual_heat.py:162-166,189-201,404-462
 *   stt_mma_sub         sttopt/mma.py:150-285 (mmasub: asymptotes, approximation, subsolv)
 *   stt_mma_subsolv     sttopt/mma.py:346-557 (subsolv)
 */
#ifndef STTB200_H
#define STTB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* stt_stream_t; /* == cudaStream_t */

enum {
  STT_OK = 0,
  STT_ERR_INVALID = 1,       /* bad argument (size, pointer, precision) */
  STT_ERR_NOT_CONVERGED = 2, /* PCG hit max_iter with a row above rtol */
  STT_ERR_BREAKDOWN = 3,     /* a non-finite PCG scalar */
  STT_ERR_TIMEOUT = 4,       /* a bounded device wait gave up */
  STT_ERR_CUDA = 5,          /* a CUDA runtime call failed */
  STT_ERR_WORKSPACE = 6      /* the workspace is smaller than required */
};

enum { STT_FP64 = 0, STT_FP32 = 1 };
enum { STT_FORM_MODAL = 0, STT_FORM_PRODUCT = 1 };
enum { STT_PROJECT_IN = 1, STT_PROJECT_OUT = 2 };

/* Last CUDA / argument error message of this thread (never NULL). */
const char* stt_last_error(void);

/* ---- level-0 operator ---------------------------------------------------------- */

/* out[s] = [P] (K(rho[h(s)]) [P] u[s] + rdiag[h(s)] * [P] u[s]) for s < nrows.
 * precision selects double (STT_FP64) or float (STT_FP32) for u, out, rho and rdiag.
 * rho_rs == 0 broadcasts one density field; rdiag may be NULL (no reaction term);
 * fixed may be NULL (no projection).  KE is a host pointer to (4d)^2 doubles. */
int stt_q4_apply(int precision, int d, int nelx, int nely, int nrows,
                 const void* u, long long u_rs, void* out, long long out_rs,
                 const void* rho, long long rho_rs, const void* rdiag, long long rdiag_rs,
                 const uint8_t* fixed, int flags, const double* KE, stt_stream_t stream);

/* out[s] = P K(rho[s]) u[s] (FP64, fixed dofs zeroed; u projected already) and in the same
 * pass dots[s][0] = u[s] . out[s], dots[s][1] = u[s] . f[s]: an adjoint load (KE = 2 KE
 * gives dL/dU = 2 K U) with its warm-start factor's dots, one pass over u.  The dots are
 * reduced in a fixed order through ws (stt_q4_apply_dots_workspace_bytes; 256-byte
 * aligned; its counters are reset on the stream).  Any KE (modal or the 8 x 8 product). */
long long stt_q4_apply_dots_workspace_bytes(int nelx, int nely, int nrows);
int stt_q4_apply_dots(int d, int nelx, int nely, int nrows, const double* u, long long u_rs,
                      double* out, long long out_rs, const double* rho, long long rho_rs,
                      const uint8_t* fixed, const double* KE, const double* f, long long f_rs,
                      double* dots, void* ws, long long ws_bytes, stt_stream_t stream);

/* out[s] = safe_div(dots[s][0], dots[s][1]) v[s] (FP64, dots [nrows][2] as written by
 * stt_q4_apply_dots): the adjoint's warm start alpha U, alpha = (U . g) / (U . F). */
int stt_adjoint_warm_start(int nrows, long long n, const double* dots, const double* v, long long v_rs,
                           double* out, long long o_rs, stt_stream_t stream);

/* The adjoint of stt_lumped_reaction: out[s][e] = (1/4) sum over e's 4 corners and their
 * d dofs of g[s].  FP64. */
int stt_lumped_reaction_adjoint(int d, int nelx, int nely, int nrows, const double* g, long long g_rs,
                                double* out, long long o_rs, stt_stream_t stream);

/* diag(K(rho)) (+ rdiag), with fixed dofs set to 1 when fixed != NULL.  FP64. */
int stt_q4_diag(int d, int nelx, int nely, int nrows, const double* rho, long long rho_rs,
                const double* rdiag, long long rdiag_rs, const uint8_t* fixed,
                double* out, long long out_rs, const double* KE, stt_stream_t stream);

/* rdiag[n * d + i] = sum over elements e touching node n of reaction[e] / 4.  FP64. */
int stt_lumped_reaction(int d, int nelx, int nely, int nrows, const double* reaction,
                        long long r_rs, double* out, long long out_rs, stt_stream_t stream);

/* How element matrices are applied, process-wide, by every later stt_hier_create and
 * level-0 apply (not by hierarchies already built): STT_FORM_MODAL (default) through the
 * element's edge modes when KE has the modal form (stt_ke_modal), else the 8 x 8 product;
 * STT_FORM_PRODUCT always the 8 x 8 product of the corner values, as the reference's
 * torch_fem.matvec (sttopt/torch_fem.py:76-82).  The modal form is faster and exact on
 * rigid translations; the product form reproduces the reference's FP64 rounding (its
 * float64 KE gives a translation a stiffness of ~1e-16 per element).  Returns the
 * previous form, or -1 for an unknown one.  No reference counterpart. */
int stt_set_element_form(int form);

/* Host only (no device work).  Returns 1 and writes m[8] when KE ((4d)^2 doubles) has
 * the modal form KE = T^T M T of the unit-square bilinear element (the reference's
 * plane-stress KE for any nu, and its diffusion KE), which the level-0 kernels then
 * apply through the element's edge modes; returns 0 for any other KE (those take the
 * generic 8 x 8 product).  m = {m00, m01, m11, m22, m44, m55, kd0, kd1}. */
int stt_ke_modal(int d, const double* KE, double* m);

/* ---- density filter ------------------------------------------------------------ */

/* xt[s] = H x[s] / Hs with H[e1, e2] = max(0, rmin - dist(e1, e2)) over the offsets
 * |d| <= ceil(rmin) - 1 (zero outside the grid) and Hs its row sums; when beta > 0 also
 * xp[s] = P(xt[s]), the Heaviside projection at threshold eta (beta = +inf: the step,
 * 1/2 at the threshold).  Element fields (nely x nelx, row-major), FP64, rmin in (0, 8]. */
int stt_cone_filter(int nelx, int nely, int nrows, double rmin, const double* x, long long x_rs,
                    double* xt, double* xp, long long o_rs, double beta, double eta,
                    stt_stream_t stream);

/* The adjoint: out[s] = H (g[s] * P'(xt[s]) / Hs) (beta > 0, xt given) or H (g[s] / Hs). */
int stt_cone_filter_adjoint(int nelx, int nely, int nrows, double rmin, const double* g,
                            long long g_rs, const double* xt, long long xt_rs, double beta,
                            double eta, double* out, long long o_rs, stt_stream_t stream);

/* ---- multigrid hierarchy ------------------------------------------------------- */

typedef struct stt_hier stt_hier;

/* Bytes of device workspace a hierarchy of hrows density fields needs. */
long long stt_hier_workspace_bytes(int d, int nelx, int nely, int hrows,
                                   int max_coarse_elements, int precision);

/* Build the Galerkin hierarchy on the device (torch_mg.build_hierarchy): level 0 is
 * K(rho) (+ lumped reaction), coarser levels the exact Galerkin products stored as
 * symmetric 9-point block stencils, the coarsest factorised by FP64 Cholesky.
 * precision STT_FP32 keeps FP32 copies for an FP32 V-cycle.  reaction may be NULL. */
int stt_hier_create(stt_hier** out, void* workspace, long long ws_bytes, int d, int nelx,
                    int nely, int hrows, const double* rho, long long rho_rs,
                    const double* reaction, long long r_rs, const uint8_t* fixed,
                    const double* KE, int max_coarse_elements, int precision,
                    stt_stream_t stream);

/* The build does not synchronise.  The levels are built on `stream`; the coarsest
 * level's factorisation (and its explicit inverse for STT_FP32) then runs on a stream of
 * the library's own, ordered after them, while `stream` goes on: every coarse solve on
 * any stream (stt_vcycle, stt_pcg_mg, ...) waits for it on the device.  The build's
 * device checks (a coarse pivot <= 0, a coarse operator beyond its planned band) are
 * reported by stt_hier_status (which waits for the factorisation and synchronises
 * `stream`) and by the first convergence check of stt_pcg_mg after its first V-cycle.
 * Work on other streams must be ordered after `stream` by the caller, as usual. */
int stt_hier_status(const stt_hier* h, stt_stream_t stream);

/* A view of h restricted to batch rows: batch row s uses hierarchy row row_map[s]
 * (device int32, caller-owned, kept alive while the view is used).  A view shares h's
 * workspace and coarse factorisation and may outlive h's handle (not its workspace). */
int stt_hier_select(const stt_hier* h, const int* row_map, stt_hier** out);
/* Releases a hierarchy or view handle.  The last handle of a hierarchy waits (host) for
 * its coarse factorisation, after which the caller may reuse the workspace. */
int stt_hier_destroy(stt_hier* h);

/* nlevels, and per level (nelx, nely, kx, ky) into dims[4 * level]. */
int stt_hier_info(const stt_hier* h, int* nlevels, int* dims, int max_levels);

/* Launch shapes of the solves on h (stt_vcycle, stt_pcg_mg, stt_level_apply; views made
 * afterwards inherit them): pcg_band, the grid rows a block of the PCG's level-0 passes
 * marches (8, 16 or 32; 0: the built-in choice, 32 or shorter while the rows give fewer
 * than two waves of blocks), and level_waves, the blocks the stencil levels' kernels aim
 * at in waves of one block per SM (1..64; 0: four).  Results do not depend on them beyond
 * the order of the block reductions.  No reference counterpart: set by this library's
 * autotuner (sttopt_b200.autotune), which times the candidates on the hierarchy. */
int stt_hier_tune(stt_hier* h, int pcg_band, int level_waves);

/* Copies of a level's Jacobi diagonal (FP64, [hrows][ndof]) and fixed flags. */
int stt_hier_level_diag(const stt_hier* h, int level, double* out, stt_stream_t stream);
int stt_hier_level_fixed(const stt_hier* h, int level, uint8_t* out, stt_stream_t stream);

/* out[s] = A_level v[s] (the projected level operator, FP64). */
int stt_level_apply(const stt_hier* h, int level, int nrows, const double* v, long long v_rs,
                    double* out, long long out_rs, stt_stream_t stream);

/* The grid transfers of torch_mg._on_node_grid with _interp_axis (restrict_ == 0:
 * out = P in, in on the cnnx x cnny coarse node grid) or _restrict_axis (restrict_ != 0:
 * out = R in = P^T in, in on the fine grid), sttopt/torch_mg.py:75-109: the x pass then
 * the y pass, factors kx, ky in {1, 2, 3}, d interleaved dofs per node, no projection.
 * FP64; nrows batch rows with their own strides. */
int stt_grid_transfer(int d, int kx, int ky, int cnnx, int cnny, int nrows, int restrict_,
                      const double* in, long long in_rs, double* out, long long out_rs,
                      stt_stream_t stream);

/* keff_matvec (sttopt/torch_mg.py:179-193): out[s] = sum_e scatter(U_e[s]^T keff[s][e]) with
 * explicit element matrices keff[s] ((4d)^2 doubles per element, row-major, the
 * reference's local dof order; k_rs = 0 shares one set over the rows).  FP64,
 * deterministic (node-centric gather, no atomics). */
int stt_keff_apply(int d, int nelx, int nely, int nrows, const double* U, long long u_rs,
                   const double* keff, long long k_rs, double* out, long long o_rs,
                   stt_stream_t stream);

/* Live timing of the plane-stress solves' steady-state p.Ap passes (pcg_pap_kernel with a
 * deferred x update), for measurement: while enabled (stt_pap_timing(1), which also resets
 * the totals) each such launch of stt_pcg_mg is bracketed by CUDA events on its stream;
 * stt_pap_timing_read returns the summed milliseconds, the launches and the batch rows
 * summed over the launches.  No reference counterpart. */
int stt_pap_timing(int enable);
int stt_pap_timing_read(double* total_ms, long long* launches, long long* rows);

/* Bytes of device workspace for stt_pcg_mg over nrows batch rows (enough for stt_vcycle
 * too). */
long long stt_solve_workspace_bytes(const stt_hier* h, int nrows, int gamma);
/* Bytes of device workspace stt_vcycle needs over nrows batch rows (its per-level
 * vectors and coarse scratch only). */
long long stt_vcycle_workspace_bytes(const stt_hier* h, int nrows, int gamma);

/* z[s] = M r[s], one V-cycle (damped Jacobi omega, n_smooth sweeps each way, gamma
 * coarse visits).  r and z are FP64; the cycle runs in the hierarchy's precision. */
int stt_vcycle(const stt_hier* h, int nrows, const double* r, long long r_rs, double* z,
               long long z_rs, double omega, int n_smooth, int gamma, void* workspace,
               long long ws_bytes, stt_stream_t stream);

/* stt_vcycle without a caller workspace.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory: plugins inside a host application that owns
 * the device memory pool and forbids outside cudaMalloc, multi-stream pipelines that
 * cannot afford cudaMalloc's implicit device synchronisation mid-run, and bindings that
 * can pass input and output buffers but cannot size and own scratch.
 * Its scratch is a fixed 32 MiB array inside this library, held by every GPU that loads
 * the library until exit; calls needing more (stt_vcycle_workspace_bytes) return
 * STT_ERR_WORKSPACE without launching.  All calls on a device share that array: calls
 * that overlap on the GPU race, so order them on one stream.  The first call on each
 * device looks up the array's device address and keeps it for the process's lifetime:
 * make that first call before any stream capture, and do not use the library across a
 * reset of the device's primary context (cudaDeviceReset), which also invalidates its
 * hierarchy handles and streams.  Results equal stt_vcycle's for the same arguments. */
int stt_vcycle_noalloc(const stt_hier* h, int nrows, const double* r, long long r_rs, double* z,
                       long long z_rs, double omega, int n_smooth, int gamma, stt_stream_t stream);

/* MG-preconditioned CG on all batch rows, entirely on the device.  x holds the warm
 * start when has_x0, else is zeroed; b must already be projected.  Outputs: rel_resid
 * [nrows] (host), conv_iter [nrows] (host, -1 = not converged), *n_iter (host).
 * flexible selects the Polak-Ribiere beta; replace_every > 0 recomputes the true
 * residual b - A x every that many iterations.  retire selects when a converged row
 * stops: 0 at once; 1 as the reference retires rows (torch_fem.py:270-331), a converged
 * row iterating on with the others until the rows short of rtol are at most 3/4 of the
 * rows left by the previous retirement, so that every row's x equals the reference's
 * (conv_iter is then the iteration at which the row stopped).  Returns
 * STT_ERR_NOT_CONVERGED when a row is above rtol after max_iter iterations. */
int stt_pcg_mg(const stt_hier* h, int nrows, const double* b, long long b_rs, double* x,
               long long x_rs, int has_x0, double rtol, int max_iter, double omega,
               int n_smooth, int gamma, int flexible, int replace_every, int retire,
               double* rel_resid, int* conv_iter, int* n_iter, void* workspace, long long ws_bytes,
               stt_stream_t stream);

/* ---- PCG vector steps for arbitrary operators (FP64) ---------------------------- */

/* dots[s * k + j] = sum_i a_j[s, i] * b_j[s, i] for the k <= 3 pairs given (NULL ends). */
int stt_vec_dots(int nrows, long long n, const double* a0, const double* b0, const double* a1,
                 const double* b1, const double* a2, const double* b2, long long rs,
                 double* dots, stt_stream_t stream);
/* x += alpha[s] p; r -= alpha[s] Ap; rr[s] = ||r[s]||^2. */
int stt_vec_cg_update(int nrows, long long n, const double* alpha, double* x, double* r,
                      const double* p, const double* Ap, long long rs, double* rr,
                      stt_stream_t stream);
/* p = z + beta[s] p. */
int stt_vec_xpay(int nrows, long long n, const double* z, const double* beta, double* p,
                 long long rs, stt_stream_t stream);

/* ---- element terms ------------------------------------------------------------- */

/* Per element e and batch row s: ce = U_e^T KE U_e; gdens = -lam_e^T KE U_e;
 * greac = -lam_e . U_e / 4.  Any of ce, gdens, greac may be NULL (lam too, if both
 * gradients are NULL).  FP64. */
int stt_element_sens(int d, int nelx, int nely, int nrows, const double* U, long long U_rs,
                     const double* lam, long long lam_rs, const double* KE, double* ce,
                     double* gdens, double* greac, long long e_rs, stt_stream_t stream);

/* ---- space-time stage glue (hard threshold t <= s / n_stage) -------------------- */

/* member[s * nel + e] = tPhys[e] <= (s + 1) / n_stage, bit-exact FP64 compare. */
int stt_stage_membership(int nel, int n_stage, const double* tPhys, uint8_t* member,
                         stt_stream_t stream);

/* For each stage s: xt = x * m_s; rho = Emin + xt^penal (Emax - Emin) (FP64);
 * F[2n+1] = -(fe / 4) sum of xt over the elements of node n, F[2n] = 0, masked by
 * fixed; fe = 1 / (nelx nely). */
int stt_stage_rows(int nelx, int nely, int n_stage, const double* x, const uint8_t* member,
                   double Emin, double Emax, double penal, const uint8_t* fixed, double* rho,
                   double* F, stt_stream_t stream);

/* grad[e] += sum_s m_s[e] * ((ce_s + gdens_s) * penal * xt^(penal - 1) * (Emax - Emin)
 *            - (fe / 4) * sum over corners of gF_s at the y dofs).  ce/gdens [n_stage][nel],
 * gF [n_stage][2 nnode]. */
int stt_stage_gradient(int nelx, int nely, int n_stage, const double* x,
                       const uint8_t* member, const double* ce, const double* gdens,
                       const double* gF, double Emin, double Emax, double penal, double* grad,
                       stt_stream_t stream);

/* ---- production stage glue (any stage mask) ------------------------------------ */

/* Rows of the one batched whole + self-weight solve.  For stage s < n_stage the mask row
 * m_s is M[s] (M != NULL) or the smooth indicator
 * max(0, 1 - (tanh(beta ti) + tanh(beta (t - ti))) / (tanh(beta ti) + tanh(beta (1 - ti))))
 * with ti = times[s] (host array), written to M_out when non-NULL; xt[s] = x * m_s.  Row
 * layout of rho and F: with has_row0, row 0 is the whole structure (rho = SIMP(x),
 * F = F0) and stage s is row s + 1.  rho[r] = Emin + xt^penal (Emax - Emin);
 * F[r][2n] = 0, F[r][2n+1] = -(fe / 4) * sum of xt over the elements of node n,
 * fe = 1 / (nelx nely) (unprojected, as the reference builds it).  Any of M_out, xt,
 * rho, F may be NULL (F needs xt).  FP64; n_stage <= 128. */
int stt_stage_glue_rows(int nelx, int nely, int n_stage, int has_row0, const double* x,
                        const double* t, const double* times, double beta, const double* M,
                        double* M_out, const double* F0, double Emin, double Emax, double penal,
                        double* xt, double* rho, double* F, stt_stream_t stream);

/* The adjoint of stt_stage_glue_rows for output gradients g_xt [n_stage][nel],
 * g_rho and g_F (rows as above; any may be NULL): gx[e] (overwritten), gt[e] (optional,
 * the smooth indicator's t gradient; the clamp's gradient passes where the unclamped
 * value is >= 0) and gM[s][e] = d/dm_s (optional).  The mask rows are the smooth
 * indicator when t (with times and beta) is given, else M. */
int stt_stage_glue_adjoint(int nelx, int nely, int n_stage, int has_row0, const double* x,
                           const double* t, const double* times, double beta, const double* M,
                           const double* g_xt, const double* g_rho, const double* g_F,
                           double Emin, double Emax, double penal, double* gx, double* gt,
                           double* gM, stt_stream_t stream);

/* Heat glue: t_e = mean over corners of (1 - T); and the adjoint load
 * g[n] = -sum over elements of w[e] / (4 scale). */
int stt_heat_element_means(int nelx, int nely, const double* T, double* t_e,
                           stt_stream_t stream);
int stt_heat_adjoint_load(int nelx, int nely, const double* w, double scale, double* g,
                          stt_stream_t stream);

/* ---- element <-> node transfers of the stage glue and the time fields ----------- */

/* Gravity load matrix C of the self-weight load (replaces gravity.gravity_load_matrix,
 * sttopt/gravity.py:15-36, and its SpMV in compliance._gravity_load,
 * sttopt/compliance.py:156): transpose == 0: out[s][n] = (fe / 4) * sum of x[s][e] over
 * the elements of node n (C x); transpose != 0: out[s][e] = (fe / 4) * sum of x[s][n]
 * over the corners of e (C^T g).  fe = 1 / (nelx nely).  FP64. */
int stt_gravity_load(int nelx, int nely, int nrows, const double* x, long long x_rs,
                     double* out, long long o_rs, int transpose, stt_stream_t stream);

/* Element means (virtual_heat.element_means, sttopt/virtual_heat.py:162-166):
 * transpose == 0: out[s][e] = mean of u[s] over e's corners; transpose != 0:
 * out[s][n] = sum over the elements of n of u[s][e] / 4 (the adjoint).  FP64. */
int stt_element_means(int nelx, int nely, int nrows, const double* u, long long u_rs,
                      double* out, long long o_rs, int transpose, stt_stream_t stream);

/* Load of the Poisson distance fit (ScalarMesh.divergence_load(w, direction_field(s)),
 * sttopt/virtual_heat.py:290-320): F[n] = sum over elements of w[e] / 4 * sum over the
 * 2 x 2 Gauss points of X . grad N_n, X = grad s / sqrt(|grad s|^2 + DBL_MIN).  FP64. */
int stt_poisson_load(int nelx, int nely, int nrows, const double* s, long long s_rs,
                     const double* w, long long w_rs, double* F, long long F_rs,
                     stt_stream_t stream);

/* Its adjoint for an output weight gF: gs = (dF/ds)^T gF (per node), gw = (dF/dw)^T gF
 * (per element); either output may be NULL. */
int stt_poisson_load_adjoint(int nelx, int nely, int nrows, const double* s, long long s_rs,
                             const double* w, long long w_rs, const double* gF, long long gF_rs,
                             double* gs, long long gs_rs, double* gw, long long gw_rs,
                             stt_stream_t stream);

/* ---- MMA subproblem (sttopt/mma.py:150-557) -----------------------------------------
 *
 * n-sized vectors and the m x n matrices (row stride ld >= n, in elements) are device
 * pointers; m-sized vectors (fval, a, b, c, d and the m-sized results y, lam, mu, s) and
 * the scalars z, zet are HOST pointers, since the m-sized algebra runs on the host.  The
 * calls synchronise the stream.  With m < n (at most 64 constraints) the per-variable
 * work runs on the device; with m >= n the whole solve runs in the library's host code.
 * counts (optional, 3 ints) receives the number of barrier levels whose Newton loop
 * stopped at its 200-iteration cap, the Newton steps taken and the line-search
 * candidates tried; cap_epsi (optional) the last capped level's epsi.  Workspace:
 * stt_mma_workspace_bytes (256-byte aligned device memory). */
size_t stt_mma_workspace_bytes(int m, long long n);

/* mmasub (sttopt/mma.py:150-285) with epsimin 1e-7: low / upp are read (iteration >= 2)
 * and overwritten with the new asymptotes; each of asyinit, asyclamp_min, asyclamp_max
 * and move is a device n-vector, or NULL for the scalar beside it.  Outputs xmma, xsi,
 * eta (device n) and ymma, zmma, lam, mu, zet, s (host). */
int stt_mma_sub(int m, long long n, int iteration, const double* xval, const double* xmin,
                const double* xmax, const double* xold1, const double* xold2, const double* df0dx,
                const double* fval, const double* dfdx, long long dfdx_ld, double* low, double* upp,
                double a0, const double* a, const double* c, const double* d,
                const double* asyinit, double asyinit_v, const double* asyclamp_min,
                double asyclamp_min_v, const double* asyclamp_max, double asyclamp_max_v,
                const double* move, double move_v, double raa0, double albefa, double asyincr,
                double asydecr, double* xmma, double* xsi, double* eta, double* ymma, double* zmma,
                double* lam, double* mu, double* zet, double* s, int* counts, double* cap_epsi,
                void* ws, size_t ws_bytes, stt_stream_t stream);

/* subsolv (sttopt/mma.py:346-557) on a given subproblem: low, upp, alfa, beta, p0, q0
 * (device n), P, Q (device m x n, row stride ld), a0 and a, b, c, d (host m). */
int stt_mma_subsolv(int m, long long n, double epsimin, const double* low, const double* upp,
                    const double* alfa, const double* beta, const double* p0, const double* q0,
                    const double* P, const double* Q, long long ld, double a0, const double* a,
                    const double* b, const double* c, const double* d, double* xmma, double* xsi,
                    double* eta, double* ymma, double* zmma, double* lam, double* mu, double* zet,
                    double* s, int* counts, double* cap_epsi, void* ws, size_t ws_bytes,
                    stt_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* STTB200_H */
