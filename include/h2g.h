/*
 * h2g.h -- C ABI of the B200 (sm_100a) solver library for the Heat3ds linear-solver path.
 *
 * The library replaces the Julia module NonUniform (src/NonUniform.jl) for par="gpu":
 * the matrix-free 7-point finite-volume operator, the 5-sweep red-black Gauss-Seidel
 * preconditioner and the PBiCGSTAB / CG drivers.  It is called with the reference's own
 * arrays: Float64, column-major (i fastest), shape (MX, MY, MZ) = (NX+2, NY+2, NZ+2)
 * including one guard layer on each side (src/common.jl:49-89).  Element (i,j,k) of the
 * Julia array (1-based) is host element (i-1) + MX*((j-1) + MY*(k-1)).
 *
 * Conventions
 *  - Every entry returns an int status (H2G_OK = 0 or one of the codes below); nothing
 *    aborts or exits.  h2g_last_error() gives a one-line message for the last failure
 *    on the calling thread.
 *  - Host pointers are copied in and out; device memory is owned by the solver handle.
 *  - A handle is not thread-safe: use one handle per host thread / Julia task.
 *  - Calls are synchronous with respect to the host unless they say otherwise; they run
 *    on the stream given to h2g_set_stream (default: the legacy default stream).
 */
#ifndef H2G_H
#define H2G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define H2G_OK 0              /* converged / done */
#define H2G_NOT_CONVERGED 1   /* maxItr reached (reference: isconverged=false, NonUniform.jl:225,349) */
#define H2G_BREAKDOWN 2       /* |rho|, (p,q) or (t,t) below FloatMin=1e-37 (NonUniform.jl:169-173, 291-294, 321-324) */
#define H2G_NONFINITE 3       /* NaN/Inf in an input array or in the iteration */
#define H2G_BAD_ARG 4         /* rejected on the host before any launch */
#define H2G_CUDA_ERROR 5      /* a CUDA runtime call failed */
#define H2G_TIMEOUT 6         /* a bounded device wait ran out (the fused sweep's TMA waits) */
#define H2G_UNSUPPORTED 7     /* input outside what the library implements (message says what) */

/* ---- precision ---------------------------------------------------------------------- */
#define H2G_FP64 0     /* FP64 throughout, same arithmetic as the reference */
#define H2G_MIXED 1    /* FP32 RB-GS preconditioner (operator tables, smoother vectors) inside FP64
                          PBiCGSTAB/CG: FP64 Krylov vectors, inner products, CalcAX and solution;
                          convergence is confirmed on the FP64 true residual (restarts if needed) */
#define H2G_MIXED_IR 2 /* FP32 operator, smoother and Krylov vectors inside FP64 iterative
                          refinement (FP64 true residual, solution accumulation, inner products);
                          its FP32 BiCGSTAB can diverge on fine grids (reported as H2G_NONFINITE) */

/* ---- smoother (NonUniform.jl:36-41: :none, :gs) -------------------------------------- */
#define H2G_SMOOTHER_NONE 0
#define H2G_SMOOTHER_GS 1

/* ---- boundary types (src/common.jl:20-24) -------------------------------------------- */
#define H2G_ISOTHERMAL 0
#define H2G_HEAT_FLUX 1
#define H2G_CONVECTION 2

/* BoundaryCondition (src/boundary_conditions.jl:15-21); faces ordered x-, x+, y-, y+, z-, z+
 * (BoundaryConditionSet, boundary_conditions.jl:24-31). */
typedef struct h2g_bc {
  int type;
  double temperature;
  double heat_flux;
  double htc;
  double ambient;
} h2g_bc;

/* The (isconverged, itr, res0) tuple returned by PBiCGSTAB!/CG! (NonUniform.jl:225, 349),
 * plus what the GPU path adds. */
typedef struct h2g_result {
  int isconverged; /* 1 if ||r_k|| / ||r_0|| < tol */
  int itr;         /* PBiCGSTAB/CG iterations (all inner iterations for H2G_MIXED_IR) */
  int outer;       /* refinement passes (H2G_MIXED_IR) or true-residual restarts (H2G_MIXED) */
  int status;      /* same value the call returns */
  double res0;     /* initial residual ||b - A theta||_2 (NonUniform.jl:263) */
  double res;      /* final relative residual ||r|| / res0 */
  long long launches; /* kernels this call launched on the device (graph iterations included) */
} h2g_result;

typedef struct h2g_solver h2g_solver;

/* ---- library ------------------------------------------------------------------------ */
const char *h2g_version(void);
const char *h2g_status_string(int status);
const char *h2g_last_error(void);

/* ---- handle lifecycle ----------------------------------------------------------------
 * Allocates the device copies of WorkBuffers (src/common.jl:71-89) for an (MX,MY,MZ)
 * grid on the current CUDA device. */
int h2g_create(int MX, int MY, int MZ, int precision, h2g_solver **out);
int h2g_destroy(h2g_solver *h);
/* stream: a cudaStream_t (NULL = legacy default stream). */
int h2g_set_stream(h2g_solver *h, void *stream);

/* Grid and coefficients of the operator (the Δh, Δt, ZC, ΔZ, HC, is_steady arguments of
 * CalcAX!/CalcRK!/rbsor_core!, NonUniform.jl:372-386, 454-466, 848-862).  ZC and dZ have
 * MZ entries (genZ!, src/Zcoord.jl:133-166); HC has 6 (set_BC_coef, boundary_conditions.jl:360-394). */
int h2g_set_grid(h2g_solver *h, const double *ZC, const double *dZ, double dx, double dy, double dt,
                 const double *HC, int is_steady);
/* wk.λ, wk.mask, wk.ρ, wk.cp (src/common.jl:52-55), guard layers included.  ρ and cp may be
 * NULL for a steady grid.  Masks must be 0 or 1. */
int h2g_set_fields(h2g_solver *h, const double *lambda, const double *mask, const double *rho,
                   const double *cp);
/* wk.b and wk.θ (src/common.jl:50-51). */
int h2g_set_rhs(h2g_solver *h, const double *b);
int h2g_get_rhs(h2g_solver *h, double *b);
int h2g_set_theta(h2g_solver *h, const double *theta);
int h2g_get_theta(h2g_solver *h, double *theta);
/* Device-side copy of θ: op 0 saves the current θ, op 1 restores it (repeat a solve from
 * the same start without a host copy). */
int h2g_theta_snapshot(h2g_solver *h, int op);

/* Iterative-refinement settings for H2G_MIXED_IR: inner relative tolerance of each FP32 solve
 * and the cap on refinement passes (defaults 1e-4 and 40). */
int h2g_set_mixed_params(h2g_solver *h, double inner_tol, int max_outer);

/* ---- solvers -------------------------------------------------------------------------
 * PBiCGSTAB!(wk, Δh, Δt, ZC, ΔZ, HC; tol, maxItr, smoother, par, verbose, is_steady)
 *   (src/NonUniform.jl:248-350) on the handle's θ, b and fields; θ is updated on the device
 *   (fetch it with h2g_get_theta).  res_hist (nullable, maxItr doubles) receives the relative
 *   residual of every iteration; verbose prints the reference's "%10d %24.14E" lines to stdout.
 *   Returns H2G_OK when converged. */
int h2g_pbicgstab(h2g_solver *h, double tol, int maxItr, int smoother, int verbose, double *res_hist,
                  h2g_result *out);
/* CG!(...) (src/NonUniform.jl:115-226), same conventions. */
int h2g_cg(h2g_solver *h, double tol, int maxItr, int smoother, int verbose, double *res_hist, h2g_result *out);

/* One-call drop-in for PBiCGSTAB!/CG! with the reference's arrays (heat3ds.jl:133-141):
 * uploads θ, b, λ, mask, ρ, cp and the grid, solves, and writes θ back.  A handle for the
 * grid size is kept between calls (not thread-safe). */
int h2g_PBiCGSTAB(int MX, int MY, int MZ, double *theta, const double *b, const double *lambda,
                  const double *mask, const double *rho, const double *cp, double dx, double dy, double dt,
                  const double *ZC, const double *dZ, const double *HC, double tol, int maxItr, int smoother,
                  int verbose, int is_steady, int precision, double *res_hist, h2g_result *out);
int h2g_CG(int MX, int MY, int MZ, double *theta, const double *b, const double *lambda, const double *mask,
           const double *rho, const double *cp, double dx, double dy, double dt, const double *ZC,
           const double *dZ, const double *HC, double tol, int maxItr, int smoother, int verbose, int is_steady,
           int precision, double *res_hist, h2g_result *out);
/* solveSOR!(θ, λ, b, mask, ρ, cp, Δh, Δt, ω, ZC, ΔZ, HC, F, tol, par; maxItr, is_steady)
 *   (src/NonUniform.jl:1004-1051): res0 = resSOR (1 if it is 0), then rbsor! passes (colour 0,
 *   colour 1) with relaxation omega in (0, 2) until sqrt(sum of r^2)/res0 < tol.  Runs in FP64
 *   whatever the handle's precision.  res_hist and verbose as for h2g_pbicgstab (the reference
 *   writes the same lines to F and stdout).  A non-finite residual stops the loop with
 *   H2G_NONFINITE (the reference would run on to maxItr). */
int h2g_sor(h2g_solver *h, double omega, double tol, int maxItr, int verbose, double *res_hist, h2g_result *out);
/* One-call drop-in for solveSOR! with the reference's arrays (FP64; handle cached as above). */
int h2g_SolveSOR(int MX, int MY, int MZ, double *theta, const double *b, const double *lambda, const double *mask,
                 const double *rho, const double *cp, double dx, double dy, double dt, double omega,
                 const double *ZC, const double *dZ, const double *HC, double tol, int maxItr, int verbose,
                 int is_steady, double *res_hist, h2g_result *out);
/* Release the handles kept by h2g_PBiCGSTAB / h2g_CG / h2g_SolveSOR. */
int h2g_release_cached(void);

/* ---- batches ----------------------------------------------------------------------------
 * Solve n independent systems at once (many power maps and grids of uneven size): every handle
 * keeps its own grid, fields, θ and b (set beforehand), gets its own non-blocking stream for the
 * batch, and its whole solve (a CUDA graph looping on the device) is issued from one of
 * `threads` host threads (<= 0: 2), so the solves run concurrently on the GPU.  method 0
 * PBiCGSTAB, 1 CG, 2 RB-SOR with omega = 1.  outs[q] receives handle q's result (the same values
 * as a lone h2g_pbicgstab/h2g_cg on that handle: kernels are deterministic).  Returns H2G_OK
 * when every member converged, else the first non-OK member status (H2G_BAD_ARG /
 * H2G_CUDA_ERROR if a member failed that way).  No reference counterpart: the reference solves
 * one system per call (heat3ds.jl:128-141). */
int h2g_batch_solve(int n, h2g_solver *const *hs, int method, double tol, int maxItr, int smoother, int threads,
                    h2g_result *outs);

/* ---- K right-hand sides on one operator (no reference counterpart) ------------------------
 * The batched workload's members of one grid size share the operator (geometry, materials,
 * boundary set) and differ in their heat maps, so in b.  h2g_create_multi makes an FP64 handle for
 * nrhs (1..64) right-hand sides: grid and fields are set once with h2g_set_grid / h2g_set_fields;
 * b and theta of every right-hand side with h2g_set_rhs_multi / h2g_set_theta_multi (nrhs
 * column-major arrays of MX*MY*MZ doubles one after another; h2g_get_theta_multi reads them back).
 * h2g_pbicgstab_multi runs PBiCGSTAB! + RB-GS (smoother 1 only) for all of them at once: every
 * stencil kernel computes a cell's coefficients once for a group of right-hand sides, and each
 * right-hand side keeps its own scalars, stop test and result (outs[nrhs]); its iterates and
 * result are bit for bit those of its lone solve (h2g_pbicgstab).  Returns H2G_OK when every
 * right-hand side converged, else the first other status. */
int h2g_create_multi(int MX, int MY, int MZ, int nrhs, h2g_solver **out);
int h2g_set_rhs_multi(h2g_solver *h, const double *b);
int h2g_set_theta_multi(h2g_solver *h, const double *theta);
int h2g_get_theta_multi(h2g_solver *h, double *theta);
int h2g_pbicgstab_multi(h2g_solver *h, double tol, int maxItr, int smoother, h2g_result *outs);

/* ---- steady adjoint (no reference counterpart) -------------------------------------------
 * Gradient of J = (sum_c w_c θ_c^p)^(1/p) (w_c >= 0 per cell, column-major with guards, e.g.
 * the cell volume on the silicon cells and 0 elsewhere; p >= 1) where θ solves the handle's
 * current system A θ = b: PBiCGSTAB! from the handle's θ to tol (θ is left at the solution),
 * then one adjoint solve A λa = dJ/dθ with the same solver (A is symmetric), then
 *   dJ_dhsrc[c]  = -V_c λa_c                  (b = -(hsrc·V + ...), calRHS!)
 *   dJ_dlnlam[c] = dJ / d ln λ_c              (λ_c scaled with its isothermal guard copy)
 * as column-major host arrays (nullable; guards 0).  out_fwd / out_adj (nullable) receive the
 * two solves' results. */
int h2g_adjoint(h2g_solver *h, const double *weights, double p, double tol, int maxItr, int smoother, double *J,
                double *dJ_dhsrc, double *dJ_dlnlam, h2g_result *out_fwd, h2g_result *out_adj);

/* Transient form (no reference counterpart): J = (sum_c w_c θ_c^p)^(1/p) on θ after nt steps of
 * h2g_transient (b rebuilt per step, PBiCGSTAB! from the previous θ; transient grid with ρ, cp
 * and the handle's hsrc, boundary set bc[6]), from the handle's θ as θ^0.  Gradients summed over
 * the steps, through the adjoint recursion mu = A^-1 lam, lam <- (db/dθ) mu.  The forward states
 * are kept every checkpoint_every steps and recomputed per segment (device memory:
 * ceil(nt/checkpoint_every) + checkpoint_every + 1 state vectors).  θ is left at θ^nt.  out.itr
 * counts the iterations of all forward, recomputed and adjoint solves. */
int h2g_adjoint_transient(h2g_solver *h, const h2g_bc *bc, int nt, const double *weights, double p, double tol,
                          int maxItr, int smoother, int checkpoint_every, double *J, double *dJ_dhsrc,
                          double *dJ_dlnlam, h2g_result *out);

/* ---- right-hand side and time stepping ---------------------------------------------------
 * wk.hsrc (src/common.jl:64, filled by HeatSrc!): volumetric heat source in W/m^3, guard layers
 * included.  A handle without one uses zero. */
int h2g_set_hsrc(h2g_solver *h, const double *hsrc);
/* calRHS!(wk, Δh, Δt, ΔZ, bc_set, qsrf, par; is_steady) (src/NonUniform.jl:57-91) with
 * apply_bc2RHS! (src/RHS.jl:23-192) on the device, with the handle's θ, hsrc, ρ·cp and grid:
 * the boundary terms of bc[6] (x-, x+, y-, y+, z-, z+; heat flux ±q·area, convection
 * ∓h·area·(θ∞ − θ), isothermal nothing) are added to b in that order, then
 * b = −(a_p0·θ + hsrc·dx·dy·dz + b) over the interior.  zero_b = 0 accumulates into the current
 * b as the reference does; zero_b = 1 starts from b = 0 (a step of a multi-step run). */
int h2g_calrhs(h2g_solver *h, const h2g_bc *bc, int zero_b);
/* The time loop of main() (src/heat3ds.jl:123-151) with θ resident on the device: nt steps of
 * [h2g_calrhs(zero_b = 1); PBiCGSTAB!/CG! (method 0/1) from the previous θ].  step_stats
 * (nullable, 5*nt doubles) receives per step the interior θmin, θmax, ||θ||_2 (the log.txt line,
 * heat3ds.jl:149-151), the iterations and the final relative residual.  out: itr = iterations of
 * all steps, outer = steps run, isconverged = every step converged, res0/res of the last step.
 * A step that does not converge is reported and the loop goes on (heat3ds.jl:144-146); a
 * non-finite residual ends it. */
int h2g_transient(h2g_solver *h, const h2g_bc *bc, int nt, int method, double tol, int maxItr, int smoother,
                  int verbose, double *step_stats, h2g_result *out);

/* ---- launch-shape tuning (no reference counterpart) ---------------------------------------
 * The smoother's colour pass has no reduction, so its launch variant changes no result.  The
 * first solve of a handle times blocks of 2, 4, 8 and 16 rows with 1 or 2 planes per thread and
 * three sources of a cell's coefficients (a few sweeps each on scratch vectors) and keeps the
 * fastest; it also times the FP64 CalcAX with each source (the same bits in every case).  The
 * sources: 0 the key tables with dd summed per cell, 1 the key tables with dd read from a
 * per-cell array, 2 the stencil-class table (the FP64 kernels and the FP32 smoother): the
 * distinct (plane, 7 stencil keys) pairs of the grid, at most 65535 and NZ <= 255 (else not
 * built; H2G_CLS=0 disables it), each with its coefficients, and a 2-byte class index per cell.  The choices are cached per grid size and
 * smoother precision for the process; H2G_RB_ROWS, H2G_RB_PLANES, H2G_RB_DD and H2G_AX_DD
 * (sources 0/1/2) in the environment force them (all four: no timing at all; a forced rows,
 * planes or source restricts the timing to it).  h2g_autotune runs the tuner now and reports its
 * choices (each pointer nullable): the colour pass's rows and planes and its source (*rb_dd), and
 * CalcAX's source (*ax_dd).  h2g_set_tuning forces a shape (rows 2, 4, 8 or 16 and planes 1 or
 * 2; rows = 0: tune again on the next solve). */
int h2g_autotune(h2g_solver *h, int *rows, int *planes, int *rb_dd, int *ax_dd);
int h2g_set_tuning(h2g_solver *h, int rows, int planes);
/* The preconditioner's sweeps 2-5 as one fused launch each (k_rb_sweep: both colours of a sweep,
 * planes of x and keys staged in shared memory by TMA, z-marching, results bit-identical to the
 * colour passes) or as two colour passes each.  The tuner times the fused sweep for several
 * numbers of z chunks, with dd summed or read, against the best colour-pass shape and keeps the
 * faster (H2G_RB_FUSED, H2G_SW_CHUNKS, H2G_SW_DD in the environment force it).  h2g_set_sweep forces
 * the choice on a handle: fused 0 (colour passes), 1 (fused, with `chunks` z chunks, 1..255, and
 * dd read from the per-cell array if dd_array) or -1 (tune again); h2g_get_sweep reports what the
 * next solve uses.  No reference counterpart (rbsor!, NonUniform.jl:936-957, runs the colours one
 * after another over the whole grid). */
int h2g_set_sweep(h2g_solver *h, int fused, int chunks, int dd_array);
int h2g_get_sweep(h2g_solver *h, int *fused, int *chunks, int *dd_array);
/* The whole preconditioner of a PBiCGSTAB iteration (first pass and 9 colour passes) as one
 * cooperative launch with a bounded grid barrier between passes (k_precond_coop), instead of ten
 * launches; results bit-identical.  FP64 handles on the colour-pass path only.  mode 1 on, 0 off,
 * -1 default (off unless H2G_RB_COOP=1 in the environment).  h2g_batch_solve runs its handles
 * without it while more than one solve is in flight (a cooperative launch needs the device to
 * itself; beside another cooperative launch a barrier would wait until its budget ran out).
 * h2g_get_coop reports what the next solve uses.  No reference counterpart. */
int h2g_set_coop(h2g_solver *h, int mode);
int h2g_get_coop(h2g_solver *h, int *on);
/* Budget of one bounded device wait (the fused sweep's waits for its TMA copies, the cooperative
 * preconditioner's grid barriers), in SM clock cycles; default about one second.  0 makes every
 * such wait give up at once: the solve then ends with H2G_TIMEOUT, copies in flight are drained
 * and the context stays usable (the failure path of the bounded waits, exercised by the tests
 * without a GPU fault). */
int h2g_set_wait_limit(h2g_solver *h, long long cycles);

/* ---- kernels of the path, callable one at a time (host arrays in and out) ---------------
 * CalcAX! (NonUniform.jl:454-511): ax = A x over the interior; guard cells of ax are 0. */
int h2g_calcax(h2g_solver *h, const double *x, double *ax);
/* CalcRK! (NonUniform.jl:372-434): r = b - A θ with the handle's θ and b; *res = ||r||_2. */
int h2g_calcrk(h2g_solver *h, double *r, double *res);
/* rbsor_core! (NonUniform.jl:848-915): one colour pass (color 0 or 1) of RB-SOR with
 * relaxation omega on x (in/out) with right-hand side b. */
int h2g_rbsor_pass(h2g_solver *h, double *x, const double *b, int color, double omega);
/* Preconditioner! (NonUniform.jl:531-559): xx = M^-1 bb, xx starting from zero. */
int h2g_preconditioner(h2g_solver *h, const double *bb, double *xx, int smoother);

/* ---- device-resident timing hooks (for benchmarks) --------------------------------------
 * Run `reps` back-to-back launches of one kernel class on the handle's resident data, on the
 * handle's stream, without synchronising: kind 0 = one RB-GS sweep (both colours) of the
 * preconditioner, kind 1 = CalcAX.  Returns the number of kernel launches issued in *launches. */
int h2g_bench_kernel(h2g_solver *h, int kind, int reps, int *launches);

/* ---- CalcRK! without device allocation -------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory: the device
 * memory belongs to someone else (a Julia program's CUDA.jl pool, a framework's caching
 * allocator), or the caller runs a time-stepping loop that must not stall on cudaMalloc/cudaFree.
 * Computes
 * r = b - A theta over the interior and *res = ||r||_2 exactly as h2g_calcrk, from the
 * reference's column-major arrays already in device memory (theta, b, lambda, mask, rho, cp: MX*MY*MZ
 * doubles; ZC, dZ: MZ doubles; rho and cp may be NULL when is_steady) and HC[6] on the host;
 * r (device, MX*MY*MZ) gets the interior, guard cells are left untouched.  Nothing is allocated:
 * the reduction uses a 512 KiB device array inside the library that every GPU loading it keeps
 * until exit, so grids with more than 65536 interior rows (NY*NZ) are rejected (H2G_BAD_ARG).
 * Calls share that array: calls that overlap on the GPU race and must be serialised.  The first
 * call on a device looks up the array's address.  stream may be NULL (legacy default stream); the
 * call copies *res to the host and synchronises the stream before it returns, so it must not be
 * issued while that stream is capturing a CUDA graph. */
int h2g_calcrk_noalloc(int MX, int MY, int MZ, const double *theta, const double *b, const double *lambda,
                       const double *mask, const double *rho, const double *cp, const double *ZC, const double *dZ,
                       double dx, double dy, double dt, const double *HC, int is_steady, double *r, double *res,
                       void *stream);

/* ---- the reference's problem set-up (what q3d does before the solve) ---------------------
 * genZ! (src/Zcoord.jl:133-166) for NZ = 30*m: Z (NZ+3 faces with extrapolated guards), ZC and dZ
 * (NZ+2 each).  m > 1 splits each of the 30 Zcase2! cells (Zcoord.jl:88-124) into m equal
 * sub-cells; the reference itself only supports NZ = 30. */
int h2g_model_zgrid(int NZ, double *Z, double *ZC, double *dZ);
/* dx = round(1.2e-3/N, digits=8) (src/heat3ds.jl:197-200). */
double h2g_model_pitch(int N);
/* fillID! (src/modelA.jl:545-556) on the GPU: the uint8 material-ID field of the IC stack for an
 * (NX+2, NY+2, NZ+2) grid, written to the host array ID (column-major); bit-identical to the
 * reference's 50^3-sample volume tests. */
int h2g_model_fill_id(int NX, int NY, int NZ, uint8_t *ID);

#ifdef __cplusplus
}
#endif
#endif /* H2G_H */
