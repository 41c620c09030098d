/*
 * mps_linsolve.h -- C ABI of the B200 multigrid / Krylov linear solver for the
 * mps3d 7-point finite-volume operators.
 *
 * The entry points replace the solver calls of the reference's equation
 * modules (plain C types only: no CUDA or torch types in the signatures; the
 * stream of the *_dev variants is a cudaStream_t passed as void*).
 *
 * Streams: a handle runs its work on its own non-blocking stream.  A *_dev
 * call given the caller's stream orders that work after what the caller's
 * stream has queued (the inputs) and makes the caller's stream wait for it
 * (the outputs).  NULL means the handle's stream itself, with no ordering
 * against any other stream; for the legacy default stream (torch's default
 * stream, among others) pass cudaStreamLegacy, ((void*)0x1), not NULL.
 * Entry points without a handle queue their work on `stream` itself (NULL is
 * then the legacy default stream).
 *
 * Entry points:
 *
 *   mps_vcycle_once   <- perform_vcycle, mgridlib/mgridsteps.f90:384-417
 *                        (one call, same arguments and in/out meaning)
 *   mps_linsolve      <- the caller loop "do i=1,nvcycles; call perform_vcycle;
 *                        if(resnorm .le. err_tol) exit" of
 *                        plasma_pde/poissoneq.f90:427-450,
 *                        plasma_pde/edeneq.f90:489-503, plasma_pde/ionseq.f90:600-614,
 *                        plasma_pde/eenergyeq.f90:817-829,
 *                        plasma_pde/neutralseq.f90:481-494, generic_pde/pdedefs.f90:304-328
 *   mps_apply_A       <- find_AX, mgridlib/discretepde.f90:672-1119 (AX only)
 *   mps_find_bvec     <- find_bvec, mgridlib/discretepde.f90:382-618 (applybcflag=.true.)
 *   mps_fill_ghosts   <- update_boundary_ghostvalues, mgridlib/discretepde.f90:1121-1267
 *
 * Array conventions are the reference's: real*8 fields ghosted by one layer
 * (-g_nglayers+1 : l+g_nglayers, par_decompose.f90:18) in Fortran order
 * (i fastest); vel carries a trailing NDIM=3 axis; face arrays are
 * left/right (ly,lz), bottom/top (lx,lz), back/front (lx,ly)
 * (globalvars.f90:57-66); faces are ordered LEFT, RIGHT, BOTTOM, TOP, BACK,
 * FRONT (globalvars.f90:11-17).  The reference's character(4) codes map to
 * the MPS_BC_* integers below.
 *
 * Errors are returned as an integer status; the library never aborts, traps
 * or exits (the reference calls abort()/MPI_Abort at gmres.f90:398 and
 * mgridsteps.f90:359).
 */
#ifndef MPS_LINSOLVE_H
#define MPS_LINSOLVE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
enum mps_status {
    MPS_OK = 0,
    MPS_ERR_NOT_CONVERGED = 1, /* maxit reached; the reference silently accepts this */
    MPS_ERR_NAN = 2,           /* NaN/Inf in a residual or Krylov quantity (gmres.f90:113-120) */
    MPS_ERR_BREAKDOWN = 3,     /* singular coarse operator or Krylov breakdown */
    MPS_ERR_BAD_ARG = 4,
    MPS_ERR_TIMEOUT = 5,       /* a bounded device-side wait expired */
    MPS_ERR_CUDA = 6,
    MPS_ERR_NOMEM = 7,
    MPS_ERR_TOO_LARGE = 8      /* grid beyond MPS_NOALLOC_MAX_CELLS (mps_apply_A_noalloc) */
};

/* ---- boundary-condition codes (discretepde.f90; PERI is an extension) ---- */
enum { MPS_BC_DIRC = 1, MPS_BC_FLUX = 2, MPS_BC_ZGRD = 3, MPS_BC_PERI = 4, MPS_BC_DZGD = 5 };

enum { MPS_HIER_CELL = 0,      /* reference hierarchy: l/2 by integer division,
                                  8-cell average, central-slope prolongation,
                                  coarsest when a per-rank size reaches LMIN=1 */
       MPS_HIER_GEOM = 1 };    /* any size: l/2 cells with the odd cell merged into the
                                  last coarse cell, exact cell widths, volume-weighted
                                  restriction, trilinear prolongation (extension) */
enum { MPS_PREC_FP64 = 0, MPS_PREC_MIXED = 1 };  /* MIXED: FP32 V-cycle inside FP64 refinement */
enum { MPS_KRYLOV_NONE = 0, MPS_KRYLOV_FGMRES = 1 };
enum { MPS_FLUX_UPWIND = 0, MPS_FLUX_SG = 1 };
enum { MPS_TOL_RMS_ABS = 0,    /* sqrt(sum r^2 / ncells) <= tol (compute_norm, globalvars.f90:136-159) */
       MPS_TOL_REL_L2 = 1 };   /* ||b - A x||_2 / ||b||_2 <= tol */

typedef struct {
    int lx, ly, lz;                /* cells per direction (g_lx, g_ly, g_lz) */
    double llenx, lleny, llenz;    /* box lengths (g_llenx, ...; dx = llenx/lx) */
} mps_grid;

typedef struct {
    double tol;          /* default 1e-10 */
    int tol_kind;        /* MPS_TOL_*; default REL_L2 */
    int maxit;           /* outer iterations (V-cycles or FGMRES steps); default 50 */
    int nu1, nu2;        /* pre/post red-black GS sweeps; default 2,2 (mgridsteps.f90:473) */
    int hierarchy;       /* MPS_HIER_*; default GEOM */
    int ranks[3];        /* CELL only: rank layout px,py,pz fixing the coarsest level; default 1,1,1 */
    int max_coarse;      /* GEOM only: coarsen while a level has more cells; default 125 */
    int precision;       /* MPS_PREC_*; default FP64 */
    int inner_cycles;    /* MIXED: FP32 V-cycles per FP64 refinement step; default 0 = automatic */
    int krylov;          /* MPS_KRYLOV_*; default NONE (stationary V-cycle iteration) */
    int restart;         /* FGMRES restart length m; default 30 */
    int fill_ghosts;     /* 1: write solution ghosts like update_boundary_ghostvalues; default 0 */
    int use_graph;       /* 1: replay the V-cycle as a CUDA graph; default 1 */
    int transpose;       /* 1: solve with A^T (adjoint); default 0 */
    int flux;            /* MPS_FLUX_*: convective flux of the operator; default UPWIND
                            (find_AX); SG = Scharfetter-Gummel faces
                            (mps1d/source/convdiff.f90:10-64) */
} mps_solver_opts;

typedef struct {
    int status;          /* mps_status of the solve */
    int iters;           /* outer iterations done */
    int vcycles;         /* V-cycles done (all precisions) */
    int levels;          /* multigrid levels including the coarsest */
    double rel_res;      /* final ||b - A x||_2 / ||b||_2 (FP64) */
    double rms_res;      /* final sqrt(sum r^2 / ncells), the reference's norm */
    double rel_res0;     /* initial relative residual */
    double time_ms;      /* device time of the solve (CUDA events) */
    int launches;        /* kernels launched by the solve */
} mps_solve_info;

/* per-kernel-class device time of the finest level, accumulated over solves
 * while profiling is on (CUDA events around each launch on the handle's
 * stream) */
enum { MPS_PROF_SMOOTH = 0,   /* red-black colour passes, finest level */
       MPS_PROF_RESTRICT = 1, /* fused residual + restriction, finest level */
       MPS_PROF_PROLONG = 2,  /* fused prolongation + correction, finest level */
       MPS_PROF_RESID = 3,    /* FP64 residual + norm of the outer iteration */
       MPS_PROF_NCLASS = 8 };
typedef struct {
    int count[MPS_PROF_NCLASS];
    double ms[MPS_PROF_NCLASS];
    int precision_bytes;  /* word size of the V-cycle (8 FP64, 4 mixed) */
    int coeff_field;      /* 1 when the finest-level operator reads a cell coefficient field */
    long long cells;      /* finest-level cells */
} mps_profile;

typedef struct mps_handle_s* mps_handle;

/* defaults listed in mps_solver_opts */
void mps_default_opts(mps_solver_opts* o);
/* library version string */
const char* mps_version(void);

/* A handle owns a CUDA stream and the device workspace (level hierarchy,
 * coefficient pyramid, Krylov basis), reused across calls with the same grid.
 * device < 0 selects the current device. */
int mps_create(mps_handle* h, int device);
int mps_destroy(mps_handle h);
/* the handle's stream (cudaStream_t) */
void* mps_stream(mps_handle h);
/* text of the last error seen by the handle ("" when none) */
const char* mps_last_error(mps_handle h);

/* Solve A soln = b with b = find_bvec(applybcflag=.true.) + mgridsterm.
 * Host pointers (Fortran-order ghosted arrays, copied to and from the device
 * inside the call).  vel, reac and mgridsterm may be NULL (zero).  soln holds
 * the initial guess on entry and the solution on exit (interior; ghosts too
 * when opts->fill_ghosts).  Replaces the caller loop around perform_vcycle. */
int mps_linsolve(mps_handle h, const mps_grid* g, int timederiv, double dt,
                 const double* vel, const double* dcoeff, const double* reac,
                 const double* source, const int bc_code[6], const double* const bcval[6],
                 const double* mgridsterm, double* soln, const mps_solver_opts* opts,
                 mps_solve_info* info);

/* Same with device pointers, ordered with `stream` (cudaStream_t; NULL = the
 * handle's stream, unordered with other streams; see the top of this file);
 * no host<->device copies of the fields. */
int mps_linsolve_dev(mps_handle h, const mps_grid* g, int timederiv, double dt,
                     const double* vel, const double* dcoeff, const double* reac,
                     const double* source, const int bc_code[6], const double* const bcval[6],
                     const double* mgridsterm, double* soln, const mps_solver_opts* opts,
                     mps_solve_info* info, void* stream);

/* Exactly one V-cycle with perform_vcycle's meaning (host pointers):
 * soln in/out (ghosted), resnorm out = RMS norm of the post-smoothing
 * residual (mgridsteps.f90:575).  opts may be NULL (CELL hierarchy, 2/2 sweeps). */
int mps_vcycle_once(mps_handle h, const mps_grid* g, int timederiv, double dt,
                    const double* vel, const double* dcoeff, const double* reac,
                    const double* source, const int bc_code[6], const double* const bcval[6],
                    const double* mgridsterm, double* soln, double* resnorm,
                    const mps_solver_opts* opts);

/* AX = A soln (interior, Fortran order), device pointers; opts selects the flux
 * scheme and transpose. */
int mps_apply_A_dev(mps_handle h, const mps_grid* g, int timederiv, double dt,
                    const double* vel, const double* dcoeff, const double* reac,
                    const int bc_code[6], const double* soln, double* AX,
                    const mps_solver_opts* opts, void* stream);

/* b = find_bvec (applybcflag=.true.) + mgridsterm, device pointers, interior out. */
int mps_find_bvec_dev(mps_handle h, const mps_grid* g, const double* vel, const double* dcoeff,
                      const double* source, const int bc_code[6], const double* const bcval[6],
                      const double* mgridsterm, double* b, const mps_solver_opts* opts,
                      void* stream);

/* Profiling of the smoothing and transfer kernels of one level (off by
 * default): on = 1 times the finest level, on = 1 + l level l; the residual
 * class is always the finest level's.  mps_get_profile returns the
 * accumulated figures and resets them when reset != 0. */
int mps_set_profile(mps_handle h, int on);
int mps_get_profile(mps_handle h, mps_profile* p, int reset);

/* Ghost layer of a ghosted field per update_boundary_ghostvalues (+ periodic
 * wrap), device pointers. */
int mps_fill_ghosts_dev(mps_handle h, const mps_grid* g, const int bc_code[6],
                        const double* const bcval[6], double* soln, void* stream);

/* One independent problem of a batched call (device pointers, as for
 * mps_linsolve_dev). */
typedef struct mps_problem {
    mps_grid g;
    int timederiv;
    double dt;
    const double* vel;      /* NULL or all zero: batched solves take the diffusion class */
    const double* dcoeff;
    const double* reac;
    const double* source;
    int bc_code[6];
    const double* bcval[6];
    const double* mgridsterm;
    double* soln;           /* in: initial guess, out: solution (ghosted) */
} mps_problem;

#define MPS_BATCH_MAX 4096

/* Solve nprob independent problems of any sizes together: one set-up per
 * problem, then every V-cycle step of all problems as one launch, the outer
 * iterations inside one CUDA graph whose loop ends on the device when every
 * problem has converged (or reached maxit).  Replaces a loop of
 * mps_linsolve_dev calls, i.e. a loop over the reference's per-equation solve
 * loops (poissoneq.f90:427-450 and its siblings) for independent systems.
 * opts apply to every problem: stationary iteration (krylov NONE),
 * precision MIXED (FP32 V-cycles, FP64 residual and update) or FP64,
 * nu1 >= 1 and nu1+nu2 even.  infos[p] (may be NULL) gets each problem's
 * result; the return value is MPS_OK unless a problem failed to set up
 * (its status) or produced NaN (MPS_ERR_NAN).  A call that repeats the
 * previous one's problems (same sizes, boundary codes, buffers and options,
 * and inputs of the same operator class: convection, reaction field,
 * uniform coefficient and its value, zero initial guess) replays the
 * per-problem set-up as a CUDA graph captured at the second such call; the
 * buffers' contents may change between calls. */
int mps_linsolve_batched_dev(mps_handle h, int nprob, const mps_problem* probs,
                             const mps_solver_opts* opts, mps_solve_info* infos, void* stream);

/* Adjoint of a solve, operator part (extension: the reference has no
 * adjoint).  Gradients of s = lam^T A(vel, dcoeff, reac) u with respect to the
 * operator's cell fields, for interior lam and u (Fortran order, lx*ly*lz):
 * gvel (3 x interior), gdcoeff, greac (interior); any output may be NULL.
 * With x = A^{-1} b and lam = A^{-T} dL/dx (mps_linsolve_dev with
 * opts->transpose = 1), dL/dtheta = -(this result).  vel may be NULL; opts
 * selects the flux (NULL = upwind); uniform grid (dx = llen/l).  Queued on
 * `stream` (NULL = default stream), not waited for; allocates nothing.
 * The dependence of b on the fields (DIRC faces of SG operators) is not
 * included. */
int mps_operator_vjp_dev(const mps_grid* g, const double* vel, const double* dcoeff,
                         const int bc_code[6], const double* lam, const double* u,
                         const mps_solver_opts* opts, double* gvel, double* gdcoeff,
                         double* greac, void* stream);

/* ---- on-device operator assembly and the implicit plasma step ----------
 * The producers the reference runs on the host before each solve, as
 * kernels writing the solver's inputs (ghosted Fortran-order fields) in
 * device memory.  Queued on `stream` (NULL = the legacy default stream), not
 * waited for; they allocate nothing.  Mobility and diffusivity come in as
 * fields (the reference's chemistry tables are not part of this library). */

/* update_efield, plasma_pde/poissoneq.f90:565-680: first the ghosts of phi
 * (update_boundary_ghostvalues with the potential's codes and face values, in
 * place, :586-587), then E = -scale * grad(phi) by central differences
 * (:593-611; scale = potscale/lscale, :667), minmod-limited per direction
 * when limiter != 0 (gradient_limiter_flag, :614-662); efield = 3 ghosted
 * fields whose ghosts copy the first interior value (codes 'ZGRD', :582),
 * periodic faces wrapping. */
int mps_efield_dev(const mps_grid* g, const int phi_bc[6], const double* const phi_bcval[6], double* phi,
                   double scale, int limiter, double* efield, void* stream);

/* eden_update_transport, plasma_pde/edeneq.f90:360-444: vel = mu_e E *
 * scaling[0] (mu_e signed, negative for electrons), dcoeff = D * scaling[1]
 * (D = |mu_e| te when dco is NULL), source = prod * scaling[2] (prod may be
 * NULL) + n_old/dt when timederiv (:441); ghosts zero.  scaling NULL = 1,1,1
 * (SI units; the reference's vel/dcoeff/source_scaling, edeneq.f90:82-85). */
int mps_eden_transport_dev(const mps_grid* g, const double* efield, const double* mu_e, const double* dco,
                           const double* te, const double* prod, const double* n_old, int timederiv, double dt,
                           const double scaling[3], double* vel, double* dcoeff, double* source, void* stream);

/* poisson_update_transport, plasma_pde/poissoneq.f90:335-385: source =
 * (sum_s charge[s] n_ion[s] - n_e) * scale (scale = ECHARGE/EPS0 *
 * source_scaling) + phi_old/dt when phi_old is given (:382); n_ion holds
 * nspec ghosted fields one after another, charge is a device array. */
int mps_poisson_source_dev(const mps_grid* g, const double* n_e, int nspec, const double* n_ion,
                           const double* charge, double scale, const double* phi_old, double dt, double* source,
                           void* stream);

/* The potential and electron parts of one implicit time step
 * (plasma_pde/solve_manager.f90:363-502): Poisson source, potential solve,
 * E field, electron operator, implicit electron solve from n_old, the floor
 * n_e >= nemin and the electron ghosts (eden_solve, edeneq.f90:446-525).
 * All fields are device pointers in the reference's ghosted layout. */
typedef struct mps_plasma_step {
    mps_grid g;
    /* potential */
    int phi_bc[6];
    const double* phi_bcval[6];   /* face values of DIRC/FLUX faces */
    const double* eps;            /* permittivity: the Poisson operator's dcoeff */
    double* phi;                  /* in: initial guess; out: potential with its ghosts */
    double rho_scale;             /* ECHARGE/EPS0 * source_scaling */
    int nion;                     /* ion species in n_ion */
    const double* n_ion;          /* nion ghosted densities, one after another */
    const double* ion_charge;     /* nion charge numbers (device) */
    double* phi_source;           /* workspace: the Poisson source */
    /* electrons */
    int ne_bc[6];
    const double* ne_bcval[6];
    double* n_e;                  /* in: n_old; out: n_new, floored, ghosts set */
    const double* mu_e;           /* signed electron mobility */
    const double* d_e;            /* diffusivity, or NULL: |mu_e| te */
    const double* te;             /* electron temperature in volts (when d_e is NULL) */
    const double* prod_e;         /* production, or NULL */
    double dt;
    double nemin;                 /* floor of n_e */
    double efield_scale;          /* potscale/lscale; 1 in SI units */
    int limiter;                  /* 1: minmod-limited E */
    double vel_scaling, dcoeff_scaling, source_scaling;
    double* efield;               /* out: E (3 fields) */
    double* vel;                  /* out: electron drift (3 fields) */
    double* dcoeff;               /* out: electron diffusivity */
    double* source;               /* out: electron source */
} mps_plasma_step;

/* hp solves the potential (opts_phi), he the electrons (opts_e: typically
 * flux SG with FGMRES); two handles keep both workspaces resident.  The step
 * is ordered on `stream` (NULL = the legacy default stream).  Returns the
 * first failing status (MPS_ERR_NOT_CONVERGED of a solve is passed on after
 * the step completes). */
int mps_plasma_step_dev(mps_handle hp, mps_handle he, const mps_plasma_step* step,
                        const mps_solver_opts* opts_phi, const mps_solver_opts* opts_e,
                        mps_solve_info* info_phi, mps_solve_info* info_e, void* stream);

/* ---- VTK output from device buffers (mgridlib/cartwrite.f90) ------------
 * The reference's RectilinearGrid files byte for byte: XML header, raw
 * appended Float64 cell data (4-byte size, then the interior in Fortran
 * order), node coordinates off + (i-1) len/l.  fields are ghosted device
 * arrays (their interiors are written); names are C strings (trailing blanks
 * dropped, as Fortran's trim does).  The cell data are gathered and copied
 * on `stream` (NULL = the legacy default stream) while the previous field is
 * written; the call returns when the file is complete. */

/* Writeserialvtrfile, cartwrite.f90:8-161: <filename>.vtr; off may be NULL (0). */
int mps_write_vtr_dev(const char* filename, const mps_grid* g, const double off[3], int nscalars,
                      const char* const* names, const double* const* fields, void* stream);
/* Writevtrfile, cartwrite.f90:163-317: <dirname>/file_<rank, 8 digits>.vtr,
 * the piece of rank `rank` at 1-based block index pind (g = the piece's own
 * cells and lengths, off = its origin). */
int mps_write_vtr_piece_dev(const char* dirname, int rank, const int pind[3], const mps_grid* g,
                            const double off[3], int nscalars, const char* const* names,
                            const double* const* fields, void* stream);
/* Writepvtrfile, cartwrite.f90:319-438: creates dirname and writes
 * <dirname>.pvtr, the index of px*py*pz pieces of lx*ly*lz cells (host only). */
int mps_write_pvtr(const char* dirname, const int lxyz[3], const int pxyz[3], int nscalars,
                   const char* const* names);

/* AX = A soln like mps_apply_A_dev, for callers that must not allocate device
 * memory.  No counterpart in the reference: its find_AX works on arrays the
 * caller already owns, so it never needed one.  Callers that cannot allocate
 * are, for example, a time-stepping code whose memory pool (its own or
 * torch's caching allocator) already holds the free HBM, so that cudaMalloc
 * would fail, and a code that keeps the device busy on its own streams, which
 * cudaFree would stall by waiting for the whole device.
 *
 * No handle: the call works on the current device and calls no cudaMalloc,
 * cudaFree or allocating library routine.  Its scratch is one static device
 * array of MPS_NOALLOC_SCRATCH_BYTES (32 MiB).  The CUDA runtime reserves it
 * on a device when it loads this library's code there -- under the default
 * lazy module loading that is the first mps_apply_A_noalloc call on that
 * device (with CUDA_MODULE_LOADING=EAGER, the creation of the device's
 * context) -- and keeps it until the process exits.  That first call also
 * looks up the array's address on the device.  So make the first call on
 * each device early: before the caller's memory pool takes the free HBM
 * (else the reservation itself can fail, as MPS_ERR_CUDA) and before any
 * stream capture begins.  Sizes: round_up(lx, 16) * ly * lz must not
 * exceed MPS_NOALLOC_MAX_CELLS (64^3), else MPS_ERR_TOO_LARGE and nothing is
 * launched.  The work is queued on `stream` (NULL = the default stream) and
 * AX is ready when the stream reaches that point.  All calls share the one
 * array, so two calls that overlap on the GPU (other streams, other host
 * threads) race and corrupt each other's results: serialise them.  opts may
 * be NULL (upwind flux, no transpose); only its flux and transpose are read. */
#define MPS_NOALLOC_MAX_CELLS 262144
#define MPS_NOALLOC_SCRATCH_BYTES (16LL * 8LL * MPS_NOALLOC_MAX_CELLS)
int mps_apply_A_noalloc(const mps_grid* g, int timederiv, double dt, const double* vel,
                        const double* dcoeff, const double* reac, const int bc_code[6],
                        const double* soln, double* AX, const mps_solver_opts* opts, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MPS_LINSOLVE_H */
