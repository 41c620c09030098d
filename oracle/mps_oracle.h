/*
 * mps_oracle.h -- FP64 CPU restatement of the mps3d mgridlib linear-solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * implementation is compared against; it is never linked into, loaded by or
 * called from the product library (mps3d_b200/).  Only tests/, the smoke()
 * check in __graft_entry__.py and the cpu_baseline leg of bench.py use it.
 *
 * Two layers:
 *   (A) a literal restatement of the reference Fortran (ghosted arrays in
 *       Fortran order, find_AX / find_bvec / red-black Gauss-Seidel / FAS
 *       V-cycle / GMRES bottom solve), each function citing the reference
 *       file:line it follows;
 *   (B) extensions the reference does not have (periodic faces, the
 *       "geom" hierarchy for any size (ceil coarsening, exact cell widths,
 *       trilinear prolongation), Scharfetter-Gummel rows taken
 *       from the 1D code, transposed operators, right-preconditioned FGMRES),
 *       built on an explicit 7-point row representation and checked against
 *       layer (A) where the two overlap.
 *
 * Parity pinning: the reference cannot be compiled here (Fortran/MPI, no
 * gfortran or mpif90 in the image).  The restatement is pinned by the
 * reference's own known-answer decks (tests/Laplace_test: phi = x exactly;
 * tests/gpde_test: steady phi = 0.5(x^2 - x)), see tests/test_oracle_kat.py.
 */
#ifndef MPS_ORACLE_H
#define MPS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Face order and BC codes follow globalvars.f90:11-17 and the character(4)
 * codes of discretepde.f90 ('DIRC','FLUX','ZGRD'); PERI is an extension. */
enum { ORC_LEFT = 0, ORC_RIGHT, ORC_BOTTOM, ORC_TOP, ORC_BACK, ORC_FRONT };
enum { ORC_DIRC = 1, ORC_FLUX = 2, ORC_ZGRD = 3, ORC_PERI = 4, ORC_DZGD = 5 };
enum { ORC_HIER_CELL = 0, ORC_HIER_GEOM = 1 };
enum { ORC_FLUX_UPWIND = 0, ORC_FLUX_SG = 1 };

typedef struct {
    int lx, ly, lz;                 /* cells per direction */
    double llenx, lleny, llenz;     /* physical lengths */
    int px, py, pz;                 /* rank layout (CELL hierarchy coarsest rule) */
    int hier;                       /* ORC_HIER_CELL or ORC_HIER_GEOM */
    int max_coarse;                 /* GEOM: coarsen while cells > max_coarse */
    int nu1, nu2;                   /* pre/post smoothing sweeps (reference: 2,2) */
} orc_grid;

/* ---- layer (A): literal restatement (ghosted Fortran-order arrays) ---- */
void orc_find_AX(const orc_grid* g, const double* soln, int timederiv, double dt,
                 const double* vel, const double* dcoeff, const double* reac,
                 const int* bc, double* AX, double* diag, double* offdiag);
void orc_find_bvec(const orc_grid* g, const double* vel, const double* dcoeff,
                   const double* source, const int* bc, const double* const* bcvals,
                   const double* mgridsource, int applybc, double* b);
void orc_gs_smooth(const orc_grid* g, double* soln, int timederiv, double dt,
                   int applybc, const double* mgridsource, double* res,
                   const double* vel, const double* dcoeff, const double* reac,
                   const double* source, const int* bc, const double* const* bcvals,
                   int niter);
int orc_vcycle(const orc_grid* g, double* soln, int timederiv, double dt,
               const double* vel, const double* dcoeff, const double* reac,
               const double* source, const int* bc, const double* const* bcvals,
               const double* mgridsterm, double* resnorm);
/* caller loop (poissoneq.f90:427-450 / pdedefs.f90:304-328) extended with
 * a relative-residual stop; returns cycles used, fills rel/rms histories */
int orc_solve(const orc_grid* g, double* soln, int timederiv, double dt,
              const double* vel, const double* dcoeff, const double* reac,
              const double* source, const int* bc, const double* const* bcvals,
              int maxit, double tol, int tol_kind, double* rel_hist, double* rms_hist);
double orc_rel_residual(const orc_grid* g, const double* soln, int timederiv, double dt,
                        const double* vel, const double* dcoeff, const double* reac,
                        const double* source, const int* bc, const double* const* bcvals,
                        double* rms_out);
void orc_fill_ghosts(const orc_grid* g, double* soln, const int* bc,
                     const double* const* bcvals);

/* ---- layer (B): 7-point rows (extension machinery) ----
 * rows layout: 7 interior arrays [d, xm, xp, ym, yp, zm, zp], each lx*ly*lz,
 * i fastest; A u (c) = d u_c + xm u_{c-x} + xp u_{c+x} + ...  (periodic
 * neighbours wrap; off-domain coefficients are zero). */
void orc_build_rows(const orc_grid* g, int flux, int timederiv, double dt,
                    const double* vel, const double* dcoeff, const double* reac,
                    const int* bc, double* rows);
void orc_build_rhs(const orc_grid* g, int flux, const double* vel, const double* dcoeff,
                   const double* source, const int* bc, const double* const* bcvals,
                   double* b);
void orc_rows_apply(const orc_grid* g, const int* bc, const double* rows,
                    const double* u, double* Au);
void orc_rows_transpose(const orc_grid* g, const int* bc, const double* rows, double* rowsT);
/* gradients of lam^T A(vel, dcoeff, reac) u (interior lam, u; uniform grid)
 * with respect to vel (3 x interior), dcoeff and reac (interior) */
void orc_operator_vjp(const orc_grid* g, int flux, const double* vel, const double* dcoeff, const int* bc,
                      const double* lam, const double* u, double* gvel, double* gd, double* greac);
void orc_sg_face_d(double cL, double cR, double DL, double DR, double dx, double* dwL, double* dwR);
void orc_sg_face(double cL, double cR, double DL, double DR, double dx,
                 double* wL, double* wR);
/* correction-scheme V-cycle over rows operators (coarse rows rediscretised
 * from restricted vel/dcoeff/reac); u interior, f interior */
typedef struct orc_mg orc_mg;
orc_mg* orc_mg_create(const orc_grid* g, int flux, int timederiv, double dt,
                      const double* vel, const double* dcoeff, const double* reac,
                      const int* bc, int transpose);
void orc_mg_destroy(orc_mg* mg);
int orc_mg_levels(const orc_mg* mg, int* dims /* 3*levels */);
void orc_mg_vcycle(orc_mg* mg, double* u, const double* f);
const double* orc_mg_rows(const orc_mg* mg, int level);
/* right-preconditioned FGMRES(m), FP64, preconditioner = one V-cycle */
int orc_fgmres(orc_mg* mg, const double* b, double* x, int m, int maxit, double tol,
               double* relres_out);
/* stationary V-cycle iteration on rows operators: x += V(b - A x) */
int orc_mg_solve(orc_mg* mg, const double* b, double* x, int maxit, double tol,
                 double* relres_out);

/* OpenMP threads of the oracle's parallel loops (<= 0: unchanged) */
void orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
