/*
 * mps_oracle.c -- FP64 CPU restatement of the mps3d mgridlib linear solve.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Never part of the product path.
 *
 * Array conventions (identical to the reference):
 *   ghosted fields  (lx+2)(ly+2)(lz+2), Fortran order, index 0 and l+1 are
 *                   the ghost layers (g_nglayers = 1, par_decompose.f90:18);
 *   interior fields lx*ly*lz, Fortran order, 1-based (i,j,k) -> (i-1)+lx*(..);
 *   vel             3 ghosted fields back to back (vel(:,:,:,NDIM));
 *   bcvals[6]       left/right (ly,lz), bottom/top (lx,lz), back/front (lx,ly)
 *                   (globalvars.f90:57-66, allocate_bcvalues :201-222).
 * A periodic face (extension) is treated exactly like an MPI processor
 * boundary of the reference whose neighbour is the opposite side of the
 * domain: the face loop runs over it and the "ghost" values are read from the
 * wrapped interior cells (exchangehalodata, par_decompose.f90:122-296).
 */
#include "mps_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NEARZERO 1.0e-25 /* globalvars.f90:19 */
#define LMIN 1           /* globalvars.f90:23 */
#define ERRTOLR 1.0e-11  /* globalvars.f90:29 */

typedef struct { int lx, ly, lz; } dims3;

#define GX(i, j, k) ((long)(i) + (long)(lx + 2) * ((long)(j) + (long)(ly + 2) * (long)(k)))
#define IX(i, j, k) ((long)((i)-1) + (long)lx * ((long)((j)-1) + (long)ly * (long)((k)-1)))

static inline long ngh(int lx, int ly, int lz) { return (long)(lx + 2) * (ly + 2) * (lz + 2); }
static inline long nin(int lx, int ly, int lz) { return (long)lx * ly * lz; }

static inline int wrap1(int i, int n) { return i < 1 ? i + n : (i > n ? i - n : i); }

static double* zalloc(long n) { return (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

/* ======================================================================
 * layer (A): literal restatement
 * ==================================================================== */

/* findcellcontributions, discretepde.f90:620-670 */
static inline void cellcontrib(double soln_l, double soln_r, double k_l, double k_r,
                               double vel_l, double vel_r, double a_by_v, double d_lr,
                               double* diag_l, double* diag_r, double* off_l, double* off_r)
{
    double k_half, vel_half;
    *diag_l = 0.0; *diag_r = 0.0; *off_l = 0.0; *off_r = 0.0;
    k_half = 0.5 * (k_l + k_r);
    *diag_l = *diag_l + (k_half / d_lr) * a_by_v;
    *diag_r = *diag_r + (k_half / d_lr) * a_by_v;
    *off_l = *off_l - soln_r * (k_half / d_lr) * a_by_v;
    *off_r = *off_r - soln_l * (k_half / d_lr) * a_by_v;
    vel_half = 0.5 * (vel_l + vel_r);
    if (vel_half > 0.0) {
        *diag_l = *diag_l + vel_half * a_by_v;
        *off_r = *off_r - vel_half * soln_l * a_by_v;
    } else {
        *diag_r = *diag_r - vel_half * a_by_v;
        *off_l = *off_l + vel_half * soln_r * a_by_v;
    }
}

/* find_AX, discretepde.f90:672-1119.  Physical faces: lrank<0 etc. */
void orc_find_AX(const orc_grid* g, const double* soln, int timederiv, double dt,
                 const double* vel, const double* dcoeff, const double* reac,
                 const int* bc, double* AX, double* diag, double* offdiag)
{
    const int lx = g->lx, ly = g->ly, lz = g->lz;
    const double dx = g->llenx / lx, dy = g->lleny / ly, dz = g->llenz / lz;
    const long ng = ngh(lx, ly, lz), n = nin(lx, ly, lz);
    const double* velx = vel;
    const double* vely = vel + ng;
    const double* velz = vel + 2 * ng;
    const int perx = bc[ORC_LEFT] == ORC_PERI, pery = bc[ORC_BOTTOM] == ORC_PERI,
              perz = bc[ORC_BACK] == ORC_PERI;
    memset(AX, 0, sizeof(double) * n);
    memset(diag, 0, sizeof(double) * n);
    memset(offdiag, 0, sizeof(double) * n);

    /* X direction, :754-796 */
    {
        int imin = perx ? 0 : 1, imax = perx ? lx : lx - 1;
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= lz; k++)
            for (int j = 1; j <= ly; j++)
                for (int i = imin; i <= imax; i++) {
                    int lcell = i, rcell = i + 1;
                    int lw = perx ? wrap1(lcell, lx) : lcell, rw = perx ? wrap1(rcell, lx) : rcell;
                    double dl, dr, ol, orr;
                    cellcontrib(soln[GX(lw, j, k)], soln[GX(rw, j, k)], dcoeff[GX(lw, j, k)],
                                dcoeff[GX(rw, j, k)], velx[GX(lw, j, k)], velx[GX(rw, j, k)],
                                1.0 / dx, dx, &dl, &dr, &ol, &orr);
                    if (lcell > 0) { diag[IX(lcell, j, k)] += dl; offdiag[IX(lcell, j, k)] += ol; }
                    if (rcell <= lx) { diag[IX(rcell, j, k)] += dr; offdiag[IX(rcell, j, k)] += orr; }
                }
    }
    /* X boundaries, :798-865 */
    if (!perx) {
        for (int side = 0; side < 2; side++) {
            int code = bc[side], i = side == 0 ? 1 : lx;
            for (int k = 1; k <= lz; k++)
                for (int j = 1; j <= ly; j++) {
                    double vb = velx[GX(i, j, k)];
                    if (code == ORC_DIRC) {
                        diag[IX(i, j, k)] += 2.0 * dcoeff[GX(i, j, k)] / (dx * dx);
                        if (side == 0 && vb < 0.0) diag[IX(i, j, k)] -= vb / dx;
                        if (side == 1 && vb > 0.0) diag[IX(i, j, k)] += vb / dx;
                    } else if (code == ORC_ZGRD) {
                        if (side == 0) diag[IX(i, j, k)] -= vb / dx;
                        else diag[IX(i, j, k)] += vb / dx;
                    }
                }
        }
    }
    /* Y direction, :871-917 */
    {
        int jmin = pery ? 0 : 1, jmax = pery ? ly : ly - 1;
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= lz; k++)
            for (int j = jmin; j <= jmax; j++) {
                int lcell = j, rcell = j + 1;
                int lw = pery ? wrap1(lcell, ly) : lcell, rw = pery ? wrap1(rcell, ly) : rcell;
                for (int i = 1; i <= lx; i++) {
                    double dl, dr, ol, orr;
                    cellcontrib(soln[GX(i, lw, k)], soln[GX(i, rw, k)], dcoeff[GX(i, lw, k)],
                                dcoeff[GX(i, rw, k)], vely[GX(i, lw, k)], vely[GX(i, rw, k)],
                                1.0 / dy, dy, &dl, &dr, &ol, &orr);
                    if (lcell > 0) { diag[IX(i, lcell, k)] += dl; offdiag[IX(i, lcell, k)] += ol; }
                    if (rcell <= ly) { diag[IX(i, rcell, k)] += dr; offdiag[IX(i, rcell, k)] += orr; }
                }
            }
    }
    /* Y boundaries, :919-985 */
    if (!pery) {
        for (int side = 0; side < 2; side++) {
            int code = bc[2 + side], j = side == 0 ? 1 : ly;
            for (int k = 1; k <= lz; k++)
                for (int i = 1; i <= lx; i++) {
                    double vb = vely[GX(i, j, k)];
                    if (code == ORC_DIRC) {
                        diag[IX(i, j, k)] += 2.0 * dcoeff[GX(i, j, k)] / (dy * dy);
                        if (side == 0 && vb < 0.0) diag[IX(i, j, k)] -= vb / dy;
                        if (side == 1 && vb > 0.0) diag[IX(i, j, k)] += vb / dy;
                    } else if (code == ORC_ZGRD) {
                        if (side == 0) diag[IX(i, j, k)] -= vb / dy;
                        else diag[IX(i, j, k)] += vb / dy;
                    }
                }
        }
    }
    /* Z direction, :992-1034 (j outermost for threading; per-cell order kept) */
    {
        int kmin = perz ? 0 : 1, kmax = perz ? lz : lz - 1;
#pragma omp parallel for schedule(static)
        for (int j = 1; j <= ly; j++)
            for (int k = kmin; k <= kmax; k++) {
                int lcell = k, rcell = k + 1;
                int lw = perz ? wrap1(lcell, lz) : lcell, rw = perz ? wrap1(rcell, lz) : rcell;
                for (int i = 1; i <= lx; i++) {
                    double dl, dr, ol, orr;
                    cellcontrib(soln[GX(i, j, lw)], soln[GX(i, j, rw)], dcoeff[GX(i, j, lw)],
                                dcoeff[GX(i, j, rw)], velz[GX(i, j, lw)], velz[GX(i, j, rw)],
                                1.0 / dz, dz, &dl, &dr, &ol, &orr);
                    if (lcell > 0) { diag[IX(i, j, lcell)] += dl; offdiag[IX(i, j, lcell)] += ol; }
                    if (rcell <= lz) { diag[IX(i, j, rcell)] += dr; offdiag[IX(i, j, rcell)] += orr; }
                }
            }
    }
    /* Z boundaries, :1037-1100 */
    if (!perz) {
        for (int side = 0; side < 2; side++) {
            int code = bc[4 + side], k = side == 0 ? 1 : lz;
            for (int j = 1; j <= ly; j++)
                for (int i = 1; i <= lx; i++) {
                    double vb = velz[GX(i, j, k)];
                    if (code == ORC_DIRC) {
                        diag[IX(i, j, k)] += 2.0 * dcoeff[GX(i, j, k)] / (dz * dz);
                        if (side == 0 && vb < 0.0) diag[IX(i, j, k)] -= vb / dz;
                        if (side == 1 && vb > 0.0) diag[IX(i, j, k)] += vb / dz;
                    } else if (code == ORC_ZGRD) {
                        if (side == 0) diag[IX(i, j, k)] -= vb / dz;
                        else diag[IX(i, j, k)] += vb / dz;
                    }
                }
        }
    }
    /* reaction, time derivative, AX = diag*u + offdiag: :1102-1116 */
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) {
                long c = IX(i, j, k);
                diag[c] = diag[c] - reac[GX(i, j, k)];
                if (timederiv) diag[c] = diag[c] + 1.0 / dt;
                AX[c] = diag[c] * soln[GX(i, j, k)] + offdiag[c];
            }
}

/* find_bvec, discretepde.f90:382-618 */
void orc_find_bvec(const orc_grid* g, const double* vel, const double* dcoeff,
                   const double* source, const int* bc, const double* const* bcvals,
                   const double* mgridsource, int applybc, double* b)
{
    const int lx = g->lx, ly = g->ly, lz = g->lz;
    const double dx = g->llenx / lx, dy = g->lleny / ly, dz = g->llenz / lz;
    const long ng = ngh(lx, ly, lz), n = nin(lx, ly, lz);
    memset(b, 0, sizeof(double) * n);
    if (applybc) {
        for (int side = 0; side < 2; side++) { /* LEFT/RIGHT :428-486 */
            int code = bc[side], i = side == 0 ? 1 : lx;
            const double* bv = bcvals[side];
            if (code == ORC_DIRC) {
                for (int k = 1; k <= lz; k++)
                    for (int j = 1; j <= ly; j++) {
                        double vb = vel[GX(i, j, k)], gv = bv[(j - 1) + (long)ly * (k - 1)];
                        long c = IX(i, j, k);
                        b[c] = b[c] + 2.0 * dcoeff[GX(i, j, k)] * gv / (dx * dx);
                        if (side == 0 && vb > 0.0) b[c] = b[c] + vb * gv / dx;
                        if (side == 1 && vb < 0.0) b[c] = b[c] - vb * gv / dx;
                    }
            } else if (code == ORC_FLUX) {
                for (int k = 1; k <= lz; k++)
                    for (int j = 1; j <= ly; j++)
                        b[IX(i, j, k)] -= bv[(j - 1) + (long)ly * (k - 1)] / dx;
            }
        }
        for (int side = 0; side < 2; side++) { /* BOTTOM/TOP :488-546 */
            int code = bc[2 + side], j = side == 0 ? 1 : ly;
            const double* bv = bcvals[2 + side];
            if (code == ORC_DIRC) {
                for (int k = 1; k <= lz; k++)
                    for (int i = 1; i <= lx; i++) {
                        double vb = vel[ng + GX(i, j, k)], gv = bv[(i - 1) + (long)lx * (k - 1)];
                        long c = IX(i, j, k);
                        b[c] = b[c] + 2.0 * dcoeff[GX(i, j, k)] * gv / (dy * dy);
                        if (side == 0 && vb > 0.0) b[c] = b[c] + vb * gv / dy;
                        if (side == 1 && vb < 0.0) b[c] = b[c] - vb * gv / dy;
                    }
            } else if (code == ORC_FLUX) {
                for (int k = 1; k <= lz; k++)
                    for (int i = 1; i <= lx; i++)
                        b[IX(i, j, k)] -= bv[(i - 1) + (long)lx * (k - 1)] / dy;
            }
        }
        for (int side = 0; side < 2; side++) { /* BACK/FRONT :548-606 */
            int code = bc[4 + side], k = side == 0 ? 1 : lz;
            const double* bv = bcvals[4 + side];
            if (code == ORC_DIRC) {
                for (int j = 1; j <= ly; j++)
                    for (int i = 1; i <= lx; i++) {
                        double vb = vel[2 * ng + GX(i, j, k)], gv = bv[(i - 1) + (long)lx * (j - 1)];
                        long c = IX(i, j, k);
                        b[c] = b[c] + 2.0 * dcoeff[GX(i, j, k)] * gv / (dz * dz);
                        if (side == 0 && vb > 0.0) b[c] = b[c] + vb * gv / dz;
                        if (side == 1 && vb < 0.0) b[c] = b[c] - vb * gv / dz;
                    }
            } else if (code == ORC_FLUX) {
                for (int j = 1; j <= ly; j++)
                    for (int i = 1; i <= lx; i++)
                        b[IX(i, j, k)] -= bv[(i - 1) + (long)lx * (j - 1)] / dz;
            }
        }
    }
    /* :610-616 */
    for (long c = 0; c < n; c++) b[c] = b[c] + (mgridsource ? mgridsource[c] : 0.0);
    if (applybc)
        for (int k = 1; k <= lz; k++)
            for (int j = 1; j <= ly; j++)
                for (int i = 1; i <= lx; i++) b[IX(i, j, k)] += source[GX(i, j, k)];
}

/* red = odd (gi+gj+gk) with 1-based global indices (find_redblack_indices,
 * discretepde.f90:13-63); red is updated first (:207-227). */
static void colour_update(int lx, int ly, int lz, double* soln, const double* b,
                          const double* offdiag, const double* diag, int red)
{
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) {
                int odd = (i + j + k) & 1;
                if (odd == red) {
                    long c = IX(i, j, k);
                    soln[GX(i, j, k)] = (b[c] - offdiag[c]) / diag[c];
                }
            }
}

/* perform_gseidel_smoothing, discretepde.f90:132-236 */
void orc_gs_smooth(const orc_grid* g, double* soln, int timederiv, double dt,
                   int applybc, const double* mgridsource, double* res,
                   const double* vel, const double* dcoeff, const double* reac,
                   const double* source, const int* bc, const double* const* bcvals,
                   int niter)
{
    const int lx = g->lx, ly = g->ly, lz = g->lz;
    const long n = nin(lx, ly, lz);
    double* AX = zalloc(n);
    double* diag = zalloc(n);
    double* off = zalloc(n);
    double* b = zalloc(n);
    orc_find_bvec(g, vel, dcoeff, source, bc, bcvals, mgridsource, applybc, b);
    for (int it = 0; it < niter; it++) {
        orc_find_AX(g, soln, timederiv, dt, vel, dcoeff, reac, bc, AX, diag, off);
        colour_update(lx, ly, lz, soln, b, off, diag, 1);
        orc_find_AX(g, soln, timederiv, dt, vel, dcoeff, reac, bc, AX, diag, off);
        colour_update(lx, ly, lz, soln, b, off, diag, 0);
    }
    orc_find_AX(g, soln, timederiv, dt, vel, dcoeff, reac, bc, AX, diag, off);
    for (long c = 0; c < n; c++) res[c] = b[c] - AX[c];
    free(AX); free(diag); free(off); free(b);
}

/* ---- hierarchy sizes ----
 * CELL: lx/2 by integer division (mgridsteps.f90:21-23), stop when any local
 *       size (global / ranks) <= LMIN (:512).
 * GEOM (extension): l/2 coarse cells (pairs; for an odd size the last
 *       coarse cell takes three; a size of 1 stays 1); stop when the level
 *       holds <= max_coarse cells. */
static dims3 coarse_dims(const orc_grid* g, dims3 f)
{
    dims3 c;
    if (g->hier == ORC_HIER_CELL) {
        c.lx = g->px * ((f.lx / g->px) / 2);
        c.ly = g->py * ((f.ly / g->py) / 2);
        c.lz = g->pz * ((f.lz / g->pz) / 2);
    } else {
        c.lx = f.lx > 1 ? f.lx / 2 : 1;
        c.ly = f.ly > 1 ? f.ly / 2 : 1;
        c.lz = f.lz > 1 ? f.lz / 2 : 1;
    }
    return c;
}

static int is_coarsest(const orc_grid* g, dims3 d)
{
    if (g->hier == ORC_HIER_CELL)
        return (d.lx / g->px) <= LMIN || (d.ly / g->py) <= LMIN || (d.lz / g->pz) <= LMIN;
    return nin(d.lx, d.ly, d.lz) <= g->max_coarse ||
           (d.lx == 1 && d.ly == 1 && d.lz == 1);
}

/* Cell widths per level (GEOM hierarchy).  Coarse cells are pairs of fine
 * cells; when a size is odd the last coarse cell takes three.  Every level is
 * then uniform except for its last cell, whose width is tracked exactly:
 * w = regular width, wl = width of the last cell (wl/w -> 1 with depth).  The CELL hierarchy keeps the
 * reference's dx = llen/l at every level (find_AX, discretepde.f90:724-726). */
typedef struct { int n[3]; double w[3], wl[3]; } geo3;

static geo3 geo_fine(const orc_grid* g)
{
    geo3 G;
    G.n[0] = g->lx; G.n[1] = g->ly; G.n[2] = g->lz;
    const double L[3] = {g->llenx, g->lleny, g->llenz};
    for (int a = 0; a < 3; a++) G.w[a] = G.wl[a] = L[a] / G.n[a];
    return G;
}

static geo3 geo_coarse(const orc_grid* g, geo3 f)
{
    dims3 fd = {f.n[0], f.n[1], f.n[2]};
    dims3 cd = coarse_dims(g, fd);
    geo3 c;
    c.n[0] = cd.lx; c.n[1] = cd.ly; c.n[2] = cd.lz;
    const double L[3] = {g->llenx, g->lleny, g->llenz};
    for (int a = 0; a < 3; a++) {
        if (g->hier == ORC_HIER_CELL) {
            c.w[a] = c.wl[a] = L[a] / c.n[a];
        } else if (f.n[a] == 1) {
            c.w[a] = c.wl[a] = f.wl[a];
        } else {
            c.w[a] = 2.0 * f.w[a];
            c.wl[a] = (f.n[a] & 1) ? 2.0 * f.w[a] + f.wl[a] : f.w[a] + f.wl[a];
            if (c.n[a] == 1) c.w[a] = c.wl[a];
        }
    }
    return c;
}

static inline double cwidth(const geo3* G, int ax, int i0) /* 0-based index */
{
    return i0 == G->n[ax] - 1 ? G->wl[ax] : G->w[ax];
}

/* children of coarse cell I (1-based) along one direction: 2I-1 and 2I, plus
 * 2I+1 for the last coarse cell of an odd size */
static inline int child_lo(int I) { return 2 * I - 1; }
static inline int child_n(int I, int nf, int nc) { return nf == 1 ? 1 : (I == nc ? nf - 2 * (nc - 1) : 2); }

/* restriction, mgridsteps.f90:11-53 (8-cell average).  UNIFORM: the
 * volume-weighted average of the children that exist (equal to the 8-cell
 * average when all children are regular cells). */
static void restrict_fieldg(const orc_grid* g, const geo3* fg, const geo3* cg, const double* fine,
                            int fine_ghosted, double* coarse, int coarse_ghosted)
{
    const int cell = g->hier == ORC_HIER_CELL;
    dims3 f = {fg->n[0], fg->n[1], fg->n[2]}, c = {cg->n[0], cg->n[1], cg->n[2]};
#pragma omp parallel for schedule(static)
    for (int K = 1; K <= c.lz; K++)
        for (int J = 1; J <= c.ly; J++)
            for (int I = 1; I <= c.lx; I++) {
                double s = 0.0, vol = 0.0;
                int nx = cell ? 2 : child_n(I, f.lx, c.lx), ny = cell ? 2 : child_n(J, f.ly, c.ly),
                    nz = cell ? 2 : child_n(K, f.lz, c.lz);
                /* reference summation order: x, then y, then z */
                for (int dk = 0; dk < nz; dk++)
                    for (int dj = 0; dj < ny; dj++)
                        for (int di = 0; di < nx; di++) {
                            int i = child_lo(I) + di, j = child_lo(J) + dj, k = child_lo(K) + dk;
                            long src;
                            int lx = f.lx, ly = f.ly;
                            src = fine_ghosted ? GX(i, j, k) : IX(i, j, k);
                            if (cell) {
                                s += fine[src];
                            } else {
                                double v = cwidth(fg, 0, i - 1) * cwidth(fg, 1, j - 1) * cwidth(fg, 2, k - 1);
                                s += v * fine[src];
                                vol += v;
                            }
                        }
                double val = cell ? s * (1.0 / 8.0) : s / vol;
                int lx = c.lx, ly = c.ly;
                long dst = coarse_ghosted ? GX(I, J, K) : IX(I, J, K);
                coarse[dst] = val;
            }
}

static void restrict_field(const orc_grid* g, dims3 f, dims3 c, const double* fine, int fine_ghosted,
                           double* coarse, int coarse_ghosted)
{
    /* CELL only (uniform widths) */
    geo3 fg, cg;
    fg.n[0] = f.lx; fg.n[1] = f.ly; fg.n[2] = f.lz;
    cg.n[0] = c.lx; cg.n[1] = c.ly; cg.n[2] = c.lz;
    for (int a = 0; a < 3; a++) { fg.w[a] = fg.wl[a] = 1.0; cg.w[a] = cg.wl[a] = 1.0; }
    restrict_fieldg(g, &fg, &cg, fine, fine_ghosted, coarse, coarse_ghosted);
}

/* restrict_boundary, mgridsteps.f90:55-128 (average of 4 children; UNIFORM:
 * of the children that exist) */
static void restrict_bcvals(dims3 f, dims3 c, int cell, const double* const* bf, double** bcoarse)
{
    int fa[3][2] = {{f.ly, f.lz}, {f.lx, f.lz}, {f.lx, f.ly}};
    int ca[3][2] = {{c.ly, c.lz}, {c.lx, c.lz}, {c.lx, c.ly}};
    for (int face = 0; face < 6; face++) {
        int ax = face / 2;
        int n1 = fa[ax][0], c1 = ca[ax][0], c2 = ca[ax][1];
        for (int b = 1; b <= c2; b++)
            for (int a = 1; a <= c1; a++) {
                int na = cell ? 2 : child_n(a, fa[ax][0], c1), nb = cell ? 2 : child_n(b, fa[ax][1], c2);
                double s = 0.0;
                for (int db = 0; db < nb; db++)
                    for (int da = 0; da < na; da++)
                        s += bf[face][(child_lo(a) + da - 1) + (long)n1 * (child_lo(b) + db - 1)];
                bcoarse[face][(a - 1) + (long)c1 * (b - 1)] = s * (1.0 / (double)(na * nb));
            }
    }
}

/* update_boundary_ghostvalues, discretepde.f90:1121-1267 (+ periodic wrap) */
static void ghost_update(dims3 d, double* u, const int* bc, const double* const* bcv)
{
    const int lx = d.lx, ly = d.ly, lz = d.lz;
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++) {
            long jk = (j - 1) + (long)ly * (k - 1);
            if (bc[ORC_LEFT] == ORC_PERI) {
                u[GX(0, j, k)] = u[GX(lx, j, k)];
                u[GX(lx + 1, j, k)] = u[GX(1, j, k)];
            } else {
                u[GX(0, j, k)] = bc[ORC_LEFT] == ORC_DIRC ? 2.0 * bcv[0][jk] - u[GX(1, j, k)] : u[GX(1, j, k)];
                u[GX(lx + 1, j, k)] = bc[ORC_RIGHT] == ORC_DIRC ? 2.0 * bcv[1][jk] - u[GX(lx, j, k)] : u[GX(lx, j, k)];
            }
        }
    for (int k = 1; k <= lz; k++)
        for (int i = 1; i <= lx; i++) {
            long ik = (i - 1) + (long)lx * (k - 1);
            if (bc[ORC_BOTTOM] == ORC_PERI) {
                u[GX(i, 0, k)] = u[GX(i, ly, k)];
                u[GX(i, ly + 1, k)] = u[GX(i, 1, k)];
            } else {
                u[GX(i, 0, k)] = bc[ORC_BOTTOM] == ORC_DIRC ? 2.0 * bcv[2][ik] - u[GX(i, 1, k)] : u[GX(i, 1, k)];
                u[GX(i, ly + 1, k)] = bc[ORC_TOP] == ORC_DIRC ? 2.0 * bcv[3][ik] - u[GX(i, ly, k)] : u[GX(i, ly, k)];
            }
        }
    for (int j = 1; j <= ly; j++)
        for (int i = 1; i <= lx; i++) {
            long ij = (i - 1) + (long)lx * (j - 1);
            if (bc[ORC_BACK] == ORC_PERI) {
                u[GX(i, j, 0)] = u[GX(i, j, lz)];
                u[GX(i, j, lz + 1)] = u[GX(i, j, 1)];
            } else {
                u[GX(i, j, 0)] = bc[ORC_BACK] == ORC_DIRC ? 2.0 * bcv[4][ij] - u[GX(i, j, 1)] : u[GX(i, j, 1)];
                u[GX(i, j, lz + 1)] = bc[ORC_FRONT] == ORC_DIRC ? 2.0 * bcv[5][ij] - u[GX(i, j, lz)] : u[GX(i, j, lz)];
            }
        }
}

void orc_fill_ghosts(const orc_grid* g, double* soln, const int* bc, const double* const* bcvals)
{
    dims3 d = {g->lx, g->ly, g->lz};
    ghost_update(d, soln, bc, bcvals);
}

/* prolongation1, mgridsteps.f90:170-216 (CELL): e_f = e_c + sum_ax alpha_ax *
 * (e_c[I+1] - e_c[I-1]) with alpha = -1/8 / +1/8 (0.25*0.5*..., :197-209);
 * the odd last fine cell has no parent and is not corrected.
 * GEOM: tensor-product linear interpolation between the coarse centres that
 * bracket the fine centre, positions measured in units of the fine regular
 * width; ghost centres mirror across the wall with the value -e (Dirichlet)
 * or +e (other faces), or wrap for periodic faces.  (The additive central-
 * slope form loses its two-grid rate next to an odd last cell in 3D; the
 * tensor-product form keeps the even-size rate.) */
/* value of the coarse correction at ghosted index (qx,qy,qz), where any of
 * the indices may be a ghost (0 or n+1): each ghost axis maps back to the
 * adjacent interior cell with the sign of its face rule (Dirichlet -1,
 * other +1) or wraps for a periodic face.  Equals the face ghosts that
 * update_boundary_ghostvalues sets, extended to edges and corners. */
static double ghost_val(dims3 c, const double* ec, const int* bc, int qx, int qy, int qz)
{
    int q[3] = {qx, qy, qz}, n[3] = {c.lx, c.ly, c.lz};
    double sgn = 1.0;
    for (int a = 0; a < 3; a++) {
        if (q[a] >= 1 && q[a] <= n[a]) continue;
        int side = q[a] < 1 ? 0 : 1;
        if (bc[2 * a] == ORC_PERI) q[a] = q[a] < 1 ? n[a] : 1;
        else {
            if (bc[2 * a + side] == ORC_DIRC) sgn = -sgn;
            q[a] = q[a] < 1 ? 1 : n[a];
        }
    }
    int lx = c.lx, ly = c.ly;
    return sgn * ec[GX(q[0], q[1], q[2])];
}

typedef struct { int j0, j1; double t; } lin1; /* e = (1-t) e[j0] + t e[j1]; j = -1 / nc: ghost */

static lin1 geom_lin(const geo3* fg, const geo3* cg, int ax, int i0, int per)
{
    lin1 r;
    const int nf = fg->n[ax], nc = cg->n[ax];
    if (nf == nc) { r.j0 = r.j1 = i0; r.t = 0.0; return r; }
    const double rf = fg->wl[ax] / fg->w[ax], Rc = cg->wl[ax] / fg->w[ax];
    const double xf = (i0 == nf - 1) ? (nf - 1) + 0.5 * rf : i0 + 0.5;
    const double Ltot = 2.0 * (nc - 1) + Rc;
    const double X0 = (nc == 1) ? 0.5 * Rc : 1.0;
    const double Xl = 2.0 * (nc - 1) + 0.5 * Rc;
    int I = (i0 >> 1) < nc - 1 ? (i0 >> 1) : nc - 1;
    double XI = (I == nc - 1) ? Xl : 2.0 * I + 1.0;
    int J = xf >= XI ? I : I - 1;
    double XJ, XJ1;
    if (J < 0) XJ = per ? Xl - Ltot : -X0;
    else XJ = (J == nc - 1) ? Xl : 2.0 * J + 1.0;
    if (J + 1 > nc - 1) XJ1 = per ? X0 + Ltot : 2.0 * Ltot - Xl;
    else XJ1 = (J + 1 == nc - 1) ? Xl : 2.0 * (J + 1) + 1.0;
    r.j0 = J;
    r.j1 = J + 1;
    r.t = (xf - XJ) / (XJ1 - XJ);
    return r;
}

/* coarse value with ghost rule (1-based index into a ghosted coarse array
 * whose face ghosts are already set by ghost_update); jz is 0-based along ax */
static void prolongg(const orc_grid* g, const geo3* fg, const geo3* cg, const int* bc, const double* ec,
                     double* ef)
{
    const int cell = g->hier == ORC_HIER_CELL;
    dims3 f = {fg->n[0], fg->n[1], fg->n[2]}, c = {cg->n[0], cg->n[1], cg->n[2]};
    const int per[3] = {bc[0] == ORC_PERI, bc[2] == ORC_PERI, bc[4] == ORC_PERI};
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= f.lz; k++)
        for (int j = 1; j <= f.ly; j++)
            for (int i = 1; i <= f.lx; i++) {
                if (cell) {
                    int I = (i + 1) / 2, J = (j + 1) / 2, K = (k + 1) / 2;
                    if (I > c.lx || J > c.ly || K > c.lz) continue; /* odd last cell dropped */
                    int lx = c.lx, ly = c.ly;
                    double e0 = ec[GX(I, J, K)];
                    double ax = (i & 1) ? -0.125 : 0.125;
                    double ay = (j & 1) ? -0.125 : 0.125;
                    double az = (k & 1) ? -0.125 : 0.125;
                    double dxv = ec[GX(I + 1, J, K)] - ec[GX(I - 1, J, K)];
                    double dyv = ec[GX(I, J + 1, K)] - ec[GX(I, J - 1, K)];
                    double dzv = ec[GX(I, J, K + 1)] - ec[GX(I, J, K - 1)];
                    double v = e0 + ((ax * dxv + ay * dyv) + az * dzv);
                    lx = f.lx; ly = f.ly;
                    ef[GX(i, j, k)] = v;
                    continue;
                }
                lin1 L3[3] = {geom_lin(fg, cg, 0, i - 1, per[0]), geom_lin(fg, cg, 1, j - 1, per[1]),
                              geom_lin(fg, cg, 2, k - 1, per[2])};
                /* ghosted coarse array: 0-based index q maps to q+1; ghosts at 0 and n+1
                 * hold the face rule, which for a 1-D bracket is the value we need */
                double v = 0.0;
                for (int cz = 0; cz < 2; cz++) {
                    double wz = cz ? L3[2].t : 1.0 - L3[2].t;
                    if (wz == 0.0) continue;
                    int qz = (cz ? L3[2].j1 : L3[2].j0) + 1;
                    for (int cy = 0; cy < 2; cy++) {
                        double wy = cy ? L3[1].t : 1.0 - L3[1].t;
                        if (wy == 0.0) continue;
                        int qy = (cy ? L3[1].j1 : L3[1].j0) + 1;
                        for (int cx = 0; cx < 2; cx++) {
                            double wx = cx ? L3[0].t : 1.0 - L3[0].t;
                            if (wx == 0.0) continue;
                            int qx = (cx ? L3[0].j1 : L3[0].j0) + 1;
                            int lx = c.lx, ly = c.ly;
                            v += wz * wy * wx * ghost_val(c, ec, bc, qx, qy, qz);
                        }
                    }
                }
                int lx = f.lx, ly = f.ly;
                ef[GX(i, j, k)] = v;
            }
}

static void prolong(int cell, dims3 f, dims3 c, const double* ec, double* ef)
{
    /* CELL only */
    orc_grid g;
    memset(&g, 0, sizeof(g));
    g.hier = ORC_HIER_CELL;
    geo3 fg, cg;
    fg.n[0] = f.lx; fg.n[1] = f.ly; fg.n[2] = f.lz;
    cg.n[0] = c.lx; cg.n[1] = c.ly; cg.n[2] = c.lz;
    for (int a = 0; a < 3; a++) { fg.w[a] = fg.wl[a] = cg.w[a] = cg.wl[a] = 1.0; }
    int bc[6] = {0, 0, 0, 0, 0, 0};
    (void)cell;
    prolongg(&g, &fg, &cg, bc, ec, ef);
}

/* ---- GMRES bottom solve: gmres.f90:9-434 with gseidel_precond
 *      (discretepde.f90:238-337) ---- */
typedef struct {
    const orc_grid* g;
    int timederiv; double dt;
    const double *vel, *dcoeff, *reac;
    const int* bc;
    double *AX, *diag, *off;
} opctx;

static void op_AX(opctx* o, const double* x, double* Ax_interior)
{
    orc_find_AX(o->g, x, o->timederiv, o->dt, o->vel, o->dcoeff, o->reac, o->bc, Ax_interior, o->diag, o->off);
}

/* gseidel_precond: MinvX ghosted out, X ghosted in (interior used) */
static void gs_precond(opctx* o, double* MinvX, const double* X, int niter)
{
    const int lx = o->g->lx, ly = o->g->ly, lz = o->g->lz;
    const long ng = ngh(lx, ly, lz);
    memset(MinvX, 0, sizeof(double) * ng);
    if ((long)lx * ly * lz == 1) {
        op_AX(o, MinvX, o->AX);
        MinvX[GX(1, 1, 1)] = X[GX(1, 1, 1)] / o->diag[0];
        return;
    }
    for (int it = 0; it < niter; it++) {
        op_AX(o, MinvX, o->AX);
        for (int k = 1; k <= lz; k++)
            for (int j = 1; j <= ly; j++)
                for (int i = 1; i <= lx; i++)
                    if (((i + j + k) & 1) == 1) {
                        long c = IX(i, j, k);
                        MinvX[GX(i, j, k)] = (X[GX(i, j, k)] - o->off[c]) / o->diag[c];
                    }
        op_AX(o, MinvX, o->AX);
        for (int k = 1; k <= lz; k++)
            for (int j = 1; j <= ly; j++)
                for (int i = 1; i <= lx; i++)
                    if (((i + j + k) & 1) == 0) {
                        long c = IX(i, j, k);
                        MinvX[GX(i, j, k)] = (X[GX(i, j, k)] - o->off[c]) / o->diag[c];
                    }
    }
}

static double findnorm(const double* v, long n)
{
    double s = 0.0;
    for (long i = 0; i < n; i++) s += v[i] * v[i];
    return sqrt(s);
}

static int isit_nan(double x) /* gmres.f90:436-450 */
{
    int r = 0;
    if (x != x) r = 1;
    if ((x / x != 1.0) && (x != 0.0)) r = 1;
    return r;
}

/* performgmres, gmres.f90:197-434 (left preconditioned, classical GS).
 * Returns 0 on success, 2 when a NaN/Inf was detected (the reference aborts). */
static int performgmres(opctx* o, const double* b, double* x, int maxkspdim, int nrestarts, double tol)
{
    const int lx = o->g->lx, ly = o->g->ly, lz = o->g->lz;
    const long ng = ngh(lx, ly, lz), n = nin(lx, ly, lz);
    const int m = maxkspdim;
    double* bg = zalloc(ng);
    double* Minvb = zalloc(ng);
    double* Ax0 = zalloc(n);
    double* r0 = zalloc(ng);
    double* r = zalloc(ng);
    double* x0 = zalloc(ng);
    double* V = zalloc(ng * (m + 1));
    double* H = zalloc((long)(m + 1) * m);
    double* y = zalloc(m);
    double* cs = zalloc(m);
    double* sn = zalloc(m);
    double* be = zalloc(m + 1);
    double* Avj = zalloc(ng);
    double* MinvAvj = zalloc(ng);
    double* w = zalloc(ng);
    int status = 0;
#define HM(i, j) H[(long)((i)-1) + (long)(m + 1) * ((j)-1)]
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) bg[GX(i, j, k)] = b[IX(i, j, k)];
    for (int rs = 0; rs < nrestarts; rs++) {
        memset(H, 0, sizeof(double) * (m + 1) * m);
        memset(V, 0, sizeof(double) * ng * (m + 1));
        memset(be, 0, sizeof(double) * (m + 1));
        memset(cs, 0, sizeof(double) * m);
        memset(sn, 0, sizeof(double) * m);
        memset(y, 0, sizeof(double) * m);
        memset(r0, 0, sizeof(double) * ng);
        gs_precond(o, Minvb, bg, 1);
        double b_norm = findnorm(Minvb, ng);
        if (b_norm == 0.0) { memset(x, 0, sizeof(double) * ng); break; }
        memcpy(x0, x, sizeof(double) * ng);
        op_AX(o, x0, Ax0);
        for (int k = 1; k <= lz; k++)
            for (int j = 1; j <= ly; j++)
                for (int i = 1; i <= lx; i++) r0[GX(i, j, k)] = b[IX(i, j, k)] - Ax0[IX(i, j, k)];
        gs_precond(o, r, r0, 1);
        double beta = findnorm(r, ng);
        for (long q = 0; q < ng; q++) V[q] = r[q] / beta;
        be[0] = beta;
        beta = findnorm(r, ng);
        if (fabs(beta) < tol) break;
        memcpy(x0, x, sizeof(double) * ng);
        for (long q = 0; q < ng; q++) V[q] = r[q] / beta;
        int optk = m, lucky = 0;
        double residnorm = 0.0;
        for (int kd = 1; kd <= m; kd++) {
            memcpy(x, x0, sizeof(double) * ng);
            /* arnoldialgorithm, gmres.f90:9-122 */
            double* vj = V + ng * (kd - 1);
            memset(Avj, 0, sizeof(double) * ng);
            double* Avi = zalloc(n);
            op_AX(o, vj, Avi);
            for (int k = 1; k <= lz; k++)
                for (int j = 1; j <= ly; j++)
                    for (int i = 1; i <= lx; i++) Avj[GX(i, j, k)] = Avi[IX(i, j, k)];
            free(Avi);
            gs_precond(o, MinvAvj, Avj, 1);
            memcpy(w, MinvAvj, sizeof(double) * ng);
            for (int ii = 1; ii <= kd; ii++) {
                const double* vi = V + ng * (ii - 1);
                double h = 0.0;
                for (int k = 1; k <= lz; k++)
                    for (int j = 1; j <= ly; j++)
                        for (int i = 1; i <= lx; i++) h += MinvAvj[GX(i, j, k)] * vi[GX(i, j, k)];
                HM(ii, kd) = h;
                for (long q = 0; q < ng; q++) w[q] = w[q] - h * vi[q];
            }
            HM(kd + 1, kd) = findnorm(w, ng);
            int nanflag = 0;
            if (HM(kd + 1, kd) > NEARZERO) {
                for (long q = 0; q < ng; q++) V[ng * kd + q] = w[q] / HM(kd + 1, kd);
            } else if (!isit_nan(HM(kd + 1, kd))) {
                lucky = 1;
            } else {
                nanflag = 1;
            }
            if (nanflag) { status = 2; goto done; }
            /* triangularize, gmres.f90:159-195 */
            for (int i = 1; i <= kd - 1; i++) {
                double t = cs[i - 1] * HM(i, kd) + sn[i - 1] * HM(i + 1, kd);
                HM(i + 1, kd) = -sn[i - 1] * HM(i, kd) + cs[i - 1] * HM(i + 1, kd);
                HM(i, kd) = t;
            }
            double rr = HM(kd, kd), ss = HM(kd + 1, kd), c, s;
            if (rr == 0.0) { c = 0.0; s = 1.0; } /* givens_rotate :144-157 */
            else { c = rr / sqrt(rr * rr + ss * ss); s = ss / sqrt(rr * rr + ss * ss); }
            HM(kd, kd) = c * HM(kd, kd) + s * HM(kd + 1, kd);
            HM(kd + 1, kd) = 0.0;
            cs[kd - 1] = c; sn[kd - 1] = s;
            be[kd] = -s * be[kd - 1];
            be[kd - 1] = c * be[kd - 1];
            residnorm = fabs(be[kd]);
            if (lucky) { optk = kd; break; }
        }
        /* uppertrisolve, gmres.f90:124-142 */
        for (int i = optk; i >= 1; i--) {
            y[i - 1] = be[i - 1];
            for (int j = i + 1; j <= optk; j++) y[i - 1] -= HM(i, j) * y[j - 1];
            y[i - 1] /= HM(i, i);
        }
        for (int j = 1; j <= optk; j++)
            for (long q = 0; q < ng; q++) x[q] = x[q] + y[j - 1] * V[ng * (j - 1) + q];
        if (residnorm / b_norm <= tol || lucky) break;
    }
done:
#undef HM
    free(bg); free(Minvb); free(Ax0); free(r0); free(r); free(x0); free(V); free(H);
    free(y); free(cs); free(sn); free(be); free(Avj); free(MinvAvj); free(w);
    return status;
}

/* bottomsolve, mgridsteps.f90:218-382 (single global domain: the gather is
 * the identity).  serial_bcvals are zero in the reference (:222-223, :514). */
static int bottomsolve(const orc_grid* g, double* soln, int timederiv, double dt,
                       const double* vel, const double* dcoeff, const double* reac,
                       const double* source, const int* bc, int applybc,
                       const double* mgridsterm)
{
    const int lx = g->lx, ly = g->ly, lz = g->lz;
    const long n = nin(lx, ly, lz), ng = ngh(lx, ly, lz);
    double* zeros[6];
    double* b = zalloc(n);
    double* x = zalloc(ng);
    for (int f = 0; f < 6; f++) zeros[f] = zalloc((long)(lx + ly + lz) * (lx + ly + lz));
    /* the gather copies interior values only (:314-326) */
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) x[GX(i, j, k)] = soln[GX(i, j, k)];
    double* vel_s = zalloc(3 * ng);
    double* dc_s = zalloc(ng);
    double* re_s = zalloc(ng);
    double* so_s = zalloc(ng);
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) {
                long q = GX(i, j, k);
                for (int d = 0; d < 3; d++) vel_s[d * ng + q] = vel[d * ng + q];
                dc_s[q] = dcoeff[q]; re_s[q] = reac[q]; so_s[q] = source[q];
            }
    orc_find_bvec(g, vel_s, dc_s, so_s, bc, (const double* const*)zeros, mgridsterm, applybc, b);
    opctx o = {g, timederiv, dt, vel_s, dc_s, re_s, bc, zalloc(n), zalloc(n), zalloc(n)};
    int st = performgmres(&o, b, x, (int)n, 1, ERRTOLR * 0.0001);
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) soln[GX(i, j, k)] = x[GX(i, j, k)];
    free(o.AX); free(o.diag); free(o.off);
    free(vel_s); free(dc_s); free(re_s); free(so_s);
    for (int f = 0; f < 6; f++) free(zeros[f]);
    free(b); free(x);
    return st;
}

static double compute_norm(const double* var, long n) /* globalvars.f90:136-159 */
{
    double s = 0.0;
    for (long c = 0; c < n; c++) s += var[c] * var[c];
    return sqrt(s / (double)n);
}

static int vcycle_rec(const orc_grid* g, int is_fine, double* soln, int timederiv, double dt,
                      const double* vel, const double* dcoeff, const double* reac,
                      const double* source, const int* bc, const double* const* bcvals,
                      const double* mgridsterm, double* resnorm)
{
    const int lx = g->lx, ly = g->ly, lz = g->lz;
    dims3 f = {lx, ly, lz};
    int applybc = is_fine; /* :506-510 */
    if (is_coarsest(g, f)) {
        *resnorm = 0.0;
        return bottomsolve(g, soln, timederiv, dt, vel, dcoeff, reac, source, bc, applybc, mgridsterm);
    }
    dims3 c = coarse_dims(g, f);
    orc_grid gc = *g;
    gc.lx = c.lx; gc.ly = c.ly; gc.lz = c.lz;
    const long n = nin(lx, ly, lz), ng = ngh(lx, ly, lz);
    const long nc = nin(c.lx, c.ly, c.lz), ngc = ngh(c.lx, c.ly, c.lz);
    const int cell = g->hier == ORC_HIER_CELL;
    double* res = zalloc(n);
    double* rres = zalloc(nc);
    double* rsold = zalloc(ngc);
    double* rsnew = zalloc(ngc);
    double* e2h = zalloc(ngc);
    double* eh = zalloc(ng);
    double* rsterm = zalloc(nc);
    double* vel_c = zalloc(3 * ngc);
    double* dc_c = zalloc(ngc);
    double* re_c = zalloc(ngc);
    double* so_c = zalloc(ngc);
    double* AXc = zalloc(nc);
    double* d1 = zalloc(nc);
    double* d2 = zalloc(nc);
    double* bcc[6];
    int fa[3] = {c.ly * c.lz, c.lx * c.lz, c.lx * c.ly};
    for (int q = 0; q < 6; q++) bcc[q] = zalloc(fa[q / 2]);
    int st;

    orc_gs_smooth(g, soln, timederiv, dt, applybc, mgridsterm, res, vel, dcoeff, reac, source, bc,
                  bcvals, g->nu1); /* :523-527 */
    restrict_field(g, f, c, soln, 1, rsold, 1);               /* :529 */
    restrict_field(g, f, c, res, 0, rres, 0);                 /* :531 */
    for (int d = 0; d < 3; d++)                                /* :533-535 */
        restrict_field(g, f, c, vel + d * ng, 1, vel_c + d * ngc, 1);
    restrict_field(g, f, c, dcoeff, 1, dc_c, 1);              /* :537 */
    restrict_field(g, f, c, reac, 1, re_c, 1);                /* :538 */
    restrict_field(g, f, c, source, 1, so_c, 1);              /* :539 */
    restrict_bcvals(f, c, cell, bcvals, bcc);                 /* :542 */
    orc_find_AX(&gc, rsold, timederiv, dt, vel_c, dc_c, re_c, bc, AXc, d1, d2); /* :544-548 */
    for (long q = 0; q < nc; q++) rsterm[q] = AXc[q] + rres[q]; /* :550 */
    ghost_update(c, rsold, bc, (const double* const*)bcc);    /* :552 */
    memcpy(rsnew, rsold, sizeof(double) * ngc);               /* :554 */
    double rn2h;
    st = vcycle_rec(&gc, 0, rsnew, timederiv, dt, vel_c, dc_c, re_c, so_c, bc,
                    (const double* const*)bcc, rsterm, &rn2h); /* :555-558 */
    ghost_update(c, rsnew, bc, (const double* const*)bcc);    /* :560 */
    for (long q = 0; q < ngc; q++) e2h[q] = rsnew[q] - rsold[q]; /* :562 */
    prolong(cell, f, c, e2h, eh);                             /* :565 */
    for (long q = 0; q < ng; q++) soln[q] = soln[q] + eh[q];  /* :567 */
    orc_gs_smooth(g, soln, timederiv, dt, applybc, mgridsterm, res, vel, dcoeff, reac, source, bc,
                  bcvals, g->nu2); /* :569-573 */
    *resnorm = compute_norm(res, n);                          /* :575 */
    free(res); free(rres); free(rsold); free(rsnew); free(e2h); free(eh); free(rsterm);
    free(vel_c); free(dc_c); free(re_c); free(so_c); free(AXc); free(d1); free(d2);
    for (int q = 0; q < 6; q++) free(bcc[q]);
    return st;
}

/* perform_vcycle, mgridsteps.f90:384-579 */
int orc_vcycle(const orc_grid* g, double* soln, int timederiv, double dt,
               const double* vel, const double* dcoeff, const double* reac,
               const double* source, const int* bc, const double* const* bcvals,
               const double* mgridsterm, double* resnorm)
{
    const long n = nin(g->lx, g->ly, g->lz);
    double* zero = NULL;
    if (g->hier != ORC_HIER_CELL) return 4; /* the restatement is the reference hierarchy */
    if (!mgridsterm) { zero = zalloc(n); mgridsterm = zero; }
    int st = vcycle_rec(g, 1, soln, timederiv, dt, vel, dcoeff, reac, source, bc, bcvals,
                        mgridsterm, resnorm);
    free(zero);
    return st;
}

double orc_rel_residual(const orc_grid* g, const double* soln, int timederiv, double dt,
                        const double* vel, const double* dcoeff, const double* reac,
                        const double* source, const int* bc, const double* const* bcvals,
                        double* rms_out)
{
    const long n = nin(g->lx, g->ly, g->lz);
    double* b = zalloc(n);
    double* AX = zalloc(n);
    double* d = zalloc(n);
    double* o = zalloc(n);
    orc_find_bvec(g, vel, dcoeff, source, bc, bcvals, NULL, 1, b);
    orc_find_AX(g, soln, timederiv, dt, vel, dcoeff, reac, bc, AX, d, o);
    double rr = 0.0, bb = 0.0;
    for (long c = 0; c < n; c++) {
        double r = b[c] - AX[c];
        rr += r * r;
        bb += b[c] * b[c];
    }
    if (rms_out) *rms_out = sqrt(rr / (double)n);
    free(b); free(AX); free(d); free(o);
    return bb > 0.0 ? sqrt(rr) / sqrt(bb) : sqrt(rr);
}

/* caller loop: poissoneq.f90:427-450, pdedefs.f90:304-328 (tol_kind 0 = the
 * reference's RMS of the post-smoothing residual, 1 = ||b-Ax||/||b||) */
int orc_solve(const orc_grid* g, double* soln, int timederiv, double dt,
              const double* vel, const double* dcoeff, const double* reac,
              const double* source, const int* bc, const double* const* bcvals,
              int maxit, double tol, int tol_kind, double* rel_hist, double* rms_hist)
{
    const long n = nin(g->lx, g->ly, g->lz);
    double* sterm = zalloc(n);
    int it;
    for (it = 0; it < maxit; it++) {
        double resnorm = 0.0, rms = 0.0;
        memset(sterm, 0, sizeof(double) * n);
        int st = orc_vcycle(g, soln, timederiv, dt, vel, dcoeff, reac, source, bc, bcvals, sterm, &resnorm);
        if (st) { free(sterm); return -st; }
        double rel = orc_rel_residual(g, soln, timederiv, dt, vel, dcoeff, reac, source, bc, bcvals, &rms);
        if (rel_hist) rel_hist[it] = rel;
        if (rms_hist) rms_hist[it] = resnorm;
        if ((tol_kind == 0 && resnorm <= tol) || (tol_kind == 1 && rel <= tol)) { it++; break; }
    }
    free(sterm);
    return it;
}

/* ======================================================================
 * layer (B): 7-point rows
 * ==================================================================== */

/* find_sg_exponential_flux, mps1d/source/convdiff.f90:10-64 */
void orc_sg_face(double cL, double cR, double DL, double DR, double dx, double* wL, double* wR)
{
    const double eps = 1.0e-10;
    double c_half = 0.5 * (cL + cR);
    double D_half = 2.0 * DL * DR / (DL + DR + eps);
    double sign_c = c_half <= 0.0 ? -1.0 : 1.0;
    *wL = 0.0; *wR = 0.0;
    if (fabs(D_half) < eps) {
        *wL = cL * 0.5 * (1.0 + sign_c);
        *wR = cR * 0.5 * (1.0 - sign_c);
    } else {
        double Pe = c_half * dx / D_half;
        if (fabs(Pe) < eps) {
            *wL = D_half / dx;
            *wR = -D_half / dx;
        } else if (Pe > 0.0) {
            *wL = c_half / (1.0 - exp(-Pe));
            *wR = -c_half * exp(-Pe) / (1.0 - exp(-Pe));
        } else {
            *wL = c_half * exp(Pe) / (exp(Pe) - 1.0);
            *wR = -c_half / (exp(Pe) - 1.0);
        }
    }
}

/* derivatives of orc_sg_face with respect to (cL, cR, DL, DR), differentiated
 * branch by branch from the closed forms above (extension: the reference has
 * no adjoint).  dwL[q], dwR[q] for q = cL, cR, DL, DR. */
void orc_sg_face_d(double cL, double cR, double DL, double DR, double dx, double* dwL, double* dwR)
{
    const double eps = 1.0e-10;
    const double c = 0.5 * (cL + cR);
    const double S = DL + DR + eps;
    const double D = 2.0 * DL * DR / S;
    const double dD_dL = 2.0 * DR * (DR + eps) / (S * S), dD_dR = 2.0 * DL * (DL + eps) / (S * S);
    double wLc = 0.0, wLD = 0.0, wRc = 0.0, wRD = 0.0;
    for (int q = 0; q < 4; q++) dwL[q] = dwR[q] = 0.0;
    if (fabs(D) < eps) {
        const double sgn = c <= 0.0 ? -1.0 : 1.0;
        dwL[0] = 0.5 * (1.0 + sgn);
        dwR[1] = 0.5 * (1.0 - sgn);
        return;
    }
    const double Pe = c * dx / D;
    if (fabs(Pe) < eps) {
        wLD = 1.0 / dx;
        wRD = -1.0 / dx;
    } else if (fabs(Pe) < 1.0e-2) {
        /* the closed forms below cancel as Pe -> 0: Taylor series of the same
         * weights, wL = c/(1 - e^-Pe) = (D/dx)(1 + Pe/2 + Pe^2/12 - Pe^4/720 + ...),
         * wR = c - wL, truncated after the Pe^6 terms */
        const double P2 = Pe * Pe;
        wLc = 0.5 + Pe / 6.0 - P2 * Pe / 180.0 + P2 * P2 * Pe / 5040.0;
        wRc = 1.0 - wLc;
        wLD = (1.0 - P2 / 12.0 + P2 * P2 / 240.0 - P2 * P2 * P2 / 6048.0) / dx;
        wRD = -wLD;
    } else if (Pe > 0.0) {
        const double E = exp(-Pe), q1 = 1.0 - E;
        wLc = 1.0 / q1 - Pe * E / (q1 * q1);
        wLD = c * E * Pe / (D * q1 * q1);
        wRc = -E / q1 + Pe * E / (q1 * q1);
        wRD = -c * E * Pe / (D * q1 * q1);
    } else {
        const double P = exp(Pe), q1 = P - 1.0;
        wLc = P / q1 - Pe * P / (q1 * q1);
        wLD = c * P * Pe / (D * q1 * q1);
        wRc = -1.0 / q1 + Pe * P / (q1 * q1);
        wRD = -c * P * Pe / (D * q1 * q1);
    }
    dwL[0] = 0.5 * wLc; dwL[1] = 0.5 * wLc; dwL[2] = wLD * dD_dL; dwL[3] = wLD * dD_dR;
    dwR[0] = 0.5 * wRc; dwR[1] = 0.5 * wRc; dwR[2] = wRD * dD_dL; dwR[3] = wRD * dD_dR;
}

/* gradients of s = lam^T A(vel, dcoeff, reac) u with respect to the cell
 * fields (interior arrays lam, u; uniform grid), accumulated face by face:
 * a face (L, R) with flux F = wL u_L + wR u_R adds F (lam_L - lam_R) / h to s,
 * boundary and diagonal terms add lam_c u_c times their coefficient. */
void orc_operator_vjp(const orc_grid* g, int flux, const double* vel, const double* dcoeff, const int* bc,
                      const double* lam, const double* u, double* gvel, double* gd, double* greac)
{
    const int lx = g->lx, ly = g->ly, lz = g->lz;
    const long ng = ngh(lx, ly, lz), n = nin(lx, ly, lz);
    const int L[3] = {lx, ly, lz};
    const double h[3] = {g->llenx / lx, g->lleny / ly, g->llenz / lz};
    memset(gvel, 0, sizeof(double) * 3 * n);
    memset(gd, 0, sizeof(double) * n);
    for (long c = 0; c < n; c++) greac[c] = -lam[c] * u[c];
    for (int ax = 0; ax < 3; ax++) {
        const double* v = vel + ax * ng;
        double* gv = gvel + ax * n;
        const int per = bc[2 * ax] == ORC_PERI;
        const double hx = h[ax];
        for (int k = 1; k <= lz; k++)
            for (int j = 1; j <= ly; j++)
                for (int i = 1; i <= lx; i++) {
                    int idx[3] = {i, j, k};
                    const int pos = idx[ax];
                    const long c = IX(i, j, k);
                    const double vc = v[GX(i, j, k)], kc = dcoeff[GX(i, j, k)];
                    if (pos < L[ax] || per) {
                        int r3[3] = {i, j, k};
                        r3[ax] = pos < L[ax] ? pos + 1 : 1;
                        const long cr = IX(r3[0], r3[1], r3[2]);
                        const double vr = v[GX(r3[0], r3[1], r3[2])], kr = dcoeff[GX(r3[0], r3[1], r3[2])];
                        double dwL[4], dwR[4];
                        if (flux == ORC_FLUX_SG) {
                            orc_sg_face_d(vc, vr, kc, kr, hx, dwL, dwR);
                        } else {
                            const double vh = 0.5 * (vc + vr);
                            const double a = 0.5 / hx;
                            dwL[0] = dwL[1] = vh > 0.0 ? 0.5 : 0.0;
                            dwR[0] = dwR[1] = vh > 0.0 ? 0.0 : 0.5;
                            dwL[2] = dwL[3] = a;
                            dwR[2] = dwR[3] = -a;
                        }
                        const double m = (lam[c] - lam[cr]) / hx;
                        gv[c] += m * (dwL[0] * u[c] + dwR[0] * u[cr]);
                        gv[cr] += m * (dwL[1] * u[c] + dwR[1] * u[cr]);
                        gd[c] += m * (dwL[2] * u[c] + dwR[2] * u[cr]);
                        gd[cr] += m * (dwL[3] * u[c] + dwR[3] * u[cr]);
                    }
                    if (!per && (pos == 1 || pos == L[ax])) {
                        for (int side = 0; side < 2; side++) {
                            if ((side == 0 && pos != 1) || (side == 1 && pos != L[ax])) continue;
                            const int code = bc[2 * ax + side];
                            const double lu = lam[c] * u[c];
                            if (code == ORC_DIRC) {
                                if (flux == ORC_FLUX_SG) {
                                    double dwL[4], dwR[4];
                                    orc_sg_face_d(vc, vc, kc, kc, 0.5 * hx, dwL, dwR);
                                    if (side == 0) {
                                        gv[c] -= lu * (dwR[0] + dwR[1]) / hx;
                                        gd[c] -= lu * (dwR[2] + dwR[3]) / hx;
                                    } else {
                                        gv[c] += lu * (dwL[0] + dwL[1]) / hx;
                                        gd[c] += lu * (dwL[2] + dwL[3]) / hx;
                                    }
                                } else {
                                    gd[c] += lu * 2.0 / (hx * hx);
                                    if (side == 0 && vc < 0.0) gv[c] -= lu / hx;
                                    if (side == 1 && vc > 0.0) gv[c] += lu / hx;
                                }
                            } else if (code == ORC_ZGRD) {
                                gv[c] += side == 0 ? -lu / hx : lu / hx;
                            }
                        }
                    }
                }
    }
}

#define R7(q, c) rows[(long)(q) * n + (c)]

/* upwind rows from the find_AX formulas (discretepde.f90:620-1116); SG rows
 * from the 1D flux applied per face (convdiff.f90:280-288) with the same
 * boundary treatment as find_AX for ZGRD and a half-cell SG flux for DIRC.
 * A face between cells of widths wa, wb has centre distance d = (wa+wb)/2;
 * its flux per unit area is F = wL*u_L + wR*u_R and row L gains +F/w_L, row
 * R gains -F/w_R (on uniform cells: find_AX's (k_half/dx)*(1/dx) etc.). */
static void build_rows_geo(const geo3* G, int flux, int timederiv, double dt, const double* vel,
                           const double* dcoeff, const double* reac, const int* bc, double* rows)
{
    const int lx = G->n[0], ly = G->n[1], lz = G->n[2];
    const long ng = ngh(lx, ly, lz), n = nin(lx, ly, lz);
    const int L[3] = {lx, ly, lz};
    memset(rows, 0, sizeof(double) * 7 * n);
    for (int ax = 0; ax < 3; ax++) {
        const double* v = vel + ax * ng;
        const int per = bc[2 * ax] == ORC_PERI;
        for (int k = 1; k <= lz; k++)
            for (int j = 1; j <= ly; j++)
                for (int i = 1; i <= lx; i++) {
                    int idx[3] = {i, j, k};
                    int pos = idx[ax];
                    long c = IX(i, j, k);
                    const double wc = cwidth(G, ax, pos - 1);
                    /* face on the + side of this cell (between pos and pos+1) */
                    if (pos < L[ax] || per) {
                        int r3[3] = {i, j, k};
                        r3[ax] = pos < L[ax] ? pos + 1 : 1;
                        long cr = IX(r3[0], r3[1], r3[2]);
                        const double wn = cwidth(G, ax, r3[ax] - 1);
                        const double d = 0.5 * (wc + wn);
                        double kl = dcoeff[GX(i, j, k)], kr = dcoeff[GX(r3[0], r3[1], r3[2])];
                        double vl = v[GX(i, j, k)], vr = v[GX(r3[0], r3[1], r3[2])];
                        double wL, wR;
                        if (flux == ORC_FLUX_SG) {
                            orc_sg_face(vl, vr, kl, kr, d, &wL, &wR);
                        } else {
                            double kh = 0.5 * (kl + kr) / d;
                            double vh = 0.5 * (vl + vr);
                            wL = kh; wR = -kh;
                            if (vh > 0.0) wL += vh;
                            else wR += vh;
                        }
                        const double al = 1.0 / wc, ar = 1.0 / wn;
                        R7(0, c) += wL * al;
                        R7(2 + 2 * ax, c) += wR * al;
                        R7(0, cr) -= wR * ar;
                        R7(1 + 2 * ax, cr) -= wL * ar;
                    }
                    /* physical boundary faces */
                    if (!per && (pos == 1 || pos == L[ax])) {
                        for (int side = 0; side < 2; side++) {
                            if ((side == 0 && pos != 1) || (side == 1 && pos != L[ax])) continue;
                            int code = bc[2 * ax + side];
                            double vb = v[GX(i, j, k)], kb = dcoeff[GX(i, j, k)];
                            if (code == ORC_DIRC) {
                                if (flux == ORC_FLUX_SG) {
                                    double wL, wR;
                                    orc_sg_face(vb, vb, kb, kb, 0.5 * wc, &wL, &wR);
                                    if (side == 0) R7(0, c) -= wR / wc; /* F = wL g + wR u */
                                    else R7(0, c) += wL / wc;           /* F = wL u + wR g */
                                } else {
                                    R7(0, c) += 2.0 * kb / (wc * wc);
                                    if (side == 0 && vb < 0.0) R7(0, c) -= vb / wc;
                                    if (side == 1 && vb > 0.0) R7(0, c) += vb / wc;
                                }
                            } else if (code == ORC_ZGRD) {
                                if (side == 0) R7(0, c) -= vb / wc;
                                else R7(0, c) += vb / wc;
                            }
                        }
                    }
                }
    }
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) {
                long c = IX(i, j, k);
                R7(0, c) -= reac[GX(i, j, k)];
                if (timederiv) R7(0, c) += 1.0 / dt;
            }
}

void orc_build_rows(const orc_grid* g, int flux, int timederiv, double dt,
                    const double* vel, const double* dcoeff, const double* reac,
                    const int* bc, double* rows)
{
    geo3 G = geo_fine(g);
    build_rows_geo(&G, flux, timederiv, dt, vel, dcoeff, reac, bc, rows);
}

void orc_build_rhs(const orc_grid* g, int flux, const double* vel, const double* dcoeff,
                   const double* source, const int* bc, const double* const* bcvals, double* b)
{
    if (flux != ORC_FLUX_SG) {
        orc_find_bvec(g, vel, dcoeff, source, bc, bcvals, NULL, 1, b);
        return;
    }
    const int lx = g->lx, ly = g->ly, lz = g->lz;
    const long ng = ngh(lx, ly, lz), n = nin(lx, ly, lz);
    const double h[3] = {g->llenx / lx, g->lleny / ly, g->llenz / lz};
    const int L[3] = {lx, ly, lz};
    memset(b, 0, sizeof(double) * n);
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) {
                long c = IX(i, j, k);
                int idx[3] = {i, j, k};
                for (int ax = 0; ax < 3; ax++) {
                    if (bc[2 * ax] == ORC_PERI) continue;
                    for (int side = 0; side < 2; side++) {
                        int pos = idx[ax];
                        if ((side == 0 && pos != 1) || (side == 1 && pos != L[ax])) continue;
                        int code = bc[2 * ax + side];
                        long fi;
                        if (ax == 0) fi = (j - 1) + (long)ly * (k - 1);
                        else if (ax == 1) fi = (i - 1) + (long)lx * (k - 1);
                        else fi = (i - 1) + (long)lx * (j - 1);
                        double gv = bcvals[2 * ax + side][fi];
                        double dx = h[ax];
                        if (code == ORC_DIRC) {
                            double vb = vel[ax * ng + GX(i, j, k)], kb = dcoeff[GX(i, j, k)];
                            double wL, wR;
                            orc_sg_face(vb, vb, kb, kb, 0.5 * dx, &wL, &wR);
                            if (side == 0) b[c] += wL * gv / dx;
                            else b[c] -= wR * gv / dx;
                        } else if (code == ORC_FLUX) {
                            b[c] -= gv / dx;
                        }
                    }
                }
                b[c] += source[GX(i, j, k)];
            }
}

static inline long nbr(int lx, int ly, int lz, const int* bc, int i, int j, int k, int q)
{
    /* q: 1 xm, 2 xp, 3 ym, 4 yp, 5 zm, 6 zp; -1 when outside */
    int d = (q - 1) / 2, s = (q & 1) ? -1 : 1;
    int p[3] = {i, j, k}, L[3] = {lx, ly, lz};
    p[d] += s;
    if (p[d] < 1 || p[d] > L[d]) {
        if (bc[2 * d] != ORC_PERI) return -1;
        p[d] = p[d] < 1 ? L[d] : 1;
    }
    return IX(p[0], p[1], p[2]);
}

void orc_rows_apply(const orc_grid* g, const int* bc, const double* rows, const double* u, double* Au)
{
    const int lx = g->lx, ly = g->ly, lz = g->lz;
    const long n = nin(lx, ly, lz);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) {
                long c = IX(i, j, k);
                double s = R7(0, c) * u[c];
                for (int q = 1; q <= 6; q++) {
                    long m = nbr(lx, ly, lz, bc, i, j, k, q);
                    if (m >= 0) s += R7(q, c) * u[m];
                }
                Au[c] = s;
            }
}

/* (A^T)_{c,m} = A_{m,c}: the xp coefficient of row c of A^T is the xm
 * coefficient of row c+x of A, etc. */
void orc_rows_transpose(const orc_grid* g, const int* bc, const double* rows, double* rowsT)
{
    const int lx = g->lx, ly = g->ly, lz = g->lz;
    const long n = nin(lx, ly, lz);
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) {
                long c = IX(i, j, k);
                rowsT[c] = R7(0, c);
                for (int q = 1; q <= 6; q++) {
                    long m = nbr(lx, ly, lz, bc, i, j, k, q);
                    int opp = (q & 1) ? q + 1 : q - 1;
                    rowsT[(long)q * n + c] = m >= 0 ? rows[(long)opp * n + m] : 0.0;
                }
            }
}

/* ---- correction-scheme multigrid over rows ---- */
struct orc_mg {
    orc_grid g;
    int bc[6];
    int nlev;
    dims3 d[32];
    geo3 geo[32];
    double* rows[32];
    double* u[32];
    double* f[32];
    double* r[32];
    double* lu;  /* coarsest LU (row-major, n x n) */
    int* piv;
};

const double* orc_mg_rows(const orc_mg* mg, int level) { return mg->rows[level]; }

int orc_mg_levels(const orc_mg* mg, int* dims)
{
    for (int l = 0; l < mg->nlev && dims; l++) {
        dims[3 * l] = mg->d[l].lx; dims[3 * l + 1] = mg->d[l].ly; dims[3 * l + 2] = mg->d[l].lz;
    }
    return mg->nlev;
}

orc_mg* orc_mg_create(const orc_grid* g, int flux, int timederiv, double dt,
                      const double* vel, const double* dcoeff, const double* reac,
                      const int* bc, int transpose)
{
    orc_mg* mg = (orc_mg*)calloc(1, sizeof(orc_mg));
    mg->g = *g;
    memcpy(mg->bc, bc, sizeof(int) * 6);
    dims3 d = {g->lx, g->ly, g->lz};
    geo3 G = geo_fine(g);
    long ng = ngh(d.lx, d.ly, d.lz);
    double* v = zalloc(3 * ng);
    double* kc = zalloc(ng);
    double* rc = zalloc(ng);
    memcpy(v, vel, sizeof(double) * 3 * ng);
    memcpy(kc, dcoeff, sizeof(double) * ng);
    memcpy(rc, reac, sizeof(double) * ng);
    int l = 0;
    for (;;) {
        long n = nin(d.lx, d.ly, d.lz);
        mg->d[l] = d;
        mg->geo[l] = G;
        mg->rows[l] = zalloc(7 * n);
        build_rows_geo(&G, flux, timederiv, dt, v, kc, rc, bc, mg->rows[l]);
        if (transpose) {
            orc_grid gl = *g;
            gl.lx = d.lx; gl.ly = d.ly; gl.lz = d.lz;
            double* t = zalloc(7 * n);
            orc_rows_transpose(&gl, bc, mg->rows[l], t);
            free(mg->rows[l]);
            mg->rows[l] = t;
        }
        mg->u[l] = zalloc(n);
        mg->f[l] = zalloc(n);
        mg->r[l] = zalloc(n);
        if (is_coarsest(g, d) || l == 31) break;
        geo3 Gc = geo_coarse(g, G);
        dims3 c = {Gc.n[0], Gc.n[1], Gc.n[2]};
        long ngc = ngh(c.lx, c.ly, c.lz);
        double* vc = zalloc(3 * ngc);
        double* kcc = zalloc(ngc);
        double* rcc = zalloc(ngc);
        for (int q = 0; q < 3; q++) restrict_fieldg(g, &G, &Gc, v + q * ng, 1, vc + q * ngc, 1);
        restrict_fieldg(g, &G, &Gc, kc, 1, kcc, 1);
        restrict_fieldg(g, &G, &Gc, rc, 1, rcc, 1);
        free(v); free(kc); free(rc);
        v = vc; kc = kcc; rc = rcc;
        d = c; G = Gc; ng = ngc; l++;
    }
    free(v); free(kc); free(rc);
    mg->nlev = l + 1;
    /* dense LU (partial pivoting) of the coarsest operator */
    {
        dims3 c = mg->d[l];
        int lx = c.lx, ly = c.ly, lz = c.lz;
        long n = nin(lx, ly, lz);
        double* A = zalloc(n * n);
        const double* rows = mg->rows[l];
        for (int k = 1; k <= lz; k++)
            for (int j = 1; j <= ly; j++)
                for (int i = 1; i <= lx; i++) {
                    long cc = IX(i, j, k);
                    A[cc * n + cc] += rows[cc];
                    for (int q = 1; q <= 6; q++) {
                        long m = nbr(lx, ly, lz, bc, i, j, k, q);
                        if (m >= 0) A[cc * n + m] += rows[(long)q * n + cc];
                    }
                }
        int* piv = (int*)calloc((size_t)n, sizeof(int));
        for (long p = 0; p < n; p++) {
            long best = p;
            for (long r = p + 1; r < n; r++)
                if (fabs(A[r * n + p]) > fabs(A[best * n + p])) best = r;
            piv[p] = (int)best;
            if (best != p)
                for (long q = 0; q < n; q++) { double t = A[p * n + q]; A[p * n + q] = A[best * n + q]; A[best * n + q] = t; }
            double dp = A[p * n + p];
            for (long r = p + 1; r < n; r++) {
                double fct = (dp != 0.0) ? A[r * n + p] / dp : 0.0;
                A[r * n + p] = fct;
                for (long q = p + 1; q < n; q++) A[r * n + q] -= fct * A[p * n + q];
            }
        }
        mg->lu = A;
        mg->piv = piv;
    }
    return mg;
}

void orc_mg_destroy(orc_mg* mg)
{
    if (!mg) return;
    for (int l = 0; l < mg->nlev; l++) { free(mg->rows[l]); free(mg->u[l]); free(mg->f[l]); free(mg->r[l]); }
    free(mg->lu); free(mg->piv); free(mg);
}

/* one colour pass: every cell of the colour takes its new value from the
 * state at the start of the pass (the reference computes offdiag for all
 * cells with find_AX before updating a colour, discretepde.f90:204-227) */
static void rows_colour(const orc_mg* mg, int l, double* u, const double* f, int red)
{
    const dims3 d = mg->d[l];
    const int lx = d.lx, ly = d.ly, lz = d.lz;
    const long n = nin(lx, ly, lz);
    const double* rows = mg->rows[l];
    double* nu = mg->r[l];
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++) {
                if (((i + j + k) & 1) != red) continue;
                long c = IX(i, j, k);
                double s = 0.0;
                for (int q = 1; q <= 6; q++) {
                    long m = nbr(lx, ly, lz, mg->bc, i, j, k, q);
                    if (m >= 0) s += R7(q, c) * u[m];
                }
                nu[c] = (f[c] - s) / R7(0, c);
            }
    for (int k = 1; k <= lz; k++)
        for (int j = 1; j <= ly; j++)
            for (int i = 1; i <= lx; i++)
                if (((i + j + k) & 1) == red) u[IX(i, j, k)] = nu[IX(i, j, k)];
}

static void coarse_solve(const orc_mg* mg, double* u, const double* f)
{
    const dims3 d = mg->d[mg->nlev - 1];
    long n = nin(d.lx, d.ly, d.lz);
    const double* A = mg->lu;
    double* y = zalloc(n);
    memcpy(y, f, sizeof(double) * n);
    for (long p = 0; p < n; p++) {
        long q = mg->piv[p];
        if (q != p) { double t = y[p]; y[p] = y[q]; y[q] = t; }
        for (long r = p + 1; r < n; r++) y[r] -= A[r * n + p] * y[p];
    }
    for (long p = n - 1; p >= 0; p--) {
        double s = y[p];
        for (long q = p + 1; q < n; q++) s -= A[p * n + q] * u[q];
        u[p] = (A[p * n + p] != 0.0) ? s / A[p * n + p] : 0.0;
    }
    free(y);
}

static void mg_rec(orc_mg* mg, int l, double* u, const double* f)
{
    if (l == mg->nlev - 1) { coarse_solve(mg, u, f); return; }
    const dims3 fd = mg->d[l], cd = mg->d[l + 1];
    const int cell = mg->g.hier == ORC_HIER_CELL;
    const long n = nin(fd.lx, fd.ly, fd.lz), nc = nin(cd.lx, cd.ly, cd.lz);
    for (int s = 0; s < mg->g.nu1; s++) { rows_colour(mg, l, u, f, 1); rows_colour(mg, l, u, f, 0); }
    double* r = zalloc(n);
    {
        orc_grid gl = mg->g; gl.lx = fd.lx; gl.ly = fd.ly; gl.lz = fd.lz;
        orc_rows_apply(&gl, mg->bc, mg->rows[l], u, r);
    }
#pragma omp parallel for schedule(static)
    for (long c = 0; c < n; c++) r[c] = f[c] - r[c];
    double* fc = mg->f[l + 1];
    double* uc = mg->u[l + 1];
    restrict_fieldg(&mg->g, &mg->geo[l], &mg->geo[l + 1], r, 0, fc, 0);
    memset(uc, 0, sizeof(double) * nc);
    mg_rec(mg, l + 1, uc, fc);
    /* ghosted copy of the coarse correction with the prolongation ghosts:
     * DIRC -> -e, other physical -> +e, periodic -> wrap */
    long ngc = ngh(cd.lx, cd.ly, cd.lz);
    double* eg = zalloc(ngc);
    double* zb[6];
    int fa[3] = {cd.ly * cd.lz, cd.lx * cd.lz, cd.lx * cd.ly};
    for (int q = 0; q < 6; q++) zb[q] = zalloc(fa[q / 2]);
    {
        int lx = cd.lx, ly = cd.ly;
        for (int k = 1; k <= cd.lz; k++)
            for (int j = 1; j <= cd.ly; j++)
                for (int i = 1; i <= cd.lx; i++) {
                    long src = (i - 1) + (long)cd.lx * ((j - 1) + (long)cd.ly * (k - 1));
                    eg[GX(i, j, k)] = uc[src];
                }
    }
    ghost_update(cd, eg, mg->bc, (const double* const*)zb);
    long ngf = ngh(fd.lx, fd.ly, fd.lz);
    double* ef = zalloc(ngf);
    prolongg(&mg->g, &mg->geo[l], &mg->geo[l + 1], mg->bc, eg, ef);
    {
        int lx = fd.lx, ly = fd.ly;
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= fd.lz; k++)
            for (int j = 1; j <= fd.ly; j++)
                for (int i = 1; i <= fd.lx; i++)
                    u[(i - 1) + (long)fd.lx * ((j - 1) + (long)fd.ly * (k - 1))] += ef[GX(i, j, k)];
    }
    for (int s = 0; s < mg->g.nu2; s++) { rows_colour(mg, l, u, f, 1); rows_colour(mg, l, u, f, 0); }
    for (int q = 0; q < 6; q++) free(zb[q]);
    free(eg); free(ef); free(r);
}

void orc_mg_vcycle(orc_mg* mg, double* u, const double* f) { mg_rec(mg, 0, u, f); }

static double dot(const double* a, const double* b, long n)
{
    double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
    for (long i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* host threads of the oracle's OpenMP loops (the CPU baseline times one
 * thread and all threads) */
void orc_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int orc_get_threads(void) { return omp_get_max_threads(); }

int orc_mg_solve(orc_mg* mg, const double* b, double* x, int maxit, double tol, double* relres_out)
{
    const dims3 d = mg->d[0];
    const long n = nin(d.lx, d.ly, d.lz);
    orc_grid gl = mg->g; gl.lx = d.lx; gl.ly = d.ly; gl.lz = d.lz;
    double* r = zalloc(n);
    double* e = zalloc(n);
    double bn = sqrt(dot(b, b, n));
    if (bn == 0.0) bn = 1.0;
    int it = 0;
    double rel = 0.0;
    for (;;) {
        orc_rows_apply(&gl, mg->bc, mg->rows[0], x, r);
#pragma omp parallel for schedule(static)
        for (long c = 0; c < n; c++) r[c] = b[c] - r[c];
        rel = sqrt(dot(r, r, n)) / bn;
        if (relres_out) relres_out[it] = rel;
        if (rel <= tol || it >= maxit) break;
        memset(e, 0, sizeof(double) * n);
        orc_mg_vcycle(mg, e, r);
#pragma omp parallel for schedule(static)
        for (long c = 0; c < n; c++) x[c] += e[c];
        it++;
    }
    free(r); free(e);
    return it;
}

/* right-preconditioned FGMRES(m): the flexible form of the 1D
 * MG-preconditioned GMRES (mps1d/source/gmres.f90:182-375 with
 * mgridprecond, convdiff.f90:659-689); CGS2 orthogonalisation. */
int orc_fgmres(orc_mg* mg, const double* b, double* x, int m, int maxit, double tol, double* relres_out)
{
    const dims3 d = mg->d[0];
    const long n = nin(d.lx, d.ly, d.lz);
    orc_grid gl = mg->g; gl.lx = d.lx; gl.ly = d.ly; gl.lz = d.lz;
    double* V = zalloc(n * (m + 1));
    double* Z = zalloc(n * m);
    double* w = zalloc(n);
    double* H = zalloc((long)(m + 1) * m);
    double* cs = zalloc(m);
    double* sn = zalloc(m);
    double* gq = zalloc(m + 1);
    double* y = zalloc(m);
    double bn = sqrt(dot(b, b, n));
    if (bn == 0.0) bn = 1.0;
    int total = 0;
    double rel = 0.0;
#define HH(i, j) H[(long)(i) + (long)(m + 1) * (j)]
    for (;;) {
        orc_rows_apply(&gl, mg->bc, mg->rows[0], x, w);
        for (long c = 0; c < n; c++) w[c] = b[c] - w[c];
        double beta = sqrt(dot(w, w, n));
        rel = beta / bn;
        if (relres_out) relres_out[total] = rel;
        if (rel <= tol || total >= maxit) break;
        for (long c = 0; c < n; c++) V[c] = w[c] / beta;
        memset(gq, 0, sizeof(double) * (m + 1));
        memset(H, 0, sizeof(double) * (m + 1) * m);
        gq[0] = beta;
        int j;
        for (j = 0; j < m && total < maxit; j++) {
            double* z = Z + n * j;
            memset(z, 0, sizeof(double) * n);
            orc_mg_vcycle(mg, z, V + n * j);
            orc_rows_apply(&gl, mg->bc, mg->rows[0], z, w);
            for (int pass = 0; pass < 2; pass++)
                for (int i = 0; i <= j; i++) {
                    double h = dot(V + n * i, w, n);
                    HH(i, j) += h;
#pragma omp parallel for schedule(static)
                    for (long c = 0; c < n; c++) w[c] -= h * V[n * i + c];
                }
            double hn = sqrt(dot(w, w, n));
            HH(j + 1, j) = hn;
            if (hn > 0.0)
                for (long c = 0; c < n; c++) V[n * (j + 1) + c] = w[c] / hn;
            for (int i = 0; i < j; i++) {
                double t = cs[i] * HH(i, j) + sn[i] * HH(i + 1, j);
                HH(i + 1, j) = -sn[i] * HH(i, j) + cs[i] * HH(i + 1, j);
                HH(i, j) = t;
            }
            double a = HH(j, j), bb = HH(j + 1, j), rr = sqrt(a * a + bb * bb);
            cs[j] = rr == 0.0 ? 1.0 : a / rr;
            sn[j] = rr == 0.0 ? 0.0 : bb / rr;
            HH(j, j) = cs[j] * a + sn[j] * bb;
            HH(j + 1, j) = 0.0;
            gq[j + 1] = -sn[j] * gq[j];
            gq[j] = cs[j] * gq[j];
            total++;
            if (relres_out) relres_out[total] = fabs(gq[j + 1]) / bn;
            if (fabs(gq[j + 1]) / bn <= tol || hn == 0.0) { j++; break; }
        }
        for (int i = j - 1; i >= 0; i--) {
            double s = gq[i];
            for (int q = i + 1; q < j; q++) s -= HH(i, q) * y[q];
            y[i] = s / HH(i, i);
        }
        for (int i = 0; i < j; i++)
#pragma omp parallel for schedule(static)
            for (long c = 0; c < n; c++) x[c] += y[i] * Z[n * i + c];
    }
#undef HH
    free(V); free(Z); free(w); free(H); free(cs); free(sn); free(gq); free(y);
    return total;
}
