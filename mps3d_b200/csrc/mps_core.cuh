// mps_core.cuh -- device-side data layout and per-cell stencil arithmetic of
// the B200 multigrid solver.
//
// Layout ("red/black split"): every level-l field of nx*ny*nz cells is stored
// as two colour halves.  Cell (i,j,k) (0-based) has colour c = (i+j+k)&1
// (c = 0 is the reference's "red": odd (gi+gj+gk) with 1-based indices,
// mgridlib/discretepde.f90:49-57, updated first, :207-227) and lives at
//     half c, offset (i>>1) + P*(j + ny*k)
// with P >= ceil(nx/2) a padded row pitch.  A colour pass therefore reads one
// half densely (the other colour) and writes the other densely: no lanes
// carry the wrong colour and no DRAM sector is half used.  Pad entries are
// zero and never written.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace mps {

enum { BC_DIRC = 1, BC_FLUX = 2, BC_ZGRD = 3, BC_PERI = 4, BC_DZGD = 5 };
enum { F_LEFT = 0, F_RIGHT, F_BOTTOM, F_TOP, F_BACK, F_FRONT };

// unsigned division by a run-time invariant d (n < 2^31): q = (n*M) >> s
struct FastDiv {
    unsigned long long M;
    int s;
    unsigned d;
    __host__ void init(unsigned dv)
    {
        d = dv;
        int l = 0;
        while ((1ull << l) < dv) l++;
        s = 32 + l;
        M = ((1ull << s) + dv - 1) / dv;
    }
    __host__ __device__ __forceinline__ unsigned div(unsigned n) const
    {
        return (unsigned)(((unsigned long long)n * M) >> s);
    }
};

// geometry of one level in split layout.  Cell widths: every level is
// uniform along an axis except possibly its last cell (the geometric
// hierarchy merges the odd cell of an odd size into the last coarse cell);
// w = regular width, wl = last-cell width.  Face coefficients of a row are
// 1/(d * w_row) with d the distance between the two centres: cr between
// regular cells, cl in the row of the last cell, cp in the row of its
// regular neighbour; Dirichlet faces 2/w^2 (dr) or 2/wl^2 (dlast).  On a
// uniform level all of them reduce to find_AX's 1/dx^2 and 2/dx^2.
struct Lev {
    int nx, ny, nz;   // cells
    int nh;           // (nx+1)/2: max cells of one colour in an x row
    int P;            // padded pitch (elements) of a colour row
    long long half;   // P*ny*nz: elements of one colour half
    int per[3];       // periodic flags x,y,z
    int bc[6];        // BC codes LEFT..FRONT
    double w[3], wl[3];
    double cr[3], cl[3], cp[3], dr[3], dlast[3];
    int fast_lo[3], fast_hi[3];  // index range per axis where a row has six
                                 // neighbours of the other colour at regular
                                 // spacing (interior fast path)
    FastDiv divP, divNy;
    unsigned rows;    // ny*nz
};

__host__ __device__ __forceinline__ int lev_n(const Lev& L, int ax) { return ax == 0 ? L.nx : (ax == 1 ? L.ny : L.nz); }
// face coefficient of row i towards neighbour m along ax
__host__ __device__ __forceinline__ double fcoef(const Lev& L, int ax, int i, int m)
{
    const int n = lev_n(L, ax);
    return i == n - 1 ? L.cl[ax] : (m == n - 1 ? L.cp[ax] : L.cr[ax]);
}
__host__ __device__ __forceinline__ double dcoef(const Lev& L, int ax, int i)
{
    return i == lev_n(L, ax) - 1 ? L.dlast[ax] : L.dr[ax];
}
__host__ __device__ __forceinline__ double cwidth(const Lev& L, int ax, int i)
{
    return i == lev_n(L, ax) - 1 ? L.wl[ax] : L.w[ax];
}

// one entry of a 1-D prolongation table: e_f = (1-t) e[j0] + t e[j1]
struct Lin {
    int j0, j1;
    double t;
};

// transfer between level l (fine) and l+1 (coarse)
struct Xfer {
    const Lin* tab[3];  // per-axis tables over the fine index (geometric hierarchy)
    int geom;         // 0: the reference's CELL transfers, 1: geometric
    int nf[3], nc[3];
    double rf[3], Rc[3];  // wl_f / w_f and wl_c / w_f
    int per[3];
};

__host__ __device__ __forceinline__ long long soff(const Lev& L, int i, int j, int k)
{
    return (long long)(i >> 1) + (long long)L.P * ((long long)j + (long long)L.ny * k);
}
__host__ __device__ __forceinline__ int scol(int i, int j, int k) { return (i + j + k) & 1; }

// decode a flattened (h, j, k) thread index of colour c -> (i, j, k); false when padding
__device__ __forceinline__ bool decode(const Lev& L, unsigned t, int c, int& i, int& j, int& k)
{
    unsigned row = L.divP.div(t);
    unsigned hh = t - row * (unsigned)L.P;
    if (row >= L.rows) return false;
    unsigned kk = L.divNy.div(row);
    j = (int)(row - kk * (unsigned)L.ny);
    k = (int)kk;
    i = 2 * (int)hh + ((j + k + c) & 1);
    return i < L.nx;
}

// decode a flattened natural index (i fastest) -> (i,j,k)
struct NatDiv {
    FastDiv dx, dy;
    int nx, ny;
};

template <class T>
struct Split {  // a field in split layout: c[0] red half, c[1] black half
    T* c[2];
    __device__ __forceinline__ T get(const Lev& L, int i, int j, int k) const
    {
        return c[scol(i, j, k)][soff(L, i, j, k)];
    }
};
template <class T>
struct CSplit {
    const T* c[2];
    __device__ __forceinline__ T get(const Lev& L, int i, int j, int k) const
    {
        return __ldg(&c[scol(i, j, k)][soff(L, i, j, k)]);
    }
    __device__ __forceinline__ T at(int col, int off) const { return __ldg(&c[col][off]); }
};

// neighbour along axis ax (0..2), direction s (-1/+1); returns false at a
// physical (non-periodic) boundary
__device__ __forceinline__ bool nbr(const Lev& L, int ax, int s, int& i, int& j, int& k)
{
    int n = ax == 0 ? L.nx : (ax == 1 ? L.ny : L.nz);
    int& p = ax == 0 ? i : (ax == 1 ? j : k);
    int q = p + s;
    if (q < 0 || q >= n) {
        if (!L.per[ax]) return false;
        q = q < 0 ? q + n : q - n;
    }
    p = q;
    return true;
}

// ---- operator classes -------------------------------------------------
// KOp: -div(k grad u) + dex*u with a cell coefficient k and the reference's
// arithmetic face mean k_half = (k_l + k_r)/2 (findcellcontributions,
// discretepde.f90:646-652), Dirichlet face 2 k_c/dx^2 (:810), no convection.
// dex = -reac + 1/dt (:1103-1106).  k or dex may be uniform (pointer null).
template <class T>
struct KOp {
    const T* k[2];
    T kc;
    const T* dex[2];
    T dexc;
};
// ROp: explicit rows d, xm, xp, ym, yp, zm, zp (each a split field); used for
// convection (upwind or Scharfetter-Gummel) and for transposed operators.
template <class T>
struct ROp {
    const T* r[7][2];
};

template <class T>
__device__ __forceinline__ T kval(const KOp<T>& op, const Lev& L, int i, int j, int k)
{
    return op.k[0] ? __ldg(&op.k[scol(i, j, k)][soff(L, i, j, k)]) : op.kc;
}

// diag and sum_n a_n u_n of row (i,j,k)
template <class T, class U>
__device__ __forceinline__ void row_eval(const KOp<T>& op, const Lev& L, const U& u, int i, int j,
                                         int k, T& diag, T& off)
{
    const T kc = kval(op, L, i, j, k);
    T d = op.dex[0] ? __ldg(&op.dex[scol(i, j, k)][soff(L, i, j, k)]) : op.dexc;
    T o = T(0);
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
        const int p = ax == 0 ? i : (ax == 1 ? j : k);
#pragma unroll
        for (int s = -1; s <= 1; s += 2) {
            int a = i, b = j, c = k;
            if (nbr(L, ax, s, a, b, c)) {
                const int q = ax == 0 ? a : (ax == 1 ? b : c);
                T w = T(0.5) * (kc + kval(op, L, a, b, c)) * (T)fcoef(L, ax, p, q);
                d += w;
                o -= w * u.get(L, a, b, c);
            } else if (L.bc[2 * ax + (s > 0)] == BC_DIRC) {
                d += kc * (T)dcoef(L, ax, p);
            }
        }
    }
    diag = d;
    off = o;
}

template <class T, class U>
__device__ __forceinline__ void row_eval(const ROp<T>& op, const Lev& L, const U& u, int i, int j,
                                         int k, T& diag, T& off)
{
    const int c = scol(i, j, k);
    const long long o0 = soff(L, i, j, k);
    T d = __ldg(&op.r[0][c][o0]);
    T o = T(0);
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
#pragma unroll
        for (int s = -1; s <= 1; s += 2) {
            int a = i, b = j, cc = k;
            if (nbr(L, ax, s, a, b, cc)) {
                T w = __ldg(&op.r[1 + 2 * ax + (s > 0)][c][o0]);
                o += w * u.get(L, a, b, cc);
            }
        }
    }
    diag = d;
    off = o;
}

// interior fast path: the six neighbours of (i,j,k) have the other colour and
// sit at 32-bit offsets o+q-1, o+q (x), o-+P (y), o-+P*ny (z) of the other
// half, q = i&1; all faces have the regular coefficient cr.
__device__ __forceinline__ bool is_fast(const Lev& L, int i, int j, int k)
{
    return i >= L.fast_lo[0] && i <= L.fast_hi[0] && j >= L.fast_lo[1] && j <= L.fast_hi[1] &&
           k >= L.fast_lo[2] && k <= L.fast_hi[2];
}

template <class T, class U>
__device__ __forceinline__ void row_eval_fast(const KOp<T>& op, const Lev& L, const U& u, int i, int j, int k,
                                              T& diag, T& off)
{
    const int cc = (i + j + k) & 1, oc = cc ^ 1;
    const int o = (i >> 1) + L.P * (j + L.ny * k);
    const int q = i & 1, sy = L.P, sz = L.P * L.ny;
    const int n0 = o + q - 1, n1 = o + q, n2 = o - sy, n3 = o + sy, n4 = o - sz, n5 = o + sz;
    const T cx = (T)L.cr[0], cy = (T)L.cr[1], cz = (T)L.cr[2];
    const T d0 = op.dex[0] ? __ldg(&op.dex[cc][o]) : op.dexc;
    const T u0 = u.at(oc, n0), u1 = u.at(oc, n1), u2 = u.at(oc, n2), u3 = u.at(oc, n3), u4 = u.at(oc, n4),
            u5 = u.at(oc, n5);
    if (op.k[0]) {
        const T* ko = op.k[oc];
        const T kc = __ldg(&op.k[cc][o]);
        const T w0 = (kc + __ldg(&ko[n0])) * cx, w1 = (kc + __ldg(&ko[n1])) * cx;
        const T w2 = (kc + __ldg(&ko[n2])) * cy, w3 = (kc + __ldg(&ko[n3])) * cy;
        const T w4 = (kc + __ldg(&ko[n4])) * cz, w5 = (kc + __ldg(&ko[n5])) * cz;
        diag = d0 + T(0.5) * (((w0 + w1) + (w2 + w3)) + (w4 + w5));
        off = T(-0.5) * (((w0 * u0 + w1 * u1) + (w2 * u2 + w3 * u3)) + (w4 * u4 + w5 * u5));
    } else {
        const T kc = op.kc;
        diag = d0 + T(2) * kc * ((cx + cy) + cz);
        off = -kc * ((cx * (u0 + u1) + cy * (u2 + u3)) + cz * (u4 + u5));
    }
}

template <class T, class U>
__device__ __forceinline__ void row_eval_fast(const ROp<T>& op, const Lev& L, const U& u, int i, int j, int k,
                                              T& diag, T& off)
{
    const int cc = (i + j + k) & 1, oc = cc ^ 1;
    const int o = (i >> 1) + L.P * (j + L.ny * k);
    const int q = i & 1, sy = L.P, sz = L.P * L.ny;
    diag = __ldg(&op.r[0][cc][o]);
    off = ((__ldg(&op.r[1][cc][o]) * u.at(oc, o + q - 1) + __ldg(&op.r[2][cc][o]) * u.at(oc, o + q)) +
           (__ldg(&op.r[3][cc][o]) * u.at(oc, o - sy) + __ldg(&op.r[4][cc][o]) * u.at(oc, o + sy))) +
          (__ldg(&op.r[5][cc][o]) * u.at(oc, o - sz) + __ldg(&op.r[6][cc][o]) * u.at(oc, o + sz));
}

// dispatch: fast path in the interior, general path at boundaries, periodic
// seams and next to a non-uniform last cell
template <class T, class Op, class U>
__device__ __forceinline__ void row_any(const Op& op, const Lev& L, const U& u, int i, int j, int k, T& diag,
                                        T& off)
{
    if (is_fast(L, i, j, k)) row_eval_fast(op, L, u, i, j, k, diag, off);
    else row_eval(op, L, u, i, j, k, diag, off);
}

// red-black Gauss-Seidel point update u_c = (f_c - offdiag)/diag
// (perform_gseidel_smoothing, discretepde.f90:212,226)
template <class T>
__device__ __forceinline__ T gs_value(T f, T diag, T off)
{
    return (f - off) / diag;
}

// Scharfetter-Gummel face weights (find_sg_exponential_flux,
// mps1d/source/convdiff.f90:10-64): flux = wL*uL + wR*uR
__host__ __device__ inline void sg_face(double cL, double cR, double DL, double DR, double dx, double& wL,
                                        double& wR)
{
    const double eps = 1.0e-10;
    double c_half = 0.5 * (cL + cR);
    double D_half = 2.0 * DL * DR / (DL + DR + eps);
    double sign_c = c_half <= 0.0 ? -1.0 : 1.0;
    wL = 0.0;
    wR = 0.0;
    if (fabs(D_half) < eps) {
        wL = cL * 0.5 * (1.0 + sign_c);
        wR = cR * 0.5 * (1.0 - sign_c);
    } else {
        double Pe = c_half * dx / D_half;
        if (fabs(Pe) < eps) {
            wL = D_half / dx;
            wR = -D_half / dx;
        } else if (Pe > 0.0) {
            wL = c_half / (1.0 - exp(-Pe));
            wR = -c_half * exp(-Pe) / (1.0 - exp(-Pe));
        } else {
            wL = c_half * exp(Pe) / (exp(Pe) - 1.0);
            wR = -c_half / (exp(Pe) - 1.0);
        }
    }
}

// upwind face weights of findcellcontributions (discretepde.f90:646-668)
// written as a flux per unit area F = wL*uL + wR*uR over a centre distance d
__host__ __device__ inline void upwind_face(double vl, double vr, double kl, double kr, double d, double& wL,
                                            double& wR)
{
    double kh = 0.5 * (kl + kr) / d;
    double vh = 0.5 * (vl + vr);
    wL = kh;
    wR = -kh;
    if (vh > 0.0) wL += vh;
    else wR += vh;
}

// geometric prolongation bracket along one axis: the fine centre of index i0
// lies between coarse centres j0 = J and j1 = J+1 (either may be a ghost,
// -1 or nc), e = (1-t) e[j0] + t e[j1].  Positions in units of the fine
// regular width; ghost centres mirror across the wall or wrap (periodic).
__host__ __device__ __forceinline__ void geom_lin(const Xfer& X, int ax, int i0, int& j0, int& j1, double& t)
{
    const int nf = X.nf[ax], nc = X.nc[ax];
    if (nf == nc) { j0 = j1 = i0; t = 0.0; return; }
    const int per = X.per[ax];
    const double rf = X.rf[ax], Rc = X.Rc[ax];
    const double xf = (i0 == nf - 1) ? (nf - 1) + 0.5 * rf : i0 + 0.5;
    const double Ltot = 2.0 * (nc - 1) + Rc;
    const double X0 = (nc == 1) ? 0.5 * Rc : 1.0;
    const double Xl = 2.0 * (nc - 1) + 0.5 * Rc;
    const int I = (i0 >> 1) < nc - 1 ? (i0 >> 1) : nc - 1;
    const double XI = (I == nc - 1) ? Xl : 2.0 * I + 1.0;
    const int J = xf >= XI ? I : I - 1;
    double XJ, XJ1;
    if (J < 0) XJ = per ? Xl - Ltot : -X0;
    else XJ = (J == nc - 1) ? Xl : 2.0 * J + 1.0;
    if (J + 1 > nc - 1) XJ1 = per ? X0 + Ltot : 2.0 * Ltot - Xl;
    else XJ1 = (J + 1 == nc - 1) ? Xl : 2.0 * (J + 1) + 1.0;
    j0 = J;
    j1 = J + 1;
    t = (xf - XJ) / (XJ1 - XJ);
}

}  // namespace mps
