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

// unsigned division by a run-time invariant d with a 32-bit multiply-high
// (Granlund-Montgomery): q = (t + ((n - t) >> 1)) >> (l - 1), t = mulhi(M, n),
// l = ceil(log2 d), M = floor(2^32 (2^l - d) / d) + 1; exact for all 32-bit n
struct FastDiv {
    unsigned M;
    int l;
    unsigned d;
    __host__ void init(unsigned dv)
    {
        d = dv;
        l = 0;
        while ((1ull << l) < dv) l++;
        M = (unsigned)(((1ull << 32) * ((1ull << l) - dv)) / dv + 1);
    }
    __host__ __device__ __forceinline__ unsigned div(unsigned n) const
    {
        if (d == 1) return n;
#ifdef __CUDA_ARCH__
        const unsigned t = __umulhi(M, n);
#else
        const unsigned t = (unsigned)(((unsigned long long)M * n) >> 32);
#endif
        return (t + ((n - t) >> 1)) >> (l - 1);
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
    int uniform;      // all cells of the level have the regular widths
    FastDiv divP, divNy, divG;  // by P, ny, P/4
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

// select one of two pointers without indexing a parameter array with a
// run-time index (which would copy the array to local memory)
template <class P>
__host__ __device__ __forceinline__ P sel(const P* two, int c)
{
    return c ? two[1] : two[0];
}

template <class T>
struct Split {  // a field in split layout: c[0] red half, c[1] black half
    T* c[2];
    __host__ __device__ __forceinline__ T* half(int col) const { return col ? c[1] : c[0]; }
    __device__ __forceinline__ T get(const Lev& L, int i, int j, int k) const
    {
        return half(scol(i, j, k))[soff(L, i, j, k)];
    }
};
template <class T>
struct CSplit {
    const T* c[2];
    __host__ __device__ __forceinline__ const T* half(int col) const { return col ? c[1] : c[0]; }
    __device__ __forceinline__ T get(const Lev& L, int i, int j, int k) const
    {
        return __ldg(&half(scol(i, j, k))[soff(L, i, j, k)]);
    }
    __device__ __forceinline__ T at(int col, int off) const { return __ldg(&half(col)[off]); }
    __device__ __forceinline__ const T* ptr(int col) const { return half(col); }
    __device__ __forceinline__ T ld(const T* p, int off) const { return __ldg(&p[off]); }
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
    return op.k[0] ? __ldg(&sel(op.k, scol(i, j, k))[soff(L, i, j, k)]) : op.kc;
}

// ---- row evaluation: diag and sum_n a_n u_n of row (i,j,k) ----
// Branch-light and free of local memory: each face is handled by an
// axis-templated helper (compile-time field indices, no references or
// arrays), the neighbour's colour and split offset are computed directly,
// periodic faces wrap, physical faces add their Dirichlet term.

// neighbour index along AX in direction S, wrapped when periodic; false at a
// physical boundary
template <int AX, int S>
__device__ __forceinline__ bool nbr_idx(const Lev& L, int p, int& q)
{
    const int n = AX == 0 ? L.nx : (AX == 1 ? L.ny : L.nz);
    q = p + S;
    if (q < 0 || q >= n) {
        if (!L.per[AX]) return false;
        q = q < 0 ? n - 1 : 0;
    }
    return true;
}

template <int AX>
__device__ __forceinline__ double fcoef_ax(const Lev& L, int p, int q)
{
    const int n = AX == 0 ? L.nx : (AX == 1 ? L.ny : L.nz);
    return p == n - 1 ? L.cl[AX] : (q == n - 1 ? L.cp[AX] : L.cr[AX]);
}
template <int AX>
__device__ __forceinline__ double dcoef_ax(const Lev& L, int p)
{
    const int n = AX == 0 ? L.nx : (AX == 1 ? L.ny : L.nz);
    return p == n - 1 ? L.dlast[AX] : L.dr[AX];
}

template <class T, int AX, int S, class U>
__device__ __forceinline__ void kface(const KOp<T>& op, const Lev& L, const U& u, int i, int j, int k, T kc,
                                      T& d, T& acc)
{
    const int p = AX == 0 ? i : (AX == 1 ? j : k);
    int q;
    if (nbr_idx<AX, S>(L, p, q)) {
        const int a = AX == 0 ? q : i, b = AX == 1 ? q : j, c = AX == 2 ? q : k;
        const int cn = (a + b + c) & 1;
        const int on = (a >> 1) + L.P * (b + L.ny * c);
        const T kn = op.k[0] ? __ldg(&sel(op.k, cn)[on]) : op.kc;
        const T w = T(0.5) * (kc + kn) * (T)fcoef_ax<AX>(L, p, q);
        d += w;
        acc += w * u.at(cn, on);
    } else if (L.bc[2 * AX + (S > 0 ? 1 : 0)] == BC_DIRC) {
        d += kc * (T)dcoef_ax<AX>(L, p);
    }
}

template <class T, class U>
__device__ __forceinline__ void row_eval(const KOp<T>& op, const Lev& L, const U& u, int i, int j, int k,
                                         T& diag, T& off)
{
    const int cc = (i + j + k) & 1;
    const int o = (i >> 1) + L.P * (j + L.ny * k);
    const T kc = op.k[0] ? __ldg(&sel(op.k, cc)[o]) : op.kc;
    T d = op.dex[0] ? __ldg(&sel(op.dex, cc)[o]) : op.dexc;
    T acc = T(0);
    kface<T, 0, -1>(op, L, u, i, j, k, kc, d, acc);
    kface<T, 0, 1>(op, L, u, i, j, k, kc, d, acc);
    kface<T, 1, -1>(op, L, u, i, j, k, kc, d, acc);
    kface<T, 1, 1>(op, L, u, i, j, k, kc, d, acc);
    kface<T, 2, -1>(op, L, u, i, j, k, kc, d, acc);
    kface<T, 2, 1>(op, L, u, i, j, k, kc, d, acc);
    diag = d;
    off = -acc;
}

template <class T, int AX, int S, class U>
__device__ __forceinline__ void rface(const ROp<T>& op, const Lev& L, const U& u, int i, int j, int k, int cc,
                                      int o, T& acc)
{
    const int p = AX == 0 ? i : (AX == 1 ? j : k);
    int q;
    if (nbr_idx<AX, S>(L, p, q)) {
        const int a = AX == 0 ? q : i, b = AX == 1 ? q : j, c = AX == 2 ? q : k;
        const int cn = (a + b + c) & 1;
        const int on = (a >> 1) + L.P * (b + L.ny * c);
        acc += __ldg(&sel(op.r[1 + 2 * AX + (S > 0 ? 1 : 0)], cc)[o]) * u.at(cn, on);
    }
}

template <class T, class U>
__device__ __forceinline__ void row_eval(const ROp<T>& op, const Lev& L, const U& u, int i, int j, int k,
                                         T& diag, T& off)
{
    const int cc = (i + j + k) & 1;
    const int o = (i >> 1) + L.P * (j + L.ny * k);
    T acc = T(0);
    rface<T, 0, -1>(op, L, u, i, j, k, cc, o, acc);
    rface<T, 0, 1>(op, L, u, i, j, k, cc, o, acc);
    rface<T, 1, -1>(op, L, u, i, j, k, cc, o, acc);
    rface<T, 1, 1>(op, L, u, i, j, k, cc, o, acc);
    rface<T, 2, -1>(op, L, u, i, j, k, cc, o, acc);
    rface<T, 2, 1>(op, L, u, i, j, k, cc, o, acc);
    diag = __ldg(&sel(op.r[0], cc)[o]);
    off = acc;
}

// ---- uniform levels (every level of the reference hierarchy, and the
// finest level always): the six neighbours of an interior cell have the other
// colour at offsets o+q-1, o+q (x, q = i&1), o-+P (y), o-+P*ny (z) of the
// other half, read through one base pointer per field.  Boundary cells patch
// the offset of a missing face: a physical face keeps a valid offset with
// weight 0 and adds its Dirichlet term to the diagonal; a periodic face
// points at the wrapped cell.  When a periodic size is odd the wrapped cell
// has the same colour (a "seam"): that face is left out of the main loop and
// added in a rare fix-up from the same-colour arrays.
struct Nb6 {
    int o[6];   // offsets into the half of the neighbour's colour
    int m[6];   // 1 = face in the main (other-colour) loop
    int dirc;   // bit f: physical Dirichlet face f
    int seam;   // bit f: periodic face whose neighbour has the same colour
};

__device__ __forceinline__ void nb6(const Lev& L, int i, int j, int k, int cc, int o, Nb6& N)
{
    const int q = i & 1, sy = L.P, sz = L.P * L.ny;
    N.o[0] = o + q - 1; N.o[1] = o + q; N.o[2] = o - sy; N.o[3] = o + sy; N.o[4] = o - sz; N.o[5] = o + sz;
#pragma unroll
    for (int f = 0; f < 6; f++) N.m[f] = 1;
    N.dirc = 0;
    N.seam = 0;
    const int row = j + L.ny * k;
    if (i == 0) {
        if (L.per[0]) {
            const int a = L.nx - 1;
            N.o[0] = (a >> 1) + L.P * row;
            if (((a + j + k) & 1) == cc) { N.seam |= 1; N.m[0] = 0; }
        } else { N.m[0] = 0; N.o[0] = o; N.dirc |= (L.bc[0] == BC_DIRC) << 0; }
    }
    if (i == L.nx - 1) {
        if (L.per[0]) {
            N.o[1] = L.P * row;
            if (((j + k) & 1) == cc) { N.seam |= 2; N.m[1] = 0; }
        } else { N.m[1] = 0; N.o[1] = o; N.dirc |= (L.bc[1] == BC_DIRC) << 1; }
    }
    if (j == 0) {
        if (L.per[1]) {
            const int b = L.ny - 1;
            N.o[2] = (i >> 1) + L.P * (b + L.ny * k);
            if (((i + b + k) & 1) == cc) { N.seam |= 4; N.m[2] = 0; }
        } else { N.m[2] = 0; N.o[2] = o; N.dirc |= (L.bc[2] == BC_DIRC) << 2; }
    }
    if (j == L.ny - 1) {
        if (L.per[1]) {
            N.o[3] = (i >> 1) + L.P * (L.ny * k);
            if (((i + k) & 1) == cc) { N.seam |= 8; N.m[3] = 0; }
        } else { N.m[3] = 0; N.o[3] = o; N.dirc |= (L.bc[3] == BC_DIRC) << 3; }
    }
    if (k == 0) {
        if (L.per[2]) {
            const int c = L.nz - 1;
            N.o[4] = (i >> 1) + L.P * (j + L.ny * c);
            if (((i + j + c) & 1) == cc) { N.seam |= 16; N.m[4] = 0; }
        } else { N.m[4] = 0; N.o[4] = o; N.dirc |= (L.bc[4] == BC_DIRC) << 4; }
    }
    if (k == L.nz - 1) {
        if (L.per[2]) {
            N.o[5] = (i >> 1) + L.P * j;
            if (((i + j) & 1) == cc) { N.seam |= 32; N.m[5] = 0; }
        } else { N.m[5] = 0; N.o[5] = o; N.dirc |= (L.bc[5] == BC_DIRC) << 5; }
    }
}

template <class T, class U>
__device__ __forceinline__ void row_eval_uni(const KOp<T>& op, const Lev& L, const U& u, int i, int j, int k,
                                             T& diag, T& off)
{
    const int cc = (i + j + k) & 1, oc = cc ^ 1;
    const int o = (i >> 1) + L.P * (j + L.ny * k);
    Nb6 N;
    nb6(L, i, j, k, cc, o, N);
    const T cf[3] = {(T)L.cr[0], (T)L.cr[1], (T)L.cr[2]};
    T d = op.dex[0] ? __ldg(&sel(op.dex, cc)[o]) : op.dexc;
    const T* uo = u.ptr(oc);
    T acc = T(0);
    if (op.k[0]) {
        const T* ko = sel(op.k, oc);
        const T kc = __ldg(&sel(op.k, cc)[o]);
        T wsum = T(0);
#pragma unroll
        for (int f = 0; f < 6; f++) {
            const T kn = __ldg(&ko[N.o[f]]);
            const T w = N.m[f] ? (kc + kn) * cf[f >> 1] : T(0);
            wsum += w;
            acc += w * u.ld(uo, N.o[f]);
        }
        if (N.seam | N.dirc) {
            const T* ks = sel(op.k, cc);
            const T* us = u.ptr(cc);
#pragma unroll
            for (int f = 0; f < 6; f++) {
                if ((N.seam >> f) & 1) {
                    const T w = (kc + __ldg(&ks[N.o[f]])) * cf[f >> 1];
                    wsum += w;
                    acc += w * u.ld(us, N.o[f]);
                }
                if ((N.dirc >> f) & 1) wsum += T(4) * kc * cf[f >> 1];
            }
        }
        d += T(0.5) * wsum;
        acc *= T(0.5);
    } else {
        const T kc = op.kc;
        T wsum = T(0);
#pragma unroll
        for (int f = 0; f < 6; f++) {
            const T w = N.m[f] ? cf[f >> 1] : T(0);
            wsum += w;
            acc += w * u.ld(uo, N.o[f]);
        }
        if (N.seam | N.dirc) {
            const T* us = u.ptr(cc);
#pragma unroll
            for (int f = 0; f < 6; f++) {
                if ((N.seam >> f) & 1) {
                    wsum += cf[f >> 1];
                    acc += cf[f >> 1] * u.ld(us, N.o[f]);
                }
                if ((N.dirc >> f) & 1) wsum += T(2) * cf[f >> 1];
            }
        }
        d += kc * wsum;
        acc *= kc;
    }
    diag = d;
    off = -acc;
}

template <class T, class U>
__device__ __forceinline__ void row_eval_uni(const ROp<T>& op, const Lev& L, const U& u, int i, int j, int k,
                                             T& diag, T& off)
{
    const int cc = (i + j + k) & 1, oc = cc ^ 1;
    const int o = (i >> 1) + L.P * (j + L.ny * k);
    Nb6 N;
    nb6(L, i, j, k, cc, o, N);
    const T* uo = u.ptr(oc);
    T acc = T(0);
    // missing physical faces have zero row coefficients; seam faces read the
    // same colour
#pragma unroll
    for (int f = 0; f < 6; f++) {
        const T a = __ldg(&sel(op.r[1 + f], cc)[o]);
        acc += ((N.seam >> f) & 1) ? T(0) : a * u.ld(uo, N.o[f]);
    }
    if (N.seam) {
        const T* us = u.ptr(cc);
#pragma unroll
        for (int f = 0; f < 6; f++)
            if ((N.seam >> f) & 1) acc += __ldg(&sel(op.r[1 + f], cc)[o]) * u.ld(us, N.o[f]);
    }
    diag = __ldg(&sel(op.r[0], cc)[o]);
    off = acc;
}

// all stencil kernels evaluate rows through this entry point (the branch is
// uniform across a launch)
template <class T, class Op, class U>
__device__ __forceinline__ void row_any(const Op& op, const Lev& L, const U& u, int i, int j, int k, T& diag,
                                        T& off)
{
    if (L.uniform) row_eval_uni(op, L, u, i, j, k, diag, off);
    else row_eval(op, L, u, i, j, k, diag, off);
}

// red-black Gauss-Seidel point update u_c = (f_c - offdiag)/diag
// (perform_gseidel_smoothing, discretepde.f90:212,226)
template <class T>
__device__ __forceinline__ T gs_value(T f, T diag, T off)
{
    return (f - off) / diag;
}
// FP32 V-cycles are a preconditioner: the approximate divide (2 ulp) is used
template <>
__device__ __forceinline__ float gs_value<float>(float f, float diag, float off)
{
    return __fdividef(f - off, diag);
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
