// mps_subcycle.cuh -- the bottom of a V-cycle in one thread block.
//
// Below a few thousand cells a level's work is smaller than the cost of
// launching it: every red-black pass, transfer and the coarsest solve is a
// dependent launch of about 4 us inside the captured graphs, while one block
// of 1024 threads does a 16^3 colour pass in about 2 us and an 8^3 one in
// about 0.6 us from shared memory (clock64 phase times on a B200).  k_subcycle
// therefore runs the whole correction-scheme V-cycle from a top level of at
// most SUB_MAX_CELLS cells down to the coarsest and back in one launch of one
// block, replacing 2(nu1+nu2)+2 launches per level and the coarsest solve
// (21 launches per V-cycle below 32^3 at 257^3: 45 us against about 85 us).
// Every level's u and coefficient live in shared memory with one ghost layer
// (i fastest), f and the diagonal extra in natural order; the cell loops run
// over per-level row tables (no index division per cell) with branch-free face
// sums (per-axis neighbour offsets and face coefficients); the passes update
// in place (no cell of the levels it accepts has a neighbour of its own colour,
// so in-place is the same as the out-of-place "Jacobi within a colour" rule of
// perform_gseidel_smoothing, mgridlib/discretepde.f90:202-229); __syncthreads
// separates the phases.  What is constant over a solve (coefficients with
// their ghost values, diagonal extras, the coarsest inverse when it fits) is
// assembled once per solve into a device image (k_sub_image) that each launch
// copies with 16-byte loads.
//
// The discrete operators and transfers are the per-level kernels' own, on the
// geometric hierarchy with cell-coefficient operators (KOp): find_AX's
// arithmetic face mean k_half = (k_c + k_n)/2 times the level's face
// coefficient (discretepde.f90:646-652, Dirichlet faces 2k_c/dx^2 at :810),
// the volume-weighted mean of the children's residuals (restriction of the
// residual, mgridsteps.f90:11-53 and :531, exact widths), the trilinear
// prolongation with the coarse ghost rule (the geometric form of
// prolongation1, :170-216) and u = A^{-1} f with the precomputed dense inverse
// (in place of bottomsolve's exact GMRES, :218-382).
#pragma once

#include "mps_kernels.cuh"

namespace mps {

constexpr int SUB_MAXL = 8;               // levels of one launch, the coarsest included
constexpr int SUB_TPB = 1024;             // threads of the block
constexpr int SUB_MAX_CELLS = 8192;       // cells of the top level at most
constexpr int SUB_SMEM_MAX = 200 * 1024;  // shared-memory bytes at most
constexpr int SUB_MAX_AX = 160;           // axis entries of all levels (sum of nx+ny+nz)
constexpr int SUB_MAX_ROWS = 2048;        // rows of all levels (sum of ny*nz)

// one prolongation bracket (geom_lin) in the block's working type
template <class T>
struct SubLin {
    int j0, j1;
    T t;
};

// one cell position p along one axis of a level: the offsets of its two
// neighbours in the ghosted layout and the coefficients of its two faces.
// In-grid faces carry Lev's face coefficient (cr, or cl / cp next to a merged
// last cell), periodic faces wrap (the offset reaches the opposite cell),
// physical faces point at the ghost cell and carry the Dirichlet coefficient
// dr / dlast, or 0 (zero-gradient and flux faces add nothing).
template <class T>
struct SubAx {
    int om, op;  // neighbour offsets (elements of the ghosted layout)
    T cm, cp;    // face coefficients
};

// one row (j, k) of a level: its first cell's ghosted and natural indices
struct SubRow {
    int j, k, g0, n0;
};

// one level as the block's loops read it
template <class T>
struct SubGeo {
    int nx, ny, nz, nh;
    int rows;              // ny*nz
    int gx, gy;            // ghosted row and plane sizes: nx+2 (or a padded pitch), ny+2
    int pitch;             // row pitch of the level's split layout (Lev::P)
    int per;               // bit a: periodic axis a
    int dirc;              // bit f: Dirichlet face f (LEFT..FRONT)
    int ax0;               // first axis entry of the level (x, then y at +nx, z at +nx+ny)
    int row0;              // first row entry of the level
    int rc, rn;            // rows per trip of the colour loops (threads / nh) and of the cell loops (threads / nx)
    FastDiv dnh, dny, dnx; // by (nx+1)/2, ny, nx
    T w[3], wl[3];         // regular and last cell widths
};

template <class T>
struct SubPlan {
    int nl;                   // levels; geo[nl-1] is the coarsest
    int nu1, nu2;             // pre/post red-black sweeps
    int only_black;           // the prolongation corrects the black cells only (nu2 >= 1)
    int gsz;                  // lanes per row of the coarsest solve (power of two, <= 32)
    int nlin, nax, nrow;      // prolongation brackets / axis entries / rows
    int lin_off, ax_off, row_off;  // their byte offsets in shared memory
    int img_off, img_bytes;   // the solve-constant part of shared memory (coefficients, diagonal extras,
                              // coarsest inverse), copied from an image built once per solve (k_sub_image)
    int ainv_off;             // byte offset of the coarsest inverse (column major, FP64); -1: read from device memory
    T kc, dexc;               // uniform coefficient / diagonal extra (when no field)
    int rlog[SUB_MAXL];       // log2 of the lanes per coarse cell of the restriction geo[s] -> geo[s+1]
    int rrows[SUB_MAXL];      // coarse rows per trip of that restriction: (threads >> rlog) / coarse nx
    int ou[SUB_MAXL], ok[SUB_MAXL];  // ghosted fields (elements of T), ok -1: uniform coefficient
    int of[SUB_MAXL], od[SUB_MAXL];  // natural-order fields, od -1: uniform diagonal extra
    int lin0[SUB_MAXL][3];    // first bracket of level s along axis a
    const T* k[SUB_MAXL][2];              // cell coefficient (split halves) or null (image build)
    const T* dex[SUB_MAXL][2];            // diagonal extra -reac + 1/dt (split halves) or null (image build)
    SubGeo<T> geo[SUB_MAXL];
    SubAx<T> ax[SUB_MAX_AX];  // axis entries of every level
    SubLin<T> lin[SUB_MAX_AX];  // prolongation brackets of every transfer (by fine index)
};

// shared-memory views of one launch
template <class T>
struct SubMem {
    T* fld;
    const SubLin<T>* lin;
    const SubAx<T>* ax;
    const SubRow* row;
};

// the face sums of row (i,j,k): ds = sum of (k_c + k_n) * coef over the six
// faces, as = sum of (k_c + k_n) * coef * u_n (twice the face weights of
// find_AX's arithmetic mean; ghost cells of physical faces hold u = 0 and
// k = k_c, so a Dirichlet face adds 2 k_c dcoef to ds and zero-gradient faces
// nothing).  A u = (dex + ds/2) u - as/2.
template <class T, bool KF>
__device__ __forceinline__ void sub_faces(const SubAx<T>* __restrict__ axt, int ax0, int nx, int ny,
                                          const T* __restrict__ u, const T* __restrict__ kg, T kc, int i, int j,
                                          int k, int g, T& ds, T& as)
{
    const SubAx<T> X = axt[ax0 + i], Y = axt[ax0 + nx + j], Z = axt[ax0 + nx + ny + k];
    if (KF) {
        const T wa = (kc + kg[g + X.om]) * X.cm, wb = (kc + kg[g + X.op]) * X.cp;
        const T wc = (kc + kg[g + Y.om]) * Y.cm, wd = (kc + kg[g + Y.op]) * Y.cp;
        const T we = (kc + kg[g + Z.om]) * Z.cm, wf = (kc + kg[g + Z.op]) * Z.cp;
        ds = ((wa + wb) + (wc + wd)) + (we + wf);
        as = ((wa * u[g + X.om] + wb * u[g + X.op]) + (wc * u[g + Y.om] + wd * u[g + Y.op])) +
             (we * u[g + Z.om] + wf * u[g + Z.op]);
    } else {
        const T k2 = kc + kc;
        ds = k2 * (((X.cm + X.cp) + (Y.cm + Y.cp)) + (Z.cm + Z.cp));
        as = k2 * (((X.cm * u[g + X.om] + X.cp * u[g + X.op]) + (Y.cm * u[g + Y.om] + Y.cp * u[g + Y.op])) +
                   (Z.cm * u[g + Z.om] + Z.cp * u[g + Z.op]));
    }
}

template <class T>
__device__ __forceinline__ int sub_gidx(const SubGeo<T>& G, int i, int j, int k)
{
    return (i + 1) + G.gx * ((j + 1) + G.gy * (k + 1));
}

// one red-black colour pass of level s, in place.  Thread t takes the cells
// h = t mod nh of the rows t / nh, t / nh + rc, ...
template <class T, bool KF, bool DF>
__device__ __forceinline__ void sub_colour(const SubPlan<T>& P, const SubMem<T>& M, int s, int c)
{
    const SubGeo<T>& G = P.geo[s];
    const int nx = G.nx, ny = G.ny, nh = G.nh, rows = G.rows, rc = G.rc, ax0 = G.ax0;
    T* u = M.fld + P.ou[s];
    const T* kg = KF ? M.fld + P.ok[s] : nullptr;
    const T* f = M.fld + P.of[s];
    const T* df = DF ? M.fld + P.od[s] : nullptr;
    const SubRow* rt = M.row + G.row0;
    const T kc0 = P.kc, dexc = P.dexc;
    const int r0 = (int)G.dnh.div(threadIdx.x);
    const int h = (int)threadIdx.x - r0 * nh;
    if (r0 < rc) {
        for (int r = r0; r < rows; r += rc) {
            const SubRow R = rt[r];
            const int i = 2 * h + ((R.j + R.k + c) & 1);
            if (i >= nx) continue;
            const int g = R.g0 + i, idx = R.n0 + i;
            const T kc = KF ? kg[g] : kc0;
            T ds, as;
            sub_faces<T, KF>(M.ax, ax0, nx, ny, u, kg, kc, i, R.j, R.k, g, ds, as);
            const T d = (DF ? df[idx] : dexc) + T(0.5) * ds;
            u[g] = gs_value<T>(f[idx], d, T(-0.5) * as);
        }
    }
    __syncthreads();
}

// f_{s+1} = R(f_s - A_s u_s), u_{s+1} = 0: 2^rlog lanes per coarse cell, each
// a share of the children; the volume-weighted mean over the children (the
// geometric hierarchy's restriction, resid_restrict_part).  After a black
// pass the black residuals vanish up to rounding (each black cell has just
// solved its own row against its red neighbours), so only red children are
// evaluated when there is pre-smoothing; every child counts in the volume.
template <class T, bool KF, bool DF>
__device__ __forceinline__ void sub_restrict(const SubPlan<T>& P, const SubMem<T>& M, int s)
{
    const SubGeo<T>& F = P.geo[s];
    const SubGeo<T>& C = P.geo[s + 1];
    const int fnx = F.nx, fny = F.ny, fnz = F.nz, ax0 = F.ax0;
    const T* u = M.fld + P.ou[s];
    const T* kg = KF ? M.fld + P.ok[s] : nullptr;
    const T* f = M.fld + P.of[s];
    const T* df = DF ? M.fld + P.od[s] : nullptr;
    T* fc = M.fld + P.of[s + 1];
    T* uc = M.fld + P.ou[s + 1];
    const SubRow* ft = M.row + F.row0;
    const SubRow* ct = M.row + C.row0;
    const T kc0 = P.kc, dexc = P.dexc;
    const bool red_only = P.nu1 >= 1;
    const int lg = P.rlog[s], G = 1 << lg, rr = P.rrows[s];
    const int part = (int)threadIdx.x & (G - 1);
    const int slot = (int)threadIdx.x >> lg;
    const int r0 = (int)C.dnx.div((unsigned)slot);
    const int I = slot - r0 * C.nx;
    const bool on = r0 < rr;
    const int trips = (C.rows + rr - 1) / rr;
    const int cnx = C.nx, cny = C.ny, cnz = C.nz;
    for (int tr = 0; tr < trips; tr++) {  // the same trips for every lane (shuffles below)
        const int r = r0 + tr * rr;
        const bool valid = on && r < C.rows;
        T sum = T(0), vol = T(0);
        SubRow CR{0, 0, 0, 0};
        if (valid) {
            CR = ct[r];
            const int J = CR.j, K = CR.k;
            const int lo0 = fnx == cnx ? I : 2 * I, n0 = fnx == cnx ? 1 : (I == cnx - 1 ? fnx - 2 * (cnx - 1) : 2);
            const int lo1 = fny == cny ? J : 2 * J, n1 = fny == cny ? 1 : (J == cny - 1 ? fny - 2 * (cny - 1) : 2);
            const int lo2 = fnz == cnz ? K : 2 * K, n2 = fnz == cnz ? 1 : (K == cnz - 1 ? fnz - 2 * (cnz - 1) : 2);
            int ch = 0;
            for (int dk = 0; dk < n2; dk++)
                for (int dj = 0; dj < n1; dj++) {
                    const int j = lo1 + dj, k = lo2 + dk;
                    const SubRow FR = ft[j + fny * k];
                    const T vyz = (j == fny - 1 ? F.wl[1] : F.w[1]) * (k == fnz - 1 ? F.wl[2] : F.w[2]);
                    for (int di = 0; di < n0; di++, ch++) {
                        if ((ch & (G - 1)) != part) continue;
                        const int i = lo0 + di;
                        const T v = (i == fnx - 1 ? F.wl[0] : F.w[0]) * vyz;
                        vol += v;
                        if (red_only && ((i + j + k) & 1)) continue;
                        const int g = FR.g0 + i, idx = FR.n0 + i;
                        const T kc = KF ? kg[g] : kc0;
                        T ds, as;
                        sub_faces<T, KF>(M.ax, ax0, fnx, fny, u, kg, kc, i, j, k, g, ds, as);
                        const T d = (DF ? df[idx] : dexc) + T(0.5) * ds;
                        const T rv = f[idx] - (d * u[g] - T(0.5) * as);
                        sum += v * rv;
                    }
                }
        }
        for (int o = G >> 1; o > 0; o >>= 1) {
            sum += __shfl_xor_sync(0xffffffffu, sum, o);
            vol += __shfl_xor_sync(0xffffffffu, vol, o);
        }
        if (valid && part == 0) {
            fc[CR.n0 + I] = sum / vol;
            uc[CR.g0 + I] = T(0);
        }
    }
    __syncthreads();
}

// coarse value at (x,y,z), any index possibly a ghost (-1 or n): periodic
// axes wrap, Dirichlet faces mirror with a sign flip, other faces copy (the
// ghost rule of coarse_at)
template <class T>
__device__ __forceinline__ T sub_coarse(const SubGeo<T>& C, const T* e, int x, int y, int z)
{
    int q[3] = {x, y, z};
    const int n[3] = {C.nx, C.ny, C.nz};
    T sgn = T(1);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (q[a] >= 0 && q[a] < n[a]) continue;
        const int side = q[a] < 0 ? 0 : 1;
        if ((C.per >> a) & 1) q[a] = q[a] < 0 ? n[a] - 1 : 0;
        else {
            if ((C.dirc >> (2 * a + side)) & 1) sgn = -sgn;
            q[a] = q[a] < 0 ? 0 : n[a] - 1;
        }
    }
    return sgn * e[sub_gidx(C, q[0], q[1], q[2])];
}

// u_s += P u_{s+1} at one fine cell: tensor-product linear interpolation
// between the bracketing coarse centres (the transfer's staged brackets)
template <class T>
__device__ __forceinline__ void sub_prolong_cell(const SubPlan<T>& P, const SubMem<T>& M, int s, T* u,
                                                 const T* e, int i, int j, int k, int g)
{
    const SubGeo<T>& C = P.geo[s + 1];
    const SubLin<T> lx = M.lin[P.lin0[s][0] + i], ly = M.lin[P.lin0[s][1] + j], lz = M.lin[P.lin0[s][2] + k];
    T c000, c100, c010, c110, c001, c101, c011, c111;
    if (lx.j0 >= 0 && lx.j1 < C.nx && ly.j0 >= 0 && ly.j1 < C.ny && lz.j0 >= 0 && lz.j1 < C.nz) {
        const int b00 = sub_gidx(C, 0, ly.j0, lz.j0), b10 = sub_gidx(C, 0, ly.j1, lz.j0);
        const int b01 = sub_gidx(C, 0, ly.j0, lz.j1), b11 = sub_gidx(C, 0, ly.j1, lz.j1);
        c000 = e[b00 + lx.j0]; c100 = e[b00 + lx.j1];
        c010 = e[b10 + lx.j0]; c110 = e[b10 + lx.j1];
        c001 = e[b01 + lx.j0]; c101 = e[b01 + lx.j1];
        c011 = e[b11 + lx.j0]; c111 = e[b11 + lx.j1];
    } else {
        c000 = sub_coarse(C, e, lx.j0, ly.j0, lz.j0); c100 = sub_coarse(C, e, lx.j1, ly.j0, lz.j0);
        c010 = sub_coarse(C, e, lx.j0, ly.j1, lz.j0); c110 = sub_coarse(C, e, lx.j1, ly.j1, lz.j0);
        c001 = sub_coarse(C, e, lx.j0, ly.j0, lz.j1); c101 = sub_coarse(C, e, lx.j1, ly.j0, lz.j1);
        c011 = sub_coarse(C, e, lx.j0, ly.j1, lz.j1); c111 = sub_coarse(C, e, lx.j1, ly.j1, lz.j1);
    }
    const T tx = lx.t, ty = ly.t, tz = lz.t;
    const T x00 = c000 + tx * (c100 - c000), x10 = c010 + tx * (c110 - c010);
    const T x01 = c001 + tx * (c101 - c001), x11 = c011 + tx * (c111 - c011);
    const T y0 = x00 + ty * (x10 - x00), y1 = x01 + ty * (x11 - x01);
    u[g] += y0 + tz * (y1 - y0);
}

template <class T>
__device__ __forceinline__ void sub_prolong(const SubPlan<T>& P, const SubMem<T>& M, int s)
{
    const SubGeo<T>& G = P.geo[s];
    const int nx = G.nx, rows = G.rows;
    T* u = M.fld + P.ou[s];
    const T* e = M.fld + P.ou[s + 1];
    const SubRow* rt = M.row + G.row0;
    if (P.only_black) {  // the first post-smoothing pass rewrites the red cells
        const int r0 = (int)G.dnh.div(threadIdx.x);
        const int h = (int)threadIdx.x - r0 * G.nh;
        if (r0 < G.rc)
            for (int r = r0; r < rows; r += G.rc) {
                const SubRow R = rt[r];
                const int i = 2 * h + ((R.j + R.k + 1) & 1);
                if (i >= nx) continue;
                sub_prolong_cell(P, M, s, u, e, i, R.j, R.k, R.g0 + i);
            }
    } else {
        const int r0 = (int)G.dnx.div(threadIdx.x);
        const int i = (int)threadIdx.x - r0 * nx;
        if (r0 < G.rn)
            for (int r = r0; r < rows; r += G.rn) {
                const SubRow R = rt[r];
                sub_prolong_cell(P, M, s, u, e, i, R.j, R.k, R.g0 + i);
            }
    }
    __syncthreads();
}

// u = A^{-1} f on the coarsest level (FP64 sums, as coarse_solve_body); gsz
// lanes per row, shuffle-summed; the inverse is staged in shared memory
template <class T>
__device__ __forceinline__ void sub_coarse_solve(const SubPlan<T>& P, const SubMem<T>& M, const double* ainv)
{
    const int s = P.nl - 1;
    const SubGeo<T>& C = P.geo[s];
    const int n = C.nx * C.rows;
    const T* f = M.fld + P.of[s];
    T* u = M.fld + P.ou[s];
    const SubRow* rt = M.row + C.row0;
    const int G = P.gsz;
    const int per_trip = SUB_TPB / G;
    for (int q0 = 0; q0 < n; q0 += per_trip) {
        const int r = q0 + (int)threadIdx.x / G, part = (int)threadIdx.x % G;
        double acc = 0.0;
        if (r < n)
            for (int q = part; q < n; q += G) acc += ainv[q * n + r] * (double)f[q];
        for (int o = G >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (r < n && part == 0) {
            const int row = (int)C.dnx.div((unsigned)r);
            u[rt[row].g0 + (r - row * C.nx)] = (T)acc;
        }
    }
    __syncthreads();
}

// the solve-constant image (k_subcycle copies it to shared memory at
// P.img_off): every level's coefficient in the ghosted layout (ghost cells of
// physical faces hold the adjacent cell's value), every level's diagonal
// extra in natural order, the coarsest inverse.  Built once per solve.
template <class T, bool KF, bool DF>
__global__ void __launch_bounds__(SUB_TPB) k_sub_image(const __grid_constant__ SubPlan<T> P,
                                                       unsigned char* __restrict__ img,
                                                       const double* __restrict__ AinvT, int ncoarse)
{
    pdl_wait();
    T* base = reinterpret_cast<T*>(img - P.img_off);  // element offsets of the shared-memory layout
    for (int s = 0; s < P.nl; s++) {
        const SubGeo<T>& G = P.geo[s];
        const int n = G.nx * G.rows;
        for (int t = threadIdx.x; t < n; t += SUB_TPB) {
            const int r = (int)G.dnx.div((unsigned)t), i = t - r * G.nx;
            const int k = (int)G.dny.div((unsigned)r), j = r - k * G.ny;
            const int c = (i + j + k) & 1;
            const int o = (i >> 1) + G.pitch * r;
            if (KF) {
                const T v = sel(P.k[s], c)[o];
                const int g = sub_gidx(G, i, j, k);
                T* kg = base + P.ok[s];
                kg[g] = v;
                // physical-face ghosts (periodic ones are never read)
                if (i == 0) kg[g - 1] = v;
                if (i == G.nx - 1) kg[g + 1] = v;
                if (j == 0) kg[g - G.gx] = v;
                if (j == G.ny - 1) kg[g + G.gx] = v;
                if (k == 0) kg[g - G.gx * G.gy] = v;
                if (k == G.nz - 1) kg[g + G.gx * G.gy] = v;
            }
            if (DF) base[P.od[s] + t] = sel(P.dex[s], c)[o];
        }
    }
    if (P.ainv_off >= 0) {
        double* ai = reinterpret_cast<double*>(img + (P.ainv_off - P.img_off));
        for (int e = threadIdx.x; e < ncoarse * ncoarse; e += SUB_TPB) ai[e] = AinvT[e];
    }
    SubLin<T>* lin = reinterpret_cast<SubLin<T>*>(img + (P.lin_off - P.img_off));
    SubAx<T>* axt = reinterpret_cast<SubAx<T>*>(img + (P.ax_off - P.img_off));
    SubRow* rowt = reinterpret_cast<SubRow*>(img + (P.row_off - P.img_off));
    for (int e = threadIdx.x; e < P.nlin; e += SUB_TPB) lin[e] = P.lin[e];
    for (int e = threadIdx.x; e < P.nax; e += SUB_TPB) axt[e] = P.ax[e];
    for (int s = 0; s < P.nl; s++) {
        const SubGeo<T>& G = P.geo[s];
        for (int r = threadIdx.x; r < G.rows; r += SUB_TPB) {
            const int k = (int)G.dny.div((unsigned)r), j = r - k * G.ny;
            SubRow R;
            R.j = j;
            R.k = k;
            R.g0 = sub_gidx(G, 0, j, k);
            R.n0 = G.nx * r;
            rowt[G.row0 + r] = R;
        }
    }
}

// the V-cycle from geo[0] (zero initial guess, right-hand side fin) down to
// the coarsest and back; the result is written to uout (split layout)
template <class T, bool KF, bool DF>
__global__ void __launch_bounds__(SUB_TPB, 1) k_subcycle(const __grid_constant__ SubPlan<T> P, CSplit<T> fin,
                                                          Split<T> uout, const uint4* __restrict__ img,
                                                          const double* __restrict__ AinvT)
{
    pdl_wait();
    extern __shared__ __align__(16) unsigned char sub_smem[];
    SubMem<T> M;
    M.fld = reinterpret_cast<T*>(sub_smem);
    SubLin<T>* lin = reinterpret_cast<SubLin<T>*>(sub_smem + P.lin_off);
    SubAx<T>* axt = reinterpret_cast<SubAx<T>*>(sub_smem + P.ax_off);
    SubRow* rowt = reinterpret_cast<SubRow*>(sub_smem + P.row_off);
    M.lin = lin;
    M.ax = axt;
    M.row = rowt;
    // the solve-constant image (coefficients, diagonal extras, inverse, row
    // and axis tables, brackets) and the top level's right-hand side from
    // device memory (loads issued in batches before their stores), zero u
    // (ghosts included)
    {
        uint4* dst = reinterpret_cast<uint4*>(sub_smem + P.img_off);
        const int nv = P.img_bytes >> 4;
        constexpr int B = 4;
        for (int e0 = 0; e0 < nv; e0 += B * SUB_TPB) {
            uint4 v[B];
#pragma unroll
            for (int b = 0; b < B; b++) {
                const int e = e0 + b * SUB_TPB + (int)threadIdx.x;
                if (e < nv) v[b] = __ldg(&img[e]);
            }
#pragma unroll
            for (int b = 0; b < B; b++) {
                const int e = e0 + b * SUB_TPB + (int)threadIdx.x;
                if (e < nv) dst[e] = v[b];
            }
        }
    }
    for (int s = 0; s < P.nl; s++) {
        const SubGeo<T>& G = P.geo[s];
        const int ng = G.gx * G.gy * (G.nz + 2);
        T* u = M.fld + P.ou[s];
        for (int e = threadIdx.x; e < ng; e += SUB_TPB) u[e] = T(0);
    }
    {
        const SubGeo<T>& G = P.geo[0];
        T* f = M.fld + P.of[0];
        const int n = G.nx * G.rows;
        constexpr int B = 8;
        for (int t0 = 0; t0 < n; t0 += B * SUB_TPB) {
            T v[B];
#pragma unroll
            for (int b = 0; b < B; b++) {
                const int t = t0 + b * SUB_TPB + (int)threadIdx.x;
                if (t < n) {
                    const int r = (int)G.dnx.div((unsigned)t), i = t - r * G.nx;
                    const int k = (int)G.dny.div((unsigned)r), j = r - k * G.ny;
                    v[b] = fin.at((i + j + k) & 1, (i >> 1) + G.pitch * r);
                }
            }
#pragma unroll
            for (int b = 0; b < B; b++) {
                const int t = t0 + b * SUB_TPB + (int)threadIdx.x;
                if (t < n) f[t] = v[b];
            }
        }
    }
    __syncthreads();
    for (int s = 0; s < P.nl - 1; s++) {
        for (int sw = 0; sw < P.nu1; sw++) {
            sub_colour<T, KF, DF>(P, M, s, 0);
            sub_colour<T, KF, DF>(P, M, s, 1);
        }
        sub_restrict<T, KF, DF>(P, M, s);
    }
    sub_coarse_solve<T>(P, M, P.ainv_off >= 0 ? reinterpret_cast<const double*>(sub_smem + P.ainv_off) : AinvT);
    for (int s = P.nl - 2; s >= 0; s--) {
        sub_prolong<T>(P, M, s);
        for (int sw = 0; sw < P.nu2; sw++) {
            sub_colour<T, KF, DF>(P, M, s, 0);
            sub_colour<T, KF, DF>(P, M, s, 1);
        }
    }
    {
        const SubGeo<T>& G = P.geo[0];
        const T* u = M.fld + P.ou[0];
        const int r0 = (int)G.dnx.div(threadIdx.x);
        const int i = (int)threadIdx.x - r0 * G.nx;
        if (r0 < G.rn) {
#pragma unroll 4
            for (int r = r0; r < G.rows; r += G.rn) {
                const SubRow R = rowt[G.row0 + r];
                uout.half((i + R.j + R.k) & 1)[(i >> 1) + G.pitch * r] = u[R.g0 + i];
            }
        }
    }
}

}  // namespace mps
