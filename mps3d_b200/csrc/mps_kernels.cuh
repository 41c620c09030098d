// mps_kernels.cuh -- CUDA kernels of the B200 multigrid / Krylov solver.
// All kernels are memory-bound 7-point stencils, transfers or reductions
// (arithmetic intensity well below the FP64 ridge); none uses tensor cores.
#pragma once

#include "mps_core.cuh"

namespace mps {

constexpr int TPB = 256;

// Programmatic dependent launch: a kernel launched with the programmatic
// stream-serialization attribute may be scheduled while its predecessor is
// still running; this wait (first statement of every kernel) blocks until
// the predecessor grid has completed and its writes are visible.  For an
// ordinary launch it returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

struct RedBuf {
    double* partial;      // [2 * maxblocks]
    unsigned* counter;    // zero-initialised
    double* out;          // [2]: sum r^2, sum f^2
};

__device__ __forceinline__ double block_sum(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    __syncthreads();
    return s;  // valid in thread 0
}

template <class T>
struct ZeroU {  // accessor of a field known to be zero
    __device__ __forceinline__ T get(const Lev&, int, int, int) const { return T(0); }
    __device__ __forceinline__ T at(int, int) const { return T(0); }
    __device__ __forceinline__ const T* ptr(int) const { return nullptr; }
    __device__ __forceinline__ T ld(const T*, int) const { return T(0); }
};
template <class T>
struct OtherOnlyU {  // colour c known zero, the other colour read from memory
    const T* other;  // half 1-c
    int c;
    __device__ __forceinline__ T get(const Lev& L, int i, int j, int k) const
    {
        return scol(i, j, k) == c ? T(0) : __ldg(&other[soff(L, i, j, k)]);
    }
    __device__ __forceinline__ T at(int col, int off) const { return col == c ? T(0) : __ldg(&other[off]); }
    __device__ __forceinline__ const T* ptr(int col) const { return col == c ? nullptr : other; }
    __device__ __forceinline__ T ld(const T* p, int off) const { return p ? __ldg(&p[off]) : T(0); }
};

// ---------------------------------------------------------------------
// one colour pass of red-black Gauss-Seidel, out of place:
//   out[c] = (f[c] - offdiag(u)) / diag, u = state at the start of the pass
// (perform_gseidel_smoothing, discretepde.f90:202-229; the reference
// computes offdiag of all cells before updating a colour, so cells of one
// colour never see each other's new values -- the same rule holds here at
// periodic seams of odd size where equal colours touch)
// ---------------------------------------------------------------------
template <class T, class Op, class U>
__device__ __forceinline__ void colour_body(const Lev& L, const Op& op, int c, const U& u, T* __restrict__ out,
                                            const T* __restrict__ f, unsigned t)
{
    int i, j, k;
    if (!decode(L, t, c, i, j, k)) return;
    T diag, off;
    row_any<T>(op, L, u, i, j, k, diag, off);
    out[t] = gs_value(__ldg(&f[t]), diag, off);
}

template <class T, class Op, class U>
__global__ void __launch_bounds__(TPB) k_colour(Lev L, Op op, int c, U u, T* __restrict__ out,
                                                const T* __restrict__ f)
{
    pdl_wait();
    colour_body<T, Op, U>(L, op, c, u, out, f, blockIdx.x * TPB + threadIdx.x);
}

// ---------------------------------------------------------------------
// colour pass on a uniform level, four consecutive cells of one colour per
// thread (16-byte vector loads).  Row (j,k), group g: split offsets
// o0..o0+3 with o0 = 4g + P*(j+ny*k); i = 2(4g+e)+q, q = (j+k+c)&1.  The x
// neighbours of the group are the other colour at o0+q-1 .. o0+q+3 (one
// vector plus one scalar), the y/z neighbours one vector each.  Elements past
// the end of the row (pads) are written as 0.  Same semantics as k_colour.
// ---------------------------------------------------------------------
template <class T, int W>
struct VecW {
    T v[W];
};
// 256-bit global accesses (sm_100): one instruction for 8 floats or 4
// doubles; the address must be 32-byte aligned (groups start at multiples of
// W elements of rows whose pitch P is a multiple of 8)
template <class T, int W>
__device__ __forceinline__ VecW<T, W> ldv(const T* p)
{
    VecW<T, W> r;
    if constexpr (sizeof(T) * W == 32) {
        if constexpr (sizeof(T) == 4) {
            asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]), "=f"(r.v[5]),
                  "=f"(r.v[6]), "=f"(r.v[7])
                : "l"(p));
        } else {
            asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
                : "=d"(r.v[0]), "=d"(r.v[1]), "=d"(r.v[2]), "=d"(r.v[3])
                : "l"(p));
        }
    } else if constexpr (sizeof(T) * W == 16) {
        if constexpr (sizeof(T) == 4) {
            const float4 a = __ldg(reinterpret_cast<const float4*>(p));
            r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
        } else {
            const double2 a = __ldg(reinterpret_cast<const double2*>(p));
            r.v[0] = a.x; r.v[1] = a.y;
        }
    } else if constexpr (sizeof(T) * W == 8 && sizeof(T) == 4) {
        const float2 a = __ldg(reinterpret_cast<const float2*>(p));
        r.v[0] = a.x; r.v[1] = a.y;
    } else {
        static_assert(W == 1, "vector width: 1, 2, 4 or 8 floats; 1, 2 or 4 doubles");
        r.v[0] = __ldg(p);
    }
    return r;
}
template <class T, int W>
__device__ __forceinline__ void stv(T* p, const VecW<T, W>& r)
{
    if constexpr (sizeof(T) * W == 32) {
        if constexpr (sizeof(T) == 4) {
            asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(r.v[0]), "f"(r.v[1]),
                         "f"(r.v[2]), "f"(r.v[3]), "f"(r.v[4]), "f"(r.v[5]), "f"(r.v[6]), "f"(r.v[7])
                         : "memory");
        } else {
            asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(r.v[0]), "d"(r.v[1]), "d"(r.v[2]),
                         "d"(r.v[3])
                         : "memory");
        }
    } else if constexpr (sizeof(T) * W == 16) {
        if constexpr (sizeof(T) == 4) *reinterpret_cast<float4*>(p) = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
        else *reinterpret_cast<double2*>(p) = make_double2(r.v[0], r.v[1]);
    } else if constexpr (sizeof(T) * W == 8 && sizeof(T) == 4) {
        *reinterpret_cast<float2*>(p) = make_float2(r.v[0], r.v[1]);
    } else {
        static_assert(W == 1, "vector width: 1, 2, 4 or 8 floats; 1, 2 or 4 doubles");
        p[0] = r.v[0];
    }
}
template <class T, int W>
__device__ __forceinline__ VecW<T, W> zerov()
{
    VecW<T, W> r;
#pragma unroll
    for (int e = 0; e < W; e++) r.v[e] = T(0);
    return r;
}

// the row neighbour along y or z of a group (AX = 1 or 2, S = -1/+1): vectors
// of u and k values and the face status (wrapped row for periodic faces,
// same-colour arrays across an odd periodic seam)
template <class T, int W, int AX, int S, bool IN = false>
__device__ __forceinline__ void yz_face(const Lev& L, int j, int k, int h0, int cc, const T* uo, const T* us,
                                        const T* ko, const T* ks, bool kfield, VecW<T, W>& u4, VecW<T, W>& k4,
                                        int& mask, int& dirc)
{
    const int n = AX == 1 ? L.ny : L.nz;
    const int p = AX == 1 ? j : k;
    int pq = p + S;
    mask = 1;
    dirc = 0;
    const T* ub = uo;
    const T* kb = ko;
    if (!IN && (pq < 0 || pq >= n)) {  // IN: rows known to be inside the grid
        if (!L.per[AX]) {  // physical face: no neighbour
            mask = 0;
            dirc = L.bc[2 * AX + (S > 0 ? 1 : 0)] == BC_DIRC;
            u4 = zerov<T, W>();
            k4 = zerov<T, W>();
            return;
        }
        pq = pq < 0 ? n - 1 : 0;
        const int jj = AX == 1 ? pq : j, kk = AX == 2 ? pq : k;
        const int ncol = ((2 * h0 + ((j + k + cc) & 1)) + jj + kk) & 1;
        if (ncol == cc) { ub = us; kb = ks; }
    }
    const int jj = AX == 1 ? pq : j, kk = AX == 2 ? pq : k;
    const int off = h0 + L.P * (jj + L.ny * kk);
    u4 = ub ? ldv<T, W>(ub + off) : zerov<T, W>();
    k4 = kfield ? ldv<T, W>(kb + off) : zerov<T, W>();
}

// Row evaluation of W consecutive cells of one colour (vector loads).  Row
// (j,k), group g: split offsets o0..o0+W-1 with o0 = W g + P (j + ny k);
// i = 2(W g + e) + q, q = (j+k+c)&1.  The x neighbours of the group are the
// other colour at o0+q-1 .. o0+q+W-1 (one vector plus one scalar), the y/z
// neighbours one vector each.  Returns diag and offdiag (sum_n a_n u_n) per
// element; elements with i >= nx are padding.  UNI: every face has the
// regular coefficient (a uniform level); otherwise the faces touching the
// last cell of an axis (a merged odd cell of the geometric hierarchy) take
// their own coefficients, as in row_eval (fcoef_ax / dcoef_ax).
template <int AX, bool UNI>
__device__ __forceinline__ double face_c(const Lev& L, int p, int q)
{
    if (UNI) return L.cr[AX];
    return fcoef_ax<AX>(L, p, q);
}
template <int AX, bool UNI>
__device__ __forceinline__ double dir_c(const Lev& L, int p)
{
    if (UNI) return L.dr[AX];
    return dcoef_ax<AX>(L, p);
}

// The x faces and the diagonal of W cells of one row, given the y/z face
// sums (acc = sum w u_n, wsum = sum w, byz = Dirichlet y/z boundary weight)
// and the other colour's vectors at the row's own offsets (ax: u, akx: k).
// IN: every cell of the group has all six neighbours inside the grid (no
// boundary code is generated)
template <class T, int W, class U, bool UNI, bool IN = false>
__device__ __forceinline__ void row_finish(const Lev& L, const KOp<T>& op, int c, const U& u, int row, int j, int k,
                                           int h0, int q, int o0, const VecW<T, W>& kc4, const VecW<T, W>& acc,
                                           const VecW<T, W>& wsum, T byz, const VecW<T, W>& ax,
                                           const VecW<T, W>& akx, VecW<T, W>& diag, VecW<T, W>& off)
{
    const int cc = c, oc = c ^ 1;
    const bool kfield = op.k[0] != nullptr;
    const T* uo = u.ptr(oc);
    const T* us = u.ptr(cc);
    const T* ko = kfield ? sel(op.k, oc) : nullptr;
    const T* ks = kfield ? sel(op.k, cc) : nullptr;
    // x neighbours: A = other colour at o0..o0+W-1, S = o0+W (q=1) or o0-1 (q=0)
    const int so = q ? o0 + W : o0 - 1;
    const bool sok = IN || (q ? (h0 + W < L.P) : (h0 > 0));
    T sx = T(0), skx = T(0);
    if (sok) {
        sx = u.ld(uo, so);
        skx = kfield ? __ldg(ko + so) : T(0);
    }
    const int nx1 = L.nx - 1;
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = 2 * (h0 + e) + q;
        T uxm, kxm, uxp, kxp;
        if (q) {
            uxm = ax.v[e]; kxm = akx.v[e];
            uxp = e < W - 1 ? ax.v[e + 1] : sx; kxp = e < W - 1 ? akx.v[e + 1] : skx;
        } else {
            uxm = e > 0 ? ax.v[e - 1] : sx; kxm = e > 0 ? akx.v[e - 1] : skx;
            uxp = ax.v[e]; kxp = akx.v[e];
        }
        T mxm = T(1), mxp = T(1);
        T bx = T(0);
        if (!IN && i == 0) {  // x- boundary / periodic wrap
            if (L.per[0]) {
                const int a = nx1;
                const int wo = (a >> 1) + L.P * row;
                const bool same = ((a + j + k) & 1) == cc;
                uxm = u.ld(same ? us : uo, wo);
                kxm = kfield ? __ldg((same ? ks : ko) + wo) : T(0);
            } else {
                mxm = T(0);
                if (L.bc[0] == BC_DIRC) bx += (T)dir_c<0, UNI>(L, i);
            }
        }
        if (!IN && i == nx1) {  // x+ boundary / periodic wrap
            if (L.per[0]) {
                const int wo = L.P * row;
                const bool same = ((j + k) & 1) == cc;
                uxp = u.ld(same ? us : uo, wo);
                kxp = kfield ? __ldg((same ? ks : ko) + wo) : T(0);
            } else {
                mxp = T(0);
                if (L.bc[1] == BC_DIRC) bx += (T)dir_c<0, UNI>(L, i);
            }
        }
        const T cxm = (T)face_c<0, UNI>(L, i, i > 0 ? i - 1 : nx1), cxp = (T)face_c<0, UNI>(L, i, i < nx1 ? i + 1 : 0);
        const T kc = kfield ? kc4.v[e] : op.kc;
        const T d0 = op.dex[0] ? __ldg(sel(op.dex, cc) + o0 + e) : op.dexc;
        T w0, w1;
        if (kfield) { w0 = mxm * (kc + kxm) * cxm; w1 = mxp * (kc + kxp) * cxp; }
        else { w0 = mxm * cxm; w1 = mxp * cxp; }
        const T ws = wsum.v[e] + (w0 + w1);
        const T ac = acc.v[e] + (w0 * uxm + w1 * uxp);
        const T bnd = bx + byz;
        if (kfield) { diag.v[e] = d0 + T(0.5) * ws + kc * bnd; off.v[e] = T(-0.5) * ac; }
        else { diag.v[e] = d0 + kc * (ws + bnd); off.v[e] = -kc * ac; }
    }
}

// one y or z face of a group added to the face sums (mask 0: no neighbour)
template <class T, int W>
__device__ __forceinline__ void add_face(bool kfield, const VecW<T, W>& kc4, const VecW<T, W>& un,
                                         const VecW<T, W>& kn, int m, T cf, VecW<T, W>& acc, VecW<T, W>& wsum)
{
    if (!m) return;
#pragma unroll
    for (int e = 0; e < W; e++) {
        const T w = kfield ? (kc4.v[e] + kn.v[e]) * cf : cf;
        wsum.v[e] += w;
        acc.v[e] += w * un.v[e];
    }
}

template <class T, int W, class U, bool UNI = true, bool IN = false>
__device__ __forceinline__ void group_rows(const Lev& L, const KOp<T>& op, int c, const U& u, int row, int j,
                                           int k, int h0, int q, int o0, VecW<T, W>& diag, VecW<T, W>& off)
{
    const int cc = c, oc = c ^ 1;
    const bool kfield = op.k[0] != nullptr;
    const T* uo = u.ptr(oc);
    const T* us = u.ptr(cc);
    const T* ko = kfield ? sel(op.k, oc) : nullptr;
    const T* ks = kfield ? sel(op.k, cc) : nullptr;
    // y and z face coefficients of this row (the wrapped neighbour of a
    // periodic face is the last cell when p = 0)
    const int ny1 = L.ny - 1, nz1 = L.nz - 1;
    const T cym = (T)face_c<1, UNI>(L, j, j > 0 ? j - 1 : ny1), cyp = (T)face_c<1, UNI>(L, j, j < ny1 ? j + 1 : 0);
    const T czm = (T)face_c<2, UNI>(L, k, k > 0 ? k - 1 : nz1), czp = (T)face_c<2, UNI>(L, k, k < nz1 ? k + 1 : 0);

    VecW<T, W> acc = zerov<T, W>(), wsum = zerov<T, W>();
    const VecW<T, W> kc4 = kfield ? ldv<T, W>(ks + o0) : zerov<T, W>();
    int dcount_y = 0, dcount_z = 0;
    // y and z faces, accumulated one at a time
#define MPS_YZ(AXV, SV, CF, DC)                                                                      \
    {                                                                                                \
        VecW<T, W> un, kn;                                                                           \
        int m, dd;                                                                                   \
        yz_face<T, W, AXV, SV, IN>(L, j, k, h0, cc, uo, us, ko, ks, kfield, un, kn, m, dd);          \
        DC += dd;                                                                                    \
        add_face<T, W>(kfield, kc4, un, kn, m, CF, acc, wsum);                                       \
    }
    MPS_YZ(1, -1, cym, dcount_y)
    MPS_YZ(1, 1, cyp, dcount_y)
    MPS_YZ(2, -1, czm, dcount_z)
    MPS_YZ(2, 1, czp, dcount_z)
#undef MPS_YZ
    const T byz = (T)dcount_y * (T)dir_c<1, UNI>(L, j) + (T)dcount_z * (T)dir_c<2, UNI>(L, k);
    const VecW<T, W> ax = uo ? ldv<T, W>(uo + o0) : zerov<T, W>();
    const VecW<T, W> akx = kfield ? ldv<T, W>(ko + o0) : zerov<T, W>();
    row_finish<T, W, U, UNI, IN>(L, op, c, u, row, j, k, h0, q, o0, kc4, acc, wsum, byz, ax, akx, diag, off);
}

// decode the group index of a vector launch
struct GroupIdx {
    int row, j, k, h0, q, o0;
};
template <int W>
__device__ __forceinline__ bool group_decode(const Lev& L, const FastDiv& divG, int c, GroupIdx& G)
{
    const unsigned ng = (unsigned)L.P / W;
    const unsigned t = blockIdx.x * TPB + threadIdx.x;
    const unsigned row = divG.div(t);
    if (row >= L.rows) return false;
    G.row = (int)row;
    G.k = (int)L.divNy.div(row);
    G.j = (int)row - G.k * L.ny;
    G.h0 = W * (int)(t - row * ng);
    G.q = (G.j + G.k + c) & 1;
    G.o0 = G.h0 + L.P * (int)row;
    return true;
}

// colour pass, W cells of colour c per thread (vector loads).  Elements past
// the end of the row (pads) are written as 0.  Same results as k_colour.
// cells per thread and minimum resident blocks of the finest level's colour
// pass and residual; measured on the 257^3 plasma Poisson solve with the
// interior / shell split: FP32 4 cells (128-bit accesses) at 4 blocks of 256
// per SM, 52.1 us per pass (8 cells at 3 blocks: 54.7, at 4: 56.2, at 2:
// 54.1; 4 cells at 3 blocks: 53.4, at 5: 54.9; 2 cells at 6: 57.7); FP64 4
// cells (256-bit accesses) at 3 blocks
#ifndef MPS_COLOUR_W32
#define MPS_COLOUR_W32 4
#endif
#ifndef MPS_COLOUR_W64
#define MPS_COLOUR_W64 4
#endif
#ifndef MPS_COLOUR_MINB32
#define MPS_COLOUR_MINB32 4
#endif
#ifndef MPS_COLOUR_MINB64
#define MPS_COLOUR_MINB64 3
#endif
template <class T>
struct ColourShape {
    static constexpr int W = sizeof(T) == 4 ? MPS_COLOUR_W32 : MPS_COLOUR_W64;
    static constexpr int MINB = sizeof(T) == 4 ? MPS_COLOUR_MINB32 : MPS_COLOUR_MINB64;
};
// the colour pass of the levels below the finest: half the width and 4
// blocks per SM (at 128^3 the finest shape's 512 blocks are 1.15 waves of
// 3 per SM); measured on the 257^3 plasma Poisson solve: 14.76 ms mixed /
// 25.48 ms FP64 against 15.19 / 25.87 with the finest shape, 4 blocks per
// SM at the finest width no better, 2 FP32 / 1 FP64 cells worse
#ifndef MPS_COARSE_W32
#define MPS_COARSE_W32 4
#endif
#ifndef MPS_COARSE_MINB32
#define MPS_COARSE_MINB32 4
#endif
#ifndef MPS_COARSE_W64
#define MPS_COARSE_W64 2
#endif
#ifndef MPS_COARSE_MINB64
#define MPS_COARSE_MINB64 4
#endif
template <class T>
struct CoarseShape {
    static constexpr int W = sizeof(T) == 4 ? MPS_COARSE_W32 : MPS_COARSE_W64;
    static constexpr int MINB = sizeof(T) == 4 ? MPS_COARSE_MINB32 : MPS_COARSE_MINB64;
};
// the colour pass of the levels two or more below the finest (64^3 and
// smaller at 257^3): one cell per thread -- these launches are bound by the
// latency of a thread's work, not by bytes (measured: 14.23 ms mixed /
// 23.64 ms FP64 with one cell per thread here and in the transfers, against
// 14.53 / 23.92 with the 128^3 level's shapes)
#ifndef MPS_SMALL_W32
#define MPS_SMALL_W32 1
#endif
#ifndef MPS_SMALL_W64
#define MPS_SMALL_W64 1
#endif
template <class T>
struct SmallShape {
    static constexpr int W = sizeof(T) == 4 ? MPS_SMALL_W32 : MPS_SMALL_W64;
    static constexpr int MINB = sizeof(T) == 4 ? MPS_COARSE_MINB32 : MPS_COARSE_MINB64;
};

template <class T, int W, class U, int MB = ColourShape<T>::MINB>
__global__ void __launch_bounds__(TPB, MB) k_colourv(Lev L, KOp<T> op, int c, U u, T* __restrict__ out,
                                                    const T* __restrict__ f, FastDiv divG)
{
    pdl_wait();
    GroupIdx G;
    if (!group_decode<W>(L, divG, c, G)) return;
    const VecW<T, W> f4 = ldv<T, W>(f + G.o0);
    VecW<T, W> diag, off;
    if (L.uniform) group_rows<T, W, U, true>(L, op, c, u, G.row, G.j, G.k, G.h0, G.q, G.o0, diag, off);
    else group_rows<T, W, U, false>(L, op, c, u, G.row, G.j, G.k, G.h0, G.q, G.o0, diag, off);
    VecW<T, W> res;
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = 2 * (G.h0 + e) + G.q;
        res.v[e] = i < L.nx ? gs_value(f4.v[e], diag.v[e], off.v[e]) : T(0);
    }
    stv<T, W>(out + G.o0, res);
}

// residual of colour c on a uniform level, W cells per thread: r = f - A u
// (u, f of type T), optional r out (type R, split half c), and the sums of
// r^2 and f^2 reduced deterministically (accumulate = add to rb.out, for the
// second colour)
#ifndef MPS_RESID_W64
#define MPS_RESID_W64 MPS_COLOUR_W64
#endif
#ifndef MPS_RESID_MINB64
#define MPS_RESID_MINB64 MPS_COLOUR_MINB64
#endif
template <class T>
struct ResidShape {
    static constexpr int W = sizeof(T) == 4 ? MPS_COLOUR_W32 : MPS_RESID_W64;
    static constexpr int MINB = sizeof(T) == 4 ? MPS_COLOUR_MINB32 : MPS_RESID_MINB64;
};
template <class T, int W, class R>
__global__ void __launch_bounds__(TPB, ResidShape<T>::MINB) k_residv(Lev L, KOp<T> op, int c, CSplit<T> u,
                                                                       const T* __restrict__ f, R* __restrict__ rout,
                                                                       RedBuf rb, int accumulate, FastDiv divG)
{
    pdl_wait();
    __shared__ double sh[32];
    double rr = 0.0, ff = 0.0;
    const unsigned ngroups = (unsigned)(L.P / W) * L.rows;
    // grid-stride: a few hundred blocks keep the norm reduction's tail short
    for (unsigned base = blockIdx.x * TPB; base < ngroups; base += gridDim.x * TPB) {
        GroupIdx G;
        const unsigned t = base + threadIdx.x;
        const unsigned row = divG.div(t);
        if (row >= L.rows) continue;
        G.row = (int)row;
        G.k = (int)L.divNy.div(row);
        G.j = (int)row - G.k * L.ny;
        G.h0 = W * (int)(t - row * (unsigned)(L.P / W));
        G.o0 = G.h0 + L.P * (int)row;
        // c < 0: both colours of the group, one after the other (the second
        // colour's neighbours were just read as the first colour's centres)
        const int c0 = c < 0 ? 0 : c, c1 = c < 0 ? 1 : c;
        for (int cc = c0; cc <= c1; cc++) {
            G.q = (G.j + G.k + cc) & 1;
            VecW<T, W> diag, off;
            group_rows<T, W, CSplit<T>>(L, op, cc, u, G.row, G.j, G.k, G.h0, G.q, G.o0, diag, off);
            const T* fh = c < 0 ? f + (cc ? L.half : 0) : f;
            const VecW<T, W> f4 = ldv<T, W>(fh + G.o0);
            const VecW<T, W> u4 = ldv<T, W>(u.half(cc) + G.o0);
            VecW<R, W> r4;
#pragma unroll
            for (int e = 0; e < W; e++) {
                const int i = 2 * (G.h0 + e) + G.q;
                const T r = f4.v[e] - (diag.v[e] * u4.v[e] + off.v[e]);
                const bool ok = i < L.nx;
                r4.v[e] = ok ? (R)r : R(0);
                if (ok) {
                    rr += (double)r * (double)r;
                    ff += (double)f4.v[e] * (double)f4.v[e];
                }
            }
            if (rout) stv<R, W>(rout + (c < 0 && cc ? L.half : 0) + G.o0, r4);
        }
    }
    const double a = block_sum(rr, sh);
    const double b = block_sum(ff, sh);
    if (!rb.partial) return;
    // finish: last block sums the partials in block order
    __shared__ bool last;
    if (threadIdx.x == 0) {
        rb.partial[2 * blockIdx.x] = a;
        rb.partial[2 * blockIdx.x + 1] = b;
        __threadfence();
        last = (atomicAdd(rb.counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double sa = 0.0, sb = 0.0;
    for (unsigned qd = threadIdx.x; qd < gridDim.x; qd += blockDim.x) {
        sa += ((volatile double*)rb.partial)[2 * qd];
        sb += ((volatile double*)rb.partial)[2 * qd + 1];
    }
    sa = block_sum(sa, sh);
    sb = block_sum(sb, sh);
    if (threadIdx.x == 0) {
        rb.out[0] = accumulate ? rb.out[0] + sa : sa;
        rb.out[1] = accumulate ? rb.out[1] + sb : sb;
        *rb.counter = 0u;
    }
}

// ---------------------------------------------------------------------
// residual r = f - A u on the fine level fused with the restriction to the
// coarse level: coarse value = mean of r over the children {2I,2I+1}^3 that
// exist (restriction, mgridsteps.f90:11-53, applied to the residual at :531).
// One thread per coarse cell, natural order.
// ---------------------------------------------------------------------
// the coarse level's first red pass from a zero state, written with the
// restriction: u(red) = f / diag (gs_value with a zero off-diagonal part, as the
// zero-state colour pass computes it); d holds the coarse rows' diagonals
// (red half).  u == nullptr: no such write.
template <class T>
struct RedZ {
    T* u;
    const T* d;
};

// the red pass from zero at coarse cell (I,J,K) (split offset o) whose
// right-hand side is v
template <class T>
__device__ __forceinline__ void redz_put(const RedZ<T>& rz, int colour, long long o, T v)
{
    if (rz.u && colour == 0) rz.u[o] = gs_value<T>(v, __ldg(&rz.d[o]), T(0));
}

// the share `part` of `nparts` of the children of coarse cell (I,J,K):
// sum of width-weighted residuals and of the weights
template <class T, class Op>
__device__ __forceinline__ void resid_restrict_part(const Lev& F, const Op& op, const CSplit<T>& u,
                                                    const CSplit<T>& f, const Lev& C, int geom, int I, int J, int K,
                                                    int part, int nparts, T& s, T& vol)
{
    const int cI[3] = {I, J, K};
    int lo[3], cnt[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const int nf = lev_n(F, a), nc = lev_n(C, a);
        lo[a] = nf == nc ? cI[a] : 2 * cI[a];
        cnt[a] = nf == nc ? 1 : ((geom && cI[a] == nc - 1) ? nf - 2 * (nc - 1) : 2);
    }
    s = T(0);
    vol = T(0);
    const int total = cnt[0] * cnt[1] * cnt[2];
    for (int ch = part; ch < total; ch += nparts) {
        const int di = ch % cnt[0], dj = (ch / cnt[0]) % cnt[1], dk = ch / (cnt[0] * cnt[1]);
        const int i = lo[0] + di, j = lo[1] + dj, k = lo[2] + dk;
        const T v = geom ? (T)(cwidth(F, 0, i) * cwidth(F, 1, j) * cwidth(F, 2, k)) : T(1);
        T diag, off;
        row_any<T>(op, F, u, i, j, k, diag, off);
        const T r = f.get(F, i, j, k) - (diag * u.get(F, i, j, k) + off);
        s += v * r;
        vol += v;
    }
}

template <class T, class Op>
__device__ __forceinline__ void resid_restrict_body(const Lev& F, const Op& op, const CSplit<T>& u,
                                                    const CSplit<T>& f, const Lev& C, const Split<T>& fc, int geom,
                                                    unsigned t, RedZ<T> rz = RedZ<T>{nullptr, nullptr})
{
    const unsigned ncx = C.nx, ncy = C.ny;
    if (t >= ncx * ncy * (unsigned)C.nz) return;
    const unsigned K = t / (ncx * ncy);
    const unsigned rem = t - K * ncx * ncy;
    const unsigned J = rem / ncx;
    const unsigned I = rem - J * ncx;
    T s, vol;
    resid_restrict_part<T, Op>(F, op, u, f, C, geom, (int)I, (int)J, (int)K, 0, 1, s, vol);
    const T v = geom ? s / vol : s * (T(1) / vol);
    fc.half(scol(I, J, K))[soff(C, I, J, K)] = v;
    redz_put(rz, scol(I, J, K), soff(C, I, J, K), v);
}

template <class T, class Op>
__global__ void __launch_bounds__(TPB) k_resid_restrict(Lev F, Op op, CSplit<T> u, CSplit<T> f, Lev C,
                                                        Split<T> fc, int geom, RedZ<T> rz)
{
    pdl_wait();
    resid_restrict_body<T, Op>(F, op, u, f, C, fc, geom, blockIdx.x * TPB + threadIdx.x, rz);
}

// ---------------------------------------------------------------------
// fused residual + restriction in two launches.  Bulk: the coarse cells
// whose 2x2x2 children are regular cells away from odd periodic seams (a
// box).  After a black pass the black residual vanishes there, and the red
// child of coarse cell I in fine row (j,k) sits at split offset I of that
// row's red half, so one thread takes W consecutive coarse cells of one
// coarse row: the red residuals of the four fine rows (2J+dj, 2K+dk) with the
// vector row evaluation, summed and scaled by 1/8 (equal children).  No
// residual is stored.  Shell: every other coarse cell, with the general body
// (all children, residual evaluated on the fly).
// ---------------------------------------------------------------------
struct Box {
    int lo[3], hi[3];
};

// the fused residual + restriction keeps 4 cells per thread (its thread
// holds the sums of four fine rows; 8 FP32 cells spill)
#ifndef MPS_RESTRICT_W64
#define MPS_RESTRICT_W64 4
#endif
#ifndef MPS_RESTRICT_MINB64
#define MPS_RESTRICT_MINB64 3
#endif
#ifndef MPS_RESTRICT_W32
#define MPS_RESTRICT_W32 4
#endif
// prolongation: 2 cells per thread (measured at 257^3: 41.3 / 59.4 us FP32 /
// FP64 against 45.7 / 73.9 with 4 and 87 with 8 FP32 cells)
#ifndef MPS_PROLONG_W32
#define MPS_PROLONG_W32 2
#endif
#ifndef MPS_PROLONG_W64
#define MPS_PROLONG_W64 2
#endif
#ifndef MPS_RESTRICT_MINB32
#define MPS_RESTRICT_MINB32 4
#endif
template <class T>
struct RestrictShape {
    static constexpr int W = sizeof(T) == 4 ? MPS_RESTRICT_W32 : MPS_RESTRICT_W64;
    static constexpr int MINB = sizeof(T) == 4 ? MPS_RESTRICT_MINB32 : MPS_RESTRICT_MINB64;
};
// cells per thread of the prolongation bulk on the finest level
template <class T>
struct ProlongShape {
    static constexpr int W = sizeof(T) == 4 ? MPS_PROLONG_W32 : MPS_PROLONG_W64;
};
// restriction and prolongation from the levels below the finest: 2 cells
// per thread (measured on the 257^3 plasma Poisson solve: 14.49 ms mixed /
// 25.03 ms FP64 against 14.76 / 25.45 with 4; 1 cell per thread within
// noise of 2)
#ifndef MPS_XFER_COARSE_W32
#define MPS_XFER_COARSE_W32 2
#endif
#ifndef MPS_XFER_COARSE_W64
#define MPS_XFER_COARSE_W64 2
#endif
#ifndef MPS_XFER_COARSE_MINB32
#define MPS_XFER_COARSE_MINB32 4
#endif
#ifndef MPS_XFER_COARSE_MINB64
#define MPS_XFER_COARSE_MINB64 4
#endif
template <class T>
struct CoarseXferShape {
    static constexpr int W = sizeof(T) == 4 ? MPS_XFER_COARSE_W32 : MPS_XFER_COARSE_W64;
    static constexpr int MINB = sizeof(T) == 4 ? MPS_XFER_COARSE_MINB32 : MPS_XFER_COARSE_MINB64;
};
#ifndef MPS_XFER_SMALL_W
#define MPS_XFER_SMALL_W 1
#endif
template <class T>
struct SmallXferShape {
    static constexpr int W = MPS_XFER_SMALL_W > 0 ? MPS_XFER_SMALL_W : CoarseXferShape<T>::W;
    static constexpr int MINB = CoarseXferShape<T>::MINB;
};

// the r-th row (j,k) of an ny x nz set outside the rectangle [lo1,hi1] x [lo2,hi2]
__device__ __forceinline__ void shell_row(unsigned r, int ny, const Box& b, int& j, int& k)
{
    const unsigned uny = (unsigned)ny;
    const unsigned yin = (unsigned)(b.hi[1] - b.lo[1] + 1), yout = uny - yin;
    const unsigned s1 = (unsigned)b.lo[2] * uny;
    if (r < s1) { k = (int)(r / uny); j = (int)(r - (unsigned)k * uny); return; }
    r -= s1;
    const unsigned zin = (unsigned)(b.hi[2] - b.lo[2] + 1);
    const unsigned s2 = zin * yout;
    if (r < s2) {
        const unsigned kk = r / yout;
        k = b.lo[2] + (int)kk;
        const unsigned q = r - kk * yout;
        j = (int)(q < (unsigned)b.lo[1] ? q : b.hi[1] + 1 + (q - b.lo[1]));
        return;
    }
    r -= s2;
    const unsigned kk = r / uny;
    k = b.hi[2] + 1 + (int)kk;
    j = (int)(r - kk * uny);
}

// W cells of one row of colour c of the explicit-row operator whose six
// neighbours are inside the grid and of the other colour: the colour's seven
// row arrays and the other colour's neighbour rows as vectors, the x
// neighbours from the row's own vector plus one scalar; faces summed in
// row_eval's order (x-, x+, y-, y+, z-, z+)
template <class T, int W, class U>
__device__ __forceinline__ void rop_group(const Lev& L, const ROp<T>& op, int c, const U& u, int row, int h0,
                                          int q, int o0, VecW<T, W>& diag, VecW<T, W>& off)
{
    const int oc = c ^ 1;
    const T* uo = u.ptr(oc);
    const int sy = L.P, sz = L.P * L.ny;
    auto ldu = [&](int o) { return uo ? ldv<T, W>(uo + o) : zerov<T, W>(); };
    const VecW<T, W> ax = ldu(o0);
    const int so = q ? o0 + W : o0 - 1;
    const T sx = uo ? __ldg(uo + so) : T(0);
    const VecW<T, W> uym = ldu(o0 - sy), uyp = ldu(o0 + sy), uzm = ldu(o0 - sz), uzp = ldu(o0 + sz);
    VecW<T, W> r[7];
#pragma unroll
    for (int f = 0; f < 7; f++) r[f] = ldv<T, W>(sel(op.r[f], c) + o0);
#pragma unroll
    for (int e = 0; e < W; e++) {
        T uxm, uxp;
        if (q) {
            uxm = ax.v[e];
            uxp = e < W - 1 ? ax.v[e + 1] : sx;
        } else {
            uxm = e > 0 ? ax.v[e - 1] : sx;
            uxp = ax.v[e];
        }
        T acc = T(0);
        acc += r[1].v[e] * uxm;
        acc += r[2].v[e] * uxp;
        acc += r[3].v[e] * uym.v[e];
        acc += r[4].v[e] * uyp.v[e];
        acc += r[5].v[e] * uzm.v[e];
        acc += r[6].v[e] * uzp.v[e];
        diag.v[e] = r[0].v[e];
        off.v[e] = acc;
    }
}

// the W coarse cells I = h0 .. h0+W-1 of coarse row (J, K) from their four
// red fine rows; IN: every fine cell involved has its neighbours inside the
// grid and regular faces (no boundary code)
template <class T, int W, bool UNI, bool IN, class Op = KOp<T>>
__device__ __forceinline__ void restrict_cells(const Lev& F, const Op& op, const CSplit<T>& u,
                                               const T* __restrict__ fred, const Lev& C, const Split<T>& fc,
                                               const Box& bx, int J, int K, int h0,
                                               const RedZ<T>& rz = RedZ<T>{nullptr, nullptr})
{
    VecW<T, W> s = zerov<T, W>();
#pragma unroll
    for (int dk = 0; dk < 2; dk++)
#pragma unroll
        for (int dj = 0; dj < 2; dj++) {
            const int j = 2 * J + dj, k = 2 * K + dk;
            const int row = j + F.ny * k;
            const int q = (j + k) & 1;
            const int o0 = h0 + F.P * row;
            VecW<T, W> diag, off;
            if constexpr (std::is_same<Op, KOp<T>>::value) {
                group_rows<T, W, CSplit<T>, UNI, IN>(F, op, 0, u, row, j, k, h0, q, o0, diag, off);
            } else if constexpr (IN) {
                rop_group<T, W, CSplit<T>>(F, op, 0, u, row, h0, q, o0, diag, off);
            } else {  // explicit rows near the boundary: cell by cell
#pragma unroll
                for (int e = 0; e < W; e++) {
                    const int i = 2 * (h0 + e) + q;
                    diag.v[e] = T(0);
                    off.v[e] = T(0);
                    if (i < F.nx) row_any<T>(op, F, u, i, j, k, diag.v[e], off.v[e]);
                }
            }
            const VecW<T, W> f4 = ldv<T, W>(fred + o0);
            const VecW<T, W> u4 = ldv<T, W>(u.c[0] + o0);
#pragma unroll
            for (int e = 0; e < W; e++) s.v[e] += f4.v[e] - (diag.v[e] * u4.v[e] + off.v[e]);
        }
    const long long cb = (long long)C.P * (J + (long long)C.ny * K);
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int I = h0 + e;
        if (I >= bx.lo[0] && I <= bx.hi[0]) {
            const T v = s.v[e] * T(0.125);
            fc.half((I + J + K) & 1)[(I >> 1) + cb] = v;
            // (the 4-cell form of the finest level has no registers to spare)
            if constexpr (W <= 2) redz_put(rz, (I + J + K) & 1, (I >> 1) + cb, v);
        }
    }
}

// Block (or block-sized chunk) b of a split launch: the interior and x-end
// chunks are interleaved in proportion, so that the ends of a row run while
// the row's neighbours are still in L2 (the x-end chunks follow the same
// row order as the interior ones); the face rows come last.  part: 0
// interior, 1 x ends, 2 face rows; idx: the chunk within its part.
__device__ __forceinline__ void split_chunk(unsigned nb_in, unsigned nb_xe, unsigned b, int& part, unsigned& idx)
{
    const unsigned m = nb_in + nb_xe;
    if (b >= m) {
        part = 2;
        idx = b - m;
        return;
    }
    const unsigned lo = (unsigned)(((unsigned long long)b * nb_xe) / m);
    const unsigned hi = (unsigned)(((unsigned long long)(b + 1) * nb_xe) / m);
    if (hi > lo) {
        part = 1;
        idx = lo;
    } else {
        part = 0;
        idx = b - lo;
    }
}

// the bulk of the restriction in two parts: interior coarse rows [J0, J0+nJ)
// x [K0, K0+nK) with groups [ga, gb] (no boundary code), then the rest of
// the bulk -- the other groups of those rows, and every group of the coarse
// rows outside that rectangle (cells outside the box return)
struct RestrictSplit {
    FastDiv gin;      // by the interior groups
    FastDiv yin;      // by nJ
    FastDiv gx;       // by the other groups of a row (G - gin)
    FastDiv g;        // by the groups of a row (G = fine P / W)
    int ga, gb, J0, K0;
    unsigned n_in, n_xe, n_out;
    unsigned nb_in, nb_xe, nb_out;  // blocks of the three parts (interleaved by split_chunk)
    Box rect;         // the interior coarse rows (y/z bounds)
};

template <class T, int W, bool UNI, class Op = KOp<T>>
__device__ __forceinline__ void resid_restrict_bulk(const Lev& F, const Op& op, const CSplit<T>& u,
                                                    const T* __restrict__ fred, const Lev& C, const Split<T>& fc,
                                                    const Box& bx, const RestrictSplit& rs, unsigned blk,
                                                    const RedZ<T>& rz = RedZ<T>{nullptr, nullptr})
{
    int part;
    unsigned idx;
    split_chunk(rs.nb_in, rs.nb_xe, blk, part, idx);
    if (part == 0) {
        const unsigned t = idx * TPB + threadIdx.x;
        if (t >= rs.n_in) return;
        const unsigned r = rs.gin.div(t);
        const int g = rs.ga + (int)(t - r * rs.gin.d);
        const unsigned kk = rs.yin.div(r);
        restrict_cells<T, W, true, true, Op>(F, op, u, fred, C, fc, bx, rs.J0 + (int)(r - kk * rs.yin.d),
                                         rs.K0 + (int)kk, W * g, rz);
        return;
    }
    const unsigned t = idx * TPB + threadIdx.x;
    int J, K, g;
    if (part == 1) {
        if (t >= rs.n_xe) return;
        const unsigned r = rs.gx.div(t);
        const unsigned e = t - r * rs.gx.d;
        g = e < (unsigned)rs.ga ? (int)e : rs.gb + 1 + (int)(e - rs.ga);
        const unsigned kk = rs.yin.div(r);
        J = rs.J0 + (int)(r - kk * rs.yin.d);
        K = rs.K0 + (int)kk;
    } else {
        if (t >= rs.n_out) return;
        const unsigned r = rs.g.div(t);
        g = (int)(t - r * rs.g.d);
        shell_row(r, C.ny, rs.rect, J, K);
    }
    if (J < bx.lo[1] || J > bx.hi[1] || K < bx.lo[2] || K > bx.hi[2]) return;
    const int h0 = W * g;
    if (h0 > bx.hi[0] || h0 + W - 1 < bx.lo[0]) return;
    restrict_cells<T, W, UNI, false, Op>(F, op, u, fred, C, fc, bx, J, K, h0, rz);
}

// the t-th cell of an n[0] x n[1] x n[2] grid outside box b: z slabs first,
// then y slabs of the remaining planes, then the x ends of the remaining rows
__device__ __forceinline__ void shell_cell(unsigned t, const int n[3], const Box& b, int& I, int& J, int& K)
{
    const unsigned nx = n[0], ny = n[1];
    const unsigned zin = b.hi[2] - b.lo[2] + 1, yin = b.hi[1] - b.lo[1] + 1;
    const unsigned yout = ny - yin, xout = nx - (b.hi[0] - b.lo[0] + 1);
    const unsigned plane = ny * nx;
    const unsigned s1 = ((unsigned)n[2] - zin) * plane;
    if (t < s1) {
        const unsigned p = t / plane, r = t - p * plane;
        K = (int)(p < (unsigned)b.lo[2] ? p : b.hi[2] + 1 + (p - b.lo[2]));
        J = (int)(r / nx);
        I = (int)(r - (unsigned)J * nx);
        return;
    }
    t -= s1;
    const unsigned s2 = zin * yout * nx;
    if (t < s2) {
        const unsigned p = t / (yout * nx), r = t - p * yout * nx;
        K = b.lo[2] + (int)p;
        const unsigned q = r / nx;
        J = (int)(q < (unsigned)b.lo[1] ? q : b.hi[1] + 1 + (q - b.lo[1]));
        I = (int)(r - q * nx);
        return;
    }
    t -= s2;
    const unsigned p = t / (yin * xout), r = t - p * yin * xout;
    K = b.lo[2] + (int)p;
    const unsigned q = r / xout, m = r - q * xout;
    J = b.lo[1] + (int)q;
    I = (int)(m < (unsigned)b.lo[0] ? m : b.hi[0] + 1 + (m - b.lo[0]));
}

// eight lanes per shell cell, each summing a share of the children (every
// lane of the warp takes part in the shuffles)
template <class T, class Op, bool RZ = true>
__device__ __forceinline__ void resid_restrict_shell(const Lev& F, const Op& op, const CSplit<T>& u,
                                                     const CSplit<T>& f, const Lev& C, const Split<T>& fc, int geom,
                                                     const Box& bx, unsigned count, unsigned t,
                                                     const RedZ<T>& rz = RedZ<T>{nullptr, nullptr})
{
    const unsigned cell = t >> 3;
    const int part = (int)(t & 7);
    const bool ok = cell < count;
    int I = 0, J = 0, K = 0;
    T s = T(0), vol = T(0);
    if (ok) {
        const int n[3] = {C.nx, C.ny, C.nz};
        shell_cell(cell, n, bx, I, J, K);
        resid_restrict_part<T, Op>(F, op, u, f, C, geom, I, J, K, part, 8, s, vol);
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o, 8);
        vol += __shfl_xor_sync(0xffffffffu, vol, o, 8);
    }
    if (ok && part == 0) {
        const T v = geom ? s / vol : s * (T(1) / vol);
        fc.half(scol(I, J, K))[soff(C, I, J, K)] = v;
        if constexpr (RZ) redz_put(rz, scol(I, J, K), soff(C, I, J, K), v);
    }
}

// bulk and shell in one launch: blocks [0, nb_bulk) take the bulk rows,
// the rest the shell cells
// UNI: the fine level is uniform
template <class T, int W, int MB, bool UNI, class Op = KOp<T>>
__global__ void __launch_bounds__(TPB, MB) k_resid_restrict_v(Lev F, Op op, CSplit<T> u,
                                                                                 const T* __restrict__ fred, Lev C,
                                                                                 Split<T> fc, RestrictSplit rs, Box bx,
                                                                                 unsigned nb_bulk, int geom,
                                                                                 unsigned shell, RedZ<T> rz)
{
    pdl_wait();
    if (blockIdx.x < nb_bulk) {
        resid_restrict_bulk<T, W, UNI, Op>(F, op, u, fred, C, fc, bx, rs, blockIdx.x, rz);
    } else {
        CSplit<T> f;
        f.c[0] = fred;
        f.c[1] = fred + F.half;
        resid_restrict_shell<T, Op, (W <= 2)>(F, op, u, f, C, fc, geom, bx, shell,
                                              (blockIdx.x - nb_bulk) * TPB + threadIdx.x, rz);
    }
}

// the red pass of a colour pass from a zero state, elementwise: u(red) =
// f(red) / diag with the red rows' diagonals of k_diag_red (no neighbour is
// read: every one is zero); pads untouched
template <class T>
__global__ void __launch_bounds__(TPB) k_red_from_zero(Lev L, const T* __restrict__ f, const T* __restrict__ d,
                                                       T* __restrict__ out)
{
    pdl_wait();
    const unsigned t = blockIdx.x * TPB + threadIdx.x;
    int i, j, k;
    if (!decode(L, t, 0, i, j, k)) return;
    out[t] = gs_value<T>(f[t], d[t], T(0));
}

// the diagonal of every red row of a level (the zero-state colour pass's
// divisor), for the red pass written with the restriction
template <class T, class Op>
__global__ void __launch_bounds__(TPB) k_diag_red(Lev L, Op op, T* __restrict__ d)
{
    pdl_wait();
    const unsigned t = blockIdx.x * TPB + threadIdx.x;
    int i, j, k;
    if (!decode(L, t, 0, i, j, k)) return;
    T diag, off;
    row_any<T>(op, L, ZeroU<T>(), i, j, k, diag, off);
    d[soff(L, i, j, k)] = diag;
}

// coarse ghost rule for the correction (update_boundary_ghostvalues applied
// to restrictsolnnew - restrictsolnold, mgridsteps.f90:552-562): Dirichlet
// faces mirror with a sign flip, other physical faces copy, periodic wraps
template <class T>
__device__ __forceinline__ T coarse_nbr(const Lev& C, const CSplit<T>& e, int I, int J, int K, int ax, int s,
                                        T e0)
{
    int a = I, b = J, c = K;
    if (nbr(C, ax, s, a, b, c)) return e.get(C, a, b, c);
    return C.bc[2 * ax + (s > 0)] == BC_DIRC ? -e0 : e0;
}

// coarse correction at (I,J,K) where any index may be a ghost (-1 or n):
// each ghost axis maps to the adjacent cell with the sign of its face rule
// (Dirichlet -1, other +1) or wraps (periodic); equals the face ghosts of
// update_boundary_ghostvalues, extended to edges and corners
template <class T>
__device__ __forceinline__ T coarse_at(const Lev& C, const CSplit<T>& e, int I, int J, int K)
{
    int q[3] = {I, J, K};
    T sgn = T(1);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const int n = lev_n(C, a);
        if (q[a] >= 0 && q[a] < n) continue;
        const int side = q[a] < 0 ? 0 : 1;
        if (C.per[a]) q[a] = q[a] < 0 ? n - 1 : 0;
        else {
            if (C.bc[2 * a + side] == BC_DIRC) sgn = -sgn;
            q[a] = q[a] < 0 ? 0 : n - 1;
        }
    }
    return sgn * e.get(C, q[0], q[1], q[2]);
}

// ---------------------------------------------------------------------
// prolongation + correction u_f += P e_c.  CELL: prolongation1
// (mgridsteps.f90:170-216, correction :567): e_c + sum_ax +-1/8 *
// (e[I+1]-e[I-1]), odd last fine cell uncorrected.  GEOM: tensor-product
// linear interpolation between the bracketing coarse centres.  One thread
// per fine cell.
// ---------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void prolong_body(const Lev& F, const Split<T>& u, const Lev& C, const CSplit<T>& e,
                                             const Xfer& X, int only_col, unsigned t)
{
    unsigned i, j, k;
    if (only_col < 0) {  // all cells, natural order
        const unsigned nx = F.nx, ny = F.ny;
        if (t >= nx * ny * (unsigned)F.nz) return;
        k = t / (nx * ny);
        unsigned rem = t - k * nx * ny;
        j = rem / nx;
        i = rem - j * nx;
    } else if (only_col == 2) {  // red cells on the odd periodic seam planes
        int ii, jj, kk;
        if (!decode(F, t, 0, ii, jj, kk)) return;
        const bool seam = (F.per[0] && (F.nx & 1) && (ii == 0 || ii == F.nx - 1)) ||
                          (F.per[1] && (F.ny & 1) && (jj == 0 || jj == F.ny - 1)) ||
                          (F.per[2] && (F.nz & 1) && (kk == 0 || kk == F.nz - 1));
        if (!seam) return;
        i = ii; j = jj; k = kk;
    } else {  // the cells of one colour, split order (coalesced on that half)
        int ii, jj, kk;
        if (!decode(F, t, only_col, ii, jj, kk)) return;
        i = ii; j = jj; k = kk;
    }
    T v;
    if (!X.geom) {
        int I = i >> 1, J = j >> 1, K = k >> 1;
        if (I >= C.nx || J >= C.ny || K >= C.nz) return;  // odd last cell dropped
        const T e0 = e.get(C, I, J, K);
        const T ax = (i & 1) ? T(0.125) : T(-0.125);
        const T ay = (j & 1) ? T(0.125) : T(-0.125);
        const T az = (k & 1) ? T(0.125) : T(-0.125);
        const T dx = coarse_at(C, e, I + 1, J, K) - coarse_at(C, e, I - 1, J, K);
        const T dy = coarse_at(C, e, I, J + 1, K) - coarse_at(C, e, I, J - 1, K);
        const T dz = coarse_at(C, e, I, J, K + 1) - coarse_at(C, e, I, J, K - 1);
        v = e0 + ((ax * dx + ay * dy) + az * dz);
    } else {
        const Lin lx = X.tab[0][i], ly = X.tab[1][j], lz = X.tab[2][k];
        const T tx = (T)lx.t, ty = (T)ly.t, tz = (T)lz.t;
        const bool inner = lx.j0 >= 0 && lx.j1 < C.nx && ly.j0 >= 0 && ly.j1 < C.ny && lz.j0 >= 0 && lz.j1 < C.nz;
        T c000, c100, c010, c110, c001, c101, c011, c111;
        if (inner) {
            c000 = e.get(C, lx.j0, ly.j0, lz.j0); c100 = e.get(C, lx.j1, ly.j0, lz.j0);
            c010 = e.get(C, lx.j0, ly.j1, lz.j0); c110 = e.get(C, lx.j1, ly.j1, lz.j0);
            c001 = e.get(C, lx.j0, ly.j0, lz.j1); c101 = e.get(C, lx.j1, ly.j0, lz.j1);
            c011 = e.get(C, lx.j0, ly.j1, lz.j1); c111 = e.get(C, lx.j1, ly.j1, lz.j1);
        } else {
            c000 = coarse_at(C, e, lx.j0, ly.j0, lz.j0); c100 = coarse_at(C, e, lx.j1, ly.j0, lz.j0);
            c010 = coarse_at(C, e, lx.j0, ly.j1, lz.j0); c110 = coarse_at(C, e, lx.j1, ly.j1, lz.j0);
            c001 = coarse_at(C, e, lx.j0, ly.j0, lz.j1); c101 = coarse_at(C, e, lx.j1, ly.j0, lz.j1);
            c011 = coarse_at(C, e, lx.j0, ly.j1, lz.j1); c111 = coarse_at(C, e, lx.j1, ly.j1, lz.j1);
        }
        const T x00 = c000 + tx * (c100 - c000), x10 = c010 + tx * (c110 - c010);
        const T x01 = c001 + tx * (c101 - c001), x11 = c011 + tx * (c111 - c011);
        const T y0 = x00 + ty * (x10 - x00), y1 = x01 + ty * (x11 - x01);
        v = y0 + tz * (y1 - y0);
    }
    T* p = &u.half(scol(i, j, k))[soff(F, i, j, k)];
    *p = *p + v;
}

template <class T>
__global__ void __launch_bounds__(TPB) k_prolong_correct(Lev F, Split<T> u, Lev C, CSplit<T> e, Xfer X, int only_col)
{
    pdl_wait();
    prolong_body<T>(F, u, C, e, X, only_col, blockIdx.x * TPB + threadIdx.x);
}

// ---------------------------------------------------------------------
// prolongation + correction on the geometric hierarchy, W cells of one colour
// per thread along a fine row.  Inside a box of fine indices the bracketing
// coarse centres are regular (fine 2I: 1/4 e[I-1] + 3/4 e[I]; fine 2I+1:
// 3/4 e[I] + 1/4 e[I+1]); elsewhere the per-axis tables give the brackets and
// the coarse ghost rule applies (same numbers as k_prolong_correct).
// mode 0: black cells of the groups whose cells all lie inside the box;
// mode 3: the other groups of the rows inside the box in (y,z); mode 1:
// black cells of the other rows; mode 2: red cells on odd periodic seam
// planes (read by the next red pass), one cell per thread.

template <class T>
__device__ __forceinline__ void lin_axis(const Xfer& X, int ax, int i, bool regular, int& a, int& b, T& t)
{
    if (regular) {
        const int I = i >> 1;
        if (i & 1) { a = I; b = I + 1; t = T(0.25); }
        else { a = I - 1; b = I; t = T(0.75); }
    } else {
        const Lin L = X.tab[ax][i];
        a = L.j0;
        b = L.j1;
        t = (T)L.t;
    }
}

template <class T>
__device__ __forceinline__ T coarse_val(const Lev& C, const CSplit<T>& e, int x, int y, int z)
{
    if (x >= 0 && x < C.nx && y >= 0 && y < C.ny && z >= 0 && z < C.nz)
        return __ldg(&e.half((x + y + z) & 1)[(x >> 1) + (long long)C.P * (y + (long long)C.ny * z)]);
    return coarse_at(C, e, x, y, z);
}

template <class T>
__device__ __forceinline__ T trilinear(const Lev& C, const CSplit<T>& e, int x0, int x1, T tx, int y0, int y1, T ty,
                                       int z0, int z1, T tz)
{
    const T c000 = coarse_val(C, e, x0, y0, z0), c100 = coarse_val(C, e, x1, y0, z0);
    const T c010 = coarse_val(C, e, x0, y1, z0), c110 = coarse_val(C, e, x1, y1, z0);
    const T c001 = coarse_val(C, e, x0, y0, z1), c101 = coarse_val(C, e, x1, y0, z1);
    const T c011 = coarse_val(C, e, x0, y1, z1), c111 = coarse_val(C, e, x1, y1, z1);
    const T x00 = c000 + tx * (c100 - c000), x10 = c010 + tx * (c110 - c010);
    const T x01 = c001 + tx * (c101 - c001), x11 = c011 + tx * (c111 - c011);
    const T y0v = x00 + ty * (x10 - x00), y1v = x01 + ty * (x11 - x01);
    return y0v + tz * (y1v - y0v);
}

// divisors of the thread decode (32-bit multiply-high division)
struct ProlongDiv {
    FastDiv g;    // by the groups per row, P / W
    FastDiv yin;  // by the rows of the box along y
    FastDiv nh;   // by the cells of one colour per row, (nx+1)/2
    FastDiv gin;  // by the groups whose cells all lie in the box along x
    FastDiv gout; // by the other groups of a row
    FastDiv yin2; // by the row pairs of the box along y
    int g_lo, g_hi;  // the groups in the box: [g_lo, g_hi]
};

// the four parts of a prolongation in one launch: consecutive block ranges
// take modes 0, 3, 1, 2 (cnt: threads of each part; mode 2 has its own box
// and divisors).  Mode 0 threads take W cells of a 2 x 2 block of rows (the
// box starts at odd j, k and spans an even number of rows along y and z).
struct ProlongParts {
    unsigned cnt[4];   // modes 0, 3, 1, 2
    unsigned blk0[5];  // first block of each part, and the total
};

// block blk (TPB threads) of the prolongation bulk: the parts in pp's order
template <class T, int W>
__device__ __forceinline__ void prolong_v_block(const Lev& F, const Split<T>& u, const Lev& C, const CSplit<T>& e,
                                                const Xfer& X, const Box& pbox, const ProlongDiv& pdiv,
                                                const Box& sbox, const ProlongDiv& sdiv, const ProlongParts& pp,
                                                unsigned blk)
{
    int part = 0;
    while (part < 3 && blk >= pp.blk0[part + 1]) part++;
    const int mode = part == 0 ? 0 : (part == 1 ? 3 : (part == 2 ? 1 : 2));
    const unsigned t = (blk - pp.blk0[part]) * TPB + threadIdx.x;
    if (t >= pp.cnt[part]) return;
    // field-wise selection keeps both parameter structs out of local memory
    const bool m2 = mode == 2;
    Box bx;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        bx.lo[a] = m2 ? sbox.lo[a] : pbox.lo[a];
        bx.hi[a] = m2 ? sbox.hi[a] : pbox.hi[a];
    }
    ProlongDiv dv = pdiv;
    dv.yin.M = m2 ? sdiv.yin.M : pdiv.yin.M;
    dv.yin.l = m2 ? sdiv.yin.l : pdiv.yin.l;
    dv.yin.d = m2 ? sdiv.yin.d : pdiv.yin.d;
    int j, k, h0, c, nel;
    if (mode == 0 || mode == 3) {
        // rows inside the box; mode 0: the groups inside along x (every cell
        // regular, no divergent path in the warp), mode 3: the row ends
        unsigned r, g;
        if (mode == 0) {
            r = dv.gin.div(t);  // the row pair
            g = dv.g_lo + (t - r * dv.gin.d);
            const unsigned kk = dv.yin2.div(r);
            k = bx.lo[2] + 2 * (int)kk;
            j = bx.lo[1] + 2 * (int)(r - kk * dv.yin2.d);
        } else {
            r = dv.gout.div(t);  // the row
            const unsigned e = t - r * dv.gout.d;
            g = e < (unsigned)dv.g_lo ? e : dv.g_hi + 1 + (e - dv.g_lo);
            const unsigned kk = dv.yin.div(r);
            k = bx.lo[2] + (int)kk;
            j = bx.lo[1] + (int)(r - kk * dv.yin.d);
        }
        h0 = W * (int)g;
        c = 1;
        nel = W;
    } else if (mode == 1) {
        const unsigned r = dv.g.div(t);
        h0 = W * (int)(t - r * dv.g.d);
        shell_row(r, F.ny, bx, j, k);
        c = 1;
        nel = W;
    } else {
        // red seam cells: full rows on y/z seam planes, then the two x ends
        // of every other row (bx.lo/hi[1..2] delimit the rows off the planes)
        const bool sx = F.per[0] && (F.nx & 1);
        const unsigned rows_in = (unsigned)(bx.hi[1] - bx.lo[1] + 1) * (unsigned)(bx.hi[2] - bx.lo[2] + 1);
        const unsigned rows_out = (unsigned)F.ny * (unsigned)F.nz - rows_in;
        int i;
        if (t < rows_out * dv.nh.d) {
            const unsigned r = dv.nh.div(t);
            shell_row(r, F.ny, bx, j, k);
            i = 2 * (int)(t - r * dv.nh.d) + ((j + k) & 1);
        } else {
            if (!sx) return;
            const unsigned t2 = t - rows_out * dv.nh.d;
            const unsigned r = t2 >> 1;
            const unsigned kk = dv.yin.div(r);
            k = bx.lo[2] + (int)kk;
            j = bx.lo[1] + (int)(r - kk * dv.yin.d);
            i = (t2 & 1) ? F.nx - 1 : 0;
            if (((i + j + k) & 1) != 0) return;  // not red
        }
        if (i >= F.nx) return;
        int x0, x1, y0, y1, z0, z1;
        T tx, ty, tz;
        lin_axis<T>(X, 0, i, false, x0, x1, tx);
        lin_axis<T>(X, 1, j, false, y0, y1, ty);
        lin_axis<T>(X, 2, k, false, z0, z1, tz);
        T* p = &u.c[0][(i >> 1) + (long long)F.P * (j + (long long)F.ny * k)];
        *p = *p + trilinear<T>(C, e, x0, x1, tx, y0, y1, ty, z0, z1, tz);
        return;
    }
    (void)nel;
    if (mode == 0) {
        // rows (j, k), (j+1, k), (j, k+1), (j+1, k+1) with j, k odd: along y
        // both rows lie between coarse rows J0 and J0+1 (weights 0.25 for j,
        // 0.75 for j+1), likewise along z; all 4W cells regular.  The four
        // coarse rows, interpolated along x once for each cell parity, serve
        // the four fine rows (same lerp order as trilinear())
        const int J0 = j >> 1, K0 = k >> 1;
        const int q0 = (j + k + c) & 1;  // rows (j+1, k) and (j, k+1) have 1 - q0
        VecW<T, W> xi[2][2][2];          // [parity][y][z]
#pragma unroll
        for (int zz = 0; zz < 2; zz++)
#pragma unroll
            for (int yy = 0; yy < 2; yy++) {
                const int rb = C.P * ((J0 + yy) + C.ny * (K0 + zz));
                const int par = (J0 + yy + K0 + zz) & 1;
                T cv[W + 2];  // coarse x = h0 - 1 .. h0 + W
#pragma unroll
                for (int m = 0; m < W + 2; m++) {
                    const int x = h0 - 1 + m;
                    cv[m] = __ldg(&e.half((x + par) & 1)[(x >> 1) + rb]);
                }
#pragma unroll
                for (int qq = 0; qq < 2; qq++) {
                    const T tx = qq ? T(0.25) : T(0.75);
#pragma unroll
                    for (int el = 0; el < W; el++)
                        xi[qq][yy][zz].v[el] = cv[el + qq] + tx * (cv[el + qq + 1] - cv[el + qq]);
                }
            }
#pragma unroll
        for (int dk = 0; dk < 2; dk++)
#pragma unroll
            for (int dj = 0; dj < 2; dj++) {
                const bool qq = (q0 ^ dj ^ dk) != 0;  // selects, not an index: xi stays in registers
                const T ty = dj ? T(0.75) : T(0.25), tz = dk ? T(0.75) : T(0.25);
                T* base = u.half(c) + h0 + (long long)F.P * ((j + dj) + (long long)F.ny * (k + dk));
                VecW<T, W> u4 = ldv<T, W>(base);
#pragma unroll
                for (int el = 0; el < W; el++) {
                    const T x00 = qq ? xi[1][0][0].v[el] : xi[0][0][0].v[el];
                    const T x10 = qq ? xi[1][1][0].v[el] : xi[0][1][0].v[el];
                    const T x01 = qq ? xi[1][0][1].v[el] : xi[0][0][1].v[el];
                    const T x11 = qq ? xi[1][1][1].v[el] : xi[0][1][1].v[el];
                    const T a0 = x00 + ty * (x10 - x00);
                    const T a1 = x01 + ty * (x11 - x01);
                    u4.v[el] += a0 + tz * (a1 - a0);
                }
                stv<T, W>(base, u4);
            }
        return;
    }
    const int q = (j + k + c) & 1;
    const long long o0 = h0 + (long long)F.P * (j + (long long)F.ny * k);
    const bool reg = mode != 1;  // mode 3 rows lie in the box along y and z
    int y0, y1, z0, z1;
    T ty, tz;
    lin_axis<T>(X, 1, j, reg, y0, y1, ty);
    lin_axis<T>(X, 2, k, reg, z0, z1, tz);
    T* base = u.half(c) + o0;
#pragma unroll
    for (int el = 0; el < W; el++) {
        const int i = 2 * (h0 + el) + q;
        if (i >= F.nx) continue;
        const bool xreg = i >= bx.lo[0] && i <= bx.hi[0];
        int x0, x1;
        T tx;
        lin_axis<T>(X, 0, i, xreg, x0, x1, tx);
        base[el] = base[el] + trilinear<T>(C, e, x0, x1, tx, y0, y1, ty, z0, z1, tz);
    }
}

template <class T, int W>
__global__ void __launch_bounds__(TPB) k_prolong_v(Lev F, Split<T> u, Lev C, CSplit<T> e, Xfer X, Box pbox,
                                                   ProlongDiv pdiv, Box sbox, ProlongDiv sdiv, ProlongParts pp)
{
    pdl_wait();
    prolong_v_block<T, W>(F, u, C, e, X, pbox, pdiv, sbox, sdiv, pp, blockIdx.x);
}

// ---------------------------------------------------------------------
// Colour pass of a uniform level in two parts of one launch.  Blocks below
// nb_in take the interior: groups whose cells all have six neighbours inside
// the grid (rows 1 .. ny-2 and 1 .. nz-2, groups g_lo .. g_hi), evaluated
// with no boundary code at all.  The other blocks take the shell: first the
// x-end groups of the interior rows, then every group of the rows on the
// four y/z faces, with the general row evaluation.  Same arithmetic and
// results as k_colourv.
// ---------------------------------------------------------------------
struct ColourSplit {
    FastDiv gin;      // by the interior groups of a row
    FastDiv yin;      // by the interior rows along y (ny - 2)
    FastDiv gx;       // by the x-end groups of a row (G - gin)
    FastDiv g;        // by the groups of a row that hold a cell (G)
    int g_lo, g_hi;   // interior groups
    unsigned n_in;    // interior threads
    unsigned n_xe;    // threads of the x ends of the interior rows
    unsigned n_face;  // threads of the face rows
    unsigned nb_in;   // blocks (or block-sized chunks) of the interior part
    unsigned nb_xe;   // of the x ends
    unsigned nb_face; // of the face rows
    Box b;            // the interior rows: [1, ny-2] x [1, nz-2]
};


// UNI: the level is uniform (shell rows take the regular coefficients too);
// on a level whose last cells are merged the interior stops one cell short
// of them, so its faces are regular either way
// block blk of a split colour pass (TPB threads)
template <class T, int W, class U, bool UNI = true>
__device__ __forceinline__ void colour_split_block(const Lev& L, const KOp<T>& op, int c, const U& u,
                                                   T* __restrict__ out, const T* __restrict__ f,
                                                   const ColourSplit& cs, unsigned blk)
{
    int part;
    unsigned idx;
    split_chunk(cs.nb_in, cs.nb_xe, blk, part, idx);
    if (part == 0) {
        const unsigned t = idx * TPB + threadIdx.x;
        if (t >= cs.n_in) return;
        const unsigned r = cs.gin.div(t);
        const int g = cs.g_lo + (int)(t - r * cs.gin.d);
        const unsigned kk = cs.yin.div(r);
        const int k = 1 + (int)kk, j = 1 + (int)(r - kk * cs.yin.d);
        const int h0 = W * g;
        const int row = j + L.ny * k;
        const int q = (j + k + c) & 1;
        const int o0 = h0 + L.P * row;
        const VecW<T, W> f4 = ldv<T, W>(f + o0);
        VecW<T, W> diag, off;
        group_rows<T, W, U, true, true>(L, op, c, u, row, j, k, h0, q, o0, diag, off);
        VecW<T, W> res;
#pragma unroll
        for (int e = 0; e < W; e++) res.v[e] = gs_value(f4.v[e], diag.v[e], off.v[e]);
        stv<T, W>(out + o0, res);
        return;
    }
    const unsigned t = idx * TPB + threadIdx.x;
    int j, k, g;
    if (part == 1) {
        if (t >= cs.n_xe) return;
        const unsigned r = cs.gx.div(t);
        const unsigned e = t - r * cs.gx.d;
        g = e < (unsigned)cs.g_lo ? (int)e : cs.g_hi + 1 + (int)(e - cs.g_lo);
        const unsigned kk = cs.yin.div(r);
        k = 1 + (int)kk;
        j = 1 + (int)(r - kk * cs.yin.d);
    } else {
        if (t >= cs.n_face) return;
        const unsigned r = cs.g.div(t);
        g = (int)(t - r * cs.g.d);
        shell_row(r, L.ny, cs.b, j, k);
    }
    const int h0 = W * g;
    const int row = j + L.ny * k;
    const int q = (j + k + c) & 1;
    const int o0 = h0 + L.P * row;
    const VecW<T, W> f4 = ldv<T, W>(f + o0);
    VecW<T, W> diag, off;
    group_rows<T, W, U, UNI, false>(L, op, c, u, row, j, k, h0, q, o0, diag, off);
    VecW<T, W> res;
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = 2 * (h0 + e) + q;
        res.v[e] = i < L.nx ? gs_value(f4.v[e], diag.v[e], off.v[e]) : T(0);
    }
    stv<T, W>(out + o0, res);
}

template <class T, int W, class U, int MB, bool UNI = true>
__global__ void __launch_bounds__(TPB, MB) k_colourv_split(Lev L, KOp<T> op, int c, U u, T* __restrict__ out,
                                                           const T* __restrict__ f, ColourSplit cs)
{
    pdl_wait();
    colour_split_block<T, W, U, UNI>(L, op, c, u, out, f, cs, blockIdx.x);
}

// ---------------------------------------------------------------------
// Colour pass of the explicit-row operator (ROp: Scharfetter-Gummel and
// convection rows) in two parts of one launch, as k_colourv_split: the
// interior groups (all six neighbours inside the grid, of the other colour)
// with W cells of a row per thread -- the colour's seven row arrays and the
// other colour's neighbour rows as vectors, the x neighbours from the row's
// own vector plus one scalar -- and the shell cells one at a time through
// the general row evaluation.  The faces are summed in row_eval's order
// (x-, x+, y-, y+, z-, z+), so results equal those of k_colour.
// ---------------------------------------------------------------------
template <class T, int W, class U>
__global__ void __launch_bounds__(TPB) k_colourv_split_rop(Lev L, ROp<T> op, int c, U u, T* __restrict__ out,
                                                           const T* __restrict__ f, ColourSplit cs)
{
    pdl_wait();
    int part;
    unsigned idx;
    split_chunk(cs.nb_in, cs.nb_xe, blockIdx.x, part, idx);
    const unsigned t = idx * TPB + threadIdx.x;
    int j, k, g;
    if (part == 0) {
        if (t >= cs.n_in) return;
        const unsigned r = cs.gin.div(t);
        g = cs.g_lo + (int)(t - r * cs.gin.d);
        const unsigned kk = cs.yin.div(r);
        k = 1 + (int)kk;
        j = 1 + (int)(r - kk * cs.yin.d);
        const int h0 = W * g;
        const int row = j + L.ny * k;
        const int q = (j + k + c) & 1;
        const int o0 = h0 + L.P * row;
        const VecW<T, W> f4 = ldv<T, W>(f + o0);
        VecW<T, W> diag, off;
        rop_group<T, W, U>(L, op, c, u, row, h0, q, o0, diag, off);
        VecW<T, W> res;
#pragma unroll
        for (int e = 0; e < W; e++) res.v[e] = gs_value(f4.v[e], diag.v[e], off.v[e]);
        stv<T, W>(out + o0, res);
        return;
    }
    if (part == 1) {
        if (t >= cs.n_xe) return;
        const unsigned r = cs.gx.div(t);
        const unsigned e = t - r * cs.gx.d;
        g = e < (unsigned)cs.g_lo ? (int)e : cs.g_hi + 1 + (int)(e - cs.g_lo);
        const unsigned kk = cs.yin.div(r);
        k = 1 + (int)kk;
        j = 1 + (int)(r - kk * cs.yin.d);
    } else {
        if (t >= cs.n_face) return;
        const unsigned r = cs.g.div(t);
        g = (int)(t - r * cs.g.d);
        shell_row(r, L.ny, cs.b, j, k);
    }
    // the shell: each cell of the group through the general row evaluation
    const int q = (j + k + c) & 1;
    const int o0 = W * g + L.P * (j + L.ny * k);
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = 2 * (W * g + e) + q;
        T v = T(0);
        if (i < L.nx) {
            T diag, off;
            row_any<T>(op, L, u, i, j, k, diag, off);
            v = gs_value(__ldg(&f[o0 + e]), diag, off);
        }
        out[o0 + e] = v;
    }
}

// Residual r = f - A u of both colours on a uniform level (the outer
// residual of a solve), the interior groups without boundary code and the
// shell apart, grid-stride over each part; r optionally stored as R, the
// sums of r^2 and f^2 reduced as in k_residv.
// chunk ch (a block's worth of threads, in the interleaved order of
// split_chunk) of the split residual of both colours on a uniform level:
// r = f - A u stored as R when rout is set, the sums of r^2 and f^2 added to
// rr and ff
// ured (when set): the first red pass of a V-cycle from a zero state on the
// residual as right-hand side, ured = r / diag on the red cells (the diagonal
// of this operator, rounded to R), which the V-cycle then skips
template <class T, int W, class R, class Op = KOp<T>>
__device__ __forceinline__ void resid_split_chunk(const Lev& L, const Op& op, const CSplit<T>& u,
                                                  const T* __restrict__ f, R* __restrict__ rout,
                                                  const ColourSplit& cs, unsigned ch, double& rr, double& ff,
                                                  R* __restrict__ ured = nullptr)
{
    auto group = [&](int j, int k, int g, auto in) {
        constexpr bool IN = decltype(in)::value;
        const int row = j + L.ny * k;
        const int h0 = W * g;
        const int o0 = h0 + L.P * row;
        for (int cc = 0; cc <= 1; cc++) {
            const int q = (j + k + cc) & 1;
            VecW<T, W> diag, off;
            if constexpr (std::is_same<Op, KOp<T>>::value) {
                group_rows<T, W, CSplit<T>, true, IN>(L, op, cc, u, row, j, k, h0, q, o0, diag, off);
            } else if constexpr (IN) {
                rop_group<T, W, CSplit<T>>(L, op, cc, u, row, h0, q, o0, diag, off);
            } else {  // explicit rows near the boundary: cell by cell
#pragma unroll
                for (int e = 0; e < W; e++) {
                    const int i = 2 * (h0 + e) + q;
                    diag.v[e] = T(0);
                    off.v[e] = T(0);
                    if (i < L.nx) row_any<T>(op, L, u, i, j, k, diag.v[e], off.v[e]);
                }
            }
            const VecW<T, W> f4 = ldv<T, W>(f + (cc ? L.half : 0) + o0);
            const VecW<T, W> u4 = ldv<T, W>(u.half(cc) + o0);
            VecW<R, W> r4, z4;
#pragma unroll
            for (int e = 0; e < W; e++) {
                const T r = f4.v[e] - (diag.v[e] * u4.v[e] + off.v[e]);
                const bool ok = IN || 2 * (h0 + e) + q < L.nx;
                r4.v[e] = ok ? (R)r : R(0);
                z4.v[e] = ok ? gs_value(r4.v[e], (R)diag.v[e], R(0)) : R(0);
                if (ok) {
                    rr += (double)r * (double)r;
                    ff += (double)f4.v[e] * (double)f4.v[e];
                }
            }
            if (rout) stv<R, W>(rout + (cc ? L.half : 0) + o0, r4);
            if (ured && cc == 0) stv<R, W>(ured + o0, z4);
        }
    };
    int part;
    unsigned idx;
    split_chunk(cs.nb_in, cs.nb_xe, ch, part, idx);
    const unsigned t = idx * TPB + threadIdx.x;
    if (part == 0) {
        if (t >= cs.n_in) return;
        const unsigned r = cs.gin.div(t);
        const int g = cs.g_lo + (int)(t - r * cs.gin.d);
        const unsigned kk = cs.yin.div(r);
        group(1 + (int)(r - kk * cs.yin.d), 1 + (int)kk, g, std::true_type());
        return;
    }
    int j, k, g;
    if (part == 1) {
        if (t >= cs.n_xe) return;
        const unsigned r = cs.gx.div(t);
        const unsigned e = t - r * cs.gx.d;
        g = e < (unsigned)cs.g_lo ? (int)e : cs.g_hi + 1 + (int)(e - cs.g_lo);
        const unsigned kk = cs.yin.div(r);
        k = 1 + (int)kk;
        j = 1 + (int)(r - kk * cs.yin.d);
    } else {
        if (t >= cs.n_face) return;
        const unsigned r = cs.g.div(t);
        g = (int)(t - r * cs.g.d);
        shell_row(r, L.ny, cs.b, j, k);
    }
    group(j, k, g, std::false_type());
}

template <class T, int W, class R, class Op = KOp<T>>
__global__ void __launch_bounds__(TPB, ResidShape<T>::MINB) k_residv_split(Lev L, Op op, CSplit<T> u,
                                                                           const T* __restrict__ f,
                                                                           R* __restrict__ rout, RedBuf rb,
                                                                           ColourSplit cs, R* __restrict__ ured)
{
    pdl_wait();
    __shared__ double sh[32];
    double rr = 0.0, ff = 0.0;
    // block-sized chunks, grid-stride, in the interleaved order of split_chunk
    const unsigned nchunks = cs.nb_in + cs.nb_xe + cs.nb_face;
    for (unsigned ch = blockIdx.x; ch < nchunks; ch += gridDim.x)
        resid_split_chunk<T, W, R, Op>(L, op, u, f, rout, cs, ch, rr, ff, ured);
    const double a = block_sum(rr, sh);
    const double b = block_sum(ff, sh);
    if (!rb.partial) return;
    // finish: last block sums the partials in block order
    __shared__ bool last;
    if (threadIdx.x == 0) {
        rb.partial[2 * blockIdx.x] = a;
        rb.partial[2 * blockIdx.x + 1] = b;
        __threadfence();
        last = (atomicAdd(rb.counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double sa = 0.0, sb = 0.0;
    for (unsigned qd = threadIdx.x; qd < gridDim.x; qd += blockDim.x) {
        sa += ((volatile double*)rb.partial)[2 * qd];
        sb += ((volatile double*)rb.partial)[2 * qd + 1];
    }
    sa = block_sum(sa, sh);
    sb = block_sum(sb, sh);
    if (threadIdx.x == 0) {
        rb.out[0] = sa;
        rb.out[1] = sb;
        *rb.counter = 0u;
    }
}

// ---------------------------------------------------------------------
// exact coarsest solve: u = A^{-1} f with the inverse precomputed (column
// major, FP64).  Replaces bottomsolve's full-dimension GMRES
// (mgridsteps.f90:218-382), which is an exact solve as well.  One CTA.
// ---------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void coarse_solve_body(const Lev& C, const double* __restrict__ AinvT,
                                                  const CSplit<T>& f, const Split<T>& u, double* fs)
{
    const int n = C.nx * C.ny * C.nz;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        int i = r % C.nx, j = (r / C.nx) % C.ny, k = r / (C.nx * C.ny);
        fs[r] = (double)f.get(C, i, j, k);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        double acc = 0.0;
        for (int q = 0; q < n; q++) acc += AinvT[(long long)q * n + r] * fs[q];
        int i = r % C.nx, j = (r / C.nx) % C.ny, k = r / (C.nx * C.ny);
        u.half(scol(i, j, k))[soff(C, i, j, k)] = (T)acc;
    }
}

template <class T>
__global__ void __launch_bounds__(512) k_coarse_solve(Lev C, const double* __restrict__ AinvT, CSplit<T> f,
                                                      Split<T> u)
{
    pdl_wait();
    extern __shared__ double fs[];
    coarse_solve_body<T>(C, AinvT, f, u, fs);
}

// dense assembly of the coarsest operator (row major, FP64, pre-zeroed)
template <class T>
__device__ __forceinline__ void dense_row(const KOp<T>& op, const Lev& L, int i, int j, int k, double* A, int n)
{
    const int r = i + L.nx * (j + L.ny * k);
    const double kc = (double)kval(op, L, i, j, k);
    double d = op.dex[0] ? (double)sel(op.dex, scol(i, j, k))[soff(L, i, j, k)] : (double)op.dexc;
    for (int ax = 0; ax < 3; ax++)
        for (int s = -1; s <= 1; s += 2) {
            int a = i, b = j, c = k;
            const int p = ax == 0 ? i : (ax == 1 ? j : k);
            if (nbr(L, ax, s, a, b, c)) {
                const int q = ax == 0 ? a : (ax == 1 ? b : c);
                double w = 0.5 * (kc + (double)kval(op, L, a, b, c)) * fcoef(L, ax, p, q);
                d += w;
                A[(long long)r * n + (a + L.nx * (b + L.ny * c))] -= w;
            } else if (L.bc[2 * ax + (s > 0)] == BC_DIRC) {
                d += kc * dcoef(L, ax, p);
            }
        }
    A[(long long)r * n + r] += d;
}
template <class T>
__device__ __forceinline__ void dense_row(const ROp<T>& op, const Lev& L, int i, int j, int k, double* A, int n)
{
    const int r = i + L.nx * (j + L.ny * k);
    const int c0 = scol(i, j, k);
    const long long o0 = soff(L, i, j, k);
    A[(long long)r * n + r] += (double)sel(op.r[0], c0)[o0];
    for (int ax = 0; ax < 3; ax++)
        for (int s = -1; s <= 1; s += 2) {
            int a = i, b = j, c = k;
            if (nbr(L, ax, s, a, b, c))
                A[(long long)r * n + (a + L.nx * (b + L.ny * c))] += (double)sel(op.r[1 + 2 * ax + (s > 0)], c0)[o0];
        }
}
template <class T, class Op>
__global__ void k_dense_assemble(Lev L, Op op, double* A)
{
    pdl_wait();
    const int n = L.nx * L.ny * L.nz;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        int i = r % L.nx, j = (r / L.nx) % L.ny, k = r / (L.nx * L.ny);
        dense_row(op, L, i, j, k, A, n);
    }
}

// Gauss-Jordan inverse with partial pivoting of the n x n row-major A held in
// M = [A | I] (n x 2n, row major, prepared by k_gj_prepare); writes the
// inverse column-major to AinvT.  One CTA; status[0] |= 1 on a zero pivot.
// smem=1: the augmented matrix is staged in dynamic shared memory (small n).
// gj (per hierarchy): gj[2] = 0 when k_dense_same found the matrix equal to
// the one whose inverse AinvT already holds -- both kernels then return at
// once and status[0] takes the saved flag gj[0]; after an inversion gj[0]
// keeps its flag and gj[3] = 1 marks AinvT valid.
__global__ void __launch_bounds__(1024) k_gauss_jordan(int n, double* M, double* AinvT, int* status, int smem,
                                                       int* gj);
__global__ void k_gj_prepare(int n, const double* A, double* M, const int* gj);
// one CTA: gj[2] = 1 when A differs from prev (bit for bit) or no inverse
// was computed yet, and then prev = A
__global__ void __launch_bounds__(1024) k_dense_same(int n, const double* A, double* prev, int* gj);

// ---------------------------------------------------------------------
// residual + norm: r = f - A u; sum r^2 (and sum f^2) reduced
// deterministically (per-block partials, the last block sums them in
// block order).  Optionally writes r (converted to R) to a split field.
// ---------------------------------------------------------------------
__device__ __forceinline__ void finish_two(RedBuf rb, double a, double b, double* sh)
{
    __shared__ bool last;
    if (threadIdx.x == 0) {
        rb.partial[2 * blockIdx.x] = a;
        rb.partial[2 * blockIdx.x + 1] = b;
        __threadfence();
        unsigned prev = atomicAdd(rb.counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double sa = 0.0, sb = 0.0;
    for (unsigned q = threadIdx.x; q < gridDim.x; q += blockDim.x) {
        sa += ((volatile double*)rb.partial)[2 * q];
        sb += ((volatile double*)rb.partial)[2 * q + 1];
    }
    sa = block_sum(sa, sh);
    sb = block_sum(sb, sh);
    if (threadIdx.x == 0) {
        rb.out[0] = sa;
        rb.out[1] = sb;
        *rb.counter = 0u;
    }
}

template <class T, class Op, class R>
__global__ void __launch_bounds__(TPB) k_resid_norm(Lev L, Op op, CSplit<T> u, CSplit<T> f, Split<R> rout,
                                                    RedBuf rb)
{
    pdl_wait();
    __shared__ double sh[32];
    double rr = 0.0, ff = 0.0;
    const unsigned total = (unsigned)L.P * L.rows;
    for (int c = 0; c < 2; c++) {
        unsigned t = blockIdx.x * TPB + threadIdx.x;
        int i, j, k;
        if (t < total && decode(L, t, c, i, j, k)) {
            T diag, off;
            row_any<T>(op, L, u, i, j, k, diag, off);
            T fv = __ldg(&f.half(c)[t]);
            T r = fv - (diag * __ldg(&u.half(c)[t]) + off);
            rr += (double)r * (double)r;
            ff += (double)fv * (double)fv;
            if (rout.c[0]) rout.half(c)[t] = (R)r;
        }
    }
    double a = block_sum(rr, sh);
    double b = block_sum(ff, sh);
    finish_two(rb, a, b, sh);
}

// out = A u (FP64 out, u of any precision), split layout
template <class T, class Op, class Tu>
__global__ void __launch_bounds__(TPB) k_apply(Lev L, Op op, CSplit<Tu> u, Split<double> out)
{
    pdl_wait();
    const unsigned total = (unsigned)L.P * L.rows;
    unsigned t = blockIdx.x * TPB + threadIdx.x;
    if (t >= total) return;
    for (int c = 0; c < 2; c++) {
        int i, j, k;
        if (decode(L, t, c, i, j, k)) {
            T diag, off;
            row_eval(op, L, u, i, j, k, diag, off);
            out.half(c)[t] = (double)(diag * (T)__ldg(&u.half(c)[t]) + off);
        }
    }
}

// ---------------------------------------------------------------------
// setup: ghosted Fortran-order FP64 <-> split layout
// ---------------------------------------------------------------------
template <class T>
__global__ void k_pack(Lev L, const double* __restrict__ g, Split<T> out, double scale, double shift)
{
    pdl_wait();
    unsigned t = blockIdx.x * TPB + threadIdx.x;
    const unsigned nx = L.nx, ny = L.ny;
    if (t >= nx * ny * (unsigned)L.nz) return;
    unsigned k = t / (nx * ny);
    unsigned rem = t - k * nx * ny;
    unsigned j = rem / nx;
    unsigned i = rem - j * nx;
    long long gi = (long long)(i + 1) + (long long)(nx + 2) * ((long long)(j + 1) + (long long)(ny + 2) * (k + 1));
    double v = g ? g[gi] * scale + shift : shift;
    out.half(scol(i, j, k))[soff(L, i, j, k)] = (T)v;
}

template <class T>
__global__ void k_unpack(Lev L, CSplit<T> in, double* __restrict__ g)
{
    pdl_wait();
    unsigned t = blockIdx.x * TPB + threadIdx.x;
    const unsigned nx = L.nx, ny = L.ny;
    if (t >= nx * ny * (unsigned)L.nz) return;
    unsigned k = t / (nx * ny);
    unsigned rem = t - k * nx * ny;
    unsigned j = rem / nx;
    unsigned i = rem - j * nx;
    long long gi = (long long)(i + 1) + (long long)(nx + 2) * ((long long)(j + 1) + (long long)(ny + 2) * (k + 1));
    g[gi] = (double)in.get(L, i, j, k);
}

// interior split -> natural (unghosted) FP64
template <class T>
__global__ void k_unpack_nat(Lev L, CSplit<T> in, double* __restrict__ g)
{
    pdl_wait();
    unsigned t = blockIdx.x * TPB + threadIdx.x;
    const unsigned nx = L.nx, ny = L.ny;
    if (t >= nx * ny * (unsigned)L.nz) return;
    unsigned k = t / (nx * ny);
    unsigned rem = t - k * nx * ny;
    unsigned j = rem / nx;
    unsigned i = rem - j * nx;
    g[t] = (double)in.get(L, i, j, k);
}

// max |x| over the interior of a ghosted field (x - x(1,1,1) when rel=1),
// reduced with an integer atomicMax on the bit pattern (valid for >= 0)
__global__ void k_maxabs(Lev L, const double* __restrict__ g, int rel, unsigned long long* out);
__global__ void k_maxabs_all(Lev L, const double* __restrict__ vel, const double* __restrict__ reac,
                             const double* __restrict__ dcoeff, const double* __restrict__ source,
                             const double* __restrict__ soln, unsigned long long* out);

// update_boundary_ghostvalues (discretepde.f90:1121-1267) + periodic wrap,
// on a ghosted FP64 field; faces only (edges/corners untouched, as in the
// reference)
__global__ void k_fill_ghosts(Lev L, double* __restrict__ g, const double* bl, const double* br, const double* bb,
                              const double* bt, const double* bk, const double* bf);

// find_bvec (discretepde.f90:382-618, applybcflag=.true.) + mgridsterm, split
// FP64 out.  flux=1 uses the half-cell Scharfetter-Gummel weights for DIRC.
__global__ void k_find_bvec(Lev L, const double* __restrict__ vel, const double* __restrict__ dcoeff,
                            const double* __restrict__ source, const double* bl, const double* br,
                            const double* bb, const double* bt, const double* bk, const double* bf,
                            const double* __restrict__ sterm, int flux, Split<double> b);

// aggregation average (volume weighted for the geometric hierarchy) of a
// split FP64 field onto the next coarser level
__global__ void k_restrict_field(Lev F, CSplit<double> in, Lev C, Split<double> out, int geom);

// rows of the upwind (find_AX) or Scharfetter-Gummel operator from split FP64
// cell fields of one level

// dex = -reac + dtinv, k cast, in split layout

// ---- flat vector kernels (length n, split arrays including zero pads) ----
__global__ void k_multidot(long long n, int m, const double* const* __restrict__ V, const double* __restrict__ w,
                           double* __restrict__ partial);
__global__ void k_multidot_finish(int m, int nblocks, const double* __restrict__ partial, double* __restrict__ h,
                                  int accumulate);
__global__ void k_multiaxpy(long long n, int m, const double* const* __restrict__ V, const double* __restrict__ h,
                            double* __restrict__ w);
__global__ void k_scale_to(long long n, const double* __restrict__ w, const double* __restrict__ hn, int idx,
                           double* __restrict__ v, float* __restrict__ v32);

template <class T>
__global__ void k_build_rows(Lev L, CSplit<double> vx, CSplit<double> vy, CSplit<double> vz, CSplit<double> kf,
                             CSplit<double> reac, int has_reac, double dtinv, int flux, ROp<T> out_rows)
{
    pdl_wait();
    unsigned t = blockIdx.x * TPB + threadIdx.x;
    const unsigned nx = L.nx, ny = L.ny;
    if (t >= nx * ny * (unsigned)L.nz) return;
    int k = t / (nx * ny);
    unsigned rem = t - k * nx * ny;
    int j = rem / nx;
    int i = rem - j * nx;
    const CSplit<double>* V[3] = {&vx, &vy, &vz};
    const double kc = kf.get(L, i, j, k);
    double d = 0.0;
    double co[6] = {0, 0, 0, 0, 0, 0};
    for (int ax = 0; ax < 3; ax++) {
        const int p = ax == 0 ? i : (ax == 1 ? j : k);
        const double wc = cwidth(L, ax, p);
        const double vc = V[ax]->get(L, i, j, k);
        // a face between cells of widths wa, wb: centre distance (wa+wb)/2, flux
        // per unit area F = wL*u_L + wR*u_R; row L gains +F/w_L, row R -F/w_R
        // minus face (neighbour is the left state)
        {
            int a = i, b = j, c = k;
            if (nbr(L, ax, -1, a, b, c)) {
                const int q = ax == 0 ? a : (ax == 1 ? b : c);
                const double wn = cwidth(L, ax, q), dd = 0.5 * (wc + wn);
                double wL, wR;
                const double vn = V[ax]->get(L, a, b, c), kn = kf.get(L, a, b, c);
                if (flux == 1) sg_face(vn, vc, kn, kc, dd, wL, wR);
                else upwind_face(vn, vc, kn, kc, dd, wL, wR);
                d -= wR * (1.0 / wc);
                co[2 * ax] = -wL * (1.0 / wc);
            } else {
                const int code = L.bc[2 * ax];
                if (code == BC_DIRC) {
                    if (flux == 1) { double wL, wR; sg_face(vc, vc, kc, kc, 0.5 * wc, wL, wR); d -= wR / wc; }
                    else { d += 2.0 * kc / (wc * wc); if (vc < 0.0) d -= vc / wc; }
                } else if (code == BC_ZGRD) {
                    d -= vc / wc;
                }
            }
        }
        // plus face (this cell is the left state)
        {
            int a = i, b = j, c = k;
            if (nbr(L, ax, 1, a, b, c)) {
                const int q = ax == 0 ? a : (ax == 1 ? b : c);
                const double wn = cwidth(L, ax, q), dd = 0.5 * (wc + wn);
                double wL, wR;
                const double vn = V[ax]->get(L, a, b, c), kn = kf.get(L, a, b, c);
                if (flux == 1) sg_face(vc, vn, kc, kn, dd, wL, wR);
                else upwind_face(vc, vn, kc, kn, dd, wL, wR);
                d += wL * (1.0 / wc);
                co[2 * ax + 1] = wR * (1.0 / wc);
            } else {
                const int code = L.bc[2 * ax + 1];
                if (code == BC_DIRC) {
                    if (flux == 1) { double wL, wR; sg_face(vc, vc, kc, kc, 0.5 * wc, wL, wR); d += wL / wc; }
                    else { d += 2.0 * kc / (wc * wc); if (vc > 0.0) d += vc / wc; }
                } else if (code == BC_ZGRD) {
                    d += vc / wc;
                }
            }
        }
    }
    d = d - (has_reac ? reac.get(L, i, j, k) : 0.0) + dtinv;
    const int cc = scol(i, j, k);
    const long long o = soff(L, i, j, k);
    ((T*)sel(out_rows.r[0], cc))[o] = (T)d;
    for (int q = 0; q < 6; q++) ((T*)sel(out_rows.r[1 + q], cc))[o] = (T)co[q];
}

template <class T>
__global__ void k_transpose_rows(Lev L, ROp<T> in, ROp<T> out)
{
    pdl_wait();
    unsigned t = blockIdx.x * TPB + threadIdx.x;
    const unsigned nx = L.nx, ny = L.ny;
    if (t >= nx * ny * (unsigned)L.nz) return;
    int k = t / (nx * ny);
    unsigned rem = t - k * nx * ny;
    int j = rem / nx;
    int i = rem - j * nx;
    const int cc = scol(i, j, k);
    const long long o = soff(L, i, j, k);
    ((T*)out.r[0][cc])[o] = in.r[0][cc][o];
    for (int ax = 0; ax < 3; ax++)
        for (int s = -1; s <= 1; s += 2) {
            // coefficient of u_{c+s} in row c of A^T = coefficient of u_c in row c+s of A
            int a = i, b = j, c = k;
            T v = T(0);
            if (nbr(L, ax, s, a, b, c)) {
                const int q = 1 + 2 * ax + (s > 0 ? 0 : 1);  // opposite direction of s
                v = in.r[q][scol(a, b, c)][soff(L, a, b, c)];
            }
            ((T*)out.r[1 + 2 * ax + (s > 0)][cc])[o] = v;
        }
}

template <class T>
__global__ void k_cast_field(long long n, const double* __restrict__ in, T* __restrict__ out, double scale,
                             double shift)
{
    pdl_wait();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        out[t] = (T)((in ? in[t] : 0.0) * scale + shift);
}

template <class A, class B>
__global__ void k_axpy(long long n, double a, const A* __restrict__ x, B* __restrict__ y)
{
    pdl_wait();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        y[t] = (B)((double)y[t] + a * (double)x[t]);
}

// y0 += a x0 and y1 += a x1 in one launch (both colour halves of a split
// field: the mixed solve's FP64 update x += e)
template <class A, class B>
__global__ void k_axpy2(long long n, double a, const A* __restrict__ x0, B* __restrict__ y0,
                        const A* __restrict__ x1, B* __restrict__ y1)
{
    pdl_wait();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 2 * n;
         t += (long long)gridDim.x * blockDim.x) {
        const bool h = t >= n;
        const long long e = h ? t - n : t;
        const A* x = h ? x1 : x0;
        B* y = h ? y1 : y0;
        y[e] = (B)((double)y[e] + a * (double)x[e]);
    }
}

}  // namespace mps
