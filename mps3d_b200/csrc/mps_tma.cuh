// mps_tma.cuh -- the finest level's red-black colour pass with its rows
// staged in shared memory by the Tensor Memory Accelerator.
//
// The register-fed colour pass (k_colourv_split) is bound by issue and
// latency together: every neighbour vector is a load instruction whose
// destination registers stay reserved until the data arrive, and 64
// registers per thread limit the loads a thread keeps in flight.  Here one
// thread of each block issues bulk tensor copies (cp.async.bulk.tensor) of
// whole x-rows into shared memory, so the bytes in flight cost no
// registers and no per-element instructions, and the arithmetic reads its
// operands from shared memory.
//
// Decomposition: a block owns TJ interior rows (j0 .. j0+TJ-1) of a chunk of
// interior planes (k = kb .. ke) and marches along z.  Plane p in shared
// memory holds, for the pass's colour c and the other colour oc:
//   U  : u[oc] rows j0-1 .. j0+TJ    (TJ+2 rows: the y neighbours)
//   Ko : k[oc] rows j0-1 .. j0+TJ    (the neighbours' coefficients)
//   Kc : k[c]  rows j0 .. j0+TJ-1    (the cells' own coefficients)
//   F  : f[c]  rows j0 .. j0+TJ-1
// Computing plane k reads planes k-1, k, k+1 (the z neighbours); TMA_SLOTS
// plane slots rotate: planes k+2 .. arrive while plane k is computed, and
// the slot of plane k-1 takes the next plane once every warp is done with
// plane k.
// Each slot has an mbarrier that the copies complete (expect_tx with the
// slot's byte count); the waits are bounded and a block that gives up
// records the failure in a device word the host reads with the residual
// norms, and returns.
//
// The arithmetic is that of group_rows / row_finish for interior groups (IN:
// six in-grid neighbours; the interior of a level with merged last cells
// stops one cell short of them, so its faces are the regular ones): W
// cells of one row per thread, faces y-, y+, z-, z+ then x, the same
// operation order.  Blocks past the tiles run the shell of the pass (the
// x-end groups of the interior rows and the rows on the y/z faces) with the
// general row evaluation, as k_colourv_split does.  The copies read only
// this GPU's own memory and use no cluster multicast.
#pragma once

#include <cuda.h>

#include "mps_kernels.cuh"

namespace mps {

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes)
                 : "memory");
}
// wait for phase `parity` of the barrier; false once `limit` tries found it
// incomplete (each try suspends the thread for a bounded time)
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity, unsigned limit)
{
    const unsigned a = smem_addr(b);
    for (unsigned it = 0; it < limit; it++) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// one box of a 3-D tensor map into shared memory, completing on `bar`
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, int x, int y, int z,
                                            unsigned long long* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<unsigned long long>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// shared-memory vector of W elements at a 16-byte aligned address
template <class T, int W>
__device__ __forceinline__ VecW<T, W> lds(const T* p)
{
    VecW<T, W> r;
    if constexpr (sizeof(T) == 4) {
        static_assert(W % 4 == 0, "FP32 groups of 4");
#pragma unroll
        for (int e = 0; e < W; e += 4) {
            const float4 a = *reinterpret_cast<const float4*>(p + e);
            r.v[e] = a.x; r.v[e + 1] = a.y; r.v[e + 2] = a.z; r.v[e + 3] = a.w;
        }
    } else {
        static_assert(W % 2 == 0, "FP64 groups of 2");
#pragma unroll
        for (int e = 0; e < W; e += 2) {
            const double2 a = *reinterpret_cast<const double2*>(p + e);
            r.v[e] = a.x; r.v[e + 1] = a.y;
        }
    }
    return r;
}

// The diagonal and the off-diagonal sum of one group (W cells of one row) of
// an interior row from staged rows: U0 the other colour's row of the cells,
// Uym/Uyp/Uzm/Uzp its y and z neighbour rows, K* the other colour's
// coefficients on the same rows, Kc the cells' own coefficients.  Faces y-,
// y+, z-, z+ then x, the operation order of group_rows / row_finish for
// interior groups.
template <class T, int W, bool KF>
__device__ __forceinline__ void tile_rows(const KOp<T>& op, const T* U0, const T* Uym, const T* Uyp, const T* Uzm,
                                          const T* Uzp, const T* K0, const T* Kym, const T* Kyp, const T* Kzm,
                                          const T* Kzp, const T* Kc, int h0, int q, T cr0, T cr1, T cr2,
                                          VecW<T, W>& diag, VecW<T, W>& off)
{
    const VecW<T, W> kc4 = KF ? lds<T, W>(Kc + h0) : zerov<T, W>();
    VecW<T, W> acc = zerov<T, W>(), wsum = zerov<T, W>();
    auto face = [&](const T* Ur, const T* Kr, T cf) {
        const VecW<T, W> un = lds<T, W>(Ur + h0);
        if (KF) {
            const VecW<T, W> kn = lds<T, W>(Kr + h0);
#pragma unroll
            for (int e = 0; e < W; e++) {
                const T wt = (kc4.v[e] + kn.v[e]) * cf;
                wsum.v[e] += wt;
                acc.v[e] += wt * un.v[e];
            }
        } else {
#pragma unroll
            for (int e = 0; e < W; e++) {
                wsum.v[e] += cf;
                acc.v[e] += cf * un.v[e];
            }
        }
    };
    face(Uym, Kym, cr1);
    face(Uyp, Kyp, cr1);
    face(Uzm, Kzm, cr2);
    face(Uzp, Kzp, cr2);
    const VecW<T, W> ax = lds<T, W>(U0 + h0);
    const VecW<T, W> akx = KF ? lds<T, W>(K0 + h0) : zerov<T, W>();
    const int so = q ? h0 + W : h0 - 1;
    const T sx = U0[so];
    const T skx = KF ? K0[so] : T(0);
#pragma unroll
    for (int e = 0; e < W; e++) {
        T uxm, kxm, uxp, kxp;
        if (q) {
            uxm = ax.v[e]; kxm = akx.v[e];
            uxp = e < W - 1 ? ax.v[e + 1] : sx; kxp = e < W - 1 ? akx.v[e + 1] : skx;
        } else {
            uxm = e > 0 ? ax.v[e - 1] : sx; kxm = e > 0 ? akx.v[e - 1] : skx;
            uxp = ax.v[e]; kxp = akx.v[e];
        }
        const T kc = KF ? kc4.v[e] : op.kc;
        const T d0 = op.dexc;
        T w0, w1;
        if (KF) { w0 = (kc + kxm) * cr0; w1 = (kc + kxp) * cr0; }
        else { w0 = cr0; w1 = cr0; }
        const T ws = wsum.v[e] + (w0 + w1);
        const T ac = acc.v[e] + (w0 * uxm + w1 * uxp);
        if (KF) { diag.v[e] = d0 + T(0.5) * ws; off.v[e] = T(-0.5) * ac; }
        else { diag.v[e] = d0 + kc * ws; off.v[e] = -kc * ac; }
    }
}

// the launch description of k_colour_tma
struct TmaColour {
    int njb, nkb, tk;     // row blocks, plane chunks, planes per chunk
    int ntile;            // njb * nkb blocks of interior tiles
    int g_lo, g_hi;       // interior groups of a row
    int jhi, khi;         // interior rows 1 .. jhi, planes 1 .. khi (the split's interior box)
    unsigned n_xe;        // shell threads: x ends of the interior rows
    unsigned n_face;      // shell threads: rows on the y/z faces
    unsigned nb_shell;    // blocks of the shell part
    unsigned tile_elems;  // elements of one slot's halo tile (U, Ko), 128-byte padded
    unsigned own_elems;   // of one own tile (Kc, F), 128-byte padded
    unsigned slot_bytes;  // bytes the copies of one plane deliver
    double* flag;         // set to 1.0 when a wait gives up
};

// plane slots of a block: three planes under computation plus the copies in
// flight (TMA_SLOTS - 3 planes ahead)
#ifndef MPS_TMA_SLOTS
#define MPS_TMA_SLOTS 4
#endif
constexpr int TMA_SLOTS = MPS_TMA_SLOTS;
constexpr unsigned TMA_WAIT_LIMIT = 1u << 20;

// shared memory of one block: the slots of (U, Ko, Kc, F) plus the barriers
template <class T, bool KF>
__host__ __device__ inline size_t tma_smem_bytes(const TmaColour& tc)
{
    const size_t per = (size_t)tc.tile_elems * (KF ? 2 : 1) + (size_t)tc.own_elems * (KF ? 2 : 1);
    return TMA_SLOTS * per * sizeof(T) + TMA_SLOTS * sizeof(unsigned long long);
}

template <class T, int W, int TJ, bool KF, bool UNI = true>
__global__ void __launch_bounds__(TJ * 32) k_colour_tma(Lev L, KOp<T> op, int c, CSplit<T> u, T* __restrict__ out,
                                                        const T* __restrict__ f, ColourSplit cs, TmaColour tc,
                                                        const __grid_constant__ CUtensorMap tmU,
                                                        const __grid_constant__ CUtensorMap tmKo,
                                                        const __grid_constant__ CUtensorMap tmKc,
                                                        const __grid_constant__ CUtensorMap tmF)
{
    extern __shared__ __align__(128) unsigned char smem[];
    pdl_wait();
    if (blockIdx.x >= (unsigned)tc.ntile) {
        // the shell: x-end groups of the interior rows, then the face rows
        const unsigned nsh = tc.n_xe + tc.n_face;
        for (unsigned t = (blockIdx.x - tc.ntile) * blockDim.x + threadIdx.x; t < nsh;
             t += tc.nb_shell * blockDim.x) {
            int j, k, g;
            if (t < tc.n_xe) {
                const unsigned r = cs.gx.div(t);
                const unsigned e = t - r * cs.gx.d;
                g = e < (unsigned)cs.g_lo ? (int)e : cs.g_hi + 1 + (int)(e - cs.g_lo);
                const unsigned kk = cs.yin.div(r);
                k = 1 + (int)kk;
                j = 1 + (int)(r - kk * cs.yin.d);
            } else {
                const unsigned tt = t - tc.n_xe;
                const unsigned r = cs.g.div(tt);
                g = (int)(tt - r * cs.g.d);
                shell_row(r, L.ny, cs.b, j, k);
            }
            const int h0 = W * g;
            const int row = j + L.ny * k;
            const int q = (j + k + c) & 1;
            const int o0 = h0 + L.P * row;
            const VecW<T, W> f4 = ldv<T, W>(f + o0);
            VecW<T, W> diag, off;
            group_rows<T, W, CSplit<T>, UNI, false>(L, op, c, u, row, j, k, h0, q, o0, diag, off);
            VecW<T, W> res;
#pragma unroll
            for (int e = 0; e < W; e++) {
                const int i = 2 * (h0 + e) + q;
                res.v[e] = i < L.nx ? gs_value(f4.v[e], diag.v[e], off.v[e]) : T(0);
            }
            stv<T, W>(out + o0, res);
        }
        return;
    }

    const int P = L.P;
    const int jb = (int)blockIdx.x % tc.njb, kb = (int)blockIdx.x / tc.njb;
    const int j0 = 1 + jb * TJ;
    const int k0 = 1 + kb * tc.tk;
    const int k1 = min(k0 + tc.tk - 1, tc.khi);
    T* S = reinterpret_cast<T*>(smem);
    const unsigned per = tc.tile_elems * (KF ? 2 : 1) + tc.own_elems * (KF ? 2 : 1);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem + TMA_SLOTS * per * sizeof(T));
    auto slot = [&](int p) { return (p - (k0 - 1)) % TMA_SLOTS; };
    auto slotU = [&](int p) { return S + (size_t)slot(p) * per; };
    auto slotKo = [&](int p) { return S + (size_t)slot(p) * per + tc.tile_elems; };
    auto slotKc = [&](int p) { return S + (size_t)slot(p) * per + (KF ? 2 : 1) * tc.tile_elems; };
    auto slotF = [&](int p) { return S + (size_t)slot(p) * per + (KF ? 2 : 1) * tc.tile_elems + (KF ? tc.own_elems : 0); };
    // the copies of plane p into its slot
    auto issue = [&](int p) {
        unsigned long long* b = bar + slot(p);
        mbar_expect_tx(b, tc.slot_bytes);
        tma_load_3d(slotU(p), &tmU, 0, j0 - 1, p, b);
        if (KF) {
            tma_load_3d(slotKo(p), &tmKo, 0, j0 - 1, p, b);
            tma_load_3d(slotKc(p), &tmKc, 0, j0, p, b);
        }
        tma_load_3d(slotF(p), &tmF, 0, j0, p, b);
    };
    if (threadIdx.x == 0) {
        for (int s = 0; s < TMA_SLOTS; s++) mbar_init(bar + s, 1);
        fence_mbar_init();
        fence_async_smem();
    }
    __syncthreads();
    const int last = k1 + 1;  // the last plane any computation reads
    if (threadIdx.x == 0)
        for (int p = k0 - 1; p <= min(k0 + TMA_SLOTS - 2, last); p++) issue(p);
    // plane p is the ((p - (k0 - 1)) / TMA_SLOTS)-th copy into its slot
    auto parity = [&](int p) { return (unsigned)(((p - (k0 - 1)) / TMA_SLOTS) & 1); };

    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j = j0 + w;
    const bool row_ok = j <= tc.jhi;
    const T cr0 = (T)L.cr[0], cr1 = (T)L.cr[1], cr2 = (T)L.cr[2];
    bool failed = false;
    for (int k = k0; k <= k1; k++) {
        bool ok = true;
        if (k == k0) ok = mbar_wait(bar + slot(k - 1), parity(k - 1), TMA_WAIT_LIMIT);
        if (k == k0) ok = ok && mbar_wait(bar + slot(k), parity(k), TMA_WAIT_LIMIT);
        ok = ok && mbar_wait(bar + slot(k + 1), parity(k + 1), TMA_WAIT_LIMIT);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        if (row_ok) {
            const T* U0 = slotU(k) + (w + 1) * P;
            const T* Uym = slotU(k) + w * P;
            const T* Uyp = slotU(k) + (w + 2) * P;
            const T* Uzm = slotU(k - 1) + (w + 1) * P;
            const T* Uzp = slotU(k + 1) + (w + 1) * P;
            const T* K0 = KF ? slotKo(k) + (w + 1) * P : nullptr;
            const T* Kym = KF ? slotKo(k) + w * P : nullptr;
            const T* Kyp = KF ? slotKo(k) + (w + 2) * P : nullptr;
            const T* Kzm = KF ? slotKo(k - 1) + (w + 1) * P : nullptr;
            const T* Kzp = KF ? slotKo(k + 1) + (w + 1) * P : nullptr;
            const T* Kc = KF ? slotKc(k) + w * P : nullptr;
            const T* Fr = slotF(k) + w * P;
            const int q = (j + k + c) & 1;
            T* orow = out + (size_t)P * (j + (size_t)L.ny * k);
            for (int g = tc.g_lo + lane; g <= tc.g_hi; g += 32) {
                const int h0 = W * g;
                VecW<T, W> diag, off;
                tile_rows<T, W, KF>(op, U0, Uym, Uyp, Uzm, Uzp, K0, Kym, Kyp, Kzm, Kzp, Kc, h0, q, cr0, cr1, cr2, diag,
                                    off);
                const VecW<T, W> f4 = lds<T, W>(Fr + h0);
                VecW<T, W> res;
#pragma unroll
                for (int e = 0; e < W; e++) res.v[e] = gs_value(f4.v[e], diag.v[e], off.v[e]);
                stv<T, W>(orow + h0, res);
            }
        }
        __syncthreads();  // every warp is done with plane k - 1
        if (threadIdx.x == 0 && k + TMA_SLOTS - 1 <= last) {
            fence_async_smem();
            issue(k + TMA_SLOTS - 1);  // into the slot of plane k - 1
        }
    }
    if (failed) {
        if (threadIdx.x == 0) *tc.flag = 1.0;
        // let copies still in flight land before the block's shared memory
        // is released (bounded, as every wait here)
        for (int p = max(k0 - 1, 0); p <= last; p++) mbar_wait(bar + slot(p), parity(p), 64);
    }
}

}  // namespace mps
