// mps_apply_A_noalloc: A soln without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need
// the operator applied: a time-stepping code whose memory pool (its own, or
// torch's caching allocator) already holds the GPU's free HBM, where a
// cudaMalloc would fail or make the pool give memory back, and a code that
// keeps the device busy on its own streams, where cudaFree (which waits for
// the whole device) would stall every stream.  This entry point serves them:
// it takes no handle, owns no workspace and calls no cudaMalloc, cudaFree or
// allocating library routine.  Its scratch -- the split red/black copies of
// the coefficient fields, the seven operator rows and the split soln / AX --
// is one file-scope device array of MPS_NOALLOC_SCRATCH_BYTES (32 MiB).
// The CUDA runtime reserves it on a device when it loads this file's module
// there: with the default lazy module loading, at the first call on that
// device (the cudaGetSymbolAddress below), with CUDA_MODULE_LOADING=EAGER at
// context creation.  It stays reserved until the process exits, so every
// later call takes no device memory at all.
//
// The kernels are the ones the handle-based mps_apply_A_dev path uses for
// the row form of the operator (k_pack, k_build_rows, k_transpose_rows,
// k_apply, k_unpack_nat); only where their buffers live differs.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/mps_linsolve.h"
#include "mps_kernels.cuh"

namespace {

using namespace mps;

// 16 split arrays of at most MPS_NOALLOC_MAX_CELLS words each:
//   slots 0..6  : dcoeff, reac, vel x/y/z (then A^T rows when transposing)
//   slots 7..13 : the seven rows of A
//   slot 14     : soln (split)      slot 15 : A soln (split)
constexpr int kSlots = 16;
constexpr long long kSlotWords = MPS_NOALLOC_MAX_CELLS;
static_assert((long long)kSlots * kSlotWords * 8 == MPS_NOALLOC_SCRATCH_BYTES, "scratch size");

static __device__ __align__(256) double g_noalloc_scratch[kSlots * kSlotWords];

// Device address of g_noalloc_scratch per device.  In host code the name
// g_noalloc_scratch is only a handle for the runtime, not a device address;
// the address is looked up once per device, with that device current.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

int scratch_for_current_device(double** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MPS_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return MPS_ERR_CUDA;
        g_addr[dev] = static_cast<double*>(p);
    }
    *out = g_addr[dev];
    return MPS_OK;
}

// the finest (uniform) level's description, as the handle-based path builds it
Lev uniform_level(const mps_grid* g, const int bc[6])
{
    Lev L;
    std::memset(&L, 0, sizeof(L));
    L.nx = g->lx; L.ny = g->ly; L.nz = g->lz;
    L.nh = (L.nx + 1) / 2;
    L.P = ((L.nh + 7) / 8) * 8;
    L.half = (long long)L.P * L.ny * L.nz;
    for (int f = 0; f < 6; f++) L.bc[f] = bc[f];
    for (int a = 0; a < 3; a++) L.per[a] = bc[2 * a] == BC_PERI;
    const int n[3] = {L.nx, L.ny, L.nz};
    const double llen[3] = {g->llenx, g->lleny, g->llenz};
    for (int a = 0; a < 3; a++) {
        const double w = llen[a] / n[a];
        L.w[a] = L.wl[a] = w;
        L.cr[a] = 1.0 / (w * w);
        L.cl[a] = 1.0 / (w * w);
        L.cp[a] = 1.0 / (w * w);
        L.dr[a] = 2.0 / (w * w);
        L.dlast[a] = 2.0 / (w * w);
    }
    L.uniform = 1;
    L.divP.init((unsigned)L.P);
    L.divNy.init((unsigned)L.ny);
    L.divG.init((unsigned)(L.P / 4));
    L.rows = (unsigned)L.ny * (unsigned)L.nz;
    return L;
}

ROp<double> rows_at(double* base, const Lev& L)
{
    ROp<double> r;
    for (int q = 0; q < 7; q++) {
        r.r[q][0] = base + (size_t)q * kSlotWords;
        r.r[q][1] = base + (size_t)q * kSlotWords + L.half;
    }
    return r;
}

Split<double> split_at(double* base, const Lev& L)
{
    Split<double> s;
    s.c[0] = base;
    s.c[1] = base + L.half;
    return s;
}

CSplit<double> csplit_at(const double* base, const Lev& L)
{
    CSplit<double> s;
    s.c[0] = base;
    s.c[1] = base + L.half;
    return s;
}

unsigned blocks(long long n) { return (unsigned)((n + TPB - 1) / TPB); }

}  // namespace

extern "C" int mps_apply_A_noalloc(const mps_grid* g, int timederiv, double dt, const double* vel,
                                   const double* dcoeff, const double* reac, const int bc_code[6],
                                   const double* soln, double* AX, const mps_solver_opts* opts, void* stream)
{
    if (!g || !dcoeff || !soln || !AX || !bc_code) return MPS_ERR_BAD_ARG;
    if (g->lx < 1 || g->ly < 1 || g->lz < 1 || !(g->llenx > 0) || !(g->lleny > 0) || !(g->llenz > 0))
        return MPS_ERR_BAD_ARG;
    if (timederiv && !(dt > 0)) return MPS_ERR_BAD_ARG;
    for (int f = 0; f < 6; f++)
        if (bc_code[f] < MPS_BC_DIRC || bc_code[f] > MPS_BC_DZGD) return MPS_ERR_BAD_ARG;
    for (int a = 0; a < 3; a++)
        if ((bc_code[2 * a] == MPS_BC_PERI) != (bc_code[2 * a + 1] == MPS_BC_PERI)) return MPS_ERR_BAD_ARG;
    const int flux = opts ? opts->flux : MPS_FLUX_UPWIND;
    const int transpose = opts ? opts->transpose : 0;
    if (flux != MPS_FLUX_UPWIND && flux != MPS_FLUX_SG) return MPS_ERR_BAD_ARG;

    // the limit: each split array (x padded to a multiple of 16 cells) fits a slot
    const long long split_words = (long long)((g->lx + 15) / 16 * 16) * g->ly * g->lz;
    if (split_words > kSlotWords) return MPS_ERR_TOO_LARGE;

    double* S = nullptr;
    if (int st = scratch_for_current_device(&S)) return st;
    const Lev L = uniform_level(g, bc_code);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long ncell = (long long)L.nx * L.ny * L.nz;
    const long long ng = (long long)(L.nx + 2) * (L.ny + 2) * (L.nz + 2);
    double* slot[kSlots];
    for (int q = 0; q < kSlots; q++) slot[q] = S + (size_t)q * kSlotWords;
    auto sp = [&](int q) { return split_at(slot[q], L); };
    auto csp = [&](int q) { return csplit_at(slot[q], L); };

    // the split soln is the only array read outside the cells written in this
    // call (the padding past lx, at zero weight): clear it, so that nothing of
    // the previous call's contents can enter this one
    if (cudaMemsetAsync(slot[14], 0, sizeof(double) * 2 * L.half, s) != cudaSuccess) return MPS_ERR_CUDA;
    k_pack<double><<<blocks(ncell), TPB, 0, s>>>(L, dcoeff, sp(0), 1.0, 0.0);
    if (reac) k_pack<double><<<blocks(ncell), TPB, 0, s>>>(L, reac, sp(1), 1.0, 0.0);
    for (int a = 0; a < 3; a++)  // a missing vel is written as zeros
        k_pack<double><<<blocks(ncell), TPB, 0, s>>>(L, vel ? vel + a * ng : nullptr, sp(2 + a), 1.0, 0.0);
    k_pack<double><<<blocks(ncell), TPB, 0, s>>>(L, soln, sp(14), 1.0, 0.0);
    const double dtinv = timederiv ? 1.0 / dt : 0.0;
    const ROp<double> rowsA = rows_at(slot[7], L);
    k_build_rows<double><<<blocks(ncell), TPB, 0, s>>>(L, csp(2), csp(3), csp(4), csp(0), csp(1), reac != nullptr,
                                                       dtinv, flux, rowsA);
    ROp<double> rows = rowsA;
    if (transpose) {  // the fields in slots 0..6 are dead once the rows exist
        rows = rows_at(slot[0], L);
        k_transpose_rows<double><<<blocks(ncell), TPB, 0, s>>>(L, rowsA, rows);
    }
    k_apply<double, ROp<double>, double><<<blocks((long long)L.P * L.rows), TPB, 0, s>>>(L, rows, csp(14), sp(15));
    k_unpack_nat<double><<<blocks(ncell), TPB, 0, s>>>(L, csp(15), AX);
    if (cudaGetLastError() != cudaSuccess) return MPS_ERR_CUDA;
    return MPS_OK;
}
