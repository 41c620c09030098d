// mps_step.cu -- on-device operator assembly and the implicit plasma step.
//
// The reference assembles each equation's operator on the host before every
// solve: update_efield (plasma_pde/poissoneq.f90:565-680) differentiates the
// potential, eden_update_transport (plasma_pde/edeneq.f90:360-444) forms the
// drift vel = mu_e E, the diffusivity and the source (production plus
// n_old/dt), poisson_update_transport (plasma_pde/poissoneq.f90:335-385) the
// space-charge source.  Here those producers are kernels that write the
// solver's input fields in the reference's ghosted Fortran layout straight
// into device memory, so a time step moves no field across PCIe; and
// mps_plasma_step_dev chains them with the two solves (potential, then
// electrons) and the electron floor and ghost update of eden_solve
// (plasma_pde/edeneq.f90:446-525), the potential and electron parts of the
// time loop of plasma_pde/solve_manager.f90:363-502, behind one call.
//
// The electron mobility and diffusivity are fields supplied by the caller:
// the reference computes them per cell from its chemistry tables
// (getspecmobility / getspecdcoeff), which are not part of this library.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "../../include/mps_linsolve.h"
#include "mps_kernels.cuh"

namespace {

using namespace mps;

constexpr int STPB = 256;

unsigned nblocks(long long n) { return (unsigned)((n + STPB - 1) / STPB); }

// the level description k_fill_ghosts reads (sizes, periodic flags, codes)
Lev ghost_level(const mps_grid* g, const int bc[6])
{
    Lev L;
    std::memset(&L, 0, sizeof(L));
    L.nx = g->lx;
    L.ny = g->ly;
    L.nz = g->lz;
    for (int f = 0; f < 6; f++) L.bc[f] = bc[f];
    for (int a = 0; a < 3; a++) L.per[a] = bc[2 * a] == BC_PERI;
    return L;
}

bool bc_ok(const int bc[6])
{
    for (int f = 0; f < 6; f++)
        if (bc[f] < MPS_BC_DIRC || bc[f] > MPS_BC_DZGD) return false;
    for (int a = 0; a < 3; a++)
        if ((bc[2 * a] == MPS_BC_PERI) != (bc[2 * a + 1] == MPS_BC_PERI)) return false;
    return true;
}

bool grid_ok(const mps_grid* g)
{
    return g && g->lx >= 1 && g->ly >= 1 && g->lz >= 1 && g->llenx > 0 && g->lleny > 0 && g->llenz > 0;
}

struct Gh {  // ghosted Fortran-order indexing, (nx+2)(ny+2)(nz+2)
    int nx, ny, nz;
    long long sy, sz, n;
    __host__ __device__ Gh(int a, int b, int c)
        : nx(a), ny(b), nz(c), sy(a + 2), sz((long long)(a + 2) * (b + 2)), n((long long)(a + 2) * (b + 2) * (c + 2))
    {
    }
};

// minmodlimiter, plasma_pde/poissoneq.f90:549-563
__device__ __forceinline__ double minmod(double ntr, double dtr)
{
    if (dtr != 0.0) {
        const double r = ntr / dtr;
        return fmax(0.0, fmin(1.0, r));
    }
    return 1.0;
}

// E = -scale * grad(phi) by central differences of the ghosted potential
// (update_efield, poissoneq.f90:593-611, sign and scaling :667), optionally
// limited per direction by minmod (:614-662); one thread per ghosted cell,
// ghost cells written as zero (their values are set by the ghost pass)
__global__ void __launch_bounds__(STPB) k_efield(Gh G, const double* __restrict__ phi, double hx, double hy, double hz,
                                                 double scale, int limiter, double* __restrict__ ex,
                                                 double* __restrict__ ey, double* __restrict__ ez)
{
    const long long t = (long long)blockIdx.x * STPB + threadIdx.x;
    if (t >= G.n) return;
    const int i = (int)(t % G.sy);
    const long long r = t / G.sy;
    const int j = (int)(r % (G.ny + 2));
    const int k = (int)(r / (G.ny + 2));
    if (i < 1 || i > G.nx || j < 1 || j > G.ny || k < 1 || k > G.nz) {
        ex[t] = 0.0;
        ey[t] = 0.0;
        ez[t] = 0.0;
        return;
    }
    const double c = __ldg(&phi[t]);
    const double xm = __ldg(&phi[t - 1]), xp = __ldg(&phi[t + 1]);
    const double ym = __ldg(&phi[t - G.sy]), yp = __ldg(&phi[t + G.sy]);
    const double zm = __ldg(&phi[t - G.sz]), zp = __ldg(&phi[t + G.sz]);
    double gx = 0.5 * (xp - xm) / hx, gy = 0.5 * (yp - ym) / hy, gz = 0.5 * (zp - zm) / hz;
    if (limiter) {
        gx *= minmod(c - xm, xp - c);
        gy *= minmod(c - ym, yp - c);
        gz *= minmod(c - zm, zp - c);
    }
    ex[t] = -gx * scale;
    ey[t] = -gy * scale;
    ez[t] = -gz * scale;
}

// eden_update_transport (edeneq.f90:360-444) with the mobility and
// diffusivity as fields: vel = mu_e E * vel_scaling, dcoeff = D *
// dcoeff_scaling (D = |mu_e| Te when no D field is given: the Einstein
// relation with Te in volts), source = production * source_scaling (+
// n_old / dt with a time derivative, :441); ghosts zero (:397-400)
__global__ void __launch_bounds__(STPB) k_eden_transport(Gh G, const double* __restrict__ ex,
                                                         const double* __restrict__ ey, const double* __restrict__ ez,
                                                         const double* __restrict__ mu, const double* __restrict__ dco,
                                                         const double* __restrict__ te,
                                                         const double* __restrict__ prod,
                                                         const double* __restrict__ nold, double dtinv, double vs,
                                                         double ds, double ss, double* __restrict__ vx,
                                                         double* __restrict__ vy, double* __restrict__ vz,
                                                         double* __restrict__ dc, double* __restrict__ src)
{
    const long long t = (long long)blockIdx.x * STPB + threadIdx.x;
    if (t >= G.n) return;
    const int i = (int)(t % G.sy);
    const long long r = t / G.sy;
    const int j = (int)(r % (G.ny + 2));
    const int k = (int)(r / (G.ny + 2));
    if (i < 1 || i > G.nx || j < 1 || j > G.ny || k < 1 || k > G.nz) {
        vx[t] = 0.0;
        vy[t] = 0.0;
        vz[t] = 0.0;
        dc[t] = 0.0;
        src[t] = 0.0;
        return;
    }
    const double m = __ldg(&mu[t]);
    vx[t] = m * __ldg(&ex[t]) * vs;
    vy[t] = m * __ldg(&ey[t]) * vs;
    vz[t] = m * __ldg(&ez[t]) * vs;
    dc[t] = (dco ? __ldg(&dco[t]) : fabs(m) * __ldg(&te[t])) * ds;
    double s = prod ? __ldg(&prod[t]) * ss : 0.0;
    if (nold) s += __ldg(&nold[t]) * dtinv;
    src[t] = s;
}

// poisson_update_transport (poissoneq.f90:335-385): source = (sum_s q_s n_s -
// n_e) * scale (+ phi_old / dt with a time derivative, :382); ghosts zero
__global__ void __launch_bounds__(STPB) k_poisson_source(Gh G, const double* __restrict__ ne,
                                                         const double* __restrict__ nion, int nspec, long long sstride,
                                                         const double* __restrict__ charge, double scale,
                                                         const double* __restrict__ phiold, double dtinv,
                                                         double* __restrict__ src)
{
    const long long t = (long long)blockIdx.x * STPB + threadIdx.x;
    if (t >= G.n) return;
    const int i = (int)(t % G.sy);
    const long long r = t / G.sy;
    const int j = (int)(r % (G.ny + 2));
    const int k = (int)(r / (G.ny + 2));
    if (i < 1 || i > G.nx || j < 1 || j > G.ny || k < 1 || k > G.nz) {
        src[t] = 0.0;
        return;
    }
    double q = 0.0;
    for (int s = 0; s < nspec; s++) q += __ldg(&charge[s]) * __ldg(&nion[s * sstride + t]);
    double v = (q - __ldg(&ne[t])) * scale;
    if (phiold) v += __ldg(&phiold[t]) * dtinv;
    src[t] = v;
}

// the electron floor of eden_solve (edeneq.f90:505-514): interior n_e >= nemin
__global__ void __launch_bounds__(STPB) k_floor(Gh G, double* __restrict__ n, double nemin)
{
    const long long t = (long long)blockIdx.x * STPB + threadIdx.x;
    if (t >= G.n) return;
    const int i = (int)(t % G.sy);
    const long long r = t / G.sy;
    const int j = (int)(r % (G.ny + 2));
    const int k = (int)(r / (G.ny + 2));
    if (i < 1 || i > G.nx || j < 1 || j > G.ny || k < 1 || k > G.nz) return;
    if (n[t] < nemin) n[t] = nemin;
}

// ghosts of a ghosted field with the face rules of update_boundary_ghostvalues
// (the kernel of mps_fill_ghosts_dev); bcval may be NULL when no face is DIRC
void launch_ghosts(const mps_grid* g, const int bc[6], const double* const* bcval, double* f, cudaStream_t s)
{
    const Lev L = ghost_level(g, bc);
    const int mx = std::max(std::max(L.ny * L.nz, L.nx * L.nz), L.nx * L.ny);
    const double* b[6] = {};
    for (int q = 0; q < 6; q++) b[q] = bcval ? bcval[q] : nullptr;
    k_fill_ghosts<<<nblocks(mx), STPB, 0, s>>>(L, f, b[0], b[1], b[2], b[3], b[4], b[5]);
}

// E with the ghost rule of update_efield: every face copies its first
// interior value (efield_bc_codes = 'ZGRD', poissoneq.f90:582), periodic
// faces wrap
void launch_efield(const mps_grid* g, const int phi_bc[6], const double* phi, double scale, int limiter,
                   double* efield, cudaStream_t s)
{
    const Gh G(g->lx, g->ly, g->lz);
    double* ex = efield;
    double* ey = efield + G.n;
    double* ez = efield + 2 * G.n;
    k_efield<<<nblocks(G.n), STPB, 0, s>>>(G, phi, g->llenx / g->lx, g->lleny / g->ly, g->llenz / g->lz, scale,
                                           limiter, ex, ey, ez);
    int ebc[6];
    for (int f = 0; f < 6; f++) ebc[f] = phi_bc[f] == MPS_BC_PERI ? MPS_BC_PERI : MPS_BC_ZGRD;
    for (double* c : {ex, ey, ez}) launch_ghosts(g, ebc, nullptr, c, s);
}

}  // namespace

extern "C" {

int mps_efield_dev(const mps_grid* g, const int phi_bc[6], const double* const phi_bcval[6], double* phi,
                   double scale, int limiter, double* efield, void* stream)
{
    if (!grid_ok(g) || !phi_bc || !phi || !efield || !bc_ok(phi_bc)) return MPS_ERR_BAD_ARG;
    for (int f = 0; f < 6; f++)
        if (phi_bc[f] == MPS_BC_DIRC && !(phi_bcval && phi_bcval[f])) return MPS_ERR_BAD_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    launch_ghosts(g, phi_bc, phi_bcval, phi, s);  // update_boundary_ghostvalues(poissonsoln), :586-587
    launch_efield(g, phi_bc, phi, scale, limiter, efield, s);
    return cudaGetLastError() == cudaSuccess ? MPS_OK : MPS_ERR_CUDA;
}

int mps_eden_transport_dev(const mps_grid* g, const double* efield, const double* mu, const double* dco,
                           const double* te, const double* prod, const double* n_old, int timederiv, double dt,
                           const double scaling[3], double* vel, double* dcoeff, double* source, void* stream)
{
    if (!grid_ok(g) || !efield || !mu || !vel || !dcoeff || !source || (!dco && !te)) return MPS_ERR_BAD_ARG;
    if (timederiv && (!(dt > 0) || !n_old)) return MPS_ERR_BAD_ARG;
    const double vs = scaling ? scaling[0] : 1.0, ds = scaling ? scaling[1] : 1.0, ss = scaling ? scaling[2] : 1.0;
    const Gh G(g->lx, g->ly, g->lz);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_eden_transport<<<nblocks(G.n), STPB, 0, s>>>(G, efield, efield + G.n, efield + 2 * G.n, mu, dco, te, prod,
                                                   timederiv ? n_old : nullptr, timederiv ? 1.0 / dt : 0.0, vs, ds,
                                                   ss, vel, vel + G.n, vel + 2 * G.n, dcoeff, source);
    return cudaGetLastError() == cudaSuccess ? MPS_OK : MPS_ERR_CUDA;
}

int mps_poisson_source_dev(const mps_grid* g, const double* n_e, int nspec, const double* n_ion,
                           const double* charge, double scale, const double* phi_old, double dt, double* source,
                           void* stream)
{
    if (!grid_ok(g) || !n_e || !source || nspec < 0 || (nspec > 0 && (!n_ion || !charge))) return MPS_ERR_BAD_ARG;
    if (phi_old && !(dt > 0)) return MPS_ERR_BAD_ARG;
    const Gh G(g->lx, g->ly, g->lz);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_poisson_source<<<nblocks(G.n), STPB, 0, s>>>(G, n_e, n_ion, nspec, G.n, charge, scale, phi_old,
                                                   phi_old ? 1.0 / dt : 0.0, source);
    return cudaGetLastError() == cudaSuccess ? MPS_OK : MPS_ERR_CUDA;
}

int mps_plasma_step_dev(mps_handle hp, mps_handle he, const mps_plasma_step* S, const mps_solver_opts* opts_phi,
                        const mps_solver_opts* opts_e, mps_solve_info* info_phi, mps_solve_info* info_e,
                        void* stream)
{
    if (!hp || !he || !S) return MPS_ERR_BAD_ARG;
    const mps_grid* g = &S->g;
    if (!grid_ok(g) || !bc_ok(S->phi_bc) || !bc_ok(S->ne_bc) || !S->eps || !S->phi || !S->n_e || !S->mu_e ||
        (!S->d_e && !S->te) || !S->efield || !S->vel || !S->dcoeff || !S->source || !S->phi_source ||
        !(S->dt > 0))
        return MPS_ERR_BAD_ARG;
    for (int f = 0; f < 6; f++)
        if ((S->ne_bc[f] == MPS_BC_DIRC || S->ne_bc[f] == MPS_BC_FLUX) && !S->ne_bcval[f]) return MPS_ERR_BAD_ARG;
    // every piece runs on one stream: the kernels here on it, the solves
    // ordered with it (NULL = the legacy default stream, for both)
    if (!stream) stream = (void*)cudaStreamLegacy;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    mps_solve_info ip, ie;
    std::memset(&ip, 0, sizeof(ip));
    std::memset(&ie, 0, sizeof(ie));
    // 1. potential: space-charge source (poisson_update_transport), solve (poisson_solve)
    int st = mps_poisson_source_dev(g, S->n_e, S->nion, S->n_ion, S->ion_charge, S->rho_scale, nullptr, 1.0,
                                    S->phi_source, stream);
    if (st) return st;
    st = mps_linsolve_dev(hp, g, 0, 1.0, nullptr, S->eps, nullptr, S->phi_source, S->phi_bc, S->phi_bcval, nullptr,
                          S->phi, opts_phi, &ip, stream);
    if (info_phi) *info_phi = ip;
    if (st && st != MPS_ERR_NOT_CONVERGED) return st;
    // 2. E field (update_efield) and the electron operator (eden_update_transport)
    const int st2 = mps_efield_dev(g, S->phi_bc, S->phi_bcval, S->phi, S->efield_scale, S->limiter, S->efield,
                                   stream);
    if (st2) return st2;
    const double sc[3] = {S->vel_scaling, S->dcoeff_scaling, S->source_scaling};
    const int st3 = mps_eden_transport_dev(g, S->efield, S->mu_e, S->d_e, S->te, S->prod_e, S->n_e, 1, S->dt, sc,
                                           S->vel, S->dcoeff, S->source, stream);
    if (st3) return st3;
    // 3. implicit electron step from n_old (eden_solve), floor and ghosts
    const int st4 = mps_linsolve_dev(he, g, 1, S->dt, S->vel, S->dcoeff, nullptr, S->source, S->ne_bc, S->ne_bcval,
                                     nullptr, S->n_e, opts_e, &ie, stream);
    if (info_e) *info_e = ie;
    if (st4 && st4 != MPS_ERR_NOT_CONVERGED) return st4;
    const Gh G(g->lx, g->ly, g->lz);
    k_floor<<<nblocks(G.n), STPB, 0, s>>>(G, S->n_e, S->nemin);
    launch_ghosts(g, S->ne_bc, S->ne_bcval, S->n_e, s);
    if (cudaGetLastError() != cudaSuccess) return MPS_ERR_CUDA;
    return st ? st : st4;
}

}  // extern "C"
