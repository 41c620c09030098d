// mps_operator_vjp_dev: gradients of s = lam^T A(vel, dcoeff, reac) u with
// respect to the operator's cell fields -- the operator part of the adjoint
// of a solve.  For x = A^{-1} b and a loss L(x), the adjoint solve gives
// lam = A^{-T} dL/dx (mps_linsolve_dev with opts->transpose) and then
// dL/dtheta = -d(lam^T A(theta) x)/dtheta, which this kernel evaluates.
//
// The reference has no adjoint (extension).  The forward operator is the one
// built by k_build_rows: per face (L, R) a flux F = wL u_L + wR u_R entering
// row L as +F/h and row R as -F/h, boundary faces and the diagonal adding
// lam_c u_c times their coefficient.  One thread per interior cell computes
// the derivative with respect to its own fields from its six faces, so no
// two threads write the same output.  Uniform grids (the finest level).
//
// Scharfetter-Gummel weights in Bernoulli form, B(x) = x / (e^x - 1):
// wL = (D/h) B(-Pe), wR = -(D/h) B(Pe), Pe = c h / D, c = (cL+cR)/2,
// D = 2 DL DR / (DL + DR + 1e-10) (mps1d/source/convdiff.f90:10-64), so
//   dwL/dc = -B'(-Pe), dwR/dc = -B'(Pe),
//   dwL/dD = (B(-Pe) + Pe B'(-Pe)) / h, dwR/dD = -(B(Pe) - Pe B'(Pe)) / h.
#include <cuda_runtime.h>

#include "../../include/mps_linsolve.h"
#include "mps_core.cuh"

namespace {

using namespace mps;

constexpr int VJP_TPB = 256;

// B(x) and B'(x): Taylor series near 0 (|x| < 1e-3, truncation below 1e-16),
// the exp(-x) form for large positive x, x / expm1(x) otherwise
__device__ __forceinline__ void bernoulli(double x, double& B, double& dB)
{
    if (fabs(x) < 1.0e-3) {
        const double x2 = x * x;
        B = 1.0 - 0.5 * x + x2 / 12.0 - x2 * x2 / 720.0;
        dB = -0.5 + x / 6.0 - x2 * x / 180.0;
    } else if (x > 50.0) {
        const double e = exp(-x);
        B = x * e;
        dB = (1.0 - x) * e;
    } else {
        const double em = expm1(x);
        B = x / em;
        dB = (em - x * (em + 1.0)) / (em * em);
    }
}

// derivatives of the SG face weights with respect to (cL, cR, DL, DR),
// following the branches of sg_face
__device__ __forceinline__ void sg_face_grad(double cL, double cR, double DL, double DR, double dx, double dwL[4],
                                             double dwR[4])
{
    const double eps = 1.0e-10;
    const double c = 0.5 * (cL + cR);
    const double S = DL + DR + eps;
    const double D = 2.0 * DL * DR / S;
    for (int q = 0; q < 4; q++) dwL[q] = dwR[q] = 0.0;
    if (fabs(D) < eps) {  // upwind limit
        const double sgn = c <= 0.0 ? -1.0 : 1.0;
        dwL[0] = 0.5 * (1.0 + sgn);
        dwR[1] = 0.5 * (1.0 - sgn);
        return;
    }
    const double Pe = c * dx / D;
    double wLc = 0.0, wRc = 0.0, wLD, wRD;
    if (fabs(Pe) < eps) {
        wLD = 1.0 / dx;
        wRD = -1.0 / dx;
    } else {
        double Bm, dBm, Bp, dBp;
        bernoulli(-Pe, Bm, dBm);
        bernoulli(Pe, Bp, dBp);
        wLc = -dBm;
        wRc = -dBp;
        wLD = (Bm + Pe * dBm) / dx;
        wRD = -(Bp - Pe * dBp) / dx;
    }
    const double dD_dL = 2.0 * DR * (DR + eps) / (S * S), dD_dR = 2.0 * DL * (DL + eps) / (S * S);
    dwL[0] = dwL[1] = 0.5 * wLc;
    dwR[0] = dwR[1] = 0.5 * wRc;
    dwL[2] = wLD * dD_dL;
    dwL[3] = wLD * dD_dR;
    dwR[2] = wRD * dD_dL;
    dwR[3] = wRD * dD_dR;
}

// upwind_face (findcellcontributions) derivatives: k_half = (kL+kR)/(2d),
// v_half = (vL+vR)/2 added to the upwind weight
__device__ __forceinline__ void upwind_face_grad(double vL, double vR, double d, double dwL[4], double dwR[4])
{
    const double vh = 0.5 * (vL + vR);
    dwL[0] = dwL[1] = vh > 0.0 ? 0.5 : 0.0;
    dwR[0] = dwR[1] = vh > 0.0 ? 0.0 : 0.5;
    dwL[2] = dwL[3] = 0.5 / d;
    dwR[2] = dwR[3] = -0.5 / d;
}

struct VjpArgs {
    int n[3];
    double h[3];
    int bc[6];
    int flux;
};

__global__ void __launch_bounds__(VJP_TPB) k_operator_vjp(VjpArgs a, const double* __restrict__ vel,
                                                          const double* __restrict__ dc,
                                                          const double* __restrict__ lam,
                                                          const double* __restrict__ u, double* __restrict__ gvel,
                                                          double* __restrict__ gd, double* __restrict__ greac)
{
    const long long nx = a.n[0], ny = a.n[1], nz = a.n[2];
    const long long ncell = nx * ny * nz;
    const long long t = (long long)blockIdx.x * VJP_TPB + threadIdx.x;
    if (t >= ncell) return;
    const int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / (nx * ny));
    const long long gx = nx + 2, gy = ny + 2, ng = gx * gy * (nz + 2);
    auto G = [&](int ii, int jj, int kk) { return (long long)(ii + 1) + gx * ((long long)(jj + 1) + gy * (kk + 1)); };
    auto I = [&](int ii, int jj, int kk) { return (long long)ii + nx * ((long long)jj + ny * kk); };
    const double lc = lam[t], uc = u[t], lu = lc * uc;
    const double kc = dc[G(i, j, k)];
    double gdc = 0.0;
    for (int ax = 0; ax < 3; ax++) {
        const double* v = vel ? vel + ax * ng : nullptr;
        const double vc = v ? v[G(i, j, k)] : 0.0;
        const int n = a.n[ax];
        const int pos = ax == 0 ? i : (ax == 1 ? j : k);
        const bool per = a.bc[2 * ax] == MPS_BC_PERI;
        const double h = a.h[ax];
        double gv = 0.0;
        for (int side = 0; side < 2; side++) {
            // neighbour across this side, if any (periodic wrap)
            int m = side == 0 ? pos - 1 : pos + 1;
            bool has = m >= 0 && m < n;
            if (!has && per) { m = side == 0 ? n - 1 : 0; has = true; }
            if (has) {
                int q[3] = {i, j, k};
                q[ax] = m;
                const double vm = v ? v[G(q[0], q[1], q[2])] : 0.0;
                const double km = dc[G(q[0], q[1], q[2])];
                const long long cm = I(q[0], q[1], q[2]);
                double dwL[4], dwR[4];
                if (side == 1) {  // this cell is the left state
                    if (a.flux == MPS_FLUX_SG) sg_face_grad(vc, vm, kc, km, h, dwL, dwR);
                    else upwind_face_grad(vc, vm, h, dwL, dwR);
                    const double mu = (lc - lam[cm]) / h;
                    gv += mu * (dwL[0] * uc + dwR[0] * u[cm]);
                    gdc += mu * (dwL[2] * uc + dwR[2] * u[cm]);
                } else {  // this cell is the right state
                    if (a.flux == MPS_FLUX_SG) sg_face_grad(vm, vc, km, kc, h, dwL, dwR);
                    else upwind_face_grad(vm, vc, h, dwL, dwR);
                    const double mu = (lam[cm] - lc) / h;
                    gv += mu * (dwL[1] * u[cm] + dwR[1] * uc);
                    gdc += mu * (dwL[3] * u[cm] + dwR[3] * uc);
                }
            } else {
                const int code = a.bc[2 * ax + side];
                if (code == MPS_BC_DIRC) {
                    if (a.flux == MPS_FLUX_SG) {
                        double dwL[4], dwR[4];
                        sg_face_grad(vc, vc, kc, kc, 0.5 * h, dwL, dwR);
                        if (side == 0) {
                            gv -= lu * (dwR[0] + dwR[1]) / h;
                            gdc -= lu * (dwR[2] + dwR[3]) / h;
                        } else {
                            gv += lu * (dwL[0] + dwL[1]) / h;
                            gdc += lu * (dwL[2] + dwL[3]) / h;
                        }
                    } else {
                        gdc += lu * 2.0 / (h * h);
                        if (side == 0 && vc < 0.0) gv -= lu / h;
                        if (side == 1 && vc > 0.0) gv += lu / h;
                    }
                } else if (code == MPS_BC_ZGRD) {
                    gv += side == 0 ? -lu / h : lu / h;
                }
            }
        }
        if (gvel) gvel[ax * ncell + t] = gv;
    }
    if (gd) gd[t] = gdc;
    if (greac) greac[t] = -lu;
}

}  // namespace

extern "C" int mps_operator_vjp_dev(const mps_grid* g, const double* vel, const double* dcoeff, const int bc_code[6],
                                    const double* lam, const double* u, const mps_solver_opts* opts, double* gvel,
                                    double* gdcoeff, double* greac, void* stream)
{
    if (!g || !dcoeff || !bc_code || !lam || !u) return MPS_ERR_BAD_ARG;
    if (g->lx < 1 || g->ly < 1 || g->lz < 1 || !(g->llenx > 0) || !(g->lleny > 0) || !(g->llenz > 0))
        return MPS_ERR_BAD_ARG;
    if ((long long)g->lx * g->ly * g->lz >= (1LL << 31)) return MPS_ERR_BAD_ARG;
    VjpArgs a;
    a.n[0] = g->lx; a.n[1] = g->ly; a.n[2] = g->lz;
    a.h[0] = g->llenx / g->lx; a.h[1] = g->lleny / g->ly; a.h[2] = g->llenz / g->lz;
    for (int f = 0; f < 6; f++) {
        if (bc_code[f] < MPS_BC_DIRC || bc_code[f] > MPS_BC_DZGD) return MPS_ERR_BAD_ARG;
        a.bc[f] = bc_code[f];
    }
    for (int ax = 0; ax < 3; ax++)
        if ((bc_code[2 * ax] == MPS_BC_PERI) != (bc_code[2 * ax + 1] == MPS_BC_PERI)) return MPS_ERR_BAD_ARG;
    a.flux = opts ? opts->flux : MPS_FLUX_UPWIND;
    if (a.flux != MPS_FLUX_UPWIND && a.flux != MPS_FLUX_SG) return MPS_ERR_BAD_ARG;
    const long long n = (long long)g->lx * g->ly * g->lz;
    k_operator_vjp<<<(unsigned)((n + VJP_TPB - 1) / VJP_TPB), VJP_TPB, 0, static_cast<cudaStream_t>(stream)>>>(
        a, vel, dcoeff, lam, u, gvel, gdcoeff, greac);
    if (cudaGetLastError() != cudaSuccess) return MPS_ERR_CUDA;
    return MPS_OK;
}
