// mps_kernels.cu -- non-inline kernels of the B200 solver (setup, dense
// coarse inverse, Krylov vector kernels).
#include "mps_kernels.cuh"

namespace mps {

// ---------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_dense_same(int n, const double* A, double* prev, int* gj)
{
    pdl_wait();
    const long long nn = (long long)n * n;
    int diff = 0;
    for (long long t = threadIdx.x; t < nn; t += blockDim.x)
        diff |= __double_as_longlong(A[t]) != __double_as_longlong(prev[t]);
    const int any = __syncthreads_or(diff) || gj[3] == 0;
    if (any)
        for (long long t = threadIdx.x; t < nn; t += blockDim.x) prev[t] = A[t];
    if (threadIdx.x == 0) gj[2] = any;
}

__global__ void k_gj_prepare(int n, const double* A, double* M, const int* gj)
{
    pdl_wait();
    if (gj[2] == 0) return;  // the inverse in AinvT is current
    const long long n2 = 2LL * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n2;
         t += (long long)gridDim.x * blockDim.x) {
        long long r = t / n2, c = t - r * n2;
        M[t] = c < n ? A[r * n + c] : (c - n == r ? 1.0 : 0.0);
    }
}

__global__ void __launch_bounds__(1024) k_gauss_jordan(int n, double* Mg, double* AinvT, int* status, int smem,
                                                       int* gj)
{
    pdl_wait();
    if (gj[2] == 0) {  // the inverse in AinvT is current: its singular flag again
        if (threadIdx.x == 0 && gj[0]) atomicOr(status, 1);
        return;
    }
    // 32 x 32 threads: lanes stride columns, warps stride rows
    extern __shared__ double Ms[];
    __shared__ double fac[1024];
    __shared__ unsigned char sing[1024];
    __shared__ int s_piv;
    __shared__ double s_scale;
    const int ld = 2 * n;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    double* M = smem ? Ms : Mg;
    if (smem)
        for (int t = tid; t < 2 * n * n; t += nt) Ms[t] = Mg[t];
    for (int r = tid; r < n; r += nt) sing[r] = 0;
    __syncthreads();
    // scale of the matrix for the singular-pivot threshold (warp 0)
    if (wid == 0) {
        double mx = 0.0;
        for (int r = 0; r < n; r++)
            for (int c = lane; c < n; c += 32) mx = fmax(mx, fabs(M[r * ld + c]));
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        if (lane == 0) s_scale = mx;
    }
    __syncthreads();
    const double tiny = 1e-13 * s_scale;
    for (int p = 0; p < n; p++) {
        // pivot: largest |M[r][p]|, r >= p (warp 0)
        if (wid == 0) {
            double best = -1.0;
            int bi = p;
            for (int r = p + lane; r < n; r += 32) {
                const double v = fabs(M[r * ld + p]);
                if (v > best) { best = v; bi = r; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, best, o);
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (lane == 0) {
                s_piv = best > tiny ? bi : -1;
                if (best <= tiny) { atomicOr(status, 1); sing[p] = 1; }
            }
        }
        __syncthreads();
        const int piv = s_piv;
        if (piv < 0) continue;  // singular direction: left for the zeroed inverse row
        if (piv != p)
            for (int c = tid; c < ld; c += nt) {
                const double a = M[p * ld + c];
                M[p * ld + c] = M[piv * ld + c];
                M[piv * ld + c] = a;
            }
        __syncthreads();
        const double inv = 1.0 / M[p * ld + p];
        for (int r = tid; r < n; r += nt) fac[r] = (r == p) ? 0.0 : M[r * ld + p];
        __syncthreads();
        for (int c = p + tid; c < ld; c += nt) M[p * ld + c] *= inv;
        __syncthreads();
        for (int r = wid; r < n; r += nw) {
            const double f = fac[r];
            if (f != 0.0)
                for (int c = p + lane; c < ld; c += 32) M[r * ld + c] -= f * M[p * ld + c];
        }
        __syncthreads();
    }
    for (int r = wid; r < n; r += nw)
        for (int c = lane; c < n; c += 32) AinvT[(long long)c * n + r] = sing[r] ? 0.0 : M[r * ld + n + c];
    if (threadIdx.x == 0) {
        int any_sing = 0;
        for (int r = 0; r < n; r++) any_sing |= sing[r];
        gj[0] = any_sing;
        gj[3] = 1;
    }
}

// ---------------------------------------------------------------------
__global__ void k_maxabs(Lev L, const double* __restrict__ g, int rel, unsigned long long* out)
{
    pdl_wait();
    const unsigned nx = L.nx, ny = L.ny;
    const unsigned total = nx * ny * (unsigned)L.nz;
    const double ref = rel ? g[(long long)1 + (nx + 2) * (1 + (long long)(ny + 2) * 1)] : 0.0;
    double m = 0.0;
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        unsigned k = t / (nx * ny);
        unsigned rem = t - k * nx * ny;
        unsigned j = rem / nx;
        unsigned i = rem - j * nx;
        long long gi = (long long)(i + 1) + (long long)(nx + 2) * ((long long)(j + 1) + (long long)(ny + 2) * (k + 1));
        double v = fabs(g[gi] - ref);
        if (!(v <= 1.0e308)) v = __longlong_as_double(0x7ff8000000000000LL);  // NaN/Inf sort above all
        m = (__double_as_longlong(v) > __double_as_longlong(m)) ? v : m;
    }
    unsigned long long b = (unsigned long long)__double_as_longlong(m);
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long ob = __shfl_down_sync(0xffffffffu, b, o);
        b = ob > b ? ob : b;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, b);
}

// the maxima of |field| over the interior of every present field in one pass
// (warp per row, lanes along x): out[0] vel (3 components), out[1] reac,
// out[2] |dcoeff - dcoeff(1,1,1)|, out[3] source, out[4] soln, out[5] dcoeff;
// NaN/Inf sort above every finite value (atomicMax on the bit patterns)
__global__ void k_maxabs_all(Lev L, const double* __restrict__ vel, const double* __restrict__ reac,
                             const double* __restrict__ dcoeff, const double* __restrict__ source,
                             const double* __restrict__ soln, unsigned long long* out)
{
    pdl_wait();
    const long long gx = L.nx + 2, gy = L.ny + 2;
    const long long ng = gx * gy * (L.nz + 2);
    const double ref = dcoeff[1 + gx * (1 + gy)];
    long long m[6] = {0, 0, 0, 0, 0, 0};
    auto upd = [](long long& cur, double v) {
        v = fabs(v);
        if (!(v <= 1.0e308)) v = __longlong_as_double(0x7ff8000000000000LL);
        const long long b = __double_as_longlong(v);
        cur = b > cur ? b : cur;
    };
    const unsigned lane = threadIdx.x & 31;
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarp = (gridDim.x * blockDim.x) >> 5;
    for (unsigned row = warp; row < L.rows; row += nwarp) {
        const unsigned k = L.divNy.div(row), j = row - k * (unsigned)L.ny;
        const long long base = 1 + gx * ((long long)(j + 1) + gy * (long long)(k + 1));
        for (int i = lane; i < L.nx; i += 32) {
            const long long g = base + i;
            if (vel) {
                upd(m[0], vel[g]);
                upd(m[0], vel[g + ng]);
                upd(m[0], vel[g + 2 * ng]);
            }
            if (reac) upd(m[1], reac[g]);
            const double d = dcoeff[g];
            upd(m[2], d - ref);
            upd(m[5], d);
            upd(m[3], source[g]);
            upd(m[4], soln[g]);
        }
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
        long long b = m[q];
        for (int o = 16; o > 0; o >>= 1) {
            const long long ob = __shfl_down_sync(0xffffffffu, b, o);
            b = ob > b ? ob : b;
        }
        if (lane == 0 && b > 0) atomicMax(out + q, (unsigned long long)b);
    }
}

__global__ void k_fill_ghosts(Lev L, double* __restrict__ g, const double* bl, const double* br, const double* bb,
                              const double* bt, const double* bk, const double* bf)
{
    pdl_wait();
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const long long sx = 1, sy = nx + 2, sz = (long long)(nx + 2) * (ny + 2);
    auto G = [&](int i, int j, int k) -> double& { return g[i * sx + j * sy + k * sz]; };
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    for (int t = tid; t < ny * nz; t += stride) {  // LEFT / RIGHT over (j,k)
        int j = 1 + t % ny, k = 1 + t / ny;
        if (L.per[0]) {
            G(0, j, k) = G(nx, j, k);
            G(nx + 1, j, k) = G(1, j, k);
        } else {
            G(0, j, k) = L.bc[F_LEFT] == BC_DIRC ? 2.0 * bl[t] - G(1, j, k) : G(1, j, k);
            G(nx + 1, j, k) = L.bc[F_RIGHT] == BC_DIRC ? 2.0 * br[t] - G(nx, j, k) : G(nx, j, k);
        }
    }
    for (int t = tid; t < nx * nz; t += stride) {  // BOTTOM / TOP over (i,k)
        int i = 1 + t % nx, k = 1 + t / nx;
        if (L.per[1]) {
            G(i, 0, k) = G(i, ny, k);
            G(i, ny + 1, k) = G(i, 1, k);
        } else {
            G(i, 0, k) = L.bc[F_BOTTOM] == BC_DIRC ? 2.0 * bb[t] - G(i, 1, k) : G(i, 1, k);
            G(i, ny + 1, k) = L.bc[F_TOP] == BC_DIRC ? 2.0 * bt[t] - G(i, ny, k) : G(i, ny, k);
        }
    }
    for (int t = tid; t < nx * ny; t += stride) {  // BACK / FRONT over (i,j)
        int i = 1 + t % nx, j = 1 + t / nx;
        if (L.per[2]) {
            G(i, j, 0) = G(i, j, nz);
            G(i, j, nz + 1) = G(i, j, 1);
        } else {
            G(i, j, 0) = L.bc[F_BACK] == BC_DIRC ? 2.0 * bk[t] - G(i, j, 1) : G(i, j, 1);
            G(i, j, nz + 1) = L.bc[F_FRONT] == BC_DIRC ? 2.0 * bf[t] - G(i, j, nz) : G(i, j, nz);
        }
    }
}

__global__ void k_find_bvec(Lev L, const double* __restrict__ vel, const double* __restrict__ dcoeff,
                            const double* __restrict__ source, const double* bl, const double* br,
                            const double* bb, const double* bt, const double* bk, const double* bf,
                            const double* __restrict__ sterm, int flux, Split<double> b)
{
    pdl_wait();
    unsigned t = blockIdx.x * TPB + threadIdx.x;
    const unsigned nx = L.nx, ny = L.ny, nz = L.nz;
    if (t >= nx * ny * nz) return;
    unsigned k = t / (nx * ny);
    unsigned rem = t - k * nx * ny;
    unsigned j = rem / nx;
    unsigned i = rem - j * nx;
    const long long ng = (long long)(nx + 2) * (ny + 2) * (nz + 2);
    const long long gi = (long long)(i + 1) + (long long)(nx + 2) * ((long long)(j + 1) + (long long)(ny + 2) * (k + 1));
    double v = (sterm ? sterm[t] : 0.0) + source[gi];
    // interior cells: the source alone (the face terms below touch boundary cells)
    if (i > 0 && i + 1 < nx && j > 0 && j + 1 < ny && k > 0 && k + 1 < nz) {
        b.half(scol(i, j, k))[soff(L, i, j, k)] = v;
        return;
    }
    v = 0.0;
    const double kc = dcoeff[gi];
    const double* faceval[6] = {bl, br, bb, bt, bk, bf};
    const unsigned pos[3] = {i, j, k};
    const unsigned len[3] = {nx, ny, nz};
#pragma unroll
    for (int f = 0; f < 6; f++) {
        const int ax = f >> 1, side = f & 1;
        if (L.per[ax]) continue;
        if (side == 0 ? pos[ax] != 0 : pos[ax] != len[ax] - 1) continue;
        long long fi = ax == 0 ? (long long)j + (long long)ny * k
                               : (ax == 1 ? (long long)i + (long long)nx * k : (long long)i + (long long)nx * j);
        const double gv = faceval[f] ? faceval[f][fi] : 0.0;
        const double h = L.w[ax];
        const double vb = vel ? vel[ax * ng + gi] : 0.0;
        if (L.bc[f] == BC_DIRC) {
            if (flux == 1) {
                double wL, wR;
                sg_face(vb, vb, kc, kc, 0.5 * h, wL, wR);
                if (side == 0) v = v + wL * gv / h;
                else v = v - wR * gv / h;
            } else {
                v = v + 2.0 * kc * gv / (h * h);
                if (side == 0 && vb > 0.0) v = v + vb * gv / h;
                if (side == 1 && vb < 0.0) v = v - vb * gv / h;
            }
        } else if (L.bc[f] == BC_FLUX) {
            v = v - gv / h;
        }
    }
    v = v + (sterm ? sterm[t] : 0.0);
    v = v + source[gi];
    b.half(scol(i, j, k))[soff(L, i, j, k)] = v;
}

__global__ void k_restrict_field(Lev F, CSplit<double> in, Lev C, Split<double> out, int geom)
{
    pdl_wait();
    unsigned t = blockIdx.x * TPB + threadIdx.x;
    const unsigned ncx = C.nx, ncy = C.ny;
    if (t >= ncx * ncy * (unsigned)C.nz) return;
    unsigned K = t / (ncx * ncy);
    unsigned rem = t - K * ncx * ncy;
    unsigned J = rem / ncx;
    unsigned I = rem - J * ncx;
    const int cI[3] = {(int)I, (int)J, (int)K};
    int lo[3], cnt[3];
    for (int a = 0; a < 3; a++) {
        const int nf = lev_n(F, a), nc = lev_n(C, a);
        lo[a] = nf == nc ? cI[a] : 2 * cI[a];
        cnt[a] = nf == nc ? 1 : ((geom && cI[a] == nc - 1) ? nf - 2 * (nc - 1) : 2);
    }
    double s = 0.0, vol = 0.0;
    for (int dk = 0; dk < cnt[2]; dk++) {
        const int k = lo[2] + dk;
        const double wz = geom ? cwidth(F, 2, k) : 1.0;
        for (int dj = 0; dj < cnt[1]; dj++) {
            const int j = lo[1] + dj;
            const double wy = geom ? cwidth(F, 1, j) : 1.0;
            for (int di = 0; di < cnt[0]; di++) {
                const int i = lo[0] + di;
                const double wx = geom ? cwidth(F, 0, i) : 1.0;
                const double v = wx * wy * wz;
                s += v * in.get(F, i, j, k);
                vol += v;
            }
        }
    }
    out.half(scol(I, J, K))[soff(C, I, J, K)] = geom ? s / vol : s * (1.0 / vol);
}

__global__ void k_multidot(long long n, int m, const double* const* __restrict__ V, const double* __restrict__ w,
                           double* __restrict__ partial)
{
    pdl_wait();
    __shared__ double sh[32];
    for (int q = 0; q < m; q++) {
        const double* v = V[q];
        double s = 0.0;
        for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
             t += (long long)gridDim.x * blockDim.x)
            s += v[t] * w[t];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) partial[(long long)q * gridDim.x + blockIdx.x] = s;
    }
}

__global__ void k_multidot_finish(int m, int nblocks, const double* __restrict__ partial, double* __restrict__ h,
                                  int accumulate)
{
    pdl_wait();
    __shared__ double sh[32];
    const int q = blockIdx.x;
    if (q >= m) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partial[(long long)q * nblocks + b];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) h[q] = accumulate ? h[q] + s : s;
}

__global__ void k_multiaxpy(long long n, int m, const double* const* __restrict__ V, const double* __restrict__ h,
                            double* __restrict__ w)
{
    pdl_wait();
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        double s = w[t];
        for (int q = 0; q < m; q++) s -= h[q] * V[q][t];
        w[t] = s;
    }
}

__global__ void k_scale_to(long long n, const double* __restrict__ w, const double* __restrict__ hn, int idx,
                           double* __restrict__ v, float* __restrict__ v32)
{
    pdl_wait();
    const double inv = 1.0 / hn[idx];
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        double x = w[t] * inv;
        if (v) v[t] = x;
        if (v32) v32[t] = (float)x;
    }
}

}  // namespace mps
