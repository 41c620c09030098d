// Batched solves: many independent problems advanced together.
//
// Each problem keeps its own level hierarchy, built by the single-problem
// set-up (solve_impl with prepare_only).  The iteration then runs as a fixed
// list of batched steps -- one kernel launch per colour pass, transfer,
// coarsest solve, outer residual, correction and convergence check -- that
// cover every problem taking part in the step.  A launch is a persistent
// loop over tasks: a task is one block-sized tile of one problem, and each
// block takes a contiguous range of the step's tasks, looking up the problem
// (a binary search over the step's task prefix) and copying its descriptor
// (level, operator, buffers) into shared memory when the range enters it; it
// runs the same device function as the single-problem kernel.  Problems
// whose hierarchies are shallower simply take no part in the deeper steps;
// converged problems are skipped at run time through a per-problem flag.
//
// The outer iteration (defect correction: FP64 residual, V-cycles in T, FP64
// update) is one CUDA graph whose body is a WHILE conditional node: the check
// kernel at the end of the body clears the condition once no problem is
// active.  Every problem leaves the active set after at most maxit
// iterations, and the check kernel also counts the body's executions and
// stops at maxit + 2, so the loop always ends.
//
// The launch shape (blocks of the task loop, and the colour pass's
// cells per thread, per level depth) is picked by timing every candidate
// pair on the batch's own colour passes at the first call with a given batch
// structure.

namespace mps {

// per-problem iteration state (device)
struct BState {
    int active, iters, status, pad;
    double rel, rms, rel0;
};

// one problem of the batched operator detection (the scan of k_maxabs_all):
// its interior fields and the launch blocks it takes
struct BDetect {
    const double *vel, *reac, *dcoeff, *source, *soln;
    int nx, ny, nz;
    unsigned rows;
    FastDiv divNy;
    int blk0, nblk;
    unsigned long long* out;  // 9 words: k_maxabs_all's six maxima (two spare), dcoeff(1,1,1)
};

// the detection of every problem of a batch in one launch: each problem's
// blocks scan its rows (warp per row, as k_maxabs_all) and its first block
// also records the coefficient of cell (1,1,1)
__global__ void __launch_bounds__(256) kb_detect(const BDetect* __restrict__ dd, int np)
{
    int lo = 0, hi = np - 1;  // the problem whose block range holds this block
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (dd[mid].blk0 <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const BDetect& d = dd[lo];
    const long long gx = d.nx + 2, gy = d.ny + 2;
    const long long ng = gx * gy * (d.nz + 2);
    const double ref = d.dcoeff[1 + gx * (1 + gy)];
    if (blockIdx.x == (unsigned)d.blk0 && threadIdx.x == 0) d.out[8] = (unsigned long long)__double_as_longlong(ref);
    long long m[6] = {0, 0, 0, 0, 0, 0};
    auto upd = [](long long& cur, double v) {
        v = fabs(v);
        if (!(v <= 1.0e308)) v = __longlong_as_double(0x7ff8000000000000LL);
        const long long b = __double_as_longlong(v);
        cur = b > cur ? b : cur;
    };
    const unsigned lane = threadIdx.x & 31;
    const unsigned warp = ((blockIdx.x - d.blk0) * blockDim.x + threadIdx.x) >> 5, nwarp = (d.nblk * blockDim.x) >> 5;
    for (unsigned row = warp; row < d.rows; row += nwarp) {
        const unsigned k = d.divNy.div(row), j = row - k * (unsigned)d.ny;
        const long long base = 1 + gx * ((long long)(j + 1) + gy * (long long)(k + 1));
        for (int i = lane; i < d.nx; i += 32) {
            const long long g = base + i;
            if (d.vel) {
                upd(m[0], d.vel[g]);
                upd(m[0], d.vel[g + ng]);
                upd(m[0], d.vel[g + 2 * ng]);
            }
            if (d.reac) upd(m[1], d.reac[g]);
            const double c = d.dcoeff[g];
            upd(m[2], c - ref);
            upd(m[5], c);
            upd(m[3], d.source[g]);
            upd(m[4], d.soln[g]);
        }
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
        long long b = m[q];
        for (int o = 16; o > 0; o >>= 1) {
            const long long ob = __shfl_down_sync(0xffffffffu, b, o);
            b = ob > b ? ob : b;
        }
        if (lane == 0 && b > 0) atomicMax(d.out + q, (unsigned long long)b);
    }
}

// every problem active, no iteration done (the start of a batched solve)
__global__ void kb_reset_state(BState* st, int np)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np) st[p] = BState{1, 0, MPS_OK, 0, 0.0, 0.0, 0.0};
}

enum BKind { B_COLOUR = 0, B_RESTRICT, B_COARSE, B_PROLONG, B_OUTER, B_AXPY };

template <class T>
struct DColour {
    Lev L;
    KOp<T> op;
    const T* u0;  // state: red half
    const T* u1;  // state: black half (already offset by half)
    T* out;       // this colour's half of the other buffer
    const T* f;   // this colour's half of the right-hand side
    ColourSplit cs;  // interior groups and shell of the vector body (when split)
    int split;       // 1: the vector body's tasks follow cs (interior without boundary code, then the shell)
};
template <class T>
struct DRestrict {
    Lev F, C;
    KOp<T> op;
    const T* u0;
    const T* u1;
    const T* f;  // fine right-hand side (split base)
    T* fc;       // coarse right-hand side (split base)
    // the single solve's two-part form (w > 0: the bulk's red residuals, w
    // coarse cells of a row per thread, then the shell cells, eight lanes
    // each); w = 0: one thread per coarse cell over all its children
    RestrictSplit rs;
    Box bx;
    unsigned nb_bulk, shell;
    int w;
    int geom;
};
template <class T>
struct DCoarse {
    Lev C;
    const double* AinvT;
    const T* f;
    T* u0;
    T* u1;
};
template <class T>
struct DProlong {
    Lev F, C;
    Xfer X;
    T* u0;
    T* u1;
    const T* e0;
    const T* e1;
    int mode;  // 1: the black cells and the red cells of odd periodic seams (the
               // first post-smoothing pass rewrites the other red cells); -1: all
    // the single solve's vector bulk (w > 0: w cells of a row per thread in
    // the parts of pp, within box pb; the same cells as mode 1)
    Box pb, sb;
    ProlongDiv dv, sv;
    ProlongParts pp;
    int w;
};
template <class T>
struct DOuter {
    Lev L;
    KOp<double> op;
    const double* x;  // split base
    const double* b;  // split base
    T* r;             // split base (finest right-hand side of the T hierarchy)
    ColourSplit cs;   // interior groups and shell of the vector residual (when split)
    int split;        // 1: the tasks follow cs (BATCH_W cells of a row per thread)
};
template <class T>
struct DAxpy {
    long long half;
    const T* e0;
    const T* e1;
    double* x;
};


__device__ __forceinline__ int find_seg(const int* __restrict__ task0, int nseg, int task)
{
    int lo = 0, hi = nseg;  // task0[lo] <= task < task0[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&task0[mid]) <= task) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <class D>
__device__ __forceinline__ void load_desc(const D* __restrict__ desc, int seg, unsigned char* sbuf)
{
    const unsigned* src = reinterpret_cast<const unsigned*>(desc + seg);
    unsigned* dst = reinterpret_cast<unsigned*>(sbuf);
    for (int w = threadIdx.x; w < (int)(sizeof(D) / 4); w += blockDim.x) dst[w] = __ldg(&src[w]);
}

// The tasks of one batched step, each block taking a contiguous range: the
// segment (problem) is found, its descriptor copied into shared memory and
// its active flag read only when the range enters a new segment, and an
// inactive problem's remaining tasks are skipped at once.  Measured on the
// 64-problem batch: 52.6 / 68.2 ms (mixed / FP64) against 60.3 / 93.7 ms for
// a grid-stride loop that looked up the segment and copied the descriptor
// for every task.
#define BATCH_LOOP(D, desc, task0, pid, nseg, total, active, ...)                                               \
    __shared__ __align__(16) unsigned char sbuf_[sizeof(D)];                                                   \
    {                                                                                                          \
        const int per_ = ((total) + (int)gridDim.x - 1) / (int)gridDim.x;                                     \
        const int beg_ = (int)blockIdx.x * per_;                                                               \
        const int end_ = min((total), beg_ + per_);                                                            \
        int seg = 0, segbeg_ = 0, segend_ = beg_;                                                              \
        bool act_ = false;                                                                                     \
        for (int task = beg_; task < end_; task++) {                                                           \
            if (task >= segend_) {                                                                             \
                seg = find_seg(task0, nseg, task);                                                             \
                segbeg_ = __ldg(&(task0)[seg]);                                                                \
                segend_ = __ldg(&(task0)[seg + 1]);                                                            \
                const int prob = __ldg(&(pid)[seg]);                                                           \
                act_ = ((volatile const int*)&(active)[prob].active)[0] != 0;                                  \
                __syncthreads();                                                                               \
                if (act_) load_desc<D>(desc, seg, sbuf_);                                                      \
                __syncthreads();                                                                               \
            }                                                                                                  \
            if (!act_) {                                                                                       \
                task = segend_ - 1;                                                                            \
                continue;                                                                                      \
            }                                                                                                  \
            const D& d = *reinterpret_cast<const D*>(sbuf_);                                                   \
            const unsigned t = (unsigned)(task - segbeg_) * TPB + threadIdx.x;                                 \
            (void)t;                                                                                           \
            __VA_ARGS__                                                                                        \
        }                                                                                                      \
    }

// Shapes of the batched steps, measured on the 64-problem batch (sizes 33 to
// 129, 5 outer iterations; ms per batch, mixed / FP64):
//   colour     restriction          prolongation    mixed / FP64
//   1 cell     1 thread per cell    all cells       80.0 / 97.0
//   4 (FP32)   8 lanes per cell     black cells     67.9 / 107.0
//   4 (FP32)   8 lanes per cell     all cells       74.2 / 113.5
//   4 (both)   8 lanes per cell     black cells     67.7 / 108.6
//   4 (FP32)   1 thread per cell    black cells     59.9 / 90.6
// (colour: cells of a row per thread on levels with a vector row evaluation;
// black cells: the first post-smoothing pass rewrites the red ones).  Then,
// with the task ranges of BATCH_LOOP (52.6 / 68.2), the single solve's
// forms step by step: the colour pass and the outer residual split into
// interior groups and shell (50.7 / 60.8, then 47.2 / 60.5), the two-part
// restriction (44.4 / 55.3) and the vector prolongation bulk (40.6 / 51.6).
// Kept: the single solve's forms where a level has them (the generic
// bodies elsewhere), and the colour-pass body picked per depth by the
// autotuner together with the grid (below).
#ifndef MPS_BATCH_R8
#define MPS_BATCH_R8 0
#endif
#ifndef MPS_BATCH_PB
#define MPS_BATCH_PB 1
#endif
constexpr int BATCH_W = 4;
__host__ __device__ __forceinline__ bool batch_vector_level(const Lev& L) { return L.uniform || L.nx >= 16; }

// one group of BATCH_W cells of colour c (thread index t over (P/W) x rows)
template <class T, class U>
__device__ __forceinline__ void colour_group_body(const Lev& L, const KOp<T>& op, int c, const U& u,
                                                  T* __restrict__ out, const T* __restrict__ f, unsigned t)
{
    constexpr int W = BATCH_W;
    const unsigned ng = (unsigned)L.P / W;
    const unsigned row = L.divG.div(t);
    if (row >= L.rows) return;
    const int k = (int)L.divNy.div(row);
    const int j = (int)row - k * L.ny;
    const int h0 = W * (int)(t - row * ng);
    const int q = (j + k + c) & 1;
    const int o0 = h0 + L.P * (int)row;
    const VecW<T, W> f4 = ldv<T, W>(f + o0);
    VecW<T, W> diag, off;
    if (L.uniform) group_rows<T, W, U, true>(L, op, c, u, (int)row, j, k, h0, q, o0, diag, off);
    else group_rows<T, W, U, false>(L, op, c, u, (int)row, j, k, h0, q, o0, diag, off);
    VecW<T, W> res;
#pragma unroll
    for (int e = 0; e < W; e++) {
        const int i = 2 * (h0 + e) + q;
        res.v[e] = i < L.nx ? gs_value(f4.v[e], diag.v[e], off.v[e]) : T(0);
    }
    stv<T, W>(out + o0, res);
}

template <class T, class U>
__device__ __forceinline__ void batch_colour(const DColour<T>& d, int c, const U& u, unsigned t, int vec)
{
    if (vec && batch_vector_level(d.L)) {
        if (d.split) {
            // the task's block of the split pass (t = block * TPB + thread)
            if (d.L.uniform) colour_split_block<T, BATCH_W, U, true>(d.L, d.op, c, u, d.out, d.f, d.cs, t / TPB);
            else colour_split_block<T, BATCH_W, U, false>(d.L, d.op, c, u, d.out, d.f, d.cs, t / TPB);
        } else {
            colour_group_body<T, U>(d.L, d.op, c, u, d.out, d.f, t);
        }
    } else {
        colour_body<T, KOp<T>, U>(d.L, d.op, c, u, d.out, d.f, t);
    }
}

// vec: the vector body on the levels that have one (the task layout of the
// step must be the matching one)
template <class T>
__global__ void __launch_bounds__(TPB) kb_colour(const DColour<T>* __restrict__ desc, const int* __restrict__ task0,
                                                 const int* __restrict__ pid, int nseg, int total,
                                                 const BState* active, int c, int zs, int vec)
{
    BATCH_LOOP(DColour<T>, desc, task0, pid, nseg, total, active, {
        if (zs == 2) {
            batch_colour<T, ZeroU<T>>(d, c, ZeroU<T>(), t, vec);
        } else if (zs == 1) {
            OtherOnlyU<T> u;
            u.c = c;
            u.other = c == 0 ? d.u1 : d.u0;
            batch_colour<T, OtherOnlyU<T>>(d, c, u, t, vec);
        } else {
            CSplit<T> u;
            u.c[0] = d.u0;
            u.c[1] = d.u1;
            batch_colour<T, CSplit<T>>(d, c, u, t, vec);
        }
    })
}

template <class T>
__global__ void __launch_bounds__(TPB) kb_restrict(const DRestrict<T>* __restrict__ desc,
                                                   const int* __restrict__ task0, const int* __restrict__ pid,
                                                   int nseg, int total, const BState* active)
{
    // eight lanes per coarse cell, each a share of the children, summed by
    // shuffles (every thread of the block reaches the shuffles)
    BATCH_LOOP(DRestrict<T>, desc, task0, pid, nseg, total, active, {
        CSplit<T> u, f;
        u.c[0] = d.u0;
        u.c[1] = d.u1;
        f.c[0] = d.f;
        f.c[1] = d.f + d.F.half;
        if (d.w) {
            Split<T> fc;
            fc.c[0] = d.fc;
            fc.c[1] = d.fc + d.C.half;
            const unsigned blk = t / TPB;
            if (blk < d.nb_bulk) {
                if (d.F.uniform) {
                    if (d.w == 4) resid_restrict_bulk<T, 4, true>(d.F, d.op, u, d.f, d.C, fc, d.bx, d.rs, blk);
                    else if (d.w == 2) resid_restrict_bulk<T, 2, true>(d.F, d.op, u, d.f, d.C, fc, d.bx, d.rs, blk);
                    else resid_restrict_bulk<T, 1, true>(d.F, d.op, u, d.f, d.C, fc, d.bx, d.rs, blk);
                } else {
                    if (d.w == 4) resid_restrict_bulk<T, 4, false>(d.F, d.op, u, d.f, d.C, fc, d.bx, d.rs, blk);
                    else if (d.w == 2) resid_restrict_bulk<T, 2, false>(d.F, d.op, u, d.f, d.C, fc, d.bx, d.rs, blk);
                    else resid_restrict_bulk<T, 1, false>(d.F, d.op, u, d.f, d.C, fc, d.bx, d.rs, blk);
                }
            } else {
                resid_restrict_shell<T, KOp<T>>(d.F, d.op, u, f, d.C, fc, d.geom, d.bx, d.shell,
                                                (blk - d.nb_bulk) * TPB + threadIdx.x);
            }
            continue;
        }
        if (!MPS_BATCH_R8) {  // one thread per coarse cell over all its children
            Split<T> fc;
            fc.c[0] = d.fc;
            fc.c[1] = d.fc + d.C.half;
            resid_restrict_body<T, KOp<T>>(d.F, d.op, u, f, d.C, fc, d.geom, t);
            continue;
        }
        const unsigned ncx = d.C.nx, ncy = d.C.ny, nc = ncx * ncy * (unsigned)d.C.nz;
        const unsigned cell = t >> 3;
        const int part = (int)(t & 7u);
        T sm = T(0), vol = T(0);
        unsigned I = 0, J = 0, K = 0;
        if (cell < nc) {
            K = cell / (ncx * ncy);
            const unsigned rem = cell - K * ncx * ncy;
            J = rem / ncx;
            I = rem - J * ncx;
            resid_restrict_part<T, KOp<T>>(d.F, d.op, u, f, d.C, d.geom, (int)I, (int)J, (int)K, part, 8, sm, vol);
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            sm += __shfl_xor_sync(0xffffffffu, sm, o, 8);
            vol += __shfl_xor_sync(0xffffffffu, vol, o, 8);
        }
        if (cell < nc && part == 0) {
            T* dst = scol((int)I, (int)J, (int)K) ? d.fc + d.C.half : d.fc;
            dst[soff(d.C, (int)I, (int)J, (int)K)] = d.geom ? sm / vol : sm * (T(1) / vol);
        }
    })
}

template <class T>
__global__ void __launch_bounds__(TPB) kb_coarse(const DCoarse<T>* __restrict__ desc, const int* __restrict__ task0,
                                                 const int* __restrict__ pid, int nseg, int total,
                                                 const BState* active)
{
    __shared__ double fs[1024];
    BATCH_LOOP(DCoarse<T>, desc, task0, pid, nseg, total, active, {
        CSplit<T> f;
        f.c[0] = d.f;
        f.c[1] = d.f + d.C.half;
        Split<T> u;
        u.c[0] = d.u0;
        u.c[1] = d.u1;
        coarse_solve_body<T>(d.C, d.AinvT, f, u, fs);
        __syncthreads();
    })
}

template <class T>
__global__ void __launch_bounds__(TPB) kb_prolong(const DProlong<T>* __restrict__ desc, const int* __restrict__ task0,
                                                  const int* __restrict__ pid, int nseg, int total,
                                                  const BState* active)
{
    BATCH_LOOP(DProlong<T>, desc, task0, pid, nseg, total, active, {
        Split<T> u;
        u.c[0] = d.u0;
        u.c[1] = d.u1;
        CSplit<T> e;
        e.c[0] = d.e0;
        e.c[1] = d.e1;
        if (d.w) {
            const unsigned blk = t / TPB;
            if (d.w == 4) prolong_v_block<T, 4>(d.F, u, d.C, e, d.X, d.pb, d.dv, d.sb, d.sv, d.pp, blk);
            else if (d.w == 2) prolong_v_block<T, 2>(d.F, u, d.C, e, d.X, d.pb, d.dv, d.sb, d.sv, d.pp, blk);
            else prolong_v_block<T, 1>(d.F, u, d.C, e, d.X, d.pb, d.dv, d.sb, d.sv, d.pp, blk);
        } else if (d.mode < 0) {
            prolong_body<T>(d.F, u, d.C, e, d.X, -1, t);
        } else {
            prolong_body<T>(d.F, u, d.C, e, d.X, 1, t);
            if ((d.F.per[0] && (d.F.nx & 1)) || (d.F.per[1] && (d.F.ny & 1)) || (d.F.per[2] && (d.F.nz & 1)))
                prolong_body<T>(d.F, u, d.C, e, d.X, 2, t);
        }
    })
}

// r = b - A x in FP64 over both colours, r stored as T; per-task partial sums
// of r.r and b.b (deterministic: the check kernel adds them in task order)
template <class T>
__global__ void __launch_bounds__(TPB) kb_outer(const DOuter<T>* __restrict__ desc, const int* __restrict__ task0,
                                                const int* __restrict__ pid, int nseg, int total,
                                                const BState* active, double* __restrict__ partial)
{
    __shared__ double sh[32];
    BATCH_LOOP(DOuter<T>, desc, task0, pid, nseg, total, active, {
        double rr = 0.0, bb = 0.0;
        const unsigned n = (unsigned)d.L.P * d.L.rows;
        CSplit<double> x;
        x.c[0] = d.x;
        x.c[1] = d.x + d.L.half;
        if (d.split) resid_split_chunk<double, BATCH_W, T>(d.L, d.op, x, d.b, d.r, d.cs, t / TPB, rr, bb);
        else for (int c = 0; c < 2; c++) {
            int i, j, k;
            if (t < n && decode(d.L, t, c, i, j, k)) {
                double diag, off;
                row_any<double>(d.op, d.L, x, i, j, k, diag, off);
                const double bv = __ldg(&d.b[c * d.L.half + t]);
                const double r = bv - (diag * __ldg(&x.c[c][t]) + off);
                rr += r * r;
                bb += bv * bv;
                d.r[c * d.L.half + t] = (T)r;
            }
        }
        const double a = block_sum(rr, sh);
        const double b = block_sum(bb, sh);
        if (threadIdx.x == 0) {
            partial[2 * task] = a;
            partial[2 * task + 1] = b;
        }
    })
}

template <class T>
__global__ void __launch_bounds__(TPB) kb_axpy(const DAxpy<T>* __restrict__ desc, const int* __restrict__ task0,
                                               const int* __restrict__ pid, int nseg, int total,
                                               const BState* active)
{
    BATCH_LOOP(DAxpy<T>, desc, task0, pid, nseg, total, active, {
        if ((long long)t < 2 * d.half) {
            const T e = (long long)t < d.half ? d.e0[t] : d.e1[(long long)t - d.half];
            d.x[t] = d.x[t] + (double)e;
        }
    })
}

// one block per problem: sum the outer step's partials, update the state;
// the last block to finish sets the loop condition (when inside the graph)
__global__ void __launch_bounds__(TPB) kb_check(const int* __restrict__ task0, const int* __restrict__ pid,
                                                const double* __restrict__ partial, BState* st,
                                                const long long* __restrict__ ncell, int nprob, double tol,
                                                int tol_kind, int maxit, int count_iter, unsigned* counter,
                                                int* loops, int loop_cap, cudaGraphConditionalHandle hc,
                                                int use_handle)
{
    __shared__ double sh[32];
    __shared__ bool last;
    const int s = blockIdx.x;
    const int p = pid[s];
    const bool act = ((volatile int*)&st[p].active)[0] != 0;
    double a = 0.0, b = 0.0;
    if (act)
        for (int q = task0[s] + threadIdx.x; q < task0[s + 1]; q += blockDim.x) {
            a += partial[2 * q];
            b += partial[2 * q + 1];
        }
    a = block_sum(a, sh);
    b = block_sum(b, sh);
    if (threadIdx.x == 0) {
        if (act) {
            BState& S = st[p];
            if (count_iter) S.iters += 1;
            const double rel = b > 0.0 ? sqrt(a) / sqrt(b) : sqrt(a);
            const double rms = sqrt(a / (double)ncell[p]);
            if (!count_iter) S.rel0 = rel;
            S.rel = rel;
            S.rms = rms;
            const bool conv = tol_kind == MPS_TOL_RMS_ABS ? rms <= tol : rel <= tol;
            if (!(a <= 1.0e308)) { S.status = MPS_ERR_NAN; S.active = 0; }
            else if (conv) { S.status = MPS_OK; S.active = 0; }
            else if (S.iters >= maxit) { S.status = MPS_ERR_NOT_CONVERGED; S.active = 0; }
        }
        __threadfence();
        const unsigned prev = atomicAdd(counter, 1u);
        last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    int any = 0;
    for (int q = threadIdx.x; q < nprob; q += blockDim.x) any |= ((volatile int*)&st[q].active)[0];
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        *counter = 0u;
        const int l = *loops + 1;
        *loops = l;
        if (l >= loop_cap) any = 0;
        if (use_handle) cudaGraphSetConditional(hc, any ? 1u : 0u);
    }
}

#undef BATCH_LOOP

// ----------------------------------------------------------------------
// host side
struct BStep {
    int kind = 0, c = 0, zs = 0, depth = 0;
    size_t desc_off = 0;  // bytes into the descriptor buffer
    size_t task_off = 0;  // ints into the task buffer: task0[nseg+1], then pid[nseg]
    int nseg = 0, total = 0, grid = 0;
    // colour steps: the task layout of the vector body (BATCH_W cells per
    // thread on the levels that have one) and which of the two runs
    size_t task_off_v = 0;
    int total_v = 0, vec = 0;
};

struct BatchState {
    std::vector<std::unique_ptr<Ctx>> sub;
    // device buffers (one allocation each, grown on demand)
    unsigned char* ddesc = nullptr;
    size_t ddesc_cap = 0;
    int* dtask = nullptr;
    size_t dtask_cap = 0;
    double* dpart = nullptr;
    size_t dpart_cap = 0;
    BState* dst = nullptr;
    long long* dncell = nullptr;
    unsigned* dcounter = nullptr;
    int* dloops = nullptr;
    int cap_prob = 0;
    // captured loop
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> graph_key;
    int body_kernels = 0;
    // autotuned grid and colour-pass body per (precision, depth), keyed by
    // the batch structure
    std::vector<long long> tune_key;
    std::vector<int> tune_grid;
    std::vector<int> tune_vec;
    // operator detection of every problem (9 words each), read back at once
    unsigned long long* ddet = nullptr;
    unsigned long long* hdet = nullptr;  // page-locked
    BDetect* ddd = nullptr;              // the detection launch's problem table
    BDetect* hdd = nullptr;              // page-locked
    int det_cap = 0;
    // streams of the per-problem set-ups (independent: they overlap on the
    // device), joined to the handle's stream before the iterations
    // the tables last uploaded (a repeated batch skips the uploads: copies
    // from pageable host memory hold the host until the stream drains)
    std::vector<unsigned char> up_desc;
    std::vector<int> up_task;
    std::vector<long long> up_cells;
    static constexpr int NSET = 8;
    cudaStream_t set_s[NSET] = {};
    cudaEvent_t set_e[NSET] = {};
    cudaEvent_t start_e = nullptr;
    // a repeated batch (same problems, buffers, options and detected
    // operators) replays its set-up and its unpacking as CUDA graphs, captured
    // at the second call with that key, and reuses its step plan
    std::vector<long long> prep_key;
    int prep_calls = 0;                  // calls in a row with prep_key
    cudaGraphExec_t prep_exec = nullptr, post_exec = nullptr;
    long long prep_kernels = 0, post_kernels = 0;  // kernels in those graphs (the launch counts)
    std::shared_ptr<void> plan;          // BatchPlan<T> of prep_key
};

static void batch_release_prep(BatchState& B)
{
    if (B.prep_exec) cudaGraphExecDestroy(B.prep_exec);
    if (B.post_exec) cudaGraphExecDestroy(B.post_exec);
    B.prep_exec = B.post_exec = nullptr;
    B.plan.reset();
}

static int sub_init(Ctx& parent, Ctx& sc)
{
    sc.dev = parent.dev;
    sc.nsm = parent.nsm;
    sc.s = parent.s;
    if (cudaEventCreate(&sc.e0) != cudaSuccess || cudaEventCreate(&sc.e1) != cudaSuccess ||
        cudaMallocHost((void**)&sc.hpin, sizeof(double) * 512) != cudaSuccess ||
        cudaMalloc((void**)&sc.dmax, sizeof(unsigned long long) * 8) != cudaSuccess)
        return MPS_ERR_CUDA;
    return MPS_OK;
}

static void sub_free(Ctx& sc)
{
    destroy_graphs(sc);
    sc.ar.clear();
    sc.kar.clear();
    sc.inbuf.clear();
    for (cudaEvent_t e : sc.prof.ev) cudaEventDestroy(e);
    if (sc.dtab) cudaFree(sc.dtab);
    if (sc.dmax) cudaFree(sc.dmax);
    if (sc.hpin) cudaFreeHost(sc.hpin);
    if (sc.e0) cudaEventDestroy(sc.e0);
    if (sc.e1) cudaEventDestroy(sc.e1);
    sc.dtab = nullptr;
    sc.dmax = nullptr;
    sc.hpin = nullptr;
    sc.e0 = sc.e1 = nullptr;
}

static void batch_release_graph(BatchState& B)
{
    if (B.exec) cudaGraphExecDestroy(B.exec);
    if (B.graph) cudaGraphDestroy(B.graph);
    B.exec = nullptr;
    B.graph = nullptr;
    B.graph_key.clear();
}

static void destroy_batch(Ctx& ctx)
{
    if (!ctx.batch) return;
    BatchState& B = *ctx.batch;
    batch_release_graph(B);
    for (auto& sc : B.sub) sub_free(*sc);
    B.sub.clear();
    cudaFree(B.ddesc);
    cudaFree(B.dtask);
    cudaFree(B.dpart);
    cudaFree(B.dst);
    cudaFree(B.dncell);
    cudaFree(B.dcounter);
    cudaFree(B.dloops);
    if (B.ddet) cudaFree(B.ddet);
    if (B.hdet) cudaFreeHost(B.hdet);
    if (B.ddd) cudaFree(B.ddd);
    if (B.hdd) cudaFreeHost(B.hdd);
    for (int i = 0; i < BatchState::NSET; i++) {
        if (B.set_s[i]) cudaStreamDestroy(B.set_s[i]);
        if (B.set_e[i]) cudaEventDestroy(B.set_e[i]);
    }
    if (B.start_e) cudaEventDestroy(B.start_e);
    batch_release_prep(B);
    delete ctx.batch;
    ctx.batch = nullptr;
}

// the step list and descriptors of one batch, built by replaying each
// problem's V-cycle bookkeeping (buffer parities) on the host
template <class T>
struct BatchPlan {
    std::vector<BStep> pre, body;
    std::vector<unsigned char> desc;
    std::vector<int> task;
    int maxdepth = 0;

    template <class D>
    size_t add_desc(const D& d)
    {
        const size_t off = (desc.size() + 15) / 16 * 16;
        desc.resize(off + sizeof(D));
        std::memcpy(desc.data() + off, &d, sizeof(D));
        return off;
    }
};

template <class T>
static Hier<T>& batch_hier(Ctx& sc);
template <>
Hier<float>& batch_hier<float>(Ctx& sc) { return sc.h32; }
template <>
Hier<double>& batch_hier<double>(Ctx& sc) { return sc.h64; }

template <class T>
static void plan_batch(BatchState& B, BatchPlan<T>& P, const mps_solver_opts* o, int inner)
{
    const int np = (int)B.sub.size();
    int D = 0;
    for (auto& sc : B.sub) D = std::max(D, sc->nlev - 1);
    P.maxdepth = D;
    std::vector<std::array<int, MAXL>> ri(np), bi(np);
    for (int p = 0; p < np; p++) {
        ri[p].fill(0);
        bi[p].fill(0);
    }
    // one step over the participating problems: make(p) fills the descriptor
    auto step = [&](std::vector<BStep>& list, int kind, int depth, int c, int zs, auto want, auto make,
                    auto tasks) {
        using D = decltype(make(0));
        BStep s;
        s.kind = kind;
        s.depth = depth;
        s.c = c;
        s.zs = zs;
        std::vector<int> t0, pid;
        std::vector<D> ds;
        int total = 0;
        for (int p = 0; p < np; p++) {
            if (!want(p)) continue;
            t0.push_back(total);
            pid.push_back(p);
            ds.push_back(make(p));
            total += tasks(p);
        }
        if (pid.empty()) return;
        t0.push_back(total);
        s.nseg = (int)pid.size();
        s.total = total;
        s.desc_off = (P.desc.size() + 15) / 16 * 16;
        P.desc.resize(s.desc_off + sizeof(D) * ds.size());
        std::memcpy(P.desc.data() + s.desc_off, ds.data(), sizeof(D) * ds.size());
        s.task_off = P.task.size();
        P.task.insert(P.task.end(), t0.begin(), t0.end());
        P.task.insert(P.task.end(), pid.begin(), pid.end());
        list.push_back(s);
    };
    auto nb = [](long long n) { return (int)((n + TPB - 1) / TPB); };
    // the single solve's vector prolongation where it applies (black cells
    // and odd-seam red cells, the geometric hierarchy's regular box), with its
    // cells per thread by level index
    auto prolong_vform = [&](const Lev& F, const Lev& C, const Xfer& X, int d, Box& pb, ProlongDiv& dv, Box& sb,
                             ProlongDiv& sv, ProlongParts& pp, int& w) {
        std::memset(&pb, 0, sizeof(pb));
        std::memset(&sb, 0, sizeof(sb));
        std::memset(&dv, 0, sizeof(dv));
        std::memset(&sv, 0, sizeof(sv));
        std::memset(&pp, 0, sizeof(pp));
        w = 0;
        if (!MPS_BATCH_PB || o->nu2 < 1 || F.nx < 16 || !prolong_box(F, C, X, pb)) return false;
        w = d == 0 ? ProlongShape<T>::W : d == 1 ? CoarseXferShape<T>::W : SmallXferShape<T>::W;
        if (w != 1 && w != 2 && w != 4) {
            w = 0;
            return false;
        }
        prolong_form(F, pb, w, dv, sb, sv, pp);
        return true;
    };
    // the two-part restriction of the single solve where it applies (the red
    // residual alone is valid after a black pass), with the single solve's
    // cells per thread by level index
    auto restrict_form = [&](const Lev& F, const Lev& C, int d, RestrictSplit& rs, Box& bx, unsigned& nbb,
                             unsigned& shell, int& w) {
        std::memset(&rs, 0, sizeof(rs));
        std::memset(&bx, 0, sizeof(bx));
        nbb = shell = 0;
        w = 0;
        if (o->nu1 < 1 || F.nx < 16 || !restrict_box(F, C, bx)) return false;
        w = d == 0 ? RestrictShape<T>::W : d == 1 ? CoarseXferShape<T>::W : SmallXferShape<T>::W;
        if (w != 1 && w != 2 && w != 4) {
            w = 0;
            return false;
        }
        rs = make_restrict_split(F, C, bx, w);
        nbb = rs.nb_in + rs.nb_xe + rs.nb_out;
        shell = (unsigned)((long long)C.nx * C.ny * C.nz - box_cells(bx));
        return true;
    };
    auto cur0 = [&](int p, int d) { return batch_hier<T>(*B.sub[p]).U[d][ri[p][d]]; };
    auto cur1 = [&](int p, int d) {
        return batch_hier<T>(*B.sub[p]).U[d][bi[p][d]] + B.sub[p]->lev[d].half;
    };
    auto colour = [&](std::vector<BStep>& list, int d, int c, int zs) {
        step(
            list, B_COLOUR, d, c, zs, [&](int p) { return d < B.sub[p]->nlev - 1; },
            [&](int p) {
                Ctx& sc = *B.sub[p];
                Hier<T>& H = batch_hier<T>(sc);
                const Lev& L = sc.lev[d];
                DColour<T> x;
                x.L = L;
                x.op = H.kop[d];
                x.u0 = cur0(p, d);
                x.u1 = cur1(p, d);
                x.out = c == 0 ? H.U[d][ri[p][d] ^ 1] : H.U[d][bi[p][d] ^ 1] + L.half;
                x.f = H.F[d] + (c ? L.half : 0);
                x.split = batch_vector_level(L) && make_split(L, BATCH_W, x.cs) ? 1 : 0;
                if (!x.split) std::memset(&x.cs, 0, sizeof(x.cs));
                if (c == 0) ri[p][d] ^= 1;
                else bi[p][d] ^= 1;
                return x;
            },
            [&](int p) { return nb(B.sub[p]->lev[d].half); });
        if (list.empty() || list.back().kind != B_COLOUR || list.back().depth != d) return;
        // the task layout of the vector body over the same problems
        BStep& s = list.back();
        const int* pid = P.task.data() + s.task_off + s.nseg + 1;
        std::vector<int> t0v;
        int tot = 0;
        for (int q = 0; q < s.nseg; q++) {
            t0v.push_back(tot);
            const Lev& L = B.sub[pid[q]]->lev[d];
            ColourSplit cs;
            if (!batch_vector_level(L)) tot += nb(L.half);
            else if (make_split(L, BATCH_W, cs)) tot += (int)(cs.nb_in + cs.nb_xe + cs.nb_face);
            else tot += nb(L.half / BATCH_W);
        }
        t0v.push_back(tot);
        std::vector<int> pids(pid, pid + s.nseg);
        s.task_off_v = P.task.size();
        s.total_v = tot;
        P.task.insert(P.task.end(), t0v.begin(), t0v.end());
        P.task.insert(P.task.end(), pids.begin(), pids.end());
    };
    auto vcycle = [&](std::vector<BStep>& list, bool zero) {
        for (int d = 0; d < D; d++) {
            const bool z = d > 0 || zero;
            for (int s = 0; s < o->nu1; s++) {
                colour(list, d, 0, z && s == 0 ? 2 : 0);
                colour(list, d, 1, z && s == 0 ? 1 : 0);
            }
            step(
                list, B_RESTRICT, d, 0, 0, [&](int p) { return d < B.sub[p]->nlev - 1; },
                [&](int p) {
                    Ctx& sc = *B.sub[p];
                    Hier<T>& H = batch_hier<T>(sc);
                    DRestrict<T> x;
                    x.F = sc.lev[d];
                    x.C = sc.lev[d + 1];
                    x.op = H.kop[d];
                    x.u0 = cur0(p, d);
                    x.u1 = cur1(p, d);
                    x.f = H.F[d];
                    x.fc = H.F[d + 1];
                    x.geom = sc.xf[d].geom;
                    restrict_form(x.F, x.C, d, x.rs, x.bx, x.nb_bulk, x.shell, x.w);
                    return x;
                },
                [&](int p) {
                    const Lev& F = B.sub[p]->lev[d];
                    const Lev& C = B.sub[p]->lev[d + 1];
                    RestrictSplit rs;
                    Box bx;
                    unsigned nbb, shell;
                    int w;
                    if (restrict_form(F, C, d, rs, bx, nbb, shell, w)) return (int)(nbb + nblk(8LL * shell));
                    return nb((MPS_BATCH_R8 ? 8LL : 1LL) * C.nx * C.ny * C.nz);
                });
        }
        step(
            list, B_COARSE, D, 0, 0, [&](int) { return true; },
            [&](int p) {
                Ctx& sc = *B.sub[p];
                Hier<T>& H = batch_hier<T>(sc);
                const int d = sc.nlev - 1;
                DCoarse<T> x;
                x.C = sc.lev[d];
                x.AinvT = H.AinvT;
                x.f = H.F[d];
                x.u0 = cur0(p, d);
                x.u1 = cur1(p, d);
                return x;
            },
            [&](int) { return 1; });
        for (int d = D - 1; d >= 0; d--) {
            step(
                list, B_PROLONG, d, 0, 0, [&](int p) { return d < B.sub[p]->nlev - 1; },
                [&](int p) {
                    Ctx& sc = *B.sub[p];
                    DProlong<T> x;
                    x.F = sc.lev[d];
                    x.C = sc.lev[d + 1];
                    x.X = sc.xf[d];
                    x.u0 = cur0(p, d);
                    x.u1 = cur1(p, d);
                    x.e0 = cur0(p, d + 1);
                    x.e1 = cur1(p, d + 1);
                    x.mode = (MPS_BATCH_PB && o->nu2 >= 1) ? 1 : -1;
                    prolong_vform(x.F, x.C, x.X, d, x.pb, x.dv, x.sb, x.sv, x.pp, x.w);
                    return x;
                },
                [&](int p) {
                    const Lev& F = B.sub[p]->lev[d];
                    Box pb, sb;
                    ProlongDiv dv, sv;
                    ProlongParts pp;
                    int w;
                    if (prolong_vform(F, B.sub[p]->lev[d + 1], B.sub[p]->xf[d], d, pb, dv, sb, sv, pp, w))
                        return (int)pp.blk0[4];
                    return (MPS_BATCH_PB && o->nu2 >= 1) ? nb(F.half) : nb((long long)F.nx * F.ny * F.nz);
                });
            for (int s = 0; s < o->nu2; s++) {
                colour(list, d, 0, 0);
                colour(list, d, 1, 0);
            }
        }
    };
    auto outer = [&](std::vector<BStep>& list) {
        step(
            list, B_OUTER, 0, 0, 0, [&](int) { return true; },
            [&](int p) {
                Ctx& sc = *B.sub[p];
                DOuter<T> x;
                x.L = sc.lev[0];
                x.op = sc.kop64;
                x.x = sc.x64;
                x.b = sc.b64;
                x.r = batch_hier<T>(sc).F[0];
                x.split = sc.lev[0].uniform && make_split(sc.lev[0], BATCH_W, x.cs) ? 1 : 0;
                if (!x.split) std::memset(&x.cs, 0, sizeof(x.cs));
                return x;
            },
            [&](int p) {
                const Lev& L = B.sub[p]->lev[0];
                ColourSplit cs;
                if (L.uniform && make_split(L, BATCH_W, cs)) return (int)(cs.nb_in + cs.nb_xe + cs.nb_face);
                return nb(L.half);
            });
    };
    outer(P.pre);
    for (int c = 0; c < inner; c++) vcycle(P.body, c == 0);
    step(
        P.body, B_AXPY, 0, 0, 0, [&](int) { return true; },
        [&](int p) {
            Ctx& sc = *B.sub[p];
            DAxpy<T> x;
            x.half = sc.lev[0].half;
            x.e0 = cur0(p, 0);
            x.e1 = cur1(p, 0);
            x.x = sc.x64;
            return x;
        },
        [&](int p) { return nb(2 * B.sub[p]->lev[0].half); });
    outer(P.body);
}

template <class T>
static void launch_step(cudaStream_t s, const BStep& st, const unsigned char* ddesc, const int* dtask,
                        const BState* active, double* dpart)
{
    const int* t0 = dtask + st.task_off;
    const int* pid = t0 + st.nseg + 1;
    const unsigned g = (unsigned)std::max(1, std::min(st.grid, st.total));
    const void* dp = ddesc + st.desc_off;
    switch (st.kind) {
    case B_COLOUR:
        if (st.vec) {
            const int* tv = dtask + st.task_off_v;
            const unsigned gv = (unsigned)std::max(1, std::min(st.grid, st.total_v));
            kb_colour<T><<<gv, TPB, 0, s>>>((const DColour<T>*)dp, tv, tv + st.nseg + 1, st.nseg, st.total_v, active,
                                            st.c, st.zs, 1);
        } else {
            kb_colour<T><<<g, TPB, 0, s>>>((const DColour<T>*)dp, t0, pid, st.nseg, st.total, active, st.c, st.zs, 0);
        }
        break;
    case B_RESTRICT:
        kb_restrict<T><<<g, TPB, 0, s>>>((const DRestrict<T>*)dp, t0, pid, st.nseg, st.total, active);
        break;
    case B_COARSE:
        kb_coarse<T><<<g, TPB, 0, s>>>((const DCoarse<T>*)dp, t0, pid, st.nseg, st.total, active);
        break;
    case B_PROLONG:
        kb_prolong<T><<<g, TPB, 0, s>>>((const DProlong<T>*)dp, t0, pid, st.nseg, st.total, active);
        break;
    case B_OUTER:
        kb_outer<T><<<g, TPB, 0, s>>>((const DOuter<T>*)dp, t0, pid, st.nseg, st.total, active, dpart);
        break;
    case B_AXPY:
        kb_axpy<T><<<g, TPB, 0, s>>>((const DAxpy<T>*)dp, t0, pid, st.nseg, st.total, active);
        break;
    }
}

// the batch structure a graph (and a tuning result) is valid for
template <class T>
static std::vector<long long> batch_key(BatchState& B, const BatchPlan<T>& P, const mps_solver_opts* o, int inner)
{
    std::vector<long long> k;
    k.push_back(sizeof(T));
    k.push_back(o->nu1);
    k.push_back(o->nu2);
    k.push_back(inner);
    k.push_back((long long)B.sub.size());
    for (auto& sc : B.sub) {
        k.push_back(sc->nlev);
        for (int l = 0; l < sc->nlev; l++) {
            k.push_back(sc->lev[l].nx);
            k.push_back(sc->lev[l].ny);
            k.push_back(sc->lev[l].nz);
        }
    }
    k.push_back((long long)P.desc.size());
    k.push_back((long long)P.task.size());
    return k;
}

// candidate grids, in blocks per SM
static const int kTuneBlocksPerSM[] = {1, 2, 4, 8, 16, 32};

// time the candidate grids on the colour pass of every depth (the passes
// read and write only the V-cycle state, which the first pass of a solve
// overwrites without reading)
template <class T>
static int autotune(Ctx& ctx, BatchState& B, BatchPlan<T>& P, const unsigned char* ddesc, const int* dtask)
{
    const int D = P.maxdepth;
    B.tune_grid.assign(D + 1, 8 * ctx.nsm);
    B.tune_vec.assign(D + 1, 0);
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    for (int d = 0; d < D; d++) {
        const BStep* st = nullptr;
        for (const BStep& s : P.body)
            if (s.kind == B_COLOUR && s.depth == d && s.zs == 0) { st = &s; break; }
        if (!st) continue;
        // the grid and the body (one cell or BATCH_W cells per thread) of
        // this depth's colour passes: every pair timed, the fastest kept
        float best = 1e30f;
        for (int vec = 0; vec < 2; vec++) {
            const int total = vec ? st->total_v : st->total;
            if (vec && st->total_v == st->total) continue;  // no level of this depth has the vector body
            for (int bps : kTuneBlocksPerSM) {
                const int g = bps * ctx.nsm;
                if (g > std::max(total, ctx.nsm)) break;
                BStep s2 = *st;
                s2.grid = g;
                s2.vec = vec;
                launch_step<T>(ctx.s, s2, ddesc, dtask, B.dst, B.dpart);  // warm
                CK(cudaEventRecord(a, ctx.s));
                for (int r = 0; r < 3; r++) launch_step<T>(ctx.s, s2, ddesc, dtask, B.dst, B.dpart);
                CK(cudaEventRecord(b, ctx.s));
                CK(cudaEventSynchronize(b));
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, a, b));
                if (ms < best * 0.97f) {
                    best = ms;
                    B.tune_grid[d] = g;
                    B.tune_vec[d] = vec;
                }
            }
        }
    }
    B.tune_grid[D] = B.tune_grid[0];
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CK(cudaGetLastError());
    return 0;
}

template <class T>
static void assign_grids(BatchState& B, BatchPlan<T>& P)
{
    auto grid_of = [&](const BStep& s) {
        if (s.kind == B_COARSE) return std::min(s.total, 4736);
        if (s.kind == B_OUTER || s.kind == B_AXPY) return B.tune_grid[0];
        return B.tune_grid[std::min(s.depth, (int)B.tune_grid.size() - 1)];
    };
    auto vec_of = [&](const BStep& s) {
        return s.kind == B_COLOUR && !B.tune_vec.empty() ? B.tune_vec[std::min(s.depth, (int)B.tune_vec.size() - 1)]
                                                         : 0;
    };
    for (BStep& s : P.pre) { s.grid = grid_of(s); s.vec = vec_of(s); }
    for (BStep& s : P.body) { s.grid = grid_of(s); s.vec = vec_of(s); }
}

// everything a batch's set-up sequence depends on: word size, options, every
// problem's description (sizes, buffers, boundary codes) and what its
// detection decides (finite inputs, convection, reaction field, uniform
// coefficient and its value, zero initial guess) -- not the data itself, so
// new right-hand sides or initial guesses in the same buffers replay
static std::vector<long long> prep_key_of(int wordsize, int np, const mps_problem* probs, const mps_solver_opts* o,
                                          int inner, const unsigned long long* det, const std::vector<char>& scanned)
{
    std::vector<long long> k;
    auto bytes = [&k](const void* p, size_t n) {
        const size_t w = (n + 7) / 8;
        const size_t at = k.size();
        k.resize(at + w, 0);
        std::memcpy(k.data() + at, p, n);
    };
    k.push_back(wordsize);
    k.push_back(inner);
    k.push_back(np);
    bytes(o, sizeof(*o));
    for (int p = 0; p < np; p++) {
        bytes(&probs[p], sizeof(mps_problem));
        k.push_back(scanned[p]);
        if (scanned[p]) {
            double v[9];
            std::memcpy(v, det + 9 * p, sizeof(v));
            bool finite = true;
            for (int q = 0; q < 6; q++) finite = finite && v[q] <= 1e308;
            const bool kuni = v[2] == 0.0;
            k.push_back(finite);
            k.push_back(v[0] == 0.0);  // no convection
            k.push_back(v[1] > 0.0);   // reaction field
            k.push_back(kuni);
            k.push_back(v[4] == 0.0);  // zero initial guess
            long long kb = 0;
            if (kuni) std::memcpy(&kb, &v[8], 8);  // the uniform coefficient enters the operators
            k.push_back(kb);
        }
    }
    return k;
}

template <class T>
static int batched_solve(Ctx& ctx, int np, const mps_problem* probs, const mps_solver_opts* o, mps_solve_info* infos)
{
    if (!ctx.batch) ctx.batch = new BatchState();
    BatchState& B = *ctx.batch;
    const int inner = o->inner_cycles > 0 ? o->inner_cycles : 2;
    // ---- per-problem contexts and set-up ----
    if ((int)B.sub.size() != np) {
        batch_release_graph(B);
        batch_release_prep(B);
        B.prep_key.clear();
        for (auto& sc : B.sub) sub_free(*sc);
        B.sub.clear();
        for (int p = 0; p < np; p++) {
            B.sub.emplace_back(new Ctx());
            if (sub_init(ctx, *B.sub.back())) { ctx.err.msg = "batched: sub-context set-up failed"; return MPS_ERR_CUDA; }
        }
    }
    CK(cudaEventRecord(ctx.e0, ctx.s));
    const long long launches0 = ctx.launches;
    // operator detection of every problem, then one device->host read (each
    // problem's set-up below then needs no synchronisation of its own);
    // problems whose arguments solve_impl will refuse are not scanned
    if (np > B.det_cap) {
        if (B.ddet) cudaFree(B.ddet);
        if (B.hdet) cudaFreeHost(B.hdet);
        if (B.ddd) cudaFree(B.ddd);
        if (B.hdd) cudaFreeHost(B.hdd);
        B.ddet = nullptr;
        B.hdet = nullptr;
        B.ddd = nullptr;
        B.hdd = nullptr;
        B.det_cap = 0;
        if (cudaMalloc((void**)&B.ddet, sizeof(unsigned long long) * 9 * np) != cudaSuccess ||
            cudaMallocHost((void**)&B.hdet, sizeof(unsigned long long) * 9 * np) != cudaSuccess ||
            cudaMalloc((void**)&B.ddd, sizeof(BDetect) * np) != cudaSuccess ||
            cudaMallocHost((void**)&B.hdd, sizeof(BDetect) * np) != cudaSuccess) {
            ctx.err.msg = "batched: detection buffers";
            return MPS_ERR_NOMEM;
        }
        B.det_cap = np;
    }
    std::vector<char> scanned(np, 0);
    int ndet = 0, blocks = 0;
    for (int p = 0; p < np; p++) {
        const mps_problem& q = probs[p];
        const mps_grid& g = q.g;
        if (g.lx < 1 || g.ly < 1 || g.lz < 1 || !q.dcoeff || !q.source || !q.soln ||
            (long long)g.lx * g.ly * g.lz >= (1LL << 31) / 2)
            continue;
        bool bcok = true;
        for (int f = 0; f < 6; f++) bcok = bcok && q.bc_code[f] >= 1 && q.bc_code[f] <= 5;
        if (!bcok) continue;
        BDetect& d = B.hdd[ndet++];
        d.vel = q.vel;
        d.reac = q.reac;
        d.dcoeff = q.dcoeff;
        d.source = q.source;
        d.soln = q.soln;
        d.nx = g.lx;
        d.ny = g.ly;
        d.nz = g.lz;
        d.rows = (unsigned)g.ly * (unsigned)g.lz;
        d.divNy.init((unsigned)g.ly);
        d.blk0 = blocks;
        d.nblk = (int)std::min<long long>(((long long)d.rows + 7) / 8, 256);  // a warp per row, 8 per block
        d.out = B.ddet + 9 * p;
        blocks += d.nblk;
        scanned[p] = 1;
    }
    CK(cudaMemsetAsync(B.ddet, 0, sizeof(unsigned long long) * 9 * np, ctx.s));
    if (ndet > 0) {
        CK(cudaMemcpyAsync(B.ddd, B.hdd, sizeof(BDetect) * ndet, cudaMemcpyHostToDevice, ctx.s));
        kb_detect<<<blocks, 256, 0, ctx.s>>>(B.ddd, ndet);
        CKL();
    }
    CK(cudaMemcpyAsync(B.hdet, B.ddet, sizeof(unsigned long long) * 9 * np, cudaMemcpyDeviceToHost, ctx.s));
    CK(cudaStreamSynchronize(ctx.s));
    // the set-up of every problem: run eagerly, captured as a graph at the
    // second call with the same key (then launched), or replayed
    const std::vector<long long> pkey = prep_key_of((int)sizeof(T), np, probs, o, inner, B.hdet, scanned);
    if (pkey != B.prep_key) {
        batch_release_prep(B);
        B.prep_key = pkey;
        B.prep_calls = 0;
    }
    const bool replay = B.prep_exec != nullptr;
    const bool capture = !replay && B.prep_calls == 1;
    B.prep_calls++;
    if (!B.start_e) {
        for (int i = 0; i < BatchState::NSET; i++) {
            CK(cudaStreamCreateWithFlags(&B.set_s[i], cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&B.set_e[i], cudaEventDisableTiming));
        }
        CK(cudaEventCreateWithFlags(&B.start_e, cudaEventDisableTiming));
    }
    auto setups = [&]() -> int {
        CK(cudaEventRecord(B.start_e, ctx.s));
        const int nset = std::min(np, (int)BatchState::NSET);
        for (int i = 0; i < nset; i++) CK(cudaStreamWaitEvent(B.set_s[i], B.start_e, 0));
        for (int p = 0; p < np; p++) {
            Ctx& sc = *B.sub[p];
            sc.s = B.set_s[p % nset];
            const mps_problem& q = probs[p];
            Inputs in;
            in.vel = q.vel;
            in.dcoeff = q.dcoeff;
            in.reac = q.reac;
            in.source = q.source;
            for (int f = 0; f < 6; f++) in.bcval[f] = q.bcval[f];
            in.sterm = q.mgridsterm;
            in.soln = q.soln;
            mps_solve_info inf;
            sc.launches = 0;
            int st = solve_impl(sc, &q.g, q.timederiv, q.dt, in, q.bc_code, o, &inf, 0, 1,
                                scanned[p] ? B.hdet + 9 * p : nullptr);
            ctx.launches += sc.launches;
            if (st) {
                ctx.err.msg = "batched problem " + std::to_string(p) + ": " + sc.err.msg;
                if (infos) { std::memset(&infos[p], 0, sizeof(mps_solve_info)); infos[p].status = st; }
                return st;
            }
            if (sc.sig.opclass != 0) {
                ctx.err.msg = "batched problem " + std::to_string(p) +
                              ": batched solves take the diffusion class (no convection, upwind flux, no transpose)";
                return MPS_ERR_BAD_ARG;
            }
        }
        for (int i = 0; i < nset; i++) {
            CK(cudaEventRecord(B.set_e[i], B.set_s[i]));
            CK(cudaStreamWaitEvent(ctx.s, B.set_e[i], 0));
        }
        for (int p = 0; p < np; p++) B.sub[p]->s = ctx.s;
        return 0;
    };
    if (replay) {
        CK(cudaGraphLaunch(B.prep_exec, ctx.s));
        ctx.launches += B.prep_kernels;
    } else if (capture) {
        CK(cudaStreamBeginCapture(ctx.s, cudaStreamCaptureModeThreadLocal));
        const long long k0 = ctx.launches;
        const int st = setups();
        B.prep_kernels = ctx.launches - k0;
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(ctx.s, &g);
        if (st == 0 && ce == cudaSuccess && g) ce = cudaGraphInstantiate(&B.prep_exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (st) return st;
        if (ce != cudaSuccess || !B.prep_exec) {  // not capturable: eager from now on for this key
            cudaGetLastError();
            B.prep_exec = nullptr;
            B.prep_calls = 2;
            ctx.launches = k0;  // the captured launches never ran
            for (int p = 0; p < np; p++) B.sub[p]->s = ctx.s;
            if (int st2 = setups()) return st2;
        } else {
            CK(cudaGraphLaunch(B.prep_exec, ctx.s));
        }
    } else if (int st = setups()) {
        return st;
    }
    // ---- plan, device tables ----
    const bool plan_fresh = !replay || !B.plan;
    if (plan_fresh) {
        auto fresh = std::make_shared<BatchPlan<T>>();
        plan_batch<T>(B, *fresh, o, inner);
        B.plan = fresh;
    }
    BatchPlan<T>& P = *static_cast<BatchPlan<T>*>(B.plan.get());
    auto grow = [&](auto*& ptr, size_t& cap, size_t n, size_t elem) -> int {
        if (n <= cap) return 0;
        batch_release_graph(B);
        B.up_desc.clear();
        B.up_task.clear();
        B.up_cells.clear();
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
        if (cudaMalloc((void**)&ptr, std::max<size_t>(n, 1) * elem) != cudaSuccess) return MPS_ERR_CUDA;
        cap = n;
        return 0;
    };
    int maxtasks = 0;
    for (const BStep& s : P.body)
        if (s.kind == B_OUTER) maxtasks = std::max(maxtasks, s.total);
    if (grow(B.ddesc, B.ddesc_cap, P.desc.size(), 1) || grow(B.dtask, B.dtask_cap, P.task.size(), sizeof(int)) ||
        grow(B.dpart, B.dpart_cap, 2 * (size_t)maxtasks, sizeof(double))) {
        ctx.err.msg = "batched: device tables";
        return MPS_ERR_NOMEM;
    }
    if (np > B.cap_prob) {
        batch_release_graph(B);
        cudaFree(B.dst);
        cudaFree(B.dncell);
        cudaFree(B.dcounter);
        cudaFree(B.dloops);
        B.dst = nullptr; B.dncell = nullptr; B.dcounter = nullptr; B.dloops = nullptr;
        B.cap_prob = 0;
        if (cudaMalloc((void**)&B.dst, sizeof(BState) * np) != cudaSuccess ||
            cudaMalloc((void**)&B.dncell, sizeof(long long) * np) != cudaSuccess ||
            cudaMalloc((void**)&B.dcounter, sizeof(unsigned)) != cudaSuccess ||
            cudaMalloc((void**)&B.dloops, sizeof(int)) != cudaSuccess) {
            ctx.err.msg = "batched: state";
            return MPS_ERR_NOMEM;
        }
        CK(cudaMemsetAsync(B.dcounter, 0, sizeof(unsigned), ctx.s));
        B.cap_prob = np;
        B.up_cells.clear();
    }
    std::vector<long long> hn(np);
    for (int p = 0; p < np; p++) hn[p] = (long long)probs[p].g.lx * probs[p].g.ly * probs[p].g.lz;
    // (a replayed plan is the one uploaded last, unless a buffer was reallocated)
    if ((plan_fresh || B.up_desc.empty() || B.up_cells.empty()) &&
        (P.desc != B.up_desc || P.task != B.up_task || hn != B.up_cells)) {
        CK(cudaMemcpyAsync(B.ddesc, P.desc.data(), P.desc.size(), cudaMemcpyHostToDevice, ctx.s));
        CK(cudaMemcpyAsync(B.dtask, P.task.data(), sizeof(int) * P.task.size(), cudaMemcpyHostToDevice, ctx.s));
        CK(cudaMemcpyAsync(B.dncell, hn.data(), sizeof(long long) * np, cudaMemcpyHostToDevice, ctx.s));
        B.up_desc = P.desc;
        B.up_task = P.task;
        B.up_cells = hn;
    }
    // every problem starts active (the state the loop's check kernel updates)
    kb_reset_state<<<(np + TPB - 1) / TPB, TPB, 0, ctx.s>>>(B.dst, np);
    CKL();
    CK(cudaMemsetAsync(B.dloops, 0, sizeof(int), ctx.s));
    const BState* active = B.dst;
    // ---- launch shapes ----
    std::vector<long long> key = batch_key<T>(B, P, o, inner);
    if (key != B.tune_key) {
        int st = autotune<T>(ctx, B, P, B.ddesc, B.dtask);
        if (st) return st;
        B.tune_key = key;
    }
    assign_grids<T>(B, P);
    // ---- initial residual and check ----
    for (const BStep& s : P.pre) {
        launch_step<T>(ctx.s, s, B.ddesc, B.dtask, active, B.dpart);
        CKL();
        const int* t0 = B.dtask + s.task_off;
        kb_check<<<s.nseg, TPB, 0, ctx.s>>>(t0, t0 + s.nseg + 1, B.dpart, B.dst, B.dncell, np, o->tol, o->tol_kind,
                                            o->maxit, 0, B.dcounter, B.dloops, o->maxit + 2, 0, 0);
        CKL();
    }
    CK(cudaMemsetAsync(B.dloops, 0, sizeof(int), ctx.s));
    // ---- the loop: one graph launch ----
    key.push_back((long long)(uintptr_t)B.ddesc);
    key.push_back((long long)(uintptr_t)B.dtask);
    key.push_back((long long)(uintptr_t)B.dpart);
    key.push_back((long long)(uintptr_t)B.dst);
    key.push_back(o->maxit);
    key.push_back(o->tol_kind);
    long long tb;
    std::memcpy(&tb, &o->tol, 8);
    key.push_back(tb);
    for (const BStep& s : P.body) {
        key.push_back(s.grid);
        key.push_back(s.vec);
    }
    if (key != B.graph_key) {
        batch_release_graph(B);
        CK(cudaGraphCreate(&B.graph, 0));
        cudaGraphConditionalHandle hc;
        CK(cudaGraphConditionalHandleCreate(&hc, B.graph, 1, cudaGraphCondAssignDefault));
        // (the struct holds a union without a default constructor: zeroed storage)
        alignas(cudaGraphNodeParams) unsigned char cpbuf[sizeof(cudaGraphNodeParams)];
        std::memset(cpbuf, 0, sizeof(cpbuf));
        cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cpbuf);
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hc;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CK(cudaGraphAddNode(&node, B.graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(ctx.s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        int nk = 0;
        const BStep* last_outer = nullptr;
        for (const BStep& s : P.body) {
            launch_step<T>(ctx.s, s, B.ddesc, B.dtask, active, B.dpart);
            nk++;
            if (s.kind == B_OUTER) last_outer = &s;
        }
        const int* t0 = B.dtask + last_outer->task_off;
        kb_check<<<last_outer->nseg, TPB, 0, ctx.s>>>(t0, t0 + last_outer->nseg + 1, B.dpart, B.dst, B.dncell, np,
                                                      o->tol, o->tol_kind, o->maxit, 1, B.dcounter, B.dloops,
                                                      o->maxit + 2, hc, 1);
        nk++;
        cudaGraph_t got = nullptr;
        cudaError_t ce = cudaStreamEndCapture(ctx.s, &got);
        if (ce != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            batch_release_graph(B);
            ctx.err.msg = std::string("batched: graph capture: ") + cudaGetErrorString(ce);
            return MPS_ERR_CUDA;
        }
        CK(cudaGraphInstantiate(&B.exec, B.graph, 0));
        B.graph_key = key;
        B.body_kernels = nk;
    }
    CK(cudaGraphLaunch(B.exec, ctx.s));
    // ---- results ----
    int loops = 0;
    std::vector<BState> hs(np);
    CK(cudaMemcpyAsync(hs.data(), B.dst, sizeof(BState) * np, cudaMemcpyDeviceToHost, ctx.s));
    CK(cudaMemcpyAsync(&loops, B.dloops, sizeof(int), cudaMemcpyDeviceToHost, ctx.s));
    auto unpack = [&]() -> int {  // every solution back to its caller's ghosted array
        for (int p = 0; p < np; p++) {
            Ctx& sc = *B.sub[p];
            const Lev& L0 = sc.lev[0];
            const long long n = (long long)L0.nx * L0.ny * L0.nz;
            k_unpack<double><<<nblk(n), TPB, 0, ctx.s>>>(L0, csplit<double>(sc.x64, L0), probs[p].soln);
            CKL();
            if (o->fill_ghosts) {
                const int mx = std::max(std::max(L0.ny * L0.nz, L0.nx * L0.nz), L0.nx * L0.ny);
                const double* zf[6];
                for (int f = 0; f < 6; f++) zf[f] = probs[p].bcval[f];
                k_fill_ghosts<<<nblk(mx), TPB, 0, ctx.s>>>(L0, probs[p].soln, zf[0], zf[1], zf[2], zf[3], zf[4],
                                                            zf[5]);
                CKL();
            }
        }
        return 0;
    };
    bool post_captured = false;
    if (B.prep_exec && !B.post_exec) {  // a repeated batch: capture the unpacking too
        CK(cudaStreamBeginCapture(ctx.s, cudaStreamCaptureModeThreadLocal));
        const long long k0 = ctx.launches;
        const int st = unpack();
        B.post_kernels = ctx.launches - k0;
        post_captured = true;
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(ctx.s, &g);
        if (st == 0 && ce == cudaSuccess && g) ce = cudaGraphInstantiate(&B.post_exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (st) return st;
        if (ce != cudaSuccess) {
            cudaGetLastError();
            B.post_exec = nullptr;
        }
    }
    if (B.post_exec) {
        CK(cudaGraphLaunch(B.post_exec, ctx.s));
        if (!post_captured) ctx.launches += B.post_kernels;
    } else if (int st = unpack()) {
        return st;
    }
    CK(cudaEventRecord(ctx.e1, ctx.s));
    CK(cudaStreamSynchronize(ctx.s));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx.e0, ctx.e1));
    ctx.launches += (long long)loops * B.body_kernels;
    int worst = MPS_OK;
    for (int p = 0; p < np; p++) {
        if (infos) {
            mps_solve_info& inf = infos[p];
            std::memset(&inf, 0, sizeof(inf));
            inf.status = hs[p].active ? MPS_ERR_NOT_CONVERGED : hs[p].status;
            inf.iters = hs[p].iters;
            inf.vcycles = hs[p].iters * inner;
            inf.levels = B.sub[p]->nlev;
            inf.rel_res = hs[p].rel;
            inf.rms_res = hs[p].rms;
            inf.rel_res0 = hs[p].rel0;
            inf.time_ms = ms;
            inf.launches = (int)(ctx.launches - launches0);
        }
        if (hs[p].status == MPS_ERR_NAN) worst = MPS_ERR_NAN;
    }
    return worst;
}

}  // namespace mps
