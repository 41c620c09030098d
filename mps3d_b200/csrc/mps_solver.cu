// mps_solver.cu -- host driver and C ABI of the B200 multigrid / Krylov
// solver.  One handle = one CUDA stream + a device workspace reused across
// calls with the same grid signature.
//
// Solve structure (correction scheme; equivalent to the reference's FAS
// V-cycle, mgridlib/mgridsteps.f90:384-579, because the operator is linear):
//   V(l): nu1 red-black GS sweeps; f_{l+1} = R(f_l - A_l u_l) (fused);
//         u_{l+1} = 0; V(l+1); u_l += P u_{l+1}; nu2 sweeps.
//   coarsest: u = A^{-1} f with a precomputed dense inverse.
// Outer loops: FP64 stationary V-cycle iteration; MIXED = FP64 residual +
// FP32 V-cycles + FP64 update (defect correction); FGMRES(m) right
// preconditioned by the V-cycle with FP64 Gram-Schmidt and Givens.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <memory>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/mps_linsolve.h"

#include <cstddef>

// The Fortran module include/mps_linsolve_c.f90 declares bind(C) twins of
// these structs with the same components in the same order; a Fortran
// compiler lays them out by the C rules.  These offsets are what that module
// (and the ctypes mirror in mps3d_b200/capi.py) assume: a change of a struct
// that moves one fails here instead of corrupting a caller's arguments.
static_assert(offsetof(mps_grid, llenx) == 16 && sizeof(mps_grid) == 40, "mps_grid layout");
static_assert(offsetof(mps_solver_opts, tol_kind) == 8 && offsetof(mps_solver_opts, ranks) == 28 &&
                  offsetof(mps_solver_opts, max_coarse) == 40 && offsetof(mps_solver_opts, flux) == 72 &&
                  sizeof(mps_solver_opts) == 80,
              "mps_solver_opts layout");
static_assert(offsetof(mps_solve_info, rel_res) == 16 && offsetof(mps_solve_info, launches) == 48 &&
                  sizeof(mps_solve_info) == 56,
              "mps_solve_info layout");
static_assert(offsetof(mps_profile, ms) == 32 && offsetof(mps_profile, precision_bytes) == 96 &&
                  offsetof(mps_profile, cells) == 104 && sizeof(mps_profile) == 112,
              "mps_profile layout");
static_assert(offsetof(mps_problem, timederiv) == 40 && offsetof(mps_problem, dt) == 48 &&
                  offsetof(mps_problem, vel) == 56 && offsetof(mps_problem, bc_code) == 88 &&
                  offsetof(mps_problem, bcval) == 112 && offsetof(mps_problem, mgridsterm) == 160 &&
                  offsetof(mps_problem, soln) == 168 && sizeof(mps_problem) == 176,
              "mps_problem layout");
#include "mps_kernels.cuh"
#include "mps_tma.cuh"
#include "mps_subcycle.cuh"

#include <cudaTypedefs.h>

namespace mps {

constexpr int MAXL = 24;
constexpr int MAX_DENSE = 1024;

static inline unsigned nblk(long long n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

// launch with the programmatic stream-serialization attribute: the kernel may
// be scheduled before its predecessor on the stream finishes, and waits for it
// in its first statement (pdl_wait); inside a captured graph this becomes a
// programmatic edge, which shortens the gap between dependent launches
template <class... KArgs, class... Args>
static cudaError_t pdl_launch(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args)
{
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}


// a kernel attribute (the shared-memory limit) set once per device: the call
// costs host time, and attributes belong to each device's context
template <class F>
static bool once_per_device(int dev, signed char* state, F&& set)
{
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    if (dev < 0 || dev >= 64) return set();
    if (state[dev] == 0) state[dev] = set() ? 1 : -1;
    return state[dev] == 1;
}

struct Err {
    int code = 0;
    std::string msg;
};

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            ctx.err.code = MPS_ERR_CUDA;                                                           \
            ctx.err.msg = std::string(#call) + ": " + cudaGetErrorString(e_);                     \
            return MPS_ERR_CUDA;                                                                   \
        }                                                                                          \
    } while (0)
#define CKL()                                                                                      \
    do {                                                                                           \
        ctx.launches++;                                                                            \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess) {                                                                   \
            ctx.err.code = MPS_ERR_CUDA;                                                           \
            ctx.err.msg = std::string("launch at ") + __FILE__ + ":" + std::to_string(__LINE__) +   \
                          ": " + cudaGetErrorString(e_);                                           \
            return MPS_ERR_CUDA;                                                                   \
        }                                                                                          \
    } while (0)

struct Arena {
    std::vector<void*> blocks;
    size_t bytes = 0;
    size_t limit = 0;  // 0: no cap; else get() fails once the arena would exceed it
    void* get(size_t n)
    {
        void* p = nullptr;
        if (n == 0) n = 16;
        if (limit && bytes + n > limit) return nullptr;
        if (cudaMalloc(&p, n) != cudaSuccess) return nullptr;
        if (cudaMemset(p, 0, n) != cudaSuccess) { cudaFree(p); return nullptr; }
        blocks.push_back(p);
        bytes += n;
        return p;
    }
    void clear()
    {
        for (void* p : blocks) cudaFree(p);
        blocks.clear();
        bytes = 0;
    }
};

template <class T>
struct Hier {
    T* U[MAXL][2] = {};  // two full split buffers (2*half) per level
    T* F[MAXL] = {};     // right-hand side (split)
    T* R[MAXL] = {};     // residual scratch (split)
    T* D[MAXL] = {};     // diagonal of the red rows (levels 1 .. nlev-2; the red pass written by the restriction)
    int ri[MAXL] = {}, bi[MAXL] = {};
    KOp<T> kop[MAXL];
    ROp<T> rop[MAXL];
    double* AinvT = nullptr;
    unsigned char* subimg = nullptr;  // solve-constant image of the one-block sub-cycle (k_sub_image)
    size_t subimg_bytes = 0;
    bool sub_ok = false;              // the image is current: the V-cycle may run k_subcycle
    double* Dprev = nullptr;  // the coarsest matrix whose inverse AinvT holds
    int* gj = nullptr;        // its inversion state (k_gauss_jordan)
};

struct Signature {
    int dims[3] = {0, 0, 0};
    int bc[6] = {0, 0, 0, 0, 0, 0};
    int hier = -1, ranks[3] = {0, 0, 0}, max_coarse = 0, opclass = -1, prec = -1, krylov = -1, restart = 0;
    int has_reac = -1, kuni = -1, transpose = -1;
    bool operator==(const Signature& o) const { return std::memcmp(this, &o, sizeof(Signature)) == 0; }
};

struct Prof {
    bool on = false;
    int level = 0;  // the level whose smoothing/transfer launches are timed
    std::vector<cudaEvent_t> ev;
    std::vector<int> cls;
    int used = 0;
    int count[MPS_PROF_NCLASS] = {};
    double ms[MPS_PROF_NCLASS] = {};
    int precision_bytes = 8, coeff_field = 0;
    long long cells = 0;
};

// a captured iteration, replayed with cudaGraphLaunch; keyed by everything
// that is baked into its kernel parameters
struct GraphKey {
    Signature sig;
    int kind = -1, prec = -1, inner = 0, nu1 = 0, nu2 = 0, nlev = 0, flux = 0, transpose = 0, prof = 0;
    double kc = 0, dexc = 0;
    const void* ws = nullptr;  // workspace identity (first arena block)
    bool operator==(const GraphKey& o) const
    {
        return sig == o.sig && kind == o.kind && prec == o.prec && inner == o.inner && nu1 == o.nu1 &&
               nu2 == o.nu2 && nlev == o.nlev && flux == o.flux && transpose == o.transpose && prof == o.prof &&
               kc == o.kc &&
               dexc == o.dexc && ws == o.ws;
    }
};
struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
    std::vector<cudaEvent_t> ev;  // profiling event-record nodes (pairs)
    std::vector<int> cls;
};

struct BatchState;

struct Ctx {
    int dev = 0;
    int nsm = 148;  // streaming multiprocessors of the device
    BatchState* batch = nullptr;  // batched solves (mps_linsolve_batched_dev)
    long long launches = 0;
    Prof prof;
    std::vector<GraphEntry> graphs;
    GraphEntry* capturing = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    Err err;
    Arena ar;       // grid-dependent workspace (both precisions)
    Arena kar;      // Krylov basis (FGMRES), keyed by (length, restart)
    long long kar_n = 0;
    int kar_m = 0;
    Arena inbuf;    // host-API staging of the inputs
    struct Lane {   // one host thread of the pageable copies: a stream, two pinned buffers
        cudaStream_t s = nullptr;
        double* pin[2] = {nullptr, nullptr};
        cudaEvent_t ev[2] = {nullptr, nullptr};
    };
    std::vector<Lane> lanes;  // created at the first host call with pageable arrays
    bool tma_ok = false;      // the shared-memory colour pass can run (set at workspace set-up)
    bool tma_allowed = true;  // MPS_TMA=0 at handle creation: the register-fed kernels only (for comparisons)
    bool red0_ready = false;  // the finest level's first red pass from zero was written by the outer residual
    bool redz[MAXL] = {};     // level l's first red pass from zero was written by the restriction into it
    bool sub_allowed = true;  // MPS_SUBCYCLE=0 at handle creation: one launch per pass on every level (for comparisons)
    int sub_l0 = -1;          // first level of the one-block sub-cycle (k_subcycle), -1: none
    size_t inbuf_bytes = 0;
    Signature sig;
    int nlev = 0;
    Lev lev[MAXL];
    Xfer xf[MAXL];
    Lin* dtab = nullptr;      // device prolongation tables of the current plan
    size_t dtab_n = 0;
    std::vector<Lin> htab;
    // FP64 coefficient pyramid (split cell fields)
    double* pk[MAXL] = {};
    double* preac[MAXL] = {};
    double* pv[3][MAXL] = {};
    double* dex64[MAXL] = {};
    float* k32[MAXL] = {};
    float* dex32[MAXL] = {};
    double* rows64[MAXL] = {};
    float* rows32[MAXL] = {};
    Hier<double> h64;
    Hier<float> h32;
    double* x64 = nullptr;  // outer iterate (mixed / fgmres)
    double* b64 = nullptr;
    KOp<double> kop64;      // fine-level FP64 operator for outer residuals
    ROp<double> rop64;
    double* dense = nullptr;
    double* gjM = nullptr;
    int* dstatus = nullptr;
    RedBuf rb;
    unsigned long long* dmax = nullptr;
    double* hpin = nullptr;  // pinned host scratch
    // FGMRES
    double* V = nullptr;
    void* Z = nullptr;
    double* w = nullptr;
    double* hcol = nullptr;
    double** Vptr = nullptr;
    double* dpart = nullptr;
    int mdot_blocks = 0;
    double* zero_face = nullptr;
    size_t zero_face_n = 0;
};

}  // namespace mps

struct mps_handle_s {
    mps::Ctx ctx;
};

namespace mps {

// ----------------------------------------------------------------------
static Lev make_lev(int nx, int ny, int nz, const double w[3], const double wl[3], const int bc[6])
{
    Lev L;
    std::memset(&L, 0, sizeof(L));
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.nh = (nx + 1) / 2;
    L.P = ((L.nh + 7) / 8) * 8;
    L.half = (long long)L.P * ny * nz;
    for (int f = 0; f < 6; f++) L.bc[f] = bc[f];
    for (int a = 0; a < 3; a++) L.per[a] = bc[2 * a] == BC_PERI;
    const int n[3] = {nx, ny, nz};
    for (int a = 0; a < 3; a++) {
        const double ww = w[a], wwl = wl[a];
        L.w[a] = ww;
        L.wl[a] = wwl;
        const double dl = 0.5 * (ww + wwl);
        L.cr[a] = 1.0 / (ww * ww);
        L.cl[a] = n[a] == 1 ? 1.0 / (wwl * wwl) : 1.0 / (dl * wwl);
        L.cp[a] = 1.0 / (dl * ww);
        L.dr[a] = 2.0 / (ww * ww);
        L.dlast[a] = 2.0 / (wwl * wwl);
    }
    L.uniform = (w[0] == wl[0] && w[1] == wl[1] && w[2] == wl[2]) ? 1 : 0;
    L.divP.init((unsigned)L.P);
    L.divNy.init((unsigned)ny);
    L.divG.init((unsigned)(L.P / 4));
    L.rows = (unsigned)ny * (unsigned)nz;
    return L;
}

static Lev make_lev_uniform(int nx, int ny, int nz, const double llen[3], const int bc[6])
{
    const double w[3] = {llen[0] / nx, llen[1] / ny, llen[2] / nz};
    return make_lev(nx, ny, nz, w, w, bc);
}

// level sizes and cell widths.  CELL = the reference (l/2 by integer division,
// mgridsteps.f90:21-23; dx = llen/l on every level, find_AX :724-726; coarsest
// when a per-rank size reaches LMIN=1, :512).  GEOM = l/2 with the odd cell of
// an odd size merged into the last coarse cell and exact widths; coarsest when
// a level has at most max_coarse cells.
static int plan_levels(const mps_grid* g, const mps_solver_opts* o, const int bc[6], Lev* lev, Xfer* xf,
                       std::string& why)
{
    int d[3] = {g->lx, g->ly, g->lz};
    const double llen[3] = {g->llenx, g->lleny, g->llenz};
    double w[3], wl[3];
    for (int a = 0; a < 3; a++) w[a] = wl[a] = llen[a] / d[a];
    int n = 0;
    const int* P = o->ranks;
    const bool cell = o->hierarchy == MPS_HIER_CELL;
    if (cell) {
        for (int a = 0; a < 3; a++)
            if (P[a] < 1 || d[a] % P[a] != 0) { why = "CELL hierarchy: size not divisible by ranks"; return -1; }
    }
    for (;;) {
        lev[n] = make_lev(d[0], d[1], d[2], w, wl, bc);
        long long cells = (long long)d[0] * d[1] * d[2];
        bool coarsest;
        if (cell)
            coarsest = d[0] / P[0] <= 1 || d[1] / P[1] <= 1 || d[2] / P[2] <= 1;
        else
            coarsest = cells <= o->max_coarse || (d[0] == 1 && d[1] == 1 && d[2] == 1);
        if (coarsest || n == MAXL - 1) {
            if (!coarsest) { why = "too many levels"; return -1; }
            if (cells > MAX_DENSE) { why = "coarsest level too large for the dense solve"; return -1; }
            return n + 1;
        }
        int c[3];
        double cw[3], cwl[3];
        Xfer X;
        std::memset(&X, 0, sizeof(X));
        X.geom = !cell;
        for (int a = 0; a < 3; a++) {
            if (cell) {
                int l = d[a] / P[a];
                if ((l & 1) && P[a] > 1) { why = "CELL hierarchy: odd per-rank size with several ranks"; return -1; }
                c[a] = P[a] * (l / 2);
                cw[a] = cwl[a] = llen[a] / c[a];
            } else if (d[a] == 1) {
                c[a] = 1;
                cw[a] = cwl[a] = wl[a];
            } else {
                c[a] = d[a] / 2;
                cw[a] = 2.0 * w[a];
                cwl[a] = (d[a] & 1) ? 2.0 * w[a] + wl[a] : w[a] + wl[a];
                if (c[a] == 1) cw[a] = cwl[a];
            }
            X.nf[a] = d[a];
            X.nc[a] = c[a];
            X.rf[a] = wl[a] / w[a];
            X.Rc[a] = cwl[a] / w[a];
            X.per[a] = bc[2 * a] == BC_PERI;
        }
        xf[n] = X;
        for (int a = 0; a < 3; a++) { d[a] = c[a]; w[a] = cw[a]; wl[a] = cwl[a]; }
        n++;
    }
}

template <class T>
static Split<T> cur(Hier<T>& H, const Lev& L, int l)
{
    Split<T> s;
    s.c[0] = H.U[l][H.ri[l]];
    s.c[1] = H.U[l][H.bi[l]] + L.half;
    return s;
}
template <class T>
static CSplit<T> ccur(Hier<T>& H, const Lev& L, int l)
{
    CSplit<T> s;
    s.c[0] = H.U[l][H.ri[l]];
    s.c[1] = H.U[l][H.bi[l]] + L.half;
    return s;
}
template <class T>
static CSplit<T> csplit(const T* base, const Lev& L)
{
    CSplit<T> s;
    s.c[0] = base;
    s.c[1] = base + L.half;
    return s;
}
template <class T>
static Split<T> split(T* base, const Lev& L)
{
    Split<T> s;
    s.c[0] = base;
    s.c[1] = base + L.half;
    return s;
}

// ---- finest-level profiling (events around launches on the handle's stream) ----
static void prof_begin(Ctx& ctx, int cls)
{
    Prof& P = ctx.prof;
    if (!P.on) return;
    if (ctx.capturing) {  // event-record node inside the graph being captured
        GraphEntry& G = *ctx.capturing;
        cudaEvent_t a;
        if (cudaEventCreate(&a) != cudaSuccess) return;
        G.ev.push_back(a);
        G.cls.push_back(cls);
        cudaEventRecordWithFlags(a, ctx.s, cudaEventRecordExternal);
        return;
    }
    if (P.used + 2 > (int)P.ev.size()) {
        for (int q = 0; q < 256; q++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return;
            P.ev.push_back(e);
        }
    }
    cudaEventRecord(P.ev[P.used], ctx.s);
    P.cls.push_back(cls);
}
static void prof_end(Ctx& ctx)
{
    Prof& P = ctx.prof;
    if (!P.on) return;
    if (ctx.capturing) {
        GraphEntry& G = *ctx.capturing;
        if (G.ev.size() != 2 * G.cls.size() - 1) return;
        cudaEvent_t b;
        if (cudaEventCreate(&b) != cudaSuccess) return;
        G.ev.push_back(b);
        cudaEventRecordWithFlags(b, ctx.s, cudaEventRecordExternal);
        return;
    }
    if (P.cls.size() * 2 != (size_t)P.used + 2) return;
    cudaEventRecord(P.ev[P.used + 1], ctx.s);
    P.used += 2;
}
// after a synchronize that followed a replay of G: add its event pairs
static void prof_collect_graph(Ctx& ctx, const GraphEntry& G)
{
    Prof& P = ctx.prof;
    if (!P.on) return;
    for (size_t q = 0; q < G.cls.size() && 2 * q + 1 < G.ev.size(); q++) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, G.ev[2 * q], G.ev[2 * q + 1]) == cudaSuccess) {
            P.ms[G.cls[q]] += ms;
            P.count[G.cls[q]]++;
        }
    }
}
static void destroy_graphs(Ctx& ctx)
{
    for (GraphEntry& G : ctx.graphs) {
        if (G.exec) cudaGraphExecDestroy(G.exec);
        for (cudaEvent_t e : G.ev) cudaEventDestroy(e);
    }
    ctx.graphs.clear();
}

static void prof_collect(Ctx& ctx)  // after a stream synchronize
{
    Prof& P = ctx.prof;
    for (size_t q = 0; q < P.cls.size() && (int)(2 * q + 1) < P.used; q++) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, P.ev[2 * q], P.ev[2 * q + 1]) == cudaSuccess) {
            P.ms[P.cls[q]] += ms;
            P.count[P.cls[q]]++;
        }
    }
    P.cls.clear();
    P.used = 0;
}

// Replay the captured graph for `key`, capturing `body` first when needed.
// Graphs hold kernel parameters (buffer pointers, operator constants) by
// value; the red/black buffer parities return to their start after an even
// number of sweeps per level, which the callers guarantee.  Returns the entry.
template <class F>
static int run_graph(Ctx& ctx, const GraphKey& key, GraphEntry** out, F&& body)
{
    GraphEntry* G = nullptr;
    for (GraphEntry& e : ctx.graphs)
        if (e.key == key) { G = &e; break; }
    if (!G) {
        if (ctx.graphs.size() >= 16) destroy_graphs(ctx);
        ctx.graphs.emplace_back();
        G = &ctx.graphs.back();
        G->key = key;
        cudaGraph_t graph = nullptr;
        const long long l0 = ctx.launches;
        if (cudaStreamBeginCapture(ctx.s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            ctx.graphs.pop_back();
            ctx.err.msg = "stream capture failed to start";
            return MPS_ERR_CUDA;
        }
        ctx.capturing = G;
        int st = body();
        ctx.capturing = nullptr;
        cudaError_t ce = cudaStreamEndCapture(ctx.s, &graph);
        if (st || ce != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            for (cudaEvent_t e : G->ev) cudaEventDestroy(e);
            ctx.graphs.pop_back();
            cudaGetLastError();
            if (!st) { ctx.err.msg = std::string("stream capture: ") + cudaGetErrorString(ce); st = MPS_ERR_CUDA; }
            return st;
        }
        G->kernels = (int)(ctx.launches - l0);
        ctx.launches = l0;
        ce = cudaGraphInstantiate(&G->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) {
            for (cudaEvent_t e : G->ev) cudaEventDestroy(e);
            ctx.graphs.pop_back();
            ctx.err.msg = std::string("graph instantiate: ") + cudaGetErrorString(ce);
            return MPS_ERR_CUDA;
        }
    }
    if (cudaGraphLaunch(G->exec, ctx.s) != cudaSuccess) {
        ctx.err.msg = "graph launch failed";
        return MPS_ERR_CUDA;
    }
    ctx.launches += G->kernels;
    *out = G;
    return 0;
}

static bool odd_periodic(const Lev& L)
{
    return (L.per[0] && (L.nx & 1)) || (L.per[1] && (L.ny & 1)) || (L.per[2] && (L.nz & 1));
}

// ---- transfer boxes ----
// coarse cells whose 2x2x2 children are regular cells of uniform coefficients
// away from odd periodic seams (false when an axis does not halve)
static bool restrict_box(const Lev& F, const Lev& C, Box& b)
{
    const int nf[3] = {F.nx, F.ny, F.nz}, nc[3] = {C.nx, C.ny, C.nz};
    for (int a = 0; a < 3; a++) {
        if (nf[a] != 2 * nc[a] && nf[a] != 2 * nc[a] + 1) return false;
        const bool seam = F.per[a] && (nf[a] & 1);
        const bool irregular_end = nf[a] != 2 * nc[a] || !F.uniform;  // unequal children
        b.lo[a] = seam ? 1 : 0;
        b.hi[a] = nc[a] - 1 - ((irregular_end || seam) ? 1 : 0);
        if (b.hi[a] < b.lo[a]) return false;
    }
    return true;
}
// fine cells whose bracketing coarse centres are regular cells (geometric hierarchy)
static bool prolong_box(const Lev& F, const Lev& C, const Xfer& X, Box& b)
{
    if (!X.geom) return false;
    const int nf[3] = {F.nx, F.ny, F.nz}, nc[3] = {C.nx, C.ny, C.nz};
    for (int a = 0; a < 3; a++) {
        if (nf[a] != 2 * nc[a] && nf[a] != 2 * nc[a] + 1) return false;
        const int creg = nc[a] - ((nf[a] != 2 * nc[a] || !F.uniform) ? 1 : 0);
        b.lo[a] = 1;
        b.hi[a] = 2 * creg - 3;
        // along y and z the regular rows go in pairs (2J+1, 2J+2) between
        // coarse rows J and J+1: an odd count leaves its last row to the shell
        if (a > 0 && ((b.hi[a] - b.lo[a] + 1) & 1)) b.hi[a]--;
        if (b.hi[a] < b.lo[a]) return false;
    }
    return true;
}
static long long box_cells(const Box& b)
{
    return (long long)(b.hi[0] - b.lo[0] + 1) * (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1);
}

// the launch description of the prolongation bulk (k_prolong_v) of fine
// level L with box pb and W cells per thread: the regular rows in 2 x 2
// blocks, their x ends, the rows outside the box, and the red cells of odd
// periodic seams; pp.blk0[4] blocks in all
static void prolong_form(const Lev& L, const Box& pb, int W, ProlongDiv& dv, Box& sb, ProlongDiv& sv,
                         ProlongParts& pp)
{
    const long long G = (L.nh + W - 1) / W;  // groups holding a cell (the rest of the P / W are pads)
    const long long rall = (long long)L.ny * L.nz;
    const long long rin = (long long)(pb.hi[1] - pb.lo[1] + 1) * (pb.hi[2] - pb.lo[2] + 1);
    dv.g.init((unsigned)G);
    dv.yin.init((unsigned)(pb.hi[1] - pb.lo[1] + 1));
    dv.yin2.init((unsigned)(pb.hi[1] - pb.lo[1] + 1) / 2);
    dv.nh.init((unsigned)((L.nx + 1) / 2));
    // groups with every cell in the box for both row parities: 2Wg >= lo,
    // 2W(g+1) - 1 <= hi
    dv.g_lo = (pb.lo[0] + 2 * W - 1) / (2 * W);
    dv.g_hi = (pb.hi[0] + 1) / (2 * W) - 1;
    const long long gin = dv.g_hi >= dv.g_lo ? dv.g_hi - dv.g_lo + 1 : 0;
    if (gin == 0) { dv.g_lo = 0; dv.g_hi = -1; }
    dv.gin.init((unsigned)std::max<long long>(gin, 1));
    dv.gout.init((unsigned)std::max<long long>(G - gin, 1));
    // red cells on odd periodic seams (read by the next red pass)
    const int sy = L.per[1] && (L.ny & 1), sz = L.per[2] && (L.nz & 1), sx = L.per[0] && (L.nx & 1);
    sb.lo[0] = 0;
    sb.hi[0] = L.nx - 1;
    sb.lo[1] = sy;
    sb.hi[1] = L.ny - 1 - sy;
    sb.lo[2] = sz;
    sb.hi[2] = L.nz - 1 - sz;
    const long long rin2 = (long long)(sb.hi[1] - sb.lo[1] + 1) * (sb.hi[2] - sb.lo[2] + 1);
    sv = dv;
    sv.yin.init((unsigned)(sb.hi[1] - sb.lo[1] + 1));
    pp.cnt[0] = (unsigned)(rin / 4 * gin);  // 2 x 2 row blocks
    pp.cnt[1] = (unsigned)(rin * (G - gin));
    pp.cnt[2] = (unsigned)((rall - rin) * G);
    pp.cnt[3] = odd_periodic(L) ? (unsigned)((rall - rin2) * ((L.nx + 1) / 2) + (sx ? 2 * rin2 : 0)) : 0u;
    pp.blk0[0] = 0;
    for (int q = 0; q < 4; q++) pp.blk0[q + 1] = pp.blk0[q] + nblk(pp.cnt[q]);
}

// colour passes and the outer residual: interior groups (no boundary code)
// and the shell as two parts of a launch (measured at 257^3: FP32 colour
// pass 54.6 against 58.3 us, FP64 91 against 126 us, outer residual 156
// against 201 us)
#ifndef MPS_COLOUR_SPLIT
#define MPS_COLOUR_SPLIT 1
#endif
#ifndef MPS_RESID_SPLIT
#define MPS_RESID_SPLIT 1
#endif

// the interior / shell decomposition of a level's groups of W cells
// (k_colourv_split, k_residv_split); false when the level has no interior
static bool make_split(const Lev& L, int W, ColourSplit& cs)
{
    // the interior: cells 1 .. n-2 along each axis; on a level with merged
    // last cells 1 .. n-3, whose faces all have the regular coefficients
    const int m = L.uniform ? 2 : 3;
    if (L.ny < m + 1 || L.nz < m + 1) return false;
    cs.g_lo = 1;
    cs.g_hi = (L.nx - m + 1) / (2 * W) - 1;
    if (cs.g_hi < cs.g_lo) return false;
    const unsigned G = (unsigned)((L.nh + W - 1) / W);
    const unsigned gin = (unsigned)(cs.g_hi - cs.g_lo + 1);
    const unsigned rin = (unsigned)(L.ny - m) * (unsigned)(L.nz - m);
    cs.gin.init(gin);
    cs.yin.init((unsigned)(L.ny - m));
    cs.gx.init(std::max(G - gin, 1u));
    cs.g.init(G);
    cs.n_in = rin * gin;
    cs.n_xe = rin * (G - gin);
    cs.n_face = ((unsigned)L.ny * (unsigned)L.nz - rin) * G;
    cs.nb_in = nblk(cs.n_in);
    cs.nb_xe = nblk(cs.n_xe);
    cs.nb_face = nblk(cs.n_face);
    cs.b.lo[0] = 0;
    cs.b.hi[0] = L.nx - 1;
    cs.b.lo[1] = 1;
    cs.b.hi[1] = L.ny - m;
    cs.b.lo[2] = 1;
    cs.b.hi[2] = L.nz - m;
    return true;
}

// the restriction bulk's interior coarse rows and groups (every fine cell
// evaluated has its neighbours inside the grid and regular faces: fine cells
// 1 .. n-2, or 1 .. n-3 on a level with merged last cells) and the rest; an
// empty interior leaves everything to the rest part
static RestrictSplit make_restrict_split(const Lev& F, const Lev& C, const Box& bx, int W)
{
    RestrictSplit rs;
    std::memset(&rs, 0, sizeof(rs));
    const int m = F.uniform ? 2 : 3;
    const int G = F.P / W;
    rs.J0 = std::max(bx.lo[1], 1);
    rs.K0 = std::max(bx.lo[2], 1);
    const int J1 = std::min(bx.hi[1], (F.ny - m - 1) / 2), K1 = std::min(bx.hi[2], (F.nz - m - 1) / 2);
    rs.ga = 1;
    rs.gb = ((F.nx - m - 1) / 2 - W + 1) / W;
    int nJ = J1 - rs.J0 + 1, nK = K1 - rs.K0 + 1, ng = rs.gb - rs.ga + 1;
    if (nJ < 1 || nK < 1 || ng < 1) {  // no interior: the rectangle is empty
        nJ = nK = 0;
        ng = 0;
        rs.ga = 0;
        rs.gb = -1;
    }
    rs.gin.init((unsigned)std::max(ng, 1));
    rs.yin.init((unsigned)std::max(nJ, 1));
    rs.gx.init((unsigned)std::max(G - ng, 1));
    rs.g.init((unsigned)G);
    rs.n_in = (unsigned)nJ * (unsigned)nK * (unsigned)ng;
    rs.n_xe = (unsigned)nJ * (unsigned)nK * (unsigned)(G - ng);
    rs.n_out = ((unsigned)C.ny * (unsigned)C.nz - (unsigned)nJ * (unsigned)nK) * (unsigned)G;
    rs.nb_in = nblk(rs.n_in);
    rs.nb_xe = nblk(rs.n_xe);
    rs.nb_out = nblk(rs.n_out);
    rs.rect.lo[0] = 0;
    rs.rect.hi[0] = C.nx - 1;
    rs.rect.lo[1] = rs.J0;
    rs.rect.hi[1] = rs.J0 + nJ - 1;
    rs.rect.lo[2] = rs.K0;
    rs.rect.hi[2] = rs.K0 + nK - 1;
    return rs;
}

// ---- the finest colour pass through shared memory (k_colour_tma) ----
#ifndef MPS_TMA_COLOUR
#define MPS_TMA_COLOUR 1
#endif
#ifndef MPS_TMA_LEVELS
#define MPS_TMA_LEVELS 1  // the finest level only
#endif
// tile rows and blocks per SM of the FP32 pass, measured on the 257^3 mixed
// solve (ms): 6 rows at 3 blocks per SM 12.72-12.75, 8 rows at 2 blocks
// 12.79-12.81, 5 rows at 4 blocks 13.40, 7 rows at 3 blocks 13.78
#ifndef MPS_TMA_BPS
#define MPS_TMA_BPS 3  // blocks per SM the tiling aims at
#endif
#ifndef MPS_TMA_TJ32
#define MPS_TMA_TJ32 6
#endif
#ifndef MPS_TMA_TJ64
#define MPS_TMA_TJ64 4
#endif
template <class T>
struct TmaShape {  // rows per block, one warp each; cells per thread
    static constexpr int TJ = sizeof(T) == 4 ? MPS_TMA_TJ32 : MPS_TMA_TJ64;
    static constexpr int W = 4;
};

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess && p)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

// 3-D map of one colour half (P x ny x nz elements) with boxes of `rows`
// full rows of one plane
template <class T>
static bool encode_half(CUtensorMap* m, const T* base, const Lev& L, int rows)
{
    auto fn = tensor_map_encoder();
    if (!fn) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)L.P, (cuuint64_t)L.ny, (cuuint64_t)L.nz};
    const cuuint64_t strides[2] = {(cuuint64_t)L.P * sizeof(T), (cuuint64_t)L.P * L.ny * sizeof(T)};
    const cuuint32_t box[3] = {(cuuint32_t)L.P, (cuuint32_t)rows, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
              const_cast<T*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the finest level's colour pass from a valid state with k_colour_tma;
// returns 1 when the pass was launched, 0 when this level or operator does
// not qualify (the caller runs the register-fed pass), < 0 on an error
template <class T>
static int colour_pass_tma(Ctx& ctx, Hier<T>& H, const KOp<T>& op, int l, int c, T* out, const T* fh)
{
    constexpr int TJ = TmaShape<T>::TJ, W = TmaShape<T>::W;
    const Lev& L = ctx.lev[l];
    // FP32 only: the FP64 pass measured slower through shared memory (104-117
    // against 87 us at 257^3), the FP32 pass faster (49.6 against 51.2 us)
    if (sizeof(T) != 4 || !ctx.tma_ok || L.P > 256 || op.dex[0] || L.ny < 3 || L.nz < 3) return 0;
    ColourSplit cs;
    if (!make_split(L, W, cs)) return 0;
    const bool kf = op.k[0] != nullptr;
    const int oc = c ^ 1;
    const T* uo = oc == 0 ? H.U[l][H.ri[l]] : H.U[l][H.bi[l]] + L.half;
    CUtensorMap mU, mKo, mKc, mF;
    std::memset(&mKo, 0, sizeof(mKo));
    std::memset(&mKc, 0, sizeof(mKc));
    if (!encode_half<T>(&mU, uo, L, TJ + 2) || !encode_half<T>(&mF, fh, L, TJ)) return 0;
    if (kf && (!encode_half<T>(&mKo, op.k[oc], L, TJ + 2) || !encode_half<T>(&mKc, op.k[c], L, TJ))) return 0;
    TmaColour tc;
    std::memset(&tc, 0, sizeof(tc));
    auto pad128 = [](unsigned elems) { return (unsigned)((elems * sizeof(T) + 127) / 128 * 128 / sizeof(T)); };
    tc.tile_elems = pad128((unsigned)L.P * (TJ + 2));
    tc.own_elems = pad128((unsigned)L.P * TJ);
    tc.slot_bytes = (unsigned)(L.P * sizeof(T)) * ((TJ + 2) * (kf ? 2 : 1) + TJ * (kf ? 2 : 1));
    const size_t smem = kf ? tma_smem_bytes<T, true>(tc) : tma_smem_bytes<T, false>(tc);
    if (smem > 220 * 1024) return 0;
    // tiles for the blocks that fit on an SM (shared memory, threads, at most
    // MPS_TMA_BPS): each tile streams its planes plus two halo planes, so
    // more tiles re-read more
    const int bps = std::max(1, std::min({(int)(227 * 1024 / (smem + 1024)), 2048 / (TJ * 32), MPS_TMA_BPS}));
    // the interior box of the split: rows 1 .. jhi, planes 1 .. khi (one cell
    // short of merged last cells); the shell blocks take every other row
    tc.jhi = cs.b.hi[1];
    tc.khi = cs.b.hi[2];
    if (cs.b.lo[1] != 1 || cs.b.lo[2] != 1 || tc.jhi < 1 || tc.khi < 1) return 0;
    tc.njb = (tc.jhi + TJ - 1) / TJ;
    const int want = std::max(1, ctx.nsm * bps / tc.njb);
    tc.tk = std::max(1, (tc.khi + want - 1) / want);
    tc.nkb = (tc.khi + tc.tk - 1) / tc.tk;
    tc.ntile = tc.njb * tc.nkb;
    tc.g_lo = cs.g_lo;
    tc.g_hi = cs.g_hi;
    tc.n_xe = cs.n_xe;
    tc.n_face = cs.n_face;
    const unsigned nsh = tc.n_xe + tc.n_face;
    tc.nb_shell = std::min<unsigned>((nsh + TJ * 32 - 1) / (TJ * 32), (unsigned)ctx.nsm * 4);
    tc.flag = ctx.rb.out + 3;
    auto launch = [&](auto kern) -> int {
        const cudaError_t e = pdl_launch(kern, tc.ntile + tc.nb_shell, TJ * 32, smem, ctx.s, L, op, c, ccur(H, L, l),
                                         out, fh, cs, tc, mU, mKo, mKc, mF);
        if (e != cudaSuccess) {
            ctx.err.code = MPS_ERR_CUDA;
            ctx.err.msg = std::string("k_colour_tma launch: ") + cudaGetErrorString(e);
            return -1;
        }
        return 1;
    };
    if (L.uniform) return kf ? launch(k_colour_tma<T, W, TJ, true, true>) : launch(k_colour_tma<T, W, TJ, false, true>);
    return kf ? launch(k_colour_tma<T, W, TJ, true, false>) : launch(k_colour_tma<T, W, TJ, false, false>);
}

// the attributes the shared-memory colour pass needs, set outside any stream
// capture (at workspace set-up); false when the device or driver cannot run it
static bool tma_prepare(int dev)
{
    static signed char state[64] = {};
    if (!MPS_TMA_COLOUR || !tensor_map_encoder()) return false;
    return once_per_device(dev, state, [] {
        const int bytes = 220 * 1024;
        auto set = [&](auto kern) {
            return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
        };
        constexpr int W32 = TmaShape<float>::W, J32 = TmaShape<float>::TJ;
        constexpr int W64 = TmaShape<double>::W, J64 = TmaShape<double>::TJ;
        bool ok = set(k_colour_tma<float, W32, J32, true, true>) && set(k_colour_tma<float, W32, J32, false, true>) &&
                  set(k_colour_tma<float, W32, J32, true, false>) && set(k_colour_tma<float, W32, J32, false, false>) &&
                  set(k_colour_tma<double, W64, J64, true, true>) && set(k_colour_tma<double, W64, J64, false, true>) &&
                  set(k_colour_tma<double, W64, J64, true, false>) && set(k_colour_tma<double, W64, J64, false, false>);
        if (!ok) cudaGetLastError();
        return ok;
    });
}

// the explicit-row colour pass in two parts (k_colourv_split_rop); cells
// per thread measured on the 129^3 SG step (finest pass FP32 / FP64, live
// events): one cell 17.7 / 24.7 us, 2 / 1 cells 17.3 / 24.9, 2 / 2 cells
// 17.2 / 25.4, 4 / 2 cells 21.3 / 25.5, against 20.9 / 28.8 us for k_colour
// (one cell per thread, boundary code everywhere); the solve times move
// by less than their noise (2.13-2.19 / 1.46-1.51 ms)
#ifndef MPS_ROP_SPLIT
#define MPS_ROP_SPLIT 1
#endif
#ifndef MPS_ROP_W32
#define MPS_ROP_W32 1
#endif
#ifndef MPS_ROP_W64
#define MPS_ROP_W64 1
#endif

// ---- one colour pass ----
template <class T, class Op>
static int colour_pass(Ctx& ctx, Hier<T>& H, const Op& op, int l, int c, int zero_state)
{
    const Lev& L = ctx.lev[l];
    const unsigned nb = nblk((long long)L.P * L.rows);
    T* out;
    const T* fh = H.F[l] + (c ? L.half : 0);
    if (c == 0) out = H.U[l][H.ri[l] ^ 1];
    else out = H.U[l][H.bi[l] ^ 1] + L.half;
    if (l == ctx.prof.level) prof_begin(ctx, MPS_PROF_SMOOTH);
    if constexpr (std::is_same<Op, KOp<T>>::value) {
        if (zero_state == 2 && c == 0 && H.D[l]) {  // from zero: f / diag, elementwise
            pdl_launch(k_red_from_zero<T>, nb, TPB, 0, ctx.s, L, (const T*)fh, (const T*)H.D[l], out);
            if (l == ctx.prof.level) prof_end(ctx);
            CKL();
            H.ri[l] ^= 1;
            return 0;
        }
    }
    if constexpr (std::is_same<Op, KOp<T>>::value) {
        if (l <= MPS_TMA_LEVELS - 1 && zero_state == 0) {
            const int r = colour_pass_tma<T>(ctx, H, op, l, c, out, fh);
            if (r < 0) return MPS_ERR_CUDA;
            if (r == 1) {
                if (l == ctx.prof.level) prof_end(ctx);
                CKL();
                if (c == 0) H.ri[l] ^= 1;
                else H.bi[l] ^= 1;
                return 0;
            }
        }
    }
    if constexpr (std::is_same<Op, KOp<T>>::value) {
        if (L.uniform || L.nx >= 16) {
            // vector kernel, W cells per thread (faces at a merged last cell
            // take their own coefficients inside the row evaluation); the
            // levels below the finest have their own shape
            auto launch = [&](auto wc, auto mbc) {
                constexpr int W = decltype(wc)::value, MB = decltype(mbc)::value;
                ColourSplit cs;
                if (MPS_COLOUR_SPLIT && make_split(L, W, cs)) {
                    // interior groups without boundary code, the shell apart
                    const unsigned nbt = cs.nb_in + cs.nb_xe + cs.nb_face;
                    auto go = [&](auto uc) {
                        constexpr bool UNI = decltype(uc)::value;
                        if (zero_state == 2) {
                            pdl_launch(k_colourv_split<T, W, ZeroU<T>, MB, UNI>, nbt, TPB, 0, ctx.s, L, op, c, ZeroU<T>(),
                                       out, fh, cs);
                        } else if (zero_state == 1) {
                            OtherOnlyU<T> u;
                            u.c = c;
                            u.other = c == 0 ? H.U[l][H.bi[l]] + L.half : H.U[l][H.ri[l]];
                            pdl_launch(k_colourv_split<T, W, OtherOnlyU<T>, MB, UNI>, nbt, TPB, 0, ctx.s, L, op, c, u, out,
                                       fh, cs);
                        } else {
                            pdl_launch(k_colourv_split<T, W, CSplit<T>, MB, UNI>, nbt, TPB, 0, ctx.s, L, op, c,
                                       ccur(H, L, l), out, fh, cs);
                        }
                    };
                    if (L.uniform) go(std::true_type());
                    else go(std::false_type());
                    return;
                }
                FastDiv dg;
                dg.init((unsigned)(L.P / W));
                const unsigned nbv = nblk((long long)(L.P / W) * L.rows);
                if (zero_state == 2) {
                    pdl_launch(k_colourv<T, W, ZeroU<T>, MB>, nbv, TPB, 0, ctx.s, L, op, c, ZeroU<T>(), out, fh, dg);
                } else if (zero_state == 1) {
                    OtherOnlyU<T> u;
                    u.c = c;
                    u.other = c == 0 ? H.U[l][H.bi[l]] + L.half : H.U[l][H.ri[l]];
                    pdl_launch(k_colourv<T, W, OtherOnlyU<T>, MB>, nbv, TPB, 0, ctx.s, L, op, c, u, out, fh, dg);
                } else {
                    pdl_launch(k_colourv<T, W, CSplit<T>, MB>, nbv, TPB, 0, ctx.s, L, op, c, ccur(H, L, l), out, fh,
                               dg);
                }
            };
            if (l == 0)
                launch(std::integral_constant<int, ColourShape<T>::W>(), std::integral_constant<int, ColourShape<T>::MINB>());
            else if (l == 1)
                launch(std::integral_constant<int, CoarseShape<T>::W>(), std::integral_constant<int, CoarseShape<T>::MINB>());
            else
                launch(std::integral_constant<int, SmallShape<T>::W>(), std::integral_constant<int, SmallShape<T>::MINB>());
            if (l == ctx.prof.level) prof_end(ctx);
            CKL();
            if (c == 0) H.ri[l] ^= 1;
            else H.bi[l] ^= 1;
            return 0;
        }
    }
    if constexpr (std::is_same<Op, ROp<T>>::value) {
        // explicit rows: interior groups W cells per thread, the shell cell by cell
        constexpr int W = sizeof(T) == 4 ? MPS_ROP_W32 : MPS_ROP_W64;
        ColourSplit cs;
        if (MPS_ROP_SPLIT && L.nx >= 16 && make_split(L, W, cs)) {
            const unsigned nbt = cs.nb_in + cs.nb_xe + cs.nb_face;
            if (zero_state == 2) {
                pdl_launch(k_colourv_split_rop<T, W, ZeroU<T>>, nbt, TPB, 0, ctx.s, L, op, c, ZeroU<T>(), out, fh, cs);
            } else if (zero_state == 1) {
                OtherOnlyU<T> u;
                u.c = c;
                u.other = c == 0 ? H.U[l][H.bi[l]] + L.half : H.U[l][H.ri[l]];
                pdl_launch(k_colourv_split_rop<T, W, OtherOnlyU<T>>, nbt, TPB, 0, ctx.s, L, op, c, u, out, fh, cs);
            } else {
                pdl_launch(k_colourv_split_rop<T, W, CSplit<T>>, nbt, TPB, 0, ctx.s, L, op, c, ccur(H, L, l), out, fh,
                           cs);
            }
            if (l == ctx.prof.level) prof_end(ctx);
            CKL();
            if (c == 0) H.ri[l] ^= 1;
            else H.bi[l] ^= 1;
            return 0;
        }
    }
    if (zero_state == 2) {  // whole state zero
        pdl_launch(k_colour<T, Op, ZeroU<T>>, nb, TPB, 0, ctx.s, L, op, c, ZeroU<T>(), out, fh);
    } else if (zero_state == 1) {  // colour c zero, other colour valid
        OtherOnlyU<T> u;
        u.c = c;
        u.other = c == 0 ? H.U[l][H.bi[l]] + L.half : H.U[l][H.ri[l]];
        pdl_launch(k_colour<T, Op, OtherOnlyU<T>>, nb, TPB, 0, ctx.s, L, op, c, u, out, fh);
    } else {
        pdl_launch(k_colour<T, Op, CSplit<T>>, nb, TPB, 0, ctx.s, L, op, c, ccur(H, L, l), out, fh);
    }
    if (l == ctx.prof.level) prof_end(ctx);
    CKL();
    if (c == 0) H.ri[l] ^= 1;
    else H.bi[l] ^= 1;
    return 0;
}

template <class T>
static int coarse_solve(Ctx& ctx, Hier<T>& H, int l)
{
    const Lev& L = ctx.lev[l];
    const int n = L.nx * L.ny * L.nz;
    pdl_launch(k_coarse_solve<T>, 1, 512, n * sizeof(double), ctx.s, L, H.AinvT, csplit<T>(H.F[l], L), cur(H, L, l));
    CKL();
    return 0;
}

// ---- the small levels in one block (k_subcycle) ----
// the shared-memory limit of the sub-cycle kernels, set outside any stream
// capture (at workspace set-up)
static bool sub_prepare(int dev)
{
    static signed char state[64] = {};
    return once_per_device(dev, state, [] {
        auto set = [](const void* kern) {
            return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SUB_SMEM_MAX) == cudaSuccess;
        };
        const bool ok = set((const void*)k_subcycle<float, false, false>) && set((const void*)k_subcycle<float, true, false>) &&
                        set((const void*)k_subcycle<float, false, true>) && set((const void*)k_subcycle<float, true, true>) &&
                        set((const void*)k_subcycle<double, false, false>) && set((const void*)k_subcycle<double, true, false>) &&
                        set((const void*)k_subcycle<double, false, true>) && set((const void*)k_subcycle<double, true, true>);
        if (!ok) cudaGetLastError();
        return ok;
    });
}

// first level of the one-block sub-cycle, or -1: the geometric hierarchy, a
// level below the finest with at most SUB_MAX_CELLS cells and at most
// SUB_MAXL levels from it to the coarsest (two at least), and no odd periodic
// size on those levels (cells of one colour would touch, and in-place passes
// would read new values)
static int sub_first_level(const Ctx& ctx, const mps_solver_opts* o)
{
    if (o->hierarchy != MPS_HIER_GEOM) return -1;
    const int nl = ctx.nlev;
    int l0 = -1;
    for (int l = 1; l < nl - 1; l++) {
        const Lev& L = ctx.lev[l];
        if ((long long)L.nx * L.ny * L.nz <= SUB_MAX_CELLS && nl - l <= SUB_MAXL) { l0 = l; break; }
    }
    if (l0 < 0) return -1;
    for (int l = l0; l < nl; l++) {
        if (odd_periodic(ctx.lev[l])) return -1;
        if (l < nl - 1 && !ctx.xf[l].geom) return -1;
    }
    return l0;
}

// the ghosted row pitch of a level in the block: nx+2, or 24 for FP32 rows of
// 16 cells (8 per colour), so that the four rows a warp takes in a colour pass
// (stride-2 accesses) fall on distinct banks
template <class T>
static int sub_gx(const Lev& L)
{
    return (sizeof(T) == 4 && L.nh == 8 && L.nx + 2 <= 24) ? 24 : L.nx + 2;
}

// one level of the block's plan: Lev's sizes, widths and boundary flags
template <class T>
static SubGeo<T> sub_geo(const Lev& L)
{
    SubGeo<T> G;
    std::memset(&G, 0, sizeof(G));
    G.nx = L.nx; G.ny = L.ny; G.nz = L.nz; G.nh = L.nh;
    G.rows = L.ny * L.nz;
    G.rc = SUB_TPB / L.nh;
    G.rn = SUB_TPB / L.nx;
    G.gx = sub_gx<T>(L);
    G.gy = L.ny + 2;
    G.pitch = L.P;
    for (int a = 0; a < 3; a++) {
        G.per |= L.per[a] ? 1 << a : 0;
        G.w[a] = (T)L.w[a];
        G.wl[a] = (T)L.wl[a];
    }
    for (int f = 0; f < 6; f++) G.dirc |= L.bc[f] == BC_DIRC && !L.per[f / 2] ? 1 << f : 0;
    G.dnh.init((unsigned)L.nh);
    G.dny.init((unsigned)L.ny);
    G.dnx.init((unsigned)L.nx);
    return G;
}

// the axis entries of one level (ghosted strides 1, nx+2, (nx+2)(ny+2)): the
// face coefficients of fcoef / dcoef by position, periodic faces wrapping
template <class T>
static void sub_axes(const Lev& L, SubAx<T>* out)
{
    const int n3[3] = {L.nx, L.ny, L.nz};
    const int gx = sub_gx<T>(L);
    const int st3[3] = {1, gx, gx * (L.ny + 2)};
    int e = 0;
    for (int a = 0; a < 3; a++) {
        const int n = n3[a], st = st3[a];
        const bool per = L.per[a] != 0;
        const bool dm = !per && L.bc[2 * a] == BC_DIRC, dp = !per && L.bc[2 * a + 1] == BC_DIRC;
        for (int p = 0; p < n; p++, e++) {
            SubAx<T> x;
            if (p > 0) { x.om = -st; x.cm = (T)(p == n - 1 ? L.cl[a] : L.cr[a]); }
            else if (per) { x.om = (n - 1) * st; x.cm = (T)(n == 1 ? L.cl[a] : L.cp[a]); }
            else { x.om = -st; x.cm = dm ? (T)(n == 1 ? L.dlast[a] : L.dr[a]) : T(0); }
            if (p < n - 1) { x.op = st; x.cp = (T)(p + 1 == n - 1 ? L.cp[a] : L.cr[a]); }
            else if (per) { x.op = -(n - 1) * st; x.cp = (T)L.cl[a]; }
            else { x.op = st; x.cp = dp ? (T)L.dlast[a] : T(0); }
            out[e] = x;
        }
    }
}

// the block's plan from level l0 for word type T: shared-memory layout
// (dynamic fields, the solve-constant image, tables), per-level geometry,
// axis entries and prolongation brackets.  false when it does not fit.
template <class T>
static bool sub_layout_with(const Ctx& ctx, int l0, bool kf, bool df, const mps_solver_opts* o, SubPlan<T>& P,
                            size_t& smem, bool ainv_in_smem);

// the layout with the coarsest inverse staged in shared memory when that fits,
// else read from device memory by the coarsest solve
template <class T>
static bool sub_layout(const Ctx& ctx, int l0, bool kf, bool df, const mps_solver_opts* o, SubPlan<T>& P,
                       size_t& smem)
{
    return sub_layout_with<T>(ctx, l0, kf, df, o, P, smem, true) ||
           sub_layout_with<T>(ctx, l0, kf, df, o, P, smem, false);
}

template <class T>
static bool sub_layout_with(const Ctx& ctx, int l0, bool kf, bool df, const mps_solver_opts* o, SubPlan<T>& P,
                            size_t& smem, bool ainv_in_smem)
{
    std::memset(&P, 0, sizeof(P));
    if (l0 < 1 || ctx.nlev - l0 < 2) return false;
    const int nl = ctx.nlev - l0;
    P.nl = nl;
    P.nu1 = o->nu1;
    P.nu2 = o->nu2;
    P.only_black = o->nu2 >= 1;
    int nax = 0, nrow = 0, nlin = 0;
    long long off = 0;  // elements of T: u (ghosted) and f of every level
    for (int s = 0; s < nl; s++) {
        const Lev& L = ctx.lev[l0 + s];
        // a row per thread at least in every loop; the tables' capacities
        if (L.nx > SUB_TPB || nax + L.nx + L.ny + L.nz > SUB_MAX_AX || nrow + L.ny * L.nz > SUB_MAX_ROWS)
            return false;
        P.geo[s] = sub_geo<T>(L);
        P.geo[s].ax0 = nax;
        P.geo[s].row0 = nrow;
        sub_axes<T>(L, P.ax + nax);
        nax += L.nx + L.ny + L.nz;
        nrow += L.ny * L.nz;
        P.ou[s] = (int)off; off += (long long)sub_gx<T>(L) * (L.ny + 2) * (L.nz + 2);
        P.of[s] = (int)off; off += (long long)L.nx * L.ny * L.nz;
        if (s < nl - 1) {
            const Xfer& X = ctx.xf[l0 + s];
            const int nf[3] = {L.nx, L.ny, L.nz};
            for (int a = 0; a < 3; a++) {
                P.lin0[s][a] = nlin;
                for (int i = 0; i < nf[a]; i++) {
                    Lin e;
                    geom_lin(X, a, i, e.j0, e.j1, e.t);
                    P.lin[nlin + i].j0 = e.j0;
                    P.lin[nlin + i].j1 = e.j1;
                    P.lin[nlin + i].t = (T)e.t;
                }
                nlin += nf[a];
            }
            // lanes per coarse cell: up to 8, while the coarse cells fill the
            // block and a coarse row fits one trip
            const Lev& C = ctx.lev[l0 + s + 1];
            const long long nc = (long long)C.nx * C.ny * C.nz;
            int lg = 3;
            while (lg > 0 && (nc << lg > SUB_TPB || (C.nx << lg) > SUB_TPB)) lg--;
            P.rlog[s] = lg;
            P.rrows[s] = (SUB_TPB >> lg) / C.nx;
        }
    }
    // the solve-constant image: coefficients (ghosted), diagonal extras, inverse
    off = (off + 1) & ~1LL;  // 16-byte boundary for either word size
    off = ((off * (long long)sizeof(T) + 15) & ~15LL) / (long long)sizeof(T);
    P.img_off = (int)(off * sizeof(T));
    for (int s = 0; s < nl; s++) {
        const Lev& L = ctx.lev[l0 + s];
        P.ok[s] = kf ? (int)off : -1; off += kf ? (long long)sub_gx<T>(L) * (L.ny + 2) * (L.nz + 2) : 0;
        P.od[s] = df ? (int)off : -1; off += df ? (long long)L.nx * L.ny * L.nz : 0;
    }
    size_t bytes = ((size_t)off * sizeof(T) + 15) & ~(size_t)15;
    const Lev& Cc = ctx.lev[ctx.nlev - 1];
    const long long ncs = (long long)Cc.nx * Cc.ny * Cc.nz;
    P.ainv_off = ainv_in_smem ? (int)bytes : -1;
    if (ainv_in_smem) bytes += ((size_t)(ncs * ncs) * sizeof(double) + 15) & ~(size_t)15;
    // the tables are part of the image too (built once per solve)
    P.lin_off = (int)bytes;
    bytes += ((size_t)nlin * sizeof(SubLin<T>) + 15) & ~(size_t)15;
    P.ax_off = (int)bytes;
    bytes += ((size_t)nax * sizeof(SubAx<T>) + 15) & ~(size_t)15;
    P.row_off = (int)bytes;
    bytes += ((size_t)nrow * sizeof(SubRow) + 15) & ~(size_t)15;
    P.img_bytes = (int)(bytes - P.img_off);
    P.nlin = nlin;
    P.nax = nax;
    P.nrow = nrow;
    int g = 32;
    while (g > 1 && ncs * g > SUB_TPB) g >>= 1;
    P.gsz = g;
    smem = bytes;
    return bytes <= (size_t)SUB_SMEM_MAX;
}

static cudaError_t sub_launch(const void* kern, size_t smem, cudaStream_t s, void** args)
{
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(SUB_TPB);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, kern, args);
}

// build the solve-constant image of hierarchy H (after its coefficient
// pyramid and coarsest inverse are set up); H.sub_ok tells the V-cycle
template <class T>
static int sub_image(Ctx& ctx, Hier<T>& H, const KOp<T>* ops, const mps_solver_opts* o)
{
    H.sub_ok = false;
    const int l0 = ctx.sub_l0;
    if (l0 < 1 || !H.subimg) return 0;
    const bool kf = ops[l0].k[0] != nullptr, df = ops[l0].dex[0] != nullptr;
    std::unique_ptr<SubPlan<T>> pp(new SubPlan<T>);
    SubPlan<T>& P = *pp;
    size_t smem = 0;
    if (!sub_layout<T>(ctx, l0, kf, df, o, P, smem) || (size_t)P.img_bytes > H.subimg_bytes) return 0;
    for (int s = 0; s < P.nl; s++)
        for (int c = 0; c < 2; c++) {
            P.k[s][c] = ops[l0 + s].k[c];
            P.dex[s][c] = ops[l0 + s].dex[c];
        }
    const Lev& Cc = ctx.lev[ctx.nlev - 1];
    int ncs = Cc.nx * Cc.ny * Cc.nz;
    unsigned char* img = H.subimg;
    const double* ainv = H.AinvT;
    void* args[] = {(void*)&P, (void*)&img, (void*)&ainv, (void*)&ncs};
    const void* kern = kf ? (df ? (const void*)k_sub_image<T, true, true> : (const void*)k_sub_image<T, true, false>)
                          : (df ? (const void*)k_sub_image<T, false, true> : (const void*)k_sub_image<T, false, false>);
    sub_launch(kern, 0, ctx.s, args);
    CKL();
    H.sub_ok = true;
    return 0;
}

// the V-cycle from level l0 (zero guess) to the coarsest and back in one
// launch; -1 when it does not apply (the per-level launches run instead)
template <class T>
static int subcycle(Ctx& ctx, Hier<T>& H, const KOp<T>* ops, int l0, const mps_solver_opts* o)
{
    if (!H.sub_ok || l0 != ctx.sub_l0) return -1;
    const bool kf = ops[l0].k[0] != nullptr, df = ops[l0].dex[0] != nullptr;
    std::unique_ptr<SubPlan<T>> pp(new SubPlan<T>);  // the kernel parameter (copied at launch)
    SubPlan<T>& P = *pp;
    size_t smem = 0;
    if (!sub_layout<T>(ctx, l0, kf, df, o, P, smem)) return -1;
    P.kc = ops[l0].kc;
    P.dexc = ops[l0].dexc;
    CSplit<T> fin = csplit<T>(H.F[l0], ctx.lev[l0]);
    Split<T> uout = cur(H, ctx.lev[l0], l0);
    const uint4* img = reinterpret_cast<const uint4*>(H.subimg);
    const double* ainv = H.AinvT;
    void* args[] = {(void*)&P, (void*)&fin, (void*)&uout, (void*)&img, (void*)&ainv};
    const void* kern = kf ? (df ? (const void*)k_subcycle<T, true, true> : (const void*)k_subcycle<T, true, false>)
                          : (df ? (const void*)k_subcycle<T, false, true> : (const void*)k_subcycle<T, false, false>);
    sub_launch(kern, smem, ctx.s, args);
    CKL();
    return 0;
}

template <class T, class Op>
static int vcycle_rec(Ctx& ctx, Hier<T>& H, const Op* ops, int l, const mps_solver_opts* o, bool zero_guess)
{
    if (l == ctx.nlev - 1) return coarse_solve(ctx, H, l);
    if constexpr (std::is_same<Op, KOp<T>>::value) {
        if (zero_guess && l == ctx.sub_l0) {
            const int st = subcycle(ctx, H, ops, l, o);
            if (st >= 0) return st;
        }
    }
    const Lev& L = ctx.lev[l];
    const Lev& C = ctx.lev[l + 1];
    int st;
    for (int s = 0; s < o->nu1; s++) {
        bool z = zero_guess && s == 0;
        if (z && ((l == 0 && ctx.red0_ready) || ctx.redz[l])) {
            // the red pass from zero (red = f / diag) came with the outer
            // residual (finest level) or with the restriction (coarse levels)
            H.ri[l] ^= 1;
            ctx.redz[l] = false;
        } else if ((st = colour_pass(ctx, H, ops[l], l, 0, z ? 2 : 0))) {
            return st;
        }
        if ((st = colour_pass(ctx, H, ops[l], l, 1, z ? 1 : 0))) return st;
    }
    if (o->nu1 == 0 && zero_guess) {
        // no pre-smoothing from a zero guess: materialise the zero state
        CK(cudaMemsetAsync(H.U[l][H.ri[l]], 0, sizeof(T) * L.half, ctx.s));
        CK(cudaMemsetAsync(H.U[l][H.bi[l]] + L.half, 0, sizeof(T) * L.half, ctx.s));
    }
    if (l == ctx.prof.level) prof_begin(ctx, MPS_PROF_RESTRICT);
    // the coarse level's first red pass from zero comes with its right-hand
    // side (cell-coefficient operators; not for the coarsest level, a level
    // the one-block sub-cycle takes, or from the finest level, whose
    // restriction has no registers to spare: the launches below pass rz only
    // to the forms that write it and then set the level's flag)
    RedZ<T> rz{nullptr, nullptr};
    if constexpr (std::is_same<Op, KOp<T>>::value) {
        if (l >= 1 && o->nu1 >= 1 && l + 1 < ctx.nlev - 1 && H.D[l + 1] && !(l + 1 == ctx.sub_l0 && H.sub_ok)) {
            rz.u = H.U[l + 1][H.ri[l + 1] ^ 1];
            rz.d = H.D[l + 1];
        }
    }
    bool done = false;
    {
        Box bx;
        if (o->nu1 >= 1 && L.nx >= 16 && restrict_box(L, C, bx)) {
            // red residual of the bulk's children restricted in registers, the
            // shell with the general body
            auto launch = [&](auto wc, auto mbc) {
                constexpr int W = decltype(wc)::value, MB = decltype(mbc)::value;
                const RestrictSplit rs = make_restrict_split(L, C, bx, W);
                const long long shell = (long long)C.nx * C.ny * C.nz - box_cells(bx);
                const unsigned nbb = rs.nb_in + rs.nb_xe + rs.nb_out;
                const unsigned nbs = shell > 0 ? nblk(8 * shell) : 0;
                const RedZ<T> rzw = W <= 2 ? rz : RedZ<T>{nullptr, nullptr};
                if (rzw.u) ctx.redz[l + 1] = true;
                if (L.uniform)
                    pdl_launch(k_resid_restrict_v<T, W, MB, true, Op>, nbb + nbs, TPB, 0, ctx.s, L, ops[l],
                               ccur(H, L, l), H.F[l], C, split<T>(H.F[l + 1], C), rs, bx, nbb, ctx.xf[l].geom,
                               (unsigned)shell, rzw);
                else
                    pdl_launch(k_resid_restrict_v<T, W, MB, false, Op>, nbb + nbs, TPB, 0, ctx.s, L, ops[l],
                               ccur(H, L, l), H.F[l], C, split<T>(H.F[l + 1], C), rs, bx, nbb, ctx.xf[l].geom,
                               (unsigned)shell, rzw);
            };
            if constexpr (!std::is_same<Op, KOp<T>>::value)  // explicit rows: one coarse cell per thread
                launch(std::integral_constant<int, 1>(), std::integral_constant<int, RestrictShape<T>::MINB>());
            else if (l == 0)
                launch(std::integral_constant<int, RestrictShape<T>::W>(), std::integral_constant<int, RestrictShape<T>::MINB>());
            else if (l == 1)
                launch(std::integral_constant<int, CoarseXferShape<T>::W>(), std::integral_constant<int, CoarseXferShape<T>::MINB>());
            else
                launch(std::integral_constant<int, SmallXferShape<T>::W>(), std::integral_constant<int, SmallXferShape<T>::MINB>());
            CKL();
            done = true;
        }
    }
    if (!done) {
        if (rz.u) ctx.redz[l + 1] = true;
        pdl_launch(k_resid_restrict<T, Op>, nblk((long long)C.nx * C.ny * C.nz), TPB, 0, ctx.s, 
            L, ops[l], ccur(H, L, l), csplit<T>(H.F[l], L), C, split<T>(H.F[l + 1], C), ctx.xf[l].geom, rz);
        CKL();
    }
    if (l == ctx.prof.level) prof_end(ctx);
    if ((st = vcycle_rec(ctx, H, ops, l + 1, o, true))) return st;
    if (l == ctx.prof.level) prof_begin(ctx, MPS_PROF_PROLONG);
    // the first post-smoothing pass overwrites the red cells from the black
    // ones, so only black cells need the correction (unless an odd periodic
    // seam makes red cells read red neighbours)
    Box pb{};
    auto prolong_bulk = [&](auto wc) {
        constexpr int W = decltype(wc)::value;
        ProlongDiv dv, sv;
        Box sb;
        ProlongParts pp;
        prolong_form(L, pb, W, dv, sb, sv, pp);
        pdl_launch(k_prolong_v<T, W>, pp.blk0[4], TPB, 0, ctx.s, L, cur(H, L, l), C, ccur(H, C, l + 1), ctx.xf[l],
                   pb, dv, sb, sv, pp);
    };
    if (o->nu2 >= 1 && L.nx >= 16 && prolong_box(L, C, ctx.xf[l], pb)) {
        if (l == 0) prolong_bulk(std::integral_constant<int, ProlongShape<T>::W>());
        else if (l == 1) prolong_bulk(std::integral_constant<int, CoarseXferShape<T>::W>());
        else prolong_bulk(std::integral_constant<int, SmallXferShape<T>::W>());
        CKL();
    } else if (o->nu2 >= 1) {
        pdl_launch(k_prolong_correct<T>, nblk((long long)L.P * L.rows), TPB, 0, ctx.s, L, cur(H, L, l), C,
                                                                               ccur(H, C, l + 1), ctx.xf[l], 1);
        CKL();
        if (odd_periodic(L)) {
            pdl_launch(k_prolong_correct<T>, nblk((long long)L.P * L.rows), TPB, 0, ctx.s, L, cur(H, L, l), C,
                                                                                   ccur(H, C, l + 1), ctx.xf[l], 2);
            CKL();
        }
    } else {
        pdl_launch(k_prolong_correct<T>, nblk((long long)L.nx * L.ny * L.nz), TPB, 0, ctx.s, 
            L, cur(H, L, l), C, ccur(H, C, l + 1), ctx.xf[l], -1);
        CKL();
    }
    if (l == ctx.prof.level) prof_end(ctx);
    for (int s = 0; s < o->nu2; s++) {
        if ((st = colour_pass(ctx, H, ops[l], l, 0, 0))) return st;
        if ((st = colour_pass(ctx, H, ops[l], l, 1, 0))) return st;
    }
    return 0;
}

template <class T>
static int vcycle(Ctx& ctx, Hier<T>& H, int opclass, const mps_solver_opts* o, bool zero_guess)
{
    for (int l = 0; l < MAXL; l++) ctx.redz[l] = false;  // set and consumed within one V-cycle
    if (opclass == 0) return vcycle_rec(ctx, H, H.kop, 0, o, zero_guess);
    return vcycle_rec(ctx, H, H.rop, 0, o, zero_guess);
}

// r = f - A u, sums (r.r, f.f) -> ctx.rb.out; optional r written to rout (type R);
// ured (optional): the red half that a V-cycle's first red pass from a zero
// state on rout would write (r / diag); *ured_done tells whether it was
// written (the split kernel only)
template <class T, class Op, class R>
static int resid_norm(Ctx& ctx, const Op& op, CSplit<T> u, CSplit<T> f, Split<R> rout, R* ured = nullptr,
                      bool* ured_done = nullptr)
{
    if (ured_done) *ured_done = false;
    const Lev& L = ctx.lev[0];
    prof_begin(ctx, MPS_PROF_RESID);
    if constexpr (std::is_same<Op, KOp<T>>::value) {
        if (L.uniform) {  // vector kernel, one launch per colour, norms accumulated
            constexpr int W = ResidShape<T>::W;
            FastDiv dg;
            dg.init((unsigned)(L.P / W));
            // grid-stride over one wave of resident blocks: no partial last
            // wave, and few partials for the norm reduction (measured at 257^3:
            // 193 us against 220 us for 8 blocks per SM and 233 us for one
            // thread per group)
            const unsigned nall = nblk((long long)(L.P / W) * L.rows);
            const unsigned nbv = std::min<unsigned>(nall, (unsigned)(ctx.nsm * ResidShape<T>::MINB));
            ColourSplit cs;
            if (MPS_RESID_SPLIT && make_split(L, W, cs)) {  // interior without boundary code, the shell apart
                R* ur = rout.c[0] ? ured : nullptr;
                pdl_launch(k_residv_split<T, W, R>, nbv, TPB, 0, ctx.s, L, op, u, f.half(0),
                           rout.c[0] ? rout.half(0) : nullptr, ctx.rb, cs, ur);
                CKL();
                prof_end(ctx);
                if (ured_done) *ured_done = ur != nullptr;
                return 0;
            }
            // both colours in one pass (f and rout as split bases, halves L.half apart)
            pdl_launch(k_residv<T, W, R>, nbv, TPB, 0, ctx.s, L, op, -1, u, f.half(0), rout.c[0] ? rout.half(0) : nullptr,
                                                       ctx.rb, 0, dg);
            CKL();
            prof_end(ctx);
            return 0;
        }
    } else {
        // explicit rows: interior cells without boundary code, the shell cell by cell
        ColourSplit cs;
        if (MPS_RESID_SPLIT && L.uniform && L.nx >= 16 && make_split(L, 1, cs)) {
            const unsigned nbv = std::min<unsigned>(cs.nb_in + cs.nb_xe + cs.nb_face,
                                                    (unsigned)(ctx.nsm * ResidShape<T>::MINB));
            pdl_launch(k_residv_split<T, 1, R, Op>, nbv, TPB, 0, ctx.s, L, op, u, f.half(0),
                       rout.c[0] ? rout.half(0) : nullptr, ctx.rb, cs, (R*)nullptr);
            CKL();
            prof_end(ctx);
            return 0;
        }
    }
    pdl_launch(k_resid_norm<T, Op, R>, nblk((long long)L.P * L.rows), TPB, 0, ctx.s, L, op, u, f, rout, ctx.rb);
    prof_end(ctx);
    CKL();
    return 0;
}

static int fetch(Ctx& ctx, const double* dsrc, int n)
{
    CK(cudaMemcpyAsync(ctx.hpin, dsrc, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx.s));
    CK(cudaStreamSynchronize(ctx.s));
    return 0;
}

// the residual norms (rb.out[0..1]) and the device failure word rb.out[3],
// which a kernel whose bounded wait gave up sets (k_colour_tma)
static int fetch_norms(Ctx& ctx)
{
    if (int st = fetch(ctx, ctx.rb.out, 4)) return st;
    if (ctx.hpin[3] != 0.0) {
        CK(cudaMemsetAsync(ctx.rb.out + 3, 0, sizeof(double), ctx.s));
        ctx.err.code = MPS_ERR_TIMEOUT;
        ctx.err.msg = "a bounded device-side wait expired (colour pass copies)";
        return MPS_ERR_TIMEOUT;
    }
    return 0;
}

// ----------------------------------------------------------------------
struct Inputs {  // device pointers (ghosted Fortran-order fields)
    const double* vel;
    const double* dcoeff;
    const double* reac;
    const double* source;
    const double* bcval[6];
    const double* sterm;
    double* soln;
};

template <class T>
static void alloc_hier(Ctx& ctx, Hier<T>& H, bool& ok)
{
    for (int l = 0; l < ctx.nlev; l++) {
        const Lev& L = ctx.lev[l];
        size_t b = sizeof(T) * 2 * L.half;
        H.U[l][0] = (T*)ctx.ar.get(b);
        H.U[l][1] = (T*)ctx.ar.get(b);
        H.F[l] = (T*)ctx.ar.get(b);
        H.R[l] = (T*)ctx.ar.get(b);
        H.D[l] = (l >= 1 && l < ctx.nlev - 1) ? (T*)ctx.ar.get(sizeof(T) * L.half) : nullptr;
        H.ri[l] = H.bi[l] = 0;
        ok = ok && H.U[l][0] && H.U[l][1] && H.F[l] && H.R[l] && (H.D[l] || l < 1 || l >= ctx.nlev - 1);
    }
    const Lev& C = ctx.lev[ctx.nlev - 1];
    const long long n = (long long)C.nx * C.ny * C.nz;
    H.AinvT = (double*)ctx.ar.get(sizeof(double) * n * n);
    H.Dprev = (double*)ctx.ar.get(sizeof(double) * n * n);
    H.gj = (int*)ctx.ar.get(sizeof(int) * 4);
    ok = ok && H.AinvT && H.Dprev && H.gj;
}

static int setup_workspace(Ctx& ctx, const Signature& sig, const mps_solver_opts* o, int need64, int need32)
{
    if (sig == ctx.sig) return 0;
    destroy_graphs(ctx);
    ctx.ar.clear();
    ctx.sig = Signature();
    bool ok = true;
    const int nl = ctx.nlev;
    for (int l = 0; l < nl; l++) {
        const Lev& L = ctx.lev[l];
        const size_t b64 = sizeof(double) * 2 * L.half, b32 = sizeof(float) * 2 * L.half;
        ctx.pk[l] = (double*)ctx.ar.get(b64);
        ctx.preac[l] = sig.has_reac ? (double*)ctx.ar.get(b64) : nullptr;
        ctx.dex64[l] = sig.has_reac ? (double*)ctx.ar.get(b64) : nullptr;
        for (int a = 0; a < 3; a++) ctx.pv[a][l] = sig.opclass == 1 ? (double*)ctx.ar.get(b64) : nullptr;
        ok = ok && ctx.pk[l];
        if (sig.opclass == 1) {
            ctx.rows64[l] = (need64 || l == 0) ? (double*)ctx.ar.get(7 * b64) : nullptr;  // l>0: FP64 solves
            ctx.rows32[l] = need32 ? (float*)ctx.ar.get(7 * b32) : nullptr;
        } else {
            ctx.k32[l] = (need32 && !sig.kuni) ? (float*)ctx.ar.get(b32) : nullptr;
            ctx.dex32[l] = (need32 && sig.has_reac) ? (float*)ctx.ar.get(b32) : nullptr;
        }
    }
    if (need64) alloc_hier(ctx, ctx.h64, ok);
    if (need32) alloc_hier(ctx, ctx.h32, ok);
    const Lev& L0 = ctx.lev[0];
    ctx.x64 = (double*)ctx.ar.get(sizeof(double) * 2 * L0.half);
    ctx.b64 = (double*)ctx.ar.get(sizeof(double) * 2 * L0.half);
    const Lev& C = ctx.lev[nl - 1];
    const long long nc = (long long)C.nx * C.ny * C.nz;
    ctx.dense = (double*)ctx.ar.get(sizeof(double) * nc * nc);
    ctx.gjM = (double*)ctx.ar.get(sizeof(double) * nc * nc * 2);
    ctx.dstatus = (int*)ctx.ar.get(sizeof(int) * 4);
    const unsigned maxb = nblk((long long)L0.P * L0.rows);
    ctx.rb.partial = (double*)ctx.ar.get(sizeof(double) * 2 * (maxb + 1));
    ctx.rb.counter = (unsigned*)ctx.ar.get(sizeof(unsigned) * 4);
    ctx.rb.out = (double*)ctx.ar.get(sizeof(double) * 4);
    ok = ok && ctx.x64 && ctx.b64 && ctx.dense && ctx.gjM && ctx.dstatus && ctx.rb.partial && ctx.rb.counter &&
         ctx.rb.out;
    // the one-block sub-cycle of the small levels: its first level and the
    // solve-constant images of both hierarchies
    ctx.sub_l0 = sig.opclass == 0 && ctx.sub_allowed && sub_prepare(ctx.dev) ? sub_first_level(ctx, o) : -1;
    ctx.h64.subimg = nullptr;
    ctx.h32.subimg = nullptr;
    ctx.h64.subimg_bytes = ctx.h32.subimg_bytes = 0;
    ctx.h64.sub_ok = ctx.h32.sub_ok = false;
    if (ctx.sub_l0 > 0) {
        std::unique_ptr<SubPlan<double>> p64(new SubPlan<double>);
        std::unique_ptr<SubPlan<float>> p32(new SubPlan<float>);
        size_t sm = 0;
        if (need64 && sub_layout<double>(ctx, ctx.sub_l0, !sig.kuni, sig.has_reac != 0, o, *p64, sm)) {
            ctx.h64.subimg_bytes = (size_t)p64->img_bytes;
            ctx.h64.subimg = (unsigned char*)ctx.ar.get(ctx.h64.subimg_bytes);
            ok = ok && ctx.h64.subimg;
        }
        if (need32 && sub_layout<float>(ctx, ctx.sub_l0, !sig.kuni, sig.has_reac != 0, o, *p32, sm)) {
            ctx.h32.subimg_bytes = (size_t)p32->img_bytes;
            ctx.h32.subimg = (unsigned char*)ctx.ar.get(ctx.h32.subimg_bytes);
            ok = ok && ctx.h32.subimg;
        }
    }
    if (!ok) {
        ctx.ar.clear();
        ctx.err.code = MPS_ERR_NOMEM;
        ctx.err.msg = "device allocation failed";
        return MPS_ERR_NOMEM;
    }
    // the arena zeroes new blocks with cudaMemset on the legacy stream; the
    // solver's stream does not synchronise with it, so wait here
    if (cudaDeviceSynchronize() != cudaSuccess) return MPS_ERR_CUDA;
    ctx.tma_ok = ctx.tma_allowed && tma_prepare(ctx.dev);
    ctx.sig = sig;
    return 0;
}

// FGMRES basis: V (m+1 FP64 vectors), Z (m preconditioned vectors, FP32 in
// mixed precision), w, the Hessenberg column and the dot-product partials
static int setup_krylov(Ctx& ctx, long long n, int m)
{
    if (ctx.kar_n == n && ctx.kar_m == m) return 0;
    destroy_graphs(ctx);
    ctx.kar.clear();
    ctx.kar_n = 0;
    ctx.kar_m = 0;
    bool ok = true;
    ctx.V = (double*)ctx.kar.get(sizeof(double) * n * (m + 1));
    ctx.Z = ctx.kar.get(sizeof(double) * n * m);
    ctx.w = (double*)ctx.kar.get(sizeof(double) * n);
    ctx.hcol = (double*)ctx.kar.get(sizeof(double) * 2 * (m + 2));
    ctx.Vptr = (double**)ctx.kar.get(sizeof(double*) * (m + 2));
    ctx.mdot_blocks = 592;
    ctx.dpart = (double*)ctx.kar.get(sizeof(double) * (m + 2) * ctx.mdot_blocks);
    ok = ctx.V && ctx.Z && ctx.w && ctx.hcol && ctx.Vptr && ctx.dpart;
    if (ok) {
        std::vector<double*> hp(m + 2);
        for (int j = 0; j <= m; j++) hp[j] = ctx.V + (size_t)j * n;
        hp[m + 1] = ctx.w;
        if (cudaMemcpy(ctx.Vptr, hp.data(), sizeof(double*) * (m + 2), cudaMemcpyHostToDevice) != cudaSuccess)
            ok = false;
    }
    if (!ok || cudaDeviceSynchronize() != cudaSuccess) {
        ctx.kar.clear();
        ctx.err.code = MPS_ERR_NOMEM;
        ctx.err.msg = "device allocation failed (Krylov basis)";
        return MPS_ERR_NOMEM;
    }
    ctx.kar_n = n;
    ctx.kar_m = m;
    return 0;
}

template <class T>
static void set_kop(Ctx& ctx, KOp<T>* ops, T* const* kT, T* const* dexT, double kc, double dtinv, bool kuni,
                    bool has_reac)
{
    for (int l = 0; l < ctx.nlev; l++) {
        const Lev& L = ctx.lev[l];
        KOp<T> op;
        if (kuni) { op.k[0] = op.k[1] = nullptr; op.kc = (T)kc; }
        else { op.k[0] = kT[l]; op.k[1] = kT[l] + L.half; op.kc = T(0); }
        if (has_reac) { op.dex[0] = dexT[l]; op.dex[1] = dexT[l] + L.half; op.dexc = T(0); }
        else { op.dex[0] = op.dex[1] = nullptr; op.dexc = (T)dtinv; }
        ops[l] = op;
    }
}
template <class T>
static ROp<T> make_rop(T* rows, const Lev& L)
{
    ROp<T> r;
    for (int q = 0; q < 7; q++) {
        r.r[q][0] = rows + (size_t)q * 2 * L.half;
        r.r[q][1] = rows + (size_t)q * 2 * L.half + L.half;
    }
    return r;
}

template <class T>
static int build_rows_level(Ctx& ctx, int l, T* rows, double dtinv, int flux, int transpose, T* tmp)
{
    const Lev& L = ctx.lev[l];
    const double* z = ctx.pk[l];  // any valid pointer for unused fields
    auto cs = [&](const double* p) { return csplit<double>(p ? p : z, L); };
    T* dst = transpose ? tmp : rows;
    pdl_launch(k_build_rows<T>, nblk((long long)L.nx * L.ny * L.nz), TPB, 0, ctx.s, 
        L, cs(ctx.pv[0][l]), cs(ctx.pv[1][l]), cs(ctx.pv[2][l]), cs(ctx.pk[l]), cs(ctx.preac[l]),
        ctx.preac[l] != nullptr, dtinv, flux, make_rop<T>(dst, L));
    CKL();
    if (transpose) {
        pdl_launch(k_transpose_rows<T>, nblk((long long)L.nx * L.ny * L.nz), TPB, 0, ctx.s, L, make_rop<T>(tmp, L),
                                                                                   make_rop<T>(rows, L));
        CKL();
    }
    return 0;
}

template <class T, class Op>
static int coarse_inverse(Ctx& ctx, Hier<T>& H, const Op& op)
{
    const int l = ctx.nlev - 1;
    const Lev& L = ctx.lev[l];
    const int n = L.nx * L.ny * L.nz;
    CK(cudaMemsetAsync(ctx.dense, 0, sizeof(double) * n * n, ctx.s));
    pdl_launch(k_dense_assemble<T, Op>, nblk(n), TPB, 0, ctx.s, L, op, ctx.dense);
    CKL();
    // an unchanged matrix (repeated solves with one operator) keeps its inverse
    pdl_launch(k_dense_same, 1, 1024, 0, ctx.s, n, (const double*)ctx.dense, H.Dprev, H.gj);
    CKL();
    pdl_launch(k_gj_prepare, nblk(2LL * n * n), TPB, 0, ctx.s, n, ctx.dense, ctx.gjM, (const int*)H.gj);
    CKL();
    const size_t smem = sizeof(double) * 2 * (size_t)n * n;
    static signed char gj_state[64] = {};
    const bool gj_smem = once_per_device(ctx.dev, gj_state, [] {
        return cudaFuncSetAttribute(k_gauss_jordan, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) ==
               cudaSuccess;
    });
    if (smem <= 200 * 1024 && gj_smem) {
        pdl_launch(k_gauss_jordan, 1, 1024, smem, ctx.s, n, ctx.gjM, H.AinvT, ctx.dstatus, 1, H.gj);
    } else {
        pdl_launch(k_gauss_jordan, 1, 1024, 0, ctx.s, n, ctx.gjM, H.AinvT, ctx.dstatus, 0, H.gj);
    }
    CKL();
    return 0;
}

// ----------------------------------------------------------------------
// prepare_only: stop after the set-up (hierarchy, operators, right-hand side,
// initial guess, coarsest inverse), for the batched driver
// det (optional): the operator detection of these inputs already read back
// (k_maxabs_all's eight words, then the coefficient of cell (1,1,1)); the
// batched solve detects every problem with one device->host read
static int solve_impl(Ctx& ctx, const mps_grid* g, int timederiv, double dt, const Inputs& in, const int bc[6],
                      const mps_solver_opts* o, mps_solve_info* info, int ref_norm_only, int prepare_only = 0,
                      const unsigned long long* det = nullptr)
{
    mps_solve_info inf;
    std::memset(&inf, 0, sizeof(inf));
    inf.status = MPS_OK;
    // ---- argument checks ----
    if (!g || g->lx < 1 || g->ly < 1 || g->lz < 1 || !(g->llenx > 0) || !(g->lleny > 0) || !(g->llenz > 0) ||
        !in.dcoeff || !in.source || !in.soln) {
        ctx.err.msg = "bad grid or null field";
        return MPS_ERR_BAD_ARG;
    }
    if ((long long)g->lx * g->ly * g->lz >= (1LL << 31) / 2) { ctx.err.msg = "grid too large"; return MPS_ERR_BAD_ARG; }
    for (int f = 0; f < 6; f++)
        if (bc[f] < 1 || bc[f] > 5) { ctx.err.msg = "bad BC code"; return MPS_ERR_BAD_ARG; }
    for (int a = 0; a < 3; a++)
        if ((bc[2 * a] == BC_PERI) != (bc[2 * a + 1] == BC_PERI)) {
            ctx.err.msg = "PERI must be set on both faces of a direction";
            return MPS_ERR_BAD_ARG;
        }
    if (timederiv && !(dt > 0)) { ctx.err.msg = "dt must be positive"; return MPS_ERR_BAD_ARG; }
    if (o->nu1 < 0 || o->nu2 < 0 || o->maxit < 0 || o->restart < 1 || o->restart > 250 || o->max_coarse < 1 ||
        o->max_coarse > MAX_DENSE) {
        ctx.err.msg = "bad solver option";
        return MPS_ERR_BAD_ARG;
    }
    for (int f = 0; f < 6; f++)
        if (!in.bcval[f] && (bc[f] == BC_DIRC || bc[f] == BC_FLUX)) {
            ctx.err.msg = "missing boundary values for a DIRC/FLUX face";
            return MPS_ERR_BAD_ARG;
        }
    std::string why;
    int nl = plan_levels(g, o, bc, ctx.lev, ctx.xf, why);
    if (nl < 1) { ctx.err.msg = why; return MPS_ERR_BAD_ARG; }
    ctx.nlev = nl;
    const Lev& L0 = ctx.lev[0];
    {  // 1-D prolongation tables of the geometric transfers
        size_t total = 0;
        for (int l = 0; l + 1 < nl; l++)
            for (int a = 0; a < 3; a++) total += ctx.xf[l].nf[a];
        std::vector<Lin> tab(total > 0 ? total : 1);
        size_t pos = 0;
        for (int l = 0; l + 1 < nl; l++)
            for (int a = 0; a < 3; a++) {
                for (int i = 0; i < ctx.xf[l].nf[a]; i++) {
                    Lin e;
                    geom_lin(ctx.xf[l], a, i, e.j0, e.j1, e.t);
                    tab[pos + i] = e;
                }
                pos += ctx.xf[l].nf[a];
            }
        // the device copy is kept while the tables do not change (a copy from
        // pageable host memory would hold the host until the stream drains)
        const bool same = ctx.dtab && tab.size() == ctx.htab.size() &&
                          std::memcmp(tab.data(), ctx.htab.data(), sizeof(Lin) * tab.size()) == 0;
        if (!same) {
            if (tab.size() > ctx.dtab_n) {
                if (ctx.dtab) cudaFree(ctx.dtab);
                ctx.dtab = nullptr;
                ctx.dtab_n = 0;
                CK(cudaMalloc((void**)&ctx.dtab, sizeof(Lin) * tab.size()));
                ctx.dtab_n = tab.size();
            }
            ctx.htab.swap(tab);
            CK(cudaMemcpyAsync(ctx.dtab, ctx.htab.data(), sizeof(Lin) * ctx.htab.size(), cudaMemcpyHostToDevice,
                               ctx.s));
        }
        pos = 0;
        for (int l = 0; l + 1 < nl; l++)
            for (int a = 0; a < 3; a++) {
                ctx.xf[l].tab[a] = ctx.dtab + pos;
                pos += ctx.xf[l].nf[a];
            }
    }
    const double dtinv = timederiv ? 1.0 / dt : 0.0;

    const long long launches0 = ctx.launches;
    CK(cudaEventRecord(ctx.e0, ctx.s));
    // ---- operator detection (one small device->host read) ----
    unsigned long long* dm = ctx.dmax;
    const long long ncell = (long long)L0.nx * L0.ny * L0.nz;
    const long long ng = (long long)(L0.nx + 2) * (L0.ny + 2) * (L0.nz + 2);
    unsigned long long hm[8];
    double k0 = 0.0;
    if (det) {
        std::memcpy(hm, det, sizeof(hm));
        std::memcpy(&k0, det + 8, sizeof(double));
    } else {
        CK(cudaMemsetAsync(dm, 0, sizeof(unsigned long long) * 8, ctx.s));
        const unsigned mb = std::min<unsigned>(nblk(ncell), 1184);
        pdl_launch(k_maxabs_all, mb, TPB, 0, ctx.s, L0, in.vel, in.reac, in.dcoeff, in.source, in.soln, dm);
        CKL();
        CK(cudaMemcpyAsync(hm, dm, sizeof(hm), cudaMemcpyDeviceToHost, ctx.s));
        CK(cudaMemcpyAsync(&k0, in.dcoeff + 1 + (L0.nx + 2) * (1 + (long long)(L0.ny + 2)), sizeof(double),
                           cudaMemcpyDeviceToHost, ctx.s));
        CK(cudaStreamSynchronize(ctx.s));
    }
    auto asd = [](unsigned long long b) { double d; std::memcpy(&d, &b, 8); return d; };
    const double maxvel = asd(hm[0]), maxreac = asd(hm[1]), dkvar = asd(hm[2]), maxsrc = asd(hm[3]),
                 maxsol = asd(hm[4]), maxk = asd(hm[5]);
    if (!(maxvel <= 1e308) || !(maxreac <= 1e308) || !(dkvar <= 1e308) || !(maxsrc <= 1e308) ||
        !(maxsol <= 1e308) || !(maxk <= 1e308)) {
        ctx.err.msg = "NaN or Inf in the inputs";
        inf.status = MPS_ERR_NAN;
        if (info) *info = inf;
        return MPS_ERR_NAN;
    }
    Signature sig;
    sig.dims[0] = g->lx; sig.dims[1] = g->ly; sig.dims[2] = g->lz;
    for (int f = 0; f < 6; f++) sig.bc[f] = bc[f];
    sig.hier = o->hierarchy;
    for (int a = 0; a < 3; a++) sig.ranks[a] = o->hierarchy == MPS_HIER_CELL ? o->ranks[a] : 0;
    sig.max_coarse = o->hierarchy == MPS_HIER_GEOM ? o->max_coarse : 0;
    sig.opclass = (o->transpose == 0 && o->flux == MPS_FLUX_UPWIND && maxvel == 0.0) ? 0 : 1;
    if (o->flux == MPS_FLUX_UPWIND && maxvel == 0.0) sig.opclass = 0;  // symmetric: A^T = A
    sig.prec = 0;
    sig.krylov = 0;
    sig.restart = 0;
    sig.has_reac = maxreac > 0.0;
    sig.kuni = dkvar == 0.0;
    sig.transpose = o->transpose && sig.opclass == 1;
    const bool mixed = o->precision == MPS_PREC_MIXED;
    // both hierarchies stay allocated (switching precision costs no allocation);
    // only the one this solve uses is filled
    int st = setup_workspace(ctx, sig, o, 1, 1);
    const int need64 = !mixed, need32 = mixed;
    if (st) return st;
    if (o->krylov == MPS_KRYLOV_FGMRES && (st = setup_krylov(ctx, 2 * ctx.lev[0].half, o->restart))) return st;

    // ---- coefficient pyramid (FP64) ----
    pdl_launch(k_pack<double>, nblk(ncell), TPB, 0, ctx.s, L0, in.dcoeff, split<double>(ctx.pk[0], L0), 1.0, 0.0);
    CKL();
    if (sig.has_reac) {
        pdl_launch(k_pack<double>, nblk(ncell), TPB, 0, ctx.s, L0, in.reac, split<double>(ctx.preac[0], L0), 1.0, 0.0);
        CKL();
    }
    if (sig.opclass == 1)
        for (int a = 0; a < 3; a++) {
            pdl_launch(k_pack<double>, nblk(ncell), TPB, 0, ctx.s, L0, in.vel ? in.vel + a * ng : nullptr,
                                                           split<double>(ctx.pv[a][0], L0), 1.0, 0.0);
            CKL();
        }
    for (int l = 0; l + 1 < nl; l++) {
        const Lev& F = ctx.lev[l];
        const Lev& C = ctx.lev[l + 1];
        const unsigned nb = nblk((long long)C.nx * C.ny * C.nz);
        const int geom = ctx.xf[l].geom;
        pdl_launch(k_restrict_field, nb, TPB, 0, ctx.s, F, csplit<double>(ctx.pk[l], F), C, split<double>(ctx.pk[l + 1], C),
                                                geom);
        CKL();
        if (sig.has_reac) {
            pdl_launch(k_restrict_field, nb, TPB, 0, ctx.s, F, csplit<double>(ctx.preac[l], F), C,
                                                    split<double>(ctx.preac[l + 1], C), geom);
            CKL();
        }
        if (sig.opclass == 1)
            for (int a = 0; a < 3; a++) {
                pdl_launch(k_restrict_field, nb, TPB, 0, ctx.s, F, csplit<double>(ctx.pv[a][l], F), C,
                                                        split<double>(ctx.pv[a][l + 1], C), geom);
                CKL();
            }
    }
    // ---- operators ----
    if (sig.opclass == 0) {
        for (int l = 0; l < nl; l++) {
            const long long n2 = 2 * ctx.lev[l].half;
            if (sig.has_reac) {
                pdl_launch(k_cast_field<double>, std::min<unsigned>(nblk(n2), 2368), TPB, 0, ctx.s, n2, ctx.preac[l], ctx.dex64[l], -1.0, dtinv);
                CKL();
            }
            if (need32) {
                if (!sig.kuni) {
                    pdl_launch(k_cast_field<float>, std::min<unsigned>(nblk(n2), 2368), TPB, 0, ctx.s, n2, ctx.pk[l], ctx.k32[l], 1.0, 0.0);
                    CKL();
                }
                if (sig.has_reac) {
                    pdl_launch(k_cast_field<float>, std::min<unsigned>(nblk(n2), 2368), TPB, 0, ctx.s, n2, ctx.preac[l], ctx.dex32[l], -1.0, dtinv);
                    CKL();
                }
            }
        }
        KOp<double> k64[MAXL];
        set_kop<double>(ctx, k64, ctx.pk, ctx.dex64, k0, dtinv, sig.kuni, sig.has_reac);
        ctx.kop64 = k64[0];
        if (need64) std::copy(k64, k64 + nl, ctx.h64.kop);
        if (need32) set_kop<float>(ctx, ctx.h32.kop, ctx.k32, ctx.dex32, k0, dtinv, sig.kuni, sig.has_reac);
    } else {
        for (int l = 0; l < nl; l++) {
            if (ctx.rows64[l] && (need64 || l == 0)) {
                // transposed rows need a scratch copy of the forward rows: use rows32's
                // FP64-sized neighbour (x64 is large enough only at level 0), so build into
                // the FGMRES-free scratch: the dense matrix buffer is too small; allocate once
                double* tmp = nullptr;
                if (sig.transpose) {
                    CK(cudaMallocAsync((void**)&tmp, sizeof(double) * 7 * 2 * ctx.lev[l].half, ctx.s));
                }
                if ((st = build_rows_level<double>(ctx, l, ctx.rows64[l], dtinv, o->flux, sig.transpose, tmp))) return st;
                if (tmp) CK(cudaFreeAsync(tmp, ctx.s));
                if (need64) ctx.h64.rop[l] = make_rop<double>(ctx.rows64[l], ctx.lev[l]);
            }
            if (ctx.rows32[l] && need32) {
                float* tmp = nullptr;
                if (sig.transpose) {
                    CK(cudaMallocAsync((void**)&tmp, sizeof(float) * 7 * 2 * ctx.lev[l].half, ctx.s));
                }
                if ((st = build_rows_level<float>(ctx, l, ctx.rows32[l], dtinv, o->flux, sig.transpose, tmp))) return st;
                if (tmp) CK(cudaFreeAsync(tmp, ctx.s));
                ctx.h32.rop[l] = make_rop<float>(ctx.rows32[l], ctx.lev[l]);
            }
        }
        ctx.rop64 = make_rop<double>(ctx.rows64[0], L0);
    }
    // ---- right-hand side and initial guess ----
    {
        const double* bv[6];
        for (int f = 0; f < 6; f++) bv[f] = in.bcval[f];
        pdl_launch(k_find_bvec, nblk(ncell), TPB, 0, ctx.s, L0, in.vel, in.dcoeff, in.source, bv[0], bv[1], bv[2], bv[3],
                                                    bv[4], bv[5], in.sterm, o->flux, split<double>(ctx.b64, L0));
        CKL();
        if (maxsol == 0.0) {  // a zero initial guess (every interior cell): clear instead of packing
            CK(cudaMemsetAsync(ctx.x64, 0, sizeof(double) * 2 * L0.half, ctx.s));
        } else {
            pdl_launch(k_pack<double>, nblk(ncell), TPB, 0, ctx.s, L0, in.soln, split<double>(ctx.x64, L0), 1.0, 0.0);
            CKL();
        }
    }
    // ---- coarsest inverse ----
    CK(cudaMemsetAsync(ctx.dstatus, 0, sizeof(int) * 4, ctx.s));
    if (need64) {
        if (sig.opclass == 0) st = coarse_inverse(ctx, ctx.h64, ctx.h64.kop[nl - 1]);
        else st = coarse_inverse(ctx, ctx.h64, ctx.h64.rop[nl - 1]);
    } else {
        if (sig.opclass == 0) st = coarse_inverse(ctx, ctx.h32, ctx.h32.kop[nl - 1]);
        else st = coarse_inverse(ctx, ctx.h32, ctx.h32.rop[nl - 1]);
    }
    if (st) return st;
    if (sig.opclass == 0 && !prepare_only) {  // the one-block sub-cycle's solve-constant image
        if (need64) st = sub_image(ctx, ctx.h64, ctx.h64.kop, o);
        else st = sub_image(ctx, ctx.h32, ctx.h32.kop, o);
        if (st) return st;
        // the red rows' diagonals of the levels with their own launches (the
        // restriction into such a level also writes its first red pass)
        auto diag_red = [&](auto& H) -> int {
            using TT = typename std::remove_reference<decltype(*H.D[0])>::type;
            const int lend = (ctx.sub_l0 > 0 && H.sub_ok) ? ctx.sub_l0 : nl - 1;
            for (int l = 1; l < lend && l < nl - 1; l++) {
                if (!H.D[l]) continue;
                const Lev& Ll = ctx.lev[l];
                pdl_launch(k_diag_red<TT, KOp<TT>>, nblk((long long)Ll.P * Ll.rows), TPB, 0, ctx.s, Ll, H.kop[l],
                           H.D[l]);
                CKL();
            }
            return 0;
        };
        if (need64) st = diag_red(ctx.h64);
        else st = diag_red(ctx.h32);
        if (st) return st;
    }
    if (prepare_only) {
        inf.levels = nl;
        if (info) *info = inf;
        return 0;
    }

    // ---- iterations ----
    const Lev& L = L0;
    const long long n2 = 2 * L.half;
    double bnorm = 0.0, rel = 0.0, rms = 0.0;
    int it = 0, vcycles = 0;
    auto norms = [&](double rr, double ff) {
        rel = ff > 0.0 ? std::sqrt(rr) / std::sqrt(ff) : std::sqrt(rr);
        rms = std::sqrt(rr / (double)ncell);
    };
    auto conv = [&]() { return o->tol_kind == MPS_TOL_RMS_ABS ? rms <= o->tol : rel <= o->tol; };
    Split<double> no64;
    no64.c[0] = no64.c[1] = nullptr;

    GraphKey gk;
    gk.sig = sig;
    gk.prec = mixed;
    gk.nu1 = o->nu1;
    gk.nu2 = o->nu2;
    gk.nlev = nl;
    gk.flux = o->flux;
    gk.transpose = sig.transpose;  // a symmetric operator's transposed solve replays the forward graphs
    gk.kc = sig.kuni ? k0 : 0.0;
    gk.dexc = sig.has_reac ? 0.0 : dtinv;
    gk.ws = ctx.ar.blocks.empty() ? nullptr : ctx.ar.blocks[0];
    gk.prof = ctx.prof.on ? 1 + ctx.prof.level : 0;  // profiled graphs carry event-record nodes
    // graphs need the buffer parities to return after one iteration
    const bool graphs = o->use_graph && ((o->nu1 + o->nu2) % 2 == 0);

    if (o->krylov == MPS_KRYLOV_NONE && !mixed) {
        // FP64 stationary V-cycle iteration on h64 (x lives in level-0 U)
        Hier<double>& H = ctx.h64;
        CK(cudaMemcpyAsync(H.U[0][0], ctx.x64, sizeof(double) * n2, cudaMemcpyDeviceToDevice, ctx.s));
        CK(cudaMemcpyAsync(H.F[0], ctx.b64, sizeof(double) * n2, cudaMemcpyDeviceToDevice, ctx.s));
        for (int l = 0; l < nl; l++) H.ri[l] = H.bi[l] = 0;
        auto residual = [&]() -> int {
            if (sig.opclass == 0) return resid_norm(ctx, H.kop[0], ccur(H, L, 0), csplit<double>(H.F[0], L), no64);
            return resid_norm(ctx, H.rop[0], ccur(H, L, 0), csplit<double>(H.F[0], L), no64);
        };
        auto iteration = [&]() -> int {
            int s2 = vcycle(ctx, H, sig.opclass, o, false);
            if (s2) return s2;
            return residual();
        };
        if ((st = residual())) return st;
        for (;;) {
            if ((st = fetch_norms(ctx))) return st;
            if (!(ctx.hpin[0] <= 1e308)) { inf.status = MPS_ERR_NAN; break; }
            norms(ctx.hpin[0], ctx.hpin[1]);
            if (it == 0) inf.rel_res0 = rel;
            if (ref_norm_only ? it >= o->maxit : (conv() || it >= o->maxit)) break;
            if (graphs) {
                gk.kind = 1;
                GraphEntry* G = nullptr;
                for (;;) {  // each replay ends with the residual norms of the new iterate
                    if ((st = run_graph(ctx, gk, &G, iteration))) return st;
                    if ((st = fetch_norms(ctx))) return st;
                    prof_collect_graph(ctx, *G);
                    vcycles++;
                    it++;
                    if (!(ctx.hpin[0] <= 1e308)) { inf.status = MPS_ERR_NAN; break; }
                    norms(ctx.hpin[0], ctx.hpin[1]);
                    if (ref_norm_only ? it >= o->maxit : (conv() || it >= o->maxit)) break;
                }
                break;
            }
            if ((st = iteration())) return st;
            vcycles++;
            it++;
        }
        // copy the iterate back to x64 (split, both colours)
        CK(cudaMemcpyAsync(ctx.x64, H.U[0][H.ri[0]], sizeof(double) * L.half, cudaMemcpyDeviceToDevice, ctx.s));
        CK(cudaMemcpyAsync(ctx.x64 + L.half, H.U[0][H.bi[0]] + L.half, sizeof(double) * L.half,
                           cudaMemcpyDeviceToDevice, ctx.s));
    } else if (o->krylov == MPS_KRYLOV_NONE && mixed) {
        // FP64 defect correction with FP32 V-cycles
        Hier<float>& H = ctx.h32;
        const int inner = o->inner_cycles > 0 ? o->inner_cycles : 2;
        for (int l = 0; l < nl; l++) H.ri[l] = H.bi[l] = 0;
        gk.inner = inner;
        // the residual also writes the first V-cycle's red pass from zero on the
        // finest level (r / diag) where its split kernel runs; the V-cycle then
        // skips that pass
        bool red_ready = false;
        auto residual = [&]() -> int {
            Split<float> r32 = split<float>(H.F[0], L);
            float* ured = o->nu1 >= 1 ? H.U[0][H.ri[0] ^ 1] : nullptr;
            if (sig.opclass == 0)
                return resid_norm(ctx, ctx.kop64, csplit<double>(ctx.x64, L), csplit<double>(ctx.b64, L), r32, ured,
                                  &red_ready);
            return resid_norm(ctx, ctx.rop64, csplit<double>(ctx.x64, L), csplit<double>(ctx.b64, L), r32, ured,
                              &red_ready);
        };
        auto iteration = [&]() -> int {
            int s2;
            for (int c = 0; c < inner; c++) {
                ctx.red0_ready = c == 0 && red_ready;
                s2 = vcycle(ctx, H, sig.opclass, o, c == 0);
                ctx.red0_ready = false;
                if (s2) return s2;
            }
            const unsigned ab = std::min<unsigned>(nblk(2 * L.half), 4736);
            pdl_launch(k_axpy2<float, double>, ab, TPB, 0, ctx.s, L.half, 1.0, (const float*)H.U[0][H.ri[0]], ctx.x64,
                       (const float*)(H.U[0][H.bi[0]] + L.half), ctx.x64 + L.half);
            CKL();
            return residual();
        };
        if ((st = residual())) return st;
        for (;;) {
            if ((st = fetch_norms(ctx))) return st;
            if (!(ctx.hpin[0] <= 1e308)) { inf.status = MPS_ERR_NAN; break; }
            norms(ctx.hpin[0], ctx.hpin[1]);
            if (it == 0) inf.rel_res0 = rel;
            if (conv() || it >= o->maxit) break;
            if (graphs) {
                gk.kind = 2;
                GraphEntry* G = nullptr;
                for (;;) {  // each replay ends with the residual norms of the new iterate
                    if ((st = run_graph(ctx, gk, &G, iteration))) return st;
                    if ((st = fetch_norms(ctx))) return st;
                    prof_collect_graph(ctx, *G);
                    vcycles += inner;
                    it++;
                    if (!(ctx.hpin[0] <= 1e308)) { inf.status = MPS_ERR_NAN; break; }
                    norms(ctx.hpin[0], ctx.hpin[1]);
                    if (conv() || it >= o->maxit) break;
                }
                break;
            }
            if ((st = iteration())) return st;
            vcycles += inner;
            it++;
        }
    } else {
        // FGMRES(m), right preconditioned by one V-cycle (FP32 when MIXED)
        for (int l = 0; l < nl; l++) ctx.h32.ri[l] = ctx.h32.bi[l] = ctx.h64.ri[l] = ctx.h64.bi[l] = 0;
        const int m = o->restart;
        const long long n = n2;
        const unsigned db = ctx.mdot_blocks;
        std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), gq(m + 1), y(m);
        auto HH = [&](int i, int j) -> double& { return H[(size_t)i + (size_t)(m + 1) * j]; };
        for (;;) {
            // w = b - A x, beta = ||w||
            if (sig.opclass == 0)
                st = resid_norm(ctx, ctx.kop64, csplit<double>(ctx.x64, L), csplit<double>(ctx.b64, L),
                                split<double>(ctx.w, L));
            else
                st = resid_norm(ctx, ctx.rop64, csplit<double>(ctx.x64, L), csplit<double>(ctx.b64, L),
                                split<double>(ctx.w, L));
            if (st) return st;
            if ((st = fetch_norms(ctx))) return st;
            if (!(ctx.hpin[0] <= 1e308)) { inf.status = MPS_ERR_NAN; break; }
            norms(ctx.hpin[0], ctx.hpin[1]);
            if (it == 0) { inf.rel_res0 = rel; bnorm = std::sqrt(ctx.hpin[1]); }
            if (conv() || it >= o->maxit) break;
            const double beta = std::sqrt(ctx.hpin[0]);
            // v0 = w / beta
            ctx.hpin[0] = beta;
            CK(cudaMemcpyAsync(ctx.hcol, ctx.hpin, sizeof(double), cudaMemcpyHostToDevice, ctx.s));
            pdl_launch(k_scale_to, std::min<unsigned>(nblk(n), 2368), TPB, 0, ctx.s, n, ctx.w, ctx.hcol, 0, ctx.V, nullptr);
            CKL();
            std::fill(H.begin(), H.end(), 0.0);
            std::fill(gq.begin(), gq.end(), 0.0);
            gq[0] = beta;
            int j = 0;
            bool done = false;
            for (j = 0; j < m && it < o->maxit; j++) {
                double* vj = ctx.V + (size_t)j * n;
                GraphEntry* pg = nullptr;  // the preconditioner's graph replayed this iteration
                // z_j = M^{-1} v_j (one V-cycle from zero), then w = A z_j in FP64
                if (mixed) {
                    Hier<float>& P = ctx.h32;
                    pdl_launch(k_cast_field<float>, std::min<unsigned>(nblk(n), 2368), TPB, 0, ctx.s, n, vj, P.F[0], 1.0, 0.0);
                    CKL();
                    if (graphs) {
                        gk.kind = 3;
                        if ((st = run_graph(ctx, gk, &pg, [&]() { return vcycle(ctx, P, sig.opclass, o, true); })))
                            return st;
                    } else if ((st = vcycle(ctx, P, sig.opclass, o, true))) {
                        return st;
                    }
                    float* zj = (float*)ctx.Z + (size_t)j * n;
                    CK(cudaMemcpyAsync(zj, P.U[0][P.ri[0]], sizeof(float) * L.half, cudaMemcpyDeviceToDevice, ctx.s));
                    CK(cudaMemcpyAsync(zj + L.half, P.U[0][P.bi[0]] + L.half, sizeof(float) * L.half,
                                       cudaMemcpyDeviceToDevice, ctx.s));
                    if (sig.opclass == 0)
                        pdl_launch(k_apply<double, KOp<double>, float>, nblk((long long)L.P * L.rows), TPB, 0, ctx.s, 
                            L, ctx.kop64, csplit<float>(zj, L), split<double>(ctx.w, L));
                    else
                        pdl_launch(k_apply<double, ROp<double>, float>, nblk((long long)L.P * L.rows), TPB, 0, ctx.s, 
                            L, ctx.rop64, csplit<float>(zj, L), split<double>(ctx.w, L));
                    CKL();
                } else {
                    Hier<double>& P = ctx.h64;
                    CK(cudaMemcpyAsync(P.F[0], vj, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx.s));
                    if (graphs) {
                        gk.kind = 4;
                        if ((st = run_graph(ctx, gk, &pg, [&]() { return vcycle(ctx, P, sig.opclass, o, true); })))
                            return st;
                    } else if ((st = vcycle(ctx, P, sig.opclass, o, true))) {
                        return st;
                    }
                    double* zj = (double*)ctx.Z + (size_t)j * n;
                    CK(cudaMemcpyAsync(zj, P.U[0][P.ri[0]], sizeof(double) * L.half, cudaMemcpyDeviceToDevice, ctx.s));
                    CK(cudaMemcpyAsync(zj + L.half, P.U[0][P.bi[0]] + L.half, sizeof(double) * L.half,
                                       cudaMemcpyDeviceToDevice, ctx.s));
                    if (sig.opclass == 0)
                        pdl_launch(k_apply<double, KOp<double>, double>, nblk((long long)L.P * L.rows), TPB, 0, ctx.s, 
                            L, ctx.kop64, csplit<double>(zj, L), split<double>(ctx.w, L));
                    else
                        pdl_launch(k_apply<double, ROp<double>, double>, nblk((long long)L.P * L.rows), TPB, 0, ctx.s, 
                            L, ctx.rop64, csplit<double>(zj, L), split<double>(ctx.w, L));
                    CKL();
                }
                vcycles++;
                // CGS2 against v_0..v_j: pass 1 coefficients in hcol[0..j], pass 2 in
                // hcol[m+2 ..]; the Hessenberg column is their sum
                for (int pass = 0; pass < 2; pass++) {
                    double* hp = ctx.hcol + (pass ? m + 2 : 0);
                    pdl_launch(k_multidot, db, TPB, 0, ctx.s, n, j + 1, ctx.Vptr, ctx.w, ctx.dpart);
                    CKL();
                    pdl_launch(k_multidot_finish, j + 1, TPB, 0, ctx.s, j + 1, db, ctx.dpart, hp, 0);
                    CKL();
                    pdl_launch(k_multiaxpy, std::min<unsigned>(nblk(n), 2368), TPB, 0, ctx.s, n, j + 1, ctx.Vptr, hp, ctx.w);
                    CKL();
                }
                // ||w||^2 (Vptr[m+1] points at w) into hcol[j+1]
                pdl_launch(k_multidot, db, TPB, 0, ctx.s, n, 1, ctx.Vptr + m + 1, ctx.w, ctx.dpart);
                CKL();
                pdl_launch(k_multidot_finish, 1, TPB, 0, ctx.s, 1, db, ctx.dpart, ctx.hcol + j + 1, 0);
                CKL();
                CK(cudaMemcpyAsync(ctx.hpin, ctx.hcol, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost, ctx.s));
                CK(cudaMemcpyAsync(ctx.hpin + 256, ctx.hcol + m + 2, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost,
                                   ctx.s));
                CK(cudaStreamSynchronize(ctx.s));
                if (pg) prof_collect_graph(ctx, *pg);
                for (int i = 0; i <= j; i++) HH(i, j) = ctx.hpin[i] + ctx.hpin[256 + i];
                double hn = std::sqrt(std::max(ctx.hpin[j + 1], 0.0));
                if (!(hn <= 1e308)) { inf.status = MPS_ERR_NAN; done = true; break; }
                HH(j + 1, j) = hn;
                ctx.hpin[0] = hn;
                CK(cudaMemcpyAsync(ctx.hcol + j + 1, ctx.hpin, sizeof(double), cudaMemcpyHostToDevice, ctx.s));
                if (hn > 0.0) {
                    pdl_launch(k_scale_to, std::min<unsigned>(nblk(n), 2368), TPB, 0, ctx.s, n, ctx.w, ctx.hcol, j + 1,
                                                                                    ctx.V + (size_t)(j + 1) * n, nullptr);
                    CKL();
                }
                for (int i = 0; i < j; i++) {
                    double t = cs[i] * HH(i, j) + sn[i] * HH(i + 1, j);
                    HH(i + 1, j) = -sn[i] * HH(i, j) + cs[i] * HH(i + 1, j);
                    HH(i, j) = t;
                }
                double a = HH(j, j), b = HH(j + 1, j), rr = std::sqrt(a * a + b * b);
                cs[j] = rr == 0.0 ? 1.0 : a / rr;
                sn[j] = rr == 0.0 ? 0.0 : b / rr;
                HH(j, j) = cs[j] * a + sn[j] * b;
                HH(j + 1, j) = 0.0;
                gq[j + 1] = -sn[j] * gq[j];
                gq[j] = cs[j] * gq[j];
                it++;
                const double est = std::fabs(gq[j + 1]) / (bnorm > 0 ? bnorm : 1.0);
                if ((o->tol_kind == MPS_TOL_REL_L2 && est <= o->tol) || hn == 0.0) { j++; break; }
            }
            if (done) break;
            // y = H^{-1} g ; x += Z y
            for (int i = j - 1; i >= 0; i--) {
                double s = gq[i];
                for (int q = i + 1; q < j; q++) s -= HH(i, q) * y[q];
                y[i] = (HH(i, i) != 0.0) ? s / HH(i, i) : 0.0;
            }
            for (int i = 0; i < j; i++) {
                if (mixed)
                    pdl_launch(k_axpy<float, double>, std::min<unsigned>(nblk(n), 2368), TPB, 0, ctx.s, n, y[i], (float*)ctx.Z + (size_t)i * n, ctx.x64);
                else
                    pdl_launch(k_axpy<double, double>, std::min<unsigned>(nblk(n), 2368), TPB, 0, ctx.s, n, y[i], (double*)ctx.Z + (size_t)i * n, ctx.x64);
                CKL();
            }
        }
    }
    // ---- output ----
    int gst = 0;
    CK(cudaMemcpyAsync(&gst, ctx.dstatus, sizeof(int), cudaMemcpyDeviceToHost, ctx.s));
    pdl_launch(k_unpack<double>, nblk(ncell), TPB, 0, ctx.s, L0, csplit<double>(ctx.x64, L0), in.soln);
    CKL();
    if (o->fill_ghosts) {
        const int mx = std::max(std::max(L0.ny * L0.nz, L0.nx * L0.nz), L0.nx * L0.ny);
        const double* zf[6];
        for (int f = 0; f < 6; f++) zf[f] = in.bcval[f];
        pdl_launch(k_fill_ghosts, nblk(mx), TPB, 0, ctx.s, L0, in.soln, zf[0], zf[1], zf[2], zf[3], zf[4], zf[5]);
        CKL();
    }
    CK(cudaEventRecord(ctx.e1, ctx.s));
    CK(cudaStreamSynchronize(ctx.s));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx.e0, ctx.e1));
    if (ctx.prof.on) {
        prof_collect(ctx);
        ctx.prof.precision_bytes = mixed ? 4 : 8;
        ctx.prof.coeff_field = sig.opclass == 0 ? !sig.kuni : 7;
        ctx.prof.cells = ncell;
    }
    inf.launches = (int)(ctx.launches - launches0);
    inf.iters = it;
    inf.vcycles = vcycles;
    inf.levels = nl;
    inf.rel_res = rel;
    inf.rms_res = rms;
    inf.time_ms = ms;
    if (inf.status == MPS_OK && !ref_norm_only && !conv()) inf.status = MPS_ERR_NOT_CONVERGED;
    (void)gst;
    if (info) *info = inf;
    return inf.status == MPS_ERR_NAN ? MPS_ERR_NAN : 0;
}

}  // namespace mps

#include "mps_batch.cuh"

// ======================================================================
// C ABI
// ======================================================================
using namespace mps;

extern "C" {

void mps_default_opts(mps_solver_opts* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tol = 1e-10;
    o->tol_kind = MPS_TOL_REL_L2;
    o->maxit = 50;
    o->nu1 = 2;
    o->nu2 = 2;
    o->hierarchy = MPS_HIER_GEOM;
    o->ranks[0] = o->ranks[1] = o->ranks[2] = 1;
    o->max_coarse = 125;
    o->precision = MPS_PREC_FP64;
    o->inner_cycles = 0;
    o->krylov = MPS_KRYLOV_NONE;
    o->restart = 30;
    o->fill_ghosts = 0;
    o->use_graph = 1;
    o->transpose = 0;
    o->flux = MPS_FLUX_UPWIND;
}

const char* mps_version(void) { return "mps3d_b200 0.1 (sm_100a)"; }

int mps_create(mps_handle* h, int device)
{
    if (!h) return MPS_ERR_BAD_ARG;
    *h = nullptr;
    mps_handle_s* H = new (std::nothrow) mps_handle_s();
    if (!H) return MPS_ERR_NOMEM;
    Ctx& ctx = H->ctx;
    int dev = device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) { delete H; return MPS_ERR_CUDA; }
    if (cudaSetDevice(dev) != cudaSuccess) { delete H; return MPS_ERR_CUDA; }
    ctx.dev = dev;
    // optional cap on the grid-dependent workspace (bytes, per arena), for
    // callers that share the device with other large allocations
    if (const char* cap = std::getenv("MPS_WORKSPACE_LIMIT_BYTES")) {
        const long long v = std::atoll(cap);
        if (v > 0) ctx.ar.limit = ctx.kar.limit = (size_t)v;
    }
    // the shared-memory (TMA) kernels and the register-fed ones give the same
    // results; the variable selects the register-fed ones (for comparisons)
    if (const char* tv = std::getenv("MPS_TMA")) ctx.tma_allowed = std::atoi(tv) != 0;
    // the one-block sub-cycle of the small levels and the per-level launches
    // solve the same systems; the variable selects the per-level launches
    if (const char* sv = std::getenv("MPS_SUBCYCLE")) ctx.sub_allowed = std::atoi(sv) != 0;
    if (cudaDeviceGetAttribute(&ctx.nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || ctx.nsm < 1) {
        delete H;
        return MPS_ERR_CUDA;
    }
    if (cudaStreamCreateWithFlags(&ctx.s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx.e0) != cudaSuccess || cudaEventCreate(&ctx.e1) != cudaSuccess ||
        cudaMallocHost((void**)&ctx.hpin, sizeof(double) * 512) != cudaSuccess ||
        cudaMalloc((void**)&ctx.dmax, sizeof(unsigned long long) * 8) != cudaSuccess) {
        delete H;
        return MPS_ERR_CUDA;
    }
    *h = H;
    return MPS_OK;
}

int mps_destroy(mps_handle h)
{
    if (!h) return MPS_ERR_BAD_ARG;
    Ctx& ctx = h->ctx;
    cudaSetDevice(ctx.dev);
    cudaStreamSynchronize(ctx.s);
    destroy_batch(ctx);
    destroy_graphs(ctx);
    ctx.ar.clear();
    ctx.kar.clear();
    ctx.inbuf.clear();
    for (auto& ln : ctx.lanes) {
        if (ln.s) cudaStreamSynchronize(ln.s);
        for (int b = 0; b < 2; b++) {
            if (ln.pin[b]) cudaFreeHost(ln.pin[b]);
            if (ln.ev[b]) cudaEventDestroy(ln.ev[b]);
        }
        if (ln.s) cudaStreamDestroy(ln.s);
    }
    ctx.lanes.clear();
    for (cudaEvent_t e : ctx.prof.ev) cudaEventDestroy(e);
    if (ctx.dtab) cudaFree(ctx.dtab);
    if (ctx.dmax) cudaFree(ctx.dmax);
    if (ctx.hpin) cudaFreeHost(ctx.hpin);
    if (ctx.e0) cudaEventDestroy(ctx.e0);
    if (ctx.e1) cudaEventDestroy(ctx.e1);
    if (ctx.s) cudaStreamDestroy(ctx.s);
    delete h;
    return MPS_OK;
}

void* mps_stream(mps_handle h) { return h ? (void*)h->ctx.s : nullptr; }

const char* mps_last_error(mps_handle h) { return h ? h->ctx.err.msg.c_str() : "null handle"; }

static int run_dev(mps_handle h, const mps_grid* g, int timederiv, double dt, const double* vel, const double* dcoeff,
                   const double* reac, const double* source, const int bc_code[6], const double* const bcval[6],
                   const double* sterm, double* soln, const mps_solver_opts* opts, mps_solve_info* info,
                   void* stream, int ref_norm_only)
{
    if (!h || !bc_code) return MPS_ERR_BAD_ARG;
    Ctx& ctx = h->ctx;
    ctx.err = Err();
    if (cudaSetDevice(ctx.dev) != cudaSuccess) return MPS_ERR_CUDA;
    mps_solver_opts o;
    if (opts) o = *opts;
    else mps_default_opts(&o);
    cudaStream_t user = (cudaStream_t)stream;
    cudaEvent_t ev = nullptr;
    if (user && user != ctx.s) {  // order the handle's stream after the caller's
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return MPS_ERR_CUDA;
        cudaEventRecord(ev, user);
        cudaStreamWaitEvent(ctx.s, ev, 0);
    }
    Inputs in;
    in.vel = vel; in.dcoeff = dcoeff; in.reac = reac; in.source = source; in.sterm = sterm; in.soln = soln;
    for (int f = 0; f < 6; f++) in.bcval[f] = bcval ? bcval[f] : nullptr;
    int st = solve_impl(ctx, g, timederiv, dt, in, bc_code, &o, info, ref_norm_only);
    if (ev) {
        cudaEventRecord(ev, ctx.s);
        cudaStreamWaitEvent(user, ev, 0);
        cudaEventDestroy(ev);
    }
    if (st && info) info->status = st;
    return st;
}

int mps_linsolve_batched_dev(mps_handle h, int nprob, const mps_problem* probs, const mps_solver_opts* opts,
                             mps_solve_info* infos, void* stream)
{
    if (!h) return MPS_ERR_BAD_ARG;
    Ctx& ctx = h->ctx;
    ctx.err = Err();
    if (nprob < 1 || nprob > MPS_BATCH_MAX || !probs) { ctx.err.msg = "batched: bad problem count"; return MPS_ERR_BAD_ARG; }
    if (cudaSetDevice(ctx.dev) != cudaSuccess) return MPS_ERR_CUDA;
    mps_solver_opts o;
    if (opts) o = *opts;
    else mps_default_opts(&o);
    if (o.krylov != MPS_KRYLOV_NONE || o.transpose || o.flux != MPS_FLUX_UPWIND || o.nu1 < 1 ||
        (o.nu1 + o.nu2) % 2 != 0 || (o.precision != MPS_PREC_MIXED && o.precision != MPS_PREC_FP64)) {
        ctx.err.msg = "batched: stationary iteration only (krylov NONE, upwind, no transpose), nu1 >= 1, nu1+nu2 even";
        return MPS_ERR_BAD_ARG;
    }
    cudaStream_t user = (cudaStream_t)stream;
    cudaEvent_t ev = nullptr;
    if (user && user != ctx.s) {
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return MPS_ERR_CUDA;
        cudaEventRecord(ev, user);
        cudaStreamWaitEvent(ctx.s, ev, 0);
    }
    int st = o.precision == MPS_PREC_MIXED ? batched_solve<float>(ctx, nprob, probs, &o, infos)
                                           : batched_solve<double>(ctx, nprob, probs, &o, infos);
    if (ev) {
        cudaEventRecord(ev, ctx.s);
        cudaStreamWaitEvent(user, ev, 0);
        cudaEventDestroy(ev);
    }
    if (st && st != MPS_ERR_NAN) cudaStreamSynchronize(ctx.s);
    return st;
}

int mps_set_profile(mps_handle h, int on)
{
    if (!h) return MPS_ERR_BAD_ARG;
    h->ctx.prof.on = on != 0;
    h->ctx.prof.level = on > 1 ? on - 1 : 0;
    return MPS_OK;
}

int mps_get_profile(mps_handle h, mps_profile* p, int reset)
{
    if (!h || !p) return MPS_ERR_BAD_ARG;
    Prof& P = h->ctx.prof;
    std::memset(p, 0, sizeof(*p));
    for (int c = 0; c < MPS_PROF_NCLASS; c++) { p->count[c] = P.count[c]; p->ms[c] = P.ms[c]; }
    p->precision_bytes = P.precision_bytes;
    p->coeff_field = P.coeff_field;
    p->cells = P.cells;
    if (reset)
        for (int c = 0; c < MPS_PROF_NCLASS; c++) { P.count[c] = 0; P.ms[c] = 0.0; }
    return MPS_OK;
}

int mps_linsolve_dev(mps_handle h, const mps_grid* g, int timederiv, double dt, const double* vel,
                     const double* dcoeff, const double* reac, const double* source, const int bc_code[6],
                     const double* const bcval[6], const double* mgridsterm, double* soln,
                     const mps_solver_opts* opts, mps_solve_info* info, void* stream)
{
    int st = run_dev(h, g, timederiv, dt, vel, dcoeff, reac, source, bc_code, bcval, mgridsterm, soln, opts, info,
                     stream, 0);
    if (st) return st;
    return info ? info->status : MPS_OK;
}

// host-pointer front end: stage the ghosted inputs on the device
// ---- copies between pageable host arrays and the device ----
// A pageable array cannot be read by the DMA engines directly; the driver
// would stage it through its own small pinned buffers one piece at a time.
// Here each of several host threads owns a contiguous part of the array, a
// stream and two pinned chunk buffers: it copies chunk i+1 into one buffer
// (a plain memcpy, in parallel with the other threads) while the DMA engine
// moves chunk i from the other.  Pinned (page-locked or device) arrays go
// straight to cudaMemcpyAsync on the handle's stream.
constexpr size_t kLaneChunk = 1u << 20;  // doubles per chunk buffer (8 MiB)
constexpr int kMaxLanes = 8;

static bool is_pageable(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

static int ensure_lanes(Ctx& ctx)
{
    if (!ctx.lanes.empty()) return 0;
    const unsigned hc = std::thread::hardware_concurrency();
    const int n = std::max(1, std::min<int>(kMaxLanes, hc ? (int)hc / 2 : 4));
    ctx.lanes.resize(n);
    for (auto& ln : ctx.lanes) {
        if (cudaStreamCreateWithFlags(&ln.s, cudaStreamNonBlocking) != cudaSuccess) return MPS_ERR_CUDA;
        for (int b = 0; b < 2; b++) {
            if (cudaMallocHost((void**)&ln.pin[b], sizeof(double) * kLaneChunk) != cudaSuccess) return MPS_ERR_NOMEM;
            if (cudaEventCreateWithFlags(&ln.ev[b], cudaEventDisableTiming) != cudaSuccess) return MPS_ERR_CUDA;
        }
    }
    return 0;
}

struct HostCopy {
    double* dev;        // device array
    double* host;       // pageable host array (const for H2D)
    size_t n;           // doubles
};

// all copies of one direction, each array split across the lanes; the
// handle's stream is ordered after (H2D) or the host waits for (D2H) them
static int staged_copies(Ctx& ctx, const std::vector<HostCopy>& cps, bool h2d)
{
    if (cps.empty()) return 0;
    if (int st = ensure_lanes(ctx)) return st;
    const int nl = (int)ctx.lanes.size();
    if (!h2d) {  // the results must be complete before the lanes read them
        cudaEvent_t e = ctx.e1;
        if (cudaEventRecord(e, ctx.s) != cudaSuccess) return MPS_ERR_CUDA;
        for (auto& ln : ctx.lanes)
            if (cudaStreamWaitEvent(ln.s, e, 0) != cudaSuccess) return MPS_ERR_CUDA;
    }
    std::vector<int> status(nl, 0);
    auto work = [&](int li) {
        Ctx::Lane& ln = ctx.lanes[li];
        int b = 0;
        bool used[2] = {false, false};
        for (const HostCopy& cp : cps) {
            // lane shares start on 4 KiB boundaries of the device array
            const size_t part = ((cp.n + nl - 1) / nl + 511) / 512 * 512;
            const size_t lo = std::min(cp.n, part * li), hi = std::min(cp.n, lo + part);
            for (size_t o = lo; o < hi; o += kLaneChunk) {
                const size_t m = std::min(kLaneChunk, hi - o);
                if (used[b] && cudaEventSynchronize(ln.ev[b]) != cudaSuccess) { status[li] = MPS_ERR_CUDA; return; }
                if (h2d) {
                    std::memcpy(ln.pin[b], cp.host + o, sizeof(double) * m);
                    if (cudaMemcpyAsync(cp.dev + o, ln.pin[b], sizeof(double) * m, cudaMemcpyHostToDevice, ln.s) !=
                        cudaSuccess) { status[li] = MPS_ERR_CUDA; return; }
                    if (cudaEventRecord(ln.ev[b], ln.s) != cudaSuccess) { status[li] = MPS_ERR_CUDA; return; }
                } else {
                    if (cudaMemcpyAsync(ln.pin[b], cp.dev + o, sizeof(double) * m, cudaMemcpyDeviceToHost, ln.s) !=
                            cudaSuccess ||
                        cudaStreamSynchronize(ln.s) != cudaSuccess) { status[li] = MPS_ERR_CUDA; return; }
                    std::memcpy(cp.host + o, ln.pin[b], sizeof(double) * m);
                }
                used[b] = true;
                b ^= 1;
            }
        }
        if (cudaStreamSynchronize(ln.s) != cudaSuccess) status[li] = MPS_ERR_CUDA;
    };
    std::vector<std::thread> th;
    for (int li = 1; li < nl; li++) th.emplace_back(work, li);
    work(0);
    for (auto& t : th) t.join();
    for (int st : status)
        if (st) return st;
    return 0;
}

static int run_host(mps_handle h, const mps_grid* g, int timederiv, double dt, const double* vel,
                    const double* dcoeff, const double* reac, const double* source, const int bc_code[6],
                    const double* const bcval[6], const double* mgridsterm, double* soln,
                    const mps_solver_opts* opts, mps_solve_info* info, int ref_norm_only)
{
    if (!h || !g || !dcoeff || !source || !soln || !bc_code) return MPS_ERR_BAD_ARG;
    if (g->lx < 1 || g->ly < 1 || g->lz < 1) return MPS_ERR_BAD_ARG;
    Ctx& ctx = h->ctx;
    if (cudaSetDevice(ctx.dev) != cudaSuccess) return MPS_ERR_CUDA;
    const size_t ng = (size_t)(g->lx + 2) * (g->ly + 2) * (g->lz + 2);
    const size_t ni = (size_t)g->lx * g->ly * g->lz;
    const size_t fs[6] = {(size_t)g->ly * g->lz, (size_t)g->ly * g->lz, (size_t)g->lx * g->lz,
                          (size_t)g->lx * g->lz, (size_t)g->lx * g->ly, (size_t)g->lx * g->ly};
    // one device block for the staged inputs, every field starting on a
    // 4 KiB boundary (copies into 8-byte aligned destinations ran at 37-40
    // GB/s over the host link, aligned ones at 55 GB/s)
    auto al = [](size_t n) { return (n * sizeof(double) + 4095) / 4096 * 4096 / sizeof(double); };
    size_t need = al(3 * ng) + 4 * al(ng) + al(ni) + al(fs[0] * 2 + fs[2] * 2 + fs[4] * 2);
    need *= sizeof(double);
    if (ctx.inbuf_bytes < need) {
        ctx.inbuf.clear();
        ctx.inbuf_bytes = 0;
        if (!ctx.inbuf.get(need)) return MPS_ERR_NOMEM;
        if (cudaDeviceSynchronize() != cudaSuccess) return MPS_ERR_CUDA;
        ctx.inbuf_bytes = need;
    }
    double* base = (double*)ctx.inbuf.blocks[0];
    double* d_vel = base;
    double* d_dc = d_vel + al(3 * ng);
    double* d_re = d_dc + al(ng);
    double* d_src = d_re + al(ng);
    double* d_sol = d_src + al(ng);
    double* d_st = d_sol + al(ng);
    double* d_bc = d_st + al(ni);
    const double* dbv[6];
    cudaStream_t s = ctx.s;
    // pinned (or device) arrays: one cudaMemcpyAsync each on the handle's
    // stream; pageable arrays: the staged, multi-threaded copies above
    std::vector<HostCopy> staged;
    auto h2d = [&](double* dst, const double* src, size_t n) -> int {
        if (is_pageable(src)) {
            staged.push_back({dst, const_cast<double*>(src), n});
            return 0;
        }
        return cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, s) == cudaSuccess ? 0
                                                                                                       : MPS_ERR_CUDA;
    };
    int st = 0;
    if (vel && (st = h2d(d_vel, vel, 3 * ng))) return st;
    if ((st = h2d(d_dc, dcoeff, ng))) return st;
    if (reac && (st = h2d(d_re, reac, ng))) return st;
    if ((st = h2d(d_src, source, ng))) return st;
    if ((st = h2d(d_sol, soln, ng))) return st;
    if (mgridsterm && (st = h2d(d_st, mgridsterm, ni))) return st;
    double* p = d_bc;
    for (int f = 0; f < 6; f++) {
        dbv[f] = nullptr;
        if (bcval && bcval[f]) {
            if ((st = h2d(p, bcval[f], fs[f]))) return st;
            dbv[f] = p;
        }
        p += fs[f];
    }
    if ((st = staged_copies(ctx, staged, true))) return st;  // complete when it returns
    st = run_dev(h, g, timederiv, dt, vel ? d_vel : nullptr, d_dc, reac ? d_re : nullptr, d_src, bc_code, dbv,
                 mgridsterm ? d_st : nullptr, d_sol, opts, info, nullptr, ref_norm_only);
    if (st) return st;
    if (is_pageable(soln)) {
        if ((st = staged_copies(ctx, {HostCopy{d_sol, soln, ng}}, false))) return st;
    } else {
        if (cudaMemcpyAsync(soln, d_sol, sizeof(double) * ng, cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return MPS_ERR_CUDA;
        if (cudaStreamSynchronize(s) != cudaSuccess) return MPS_ERR_CUDA;
    }
    return info ? info->status : MPS_OK;
}

int mps_linsolve(mps_handle h, const mps_grid* g, int timederiv, double dt, const double* vel, const double* dcoeff,
                 const double* reac, const double* source, const int bc_code[6], const double* const bcval[6],
                 const double* mgridsterm, double* soln, const mps_solver_opts* opts, mps_solve_info* info)
{
    return run_host(h, g, timederiv, dt, vel, dcoeff, reac, source, bc_code, bcval, mgridsterm, soln, opts, info, 0);
}

int mps_vcycle_once(mps_handle h, const mps_grid* g, int timederiv, double dt, const double* vel,
                    const double* dcoeff, const double* reac, const double* source, const int bc_code[6],
                    const double* const bcval[6], const double* mgridsterm, double* soln, double* resnorm,
                    const mps_solver_opts* opts)
{
    mps_solver_opts o;
    if (opts) o = *opts;
    else {
        mps_default_opts(&o);
        o.hierarchy = MPS_HIER_CELL;
    }
    o.maxit = 1;
    o.krylov = MPS_KRYLOV_NONE;
    o.precision = MPS_PREC_FP64;
    mps_solve_info info;
    int st = run_host(h, g, timederiv, dt, vel, dcoeff, reac, source, bc_code, bcval, mgridsterm, soln, &o, &info, 1);
    if (resnorm) *resnorm = info.rms_res;
    return st;
}

int mps_apply_A_dev(mps_handle h, const mps_grid* g, int timederiv, double dt, const double* vel,
                    const double* dcoeff, const double* reac, const int bc_code[6], const double* soln, double* AX,
                    const mps_solver_opts* opts, void* stream)
{
    if (!h || !g || !dcoeff || !soln || !AX || !bc_code) return MPS_ERR_BAD_ARG;
    Ctx& ctx = h->ctx;
    ctx.err = Err();
    if (cudaSetDevice(ctx.dev) != cudaSuccess) return MPS_ERR_CUDA;
    mps_solver_opts o;
    if (opts) o = *opts;
    else mps_default_opts(&o);
    // A u through the same operator setup as a solve: run a zero-iteration
    // solve to build the fine operator, then apply it
    o.maxit = 0;
    o.krylov = MPS_KRYLOV_NONE;
    o.precision = MPS_PREC_FP64;
    o.hierarchy = MPS_HIER_GEOM;
    const size_t ng = (size_t)(g->lx + 2) * (g->ly + 2) * (g->lz + 2);
    double* tmp = nullptr;
    double* zsrc = nullptr;
    cudaStream_t s = ctx.s;
    cudaStream_t user = (cudaStream_t)stream;
    if (user && user != s) {  // soln is read below, before the solve orders the streams
        cudaEvent_t ev = nullptr;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return MPS_ERR_CUDA;
        cudaEventRecord(ev, user);
        cudaStreamWaitEvent(s, ev, 0);
        cudaEventDestroy(ev);
    }
    if (cudaMallocAsync((void**)&tmp, sizeof(double) * ng * 2, s) != cudaSuccess) return MPS_ERR_CUDA;
    zsrc = tmp + ng;
    cudaMemcpyAsync(tmp, soln, sizeof(double) * ng, cudaMemcpyDeviceToDevice, s);
    cudaMemsetAsync(zsrc, 0, sizeof(double) * ng, s);
    int bcfix[6];
    for (int f = 0; f < 6; f++) bcfix[f] = bc_code[f];
    mps_solve_info info;
    // DIRC/FLUX faces need value arrays for find_bvec; they do not enter A
    int st = MPS_OK;
    std::vector<double*> fb;
    const double* bv[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int f = 0; f < 6 && st == MPS_OK; f++) {
        if (bc_code[f] == BC_DIRC || bc_code[f] == BC_FLUX) {
            size_t n = (f < 2) ? (size_t)g->ly * g->lz : (f < 4 ? (size_t)g->lx * g->lz : (size_t)g->lx * g->ly);
            double* d = nullptr;
            if (cudaMallocAsync((void**)&d, sizeof(double) * n, s) != cudaSuccess) {
                st = MPS_ERR_CUDA;
                break;
            }
            cudaMemsetAsync(d, 0, sizeof(double) * n, s);
            fb.push_back(d);
            bv[f] = d;
        }
    }
    if (st == MPS_OK)
        st = run_dev(h, g, timederiv, dt, vel, dcoeff, reac, zsrc, bcfix, bv, nullptr, tmp, &o, &info, stream, 1);
    if (st == MPS_OK) {
        const Lev& L = ctx.lev[0];
        double* out = nullptr;
        if (cudaMallocAsync((void**)&out, sizeof(double) * 2 * L.half, s) != cudaSuccess) {
            st = MPS_ERR_CUDA;
        } else {
            if (ctx.sig.opclass == 0)
                k_apply<double, KOp<double>, double><<<nblk((long long)L.P * L.rows), TPB, 0, s>>>(
                    L, ctx.kop64, csplit<double>(ctx.x64, L), split<double>(out, L));
            else
                k_apply<double, ROp<double>, double><<<nblk((long long)L.P * L.rows), TPB, 0, s>>>(
                    L, ctx.rop64, csplit<double>(ctx.x64, L), split<double>(out, L));
            k_unpack_nat<double><<<nblk((long long)L.nx * L.ny * L.nz), TPB, 0, s>>>(L, csplit<double>(out, L), AX);
            cudaFreeAsync(out, s);
            if (cudaGetLastError() != cudaSuccess) st = MPS_ERR_CUDA;
        }
    }
    // every exit path frees what this call allocated and waits for the stream
    for (double* d : fb) cudaFreeAsync(d, s);
    cudaFreeAsync(tmp, s);
    if (cudaStreamSynchronize(s) != cudaSuccess && st == MPS_OK) st = MPS_ERR_CUDA;
    return st;
}

int mps_find_bvec_dev(mps_handle h, const mps_grid* g, const double* vel, const double* dcoeff,
                      const double* source, const int bc_code[6], const double* const bcval[6],
                      const double* mgridsterm, double* b, const mps_solver_opts* opts, void* stream)
{
    if (!h || !g || !dcoeff || !source || !b || !bc_code) return MPS_ERR_BAD_ARG;
    Ctx& ctx = h->ctx;
    if (cudaSetDevice(ctx.dev) != cudaSuccess) return MPS_ERR_CUDA;
    for (int f = 0; f < 6; f++)
        if (bc_code[f] < 1 || bc_code[f] > 5 || (!(bcval && bcval[f]) && (bc_code[f] == BC_DIRC || bc_code[f] == BC_FLUX)))
            return MPS_ERR_BAD_ARG;
    const double llen[3] = {g->llenx, g->lleny, g->llenz};
    Lev L = make_lev_uniform(g->lx, g->ly, g->lz, llen, bc_code);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx.s;
    double* buf = nullptr;
    if (cudaMallocAsync((void**)&buf, sizeof(double) * 2 * L.half, s) != cudaSuccess) return MPS_ERR_CUDA;
    cudaMemsetAsync(buf, 0, sizeof(double) * 2 * L.half, s);
    const long long n = (long long)L.nx * L.ny * L.nz;
    k_find_bvec<<<nblk(n), TPB, 0, s>>>(L, vel, dcoeff, source, bcval[0], bcval[1], bcval[2], bcval[3], bcval[4],
                                        bcval[5], mgridsterm, opts ? opts->flux : 0, split<double>(buf, L));
    k_unpack_nat<double><<<nblk(n), TPB, 0, s>>>(L, csplit<double>(buf, L), b);
    cudaFreeAsync(buf, s);
    if (cudaGetLastError() != cudaSuccess) return MPS_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MPS_ERR_CUDA;
    return MPS_OK;
}

int mps_fill_ghosts_dev(mps_handle h, const mps_grid* g, const int bc_code[6], const double* const bcval[6],
                        double* soln, void* stream)
{
    if (!h || !g || !soln || !bc_code) return MPS_ERR_BAD_ARG;
    Ctx& ctx = h->ctx;
    if (cudaSetDevice(ctx.dev) != cudaSuccess) return MPS_ERR_CUDA;
    for (int f = 0; f < 6; f++)
        if (bc_code[f] < 1 || bc_code[f] > 5 || (!(bcval && bcval[f]) && bc_code[f] == BC_DIRC)) return MPS_ERR_BAD_ARG;
    const double llen[3] = {g->llenx, g->lleny, g->llenz};
    Lev L = make_lev_uniform(g->lx, g->ly, g->lz, llen, bc_code);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx.s;
    const int mx = std::max(std::max(L.ny * L.nz, L.nx * L.nz), L.nx * L.ny);
    k_fill_ghosts<<<nblk(mx), TPB, 0, s>>>(L, soln, bcval ? bcval[0] : nullptr, bcval ? bcval[1] : nullptr,
                                           bcval ? bcval[2] : nullptr, bcval ? bcval[3] : nullptr,
                                           bcval ? bcval[4] : nullptr, bcval ? bcval[5] : nullptr);
    if (cudaGetLastError() != cudaSuccess) return MPS_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MPS_ERR_CUDA;
    return MPS_OK;
}

}  // extern "C"
