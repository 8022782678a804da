// kernels.cuh - sm_100a kernels of the cavity time step (Eulerian impulse scheme on a staggered MAC grid).
//
// Field layout in HBM: one array per component, [z][y][x] with x fastest, exactly the reference's layout
// (backend.cu:10-12) so host copies need no reshuffle.  u: (nx+1, ny, nz), v: (nx, ny+1, nz),
// w: (nx, ny, nz+1); cell arrays (phi, rhs, residual, history) (nx, ny, nz).  T is the field type: double
// for the FP64 form, float for the mixed form.  The projection (divergence, potential, residual, gradient)
// is FP64 in both forms, as in the reference.
//
// Grid coefficients are precomputed per axis on the host (reciprocals of widths and spacings, the
// interpolation weights and wall ramps of the 4th-order Lamb stencil) and read through L1 from one table
// block per axis.
//
// Every scalar decision of a step (dt, pressure-pass count, guess rejection, errors, clock) is made on the
// device in a `Control` block, so a whole step runs without the host: the last block of a reduction kernel
// (a fixed-order, deterministic reduction) takes the decision and, inside a CUDA graph, sets the condition
// of the refinement loop's while-node.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "layout.h"

namespace cavity {

// ------------------------------------------------------------------------------------------ launch recording
// Host side.  While a recorder is installed on the calling thread, the launch helpers of a solver append their
// launch (kind, template variant, grid, dynamic shared memory and argument record) to it instead of launching:
// a batch of cavities collects every member's arguments for the same launch sequence this way and issues one
// batched launch per entry.
enum SweepKind : int { kSweepFace = 0, kSweepTile = 1, kSweepMarch = 2, kSweepPair = 3 };
enum LaunchKind : int { kLkStepBegin = 0, kLkSweep, kLkStart, kLkResidual, kLkFinish, kLkDgemm64, kLkDgemm32, kLkTc,
                        kLkPair };
struct LaunchRecord {
    int kind, variant;
    dim3 grid;
    size_t smem;
    std::vector<unsigned char> args;
};
inline thread_local std::vector<LaunchRecord>* g_launch_record = nullptr;
// number of cavities the recorded launches will cover: tile choices that depend on the size of the grid use it
inline thread_local int g_launch_batch = 1;
// FP64 transform tile forced for every cavity of a batch whose cavities differ in size (0: chosen by size)
inline thread_local int g_dgemm_tile = 0;
// a batch's FP64 passes as three paired launches (1) or six (0); -1 outside a batch
inline thread_local int g_batch_pairs = -1;
// launch a step kernel with programmatic stream serialization (see pdl_wait); inside a stream capture this makes
// the graph edge to the previous kernel a programmatic one
template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}
template <class A> inline bool record_launch(int kind, int variant, dim3 grid, size_t smem, const A& a) {
    if (!g_launch_record) return false;
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&a);
    g_launch_record->push_back(LaunchRecord{kind, variant, grid, smem, std::vector<unsigned char>(b, b + sizeof a)});
    return true;
}

constexpr int kThreads = 256;
constexpr int X = 0, Y = 1, Z = 2;

// ------------------------------------------------------------------------------------------ control block
enum ErrorCode : int {
    kOk = 0,
    kVelocityNaN = 1,      // backend.cu:890
    kRhsNaN = 2,           // backend.cu:820
    kResidualNaN = 3,      // backend.cu:838
    kNotConverged = 4,     // backend.cu:840-844
    kDeviceWait = 5,       // a bounded wait on the tensor cores ran out (no counterpart in the reference)
    kBarrierWait = 6,      // a bounded grid-barrier wait of the one-launch FDM pass ran out (no counterpart)
};
// arrival counters of the last-block reductions, and the grid barrier's arrival count and generation
enum Counter : int { kCntDiv = 0, kCntRes, kCntFinish, kCntCfl, kCntBar, kCntBarGen, kNumCounters };

struct alignas(16) Control {
    // clock, committed by the last stage of a successful step (backend.cu:945-954)
    double t, last_dt, last_cfl, phi_rel;
    long long steps;
    int dt_reason, phi_passes;
    // dt decision (backend.cu:885-899)
    double cfl_rate;            // max CFL rate of the current velocity (NaN wins)
    double prev_rates[2];
    int have_prev, pad0;
    double dt, use0;
    // current pressure solve (backend.cu:816-847)
    double rhs_norm2, res_norm2, phi_sum, rhs_norm, rel;
    int passes, use_rhs, reset_phi, zero_rhs;
    int cond, stage, pad1, pad2;
    // warm-start history: last three potential increments (backend.cu:857-873, 929-939)
    double hist_t[3], hist_scale[3];
    int hist_buf[3], hist_count;
    // status
    int error, error_passes;
    double error_value;
    long long pass_count;       // pressure passes run since creation (launch accounting)
    unsigned int counter[kNumCounters];
    unsigned int pad3[8 - kNumCounters % 8];
};

// settings that stay fixed for a solver (copied into kernel parameters)
struct Params {
    int nx, ny, nz, n_cell;
    int o4;                      // 4th-order Lamb vector
    int adaptive_dt, dt_lag, phi_extrapolate, fdm_max_passes;
    double nu, u_lid, lid_ramp_t, reinit_r, dt_fixed, dt_max, cfl_target, diffusion_limit, fdm_rtol;
    double viscous_rate;         // float-computed on the host, as backend.cu:1030-1034
};


template <class T> struct Geo {
    const T* tab[3];             // tab[a][k * stride[a] + i + kTabOffset]
    int stride[3];
    const double* dw[3];         // widths (double, float-rounded values)
    const double* dinv_sp[3];    // 1/spacing in double
    const T* lid_u;              // lid shape on the top u-faces, [z][x] with nx+1 per row
};

template <class T> __device__ __forceinline__ T tab(const Geo<T>& g, int a, int k, int i) {
    return g.tab[a][k * g.stride[a] + i + kTabOffset];
}

// flat index of component C at (x, y, z)
template <int C> __device__ __forceinline__ int fidx(const Params& p, int x, int y, int z) {
    const int ex = p.nx + (C == X), ey = p.ny + (C == Y);
    return x + ex * (y + ey * z);
}
// flat index of component C given the coordinates along axes A, B and the third axis
template <int C, int A, int B> __device__ __forceinline__ int fidx_ab(const Params& p, int va, int vb, int vd) {
    int q[3];
    q[A] = va;
    q[B] = vb;
    q[3 - A - B] = vd;
    return fidx<C>(p, q[0], q[1], q[2]);
}
__device__ __forceinline__ int cidx(const Params& p, int x, int y, int z) { return x + p.nx * (y + p.ny * z); }

__device__ __forceinline__ double lid_speed(const Params& p, double time) {     // backend.cu:623-626
    if (p.lid_ramp_t > 0) return p.u_lid * fmin(1.0, fmax(time, 0.0) / p.lid_ramp_t);
    return p.u_lid;
}

// ------------------------------------------------------------------------------------------ reductions
// Block reduction of N doubles in a fixed tree (deterministic for a fixed block size).
template <int N> struct Vec { double v[N]; };

template <int N, bool MAX>
__device__ __forceinline__ double combine(double a, double b) {
    if (MAX) return (a != a || a > b) ? a : b;       // NaN wins a max (backend.cu:427-429)
    return a + b;
}

template <int N, bool MAX>
__device__ Vec<N> block_reduce(Vec<N> x) {
    __shared__ double sh[N][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < N; k++) {
        double v = x.v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = combine<N, MAX>(v, __shfl_down_sync(0xffffffffu, v, o));
        if (lane == 0) sh[k][warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < N; k++) {
            double v = lane < kThreads / 32 ? sh[k][lane] : (MAX ? -INFINITY : 0.0);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = combine<N, MAX>(v, __shfl_down_sync(0xffffffffu, v, o));
            x.v[k] = v;
        }
    }
    __syncthreads();
    return x;   // valid in thread 0
}

// ------------------------------------------------------------------------------------------ batches
// A kernel body sees its block index and grid through a Blk: the launch's own (real_blk) when it runs for one
// cavity, or its cavity's share of a batched launch (batch_blk), where the cavities of a batch follow each other
// along grid axis z, `per` z-blocks each, and every block reads its cavity's arguments from a device array.
struct Blk {
    unsigned int x, y, z, nx, ny, nz;
};
__device__ __forceinline__ Blk real_blk() { return {blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y, gridDim.z}; }
// A batched launch runs a work list: one entry per block, naming the cavity and the block's place in that
// cavity's own launch grid, so cavities of different sizes share a launch (grid x runs over the list).
struct BatchItem {
    unsigned int cav, x, y, z, nx, ny, nz, pad;
};
// `live` holds one flag per slot of the batch: the blocks of an empty slot return at once (see Batch::set_member)
__device__ __forceinline__ Blk item_blk(const BatchItem* items, const int* live, int& cavity) {
    const BatchItem it = items[blockIdx.x];
    cavity = live[it.cav] ? (int)it.cav : -1;
    return {it.x, it.y, it.z, it.nx, it.ny, it.nz};
}
// The first transform of a pass clears the condition of the refinement loop's while-node, in the launch's first
// block: the loop would never end without it.  When that block belongs to an empty slot it still clears: the
// slot's argument record (a member's, written when the graph was built or the slot last held a cavity) names
// the same loop.
template <class A> __device__ __forceinline__ void dead_slot_clear(const A* args, const BatchItem* items) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const A& r = args[items[0].cav];
    if (r.clear_condition) cudaGraphSetConditional(r.handle, 0u);
}
__device__ __forceinline__ bool first_block() { return blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0; }
// Cells visited as columns: a block takes kThreads consecutive cells of an x-y plane (x fastest) and walks them
// up a chunk of z-layers; grid y runs over the chunks.  A thread's plane position, and so its x and y table
// values, stay fixed, and its column's values below and at the current layer carry over in registers.
// blocks of a column kernel an SM is to hold: its loads run one layer ahead, so occupancy is its memory parallelism
constexpr int kColumnBlocks = 4;
constexpr int kResidualBlocks = 3;      // the residual's pairs of cells hold more in flight per thread
struct ColumnSpan {
    int p, x, y, z0, z1;
    bool live;
};
// `per` consecutive cells of a row per thread (2: a pair starting at an even x; nx is even); s.p is the first
__device__ __forceinline__ ColumnSpan column_span(const Params& p, const Blk& k, int per = 1) {
    ColumnSpan s;
    const int plane = p.nx * p.ny;
    s.p = ((int)k.x * kThreads + (int)threadIdx.x) * per;
    s.live = s.p < plane;
    s.x = s.p % p.nx;
    s.y = s.p / p.nx;
    const int zc = (p.nz + (int)k.ny - 1) / (int)k.ny;
    s.z0 = (int)k.y * zc;
    s.z1 = min(p.nz, s.z0 + zc);
    return s;
}
// Layers of a column walk that are brought into L2 ahead of the one whose loads go out into registers: the L2
// prefetch holds no register, so it deepens the walk's memory parallelism for free.
constexpr int kColumnL2Ahead = 1;
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
// Programmatic dependent launch: the step kernels are launched so that the next kernel may start while this one
// finishes.  Every step kernel lets its dependents launch at entry and waits for its predecessor to complete
// (with all its memory visible) before it reads anything a predecessor wrote.  Both are no-ops for a kernel
// launched without the attribute.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// copy a cavity's kernel arguments into shared memory (the whole block, then a barrier)
template <class A> __device__ __forceinline__ void load_args(A& dst, const A* src) {
    static_assert(sizeof(A) % 4 == 0, "argument records are copied in words");
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(A) / 4); i += blockDim.x) d[i] = s[i];
    __syncthreads();
}

// Write this block's partials; returns true in every thread of the last block to finish, after which the
// partials of all blocks are visible to it.  The last block resets the counter for the next launch.
template <int N>
__device__ bool publish_partials(const Vec<N>& blk, double* partial, unsigned int* counter, const Blk& k) {
    __shared__ bool last;
    const unsigned int nblocks = k.nx * k.ny;
    const unsigned int b = k.x + k.nx * k.y;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < N; k++) partial[k * nblocks + b] = blk.v[k];
        __threadfence();
        const unsigned int done = atomicAdd(counter, 1u);
        last = (done == nblocks - 1);
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

template <int N>
__device__ bool publish_partials(const Vec<N>& blk, double* partial, unsigned int* counter) {
    return publish_partials(blk, partial, counter, real_blk());
}

// In the last block: reduce all partials in a fixed order (thread t combines the partials of blocks t, t + NT,
// t + 2 NT, ... in that order, then the block reduces).  Result valid in thread 0.  The loads of all N sums and
// of four block indices per thread are issued together before any is combined: this reduction is the tail of
// every reducing kernel, and the next kernel waits for it, so it should cost one L2 round trip per four
// indices, not one per sum and index.
template <int N, bool MAX>
__device__ Vec<N> final_reduce(const double* partial, const Blk& k) {
    constexpr int U = 4;
    const unsigned int nblocks = k.nx * k.ny, nt = blockDim.x;
    Vec<N> acc;
#pragma unroll
    for (int j = 0; j < N; j++) acc.v[j] = MAX ? -INFINITY : 0.0;
    for (unsigned int base = threadIdx.x; base < nblocks; base += U * nt) {
        double v[U][N];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned int i = base + u * nt;
#pragma unroll
            for (int j = 0; j < N; j++) v[u][j] = i < nblocks ? __ldcg(partial + j * nblocks + i) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (base + u * nt >= nblocks) break;
#pragma unroll
            for (int j = 0; j < N; j++) acc.v[j] = combine<N, MAX>(acc.v[j], v[u][j]);
        }
    }
    return block_reduce<N, MAX>(acc);
}
template <int N, bool MAX>
__device__ Vec<N> final_reduce(const double* partial) {
    return final_reduce<N, MAX>(partial, real_blk());
}

// ------------------------------------------------------------------------------------------ step begin
// dt from the CFL rate of the current velocity and the viscous rate (backend.cu:884-899).
struct StepBeginArgs {
    Params p;
    Control* c;
};
__device__ void step_begin_body(const Params& p, Control* c) {
    pdl_launch_dependents();
    pdl_wait();
    if (threadIdx.x != 0) return;
    if (c->error) return;          // an earlier queued step failed: leave everything as it is
    const double rates[2] = {(double)(float)c->cfl_rate, p.viscous_rate};
    double use[2] = {rates[0], rates[1]};
    if (p.dt_lag && c->have_prev) { use[0] = c->prev_rates[0]; use[1] = c->prev_rates[1]; }
    c->prev_rates[0] = rates[0];
    c->prev_rates[1] = rates[1];
    c->have_prev = 1;
    if (!isfinite(use[0])) { c->error = kVelocityNaN; c->dt = 0; return; }
    double dt;
    if (!p.adaptive_dt) { dt = p.dt_fixed; c->dt_reason = 0; }
    else {
        const double caps[3] = {p.dt_max, p.cfl_target / fmax(use[0], 1e-300), p.diffusion_limit / fmax(use[1], 1e-300)};
        int best = 0;
        for (int k = 1; k < 3; k++)
            if (caps[k] < caps[best]) best = k;
        dt = caps[best];
        c->dt_reason = best + 1;
    }
    if (p.dt_lag && c->last_dt > 0) dt = fmin(dt, 1.1 * c->last_dt);
    c->dt = dt;
    c->use0 = use[0];
}
__global__ void step_begin_kernel(Params p, Control* c) {
    if (blockIdx.x == 0) step_begin_body(p, c);
}
// one block per cavity of the batch
__global__ void step_begin_batched(const StepBeginArgs* args, const int* live) {
    if (!live[blockIdx.z]) return;
    const StepBeginArgs& a = args[blockIdx.z];
    step_begin_body(a.p, a.c);
}

// ------------------------------------------------------------------------------------------ stage constants
struct StageConst {
    double a0, b, tau;
};
__device__ __forceinline__ StageConst stage_const(int stage, const Control* c) {   // backend.cu:902-903
    StageConst s;
    if (stage == 0) { s.a0 = 0.0; s.b = 1.0; s.tau = c->t; }
    else if (stage == 1) { s.a0 = 0.75; s.b = 0.25; s.tau = c->t + c->dt; }
    else { s.a0 = 1.0 / 3.0; s.b = 2.0 / 3.0; s.tau = c->t + 0.5 * c->dt; }
    return s;
}

// ------------------------------------------------------------------------------------------ momentum sweep
// Arguments of the momentum sweep (sweep.cuh): one RK3 stage of the impulse on every face.
template <class T> struct MomentumArgs {
    Params p;
    Geo<T> g;
    const T* u[3];      // velocity of this stage
    const T* m[3];      // impulse of this stage (stage 0: the state impulse, blended on the fly)
    const T* m0[3];     // RK base (stages 1, 2)
    T* m0_out[3];       // stage 0 writes m0 here
    T* out[3];          // new impulse
    const Control* c;
    int stage;
    T r, one_minus_r;   // gauge-reset weights
    T nu;
};

// ------------------------------------------------------------------------------------------ start of a projection
// rhs = volume * div(m) in FP64 (backend.cu:334-342) and the starting potential of the solve.  In a step that is
// the warm-start guess: the potential carried by the RK combination (base, backend.cu:922-923) plus the
// extrapolated increments (backend.cu:924-925, 857-873); stage 0 also stores phi0 = r phi (backend.cu:882).
// Its residual r = rhs - L guess (backend.cu:825-829) needs the guess of neighbouring cells, so the start mode
// of the residual kernel computes it next and takes the decisions that depend on it.  A plain projection
// (initialize, kick) starts from zero with r = rhs.  The last block takes the reference's start-of-solve
// decisions (backend.cu:818-831) that need only the right-hand side: NaN (error), zero (phi = 0, no pass), and,
// starting from zero, whether the refinement loop runs.  Column walk (ColumnSpan).
template <class T> struct StartArgs {
    Params p;
    Geo<T> g;
    const T* m[3];
    double* rhs;
    double* res;
    double* guess;              // the starting potential (the buffer the solve refines)
    // step only (base == nullptr: a plain projection)
    const double* phi_state;    // stage 0: state potential
    double* phi0;               // stage 0 writes, stages 1, 2 read
    const double* phi_cur;      // stages 1, 2: potential of the previous stage
    double* base;
    const double* hist[4];
    int stage;
    Control* c;
    double* partial;
    cudaGraphConditionalHandle handle;
    int use_handle;
};

__device__ __forceinline__ void guess_coefficients(const Params& p, const Control* c, double tau, double scale,
                                                   int& b1, double& c1, int& b2, double& c2) {
    // nearest history entries in time, later first on ties (backend.cu:857-873)
    b1 = -1; b2 = -1; c1 = 0; c2 = 0;
    const int n = c->hist_count;
    if (!p.phi_extrapolate || n == 0) return;
    int order[3] = {0, 1, 2};
    for (int i = 1; i < n; i++) {          // stable insertion sort by (|t - tau|, later first)
        int k = order[i], j = i - 1;
        const double dk = fabs(c->hist_t[k] - tau);
        while (j >= 0) {
            const int o = order[j];
            const double dj = fabs(c->hist_t[o] - tau);
            const bool before = dk != dj ? dk < dj : k > o;
            if (!before) break;
            order[j + 1] = o;
            j--;
        }
        order[j + 1] = k;
    }
    const int h1 = order[0];
    int h2 = -1;
    for (int k = 1; k < n && h2 < 0; k++)
        if (fabs(c->hist_t[order[k]] - c->hist_t[h1]) > 1e-12 * fmax(1.0, fabs(c->hist_t[h1]))) h2 = order[k];
    const double w2 = h2 >= 0 ? (tau - c->hist_t[h1]) / (c->hist_t[h2] - c->hist_t[h1]) : 0.0, w1 = 1.0 - w2;
    b1 = c->hist_buf[h1];
    c1 = scale * w1 / c->hist_scale[h1];
    if (h2 >= 0) {
        b2 = c->hist_buf[h2];
        c2 = scale * w2 / c->hist_scale[h2];
    }
}

// use_handle: 0 = no graph loop, 1 = this cavity's own loop, 2 = a loop shared by a batch of cavities, which
// runs while any cavity needs it (only ever set here; the first transform of each pass clears it)
__device__ __forceinline__ void set_loop(Control* c, cudaGraphConditionalHandle h, int use_handle, int cond) {
    c->cond = cond;
    if (use_handle == 1) cudaGraphSetConditional(h, cond ? 1u : 0u);
    else if (use_handle == 2 && cond) cudaGraphSetConditional(h, 1u);
}

// decision after a residual: more passes, convergence, or the non-convergence error (backend.cu:832-845)
__device__ __forceinline__ void decide_loop(const Params& p, Control* c, cudaGraphConditionalHandle h, int use_handle) {
    const int more = c->rel > p.fdm_rtol && c->passes < p.fdm_max_passes;
    if (!more && c->rel > p.fdm_rtol) {
        c->error = kNotConverged;
        c->error_value = c->rel;
        c->error_passes = c->passes;
    }
    if (!more) c->phi_rel = c->rel;
    set_loop(c, h, use_handle, more);
}

template <class T>
__device__ void projection_start_body(const StartArgs<T>& a, const Blk& k) {
    pdl_launch_dependents();
    pdl_wait();
    Control* c = a.c;
    const Params& p = a.p;
    const int err = c->error;
    const bool have_guess = a.base != nullptr;
    const StageConst sc = stage_const(a.stage, c);
    int b1 = -1, b2 = -1;
    double c1 = 0, c2 = 0;
    if (have_guess) guess_coefficients(p, c, sc.tau, sc.b * c->dt, b1, c1, b2, c2);
    Vec<1> acc;
    acc.v[0] = 0.0;
    const ColumnSpan cs = column_span(p, k);
    if (!err && cs.live && cs.z0 < cs.z1) {
        const int x = cs.x, y = cs.y, nx = p.nx, sz = p.nx * p.ny;
        const int su = (p.nx + 1) * p.ny, sv = p.nx * (p.ny + 1);     // layer strides of the u and v faces
        const double dx = a.g.dw[X][x], dy = a.g.dw[Y][y];
        // the loads of a layer, issued one layer ahead of its arithmetic
        struct Layer { T mx0, mx1, my0, my1, mz1; double dz, ph, p0, h1, h2; };
        auto fetch = [&](int j, int ju, int jv, int z) {
            Layer v;
            v.mx0 = __ldg(a.m[X] + ju);
            v.mx1 = __ldg(a.m[X] + ju + 1);
            v.my0 = __ldg(a.m[Y] + jv);
            v.my1 = __ldg(a.m[Y] + jv + nx);
            v.mz1 = __ldg(a.m[Z] + j + sz);
            v.dz = __ldg(a.g.dw[Z] + z);
            v.ph = v.p0 = v.h1 = v.h2 = 0.0;
            if (have_guess) {
                if (a.stage == 0) v.ph = __ldg(a.phi_state + j);
                else { v.p0 = __ldg(a.phi0 + j); v.ph = __ldg(a.phi_cur + j); }
                if (b1 >= 0) v.h1 = __ldg(a.hist[b1] + j);
                if (b2 >= 0) v.h2 = __ldg(a.hist[b2] + j);
            }
            return v;
        };
        int i = cs.p + cs.z0 * sz;
        int iu = fidx<X>(p, x, y, cs.z0), iv = fidx<Y>(p, x, y, cs.z0);
        T wlo = __ldg(a.m[Z] + i);                                     // m_z on this cell's lower face
        Layer next = fetch(i, iu, iv, cs.z0);
        for (int z = cs.z0; z < cs.z1; z++, i += sz, iu += su, iv += sv) {
            const Layer l = next;
            if (z + 1 < cs.z1) next = fetch(i + sz, iu + su, iv + sv, z + 1);
            const double dz = l.dz;
            const double rhs = ((double)l.mx1 - (double)l.mx0) * (dy * dz) + ((double)l.my1 - (double)l.my0) * (dx * dz) +
                               ((double)l.mz1 - (double)wlo) * (dx * dy);
            wlo = l.mz1;
            a.rhs[i] = rhs;
            acc.v[0] += rhs * rhs;
            if (have_guess) {
                // base and guess (backend.cu:922-928, 857-873); their residual is the start mode of the
                // residual kernel, which reads the guess of the neighbouring cells
                double base;
                if (a.stage == 0) {
                    base = sc.b * (p.reinit_r * l.ph);
                    a.phi0[i] = p.reinit_r * l.ph;
                } else {
                    base = sc.a0 * l.p0 + sc.b * l.ph;
                }
                a.base[i] = base;
                double g = base;
                if (b1 >= 0) {
                    const double ex = b2 >= 0 ? c1 * l.h1 + c2 * l.h2 : c1 * l.h1;
                    g = ex + base;
                }
                a.guess[i] = g;
            } else {
                a.guess[i] = 0.0;
                a.res[i] = rhs;
            }
        }
    }
    const Vec<1> blk = block_reduce<1, false>(acc);
    if (publish_partials(blk, a.partial, &c->counter[kCntDiv], k)) {
        const Vec<1> tot = final_reduce<1, false>(a.partial, k);
        if (threadIdx.x == 0) {
            c->counter[kCntDiv] = 0;
            c->passes = 0;
            c->phi_passes = 0;
            c->reset_phi = 0;
            c->zero_rhs = 0;
            if (err) { set_loop(c, a.handle, a.use_handle, 0); return; }
            c->rhs_norm2 = tot.v[0];
            c->rhs_norm = sqrt(tot.v[0]);
            if (!isfinite(c->rhs_norm)) { c->error = kRhsNaN; set_loop(c, a.handle, a.use_handle, 0); return; }
            if (c->rhs_norm == 0.0) {                         // backend.cu:821: phi = 0
                c->zero_rhs = 1;
                c->reset_phi = 1;
                c->phi_rel = 0.0;
                c->phi_sum = 0.0;
                c->rel = 0.0;
                set_loop(c, a.handle, a.use_handle, 0);
                return;
            }
            if (!have_guess) {                                // start from phi = 0: the residual is rhs
                c->use_rhs = 1;
                c->phi_sum = 0.0;
                c->rel = 1.0;
                decide_loop(p, c, a.handle, a.use_handle);
            }
        }
    }
}
template <class T>
__global__ void __launch_bounds__(kThreads, kColumnBlocks) projection_start_kernel(StartArgs<T> a) {
    projection_start_body(a, real_blk());
}
template <class T>
__global__ void __launch_bounds__(kThreads, kColumnBlocks) projection_start_batched(const StartArgs<T>* args, const BatchItem* items, const int* live) {
    __shared__ StartArgs<T> a;
    int cav;
    const Blk k = item_blk(items, live, cav);
    if (cav < 0) return;
    load_args(a, args + cav);
    projection_start_body(a, k);
}

// ------------------------------------------------------------------------------------------ residual
// r = rhs - L phi with L the 7-point area-weighted Neumann Laplacian (backend.cu:345-359) after a pass, sum r^2
// and sum phi; the last block counts the pass and decides on the next (backend.cu:835-839).  Column walk.
struct ResidualArgs {
    Params p;
    const double* dw[3];
    const double* dinv_sp[3];
    const double* phi;
    const double* rhs;
    double* res;
    Control* c;
    double* partial;
    cudaGraphConditionalHandle handle;
    int use_handle;
    int start;                 // 1: residual of the warm-start guess at the start of a solve (phi = the guess)
};

// A cavity whose refinement loop has ended (a batch runs passes while any cavity needs one) skips the pass.
// Column walk (ColumnSpan); each cell's arithmetic is that of backend.cu:352-357.
__device__ void residual_body(const ResidualArgs& a, const Blk& k) {
    pdl_launch_dependents();
    pdl_wait();
    Control* c = a.c;
    if (!a.start && !c->cond) return;
    const Params& p = a.p;
    const int err = c->error;
    const bool skip = err || (a.start && c->zero_rhs);
    Vec<2> acc;
    acc.v[0] = 0.0;
    acc.v[1] = 0.0;
    // a pair of cells (x, x + 1) per thread, x even: 16-byte loads and stores, and the pair's inner x-neighbours
    // are its own values
    const ColumnSpan cs = column_span(p, k, 2);
    if (!skip && cs.live && cs.z0 < cs.z1) {
        const int sy = p.nx, sz = p.nx * p.ny, x = cs.x, y = cs.y;
        const bool xl = x > 0, xh = x + 2 < p.nx, yl = y > 0, yh = y + 1 < p.ny;
        const double* f = a.phi;
        const double* dwx = a.dw[X] + x;            // tables: L1 hits, read at use to keep registers for the loads
        const double* ispx = a.dinv_sp[X] + x;
        const double* ispy = a.dinv_sp[Y] + y;
        auto ld2 = [](const double* q) { return __ldg(reinterpret_cast<const double2*>(q)); };
        const double2 zero2 = make_double2(0.0, 0.0);
        // the loads of a layer that go to DRAM or to other blocks' rows, issued one layer ahead of its arithmetic;
        // the same row's outer neighbours and the z tables are L1 hits by then
        struct Layer { double2 above, n, s, rhs; };
        auto fetch = [&](int j, int z) {
            Layer v;
            v.above = z + 1 < p.nz ? ld2(f + j + sz) : zero2;
            v.n = yh ? ld2(f + j + sy) : zero2;
            v.s = yl ? ld2(f + j - sy) : zero2;
            v.rhs = ld2(a.rhs + j);
            return v;
        };
        int i = cs.p + cs.z0 * sz;
        double2 below = cs.z0 > 0 ? ld2(f + i - sz) : zero2;
        double2 cc = ld2(f + i);
        Layer next = fetch(i, cs.z0);
        for (int z = cs.z0; z < cs.z1; z++, i += sz) {
            const Layer l = next;
            if (z + 1 < cs.z1) next = fetch(i + sz, z + 1);
            if (z + 1 + kColumnL2Ahead < cs.z1) {
                const int j = i + (1 + kColumnL2Ahead) * sz;
                prefetch_l2(a.rhs + j);
                if (z + 2 + kColumnL2Ahead < p.nz) prefetch_l2(f + j + sz);
            }
            const double dz = __ldg(a.dw[Z] + z);
            const bool zh = z + 1 < p.nz;
            const double izh = zh ? __ldg(a.dinv_sp[Z] + z + 1) : 0.0, izl = __ldg(a.dinv_sp[Z] + z);
            const double west = xl ? __ldg(f + i - 1) : 0.0, east = xh ? __ldg(f + i + 2) : 0.0;
            const double dx0 = __ldg(dwx), dx1 = __ldg(dwx + 1), dy = __ldg(a.dw[Y] + y);
            const double ixl = __ldg(ispx), ixm = __ldg(ispx + 1), ixh = xh ? __ldg(ispx + 2) : 0.0;
            const double iyl = __ldg(ispy), iyh = __ldg(ispy + 1);
            // cell x (its east neighbour is the pair's other cell)
            double s0 = 0.0;
            s0 += (dy * dz) * (cc.y - cc.x) * ixm;
            if (xl) s0 -= (dy * dz) * (cc.x - west) * ixl;
            if (yh) s0 += (dx0 * dz) * (l.n.x - cc.x) * iyh;
            if (yl) s0 -= (dx0 * dz) * (cc.x - l.s.x) * iyl;
            if (zh) s0 += (dx0 * dy) * (l.above.x - cc.x) * izh;
            if (z > 0) s0 -= (dx0 * dy) * (cc.x - below.x) * izl;
            // cell x + 1 (its west neighbour is the pair's other cell)
            double s1 = 0.0;
            if (xh) s1 += (dy * dz) * (east - cc.y) * ixh;
            s1 -= (dy * dz) * (cc.y - cc.x) * ixm;
            if (yh) s1 += (dx1 * dz) * (l.n.y - cc.y) * iyh;
            if (yl) s1 -= (dx1 * dz) * (cc.y - l.s.y) * iyl;
            if (zh) s1 += (dx1 * dy) * (l.above.y - cc.y) * izh;
            if (z > 0) s1 -= (dx1 * dy) * (cc.y - below.y) * izl;
            const double r0 = l.rhs.x - s0, r1 = l.rhs.y - s1;
            *reinterpret_cast<double2*>(a.res + i) = make_double2(r0, r1);
            acc.v[0] += r0 * r0;
            acc.v[0] += r1 * r1;
            acc.v[1] += cc.x;
            acc.v[1] += cc.y;
            below = cc;
            cc = l.above;
        }
    }
    const Vec<2> blk = block_reduce<2, false>(acc);
    if (publish_partials(blk, a.partial, &c->counter[kCntRes], k)) {
        const Vec<2> tot = final_reduce<2, false>(a.partial, k);
        if (threadIdx.x == 0) {
            c->counter[kCntRes] = 0;
            if (err) { set_loop(c, a.handle, a.use_handle, 0); return; }
            if (a.start) {
                // the guess is kept unless it is no better than zero (backend.cu:825-831); a zero right-hand
                // side was decided with it
                if (c->zero_rhs) return;
                double rel = sqrt(tot.v[0]) / c->rhs_norm;
                c->res_norm2 = tot.v[0];
                c->use_rhs = 0;
                c->phi_sum = tot.v[1];
                if (rel >= 1.0) { rel = 1.0; c->use_rhs = 1; c->reset_phi = 1; c->phi_sum = 0.0; }
                c->rel = rel;
                decide_loop(p, c, a.handle, a.use_handle);
                return;
            }
            c->passes += 1;
            c->phi_passes = c->passes;
            c->pass_count += 1;
            c->use_rhs = 0;
            c->reset_phi = 0;
            c->res_norm2 = tot.v[0];
            c->phi_sum = tot.v[1];
            c->rel = sqrt(tot.v[0]) / c->rhs_norm;
            if (!isfinite(c->rel)) { c->error = kResidualNaN; set_loop(c, a.handle, a.use_handle, 0); return; }
            decide_loop(p, c, a.handle, a.use_handle);
        }
    }
}
__global__ void __launch_bounds__(kThreads, kResidualBlocks) residual_kernel(ResidualArgs a) { residual_body(a, real_blk()); }
__global__ void __launch_bounds__(kThreads, kResidualBlocks) residual_batched(const ResidualArgs* args, const BatchItem* items, const int* live) {
    __shared__ ResidualArgs a;
    int cav;
    const Blk k = item_blk(items, live, cav);
    if (cav < 0) return;
    load_args(a, args + cav);
    residual_body(a, k);
}

// ------------------------------------------------------------------------------------------ FDM transforms
// Arguments of the batched transform C[b] = A[b] (M x K) * B[b] (K x N) of the fast-diagonalisation pressure
// solve (backend.cu:792-813; kernel in fdm.cuh).  The operand that is a residual is chosen on the device (rhs
// when the guess was rejected, else the residual); the epilogue stores, scales by 1/lambda, or accumulates
// into phi.
enum Epilogue : int { kStore = 0, kScaleInvLambda = 1, kAccumulate = 2 };

template <class D> struct GemmArgs {
    int M, N, K, lda, ldb, ldc;
    long long sA, sB, sC;            // batch strides
    const D* A;
    const D* A_alt;                  // used instead of A when the control block says use_rhs
    const D* B;
    D* C;
    const D* inv_lambda;             // kScaleInvLambda
    double* phi;                     // kAccumulate target
    int epilogue;
    const Control* c;
    // loop guard: the first transform of a pass clears the refinement loop's condition, so the loop ends
    // unless the residual after the pass sets it again
    cudaGraphConditionalHandle handle;
    int clear_condition;
};

// ------------------------------------------------------------------------------------------ finish a projection
// u = m - grad(phi) with phi's mean removed (backend.cu:846, 361-371); the potential increment history
// (backend.cu:929-939); in the last stage the CFL rate of the new velocity for the next step's dt
// (backend.cu:465-472) and the clock update (backend.cu:945-954).  Column walk (ColumnSpan): a thread writes
// the lower faces of its cells, and the wall face beyond the last cell along an axis.  The solution is read from one buffer and the
// mean-removed potential written to another, since every thread also reads its neighbours' values.
template <class T> struct FinishArgs {
    Params p;
    Geo<T> g;
    const T* m[3];
    T* u_out[3];
    const double* phi;         // the pressure solution (read only: neighbours read it too)
    double* phi_out;           // the solution with its mean removed
    const double* base;        // step only: for the history increment
    double* hist[4];
    int step_mode;             // 1: stage of a step, 0: plain projection (initialize / kick)
    int last_stage;            // compute CFL + commit clock
    int stage;
    Control* c;
    double* partial;
};

template <class T>
__device__ void finish_body(const FinishArgs<T>& a, const Blk& k) {
    pdl_launch_dependents();
    pdl_wait();
    Control* c = a.c;
    const Params& p = a.p;
    const int err = c->error;
    const int zero_phi = c->reset_phi;       // the solve ended on phi = 0 (zero right-hand side, or no pass)
    Vec<1> acc;
    acc.v[0] = -INFINITY;
    // history buffer for this stage's increment: the first one no entry uses (backend.cu:930-935)
    int hb = -1;
    if (a.step_mode && p.phi_extrapolate) {
        for (int k = 0; k < 4 && hb < 0; k++) {
            bool used = false;
            for (int h = 0; h < c->hist_count; h++) used |= (c->hist_buf[h] == k);
            if (!used) hb = k;
        }
    }
    const double mean = c->phi_sum / p.n_cell;
    auto pv = [&](int j) { return zero_phi ? 0.0 : __ldg(a.phi + j) - mean; };
    const ColumnSpan cs = column_span(p, k);
    if (!err && cs.live && cs.z0 < cs.z1) {
        const int x = cs.x, y = cs.y, nx = p.nx, sy = p.nx, sz = p.nx * p.ny;
        const int su = (p.nx + 1) * p.ny, sv = p.nx * (p.ny + 1);     // layer strides of the u and v faces
        const bool xl = x > 0, xh = x + 1 < p.nx, yl = y > 0, yh = y + 1 < p.ny;
        const double ixl = a.g.dinv_sp[X][x], ixh = a.g.dinv_sp[X][x + 1];
        const double iyl = a.g.dinv_sp[Y][y], iyh = a.g.dinv_sp[Y][y + 1];
        const T wx = tab(a.g, X, kW, x), wy = tab(a.g, Y, kW, y);
        // the loads of a layer that go to DRAM or to other blocks' rows, issued one layer ahead of its arithmetic;
        // the same row's neighbours and the z tables are L1 hits by then (the faces above the cell are needed only
        // for the CFL rate of the last stage)
        const bool cfl = a.last_stage;
        struct Layer { double above, s, n, base; T mx, my, mz, my1; };
        auto fetch = [&](int j, int ju, int jv, int z) {
            Layer v;
            const bool zh = z + 1 < p.nz;
            v.above = zh ? pv(j + sz) : 0.0;
            v.s = yl ? pv(j - sy) : 0.0;
            v.n = cfl && yh ? pv(j + sy) : 0.0;
            v.base = hb >= 0 ? __ldg(a.base + j) : 0.0;
            v.mx = __ldg(a.m[X] + ju);
            v.my = __ldg(a.m[Y] + jv);
            v.mz = zh ? __ldg(a.m[Z] + j + sz) : T(0);
            v.my1 = cfl && yh ? __ldg(a.m[Y] + jv + nx) : T(0);
            return v;
        };
        int i = cs.p + cs.z0 * sz;
        int iu = fidx<X>(p, x, y, cs.z0), iv = fidx<Y>(p, x, y, cs.z0);
        double ph = pv(i);
        T wlo = T(0);                 // the w-face below this cell, as the cell below computed it
        if (cs.z0 > 0) wlo = __ldg(a.m[Z] + i) - (T)((ph - pv(i - sz)) * a.g.dinv_sp[Z][cs.z0]);
        Layer next = fetch(i, iu, iv, cs.z0);
        for (int z = cs.z0; z < cs.z1; z++, i += sz, iu += su, iv += sv) {
            const Layer l = next;
            if (z + 1 < cs.z1) next = fetch(i + sz, iu + su, iv + sv, z + 1);
            if (z + 1 + kColumnL2Ahead < cs.z1) {
                constexpr int d = 1 + kColumnL2Ahead;
                const int j = i + d * sz;
                prefetch_l2(a.m[X] + iu + d * su);
                prefetch_l2(a.m[Y] + iv + d * sv);
                prefetch_l2(a.m[Z] + j + sz);
                if (!zero_phi && z + 2 + kColumnL2Ahead < p.nz) prefetch_l2(a.phi + j + sz);
                if (hb >= 0) prefetch_l2(a.base + j);
            }
            // faces below this cell (wall faces 0), and above it at the last cell of an axis
            const bool zh = z + 1 < p.nz;
            T uf[2], vf[2], wf[2];
            uf[0] = xl ? l.mx - (T)((ph - pv(i - 1)) * ixl) : T(0);
            vf[0] = yl ? l.my - (T)((ph - l.s) * iyl) : T(0);
            wf[0] = wlo;
            wf[1] = zh ? l.mz - (T)((l.above - ph) * __ldg(a.g.dinv_sp[Z] + z + 1)) : T(0);
            a.u_out[X][iu] = uf[0];
            a.u_out[Y][iv] = vf[0];
            a.u_out[Z][i] = wf[0];
            if (!xh) a.u_out[X][iu + 1] = T(0);
            if (!yh) a.u_out[Y][iv + nx] = T(0);
            if (!zh) a.u_out[Z][i + sz] = T(0);
            if (cfl) {
                uf[1] = xh ? __ldg(a.m[X] + iu + 1) - (T)((pv(i + 1) - ph) * ixh) : T(0);
                vf[1] = yh ? l.my1 - (T)((l.n - ph) * iyh) : T(0);
                // CFL rate of the new velocity, as backend.cu:469-471 (divisions kept for identical rounding)
                const T r = fmax(fabs(uf[0]), fabs(uf[1])) / wx + fmax(fabs(vf[0]), fabs(vf[1])) / wy +
                            fmax(fabs(wf[0]), fabs(wf[1])) / tab(a.g, Z, kW, z);
                acc.v[0] = combine<1, true>(acc.v[0], (double)r);
            }
            a.phi_out[i] = ph;
            if (hb >= 0) a.hist[hb][i] = 1.0 * ph + -1.0 * l.base;
            wlo = wf[1];
            ph = l.above;
        }
    }
    // gridwide: CFL max (NaN wins) and the scalar bookkeeping in the last block
    const Vec<1> blk = block_reduce<1, true>(acc);
    if (publish_partials(blk, a.partial, &c->counter[kCntFinish], k)) {
        const Vec<1> tot = final_reduce<1, true>(a.partial, k);
        if (threadIdx.x == 0) {
            c->counter[kCntFinish] = 0;
            if (!err) {
                if (hb >= 0) {                          // push this increment, keep the last three
                    const StageConst sc = stage_const(a.stage, c);
                    int n = c->hist_count;
                    if (n == 3) {
                        for (int k = 0; k < 2; k++) {
                            c->hist_t[k] = c->hist_t[k + 1];
                            c->hist_scale[k] = c->hist_scale[k + 1];
                            c->hist_buf[k] = c->hist_buf[k + 1];
                        }
                        n = 2;
                    }
                    c->hist_t[n] = sc.tau;
                    c->hist_scale[n] = sc.b * c->dt;
                    c->hist_buf[n] = hb;
                    c->hist_count = n + 1;
                }
                if (a.last_stage) c->cfl_rate = tot.v[0];
                if (a.step_mode && a.last_stage) {
                    c->t += c->dt;
                    c->steps += 1;
                    c->last_dt = c->dt;
                    c->last_cfl = c->dt * c->use0;
                }
            }
        }
    }
}
template <class T>
__global__ void __launch_bounds__(kThreads, kColumnBlocks) finish_kernel(FinishArgs<T> a) { finish_body(a, real_blk()); }
template <class T>
__global__ void __launch_bounds__(kThreads, kColumnBlocks) finish_batched(const FinishArgs<T>* args, const BatchItem* items, const int* live) {
    __shared__ FinishArgs<T> a;
    int cav;
    const Blk k = item_blk(items, live, cav);
    if (cav < 0) return;
    load_args(a, args + cav);
    finish_body(a, k);
}

// ------------------------------------------------------------------------------------------ small kernels
// CFL rate of a velocity field (backend.cu:465-472), max over cells into c->cfl_rate.
template <class T> struct CflArgs {
    Params p;
    Geo<T> g;
    const T* u[3];
    Control* c;
    double* partial;
};
template <class T>
__global__ void __launch_bounds__(kThreads) cfl_kernel(CflArgs<T> a) {
    const Params& p = a.p;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    Vec<1> acc;
    acc.v[0] = -INFINITY;
    if (i < p.n_cell) {
        const int x = i % p.nx, y = (i / p.nx) % p.ny, z = i / (p.nx * p.ny);
        const int iu = fidx<X>(p, x, y, z), iv = fidx<Y>(p, x, y, z), iw = fidx<Z>(p, x, y, z);
        const T r = fmax(fabs(a.u[X][iu]), fabs(a.u[X][iu + 1])) / tab(a.g, X, kW, x) +
                    fmax(fabs(a.u[Y][iv]), fabs(a.u[Y][iv + p.nx])) / tab(a.g, Y, kW, y) +
                    fmax(fabs(a.u[Z][iw]), fabs(a.u[Z][iw + p.nx * p.ny])) / tab(a.g, Z, kW, z);
        acc.v[0] = (double)r;
    }
    const Vec<1> blk = block_reduce<1, true>(acc);
    if (publish_partials(blk, a.partial, &a.c->counter[kCntCfl])) {
        const Vec<1> tot = final_reduce<1, true>(a.partial);
        if (threadIdx.x == 0) {
            a.c->counter[kCntCfl] = 0;
            a.c->cfl_rate = tot.v[0];
        }
    }
}

// zero the wall faces of one component (backend.cu:373-380)
template <class T>
__global__ void zero_walls_kernel(Params p, int comp, T* f) {
    const int ex = p.nx + (comp == 0), ey = p.ny + (comp == 1), ez = p.nz + (comp == 2);
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= ex * ey * ez) return;
    const int x = i % ex, y = (i / ex) % ey, z = i / (ex * ey);
    if ((comp == 0 && (x == 0 || x == p.nx)) || (comp == 1 && (y == 0 || y == p.ny)) ||
        (comp == 2 && (z == 0 || z == p.nz)))
        f[i] = T(0);
}

// type conversions for host copies: the ABI carries velocity and impulse as float32
template <class S, class D>
__global__ void convert_kernel(const S* in, D* out, long long n) {
    const long long i = blockIdx.x * (long long)kThreads + threadIdx.x;
    if (i < n) out[i] = (D)in[i];
}
// initial impulse from double noise, rounded to float as the reference (backend.cu:1080-1082)
template <class T>
__global__ void noise_to_field_kernel(const double* in, T* out, long long n) {
    const long long i = blockIdx.x * (long long)kThreads + threadIdx.x;
    if (i < n) out[i] = in ? (T)(float)in[i] : T(0);
}

}  // namespace cavity
