// fdm.cuh - one pass of the fast-diagonalisation (FDM) pressure solve (backend.cu:801-814), as launches of the
// batched transform kernel of kernels.cuh:  t = S_z^T S_y^T S_x^T r (along x, y, z), t *= inv_lambda,
// phi += S_x S_y S_z t.  Fields are [z][y][x]; S_a is the row-major n_a x n_a eigenbasis of axis a
// (eigenvector j in column j) and ST_a its transpose.
#pragma once
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "kernels.cuh"

namespace cavity {

struct FdmOperands {
    int nx, ny, nz;
    const double* s[3];
    const double* st[3];
    const double* inv_lambda;
};

// C[b] = A[b] (M x K) * B[b] (K x N), row-major, on the FP64 tensor cores: each warp owns a 32 x 32 tile of C as
// fragments of mma.sync.m8n8k4.f64 (the FP64 MMA of sm_80 and later; Blackwell's tcgen05 has no FP64
// kind).  Operand panels are staged in shared memory with row pitches of 8 banks mod 32, so the 8 x 4 A
// fragments and 4 x 8 B fragments load without bank conflicts.  Same operand selection, skip rule,
// loop guard and epilogues as described at GemmArgs (kernels.cuh).
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* src, int src_bytes) {
    const unsigned int dst = (unsigned int)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async16z(void* smem_dst, const void* src, int src_bytes) {
    const unsigned int dst = (unsigned int)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// CTA tile BM x BN from WARPS_M x WARPS_N warps; K consumed in panels of KC with every load of a panel in
// flight at once (cp.async, zero-filled outside the matrices; two doubles per copy where rows allow).
template <int BM, int BN, int WARPS_M, int WARPS_N, int KC>
__device__ void dgemm_mma_body(const GemmArgs<double>& g, const Blk& blk, bool first) {
    pdl_launch_dependents();
    pdl_wait();
    constexpr int NT = WARPS_M * WARPS_N * 32;
    constexpr int WTM = BM / WARPS_M, WTN = BN / WARPS_N;     // warp tile
    constexpr int FM = WTM / 8, FN = WTN / 8;                   // fragments per warp tile
    constexpr int LDA = KC + 4, LDB = BN + 4;                   // row pitches of 8 banks mod 32
    __shared__ __align__(16) double As[BM * LDA];
    __shared__ __align__(16) double Bs[KC * LDB];
    if (g.clear_condition && threadIdx.x == 0 && first) cudaGraphSetConditional(g.handle, 0u);
    const Control* c = g.c;
    if (c->error || !c->cond) return;                     // failed, or this cavity's refinement has ended
    const double r2 = c->use_rhs ? c->rhs_norm2 : c->res_norm2;       // a zero residual: no pass (backend.cu:803-804)
    if (!(r2 > 0)) return;
    const int b = blk.z;
    const double* A = (g.A_alt && c->use_rhs ? g.A_alt : g.A) + b * g.sA;
    const double* B = g.B + b * g.sB;
    const int m0 = blk.y * BM, n0 = blk.x * BN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp / WARPS_N, wn = warp % WARPS_N;
    const int fr = lane >> 2, fc = lane & 3;          // fragment row / column of this lane
    // two doubles per copy when rows are even and the arrays 16-byte aligned
    const bool a2 = g.K % 2 == 0 && g.lda % 2 == 0 && ((unsigned long long)A & 15) == 0;
    const bool b2 = g.N % 2 == 0 && g.ldb % 2 == 0 && ((unsigned long long)B & 15) == 0;
    double acc[FM][FN][2];
#pragma unroll
    for (int i = 0; i < FM; i++)
#pragma unroll
        for (int j = 0; j < FN; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
    for (int k0 = 0; k0 < g.K; k0 += KC) {
        if (a2) {
            for (int e = threadIdx.x; e < BM * KC / 2; e += NT) {
                const int r = e / (KC / 2), k = 2 * (e % (KC / 2)), gm = m0 + r, gk = k0 + k;
                const bool ok = gm < g.M && gk < g.K;
                cp_async16z(&As[r * LDA + k], ok ? A + (long long)gm * g.lda + gk : A, ok ? 16 : 0);
            }
        } else {
            for (int e = threadIdx.x; e < BM * KC; e += NT) {
                const int r = e / KC, k = e % KC, gm = m0 + r, gk = k0 + k;
                const bool ok = gm < g.M && gk < g.K;
                cp_async8(&As[r * LDA + k], ok ? A + (long long)gm * g.lda + gk : A, ok ? 8 : 0);
            }
        }
        if (b2) {
            for (int e = threadIdx.x; e < KC * BN / 2; e += NT) {
                const int k = e / (BN / 2), col = 2 * (e % (BN / 2)), gk = k0 + k, gn = n0 + col;
                const bool ok = gk < g.K && gn < g.N;
                cp_async16z(&Bs[k * LDB + col], ok ? B + (long long)gk * g.ldb + gn : B, ok ? 16 : 0);
            }
        } else {
            for (int e = threadIdx.x; e < KC * BN; e += NT) {
                const int k = e / BN, col = e % BN, gk = k0 + k, gn = n0 + col;
                const bool ok = gk < g.K && gn < g.N;
                cp_async8(&Bs[k * LDB + col], ok ? B + (long long)gk * g.ldb + gn : B, ok ? 8 : 0);
            }
        }
        cp_async_wait_all();
        __syncthreads();
        const int kend = min(KC, g.K - k0);
        for (int kk = 0; kk < kend; kk += 4) {
            double af[FM], bf[FN];
#pragma unroll
            for (int i = 0; i < FM; i++) af[i] = As[(wm * WTM + i * 8 + fr) * LDA + kk + fc];
#pragma unroll
            for (int j = 0; j < FN; j++) bf[j] = Bs[(kk + fc) * LDB + wn * WTN + j * 8 + fr];
#pragma unroll
            for (int i = 0; i < FM; i++)
#pragma unroll
                for (int j = 0; j < FN; j++) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
        __syncthreads();
    }
    const int reset = c->reset_phi;
#pragma unroll
    for (int i = 0; i < FM; i++) {
        const int gm = m0 + wm * WTM + i * 8 + fr;
        if (gm >= g.M) continue;
#pragma unroll
        for (int j = 0; j < FN; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int gn = n0 + wn * WTN + j * 8 + 2 * fc + h;
                if (gn >= g.N) continue;
                const long long idx = b * g.sC + (long long)gm * g.ldc + gn;
                const double v = acc[i][j][h];
                if (g.epilogue == kStore) g.C[idx] = v;
                else if (g.epilogue == kScaleInvLambda) g.C[idx] = v * g.inv_lambda[idx];
                else g.phi[idx] = (reset ? 0.0 : g.phi[idx]) + v;
            }
    }
}

template <int BM, int BN, int WARPS_M, int WARPS_N, int KC>
__global__ void __launch_bounds__(WARPS_M * WARPS_N * 32) dgemm_mma_kernel(GemmArgs<double> g) {
    dgemm_mma_body<BM, BN, WARPS_M, WARPS_N, KC>(g, real_blk(), first_block());
}
// a batch of cavities: grid x runs over the work list (BatchItem)
template <int BM, int BN, int WARPS_M, int WARPS_N, int KC>
__global__ void __launch_bounds__(WARPS_M * WARPS_N * 32) dgemm_mma_batched(const GemmArgs<double>* args,
                                                                            const BatchItem* items, const int* live) {
    __shared__ GemmArgs<double> g;
    int cav;
    const Blk k = item_blk(items, live, cav);
    if (cav < 0) {
        dead_slot_clear(args, items);
        return;
    }
    load_args(g, args + cav);
    dgemm_mma_body<BM, BN, WARPS_M, WARPS_N, KC>(g, k, first_block());
}

// ---------------------------------------------------------------------------------------------- one-launch pass
// The six transforms of a pass as phases of one cooperative launch, separated by grid barriers: a small grid's
// transforms are each a few microseconds of latency-bound work, and one launch replaces six.  Each phase runs
// the same 32 x 32 tile body over that transform's own tile grid (grid-stride), so the arithmetic is exactly
// that of six launches.  Every barrier wait is bounded: on time-out the block sets kBarrierWait and returns.
struct FdmPassArgs {
    GemmArgs<double> g[6];
    unsigned int gx[6], gy[6], gz[6];      // each transform's tile grid
    Control* c;
};
constexpr long long kBarrierSpins = 1LL << 22;

// all blocks of the launch (co-resident: cooperative launch) meet here; false if the wait timed out
__device__ __forceinline__ bool grid_barrier(Control* c, unsigned int nblocks) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = &c->counter[kCntBarGen];
        const unsigned int g0 = *gen;
        ok = 1;
        __threadfence();
        if (atomicAdd(&c->counter[kCntBar], 1u) == nblocks - 1) {
            atomicExch(&c->counter[kCntBar], 0u);
            __threadfence();
            atomicAdd(&c->counter[kCntBarGen], 1u);
        } else {
            long long spins = 0;
            while (*gen == g0) {
                if (++spins > kBarrierSpins) {
                    atomicExch(&c->error, (int)kBarrierWait);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok;
}

__global__ void __launch_bounds__(256) fdm_pass_fused_kernel(FdmPassArgs a) {
    const unsigned int nb = gridDim.x;
    for (int p = 0; p < 6; p++) {
        const unsigned int tiles = a.gx[p] * a.gy[p] * a.gz[p];
        for (unsigned int vb = blockIdx.x; vb < tiles; vb += nb) {
            const Blk k{vb % a.gx[p], (vb / a.gx[p]) % a.gy[p], vb / (a.gx[p] * a.gy[p]), a.gx[p], a.gy[p], a.gz[p]};
            dgemm_mma_body<32, 32, 2, 4, 64>(a.g[p], k, p == 0 && vb == 0);
        }
        if (p < 5 && !grid_barrier(a.c, nb)) return;
    }
}

// one batched transform launch; the tile shape keeps at least ~two CTAs per SM on small grids.  The small tile runs
// 8 warps (2 x 4, each 16 x 8) rather than 4: more warps hide the FP64 MMA chains of a latency-bound 64^3 pass.
inline GemmArgs<double> transform_args(int M, int N, int K, const double* A, const double* A_alt, int lda, long long sA,
                                       const double* B, int ldb, long long sB, double* C, int ldc, long long sC, int epi,
                                       const double* inv_lambda, double* phi, const Control* c,
                                       cudaGraphConditionalHandle h, bool clear) {
    GemmArgs<double> g;
    g.handle = h;
    g.clear_condition = clear;
    g.M = M; g.N = N; g.K = K; g.lda = lda; g.ldb = ldb; g.ldc = ldc;
    g.sA = sA; g.sB = sB; g.sC = sC;
    g.A = A; g.A_alt = A_alt; g.B = B; g.C = C;
    g.inv_lambda = inv_lambda;
    g.phi = phi;
    g.epilogue = epi;
    g.c = c;
    return g;
}
inline void launch_transform(cudaStream_t st, int M, int N, int K, const double* A, const double* A_alt, int lda,
                             long long sA, const double* B, int ldb, long long sB, double* C, int ldc, long long sC,
                             int batch, int epi, const double* inv_lambda, double* phi, const Control* c,
                             cudaGraphConditionalHandle h, bool clear) {
    const GemmArgs<double> g = transform_args(M, N, K, A, A_alt, lda, sA, B, ldb, sB, C, ldc, sC, epi, inv_lambda, phi,
                                              c, h, clear);
    const long long tiles64 = (long long)((N + 63) / 64) * ((M + 63) / 64) * batch * g_launch_batch;
    static const int forced = [] {                 // CAVITY_DGEMM_TILE=32 or 64 forces the tile everywhere
        const char* e = std::getenv("CAVITY_DGEMM_TILE");
        return e ? std::atoi(e) : 0;
    }();
    const int tile = forced ? forced : g_dgemm_tile;
    if (tile ? tile == 64 : tiles64 >= 296) {
        dim3 grid((N + 63) / 64, (M + 63) / 64, batch);
        if (!record_launch(kLkDgemm64, 0, grid, 0, g)) launch_pdl(dgemm_mma_kernel<64, 64, 2, 2, 32>, grid, dim3(128), 0, st, g);
    } else {
        dim3 grid((N + 31) / 32, (M + 31) / 32, batch);
        if (!record_launch(kLkDgemm32, 0, grid, 0, g)) launch_pdl(dgemm_mma_kernel<32, 32, 2, 4, 64>, grid, dim3(256), 0, st, g);
    }
}

// phi += FDM(r); r_alt replaces r when the control block says use_rhs.  t1, t2: nx*ny*nz doubles of scratch.
// `clear` makes the first launch clear the condition of the enclosing graph while-node `h`.
// cooperative blocks of the one-launch pass this device holds at once (0: not available)
inline int fused_pass_capacity() {
    static const int cap = [] {
        int dev = 0, sms = 0, per = 0, coop = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && coop &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fdm_pass_fused_kernel, 256, 0) == cudaSuccess)
            return sms * per;
        return 0;
    }();
    return cap;
}
// One-launch pass: the six transforms of launch_fdm_pass with the 32 x 32 tile, as one cooperative launch.
inline void launch_fdm_pass_fused(cudaStream_t st, const FdmOperands& op, const double* r, const double* r_alt,
                                  double* phi, double* t1, double* t2, Control* c, cudaGraphConditionalHandle h,
                                  bool clear) {
    const int nx = op.nx, ny = op.ny, nz = op.nz, plane = nx * ny;
    const long long pl = plane;
    const double* il = op.inv_lambda;
    FdmPassArgs a;
    a.c = c;
    struct Shape { int M, N, batch; };
    const Shape sh[6] = {{ny * nz, nx, 1}, {ny, nx, nz}, {nz, plane, 1}, {nz, plane, 1}, {ny, nx, nz}, {ny * nz, nx, 1}};
    a.g[0] = transform_args(ny * nz, nx, nx, r, r_alt, nx, 0, op.s[0], nx, 0, t1, nx, 0, kStore, il, nullptr, c, h, clear);
    a.g[1] = transform_args(ny, nx, ny, op.st[1], nullptr, ny, 0, t1, nx, pl, t2, nx, pl, kStore, il, nullptr, c, 0, false);
    a.g[2] = transform_args(nz, plane, nz, op.st[2], nullptr, nz, 0, t2, plane, 0, t1, plane, 0, kScaleInvLambda, il,
                            nullptr, c, 0, false);
    a.g[3] = transform_args(nz, plane, nz, op.s[2], nullptr, nz, 0, t1, plane, 0, t2, plane, 0, kStore, il, nullptr, c, 0,
                            false);
    a.g[4] = transform_args(ny, nx, ny, op.s[1], nullptr, ny, 0, t2, nx, pl, t1, nx, pl, kStore, il, nullptr, c, 0, false);
    a.g[5] = transform_args(ny * nz, nx, nx, t1, nullptr, nx, 0, op.st[0], nx, 0, nullptr, nx, 0, kAccumulate, il, phi, c,
                            0, false);
    unsigned int most = 0;
    for (int p = 0; p < 6; p++) {
        a.gx[p] = (unsigned int)((sh[p].N + 31) / 32);
        a.gy[p] = (unsigned int)((sh[p].M + 31) / 32);
        a.gz[p] = (unsigned int)sh[p].batch;
        most = std::max(most, a.gx[p] * a.gy[p] * a.gz[p]);
    }
    const unsigned int blocks = std::min(most, (unsigned int)fused_pass_capacity());
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, fdm_pass_fused_kernel, a);
}
// the one-launch pass applies to a single cavity (not recording a batch) when CAVITY_FDM_FUSED=1 or the
// cavity's own choice (`want`, the autotuner's; -1 none) says so.  It is not the default: inside the step graph
// it measured slower than six launches (C2 step 0.383 against 0.368 ms), the graph's programmatic launches
// already hiding most of the gaps that the grid barriers replace.
inline bool use_fused_pass(const FdmOperands& op, int want) {
    (void)op;
    if (g_launch_record || g_dgemm_tile == 64 || fused_pass_capacity() == 0) return false;
    if (const char* e = std::getenv("CAVITY_FDM_FUSED")) return e[0] == '1';
    return want == 1;
}

inline void launch_fdm_pass(cudaStream_t st, const FdmOperands& op, const double* r, const double* r_alt, double* phi,
                            double* t1, double* t2, Control* c, cudaGraphConditionalHandle h, bool clear, int fused = -1) {
    if (use_fused_pass(op, fused)) {
        launch_fdm_pass_fused(st, op, r, r_alt, phi, t1, t2, c, h, clear);
        return;
    }
    const int nx = op.nx, ny = op.ny, nz = op.nz, plane = nx * ny;
    const long long pl = plane;
    const double* il = op.inv_lambda;
    launch_transform(st, ny * nz, nx, nx, r, r_alt, nx, 0, op.s[0], nx, 0, t1, nx, 0, 1, kStore, il,
                                      nullptr, c, h, clear);
    launch_transform(st, ny, nx, ny, op.st[1], nullptr, ny, 0, t1, nx, pl, t2, nx, pl, nz, kStore, il,
                                      nullptr, c, 0, false);
    launch_transform(st, nz, plane, nz, op.st[2], nullptr, nz, 0, t2, plane, 0, t1, plane, 0, 1,
                                      kScaleInvLambda, il, nullptr, c, 0, false);
    launch_transform(st, nz, plane, nz, op.s[2], nullptr, nz, 0, t1, plane, 0, t2, plane, 0, 1, kStore,
                                      il, nullptr, c, 0, false);
    launch_transform(st, ny, nx, ny, op.s[1], nullptr, ny, 0, t2, nx, pl, t1, nx, pl, nz, kStore, il,
                                      nullptr, c, 0, false);
    launch_transform(st, ny * nz, nx, nx, t1, nullptr, nx, 0, op.st[0], nx, 0, nullptr, nx, 0, 1,
                                      kAccumulate, il, phi, c, 0, false);
}

// Control block for a pass outside a solver: no error, a non-zero residual, accumulate into phi.
inline Control standalone_fdm_control() {
    Control c;
    memset(&c, 0, sizeof c);
    c.res_norm2 = 1.0;
    c.rhs_norm2 = 1.0;
    c.cond = 1;
    return c;
}

}  // namespace cavity
