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

// ---------------------------------------------------------------------------------------------- paired pass
// The six transforms of a pass as three launches when no axis has more than 64 cells.  Each launch chains two
// transforms through shared memory, so the intermediate between them never goes back to memory:
//   pair_xy_kernel:  t = ST_y (r S_x)                      a CTA per z-plane and block of W x-columns
//   pair_z_kernel:   t = S_z (inv_lambda .* (ST_z t))      a CTA per block of W plane columns, in place
//   pair_yx_kernel:  phi += (S_y t) ST_x                   a CTA per z-plane and block of W y-rows
// Every dot product runs over k in the same order, four at a time from a zero accumulator, as in
// dgemm_mma_body, and the values between the transforms are the same doubles, so each transform's result is
// bit for bit the six-launch pass's.  Shared-memory operands are zero outside the matrices up to the next
// multiple of 8 (rows) or 4 (k), as the six-launch pass's staged panels are.
constexpr int kPairMax = 64;                 // the largest axis a paired pass takes
constexpr int kPairPitch = kPairMax + 4;     // row pitch of a 64-wide operand: 8 banks mod 32
constexpr int kPairThreads = 256;

struct FdmPairArgs {
    int nx, ny, nz, clear_condition;
    int per;                        // tiles per CTA (pair_per); the CTA's first tile is its block index times per
    const double* s[3];
    const double* st[3];
    const double* inv_lambda;
    const double* r;
    const double* r_alt;            // used instead of r when the control block says use_rhs
    double* t;                      // nx*ny*nz doubles of scratch
    double* phi;
    const Control* c;
    cudaGraphConditionalHandle handle;
};

__device__ __forceinline__ int round_up(int v, int m) { return (v + m - 1) / m * m; }

// dst[i * p + k] = src[i * ld + k] for i < rows, k < cols, and 0 elsewhere in the R x C extent (C even, at most
// 2 LPR), as cp.async copies of two doubles where alignment allows, else of one.  LPR threads share a row, two
// columns each, so the loop needs no index division.
template <int LPR>
__device__ __forceinline__ void pair_stage(double* dst, int p, const double* src, long long ld, int rows, int cols,
                                           int R, int C) {
    constexpr int RPS = kPairThreads / LPR;         // rows in flight per sweep of the block
    const int k = 2 * (threadIdx.x % LPR);
    if (k >= C) return;
    const int n = min(2, max(0, cols - k));         // doubles of a row this thread copies (0: zero fill)
    if (ld % 2 == 0 && ((unsigned long long)src & 15) == 0) {
        for (int i = threadIdx.x / LPR; i < R; i += RPS) {
            const int m = i < rows ? n : 0;
            cp_async16z(&dst[i * p + k], m ? src + i * ld + k : src, 8 * m);
        }
    } else {
        for (int i = threadIdx.x / LPR; i < R; i += RPS) {
            const bool ok = i < rows;
            cp_async8(&dst[i * p + k], ok && n > 0 ? src + i * ld + k : src, ok && n > 0 ? 8 : 0);
            cp_async8(&dst[i * p + k + 1], ok && n > 1 ? src + i * ld + k + 1 : src, ok && n > 1 ? 8 : 0);
        }
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// acc += A[m0 .., 0 .. k4) B[0 .. k4, n0 ..) for one warp's FM x FN fragments of 8 x 8 (k4 a multiple of 4)
template <int FM, int FN>
__device__ __forceinline__ void pair_warp_mma(double (&acc)[FM][FN][2], const double* As, int lda, const double* Bs,
                                              int ldb, int k4, int m0, int n0) {
    const int lane = threadIdx.x & 31, fr = lane >> 2, fc = lane & 3;
#pragma unroll
    for (int i = 0; i < FM; i++)
#pragma unroll
        for (int j = 0; j < FN; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
    for (int kk = 0; kk < k4; kk += 4) {
        double af[FM], bf[FN];
#pragma unroll
        for (int i = 0; i < FM; i++) af[i] = As[(m0 + i * 8 + fr) * lda + kk + fc];
#pragma unroll
        for (int j = 0; j < FN; j++) bf[j] = Bs[(kk + fc) * ldb + n0 + j * 8 + fr];
#pragma unroll
        for (int i = 0; i < FM; i++)
#pragma unroll
            for (int j = 0; j < FN; j++) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
}

// The pass's entry checks (as dgemm_mma_body's): programmatic launch, the loop guard, error and residual.
// False when the block has nothing to do.
// Each kernel issues the copies that do not depend on the control block before reading it, so that their
// latencies overlap; a block with nothing to do waits for its copies to land before it exits.
__device__ __forceinline__ void pair_begin(const FdmPairArgs& a, bool first, bool clear) {
    pdl_launch_dependents();
    pdl_wait();
    if (clear && a.clear_condition && threadIdx.x == 0 && first) cudaGraphSetConditional(a.handle, 0u);
}
__device__ __forceinline__ bool pair_live(const FdmPairArgs& a) {
    const Control* c = a.c;
    if (c->error || !c->cond) return false;
    const double r2 = c->use_rhs ? c->rhs_norm2 : c->res_norm2;
    return r2 > 0;
}

template <int W> struct PairSmem {
    // two square operands of pitch kPairPitch and two 64 x W panels of pitch W + 4
    static constexpr int kPanel = W + 4;
    static constexpr size_t bytes = sizeof(double) * (2 * kPairMax * kPairPitch + 2 * kPairMax * kPanel);
};

// A CTA of a paired launch takes `a.per` consecutive tiles that share their bases (the z-planes of one column or
// row block, or consecutive plane-column blocks): the bases are staged once, and each next tile's field is copied
// under the current tile's second transform, into the buffer its first transform has finished reading.  A single
// cavity's launch has one tile per CTA; a large batch's launch several (pair_per).

// t[z] = ST_y (r[z] S_x) on columns [x0, x0 + W) of planes z: transforms 1 and 2 of the pass
template <int W>
__device__ void pair_xy_body(const FdmPairArgs& a, const Blk& blk, bool first) {
    pair_begin(a, first, true);
    constexpr int PW = PairSmem<W>::kPanel, FN = W / 8;
    extern __shared__ __align__(16) double pair_smem[];
    double* A1 = pair_smem;                         // r[z]: ny x nx
    double* A2 = A1 + kPairMax * kPairPitch;        // ST_y: ny x ny
    double* B1 = A2 + kPairMax * kPairPitch;        // S_x[:, x0 .. x0 + W)
    double* C1 = B1 + kPairMax * PW;                // r[z] S_x on those columns
    const int nx = a.nx, ny = a.ny, x0 = blk.x * W;
    const int z0 = blk.y * a.per, z1 = min(a.nz, z0 + a.per);
    const int my = round_up(ny, 8), kx = round_up(nx, 4), ky = round_up(ny, 4);
    pair_stage<W / 2>(B1, PW, a.s[X] + x0, nx, nx, min(W, nx - x0), kx, W);
    pair_stage<32>(A2, kPairPitch, a.st[Y], ny, ny, ny, my, ky);
    cp_async_commit();
    if (!pair_live(a)) {
        cp_async_wait<0>();
        return;
    }
    const double* r = a.r_alt && a.c->use_rhs ? a.r_alt : a.r;
    pair_stage<32>(A1, kPairPitch, r + (long long)z0 * nx * ny, nx, ny, nx, my, kx);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, fr = lane >> 2, fc = lane & 3;
    const int m0 = warp * 8;                        // the warp's 8 rows (y) x W columns
    for (int z = z0; z < z1; z++) {
        double acc[1][FN][2];
        if (m0 < my) {
            pair_warp_mma<1, FN>(acc, A1, kPairPitch, B1, PW, kx, m0, 0);
#pragma unroll
            for (int j = 0; j < FN; j++) {
                C1[(m0 + fr) * PW + j * 8 + 2 * fc] = acc[0][j][0];
                C1[(m0 + fr) * PW + j * 8 + 2 * fc + 1] = acc[0][j][1];
            }
        }
        __syncthreads();
        if (z + 1 < z1) {
            pair_stage<32>(A1, kPairPitch, r + (long long)(z + 1) * nx * ny, nx, ny, nx, my, kx);
            cp_async_commit();
        }
        const int y = m0 + fr;
        if (m0 < my) {
            pair_warp_mma<1, FN>(acc, A2, kPairPitch, C1, PW, ky, m0, 0);
            if (y < ny) {
                double* t = a.t + ((long long)z * ny + y) * nx;
#pragma unroll
                for (int j = 0; j < FN; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int x = x0 + j * 8 + 2 * fc + h;
                        if (x < nx) t[x] = acc[0][j][h];
                    }
            }
        }
        cp_async_wait<0>();
        __syncthreads();
    }
}

// t[:, c] = S_z (inv_lambda .* (ST_z t[:, c])) on plane columns c of blocks of W, in place: transforms 3 and 4
template <int W>
__device__ void pair_z_body(const FdmPairArgs& a, const Blk& blk, bool first) {
    pair_begin(a, first, false);
    constexpr int PW = PairSmem<W>::kPanel, FN = W / 8;
    extern __shared__ __align__(16) double pair_smem[];
    double* A1 = pair_smem;                         // ST_z
    double* A2 = A1 + kPairMax * kPairPitch;        // S_z
    double* B1 = A2 + kPairMax * kPairPitch;        // t[:, c0 .. c0 + W)
    double* C1 = B1 + kPairMax * PW;
    const int nz = a.nz, plane = a.nx * a.ny;
    const int nb = (plane + W - 1) / W, b0 = blk.x * a.per, b1 = min(nb, b0 + a.per);
    const int mz = round_up(nz, 8), kz = round_up(nz, 4);
    pair_stage<32>(A1, kPairPitch, a.st[Z], nz, nz, nz, mz, kz);
    pair_stage<W / 2>(B1, PW, a.t + b0 * W, plane, nz, min(W, plane - b0 * W), kz, W);
    cp_async_commit();
    pair_stage<32>(A2, kPairPitch, a.s[Z], nz, nz, nz, mz, kz);
    cp_async_commit();
    if (!pair_live(a)) {
        cp_async_wait<0>();
        return;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, fr = lane >> 2, fc = lane & 3;
    const int m0 = warp * 8;
    for (int b = b0; b < b1; b++) {
        const int c0 = b * W;
        double acc[1][FN][2], il[FN][2];
        if (m0 < mz) {
            const int z = m0 + fr;
#pragma unroll
            for (int j = 0; j < FN; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int c = c0 + j * 8 + 2 * fc + h;
                    il[j][h] = z < nz && c < plane ? __ldg(a.inv_lambda + (long long)z * plane + c) : 0.0;
                }
        }
        if (b == b0) cp_async_wait<1>();             // ST_z and the first block (S_z may still be in flight)
        __syncthreads();
        if (m0 < mz) {
            pair_warp_mma<1, FN>(acc, A1, kPairPitch, B1, PW, kz, m0, 0);
#pragma unroll
            for (int j = 0; j < FN; j++)
#pragma unroll
                for (int h = 0; h < 2; h++) C1[(m0 + fr) * PW + j * 8 + 2 * fc + h] = acc[0][j][h] * il[j][h];
        }
        cp_async_wait<0>();
        __syncthreads();
        if (b + 1 < b1) {
            pair_stage<W / 2>(B1, PW, a.t + c0 + W, plane, nz, min(W, plane - c0 - W), kz, W);
            cp_async_commit();
        }
        const int z = m0 + fr;
        if (m0 < mz) {
            pair_warp_mma<1, FN>(acc, A2, kPairPitch, C1, PW, kz, m0, 0);
            if (z < nz) {
                double* t = a.t + (long long)z * plane;
#pragma unroll
                for (int j = 0; j < FN; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int c = c0 + j * 8 + 2 * fc + h;
                        if (c < plane) t[c] = acc[0][j][h];
                    }
            }
        }
        cp_async_wait<0>();
        __syncthreads();
    }
}

// phi[z] += (S_y t[z]) ST_x on rows [y0, y0 + W) of planes z: transforms 5 and 6
template <int W>
__device__ void pair_yx_body(const FdmPairArgs& a, const Blk& blk, bool first) {
    pair_begin(a, first, false);
    constexpr int WN = 8 / (W / 8), FN = kPairMax / 8 / WN;   // warps along x, fragments per warp along x
    extern __shared__ __align__(16) double pair_smem[];
    double* B1 = pair_smem;                         // t[z]: ny x nx
    double* B2 = B1 + kPairMax * kPairPitch;        // ST_x: nx x nx
    double* A1 = B2 + kPairMax * kPairPitch;        // S_y[y0 .. y0 + W, :]
    double* C1 = A1 + W * kPairPitch;               // S_y t[z] on those rows
    const int nx = a.nx, ny = a.ny, y0 = blk.x * W;
    const int z0 = blk.y * a.per, z1 = min(a.nz, z0 + a.per);
    const int kx = round_up(nx, 4), ky = round_up(ny, 4), mx = round_up(nx, 8);
    const int cx = min(kPairMax, round_up(mx, 8 * FN));      // columns the active warps read: staged, zero past nx
    pair_stage<32>(A1, kPairPitch, a.s[Y] + (long long)y0 * ny, ny, min(W, ny - y0), ny, W, ky);
    pair_stage<32>(B1, kPairPitch, a.t + (long long)z0 * nx * ny, nx, ny, nx, ky, cx);
    cp_async_commit();
    pair_stage<32>(B2, kPairPitch, a.st[X], nx, nx, nx, kx, cx);
    cp_async_commit();
    if (!pair_live(a)) {
        cp_async_wait<0>();
        return;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, fr = lane >> 2, fc = lane & 3;
    const int m0 = (warp / WN) * 8, n0 = (warp % WN) * FN * 8;    // the warp's 8 rows (y) x 8 FN columns (x)
    const bool active = n0 < mx;
    const int y = y0 + m0 + fr;
    const int reset = a.c->reset_phi;
    for (int z = z0; z < z1; z++) {
        double* phi = a.phi + ((long long)z * ny + min(y, ny - 1)) * nx;
        double old[FN][2];                          // the potential this thread updates, loaded ahead
#pragma unroll
        for (int j = 0; j < FN; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int x = n0 + j * 8 + 2 * fc + h;
                old[j][h] = active && y < ny && x < nx && !reset ? phi[x] : 0.0;
            }
        if (z == z0) cp_async_wait<1>();             // S_y and the first plane (ST_x may still be in flight)
        __syncthreads();
        double acc[1][FN][2];
        if (active) {
            pair_warp_mma<1, FN>(acc, A1, kPairPitch, B1, kPairPitch, ky, m0, n0);
#pragma unroll
            for (int j = 0; j < FN; j++) {
                C1[(m0 + fr) * kPairPitch + n0 + j * 8 + 2 * fc] = acc[0][j][0];
                C1[(m0 + fr) * kPairPitch + n0 + j * 8 + 2 * fc + 1] = acc[0][j][1];
            }
        }
        cp_async_wait<0>();
        __syncthreads();
        if (z + 1 < z1) {
            pair_stage<32>(B1, kPairPitch, a.t + (long long)(z + 1) * nx * ny, nx, ny, nx, ky, cx);
            cp_async_commit();
        }
        if (active) {
            pair_warp_mma<1, FN>(acc, C1, kPairPitch, B2, kPairPitch, kx, m0, n0);
            if (y < ny) {
#pragma unroll
                for (int j = 0; j < FN; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int x = n0 + j * 8 + 2 * fc + h;
                        if (x < nx) phi[x] = old[j][h] + acc[0][j][h];
                    }
            }
        }
        cp_async_wait<0>();
        __syncthreads();
    }
}
template <int W> struct PairYxSmem {
    static constexpr size_t bytes = sizeof(double) * (2 * kPairMax * kPairPitch + 2 * W * kPairPitch);
};

enum PairPhase : int { kPairXy = 0, kPairZ = 1, kPairYx = 2 };

template <int W> __global__ void __launch_bounds__(kPairThreads, 2) pair_xy_kernel(FdmPairArgs a) {
    pair_xy_body<W>(a, real_blk(), first_block());
}
template <int W> __global__ void __launch_bounds__(kPairThreads, 2) pair_z_kernel(FdmPairArgs a) {
    pair_z_body<W>(a, real_blk(), first_block());
}
template <int W> __global__ void __launch_bounds__(kPairThreads, 2) pair_yx_kernel(FdmPairArgs a) {
    pair_yx_body<W>(a, real_blk(), first_block());
}
// a batch of cavities: grid x runs over the work list (BatchItem); the phase selects the body
template <int PHASE, int W>
__global__ void __launch_bounds__(kPairThreads, 2) pair_batched(const FdmPairArgs* args, const BatchItem* items,
                                                               const int* live) {
    __shared__ FdmPairArgs a;
    int cav;
    const Blk k = item_blk(items, live, cav);
    if (cav < 0) {
        if (PHASE == kPairXy) dead_slot_clear(args, items);
        return;
    }
    load_args(a, args + cav);
    if (PHASE == kPairXy) pair_xy_body<W>(a, k, first_block());
    else if (PHASE == kPairZ) pair_z_body<W>(a, k, first_block());
    else pair_yx_body<W>(a, k, first_block());
}
inline size_t pair_smem_bytes(int phase, int w) {
    if (w == 16) return phase == kPairYx ? PairYxSmem<16>::bytes : PairSmem<16>::bytes;
    return phase == kPairYx ? PairYxSmem<32>::bytes : PairSmem<32>::bytes;
}
// grid of one phase for an nx x ny x nz cavity with CTA width w and `per` tiles per CTA
inline dim3 pair_grid(int phase, int w, int nx, int ny, int nz, int per = 1) {
    if (phase == kPairXy) return dim3((nx + w - 1) / w, (nz + per - 1) / per);
    if (phase == kPairZ) return dim3(((nx * ny + w - 1) / w + per - 1) / per);
    return dim3((ny + w - 1) / w, (nz + per - 1) / per);
}
inline bool pair_pass_fits(int nx, int ny, int nz) {
    return nx <= kPairMax && ny <= kPairMax && nz <= kPairMax;
}
inline int current_sm_count() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 148;
    return sms;
}
// CTA width: 32 columns (rows), or 16 when a single cavity's 32-wide grid leaves SMs without a CTA (more, smaller
// CTAs: two per SM hide each other's latency).  A batch's launches all take 32.  CAVITY_PAIR_W=16 or 32 forces it.
inline int pair_width(int nx, int nz) {
    static const int forced = [] {
        const char* e = std::getenv("CAVITY_PAIR_W");
        return e ? std::atoi(e) : 0;
    }();
    static const int sms = current_sm_count();
    if (forced == 16 || forced == 32) return forced;
    if (g_launch_record) return 32;
    const long long ctas = (long long)((nx + 31) / 32) * nz;
    return ctas < sms ? 16 : 32;
}
// Tiles per CTA of a paired launch: one for a single cavity; in a batch as many as leave the whole launch (all its
// cavities counted at this one's size) three to four waves of two CTAs per SM, evened out over the axis, so that a
// CTA stages its bases once for several tiles and copies each next tile's field under the current tile's
// arithmetic.  For 64 cavities of 64^3 that is 8 planes per CTA: the batch's first passes took 2.15 ms per step
// against 2.51 with one tile per CTA, 2.19 with 4 and 2.35 with 16.  At most 8 tiles per CTA, so that in a batch of
// mixed sizes (each member counted at its own size) no CTA holds much more work than that.  CAVITY_PAIR_PER forces
// it.
inline int pair_per(int phase, int w, int nx, int ny, int nz) {
    static const int forced = [] {
        const char* e = std::getenv("CAVITY_PAIR_PER");
        return e ? std::atoi(e) : 0;
    }();
    static const int sms = current_sm_count();
    const dim3 g = pair_grid(phase, w, nx, ny, nz, 1);
    const int along = phase == kPairZ ? (int)g.x : nz;      // the tiles one CTA can take in a row
    int per = forced;
    if (per <= 0) {
        const long long tiles = (long long)g.x * g.y * std::max(g_launch_batch, 1);
        per = (int)std::min<long long>(std::min(along, 8), std::max(1LL, tiles / (6LL * sms)));
        const int chunks = (along + per - 1) / per;
        per = (along + chunks - 1) / chunks;
    }
    return std::max(1, std::min(per, along));
}
template <int W> inline cudaError_t pair_prepare_w() {
    cudaError_t r = cudaFuncSetAttribute(pair_xy_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)pair_smem_bytes(kPairXy, W));
    if (r == cudaSuccess)
        r = cudaFuncSetAttribute(pair_z_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pair_smem_bytes(kPairZ, W));
    if (r == cudaSuccess)
        r = cudaFuncSetAttribute(pair_yx_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pair_smem_bytes(kPairYx, W));
    if (r == cudaSuccess)
        r = cudaFuncSetAttribute(pair_batched<kPairXy, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pair_smem_bytes(kPairXy, W));
    if (r == cudaSuccess)
        r = cudaFuncSetAttribute(pair_batched<kPairZ, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pair_smem_bytes(kPairZ, W));
    if (r == cudaSuccess)
        r = cudaFuncSetAttribute(pair_batched<kPairYx, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pair_smem_bytes(kPairYx, W));
    return r;
}
// once per process, before any capture: the dynamic shared memory of the paired kernels
inline cudaError_t pair_prepare() {
    static const cudaError_t e = [] {
        const cudaError_t r = pair_prepare_w<32>();
        return r == cudaSuccess ? pair_prepare_w<16>() : r;
    }();
    return e;
}
template <int W>
inline void launch_pair_w(int phase, dim3 grid, cudaStream_t st, const FdmPairArgs& a) {
    const size_t smem = pair_smem_bytes(phase, W);
    if (phase == kPairXy) launch_pdl(pair_xy_kernel<W>, grid, dim3(kPairThreads), smem, st, a);
    else if (phase == kPairZ) launch_pdl(pair_z_kernel<W>, grid, dim3(kPairThreads), smem, st, a);
    else launch_pdl(pair_yx_kernel<W>, grid, dim3(kPairThreads), smem, st, a);
}
inline void launch_fdm_pass_pairs(cudaStream_t st, const FdmOperands& op, const double* r, const double* r_alt,
                                  double* phi, double* t, const Control* c, cudaGraphConditionalHandle h, bool clear) {
    FdmPairArgs a;
    a.nx = op.nx; a.ny = op.ny; a.nz = op.nz;
    a.clear_condition = clear;
    for (int k = 0; k < 3; k++) { a.s[k] = op.s[k]; a.st[k] = op.st[k]; }
    a.inv_lambda = op.inv_lambda;
    a.r = r; a.r_alt = r_alt; a.t = t; a.phi = phi; a.c = c; a.handle = h;
    const int w = pair_width(op.nx, op.nz);
    for (int ph = 0; ph < 3; ph++) {
        a.per = pair_per(ph, w, op.nx, op.ny, op.nz);
        const dim3 grid = pair_grid(ph, w, op.nx, op.ny, op.nz, a.per);
        if (record_launch(kLkPair, ph | (w << 4), grid, pair_smem_bytes(ph, w), a)) continue;
        if (w == 16) launch_pair_w<16>(ph, grid, st, a);
        else launch_pair_w<32>(ph, grid, st, a);
    }
}
// a recorded paired launch (variant: phase | width << 4) over a batch of cavities
template <int W>
inline void launch_pair_batched_w(int phase, dim3 grid, const BatchItem* items, const int* live, const FdmPairArgs* d,
                                  cudaStream_t st) {
    const size_t smem = pair_smem_bytes(phase, W);
    if (phase == kPairXy) launch_pdl(pair_batched<kPairXy, W>, grid, dim3(kPairThreads), smem, st, d, items, live);
    else if (phase == kPairZ) launch_pdl(pair_batched<kPairZ, W>, grid, dim3(kPairThreads), smem, st, d, items, live);
    else launch_pdl(pair_batched<kPairYx, W>, grid, dim3(kPairThreads), smem, st, d, items, live);
}
inline void launch_pair_batched(int variant, dim3 grid, const BatchItem* items, const int* live, const FdmPairArgs* d,
                                cudaStream_t st) {
    if ((variant >> 4) == 16) launch_pair_batched_w<16>(variant & 15, grid, items, live, d, st);
    else launch_pair_batched_w<32>(variant & 15, grid, items, live, d, st);
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
// How a pass's six transforms are launched (CAVITY_FDM_FUSED, read when a solver or batch is created or a
// standalone pass is called; else a cavity's autotuned choice; else -1: by size).
//   kPassSix:        six launches of the tile GEMM;
//   kPassOneLaunch:  one cooperative launch with grid barriers (single cavities only).  It is not a default: inside
//                    the step graph it measured slower than six launches (C2 step 0.383 against 0.368 ms), the
//                    graph's programmatic launches already hiding most of the gaps that the grid barriers replace;
//   kPassPairs:      three launches of two chained transforms each, when no axis has more than 64 cells: the
//                    default there.
// A batch's launches follow the batch's choice (g_batch_pairs), the same for every member.
enum PassForm : int { kPassSix = 0, kPassOneLaunch = 1, kPassPairs = 2 };
inline int pass_form_from_env() {
    const char* e = std::getenv("CAVITY_FDM_FUSED");
    return e && *e ? std::atoi(e) : -1;
}
inline int pass_form(const FdmOperands& op, int want) {
    const bool fits = pair_pass_fits(op.nx, op.ny, op.nz);
    if (g_launch_record) return g_batch_pairs > 0 && fits ? kPassPairs : kPassSix;
    const int f = want;
    if (f == kPassOneLaunch) return g_dgemm_tile != 64 && fused_pass_capacity() > 0 ? kPassOneLaunch : kPassSix;
    if (f == kPassSix) return kPassSix;
    return fits ? kPassPairs : kPassSix;
}

inline void launch_fdm_pass(cudaStream_t st, const FdmOperands& op, const double* r, const double* r_alt, double* phi,
                            double* t1, double* t2, Control* c, cudaGraphConditionalHandle h, bool clear, int form = -1) {
    const int f = pass_form(op, form);
    if (f == kPassOneLaunch) {
        launch_fdm_pass_fused(st, op, r, r_alt, phi, t1, t2, c, h, clear);
        return;
    }
    if (f == kPassPairs) {
        launch_fdm_pass_pairs(st, op, r, r_alt, phi, t1, c, h, clear);
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
