// fdm.cuh - one pass of the fast-diagonalisation (FDM) pressure solve (backend.cu:801-814), as launches of the
// batched transform kernel of kernels.cuh:  t = S_z^T S_y^T S_x^T r (along x, y, z), t *= inv_lambda,
// phi += S_x S_y S_z t.  Fields are [z][y][x]; S_a is the row-major n_a x n_a eigenbasis of axis a
// (eigenvector j in column j) and ST_a its transpose.
#pragma once
#include <cstring>

#include "kernels.cuh"

namespace cavity {

struct FdmOperands {
    int nx, ny, nz;
    const double* s[3];
    const double* st[3];
    const double* inv_lambda;
};

template <int BM, int BN, int BK, int TM, int TN>
inline void launch_transform(cudaStream_t st, int M, int N, int K, const double* A, const double* A_alt, int lda,
                             long long sA, const double* B, int ldb, long long sB, double* C, int ldc, long long sC,
                             int batch, int epi, const double* inv_lambda, double* phi, const Control* c,
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
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, batch);
    gemm_kernel<double, BM, BN, BK, TM, TN><<<grid, (BM / TM) * (BN / TN), 0, st>>>(g);
}

// phi += FDM(r); r_alt replaces r when the control block says use_rhs.  t1, t2: nx*ny*nz doubles of scratch.
// `clear` makes the first launch clear the condition of the enclosing graph while-node `h`.
inline void launch_fdm_pass(cudaStream_t st, const FdmOperands& op, const double* r, const double* r_alt, double* phi,
                            double* t1, double* t2, const Control* c, cudaGraphConditionalHandle h, bool clear) {
    const int nx = op.nx, ny = op.ny, nz = op.nz, plane = nx * ny;
    const long long pl = plane;
    const double* il = op.inv_lambda;
    launch_transform<32, 32, 8, 2, 2>(st, ny * nz, nx, nx, r, r_alt, nx, 0, op.s[0], nx, 0, t1, nx, 0, 1, kStore, il,
                                      nullptr, c, h, clear);
    launch_transform<32, 32, 8, 2, 2>(st, ny, nx, ny, op.st[1], nullptr, ny, 0, t1, nx, pl, t2, nx, pl, nz, kStore, il,
                                      nullptr, c, 0, false);
    launch_transform<32, 32, 8, 2, 2>(st, nz, plane, nz, op.st[2], nullptr, nz, 0, t2, plane, 0, t1, plane, 0, 1,
                                      kScaleInvLambda, il, nullptr, c, 0, false);
    launch_transform<32, 32, 8, 2, 2>(st, nz, plane, nz, op.s[2], nullptr, nz, 0, t1, plane, 0, t2, plane, 0, 1, kStore,
                                      il, nullptr, c, 0, false);
    launch_transform<32, 32, 8, 2, 2>(st, ny, nx, ny, op.s[1], nullptr, ny, 0, t2, nx, pl, t1, nx, pl, nz, kStore, il,
                                      nullptr, c, 0, false);
    launch_transform<32, 32, 8, 2, 2>(st, ny * nz, nx, nx, t1, nullptr, nx, 0, op.st[0], nx, 0, nullptr, nx, 0, 1,
                                      kAccumulate, il, phi, c, 0, false);
}

// Control block for a pass outside a solver: no error, a non-zero residual, accumulate into phi.
inline Control standalone_fdm_control() {
    Control c;
    memset(&c, 0, sizeof c);
    c.res_norm2 = 1.0;
    c.rhs_norm2 = 1.0;
    return c;
}

}  // namespace cavity
