// eigen_gpu.cu - the pressure operator's 1-D eigenbases on the GPU (solver set-up with CAVITY_EIGEN=gpu).
//
// The generalised problem K S = W S diag(lambda) of an axis (backend.cu:723-767) is solved on its symmetric
// tridiagonal form T = W^-1/2 K W^-1/2 (setup.cpp, axis_tridiagonal):
//   - eigenvalues by bisection on Sturm counts, one thread per eigenvalue, each to the resolution of doubles;
//   - eigenvectors by inverse iteration on T - lambda I, factored by Gaussian elimination with partial pivoting
//     (the tridiagonal LU of Golub and Van Loan, Matrix Computations, 4.3), three solves from a start vector
//     with no symmetry (a symmetric one would miss the antisymmetric modes of a symmetric grid).
// Eigenvalues closer than 1e-3 of the matrix norm form a cluster; one block takes a cluster and orthogonalises
// each of its vectors against the earlier ones after every solve (Gram-Schmidt), as the inverse iteration of
// LAPACK's dstein does.  On a stretched grid the low modes are closer than that, so one cluster can hold most of
// the spectrum: its recurrences run on one thread and its projections on the whole block.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "setup.h"

namespace cavity {
namespace {

void check_eigen(cudaError_t e) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("pressure solver set-up (GPU eigenbasis): ") +
                                                   cudaGetErrorString(e));
}

// number of eigenvalues of the tridiagonal (d, e) below x: negative pivots of the LDL^T factorisation of T - x I
__device__ int sturm_count(const double* d, const double* e2, int n, double x, double pivmin) {
    int count = 0;
    double q = d[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    count += q < 0.0;
    for (int i = 1; i < n; i++) {
        q = d[i] - x - e2[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        count += q < 0.0;
    }
    return count;
}

// eigenvalue k (ascending) by bisection of the Gershgorin interval [lo, hi]
__global__ void bisect_kernel(const double* d, const double* e2, int n, double lo0, double hi0, double pivmin,
                              double* lambda) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double lo = lo0, hi = hi0;
    for (int it = 0; it < 2200; it++) {
        const double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;                                    // adjacent doubles
        if (hi - lo <= 2.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)) + pivmin) break;
        if (sturm_count(d, e2, n, mid, pivmin) > k) hi = mid;
        else lo = mid;
    }
    lambda[k] = 0.5 * (lo + hi);
}

constexpr int kClusterThreads = 128;

// sum over the block (every thread gets it)
__device__ double block_sum(double v, double* red) {
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = kClusterThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// Inverse iteration for the eigenvalues of one cluster, [cluster[t], cluster[t + 1]), in block t (kClusterThreads
// threads).  Thread 0 factors T - lambda I and solves with it (sequential recurrences, on the block's workspace,
// which stays in L1); the block orthogonalises against the cluster's earlier vectors (classical Gram-Schmidt,
// twice) and normalises.  Workspace `work`: 7 arrays of n per block.  Eigenvector k goes to column k of Z.
__global__ void __launch_bounds__(kClusterThreads) inverse_iteration_kernel(const double* d, const double* e, int n,
                                                                          const double* lambda, const int* cluster,
                                                                          double tiny, double* work, double* Z) {
    __shared__ double red[kClusterThreads];
    const int t = blockIdx.x, tid = threadIdx.x;
    double* D = work + (size_t)t * 7 * n;      // U: diagonal, superdiagonals C and C2; multipliers L; swaps P
    double* C = D + n;
    double* C2 = C + n;
    double* L = C2 + n;
    double* P = L + n;
    double* B = P + n;                         // the iterate
    double* G = B + n;                         // its projections on the cluster's earlier vectors
    const int c0 = cluster[t], c1 = cluster[t + 1];
    for (int k = c0; k < c1; k++) {
        const double lam = lambda[k];
        if (tid == 0) {
            for (int i = 0; i < n; i++) {
                D[i] = d[i] - lam;
                C[i] = i + 1 < n ? e[i] : 0.0;
                C2[i] = 0.0;
            }
            for (int i = 0; i + 1 < n; i++) {
                const double sub = e[i];                   // below the diagonal in row i + 1
                const double di = D[i];
                if (fabs(di) >= fabs(sub)) {
                    const double piv = di != 0.0 ? di : tiny;
                    D[i] = piv;
                    const double m = sub / piv;
                    L[i] = m;
                    P[i] = 0.0;
                    D[i + 1] -= m * C[i];
                } else {                                   // swap rows i and i + 1
                    const double m = di / sub;
                    L[i] = m;
                    P[i] = 1.0;
                    const double ci = C[i], d1 = D[i + 1], c1n = i + 2 < n ? C[i + 1] : 0.0;
                    D[i] = sub;
                    C[i] = d1;
                    C2[i] = c1n;
                    D[i + 1] = ci - m * d1;
                    if (i + 2 < n) C[i + 1] = -m * c1n;
                }
            }
            if (D[n - 1] == 0.0) D[n - 1] = tiny;
        }
        // start vector without symmetry, in (0.5, 1.5)
        for (int i = tid; i < n; i += kClusterThreads) {
            unsigned int h = (unsigned int)(i * 2654435761u) ^ (unsigned int)(k * 40503u + 12345u);
            h ^= h >> 13;
            h *= 0x5bd1e995u;
            h ^= h >> 15;
            B[i] = 0.5 + (double)(h & 0xffffff) / 16777216.0;
        }
        __syncthreads();
        for (int iter = 0; iter < 3; iter++) {
            if (tid == 0) {
                for (int i = 0; i + 1 < n; i++) {          // apply P and L
                    if (P[i] != 0.0) {
                        const double b0 = B[i];
                        B[i] = B[i + 1];
                        B[i + 1] = b0;
                    }
                    B[i + 1] -= L[i] * B[i];
                }
                for (int i = n - 1; i >= 0; i--) {        // back substitution with U
                    double s = B[i];
                    if (i + 1 < n) s -= C[i] * B[i + 1];
                    if (i + 2 < n) s -= C2[i] * B[i + 2];
                    B[i] = s / D[i];
                }
            }
            __syncthreads();
            for (int pass = 0; pass < 2 && k > c0; pass++) {   // orthogonal to the cluster's earlier vectors
                for (int j = c0 + tid; j < k; j += kClusterThreads) {
                    double s = 0.0;
                    for (int i = 0; i < n; i++) s += Z[(long long)i * n + j] * B[i];
                    G[j - c0] = s;
                }
                __syncthreads();
                for (int i = tid; i < n; i += kClusterThreads) {
                    double v = B[i];
                    for (int j = c0; j < k; j++) v -= G[j - c0] * Z[(long long)i * n + j];
                    B[i] = v;
                }
                __syncthreads();
            }
            double part = 0.0;
            for (int i = tid; i < n; i += kClusterThreads) part += B[i] * B[i];
            const double inv = 1.0 / sqrt(block_sum(part, red));
            for (int i = tid; i < n; i += kClusterThreads) B[i] *= inv;
            __syncthreads();
        }
        for (int i = tid; i < n; i += kClusterThreads) Z[(long long)i * n + k] = B[i];
        __syncthreads();
    }
}

}  // namespace

AxisEigen axis_eigen_gpu(const AxisGrid& g) {
    const int n = g.n;
    std::vector<double> d, e;
    axis_tridiagonal(g, d, e);
    std::vector<double> e2(n, 0.0);
    double lo = INFINITY, hi = -INFINITY, norm = 0.0, emax2 = 0.0;
    for (int i = 0; i < n; i++) {
        const double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(e[i]) : 0.0);
        lo = std::min(lo, d[i] - r);
        hi = std::max(hi, d[i] + r);
        norm = std::max(norm, std::fabs(d[i]) + r);
        if (i + 1 < n) {
            e2[i] = e[i] * e[i];
            emax2 = std::max(emax2, e2[i]);
        }
    }
    const double pivmin = 2.2250738585072014e-308 * std::max(1.0, emax2);
    const double span = std::max(hi - lo, norm) * 2.220446049250313e-16 * n;
    lo -= span;
    hi += span;

    cudaStream_t st;
    check_eigen(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    double *dd = nullptr, *de = nullptr, *de2 = nullptr, *dl = nullptr, *dz = nullptr, *dw = nullptr;
    int* dc = nullptr;
    std::vector<double> lambda(n), Z((size_t)n * n);
    cudaError_t err = cudaSuccess;
    auto step = [&](cudaError_t e) {
        if (err == cudaSuccess) err = e;
    };
    step(cudaMallocAsync((void**)&dd, sizeof(double) * n, st));
    step(cudaMallocAsync((void**)&de, sizeof(double) * n, st));
    step(cudaMallocAsync((void**)&de2, sizeof(double) * n, st));
    step(cudaMallocAsync((void**)&dl, sizeof(double) * n, st));
    step(cudaMallocAsync((void**)&dz, sizeof(double) * n * n, st));
    if (err == cudaSuccess) {
        step(cudaMemcpyAsync(dd, d.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
        step(cudaMemcpyAsync(de, e.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
        step(cudaMemcpyAsync(de2, e2.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
        bisect_kernel<<<(n + 127) / 128, 128, 0, st>>>(dd, de2, n, lo, hi, pivmin, dl);
        step(cudaGetLastError());
        step(cudaMemcpyAsync(lambda.data(), dl, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        step(cudaStreamSynchronize(st));
    }
    // clusters of eigenvalues closer than 1e-3 of the norm (ascending order)
    std::vector<int> cluster{0};
    for (int k = 1; k < n; k++)
        if (lambda[k] - lambda[k - 1] > 1e-3 * norm) cluster.push_back(k);
    cluster.push_back(n);
    const int clusters = (int)cluster.size() - 1;
    if (err == cudaSuccess) {
        step(cudaMallocAsync((void**)&dc, sizeof(int) * cluster.size(), st));
        step(cudaMallocAsync((void**)&dw, sizeof(double) * 7 * (size_t)n * clusters, st));
    }
    if (err == cudaSuccess) {
        step(cudaMemcpyAsync(dc, cluster.data(), sizeof(int) * cluster.size(), cudaMemcpyHostToDevice, st));
        inverse_iteration_kernel<<<clusters, kClusterThreads, 0, st>>>(dd, de, n, dl, dc, 2.220446049250313e-16 * norm,
                                                                       dw, dz);
        step(cudaGetLastError());
        step(cudaMemcpyAsync(Z.data(), dz, sizeof(double) * n * n, cudaMemcpyDeviceToHost, st));
        step(cudaStreamSynchronize(st));
    }
    for (void* p : {(void*)dd, (void*)de, (void*)de2, (void*)dl, (void*)dz, (void*)dw, (void*)dc})
        if (p) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    check_eigen(err);
    return axis_eigen_finish(g, std::move(lambda), Z);
}

}  // namespace cavity
