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

#include "layout.h"

namespace cavity {

constexpr int kThreads = 256;
constexpr int X = 0, Y = 1, Z = 2;

// ------------------------------------------------------------------------------------------ control block
enum ErrorCode : int {
    kOk = 0,
    kVelocityNaN = 1,      // backend.cu:890
    kRhsNaN = 2,           // backend.cu:820
    kResidualNaN = 3,      // backend.cu:838
    kNotConverged = 4,     // backend.cu:840-844
};
enum Counter : int { kCntDiv = 0, kCntRes0, kCntRes, kCntFinish, kCntCfl, kNumCounters };

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
    const T* tab[3];             // tab[a][k * stride[a] + i]
    int stride[3];
    const double* dw[3];         // widths (double, float-rounded values)
    const double* dinv_sp[3];    // 1/spacing in double
    const T* lid_u;              // lid shape on the top u-faces, [z][x] with nx+1 per row
};

template <class T> __device__ __forceinline__ T tab(const Geo<T>& g, int a, int k, int i) {
    return g.tab[a][k * g.stride[a] + i];
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

// Write this block's partials; returns true in every thread of the last block to finish, after which the
// partials of all blocks are visible to it.  The last block resets the counter for the next launch.
template <int N>
__device__ bool publish_partials(const Vec<N>& blk, double* partial, unsigned int* counter) {
    __shared__ bool last;
    const unsigned int nblocks = gridDim.x * gridDim.y;
    const unsigned int b = blockIdx.x + gridDim.x * blockIdx.y;
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

// In the last block: reduce all partials in a fixed order.  Result valid in thread 0.
template <int N, bool MAX>
__device__ Vec<N> final_reduce(const double* partial) {
    const unsigned int nblocks = gridDim.x * gridDim.y;
    Vec<N> acc;
#pragma unroll
    for (int k = 0; k < N; k++) {
        double a = MAX ? -INFINITY : 0.0;
        for (unsigned int i = threadIdx.x; i < nblocks; i += blockDim.x)
            a = combine<N, MAX>(a, __ldcg(partial + k * nblocks + i));
        acc.v[k] = a;
    }
    return block_reduce<N, MAX>(acc);
}

// ------------------------------------------------------------------------------------------ step begin
// dt from the CFL rate of the current velocity and the viscous rate (backend.cu:884-899).
__global__ void step_begin_kernel(Params p, Control* c) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
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
// One RK3 stage of the impulse for every face: inviscid term I = Lamb vector - grad(u.m) (backend.cu:102-274)
// fused with the viscous flux-form Laplacian, wall/lid fluxes and the RK combination (backend.cu:279-330).
// Stage 0 also performs the gauge reset m0 = r m + (1-r) u (backend.cu:880-881) on the fly and stores m0.
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

template <class T> struct MomentumView {
    const MomentumArgs<T>& a;
    bool blend;
    __device__ __forceinline__ T mval(int C, int i) const {
        const T mv = a.m[C][i];
        return blend ? a.r * mv + a.one_minus_r * a.u[C][i] : mv;
    }
};

// Lamb term of one edge for faces normal to A with tangential axis B: (d u_B/d x_A - d u_A/d x_B) * u_B
// interpolated along A, times the stencil weight; zero where the edge or its stencil leaves the box.
template <int A, int B, int Q, class T>
__device__ __forceinline__ T lamb_edge(const MomentumArgs<T>& a, int ia, int e, int id) {
    const Params& p = a.p;
    const int na = A == X ? p.nx : A == Y ? p.ny : p.nz;
    const int nb = B == X ? p.nx : B == Y ? p.ny : p.nz;
    const int al = ia - (Q + 1) / 2, ah = ia + (Q - 1) / 2;
    const int bl = e - (Q + 1) / 2, bh = e + (Q - 1) / 2;
    if (e < 0 || e > nb || al < 0 || ah > na - 1) return T(0);
    const T s = tab(a.g, B, kRamp, e) * tab(a.g, A, kRamp, ia);
    const T wq = Q == 1 ? (p.o4 ? T(1) + s * T(0.125) : T(1)) : -s * T(0.125);
    if (wq == T(0)) return T(0);
    if (bl < 0 || bh > nb - 1) return T(0);
    const T ub_lo = a.u[B][fidx_ab<B, A, B>(p, al, e, id)];
    const T ub_hi = a.u[B][fidx_ab<B, A, B>(p, ah, e, id)];
    const T ua_lo = a.u[A][fidx_ab<A, A, B>(p, ia, bl, id)];
    const T ua_hi = a.u[A][fidx_ab<A, A, B>(p, ia, bh, id)];
    const T inv_nda = Q == 1 ? tab(a.g, A, kInvSp, ia) : tab(a.g, A, kInvNd3, ia);
    const T inv_ndb = Q == 1 ? tab(a.g, B, kInvSp, e) : tab(a.g, B, kInvNd3, e);
    const T o = (ub_hi - ub_lo) * inv_nda - (ua_hi - ua_lo) * inv_ndb;
    const T ev = Q == 1 ? tab(a.g, A, kEv1Lo, ia) * ub_lo + tab(a.g, A, kEv1Hi, ia) * ub_hi
                        : tab(a.g, A, kEv3Lo, ia) * ub_lo + tab(a.g, A, kEv3Hi, ia) * ub_hi;
    return wq * o * ev;
}

// K = u.m at the centre of cell (x, y, z) (backend.cu:218-222)
template <class T>
__device__ __forceinline__ T k_cell(const MomentumView<T>& v, int x, int y, int z) {
    const Params& p = v.a.p;
    const int a0 = fidx<X>(p, x, y, z), b0 = fidx<Y>(p, x, y, z), c0 = fidx<Z>(p, x, y, z);
    const int b1 = b0 + p.nx, c1 = c0 + p.nx * p.ny;
    const T* const* u = v.a.u;
    return T(0.5) * ((u[X][a0] * v.mval(X, a0) + u[X][a0 + 1] * v.mval(X, a0 + 1)) +
                     (u[Y][b0] * v.mval(Y, b0) + u[Y][b1] * v.mval(Y, b1)) +
                     (u[Z][c0] * v.mval(Z, c0) + u[Z][c1] * v.mval(Z, c1)));
}

template <int A, int Q, class T>
__device__ __forceinline__ T lamb_q(const MomentumArgs<T>& a, const int q[3]) {
    // tangential axes in the reference's order (backend.cu:235-236, 252-253, 269-270)
    constexpr int B1 = A == X ? Y : A == Y ? X : Y;
    constexpr int B2 = A == X ? Z : A == Y ? Z : X;
    constexpr int D1 = 3 - A - B1, D2 = 3 - A - B2;
    constexpr int up = (Q + 1) / 2, down = (Q - 1) / 2;
    const T c = Q == 1 ? T(0.5) : tab(a.g, A, kC3, q[A]);
    T L = c * (lamb_edge<A, B1, Q>(a, q[A], q[B1] + up, q[D1]) + lamb_edge<A, B1, Q>(a, q[A], q[B1] - down, q[D1]));
    L = L + c * (lamb_edge<A, B2, Q>(a, q[A], q[B2] + up, q[D2]) + lamb_edge<A, B2, Q>(a, q[A], q[B2] - down, q[D2]));
    return L;
}

template <int A, class T>
__device__ void momentum_face(const MomentumArgs<T>& a, const StageConst& sc, T dt, T lidv, int x, int y, int z) {
    const Params& p = a.p;
    const int q[3] = {x, y, z};
    const int n[3] = {p.nx, p.ny, p.nz};
    const int i = fidx<A>(p, x, y, z);
    const MomentumView<T> v{a, a.stage == 0};
    if (a.stage == 0) a.m0_out[A][i] = v.mval(A, i);
    if (q[A] == 0 || q[A] == n[A]) { a.out[A][i] = T(0); return; }
    // inviscid term
    T L = T(0);
    L = L + lamb_q<A, 1>(a, q);
    if (p.o4) {
        // the two halves of the q=3 sum are added separately, in the reference's order
        constexpr int B1 = A == X ? Y : A == Y ? X : Y;
        constexpr int B2 = A == X ? Z : A == Y ? Z : X;
        constexpr int D1 = 3 - A - B1, D2 = 3 - A - B2;
        const T c = tab(a.g, A, kC3, q[A]);
        L = L + c * (lamb_edge<A, B1, 3>(a, q[A], q[B1] + 2, q[D1]) + lamb_edge<A, B1, 3>(a, q[A], q[B1] - 1, q[D1]));
        L = L + c * (lamb_edge<A, B2, 3>(a, q[A], q[B2] + 2, q[D2]) + lamb_edge<A, B2, 3>(a, q[A], q[B2] - 1, q[D2]));
    }
    {
        int lo[3] = {x, y, z};
        lo[A]--;
        L = L - (k_cell(v, x, y, z) - k_cell(v, lo[0], lo[1], lo[2])) * tab(a.g, A, kInvSp, q[A]);
    }
    // viscous flux-form Laplacian with wall and lid fluxes (backend.cu:289-325)
    const T cc = v.mval(A, i);
    const T wall = a.u[A][i];
    const int ex = p.nx + (A == X), exy = ex * (p.ny + (A == Y));
    const int stride[3] = {1, ex, exy};
    T lap = T(0);
#pragma unroll
    for (int t = 0; t < 3; t++) {
        const int s = stride[t];
        if (t == A) {
            lap = lap + ((v.mval(A, i + s) - cc) * tab(a.g, t, kInvW, q[t]) -
                         (cc - v.mval(A, i - s)) * tab(a.g, t, kInvW, q[t] - 1)) * tab(a.g, t, kInvSp, q[t]);
            continue;
        }
        T hi = q[t] < n[t] - 1 ? (v.mval(A, i + s) - cc) * tab(a.g, t, kInvSp, q[t] + 1) : T(0);
        T lo = q[t] > 0 ? (cc - v.mval(A, i - s)) * tab(a.g, t, kInvSp, q[t]) : T(0);
        if (q[t] == 0) lo = wall * tab(a.g, t, kInvSp, 0);
        if (q[t] == n[t] - 1) {
            if (t == Y) {
                const T U = A == X ? lidv * a.g.lid_u[x + (p.nx + 1) * z] : T(0);
                hi = (U - wall) * tab(a.g, Y, kInvSp, n[Y]);
            } else {
                hi = -wall * tab(a.g, t, kInvSp, n[t]);
            }
        }
        lap = lap + (hi - lo) * tab(a.g, t, kInvW, q[t]);
    }
    T val = cc + dt * (a.nu * lap + L);
    if (a.stage > 0) val = T(sc.a0) * a.m0[A][i] + T(sc.b) * val;
    a.out[A][i] = val;
}

// grid: (ceil(max faces / kThreads), 3); blockIdx.y = component
template <class T>
__global__ void __launch_bounds__(kThreads) momentum_kernel(MomentumArgs<T> a) {
    if (a.c->error) return;
    const Params& p = a.p;
    const int comp = blockIdx.y;
    const int ex = p.nx + (comp == 0), ey = p.ny + (comp == 1), ez = p.nz + (comp == 2);
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= ex * ey * ez) return;
    const int x = i % ex, y = (i / ex) % ey, z = i / (ex * ey);
    const StageConst sc = stage_const(a.stage, a.c);
    const T dt = (T)a.c->dt;
    const T lidv = (T)lid_speed(p, sc.tau);
    if (comp == 0) momentum_face<X>(a, sc, dt, lidv, x, y, z);
    else if (comp == 1) momentum_face<Y>(a, sc, dt, lidv, x, y, z);
    else momentum_face<Z>(a, sc, dt, lidv, x, y, z);
}

// ------------------------------------------------------------------------------------------ divergence
// rhs = volume * div(m) in FP64 (backend.cu:334-342); in a step also the potential carried by the RK
// combination (base, backend.cu:922-923), the warm-start guess (backend.cu:924-925, 857-873) and, in stage 0,
// the gauge-reset potential phi0 = r phi (backend.cu:882).
template <class T> struct DivergenceArgs {
    Params p;
    Geo<T> g;
    const T* m[3];
    double* rhs;
    // step only (null in a plain projection)
    const double* phi_state;    // stage 0: state potential
    double* phi0;               // stage 0 writes, stages 1, 2 read
    const double* phi_cur;      // stages 1, 2: potential of the previous stage
    double* base;
    double* guess;              // the new potential buffer, initialised with the guess
    const double* hist[4];
    int stage;
    Control* c;
    double* partial;
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

template <class T>
__global__ void __launch_bounds__(kThreads) divergence_kernel(DivergenceArgs<T> a) {
    Control* c = a.c;
    if (c->error) return;
    const Params& p = a.p;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    Vec<1> acc;
    acc.v[0] = 0.0;
    if (i < p.n_cell) {
        const int x = i % p.nx, y = (i / p.nx) % p.ny, z = i / (p.nx * p.ny);
        const double dx = a.g.dw[X][x], dy = a.g.dw[Y][y], dz = a.g.dw[Z][z];
        const int iu = fidx<X>(p, x, y, z), iv = fidx<Y>(p, x, y, z), iw = fidx<Z>(p, x, y, z);
        const double r = ((double)a.m[X][iu + 1] - (double)a.m[X][iu]) * (dy * dz) +
                         ((double)a.m[Y][iv + p.nx] - (double)a.m[Y][iv]) * (dx * dz) +
                         ((double)a.m[Z][iw + p.nx * p.ny] - (double)a.m[Z][iw]) * (dx * dy);
        a.rhs[i] = r;
        acc.v[0] = r * r;
        if (a.base) {
            const StageConst sc = stage_const(a.stage, c);
            double base;
            if (a.stage == 0) {
                const double phi0 = p.reinit_r * a.phi_state[i];
                a.phi0[i] = phi0;
                base = sc.b * phi0;
            } else {
                base = sc.a0 * a.phi0[i] + sc.b * a.phi_cur[i];
            }
            a.base[i] = base;
            int b1, b2;
            double c1, c2;
            guess_coefficients(p, c, sc.tau, sc.b * c->dt, b1, c1, b2, c2);
            double g = base;
            if (b1 >= 0) {
                const double ex = b2 >= 0 ? c1 * a.hist[b1][i] + c2 * a.hist[b2][i] : c1 * a.hist[b1][i];
                g = ex + base;
            }
            a.guess[i] = g;
        }
    }
    const Vec<1> blk = block_reduce<1, false>(acc);
    if (publish_partials(blk, a.partial, &c->counter[kCntDiv])) {
        const Vec<1> tot = final_reduce<1, false>(a.partial);
        if (threadIdx.x == 0) {
            c->rhs_norm2 = tot.v[0];
            c->rhs_norm = sqrt(tot.v[0]);
            c->zero_rhs = 0;
            c->phi_passes = 0;
            c->passes = 0;
            if (!isfinite(c->rhs_norm)) { c->error = kRhsNaN; c->cond = 0; }
            else if (c->rhs_norm == 0.0) c->zero_rhs = 1;
            c->counter[kCntDiv] = 0;
        }
    }
}

// ------------------------------------------------------------------------------------------ residual
// r = rhs - L phi with L the 7-point area-weighted Neumann Laplacian (backend.cu:345-359), sum r^2 and
// sum phi.  `first`: the residual of the warm-start guess (or no guess), which decides the start of the
// refinement loop (backend.cu:822-831); otherwise the residual after a pass (backend.cu:835-839).
struct ResidualArgs {
    Params p;
    const double* dw[3];
    const double* dinv_sp[3];
    double* phi;
    const double* rhs;
    double* res;
    int first, have_guess;
    Control* c;
    double* partial;
    cudaGraphConditionalHandle handle;
    int use_handle;
};

__device__ __forceinline__ void set_loop(const ResidualArgs& a, Control* c, int cond) {
    c->cond = cond;
    if (a.use_handle) cudaGraphSetConditional(a.handle, cond ? 1u : 0u);
}

__global__ void __launch_bounds__(kThreads) residual_kernel(ResidualArgs a) {
    Control* c = a.c;
    const Params& p = a.p;
    const int err = c->error;
    const int zero = c->zero_rhs;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    Vec<2> acc;
    acc.v[0] = 0.0;
    acc.v[1] = 0.0;
    if (!err && i < p.n_cell) {
        if (a.first && (zero || !a.have_guess)) {
            a.phi[i] = 0.0;                    // no guess, or nothing to solve: phi = 0
        } else {
            const int x = i % p.nx, y = (i / p.nx) % p.ny, z = i / (p.nx * p.ny);
            const double dx = a.dw[X][x], dy = a.dw[Y][y], dz = a.dw[Z][z];
            const double* f = a.phi;
            const double cc = f[i];
            const int sy = p.nx, sz = p.nx * p.ny;
            double s = 0.0;
            if (x + 1 < p.nx) s += (dy * dz) * (f[i + 1] - cc) * a.dinv_sp[X][x + 1];
            if (x > 0) s -= (dy * dz) * (cc - f[i - 1]) * a.dinv_sp[X][x];
            if (y + 1 < p.ny) s += (dx * dz) * (f[i + sy] - cc) * a.dinv_sp[Y][y + 1];
            if (y > 0) s -= (dx * dz) * (cc - f[i - sy]) * a.dinv_sp[Y][y];
            if (z + 1 < p.nz) s += (dx * dy) * (f[i + sz] - cc) * a.dinv_sp[Z][z + 1];
            if (z > 0) s -= (dx * dy) * (cc - f[i - sz]) * a.dinv_sp[Z][z];
            const double r = a.rhs[i] - s;
            a.res[i] = r;
            acc.v[0] = r * r;
            acc.v[1] = cc;
        }
    }
    const Vec<2> blk = block_reduce<2, false>(acc);
    unsigned int* counter = &c->counter[a.first ? kCntRes0 : kCntRes];
    if (publish_partials(blk, a.partial, counter)) {
        const Vec<2> tot = final_reduce<2, false>(a.partial);
        if (threadIdx.x == 0) {
            *counter = 0;
            if (err) { set_loop(a, c, 0); return; }
            if (a.first) {
                c->passes = 0;
                c->phi_passes = 0;
                c->reset_phi = 0;
                if (zero) {                                           // backend.cu:821
                    c->phi_rel = 0.0;
                    c->phi_sum = 0.0;
                    c->rel = 0.0;
                    set_loop(a, c, 0);
                    return;
                }
                double rel = 1.0;
                c->use_rhs = 1;
                c->phi_sum = 0.0;
                if (a.have_guess) {
                    rel = sqrt(tot.v[0]) / c->rhs_norm;
                    c->res_norm2 = tot.v[0];
                    c->use_rhs = 0;
                    c->phi_sum = tot.v[1];
                    if (rel >= 1.0) { rel = 1.0; c->use_rhs = 1; c->reset_phi = 1; c->phi_sum = 0.0; }
                }
                c->rel = rel;
            } else {
                c->passes += 1;
                c->phi_passes = c->passes;
                c->pass_count += 1;
                c->use_rhs = 0;
                c->reset_phi = 0;
                c->res_norm2 = tot.v[0];
                c->phi_sum = tot.v[1];
                c->rel = sqrt(tot.v[0]) / c->rhs_norm;
                if (!isfinite(c->rel)) { c->error = kResidualNaN; set_loop(a, c, 0); return; }
            }
            const int more = c->rel > p.fdm_rtol && c->passes < p.fdm_max_passes;
            if (!more && c->rel > p.fdm_rtol) {
                c->error = kNotConverged;
                c->error_value = c->rel;
                c->error_passes = c->passes;
            }
            if (!more) c->phi_rel = c->rel;
            set_loop(a, c, more);
        }
    }
}

// ------------------------------------------------------------------------------------------ FDM transforms
// C[b] = A[b] (M x K) * B[b] (K x N), row-major, batched by strides: the directional transforms of the
// fast-diagonalisation pressure solve (backend.cu:792-813).  Register-blocked SIMT tiles; the operand that
// is a residual is chosen on the device (rhs when the guess was rejected, else the residual), the epilogue
// either stores, scales by 1/lambda, or accumulates into phi.
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

template <class D, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) gemm_kernel(GemmArgs<D> g) {
    if (g.clear_condition && threadIdx.x == 0 && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0)
        cudaGraphSetConditional(g.handle, 0u);
    const Control* c = g.c;
    if (c->error) return;
    // a pass with a zero residual does nothing (backend.cu:803-804)
    const double r2 = c->use_rhs ? c->rhs_norm2 : c->res_norm2;
    if (!(r2 > 0)) return;
    constexpr int NT = (BM / TM) * (BN / TN);
    __shared__ D As[BK][BM + 1];
    __shared__ D Bs[BK][BN];
    const int b = blockIdx.z;
    const D* A = (g.A_alt && c->use_rhs ? g.A_alt : g.A) + b * g.sA;
    const D* B = g.B + b * g.sB;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int tx = threadIdx.x % (BN / TN), ty = threadIdx.x / (BN / TN);
    D acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) acc[i][j] = D(0);
    for (int k0 = 0; k0 < g.K; k0 += BK) {
        for (int e = threadIdx.x; e < BM * BK; e += NT) {
            const int r = e / BK, k = e % BK;
            const int gm = m0 + r, gk = k0 + k;
            As[k][r] = (gm < g.M && gk < g.K) ? A[(long long)gm * g.lda + gk] : D(0);
        }
        for (int e = threadIdx.x; e < BK * BN; e += NT) {
            const int k = e / BN, col = e % BN;
            const int gk = k0 + k, gn = n0 + col;
            Bs[k][col] = (gk < g.K && gn < g.N) ? B[(long long)gk * g.ldb + gn] : D(0);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < BK; k++) {
            D av[TM], bv[TN];
#pragma unroll
            for (int i = 0; i < TM; i++) av[i] = As[k][ty + i * (BM / TM)];
#pragma unroll
            for (int j = 0; j < TN; j++) bv[j] = Bs[k][tx + j * (BN / TN)];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[i][j] += av[i] * bv[j];
        }
        __syncthreads();
    }
    const int reset = c->reset_phi;
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int gm = m0 + ty + i * (BM / TM);
        if (gm >= g.M) continue;
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const int gn = n0 + tx + j * (BN / TN);
            if (gn >= g.N) continue;
            const long long idx = b * g.sC + (long long)gm * g.ldc + gn;
            if (g.epilogue == kStore) g.C[idx] = acc[i][j];
            else if (g.epilogue == kScaleInvLambda) g.C[idx] = acc[i][j] * g.inv_lambda[idx];
            else g.phi[idx] = (reset ? 0.0 : g.phi[idx]) + (double)acc[i][j];
        }
    }
}

// ------------------------------------------------------------------------------------------ finish a projection
// u = m - grad(phi) with phi's mean removed (backend.cu:846, 361-371); the potential increment history
// (backend.cu:929-939); in the last stage the CFL rate of the new velocity for the next step's dt
// (backend.cu:465-472) and the clock update (backend.cu:945-954).  One thread per cell; the thread of the
// last cell along an axis also writes the wall face beyond it.  The solution is read from one buffer and the
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
__global__ void __launch_bounds__(kThreads) finish_kernel(FinishArgs<T> a) {
    Control* c = a.c;
    const Params& p = a.p;
    const int err = c->error;
    const int i = blockIdx.x * kThreads + threadIdx.x;
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
    if (!err && i < p.n_cell) {
        const double mean = c->phi_sum / p.n_cell;
        const int x = i % p.nx, y = (i / p.nx) % p.ny, z = i / (p.nx * p.ny);
        const double ph = a.phi[i] - mean;
        // faces below this cell (wall faces 0), and above it at the last cell of an axis
        const int iu = fidx<X>(p, x, y, z), iv = fidx<Y>(p, x, y, z), iw = fidx<Z>(p, x, y, z);
        const int sy = p.nx, sz = p.nx * p.ny;
        T uf[2], vf[2], wf[2];
        uf[0] = x == 0 ? T(0) : a.m[X][iu] - (T)((ph - (a.phi[i - 1] - mean)) * a.g.dinv_sp[X][x]);
        vf[0] = y == 0 ? T(0) : a.m[Y][iv] - (T)((ph - (a.phi[i - sy] - mean)) * a.g.dinv_sp[Y][y]);
        wf[0] = z == 0 ? T(0) : a.m[Z][iw] - (T)((ph - (a.phi[i - sz] - mean)) * a.g.dinv_sp[Z][z]);
        uf[1] = x == p.nx - 1 ? T(0) : a.m[X][iu + 1] - (T)(((a.phi[i + 1] - mean) - ph) * a.g.dinv_sp[X][x + 1]);
        vf[1] = y == p.ny - 1 ? T(0) : a.m[Y][iv + p.nx] - (T)(((a.phi[i + sy] - mean) - ph) * a.g.dinv_sp[Y][y + 1]);
        wf[1] = z == p.nz - 1 ? T(0) : a.m[Z][iw + sz] - (T)(((a.phi[i + sz] - mean) - ph) * a.g.dinv_sp[Z][z + 1]);
        a.u_out[X][iu] = uf[0];
        a.u_out[Y][iv] = vf[0];
        a.u_out[Z][iw] = wf[0];
        if (x == p.nx - 1) a.u_out[X][iu + 1] = uf[1];
        if (y == p.ny - 1) a.u_out[Y][iv + p.nx] = vf[1];
        if (z == p.nz - 1) a.u_out[Z][iw + sz] = wf[1];
        if (a.last_stage) {
            // CFL rate of the new velocity, as backend.cu:469-471 (divisions kept for identical rounding)
            const T r = fmax(fabs(uf[0]), fabs(uf[1])) / tab(a.g, X, kW, x) +
                        fmax(fabs(vf[0]), fabs(vf[1])) / tab(a.g, Y, kW, y) +
                        fmax(fabs(wf[0]), fabs(wf[1])) / tab(a.g, Z, kW, z);
            acc.v[0] = (double)r;
        }
        a.phi_out[i] = ph;
        if (hb >= 0) a.hist[hb][i] = 1.0 * ph + -1.0 * a.base[i];
    }
    // gridwide: CFL max (NaN wins) and the scalar bookkeeping in the last block
    const Vec<1> blk = block_reduce<1, true>(acc);
    if (publish_partials(blk, a.partial, &c->counter[kCntFinish])) {
        const Vec<1> tot = final_reduce<1, true>(a.partial);
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
