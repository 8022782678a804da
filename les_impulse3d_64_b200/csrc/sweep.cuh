// sweep.cuh - the momentum sweep: one RK3 stage of the impulse for every face (u, v and w in one launch).
//
// One thread per face computes the inviscid term I = Lamb vector - grad(u.m) (backend.cu:102-274) and fuses it
// with the viscous flux-form Laplacian, the wall and lid fluxes and the RK combination (backend.cu:279-330).
// Stage 0 also performs the gauge reset m0 = r m + (1-r) u (backend.cu:880-881) on the fly and stores m0.
// The neighbour values come through L1 (no shared-memory tile): with 40 registers a thread, eight CTAs of
// 256 threads fit an SM and hide the load latency; the coefficients come from the per-axis tables.
#pragma once
#include "kernels.cuh"

namespace cavity {

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

}  // namespace cavity
