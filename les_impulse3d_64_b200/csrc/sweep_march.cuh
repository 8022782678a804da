// sweep_march.cuh - the momentum sweep as a 2.5D march through z with the Lamb vector built edge by edge.
//
// The Lamb vector of a face sums eight edge terms (vorticity times an interpolated velocity; backend.cu:141-215),
// and every edge is shared: the narrow (q = 1) and the wide (q = 3) term of the edge between an x-face and a
// y-face enter two u-faces (as v interpolated along x) and two v-faces (as u interpolated along y), with the same
// vorticity.  The face-by-face form (sweep_tile.cuh, and the reference's kernels) evaluates each vorticity four
// times.  Here a CTA owns a TX x TY column of cells and walks up a chunk of z-layers; at each layer it first
// evaluates every edge once -
//   z-edges (x-face, y-face) of the layer:     zU (for u-faces) and zV (for v-faces), q = 1 and 3;
//   y-edges (x-face, z-face) of plane e = z+2:   yU (u-faces) and yW (w-faces);
//   x-edges (y-face, z-face) of plane e = z+2:   xV (v-faces) and xW (w-faces);
//   K = u.m of the layer's cells (backend.cu:218-222) -
// and then the three faces of each cell, which add the edge terms in the reference's order (narrow then wide,
// first then second tangential axis; backend.cu:232-272), -grad K, the viscous flux Laplacian with its wall and
// lid fluxes and the RK combination (backend.cu:279-330).  Every term is the same expression, on the same
// operands, as in the face-by-face kernel; only where it is evaluated changes.
//
// Memory: each z-layer of u, v, w and of the three impulse components is staged into shared-memory rings once
// per CTA (cp.async, zero-filled outside the box, issued one layer ahead), with the halos the stencils reach in x
// and y; the z-halos come from the rings, so nothing is re-staged along z.  Edge terms needed by neighbouring
// threads (zU, zV, yW, xW) and K go through shared memory; the yU and xV terms a thread needs only along its own
// column stay in registers, rolled from layer to layer.  Stage 0 blends the impulse m0 = r m + (1-r) u
// (backend.cu:880-881) in shared memory as each layer arrives and stores m0.
#pragma once
#include <type_traits>

#include "sweep_tile.cuh"

namespace cavity {

template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void* smem_dst, const void* src, bool valid) {
    const unsigned int dst = (unsigned int)__cvta_generic_to_shared(smem_dst);
    const int n = valid ? BYTES : 0;
    if (BYTES == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(n));
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(n));
}

template <int TX_, int TY_> struct MarchGeom {
    static constexpr int TX = TX_, TY = TY_, NT = TX * TY;
    // input boxes of one layer: width (x) x height (y), corner relative to the tile's (x0, y0)
    static constexpr int UW = TX + 3, UH = TY + 6;      // u: x-faces x0-1 .. x0+TX+1, cells y0-3 .. y0+TY+2
    static constexpr int VW = TX + 6, VH = TY + 3;      // v: cells x0-3 .. x0+TX+2, y-faces y0-1 .. y0+TY+1
    static constexpr int WW = TX + 6, WH = TY + 6;      // w: cells x0-3 .. x0+TX+2, cells y0-3 .. y0+TY+2
    static constexpr int MW = TX + 2, MH = TY + 2;      // impulse components: x0-1 .., y0-1 ..
    static constexpr int KW = TX + 1, KH = TY + 1;      // K: cells x0-1 .. x0+TX-1, y0-1 .. y0+TY-1
    static constexpr int NU = UW * UH, NV = VW * VH, NW = WW * WH, NM = MW * MH, NK = KW * KH;
    // ring slots: u, v hold layers z .. z+3 and load z+4; w holds z-faces z .. z+2 and loads z+3; the impulse
    // holds z-1 .. z+1 and loads z+2; K holds z-1, z; the w-face edge terms hold planes z .. z+2
    static constexpr int SU = 5, SW = 4, SM = 4, SK = 2, SE = 3;
    static constexpr int NZU = TX * (TY + 3);           // zU1, zU3: x-faces x0 .., y-faces y0-1 .. y0+TY+1
    static constexpr int NZV = (TX + 3) * TY;           // zV1, zV3: x-faces x0-1 .. x0+TX+1, cells y0 ..
    static constexpr int NYW = (TX + 3) * TY;           // yW1, yW3: x-faces x0-1 .. x0+TX+1, cells y0 ..
    static constexpr int NXW = TX * (TY + 3);           // xW1, xW3: cells x0 .., y-faces y0-1 .. y0+TY+1
    static constexpr int OU = 0;
    static constexpr int OV = OU + SU * NU;
    static constexpr int OW = OV + SU * NV;
    static constexpr int OM = OW + SW * NW;             // component c, slot s at OM + (c * SM + s) * NM
    static constexpr int OK = OM + 3 * SM * NM;
    static constexpr int OZU = OK + SK * NK;
    static constexpr int OZV = OZU + 2 * NZU;
    static constexpr int OYW = OZV + 2 * NZV;           // slot s: OYW + s * 2 * NYW (yW1, then yW3)
    static constexpr int OXW = OYW + SE * 2 * NYW;      // slot s: OXW + s * 2 * NXW (xW1, then xW3)
    static constexpr int ELEMS = OXW + SE * 2 * NXW;
    template <class T> static constexpr size_t smem_bytes() { return sizeof(T) * (size_t)ELEMS; }
    // halo tasks of one layer: y-edges at 3 extra x-faces, x-edges at 3 extra y-faces, z-edges (zU at 3 extra
    // y-faces, zV at 3 extra x-faces), K at the cells x0-1 (TY+1 of them) and y0-1 (TX)
    static constexpr int H_YE = 3 * TY, H_XE = 3 * TX, H_ZU = 3 * TX, H_ZV = 3 * TY, H_K = TX + TY + 1;
    static constexpr int HALO = H_YE + H_XE + H_ZU + H_ZV + H_K;
};

__device__ __forceinline__ int ring(int layer, int slots) { return (layer + 60) % slots; }

// Stage one layer (W x H box, corner (xs, ys)) of an array with extents (ex, ey, ez) into shared memory;
// elements outside the array are zero.
template <class T, int W, int H, int NT>
__device__ __forceinline__ void stage_layer(T* dst, const T* __restrict__ src, int xs, int ys, int layer, int ex, int ey,
                                            int ez) {
    const bool zin = layer >= 0 && layer < ez;
    const T* lay = src + (size_t)(zin ? layer : 0) * (size_t)ex * (size_t)ey;
    for (int e = threadIdx.x; e < W * H; e += NT) {
        const int row = e / W, col = e - row * W;
        const int gx = xs + col, gy = ys + row;
        const bool ok = zin && (unsigned)gx < (unsigned)ex && (unsigned)gy < (unsigned)ey;
        cp_async_zfill<sizeof(T)>(dst + e, ok ? lay + gx + (size_t)gy * ex : src, ok);
    }
}

// coefficients of an edge position along one axis (index i of faces along that axis)
template <class T> struct EdgeCoef {
    T ok1, l1, isp, l3, ind3, e1l, e1h, e3l, e3h;
};
template <class T> __device__ __forceinline__ EdgeCoef<T> edge_coef(const Geo<T>& g, int a, int i, int n) {
    const int c = min(max(i, -2), n + 2);
    return {tab(g, a, kOk1, c), tab(g, a, kL1, c), tab(g, a, kInvSp, c), tab(g, a, kL3, c), tab(g, a, kInvNd3, c),
            tab(g, a, kEv1Lo, c), tab(g, a, kEv1Hi, c), tab(g, a, kEv3Lo, c), tab(g, a, kEv3Hi, c)};
}

// stencil weights of an edge (the same expressions as the face-by-face kernels)
template <class T> __device__ __forceinline__ T march_w1(int o4, T okA, T okB, T lA, T lB) {
    return o4 ? okA * okB * (T(1) + (lA * lB) * T(0.125)) : okA * okB;
}
template <class T> __device__ __forceinline__ T march_w3(T lA, T lB) { return -((lA * lB) * T(0.125)); }

// edge terms: [0] narrow, [1] wide, for the two face families the edge feeds
template <class T> struct EdgeTerms {
    T f1, f3;      // first family (zU, yU, xV)
    T g1, g3;      // second family (zV, yW, xW)
};

// Shared-memory layout and rings of one CTA
template <class T, class G> struct MarchSmem {
    T* base;
    __device__ __forceinline__ T* u(int layer) const { return base + G::OU + ring(layer, G::SU) * G::NU; }
    __device__ __forceinline__ T* v(int layer) const { return base + G::OV + ring(layer, G::SU) * G::NV; }
    __device__ __forceinline__ T* w(int face) const { return base + G::OW + ring(face, G::SW) * G::NW; }
    __device__ __forceinline__ T* m(int c, int layer) const { return base + G::OM + (c * G::SM + ring(layer, G::SM)) * G::NM; }
    __device__ __forceinline__ T* k(int layer) const { return base + G::OK + ring(layer, G::SK) * G::NK; }
    __device__ __forceinline__ T* zu1() const { return base + G::OZU; }
    __device__ __forceinline__ T* zu3() const { return base + G::OZU + G::NZU; }
    __device__ __forceinline__ T* zv1() const { return base + G::OZV; }
    __device__ __forceinline__ T* zv3() const { return base + G::OZV + G::NZV; }
    __device__ __forceinline__ T* yw(int face) const { return base + G::OYW + ring(face, G::SE) * 2 * G::NYW; }
    __device__ __forceinline__ T* xw(int face) const { return base + G::OXW + ring(face, G::SE) * 2 * G::NXW; }
};

template <class T, int TX, int TY>
__device__ void sweep_march_body(const MomentumArgs<T>& a, const Blk& blk) {
    using G = MarchGeom<TX, TY>;
    constexpr int NT = G::NT, UW = G::UW, VW = G::VW, WW = G::WW, MW = G::MW, KW = G::KW;
    pdl_launch_dependents();
    pdl_wait();
    if (a.c->error) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const MarchSmem<T, G> S{reinterpret_cast<T*>(smem_raw)};
    const Params& p = a.p;
    const Geo<T>& g = a.g;
    const int nx = p.nx, ny = p.ny, nz = p.nz, o4 = p.o4;
    const int x0 = (int)blk.x * TX, y0 = (int)blk.y * TY;
    const int zc = (nz + (int)blk.nz - 1) / (int)blk.nz;
    const int z0 = (int)blk.z * zc, z1 = min(nz, z0 + zc);
    if (z0 >= z1) return;
    const bool blend = a.stage == 0;
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    const int x = x0 + tx, y = y0 + ty;
    const bool live = x < nx && y < ny;

    // ---- staging of the layers one iteration needs next: u, v (layer j+4), w (z-face j+3), impulse (j+2)
    auto stage_uv = [&](int l) {
        stage_layer<T, G::UW, G::UH, NT>(S.u(l), a.u[X], x0 - 1, y0 - 3, l, nx + 1, ny, nz);
        stage_layer<T, G::VW, G::VH, NT>(S.v(l), a.u[Y], x0 - 3, y0 - 1, l, nx, ny + 1, nz);
    };
    auto stage_w = [&](int l) { stage_layer<T, G::WW, G::WH, NT>(S.w(l), a.u[Z], x0 - 3, y0 - 3, l, nx, ny, nz + 1); };
    auto stage_m = [&](int l) {
        stage_layer<T, G::MW, G::MH, NT>(S.m(X, l), a.m[X], x0 - 1, y0 - 1, l, nx + 1, ny, nz);
        stage_layer<T, G::MW, G::MH, NT>(S.m(Y, l), a.m[Y], x0 - 1, y0 - 1, l, nx, ny + 1, nz);
        stage_layer<T, G::MW, G::MH, NT>(S.m(Z, l), a.m[Z], x0 - 1, y0 - 1, l, nx, ny, nz + 1);
    };
    // the gauge-reset blend of a staged impulse layer (stage 0), in place, from the staged velocity
    auto blend_m = [&](int l) {
        T* mu = S.m(X, l);
        T* mv = S.m(Y, l);
        T* mw = S.m(Z, l);
        const T* su = S.u(l);
        const T* sv = S.v(l);
        const T* sw = S.w(l);
        for (int e = threadIdx.x; e < G::NM; e += NT) {
            const int row = e / MW, col = e - row * MW;
            mu[e] = a.r * mu[e] + a.one_minus_r * su[(row + 2) * UW + col];
            mv[e] = a.r * mv[e] + a.one_minus_r * sv[row * VW + col + 2];
            mw[e] = a.r * mw[e] + a.one_minus_r * sw[(row + 2) * WW + col + 2];
        }
    };

    // ---- edges.  Smem views: U(a, b) of layer l at (b - y0 + 3) * UW + a - x0 + 1; V(a, b) at
    // (b - y0 + 1) * VW + a - x0 + 3; W(a, b) at (b - y0 + 3) * WW + a - x0 + 3.
    const T half = T(0.5);
    // z-edge (x-face ea, y-face eb) of layer l: f = zU, g = zV (backend.cu:141-146, 177-194)
    auto z_edge = [&](int ea, int eb, int l, const EdgeCoef<T>& cx, const EdgeCoef<T>& cy) {
        const T* su = S.u(l) + (eb - y0 + 3) * UW + ea - x0 + 1;
        const T* sv = S.v(l) + (eb - y0 + 1) * VW + ea - x0 + 3;
        EdgeTerms<T> r;
        {
            const T vl = sv[-1], vh = sv[0], ul = su[-UW], uh = su[0];
            const T wo = march_w1<T>(o4, cx.ok1, cy.ok1, cx.l1, cy.l1) * ((vh - vl) * cx.isp - (uh - ul) * cy.isp);
            r.f1 = wo * (cx.e1l * vl + cx.e1h * vh);
            r.g1 = -(wo * (cy.e1l * ul + cy.e1h * uh));
        }
        if (o4) {
            const T vl = sv[-2], vh = sv[1], ul = su[-2 * UW], uh = su[UW];
            const T wo = march_w3<T>(cx.l3, cy.l3) * ((vh - vl) * cx.ind3 - (uh - ul) * cy.ind3);
            r.f3 = wo * (cx.e3l * vl + cx.e3h * vh);
            r.g3 = -(wo * (cy.e3l * ul + cy.e3h * uh));
        } else {
            r.f3 = r.g3 = T(0);
        }
        return r;
    };
    // y-edge (x-face ea, cell cy, z-face e): f = yU, g = yW (backend.cu:153-158, 201-214)
    auto y_edge = [&](int ea, int cyy, int e, const EdgeCoef<T>& cx, const EdgeCoef<T>& cz) {
        const int ou = (cyy - y0 + 3) * UW + ea - x0 + 1;
        const T* sw = S.w(e) + (cyy - y0 + 3) * WW + ea - x0 + 3;
        EdgeTerms<T> r;
        {
            const T ul = S.u(e - 1)[ou], uh = S.u(e)[ou], wl = sw[-1], wh = sw[0];
            const T wo = march_w1<T>(o4, cz.ok1, cx.ok1, cz.l1, cx.l1) * ((uh - ul) * cz.isp - (wh - wl) * cx.isp);
            r.f1 = -(wo * (cx.e1l * wl + cx.e1h * wh));
            r.g1 = wo * (cz.e1l * ul + cz.e1h * uh);
        }
        if (o4) {
            const T ul = S.u(e - 2)[ou], uh = S.u(e + 1)[ou], wl = sw[-2], wh = sw[1];
            const T wo = march_w3<T>(cz.l3, cx.l3) * ((uh - ul) * cz.ind3 - (wh - wl) * cx.ind3);
            r.f3 = -(wo * (cx.e3l * wl + cx.e3h * wh));
            r.g3 = wo * (cz.e3l * ul + cz.e3h * uh);
        } else {
            r.f3 = r.g3 = T(0);
        }
        return r;
    };
    // x-edge (cell cx, y-face eb, z-face e): f = xV, g = xW (backend.cu:147-152, 195-200)
    auto x_edge = [&](int cxx, int eb, int e, const EdgeCoef<T>& cy, const EdgeCoef<T>& cz) {
        const int ov = (eb - y0 + 1) * VW + cxx - x0 + 3;
        const T* sw = S.w(e) + (eb - y0 + 3) * WW + cxx - x0 + 3;
        EdgeTerms<T> r;
        {
            const T wl = sw[-WW], wh = sw[0], vl = S.v(e - 1)[ov], vh = S.v(e)[ov];
            const T wo = march_w1<T>(o4, cy.ok1, cz.ok1, cy.l1, cz.l1) * ((wh - wl) * cy.isp - (vh - vl) * cz.isp);
            r.f1 = wo * (cy.e1l * wl + cy.e1h * wh);
            r.g1 = -(wo * (cz.e1l * vl + cz.e1h * vh));
        }
        if (o4) {
            const T wl = sw[-2 * WW], wh = sw[WW], vl = S.v(e - 2)[ov], vh = S.v(e + 1)[ov];
            const T wo = march_w3<T>(cy.l3, cz.l3) * ((wh - wl) * cy.ind3 - (vh - vl) * cz.ind3);
            r.f3 = wo * (cy.e3l * wl + cy.e3h * wh);
            r.g3 = -(wo * (cz.e3l * vl + cz.e3h * vh));
        } else {
            r.f3 = r.g3 = T(0);
        }
        return r;
    };
    // K = u.m of cell (cx, cy) in layer l (cx >= x0-1, cy >= y0-1)
    auto k_cell = [&](int cx, int cy, int l) {
        const T* su = S.u(l) + (cy - y0 + 3) * UW + cx - x0 + 1;
        const T* sv = S.v(l) + (cy - y0 + 1) * VW + cx - x0 + 3;
        const int ow = (cy - y0 + 3) * WW + cx - x0 + 3;
        const int om = (cy - y0 + 1) * MW + cx - x0 + 1;
        const T* mx = S.m(X, l) + om;
        const T* my = S.m(Y, l) + om;
        return half * ((su[0] * mx[0] + su[1] * mx[1]) + (sv[0] * my[0] + sv[VW] * my[MW]) +
                       (S.w(l)[ow] * S.m(Z, l)[om] + S.w(l + 1)[ow] * S.m(Z, l + 1)[om]));
    };

    // ---- the march.  Iteration j computes the y- and x-edges of z-face plane j+2 and, once j reaches the chunk,
    // K of layer j (from j = z0-1), the z-edges of layer j and the faces of layer j.
    for (int l = z0 - 3; l <= z0; l++) stage_uv(l);
    for (int l = z0 - 3; l <= z0 - 1; l++) stage_w(l);
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();

    // the yU / xV terms of this thread's own column along z: [0] plane j-1, [1] j, [2] j+1 (after the shift)
    T yu1_0 = T(0), yu1_1 = T(0), yu3_m1 = T(0), yu3_0 = T(0), yu3_1 = T(0);
    T xv1_0 = T(0), xv1_1 = T(0), xv3_m1 = T(0), xv3_0 = T(0), xv3_1 = T(0);
    // this thread's own x-face x and y-face y coefficients stay in registers for the whole march
    const EdgeCoef<T> cx_own = edge_coef(g, X, x, nx), cy_own = edge_coef(g, Y, y, ny);
    const StageConst sc = stage_const(a.stage, a.c);
    const T dt = (T)a.c->dt;
    const T lidv = (T)lid_speed(p, sc.tau);

#pragma unroll 1
    for (int j = z0 - 3; j < z1; j++) {
        if (j + 1 < z1) {
            stage_uv(j + 4);
            stage_w(j + 3);
            stage_m(j + 2);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        if (blend && j + 1 >= z0 - 1) {
            blend_m(j + 1);          // arrived at the end of the previous iteration
            __syncthreads();
        }
        const int e = j + 2;
        const EdgeCoef<T> cz_e = edge_coef(g, Z, e, nz);
        // phase A: own edges, then the halo tasks
        const EdgeTerms<T> ye = y_edge(x, y, e, cx_own, cz_e);
        const EdgeTerms<T> xe = x_edge(x, y, e, cy_own, cz_e);
        S.yw(e)[ty * (TX + 3) + tx + 1] = ye.g1;
        S.yw(e)[G::NYW + ty * (TX + 3) + tx + 1] = ye.g3;
        S.xw(e)[(ty + 1) * TX + tx] = xe.g1;
        S.xw(e)[G::NXW + (ty + 1) * TX + tx] = xe.g3;
        const bool faces = j >= z0;
        if (faces) {
            const EdgeTerms<T> ze = z_edge(x, y, j, cx_own, cy_own);
            S.zu1()[(ty + 1) * TX + tx] = ze.f1;
            S.zu3()[(ty + 1) * TX + tx] = ze.f3;
            S.zv1()[ty * (TX + 3) + tx + 1] = ze.g1;
            S.zv3()[ty * (TX + 3) + tx + 1] = ze.g3;
        }
        if (j >= z0 - 1) S.k(j)[(ty + 1) * KW + tx + 1] = k_cell(x, y, j);
        for (int t = threadIdx.x; t < G::HALO; t += NT) {
            int r = t;
            if (r < G::H_YE) {                       // y-edges at x-faces x0-1, x0+TX, x0+TX+1
                const int c = r / TY, cy = y0 + r % TY;
                const int col = c == 0 ? 0 : TX + c;     // box column (x-face x0-1+col)
                const EdgeTerms<T> h = y_edge(x0 - 1 + col, cy, e, edge_coef(g, X, x0 - 1 + col, nx), cz_e);
                S.yw(e)[(cy - y0) * (TX + 3) + col] = h.g1;
                S.yw(e)[G::NYW + (cy - y0) * (TX + 3) + col] = h.g3;
                continue;
            }
            r -= G::H_YE;
            if (r < G::H_XE) {                       // x-edges at y-faces y0-1, y0+TY, y0+TY+1
                const int c = r / TX, cx = x0 + r % TX;
                const int row = c == 0 ? 0 : TY + c;
                const EdgeTerms<T> h = x_edge(cx, y0 - 1 + row, e, edge_coef(g, Y, y0 - 1 + row, ny), cz_e);
                S.xw(e)[row * TX + cx - x0] = h.g1;
                S.xw(e)[G::NXW + row * TX + cx - x0] = h.g3;
                continue;
            }
            r -= G::H_XE;
            if (r < G::H_ZU) {                       // zU at y-faces y0-1, y0+TY, y0+TY+1
                if (!faces) continue;
                const int c = r / TX, cx = x0 + r % TX;
                const int row = c == 0 ? 0 : TY + c;
                const EdgeTerms<T> h = z_edge(cx, y0 - 1 + row, j, edge_coef(g, X, cx, nx), edge_coef(g, Y, y0 - 1 + row, ny));
                S.zu1()[row * TX + cx - x0] = h.f1;
                S.zu3()[row * TX + cx - x0] = h.f3;
                continue;
            }
            r -= G::H_ZU;
            if (r < G::H_ZV) {                       // zV at x-faces x0-1, x0+TX, x0+TX+1
                if (!faces) continue;
                const int c = r / TY, cy = y0 + r % TY;
                const int col = c == 0 ? 0 : TX + c;
                const EdgeTerms<T> h = z_edge(x0 - 1 + col, cy, j, edge_coef(g, X, x0 - 1 + col, nx), edge_coef(g, Y, cy, ny));
                S.zv1()[(cy - y0) * (TX + 3) + col] = h.g1;
                S.zv3()[(cy - y0) * (TX + 3) + col] = h.g3;
                continue;
            }
            r -= G::H_ZV;
            if (j < z0 - 1) continue;                // K at the cells x0-1 (rows y0-1 ..) and y0-1 (x0 ..)
            const int cx = r <= TY ? x0 - 1 : x0 + (r - TY - 1);
            const int cy = r <= TY ? y0 - 1 + r : y0 - 1;
            S.k(j)[(cy - y0 + 1) * KW + cx - x0 + 1] = k_cell(cx, cy, j);
        }
        __syncthreads();

        // phase B: the faces of layer j
        if (faces && live) {
            const int z = j;
            const T* kc = S.k(j) + (ty + 1) * KW + tx + 1;
            const int om = (ty + 1) * MW + tx + 1;
            const T* zu1 = S.zu1() + (ty + 1) * TX + tx;
            const T* zu3 = S.zu3() + (ty + 1) * TX + tx;
            const T* zv1 = S.zv1() + ty * (TX + 3) + tx + 1;
            const T* zv3 = S.zv3() + ty * (TX + 3) + tx + 1;
            // viscous flux-form Laplacian of component A at (x, y, z) with wall and lid fluxes, then the RK
            // combination (the expressions of viscous_rk_tile, backend.cu:289-329)
            auto finish = [&](auto Acomp, T L, T wall) {
                constexpr int A = decltype(Acomp)::value;
                const T* mc = S.m(A, z) + om;
                const T cc = mc[0];
                const T mnb[3][2] = {{mc[-1], mc[1]}, {mc[-MW], mc[MW]}, {S.m(A, z - 1)[om], S.m(A, z + 1)[om]}};
                const int q[3] = {x, y, z};
                const int n[3] = {nx, ny, nz};
                T lap = T(0);
#pragma unroll
                for (int t = 0; t < 3; t++) {
                    const T lo_v = mnb[t][0], hi_v = mnb[t][1];
                    if (t == A) {
                        lap = lap + ((hi_v - cc) * tab(g, t, kInvW, q[t]) - (cc - lo_v) * tab(g, t, kInvW, q[t] - 1)) *
                                        tab(g, t, kInvSp, q[t]);
                        continue;
                    }
                    T hi = q[t] < n[t] - 1 ? (hi_v - cc) * tab(g, t, kInvSp, q[t] + 1) : T(0);
                    T lo = q[t] > 0 ? (cc - lo_v) * tab(g, t, kInvSp, q[t]) : T(0);
                    if (q[t] == 0) lo = wall * tab(g, t, kInvSp, 0);
                    if (q[t] == n[t] - 1) {
                        if (t == Y) {
                            const T U = A == X ? lidv * g.lid_u[x + (nx + 1) * z] : T(0);
                            hi = (U - wall) * tab(g, Y, kInvSp, n[Y]);
                        } else {
                            hi = -wall * tab(g, t, kInvSp, n[t]);
                        }
                    }
                    lap = lap + (hi - lo) * tab(g, t, kInvW, q[t]);
                }
                const int i = fidx<A>(p, x, y, z);
                T val = cc + dt * (a.nu * lap + L);
                if (a.stage > 0) val = T(sc.a0) * a.m0[A][i] + T(sc.b) * val;
                a.out[A][i] = val;
            };
            // u-face x
            {
                const int i = fidx<X>(p, x, y, z);
                if (blend) a.m0_out[X][i] = S.m(X, z)[om];
                if (x == 0) a.out[X][i] = T(0);
                else {
                    T L = half * (zu1[TX] + zu1[0]) + half * (yu1_1 + yu1_0);
                    if (o4) {
                        const T c3 = tab(g, X, kC3, x);
                        L = L + c3 * (zu3[2 * TX] + zu3[-TX]);
                        L = L + c3 * (ye.f3 + yu3_m1);
                    }
                    L = L - (kc[0] - kc[-1]) * tab(g, X, kInvSp, x);
                    finish(std::integral_constant<int, X>{}, L, S.u(z)[(ty + 3) * UW + tx + 1]);
                }
                if (x == nx - 1) {
                    if (blend) a.m0_out[X][i + 1] = S.m(X, z)[om + 1];
                    a.out[X][i + 1] = T(0);
                }
            }
            // v-face y
            {
                const int i = fidx<Y>(p, x, y, z);
                if (blend) a.m0_out[Y][i] = S.m(Y, z)[om];
                if (y == 0) a.out[Y][i] = T(0);
                else {
                    T L = half * (zv1[1] + zv1[0]) + half * (xv1_1 + xv1_0);
                    if (o4) {
                        const T c3 = tab(g, Y, kC3, y);
                        L = L + c3 * (zv3[2] + zv3[-1]);
                        L = L + c3 * (xe.f3 + xv3_m1);
                    }
                    L = L - (kc[0] - kc[-KW]) * tab(g, Y, kInvSp, y);
                    finish(std::integral_constant<int, Y>{}, L, S.v(z)[(ty + 1) * VW + tx + 3]);
                }
                if (y == ny - 1) {
                    if (blend) a.m0_out[Y][i + nx] = S.m(Y, z)[om + MW];
                    a.out[Y][i + nx] = T(0);
                }
            }
            // w-face z
            {
                const int i = fidx<Z>(p, x, y, z);
                if (blend) a.m0_out[Z][i] = S.m(Z, z)[om];
                if (z == 0) a.out[Z][i] = T(0);
                else {
                    const T* xw1 = S.xw(z) + (ty + 1) * TX + tx;
                    const T* xw3 = xw1 + G::NXW;
                    const T* yw1 = S.yw(z) + ty * (TX + 3) + tx + 1;
                    const T* yw3 = yw1 + G::NYW;
                    T L = half * (xw1[TX] + xw1[0]) + half * (yw1[1] + yw1[0]);
                    if (o4) {
                        const T c3 = tab(g, Z, kC3, z);
                        L = L + c3 * (xw3[2 * TX] + xw3[-TX]);
                        L = L + c3 * (yw3[2] + yw3[-1]);
                    }
                    L = L - (kc[0] - S.k(z - 1)[(ty + 1) * KW + tx + 1]) * tab(g, Z, kInvSp, z);
                    finish(std::integral_constant<int, Z>{}, L, S.w(z)[(ty + 3) * WW + tx + 3]);
                }
                if (z == nz - 1) {
                    if (blend) a.m0_out[Z][i + nx * ny] = S.m(Z, z + 1)[om];
                    a.out[Z][i + nx * ny] = T(0);
                }
            }
        }
        // roll this column's y- and x-edge terms one plane up
        yu1_0 = yu1_1; yu1_1 = ye.f1;
        yu3_m1 = yu3_0; yu3_0 = yu3_1; yu3_1 = ye.f3;
        xv1_0 = xv1_1; xv1_1 = xe.f1;
        xv3_m1 = xv3_0; xv3_0 = xv3_1; xv3_1 = xe.f3;
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();
    }
}

template <class T, int TX, int TY>
__global__ void __launch_bounds__(TX * TY, sizeof(T) == 4 ? 3 : 1) sweep_march_kernel(MomentumArgs<T> a) {
    sweep_march_body<T, TX, TY>(a, real_blk());
}
// a batch of cavities: grid x runs over the work list (BatchItem)
template <class T, int TX, int TY>
__global__ void __launch_bounds__(TX * TY, sizeof(T) == 4 ? 3 : 1)
    sweep_march_batched(const MomentumArgs<T>* args, const BatchItem* items, const int* live) {
    __shared__ MomentumArgs<T> a;
    int cav;
    const Blk k = item_blk(items, live, cav);
    if (cav < 0) return;
    load_args(a, args + cav);
    sweep_march_body<T, TX, TY>(a, k);
}

}  // namespace cavity
