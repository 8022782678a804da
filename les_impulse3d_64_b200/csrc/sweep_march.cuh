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

// Stage rows of one layer of an array with extents (ex, ey, ez) into a W x H box (corner xs, ys) in shared memory,
// a warp per row (rows warp, warp + WARPS, ...) and a lane per column (lane, lane + 32; W <= 64); elements outside
// the array are zero.
template <class T, int W, int H, int WARPS>
__device__ __forceinline__ void stage_rows(T* dst, const T* __restrict__ src, int xs, int ys, int layer, int ex, int ey,
                                           int ez, int lane, int warp) {
    static_assert(W <= 64, "two columns per lane");
    const bool zin = layer >= 0 && layer < ez;
    const T* lay = src + (zin ? (size_t)layer * (size_t)ex * (size_t)ey : (size_t)0);
    const int gx0 = xs + lane, gx1 = xs + lane + 32;
    const bool ok0 = zin && (unsigned)gx0 < (unsigned)ex;
    const bool ok1 = lane + 32 < W && zin && (unsigned)gx1 < (unsigned)ex;
    for (int r = warp; r < H; r += WARPS) {
        const int gy = ys + r;
        const bool yok = (unsigned)gy < (unsigned)ey;
        const T* row = lay + (size_t)(yok ? gy : 0) * (size_t)ex;
        T* d = dst + r * W;
        cp_async_zfill<sizeof(T)>(d + lane, ok0 && yok ? row + gx0 : src, ok0 && yok);
        if (lane + 32 < W) cp_async_zfill<sizeof(T)>(d + lane + 32, ok1 && yok ? row + gx1 : src, ok1 && yok);
    }
}

__device__ __forceinline__ int wrap(int v, int slots) { return v >= slots ? v - slots : v; }

// the face coefficients of one axis at index i: 1/width at i and i-1, 1/spacing at i and i+1, the wide-stencil
// weight at i (the viscous flux Laplacian's and the Lamb sum's tables)
template <class T> struct FaceCoef {
    T iw0, iwm, is0, is1, c3;
};
template <class T> __device__ __forceinline__ FaceCoef<T> face_coef(const Geo<T>& g, int a, int i, int n) {
    const int c = min(max(i, -1), n + 1);
    return {tab(g, a, kInvW, c), tab(g, a, kInvW, c - 1), tab(g, a, kInvSp, c), tab(g, a, kInvSp, c + 1), tab(g, a, kC3, c)};
}

template <class T, int TX, int TY>
__device__ void sweep_march_body(const MomentumArgs<T>& a, const Blk& blk) {
    static_assert(TX == 32 && TY == 8, "a warp per row of a 32 x 8 column block; the halo tasks are laid out for 8 warps");
    using G = MarchGeom<TX, TY>;
    constexpr int UW = G::UW, VW = G::VW, WW = G::WW, MW = G::MW, KW = G::KW, EW = TX + 3;
    pdl_launch_dependents();
    pdl_wait();
    if (a.c->error) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* const base = reinterpret_cast<T*>(smem_raw);
    const Params& p = a.p;
    const Geo<T>& g = a.g;
    const int nx = p.nx, ny = p.ny, nz = p.nz, o4 = p.o4;
    const int x0 = (int)blk.x * TX, y0 = (int)blk.y * TY;
    const int zc = (nz + (int)blk.nz - 1) / (int)blk.nz;
    const int z0 = (int)blk.z * zc, z1 = min(nz, z0 + zc);
    if (z0 >= z1) return;
    const bool blend = a.stage == 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = x0 + lane, y = y0 + warp;
    const bool live = x < nx && y < ny;
    const T half = T(0.5);

    // ring slots (see MarchGeom): offsets of layer/face j + k given the slot of j
    auto U = [&](int su, int k) { return base + G::OU + wrap(su + k, G::SU) * G::NU; };
    auto V = [&](int su, int k) { return base + G::OV + wrap(su + k, G::SU) * G::NV; };
    auto Wf = [&](int sw, int k) { return base + G::OW + wrap(sw + k, G::SW) * G::NW; };
    auto M = [&](int c, int sm, int k) { return base + G::OM + (c * G::SM + wrap(sm + k, G::SM)) * G::NM; };
    auto stage = [&](int su, int sw, int sm, int lu, int lw, int lm, bool uv, bool w, bool m) {
        if (uv) {
            stage_rows<T, G::UW, G::UH, TY>(U(su, 0), a.u[X], x0 - 1, y0 - 3, lu, nx + 1, ny, nz, lane, warp);
            stage_rows<T, G::VW, G::VH, TY>(V(su, 0), a.u[Y], x0 - 3, y0 - 1, lu, nx, ny + 1, nz, lane, warp);
        }
        if (w) stage_rows<T, G::WW, G::WH, TY>(Wf(sw, 0), a.u[Z], x0 - 3, y0 - 3, lw, nx, ny, nz + 1, lane, warp);
        if (m) {
            stage_rows<T, G::MW, G::MH, TY>(M(X, sm, 0), a.m[X], x0 - 1, y0 - 1, lm, nx + 1, ny, nz, lane, warp);
            stage_rows<T, G::MW, G::MH, TY>(M(Y, sm, 0), a.m[Y], x0 - 1, y0 - 1, lm, nx, ny + 1, nz, lane, warp);
            stage_rows<T, G::MW, G::MH, TY>(M(Z, sm, 0), a.m[Z], x0 - 1, y0 - 1, lm, nx, ny, nz + 1, lane, warp);
        }
    };

    // ---- edges, from the staged boxes: U(a, b) at (b - y0 + 3) * UW + a - x0 + 1; V(a, b) at
    // (b - y0 + 1) * VW + a - x0 + 3; W(a, b) at (b - y0 + 3) * WW + a - x0 + 3.
    // z-edge (x-face ea, y-face eb) of the layer in su0/sv0: f = zU, g = zV (backend.cu:141-146, 177-194)
    auto z_edge = [&](const T* ul, const T* vl_, int ea, int eb, const EdgeCoef<T>& cx, const EdgeCoef<T>& cy) {
        const T* su = ul + (eb - y0 + 3) * UW + ea - x0 + 1;
        const T* sv = vl_ + (eb - y0 + 1) * VW + ea - x0 + 3;
        EdgeTerms<T> r;
        {
            const T vl = sv[-1], vh = sv[0], ul1 = su[-UW], uh = su[0];
            const T wo = march_w1<T>(o4, cx.ok1, cy.ok1, cx.l1, cy.l1) * ((vh - vl) * cx.isp - (uh - ul1) * cy.isp);
            r.f1 = wo * (cx.e1l * vl + cx.e1h * vh);
            r.g1 = -(wo * (cy.e1l * ul1 + cy.e1h * uh));
        }
        if (o4) {
            const T vl = sv[-2], vh = sv[1], ul3 = su[-2 * UW], uh = su[UW];
            const T wo = march_w3<T>(cx.l3, cy.l3) * ((vh - vl) * cx.ind3 - (uh - ul3) * cy.ind3);
            r.f3 = wo * (cx.e3l * vl + cx.e3h * vh);
            r.g3 = -(wo * (cy.e3l * ul3 + cy.e3h * uh));
        } else {
            r.f3 = r.g3 = T(0);
        }
        return r;
    };
    // y-edge (x-face ea, cell cyy) of z-face plane e: u of layers e-2 .. e+1 in u4[0..3], w of plane e in
    // wp: f = yU, g = yW (backend.cu:153-158, 201-214)
    auto y_edge = [&](const T* const u4[4], const T* wp, int ea, int cyy, const EdgeCoef<T>& cx, const EdgeCoef<T>& cz) {
        const int ou = (cyy - y0 + 3) * UW + ea - x0 + 1;
        const T* sw = wp + (cyy - y0 + 3) * WW + ea - x0 + 3;
        EdgeTerms<T> r;
        {
            const T ul = u4[1][ou], uh = u4[2][ou], wl = sw[-1], wh = sw[0];
            const T wo = march_w1<T>(o4, cz.ok1, cx.ok1, cz.l1, cx.l1) * ((uh - ul) * cz.isp - (wh - wl) * cx.isp);
            r.f1 = -(wo * (cx.e1l * wl + cx.e1h * wh));
            r.g1 = wo * (cz.e1l * ul + cz.e1h * uh);
        }
        if (o4) {
            const T ul = u4[0][ou], uh = u4[3][ou], wl = sw[-2], wh = sw[1];
            const T wo = march_w3<T>(cz.l3, cx.l3) * ((uh - ul) * cz.ind3 - (wh - wl) * cx.ind3);
            r.f3 = -(wo * (cx.e3l * wl + cx.e3h * wh));
            r.g3 = wo * (cz.e3l * ul + cz.e3h * uh);
        } else {
            r.f3 = r.g3 = T(0);
        }
        return r;
    };
    // x-edge (cell cxx, y-face eb) of z-face plane e: v of layers e-2 .. e+1 in v4[0..3]: f = xV, g = xW
    // (backend.cu:147-152, 195-200)
    auto x_edge = [&](const T* const v4[4], const T* wp, int cxx, int eb, const EdgeCoef<T>& cy, const EdgeCoef<T>& cz) {
        const int ov = (eb - y0 + 1) * VW + cxx - x0 + 3;
        const T* sw = wp + (eb - y0 + 3) * WW + cxx - x0 + 3;
        EdgeTerms<T> r;
        {
            const T wl = sw[-WW], wh = sw[0], vl = v4[1][ov], vh = v4[2][ov];
            const T wo = march_w1<T>(o4, cy.ok1, cz.ok1, cy.l1, cz.l1) * ((wh - wl) * cy.isp - (vh - vl) * cz.isp);
            r.f1 = wo * (cy.e1l * wl + cy.e1h * wh);
            r.g1 = -(wo * (cz.e1l * vl + cz.e1h * vh));
        }
        if (o4) {
            const T wl = sw[-2 * WW], wh = sw[WW], vl = v4[0][ov], vh = v4[3][ov];
            const T wo = march_w3<T>(cy.l3, cz.l3) * ((wh - wl) * cy.ind3 - (vh - vl) * cz.ind3);
            r.f3 = wo * (cy.e3l * wl + cy.e3h * wh);
            r.g3 = -(wo * (cz.e3l * vl + cz.e3h * vh));
        } else {
            r.f3 = r.g3 = T(0);
        }
        return r;
    };
    // K = u.m of cell (cx, cy) of a layer (u, v boxes ul, vl; w boxes of its two z-faces; impulse boxes)
    auto k_cell = [&](const T* ul, const T* vl, const T* w0, const T* w1, const T* mx, const T* my, const T* mz0,
                      const T* mz1, int cx, int cy) {
        const T* su = ul + (cy - y0 + 3) * UW + cx - x0 + 1;
        const T* sv = vl + (cy - y0 + 1) * VW + cx - x0 + 3;
        const int ow = (cy - y0 + 3) * WW + cx - x0 + 3;
        const int om = (cy - y0 + 1) * MW + cx - x0 + 1;
        return half * ((su[0] * mx[om] + su[1] * mx[om + 1]) + (sv[0] * my[om] + sv[VW] * my[om + MW]) +
                       (w0[ow] * mz0[om] + w1[ow] * mz1[om]));
    };

    // ---- this thread's coefficients: its x-face x and y-face y for the edges, and its faces' tables
    const EdgeCoef<T> cxo = edge_coef(g, X, x, nx), cyo = edge_coef(g, Y, y, ny);
    const FaceCoef<T> fx = face_coef(g, X, x, nx), fy = face_coef(g, Y, y, ny);
    const StageConst sc = stage_const(a.stage, a.c);
    const T dt = (T)a.c->dt;
    const T lidv = (T)lid_speed(p, sc.tau);
    const T a0 = T(sc.a0), b0 = T(sc.b), nu = a.nu;

    // ---- the march.  Iteration j computes the y- and x-edges of z-face plane j+2 and, once j reaches the chunk,
    // K of layer j (from j = z0-1), the z-edges of layer j and the faces of layer j.  Before the first: u, v of
    // layers z0-3 .. z0 and w of z-faces z0-3 .. z0-1.
    {
        const int su = ring(z0 - 3, G::SU), sw = ring(z0 - 3, G::SW);
        for (int k = 0; k < 4; k++) stage(wrap(su + k, G::SU), 0, 0, z0 - 3 + k, 0, 0, true, false, false);
        for (int k = 0; k < 3; k++) stage(0, wrap(sw + k, G::SW), 0, 0, z0 - 3 + k, 0, false, true, false);
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();

    // the yU / xV terms of this thread's own column along z (planes j, j+1; wide: j-1 .. j+1)
    T yu1_0 = T(0), yu1_1 = T(0), yu3_m1 = T(0), yu3_0 = T(0), yu3_1 = T(0);
    T xv1_0 = T(0), xv1_1 = T(0), xv3_m1 = T(0), xv3_0 = T(0), xv3_1 = T(0);

#pragma unroll 1
    for (int j = z0 - 3; j < z1; j++) {
        const int su = ring(j, G::SU), sw = ring(j, G::SW), sm = ring(j - 1, G::SM), se = ring(j, G::SE);
        const int sk = ring(j, G::SK);
        if (j + 1 < z1) stage(wrap(su + 4, G::SU), wrap(sw + 3, G::SW), wrap(sm + 3, G::SM), j + 4, j + 3, j + 2, true, true,
                              true);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        const T* const u4[4] = {U(su, 0), U(su, 1), U(su, 2), U(su, 3)};
        const T* const v4[4] = {V(su, 0), V(su, 1), V(su, 2), V(su, 3)};
        const T* const w0 = Wf(sw, 0);             // z-face j
        const T* const w1 = Wf(sw, 1);             // z-face j+1
        const T* const w2 = Wf(sw, 2);             // z-face j+2 (this iteration's edge plane)
        T* const mnext[3] = {M(X, sm, 2), M(Y, sm, 2), M(Z, sm, 2)};     // layer (z-face) j+1
        if (blend && j + 1 >= z0 - 1) {
            // the gauge-reset blend of the impulse layer j+1 that arrived last iteration, from u, v, w of j+1
            for (int r = warp; r < G::MH; r += TY) {
                for (int c = lane; c < MW; c += 32) {
                    const int e = r * MW + c;
                    mnext[X][e] = a.r * mnext[X][e] + a.one_minus_r * u4[1][(r + 2) * UW + c];
                    mnext[Y][e] = a.r * mnext[Y][e] + a.one_minus_r * v4[1][r * VW + c + 2];
                    mnext[Z][e] = a.r * mnext[Z][e] + a.one_minus_r * w1[(r + 2) * WW + c + 2];
                }
            }
            __syncthreads();
        }
        const int e = j + 2;
        const EdgeCoef<T> cze = edge_coef(g, Z, e, nz);
        T* const yw = base + G::OYW + wrap(se + 2, G::SE) * 2 * G::NYW;     // plane j+2
        T* const xw = base + G::OXW + wrap(se + 2, G::SE) * 2 * G::NXW;
        T* const kj = base + G::OK + sk * G::NK;
        const bool faces = j >= z0, kk = j >= z0 - 1;
        // ---- phase A: this thread's own edges and K
        const EdgeTerms<T> ye = y_edge(u4, w2, x, y, cxo, cze);
        const EdgeTerms<T> xe = x_edge(v4, w2, x, y, cyo, cze);
        yw[warp * EW + lane + 1] = ye.g1;
        yw[G::NYW + warp * EW + lane + 1] = ye.g3;
        xw[(warp + 1) * TX + lane] = xe.g1;
        xw[G::NXW + (warp + 1) * TX + lane] = xe.g3;
        T* const zu = base + G::OZU;
        T* const zv = base + G::OZV;
        if (faces) {
            const EdgeTerms<T> ze = z_edge(u4[0], v4[0], x, y, cxo, cyo);
            zu[(warp + 1) * TX + lane] = ze.f1;
            zu[G::NZU + (warp + 1) * TX + lane] = ze.f3;
            zv[warp * EW + lane + 1] = ze.g1;
            zv[G::NZV + warp * EW + lane + 1] = ze.g3;
        }
        const T* const mj[3] = {M(X, sm, 1), M(Y, sm, 1), M(Z, sm, 1)};        // layer (z-face) j
        if (kk) {
            kj[(warp + 1) * KW + lane + 1] = k_cell(u4[0], v4[0], w0, w1, mj[X], mj[Y], mj[Z], mnext[Z], x, y);
            if (warp == 0)       // the row below the block
                kj[lane + 1] = k_cell(u4[0], v4[0], w0, w1, mj[X], mj[Y], mj[Z], mnext[Z], x, y0 - 1);
            if (lane == 0) {     // the column left of the block (and its corner)
                kj[(warp + 1) * KW] = k_cell(u4[0], v4[0], w0, w1, mj[X], mj[Y], mj[Z], mnext[Z], x0 - 1, y);
                if (warp == 0) kj[0] = k_cell(u4[0], v4[0], w0, w1, mj[X], mj[Y], mj[Z], mnext[Z], x0 - 1, y0 - 1);
            }
        }
        // ---- phase A: the halo edges, one kind per warp: x-edges at the three extra y-faces (warps 0-2), zU there
        // (warps 3-5), y-edges at the three extra x-faces (warp 6) and zV there (warp 7)
        if (warp < 3) {
            const int row = warp == 0 ? 0 : TY + warp, b = y0 - 1 + row;
            const EdgeTerms<T> h = x_edge(v4, w2, x, b, edge_coef(g, Y, b, ny), cze);
            xw[row * TX + lane] = h.g1;
            xw[G::NXW + row * TX + lane] = h.g3;
        } else if (warp < 6) {
            if (faces) {
                const int row = warp == 3 ? 0 : TY + warp - 3, b = y0 - 1 + row;
                const EdgeTerms<T> h = z_edge(u4[0], v4[0], x, b, cxo, edge_coef(g, Y, b, ny));
                zu[row * TX + lane] = h.f1;
                zu[G::NZU + row * TX + lane] = h.f3;
            }
        } else if (lane < 3 * TY) {
            const int c = lane / TY, col = c == 0 ? 0 : TX + c, ea = x0 - 1 + col, cy = y0 + lane % TY;
            if (warp == 6) {
                const EdgeTerms<T> h = y_edge(u4, w2, ea, cy, edge_coef(g, X, ea, nx), cze);
                yw[(cy - y0) * EW + col] = h.g1;
                yw[G::NYW + (cy - y0) * EW + col] = h.g3;
            } else if (faces) {
                const EdgeTerms<T> h = z_edge(u4[0], v4[0], ea, cy, edge_coef(g, X, ea, nx), edge_coef(g, Y, cy, ny));
                zv[(cy - y0) * EW + col] = h.g1;
                zv[G::NZV + (cy - y0) * EW + col] = h.g3;
            }
        }
        __syncthreads();

        // ---- phase B: the faces of layer j
        if (faces && live) {
            const int z = j;
            const T* const kc = kj + (warp + 1) * KW + lane + 1;
            const T* const km = base + G::OK + wrap(sk + 1, G::SK) * G::NK + (warp + 1) * KW + lane + 1;   // layer j-1
            const int om = (warp + 1) * MW + lane + 1;
            const T* const mprev[3] = {M(X, sm, 0), M(Y, sm, 0), M(Z, sm, 0)};      // layer (z-face) j-1
            const T ispz0 = tab(g, Z, kInvSp, z), ispz1 = tab(g, Z, kInvSp, z + 1), iwz0 = tab(g, Z, kInvW, z);
            // viscous flux-form Laplacian of component A at (x, y, z) with wall and lid fluxes, then the RK
            // combination (the expressions of viscous_rk_tile, backend.cu:289-329)
            auto visc = [&](auto Acomp, T L, T wall) {
                constexpr int A = decltype(Acomp)::value;
                const T* mc = mj[A] + om;
                const T cc = mc[0];
                T lap = T(0);
                // x
                if (A == X) {
                    lap = lap + ((mc[1] - cc) * fx.iw0 - (cc - mc[-1]) * fx.iwm) * fx.is0;
                } else {
                    T hi = x < nx - 1 ? (mc[1] - cc) * fx.is1 : T(0);
                    T lo = x > 0 ? (cc - mc[-1]) * fx.is0 : T(0);
                    if (x == 0) lo = wall * fx.is0;
                    if (x == nx - 1) hi = -wall * fx.is1;
                    lap = lap + (hi - lo) * fx.iw0;
                }
                // y (the lid is the top wall)
                if (A == Y) {
                    lap = lap + ((mc[MW] - cc) * fy.iw0 - (cc - mc[-MW]) * fy.iwm) * fy.is0;
                } else {
                    T hi = y < ny - 1 ? (mc[MW] - cc) * fy.is1 : T(0);
                    T lo = y > 0 ? (cc - mc[-MW]) * fy.is0 : T(0);
                    if (y == 0) lo = wall * fy.is0;
                    if (y == ny - 1) {
                        const T Ul = A == X ? lidv * g.lid_u[x + (nx + 1) * z] : T(0);
                        hi = (Ul - wall) * fy.is1;
                    }
                    lap = lap + (hi - lo) * fy.iw0;
                }
                // z
                const T zl = mprev[A][om], zh = mnext[A][om];
                if (A == Z) {
                    lap = lap + ((zh - cc) * iwz0 - (cc - zl) * tab(g, Z, kInvW, z - 1)) * ispz0;
                } else {
                    T hi = z < nz - 1 ? (zh - cc) * ispz1 : T(0);
                    T lo = z > 0 ? (cc - zl) * ispz0 : T(0);
                    if (z == 0) lo = wall * ispz0;
                    if (z == nz - 1) hi = -wall * ispz1;
                    lap = lap + (hi - lo) * iwz0;
                }
                const int i = fidx<A>(p, x, y, z);
                T val = cc + dt * (nu * lap + L);
                if (a.stage > 0) val = a0 * a.m0[A][i] + b0 * val;
                a.out[A][i] = val;
            };
            // u-face x
            {
                const int i = fidx<X>(p, x, y, z);
                if (blend) a.m0_out[X][i] = mj[X][om];
                if (x == 0) a.out[X][i] = T(0);
                else {
                    const T* z1p = zu + (warp + 1) * TX + lane;
                    T L = half * (z1p[TX] + z1p[0]) + half * (yu1_1 + yu1_0);
                    if (o4) {
                        const T* z3p = z1p + G::NZU;
                        L = L + fx.c3 * (z3p[2 * TX] + z3p[-TX]);
                        L = L + fx.c3 * (ye.f3 + yu3_m1);
                    }
                    L = L - (kc[0] - kc[-1]) * fx.is0;
                    visc(std::integral_constant<int, X>{}, L, u4[0][(warp + 3) * UW + lane + 1]);
                }
                if (x == nx - 1) {
                    if (blend) a.m0_out[X][i + 1] = mj[X][om + 1];
                    a.out[X][i + 1] = T(0);
                }
            }
            // v-face y
            {
                const int i = fidx<Y>(p, x, y, z);
                if (blend) a.m0_out[Y][i] = mj[Y][om];
                if (y == 0) a.out[Y][i] = T(0);
                else {
                    const T* z1p = zv + warp * EW + lane + 1;
                    T L = half * (z1p[1] + z1p[0]) + half * (xv1_1 + xv1_0);
                    if (o4) {
                        const T* z3p = z1p + G::NZV;
                        L = L + fy.c3 * (z3p[2] + z3p[-1]);
                        L = L + fy.c3 * (xe.f3 + xv3_m1);
                    }
                    L = L - (kc[0] - kc[-KW]) * fy.is0;
                    visc(std::integral_constant<int, Y>{}, L, v4[0][(warp + 1) * VW + lane + 3]);
                }
                if (y == ny - 1) {
                    if (blend) a.m0_out[Y][i + nx] = mj[Y][om + MW];
                    a.out[Y][i + nx] = T(0);
                }
            }
            // w-face z
            {
                const int i = fidx<Z>(p, x, y, z);
                if (blend) a.m0_out[Z][i] = mj[Z][om];
                if (z == 0) a.out[Z][i] = T(0);
                else {
                    const T* xw1 = base + G::OXW + se * 2 * G::NXW + (warp + 1) * TX + lane;     // plane j
                    const T* xw3 = xw1 + G::NXW;
                    const T* yw1 = base + G::OYW + se * 2 * G::NYW + warp * EW + lane + 1;
                    const T* yw3 = yw1 + G::NYW;
                    T L = half * (xw1[TX] + xw1[0]) + half * (yw1[1] + yw1[0]);
                    if (o4) {
                        const T c3 = tab(g, Z, kC3, z);
                        L = L + c3 * (xw3[2 * TX] + xw3[-TX]);
                        L = L + c3 * (yw3[2] + yw3[-1]);
                    }
                    L = L - (kc[0] - km[0]) * ispz0;
                    visc(std::integral_constant<int, Z>{}, L, w0[(warp + 3) * WW + lane + 3]);
                }
                if (z == nz - 1) {
                    if (blend) a.m0_out[Z][i + nx * ny] = mnext[Z][om];
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
