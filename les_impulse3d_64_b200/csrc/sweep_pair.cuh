// sweep_pair.cuh - the FP32 momentum sweep on the shared-memory tile with two cells per thread in packed
// arithmetic (CAVITY_SWEEP=pair).
//
// The tile and its staging are the tile kernel's (tile_prologue, sweep_tile.cuh).  A thread takes the cells x and
// x + 1 (x even) of a row and evaluates their faces together in the FP32x2 instructions of sm_100
// (fma.rn.f32x2 and friends, through __ffma2_rn / __fadd2_rn / __fmul2_rn): one instruction does the arithmetic of
// both cells.  The table values of the y and z axes, the same for both cells, are read once per pair, and the
// x-neighbours the two cells share are read once.  The expressions and the order of every sum are the tile
// kernel's (backend.cu:141-330).
#pragma once
#include "sweep_tile.cuh"

namespace cavity {

// two FP32 values in one packed register pair
struct F2 {
    float2 v;
};
__device__ __forceinline__ F2 f2(float a, float b) { return {make_float2(a, b)}; }
__device__ __forceinline__ F2 f2(float s) { return {make_float2(s, s)}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return {__fmul2_rn(a.v, b.v)}; }
// a - b as a + (-1) b: the product is exact, so the result is the rounded difference
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return {__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
__device__ __forceinline__ F2 operator-(F2 a) { return {make_float2(-a.v.x, -a.v.y)}; }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ F2 sel2(bool ca, bool cb, F2 a, F2 b) {      // per component: c ? a : b
    return f2(ca ? a.v.x : b.v.x, cb ? a.v.y : b.v.y);
}
__device__ __forceinline__ F2 ld2(const float* p) { return f2(p[0], p[1]); }
// a b - c d with one rounding fewer: fma(a, b, -(c d))
__device__ __forceinline__ F2 fms2(F2 a, F2 b, F2 c, F2 d) { return fma2(a, b, -(c * d)); }
// the narrow stencil weight of an edge whose two axes are the same for both cells of the pair
__device__ __forceinline__ float w1v(int o4, float okA, float okB, float lA, float lB, float eighth) {
    return o4 ? okA * okB * (1.f + (lA * lB) * eighth) : okA * okB;
}

// viscous flux-form Laplacian and RK combination of viscous_rk_tile for the faces of component A of cells x, x + 1
template <int A, int MW, int MH, class TS0, class TS1, class TS2>
__device__ __forceinline__ F2 viscous_rk_pair(const MomentumArgs<float>& a, const float* mb, F2 wall, const StageConst& sc,
                                              float dt, float lidv, int x, int y, int z, F2 base, F2 L, const TS0& tX,
                                              const TS1& tY, const TS2& tZ) {
    const Params& p = a.p;
    const F2 cc = ld2(mb);
    const F2 zero = f2(0.f);
    F2 lap = zero;
    auto tx2 = [&](int k, int i) { return f2(tX(k, i), tX(k, i + 1)); };
    // axis X: the cells' own values differ across the pair
    {
        const F2 up = ld2(mb + 1), dn = ld2(mb - 1);
        if (A == X) {
            lap = lap + fms2(up - cc, tx2(kInvW, x), cc - dn, tx2(kInvW, x - 1)) * tx2(kInvSp, x);
        } else {
            const bool ha = x < p.nx - 1, hb = x + 1 < p.nx - 1, la = x > 0;
            F2 hi = sel2(ha, hb, (up - cc) * tx2(kInvSp, x + 1), zero);
            F2 lo = sel2(la, true, (cc - dn) * tx2(kInvSp, x), zero);
            if (x == 0) lo = f2(wall.v.x * tX(kInvSp, 0), lo.v.y);
            if (x == p.nx - 1) hi = f2(-wall.v.x * tX(kInvSp, p.nx), hi.v.y);
            if (x + 1 == p.nx - 1) hi = f2(hi.v.x, -wall.v.y * tX(kInvSp, p.nx));
            lap = lap + (hi - lo) * tx2(kInvW, x);
        }
    }
    // axes Y and Z: the same index for both cells
#pragma unroll
    for (int t = 1; t < 3; t++) {
        const auto tb = [&](int k, int idx) { return t == 1 ? tY(k, idx) : tZ(k, idx); };
        const int q = t == 1 ? y : z, n = t == 1 ? p.ny : p.nz;
        const int s = t == 1 ? MW : MW * MH;
        const F2 up = ld2(mb + s), dn = ld2(mb - s);
        if (t == A) {
            lap = lap + ((up - cc) * f2(tb(kInvW, q)) - (cc - dn) * f2(tb(kInvW, q - 1))) * f2(tb(kInvSp, q));
            continue;
        }
        F2 hi = q < n - 1 ? (up - cc) * f2(tb(kInvSp, q + 1)) : zero;
        F2 lo = q > 0 ? (cc - dn) * f2(tb(kInvSp, q)) : zero;
        if (q == 0) lo = wall * f2(tb(kInvSp, 0));
        if (q == n - 1) {
            if (t == Y) {
                const F2 U = A == X ? f2(lidv) * ld2(a.g.lid_u + x + (p.nx + 1) * z) : zero;
                hi = (U - wall) * f2(tb(kInvSp, n));
            } else {
                hi = -wall * f2(tb(kInvSp, n));
            }
        }
        lap = lap + (hi - lo) * f2(tb(kInvW, q));
    }
    F2 val = fma2(f2(dt), fma2(f2(a.nu), lap, L), cc);
    if (a.stage > 0) val = f2((float)sc.a0) * base + f2((float)sc.b) * val;
    return val;
}

template <int TY, int TZ, int NT>
__device__ void sweep_pair_body(const MomentumArgs<float>& a, const Blk& blk) {
    using T = float;
    using G = TileGeom<TY, TZ, NT, true>;           // odd row pitches: a warp reads two rows (half warps)
    constexpr int TX = G::TX;
    constexpr int UW = G::UW, UH = G::UH, VW = G::VW, VH = G::VH, WW = G::WW, WH = G::WH, MW = G::MW, MH = G::MH;
    constexpr int UP = UH * UW, VP = VH * VW, WP = WH * WW;
    constexpr int PAIR_ROWS = 2 * G::WARPS;                  // rows a sweep of the block covers (16 lanes per row)
    static_assert(TY * TZ % PAIR_ROWS == 0, "rows must divide among the half-warps");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const TileArrays<T> ta = tile_arrays<T, G>(smem_raw);
    StageConst sc;
    T dt;
    if (!tile_prologue<T, G>(a, blk, ta, sc, dt)) return;
    const T *SU = ta.SU, *SV = ta.SV, *SW = ta.SW, *MX = ta.MX, *MY = ta.MY, *MZ = ta.MZ, *Kc = ta.Kc;
    const Params& p = a.p;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int x0 = blk.x * TX, y0 = blk.y * TY, z0 = blk.z * TZ;
    const int o4 = p.o4;
    const bool blend = a.stage == 0;
    const TabSlice<T, G::SX> tX{ta.TXs, x0};
    const TabSlice<T, G::SY> tY{ta.TYs, y0};
    const TabSlice<T, G::SZ> tZ{ta.TZs, z0};
    const T lidv = (T)lid_speed(p, sc.tau);
    const F2 half = f2(0.5f);
    const T eighth = T(0.125);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int px = 2 * (lane & 15);                          // the pair's first cell within the tile row
    auto kidx = [&](int ix, int iy, int iz) { return (iz * (TY + 1) + iy) * (TX + 1) + ix; };
    auto tx2 = [&](int k, int i) { return f2(tX(k, i), tX(k, i + 1)); };
    // stencil weights of an edge: A per cell (pair), B shared (scalar)
    auto w1 = [&](F2 okA, T okB, F2 lA, T lB) {
        return o4 ? okA * f2(okB) * (f2(1.f) + (lA * f2(lB)) * f2(eighth)) : okA * f2(okB);
    };
    auto w1s = [&](T okA, F2 okB, T lA, F2 lB) {          // A shared, B per cell
        return o4 ? f2(okA) * okB * (f2(1.f) + (f2(lA) * lB) * f2(eighth)) : f2(okA) * okB;
    };
    auto w3 = [&](F2 lA, T lB) { return -((lA * f2(lB)) * f2(eighth)); };
    auto w3s = [&](T lA, F2 lB) { return -((f2(lA) * lB) * f2(eighth)); };

    // A half-warp takes RPT consecutive rows of one column of the tile, and the corner edges of each cell are
    // evaluated once for the two faces each feeds, the y- and x-edges on z-face z + 1 carrying over to the next
    // row, as in the tile kernel (sweep_tile_body); the terms are the same packed expressions as before.
    constexpr int RPT = TY * TZ / PAIR_ROWS;
    static_assert(PAIR_ROWS % TY == 0 && PAIR_ROWS / TY * RPT == TZ, "a half-warp's rows are one column of the tile");
    const int hw = 2 * warp + (lane >> 4);
    F2 cyWo = f2(0.f), cyU = f2(0.f), cyUl = f2(0.f), cyUh = f2(0.f);    // y-edge (x, z + 1)
    F2 cxWo = f2(0.f), cxV = f2(0.f), cxVl = f2(0.f), cxVh = f2(0.f);    // x-edge (y, z + 1)
#pragma unroll 1
    for (int r = 0; r < RPT; r++) {
        const int ry = hw % TY, rz = RPT * (hw / TY) + r;
        const int x = x0 + px, y = y0 + ry, z = z0 + rz;
        if (x >= nx || y >= ny || z >= nz) continue;
        const bool vb = x + 1 < nx;                           // the pair's second cell is inside
        const T* pu = SU + ((rz + 3) * UH + ry + 3) * UW + px + 1;
        const T* pv = SV + ((rz + 3) * VH + ry + 1) * VW + px + 3;
        const T* pw = SW + ((rz + 1) * WH + ry + 3) * WW + px + 3;
        const int mo = ((rz + 1) * MH + ry + 1) * MW + px + 1;
        const F2 kc = ld2(Kc + kidx(px + 1, ry + 1, rz + 1));
        const int iu = fidx<X>(p, x, y, z), iv = fidx<Y>(p, x, y, z), iw = fidx<Z>(p, x, y, z);
        const bool rk = a.stage > 0;
        const F2 zero = f2(0.f);
        const F2 bu = rk ? f2(__ldg(a.m0[X] + iu), vb ? __ldg(a.m0[X] + iu + 1) : 0.f) : zero;
        const F2 bv = rk ? f2(__ldg(a.m0[Y] + iv), vb ? __ldg(a.m0[Y] + iv + 1) : 0.f) : zero;
        const F2 bw = rk ? f2(__ldg(a.m0[Z] + iw), vb ? __ldg(a.m0[Z] + iw + 1) : 0.f) : zero;
        auto store = [&](T* out, int i, F2 v, bool zero_a) {
            st_out(out + i, zero_a ? T(0) : v.v.x);
            if (vb) st_out(out + i + 1, v.v.y);
        };

        // ---------------- the corner edges: narrow terms of two faces each
        F2 uZ0, vZ0, uY0, wY0, vX0, wX0, uY1, vX1;
        {
            const F2 ok1x = tx2(kOk1, x), l1x = tx2(kL1, x), i1x = tx2(kInvSp, x), e1lx = tx2(kEv1Lo, x),
                     e1hx = tx2(kEv1Hi, x);
            const T ok1y = tY(kOk1, y), l1y = tY(kL1, y), i1y = tY(kInvSp, y);
            const F2 e1ly = f2(tY(kEv1Lo, y)), e1hy = f2(tY(kEv1Hi, y)), e1lz = f2(tZ(kEv1Lo, z)), e1hz = f2(tZ(kEv1Hi, z));
            {   // z-edge (x, y)
                const F2 vl = ld2(pv - 1), vh = ld2(pv), ul = ld2(pu - UW), uh = ld2(pu);
                const F2 wo = w1(ok1x, ok1y, l1x, l1y) * fms2(vh - vl, i1x, uh - ul, f2(i1y));
                uZ0 = wo * fma2(e1lx, vl, e1hx * vh);
                vZ0 = -(wo * fma2(e1ly, ul, e1hy * uh));
            }
            if (r == 0) {
                const T ok1z = tZ(kOk1, z), l1z = tZ(kL1, z), i1z = tZ(kInvSp, z);
                {   // y-edge (x, z)
                    const F2 ul = ld2(pu - UP), uh = ld2(pu), wl = ld2(pw - 1), wh = ld2(pw);
                    const F2 wo = w1s(ok1z, ok1x, l1z, l1x) * fms2(uh - ul, f2(i1z), wh - wl, i1x);
                    uY0 = -(wo * fma2(e1lx, wl, e1hx * wh));
                    wY0 = wo * fma2(e1lz, ul, e1hz * uh);
                }
                {   // x-edge (y, z)
                    const F2 wl = ld2(pw - WW), wh = ld2(pw), vl = ld2(pv - VP), vh = ld2(pv);
                    const F2 wo = f2(w1v(o4, ok1y, ok1z, l1y, l1z, eighth)) * fms2(wh - wl, f2(i1y), vh - vl, f2(i1z));
                    vX0 = wo * fma2(e1ly, wl, e1hy * wh);
                    wX0 = -(wo * fma2(e1lz, vl, e1hz * vh));
                }
            } else {     // the previous row's edges on this cell's lower z-face
                uY0 = cyU;
                wY0 = cyWo * fma2(e1lz, cyUl, e1hz * cyUh);
                vX0 = cxV;
                wX0 = -(cxWo * fma2(e1lz, cxVl, e1hz * cxVh));
            }
            {   // the edges on z-face z + 1 (the next row's corner edges)
                const T ok1 = tZ(kOk1, z + 1), l1 = tZ(kL1, z + 1), i1 = tZ(kInvSp, z + 1);
                const F2 ul = ld2(pu), uh = ld2(pu + UP), wl = ld2(pw + WP - 1), wh = ld2(pw + WP);
                cyWo = w1s(ok1, ok1x, l1, l1x) * fms2(uh - ul, f2(i1), wh - wl, i1x);
                cyU = -(cyWo * fma2(e1lx, wl, e1hx * wh));
                cyUl = ul;
                cyUh = uh;
                const F2 wl2 = ld2(pw + WP - WW), wh2 = ld2(pw + WP), vl = ld2(pv), vh = ld2(pv + VP);
                cxWo = f2(w1v(o4, ok1y, ok1, l1y, l1, eighth)) * fms2(wh2 - wl2, f2(i1y), vh - vl, f2(i1));
                cxV = cxWo * fma2(e1ly, wl2, e1hy * wh2);
                cxVl = vl;
                cxVh = vh;
            }
            uY1 = cyU;
            vX1 = cxV;
        }

        // ---------------- u-faces x, x + 1: z-edges (omega_z) and y-edges (omega_y)
        {
            if (blend) {
                st_out(a.m0_out[X] + (iu), MX[mo]);
                if (vb) st_out(a.m0_out[X] + (iu + 1), MX[mo + 1]);
            }
            const F2 ok1x = tx2(kOk1, x), l1x = tx2(kL1, x), l3x = tx2(kL3, x), i1x = tx2(kInvSp, x),
                     i3x = tx2(kInvNd3, x);
            const F2 e1l = tx2(kEv1Lo, x), e1h = tx2(kEv1Hi, x), e3l = tx2(kEv3Lo, x), e3h = tx2(kEv3Hi, x);
            auto pz1 = [&](int d) {
                const int e = y + d;
                const F2 vl = ld2(pv + d * VW - 1), vh = ld2(pv + d * VW), ul = ld2(pu + (d - 1) * UW), uh = ld2(pu + d * UW);
                const F2 wo = w1(ok1x, tY(kOk1, e), l1x, tY(kL1, e)) * fms2(vh - vl, i1x, uh - ul, f2(tY(kInvSp, e)));
                return wo * fma2(e1l, vl, e1h * vh);
            };
            auto pz3 = [&](int d) {
                const int e = y + d;
                const F2 vl = ld2(pv + d * VW - 2), vh = ld2(pv + d * VW + 1), ul = ld2(pu + (d - 2) * UW),
                         uh = ld2(pu + (d + 1) * UW);
                const F2 wo = w3(l3x, tY(kL3, e)) * fms2(vh - vl, i3x, uh - ul, f2(tY(kInvNd3, e)));
                return wo * fma2(e3l, vl, e3h * vh);
            };
            auto py3 = [&](int d) {
                const int e = z + d;
                const F2 ul = ld2(pu + (d - 2) * UP), uh = ld2(pu + (d + 1) * UP), wl = ld2(pw + d * WP - 2),
                         wh = ld2(pw + d * WP + 1);
                const F2 wo = w3s(tZ(kL3, e), l3x) * fms2(uh - ul, f2(tZ(kInvNd3, e)), wh - wl, i3x);
                return -(wo * fma2(e3l, wl, e3h * wh));
            };
            F2 L = fma2(half, pz1(1) + uZ0, half * (uY1 + uY0));
            if (o4) {
                const F2 c3 = tx2(kC3, x);
                L = fma2(c3, pz3(2) + pz3(-1), L);
                L = fma2(c3, py3(2) + py3(-1), L);
            }
            L = fma2(ld2(Kc + kidx(px, ry + 1, rz + 1)) - kc, tx2(kInvSp, x), L);
            const F2 val = viscous_rk_pair<X, MW, MH>(a, MX + mo, ld2(pu), sc, dt, lidv, x, y, z, bu, L, tX, tY, tZ);
            store(a.out[X], iu, val, x == 0);
            const int xl = x + 1 == nx - 1 ? x + 1 : x == nx - 1 ? x : -1;     // the cell whose upper wall face is zero
            if (xl >= 0) {
                if (blend) st_out(a.m0_out[X] + (iu + (xl - x) + 1), MX[mo + (xl - x) + 1]);
                st_out(a.out[X] + (iu + (xl - x) + 1), T(0));
            }
        }
        // ---------------- v-faces y: z-edges (omega_z) and x-edges (omega_x)
        {
            if (blend) {
                st_out(a.m0_out[Y] + (iv), MY[mo]);
                if (vb) st_out(a.m0_out[Y] + (iv + 1), MY[mo + 1]);
            }
            if (y == 0) {
                st_out(a.out[Y] + (iv), T(0));
                if (vb) st_out(a.out[Y] + (iv + 1), T(0));
            } else {
                const T ok1y = tY(kOk1, y), l1y = tY(kL1, y), l3y = tY(kL3, y), i1y = tY(kInvSp, y), i3y = tY(kInvNd3, y);
                const F2 e1l = f2(tY(kEv1Lo, y)), e1h = f2(tY(kEv1Hi, y)), e3l = f2(tY(kEv3Lo, y)), e3h = f2(tY(kEv3Hi, y));
                auto pz1 = [&](int d) {
                    const int e = x + d;
                    const F2 vl = ld2(pv + d - 1), vh = ld2(pv + d), ul = ld2(pu + d - UW), uh = ld2(pu + d);
                    const F2 wo = w1(tx2(kOk1, e), ok1y, tx2(kL1, e), l1y) * fms2(vh - vl, tx2(kInvSp, e), uh - ul, f2(i1y));
                    return -(wo * fma2(e1l, ul, e1h * uh));
                };
                auto pz3 = [&](int d) {
                    const int e = x + d;
                    const F2 vl = ld2(pv + d - 2), vh = ld2(pv + d + 1), ul = ld2(pu + d - 2 * UW), uh = ld2(pu + d + UW);
                    const F2 wo = w3(tx2(kL3, e), l3y) * fms2(vh - vl, tx2(kInvNd3, e), uh - ul, f2(i3y));
                    return -(wo * fma2(e3l, ul, e3h * uh));
                };
                auto px3 = [&](int d) {
                    const int e = z + d;
                    const F2 wl = ld2(pw + d * WP - 2 * WW), wh = ld2(pw + d * WP + WW), vl = ld2(pv + (d - 2) * VP),
                             vh = ld2(pv + (d + 1) * VP);
                    const F2 wo = f2(-((l3y * tZ(kL3, e)) * eighth)) * fms2(wh - wl, f2(i3y), vh - vl, f2(tZ(kInvNd3, e)));
                    return wo * fma2(e3l, wl, e3h * wh);
                };
                F2 L = fma2(half, pz1(1) + vZ0, half * (vX1 + vX0));
                if (o4) {
                    const F2 c3 = f2(tY(kC3, y));
                    L = fma2(c3, pz3(2) + pz3(-1), L);
                    L = fma2(c3, px3(2) + px3(-1), L);
                }
                L = fma2(ld2(Kc + kidx(px + 1, ry, rz + 1)) - kc, f2(tY(kInvSp, y)), L);
                const F2 val = viscous_rk_pair<Y, MW, MH>(a, MY + mo, ld2(pv), sc, dt, lidv, x, y, z, bv, L, tX, tY, tZ);
                store(a.out[Y], iv, val, false);
            }
            if (y == ny - 1) {
                if (blend) {
                    st_out(a.m0_out[Y] + (iv + nx), MY[mo + MW]);
                    if (vb) st_out(a.m0_out[Y] + (iv + nx + 1), MY[mo + MW + 1]);
                }
                st_out(a.out[Y] + (iv + nx), T(0));
                if (vb) st_out(a.out[Y] + (iv + nx + 1), T(0));
            }
        }
        // ---------------- w-faces z: x-edges (omega_x) and y-edges (omega_y)
        {
            if (blend) {
                st_out(a.m0_out[Z] + (iw), MZ[mo]);
                if (vb) st_out(a.m0_out[Z] + (iw + 1), MZ[mo + 1]);
            }
            if (z == 0) {
                st_out(a.out[Z] + (iw), T(0));
                if (vb) st_out(a.out[Z] + (iw + 1), T(0));
            } else {
                const T ok1z = tZ(kOk1, z), l1z = tZ(kL1, z), l3z = tZ(kL3, z), i1z = tZ(kInvSp, z), i3z = tZ(kInvNd3, z);
                const F2 e1l = f2(tZ(kEv1Lo, z)), e1h = f2(tZ(kEv1Hi, z)), e3l = f2(tZ(kEv3Lo, z)), e3h = f2(tZ(kEv3Hi, z));
                auto px1 = [&](int d) {
                    const int e = y + d;
                    const F2 wl = ld2(pw + (d - 1) * WW), wh = ld2(pw + d * WW), vl = ld2(pv + d * VW - VP), vh = ld2(pv + d * VW);
                    const F2 wo = f2(w1v(o4, tY(kOk1, e), ok1z, tY(kL1, e), l1z, eighth)) *
                                  fms2(wh - wl, f2(tY(kInvSp, e)), vh - vl, f2(i1z));
                    return -(wo * fma2(e1l, vl, e1h * vh));
                };
                auto px3 = [&](int d) {
                    const int e = y + d;
                    const F2 wl = ld2(pw + (d - 2) * WW), wh = ld2(pw + (d + 1) * WW), vl = ld2(pv + d * VW - 2 * VP),
                             vh = ld2(pv + d * VW + VP);
                    const F2 wo = f2(-((tY(kL3, e) * l3z) * eighth)) * fms2(wh - wl, f2(tY(kInvNd3, e)), vh - vl, f2(i3z));
                    return -(wo * fma2(e3l, vl, e3h * vh));
                };
                auto py1 = [&](int d) {
                    const int e = x + d;
                    const F2 ul = ld2(pu + d - UP), uh = ld2(pu + d), wl = ld2(pw + d - 1), wh = ld2(pw + d);
                    const F2 wo = w1s(ok1z, tx2(kOk1, e), l1z, tx2(kL1, e)) * fms2(uh - ul, f2(i1z), wh - wl, tx2(kInvSp, e));
                    return wo * fma2(e1l, ul, e1h * uh);
                };
                auto py3 = [&](int d) {
                    const int e = x + d;
                    const F2 ul = ld2(pu + d - 2 * UP), uh = ld2(pu + d + UP), wl = ld2(pw + d - 2), wh = ld2(pw + d + 1);
                    const F2 wo = w3s(l3z, tx2(kL3, e)) * fms2(uh - ul, f2(i3z), wh - wl, tx2(kInvNd3, e));
                    return wo * fma2(e3l, ul, e3h * uh);
                };
                F2 L = fma2(half, px1(1) + wX0, half * (py1(1) + wY0));
                if (o4) {
                    const F2 c3 = f2(tZ(kC3, z));
                    L = fma2(c3, px3(2) + px3(-1), L);
                    L = fma2(c3, py3(2) + py3(-1), L);
                }
                L = fma2(ld2(Kc + kidx(px + 1, ry + 1, rz)) - kc, f2(tZ(kInvSp, z)), L);
                const F2 val = viscous_rk_pair<Z, MW, MH>(a, MZ + mo, ld2(pw), sc, dt, lidv, x, y, z, bw, L, tX, tY, tZ);
                store(a.out[Z], iw, val, false);
            }
            if (z == nz - 1) {
                if (blend) {
                    st_out(a.m0_out[Z] + (iw + nx * ny), MZ[mo + MW * MH]);
                    if (vb) st_out(a.m0_out[Z] + (iw + nx * ny + 1), MZ[mo + MW * MH + 1]);
                }
                st_out(a.out[Z] + (iw + nx * ny), T(0));
                if (vb) st_out(a.out[Z] + (iw + nx * ny + 1), T(0));
            }
        }
    }
}

template <int TY, int TZ, int NT>
__global__ void __launch_bounds__(NT, 2) sweep_pair_kernel(MomentumArgs<float> a) {
    sweep_pair_body<TY, TZ, NT>(a, real_blk());
}
// a batch of cavities: grid x runs over the work list (BatchItem)
template <int TY, int TZ, int NT>
__global__ void __launch_bounds__(NT, 2) sweep_pair_batched(const MomentumArgs<float>* args, const BatchItem* items,
                                                            const int* live) {
    __shared__ MomentumArgs<float> a;
    int cav;
    const Blk k = item_blk(items, live, cav);
    if (cav < 0) return;
    load_args(a, args + cav);
    sweep_pair_body<TY, TZ, NT>(a, k);
}

}  // namespace cavity
