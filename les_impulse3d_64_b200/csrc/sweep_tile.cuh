// sweep_tile.cuh - the momentum sweep on a shared-memory tile (the alternative to momentum_kernel, sweep.cuh).
//
// A CTA owns a tile of 32 x TY x TZ cells and computes the three lower faces of every cell.  It stages every
// input of the tile in shared memory first, all copies in flight at once (cp.async):
//   - the velocity with the halos the 4th-order Lamb stencil reaches: 3 cells across a component's axis, 1-2
//     along it;
//   - the impulse with a 1-cell halo; stage 0 then applies the gauge-reset blend m0 = r m + (1-r) u
//     (backend.cu:880-881) in shared memory, its u values from the velocity boxes (which contain the impulse
//     boxes' cells);
//   - the slices of the per-axis coefficient tables the tile uses.
// No thread waits on a global load while staging: every element is a cp.async, all in flight together.
// Staged values outside the box are clamped copies; every stencil term that reaches them has weight zero.
// K = u.m (backend.cu:218-222) is computed once per cell.  Each face then adds its eight edge terms
// (vorticity times interpolated velocity: backend.cu:141-215), evaluated from shared memory, in the
// reference's order: narrow then wide stencil, first then second tangential axis (backend.cu:232-238,
// 249-255, 266-272).  The narrow terms of the three edges at a cell's lower corner, each shared by two of its
// faces, are evaluated once per cell, and those on its upper z-face carry over to the cell above.  It then adds
// -grad K, the viscous flux Laplacian with its wall and lid fluxes, and the RK combination (backend.cu:279-330).
// The validity rules of the reference's stencils are folded into the weight tables (kOk1, kL1, kL3), so the edge
// arithmetic has no branches.
#pragma once
#include "sweep.cuh"

namespace cavity {

// TY x TZ rows of 32 cells per CTA, NT threads (one warp per row at a time).  ODD: every staged box gets an odd
// row pitch (one unused column where its width is even), for a kernel whose warps read two rows at once, each half
// warp every other word of its row (sweep_pair.cuh): with an even pitch both halves land on the same 16 banks and
// every such load takes two shared-memory wavefronts instead of one.
template <int TY, int TZ, int NT, bool ODD = false> struct TileGeom {
    static constexpr int TX = 32;
    static constexpr int TYc = TY, TZc = TZ;
    static constexpr int THREADS = NT, WARPS = NT / 32;
    static_assert(TY * TZ % WARPS == 0, "rows must divide among the warps");
    static constexpr int ROWS_PER_THREAD = TY * TZ / WARPS;
    static constexpr int pitch(int w) { return ODD && w % 2 == 0 ? w + 1 : w; }
    // velocity boxes: u on x-faces [x0-1, x0+TX+1] x cells [y0-3, y0+TY+2] x [z0-3, z0+TZ+2];
    // v on cells [x0-3, x0+TX+2] x y-faces [y0-1, y0+TY+1] x cells [z0-3, z0+TZ+2];
    // w on cells [x0-3, x0+TX+2] x [y0-3, y0+TY+2] x z-faces [z0-1, z0+TZ+1]
    // (UC, VC, WC, MC columns are staged per row; UW, VW, WW, MW are the row pitches)
    static constexpr int UC = TX + 3, VC = TX + 6, WC = TX + 6, MC = TX + 2;
    static constexpr int UW = pitch(UC), UH = TY + 6, UD = TZ + 6;
    static constexpr int VW = pitch(VC), VH = TY + 3, VD = TZ + 6;
    static constexpr int WW = pitch(WC), WH = TY + 6, WD = TZ + 3;
    // impulse boxes: each component on its faces / cells [lo-1, hi] along every axis
    static constexpr int MW = pitch(MC), MH = TY + 2, MD = TZ + 2;
    static constexpr int NU = UW * UH * UD, NV = VW * VH * VD, NW = WW * WH * WD, NM = MW * MH * MD;
    static constexpr int NK = (TX + 1) * (TY + 1) * (TZ + 1);  // cells [x0-1, x0+TX) x [y0-1, y0+TY) x [z0-1, z0+TZ)
    // table slices: indices [lo-2, lo+T+2] of each axis
    static constexpr int SX = TX + 5, SY = TY + 5, SZ = TZ + 5;
    static constexpr int NTAB = kNumTabs * (SX + SY + SZ);
    static constexpr int ELEMS = NU + NV + NW + 3 * NM + NK + NTAB;
    template <class T> static constexpr size_t smem_bytes() { return sizeof(T) * (size_t)ELEMS; }
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

// A store of the sweep's results (the new impulse, stage 0's RK base) to global memory, issued as st.global: a
// plain store through the arrays' generic pointers would, as far as the compiler can tell, alias the tile staged
// in shared memory, and every staged value read after it would be loaded again.
template <class T> __device__ __forceinline__ void st_out(T* p, T v) {
    const size_t g = __cvta_generic_to_global(p);
    if constexpr (sizeof(T) == 8) asm volatile("st.global.f64 [%0], %1;" ::"l"(g), "d"(v));
    else asm volatile("st.global.f32 [%0], %1;" ::"l"(g), "f"(v));
}

template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* smem_dst, const void* src) {
    const unsigned int dst = (unsigned int)__cvta_generic_to_shared(smem_dst);
    if (BYTES == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src));
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src));
}

// Global offsets of the rows (y, z) of a W x H x D box of a face array with extents (ex, ey, ez) whose corner is
// (., ys, zs), clamped into the array; rows are numbered iy + H * iz.
template <int H, int D>
__device__ __forceinline__ int box_row_base(int row, int ys, int zs, int ex, int ey, int ez) {
    const int iy = row % H, iz = row / H;
    return ex * (clampi(ys + iy, 0, ey - 1) + ey * clampi(zs + iz, 0, ez - 1));
}

// Stage a W x H x D box of a face array whose x-extent is ex and corner x is xs, coordinates clamped into the
// array, from the row offsets `rowbase` (box_row_base), rows P apart in `dst`.  Each thread keeps one column (its
// x offset and clamp) and steps through the rows NT / W at a time.
template <class T, int W, int P, int H, int D, int NT>
__device__ __forceinline__ void stage_box(T* dst, const int* rowbase, const T* __restrict__ m, int xs, int ex) {
    constexpr int RPS = NT / W, ROWS = H * D;
    const int t = threadIdx.x;
    if (t >= RPS * W) return;
    const int ix = t % W;
    const int gx = clampi(xs + ix, 0, ex - 1);
    for (int row = t / W; row < ROWS; row += RPS) cp_async_elem<sizeof(T)>(dst + row * P + ix, m + rowbase[row] + gx);
}
// Stage 0's gauge-reset blend of a staged impulse box (MC columns, row pitch MW): m <- r m + (1-r) u, with u at
// the same face from the velocity box (plane / row strides VP, VW; `uoff` its offset of the impulse box's corner)
template <class T, int MC, int MW, int MH, int MD, int NT, int VW, int VP>
__device__ __forceinline__ void blend_box(T* mb, const T* vb, int uoff, T r, T omr) {
    for (int e = threadIdx.x; e < MC * MH * MD; e += NT) {
        const int ix = e % MC, iy = (e / MC) % MH, iz = e / (MC * MH);
        const int i = (iz * MH + iy) * MW + ix;
        mb[i] = r * mb[i] + omr * vb[uoff + iz * VP + iy * VW + ix];
    }
}

// staged tables of one axis: value of table k at axis index i (i in [lo-2, lo+len+2])
template <class T, int S> struct TabSlice {
    const T* t;
    int lo;
    __device__ __forceinline__ T operator()(int k, int i) const { return t[k * S + (i - lo + 2)]; }
};

// viscous flux-form Laplacian of the impulse at a face of component A from its staged box (strides 1, MW,
// MW*MH), wall and lid fluxes, then the RK combination with the inviscid term L and the RK base value `base`
// (stages 1, 2) (backend.cu:289-329)
template <int A, class T, int MW, int MH, class TS0, class TS1, class TS2>
__device__ __forceinline__ T viscous_rk_tile(const MomentumArgs<T>& a, const T* mb, T wall, const StageConst& sc, T dt,
                                             T lidv, int x, int y, int z, T base, T L, const TS0& ts0, const TS1& ts1,
                                             const TS2& ts2) {
    const Params& p = a.p;
    const int q[3] = {x, y, z};
    const int n[3] = {p.nx, p.ny, p.nz};
    constexpr int stride[3] = {1, MW, MW * MH};
    const T cc = mb[0];
    T lap = T(0);
#pragma unroll
    for (int t = 0; t < 3; t++) {
        const auto tb = [&](int k, int idx) { return t == 0 ? ts0(k, idx) : t == 1 ? ts1(k, idx) : ts2(k, idx); };
        const int s = stride[t];
        if (t == A) {
            lap = lap + ((mb[s] - cc) * tb(kInvW, q[t]) - (cc - mb[-s]) * tb(kInvW, q[t] - 1)) * tb(kInvSp, q[t]);
            continue;
        }
        T hi = q[t] < n[t] - 1 ? (mb[s] - cc) * tb(kInvSp, q[t] + 1) : T(0);
        T lo = q[t] > 0 ? (cc - mb[-s]) * tb(kInvSp, q[t]) : T(0);
        if (q[t] == 0) lo = wall * tb(kInvSp, 0);
        if (q[t] == n[t] - 1) {
            if (t == Y) {
                const T U = A == X ? lidv * a.g.lid_u[x + (p.nx + 1) * z] : T(0);
                hi = (U - wall) * tb(kInvSp, n[Y]);
            } else {
                hi = -wall * tb(kInvSp, n[t]);
            }
        }
        lap = lap + (hi - lo) * tb(kInvW, q[t]);
    }
    T val = cc + dt * (a.nu * lap + L);
    if (a.stage > 0) val = T(sc.a0) * base + T(sc.b) * val;
    return val;
}

// The shared-memory arrays of a tile (in this order from the start of dynamic shared memory)
template <class T> struct TileArrays {
    T *SU, *SV, *SW, *MX, *MY, *MZ, *Kc, *TXs, *TYs, *TZs;
};
template <class T, class G> __device__ __forceinline__ TileArrays<T> tile_arrays(unsigned char* base) {
    TileArrays<T> t;
    t.SU = reinterpret_cast<T*>(base);
    t.SV = t.SU + G::NU;
    t.SW = t.SV + G::NV;
    t.MX = t.SW + G::NW;
    t.MY = t.MX + G::NM;
    t.MZ = t.MY + G::NM;
    t.Kc = t.MZ + G::NM;
    t.TXs = t.Kc + G::NK;
    t.TYs = t.TXs + kNumTabs * G::SX;
    t.TZs = t.TYs + kNumTabs * G::SY;
    return t;
}

// Everything a tile's faces need before their arithmetic: the staged boxes and table slices, stage 0's blend, K
// per cell, and the stage constants.  False (in every thread) when the step has failed.
template <class T, class G>
__device__ bool tile_prologue(const MomentumArgs<T>& a, const Blk& blk, const TileArrays<T>& t, StageConst& sc, T& dt) {
    constexpr int TY = G::TYc, TZ = G::TZc, NT = G::THREADS;
    pdl_launch_dependents();
    pdl_wait();
    constexpr int TX = G::TX;
    constexpr int UW = G::UW, UH = G::UH, VW = G::VW, VH = G::VH, WW = G::WW, WH = G::WH, MW = G::MW, MH = G::MH;
    constexpr int UP = UH * UW, VP = VH * VW, WP = WH * WW;      // plane strides of the velocity boxes
    T *SU = t.SU, *SV = t.SV, *SW = t.SW, *MX = t.MX, *MY = t.MY, *MZ = t.MZ, *Kc = t.Kc;
    const Params& p = a.p;
    const Geo<T>& g = a.g;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int x0 = blk.x * TX, y0 = blk.y * TY, z0 = blk.z * TZ;
    const bool blend = a.stage == 0;

    // ---- stage: row offsets of the six boxes first (one pass), then every box
    constexpr int RU = G::UH * G::UD, RV = G::VH * G::VD, RW = G::WH * G::WD, RM = G::MH * G::MD;
    __shared__ int rowbase[RU + RV + RW + 3 * RM];
    for (int e = threadIdx.x; e < RU + RV + RW + 3 * RM; e += NT) {
        int v;
        if (e < RU) v = box_row_base<G::UH, G::UD>(e, y0 - 3, z0 - 3, nx + 1, ny, nz);
        else if (e < RU + RV) v = box_row_base<G::VH, G::VD>(e - RU, y0 - 1, z0 - 3, nx, ny + 1, nz);
        else if (e < RU + RV + RW) v = box_row_base<G::WH, G::WD>(e - RU - RV, y0 - 3, z0 - 1, nx, ny, nz + 1);
        else {
            const int f = e - RU - RV - RW, comp = f / RM;
            v = box_row_base<G::MH, G::MD>(f % RM, y0 - 1, z0 - 1, nx + (comp == X), ny + (comp == Y), nz + (comp == Z));
        }
        rowbase[e] = v;
    }
    __syncthreads();
    const int* rbm = rowbase + RU + RV + RW;
    stage_box<T, G::UC, UW, UH, G::UD, NT>(SU, rowbase, a.u[X], x0 - 1, nx + 1);
    stage_box<T, G::VC, VW, VH, G::VD, NT>(SV, rowbase + RU, a.u[Y], x0 - 3, nx);
    stage_box<T, G::WC, WW, WH, G::WD, NT>(SW, rowbase + RU + RV, a.u[Z], x0 - 3, nx);
    stage_box<T, G::MC, MW, MH, G::MD, NT>(MX, rbm, a.m[X], x0 - 1, nx + 1);
    stage_box<T, G::MC, MW, MH, G::MD, NT>(MY, rbm + RM, a.m[Y], x0 - 1, nx);
    stage_box<T, G::MC, MW, MH, G::MD, NT>(MZ, rbm + 2 * RM, a.m[Z], x0 - 1, nx);
    for (int e = threadIdx.x; e < kNumTabs * (G::SX + G::SY + G::SZ); e += NT) {
        int k, i, axis, len, lo;
        if (e < kNumTabs * G::SX) { axis = X; k = e / G::SX; i = e % G::SX; len = G::SX; lo = x0; }
        else if (e < kNumTabs * (G::SX + G::SY)) {
            const int f = e - kNumTabs * G::SX;
            axis = Y; k = f / G::SY; i = f % G::SY; len = G::SY; lo = y0;
        } else {
            const int f = e - kNumTabs * (G::SX + G::SY);
            axis = Z; k = f / G::SZ; i = f % G::SZ; len = G::SZ; lo = z0;
        }
        const int n = axis == X ? nx : axis == Y ? ny : nz;
        const int idx = clampi(lo - 2 + i, -2, n + 2);
        T* dst = axis == X ? t.TXs : axis == Y ? t.TYs : t.TZs;
        cp_async_elem<sizeof(T)>(dst + k * len + i, g.tab[axis] + k * g.stride[axis] + idx + kTabOffset);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    // the control block's values, read while the copies are in flight
    const int failed = a.c->error;
    sc = stage_const(a.stage, a.c);
    dt = (T)a.c->dt;
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    if (failed) return false;
    if (blend) {      // u of each impulse-box cell: the velocity box entry 2 cells further along its cross axes
        blend_box<T, G::MC, MW, MH, G::MD, NT, UW, UP>(MX, SU, (2 * UH + 2) * UW, a.r, a.one_minus_r);
        blend_box<T, G::MC, MW, MH, G::MD, NT, VW, VP>(MY, SV, 2 * VP + 2, a.r, a.one_minus_r);
        blend_box<T, G::MC, MW, MH, G::MD, NT, WW, WP>(MZ, SW, 2 * WW + 2, a.r, a.one_minus_r);
        __syncthreads();
    }

    // ---- K = u.m per cell (x0-1+ix, y0-1+iy, z0-1+iz)
    constexpr int KW = TX + 1, KRPS = NT / KW;
    for (int e = threadIdx.x % KW + KW * (threadIdx.x / KW); threadIdx.x < KRPS * KW && e < G::NK; e += KRPS * KW) {
        const int ix = threadIdx.x % KW, r = e / KW, iy = r % (TY + 1), iz = r / (TY + 1);
        const T* u0 = SU + ((iz + 2) * UH + iy + 2) * UW + ix;
        const T* v0 = SV + ((iz + 2) * VH + iy) * VW + 2 + ix;
        const T* w0 = SW + (iz * WH + iy + 2) * WW + 2 + ix;
        const int mi = (iz * MH + iy) * MW + ix;
        Kc[e] = T(0.5) * ((u0[0] * MX[mi] + u0[1] * MX[mi + 1]) + (v0[0] * MY[mi] + v0[VW] * MY[mi + MW]) +
                          (w0[0] * MZ[mi] + w0[WP] * MZ[mi + MH * MW]));
    }
    __syncthreads();
    return true;
}

template <class T, int TY, int TZ, int NT>
__device__ void sweep_tile_body(const MomentumArgs<T>& a, const Blk& blk) {
    using G = TileGeom<TY, TZ, NT>;
    constexpr int TX = G::TX, RPT = G::ROWS_PER_THREAD;
    constexpr int UW = G::UW, UH = G::UH, VW = G::VW, VH = G::VH, WW = G::WW, WH = G::WH, MW = G::MW, MH = G::MH;
    constexpr int UP = UH * UW, VP = VH * VW, WP = WH * WW;      // plane strides of the velocity boxes
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const TileArrays<T> ta = tile_arrays<T, G>(smem_raw);
    StageConst sc;
    T dt;
    if (!tile_prologue<T, G>(a, blk, ta, sc, dt)) return;
    T *SU = ta.SU, *SV = ta.SV, *SW = ta.SW, *MX = ta.MX, *MY = ta.MY, *MZ = ta.MZ, *Kc = ta.Kc;
    const Params& p = a.p;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int x0 = blk.x * TX, y0 = blk.y * TY, z0 = blk.z * TZ;
    const int o4 = p.o4;
    const bool blend = a.stage == 0;
    const TabSlice<T, G::SX> tX{ta.TXs, x0};
    const TabSlice<T, G::SY> tY{ta.TYs, y0};
    const TabSlice<T, G::SZ> tZ{ta.TZs, z0};

    const T lidv = (T)lid_speed(p, sc.tau);
    const T half = T(0.5), eighth = T(0.125);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto kidx = [&](int ix, int iy, int iz) { return (iz * (TY + 1) + iy) * (TX + 1) + ix; };
    // stencil weights of an edge between axis indices ia (axis A) and ib (axis B)
    auto w1 = [&](T okA, T okB, T lA, T lB) { return o4 ? okA * okB * (T(1) + (lA * lB) * eighth) : okA * okB; };
    auto w3 = [&](T lA, T lB) { return -((lA * lB) * eighth); };

    // A warp takes RPT consecutive rows of one column of the tile: cells (y, z), (y, z + 1), ...  The three edges
    // at a cell's lower corner each feed two of its faces with the narrow stencil (the z-edge at x-face x, y-face
    // y its u- and v-faces; the y-edge at x-face x, z-face z its u- and w-faces; the x-edge at y-face y, z-face z
    // its v- and w-faces), so each is evaluated once per cell; the y- and x-edges on z-face z + 1, which the
    // cell's u- and v-faces reach, are the next row's corner edges and carry over in registers.  Every term is
    // the same expression on the same operands as when each face evaluated its own.
    static_assert(G::WARPS % TY == 0 && G::WARPS / TY * RPT == TZ, "a warp's rows are one column of the tile");
    T cyWo = T(0), cyU = T(0), cyUl = T(0), cyUh = T(0);     // y-edge (x, z + 1): weighted omega_y, u-face term, u
    T cxWo = T(0), cxV = T(0), cxVl = T(0), cxVh = T(0);     // x-edge (y, z + 1): weighted omega_x, v-face term, v
#pragma unroll 1
    for (int k = 0; k < RPT; k++) {
        const int ry = warp % TY, rz = RPT * (warp / TY) + k;
        const int x = x0 + lane, y = y0 + ry, z = z0 + rz;
        if (x >= nx || y >= ny || z >= nz) continue;
        const T* pu = SU + ((rz + 3) * UH + ry + 3) * UW + lane + 1;   // u at x-face x, cells (y, z)
        const T* pv = SV + ((rz + 3) * VH + ry + 1) * VW + lane + 3;   // v at cell x, y-face y, cell z
        const T* pw = SW + ((rz + 1) * WH + ry + 3) * WW + lane + 3;   // w at cells (x, y), z-face z
        const int mo = ((rz + 1) * MH + ry + 1) * MW + lane + 1;        // this cell's lower faces in the impulse boxes
        const T kc = Kc[kidx(lane + 1, ry + 1, rz + 1)];
        // the RK base of the three faces (stages 1, 2), loaded here so that the faces' arithmetic hides the wait
        const int iu = fidx<X>(p, x, y, z), iv = fidx<Y>(p, x, y, z), iw = fidx<Z>(p, x, y, z);
        const bool rk = a.stage > 0;
        const T bu = rk ? __ldg(a.m0[X] + iu) : T(0), bv = rk ? __ldg(a.m0[Y] + iv) : T(0),
                bw = rk ? __ldg(a.m0[Z] + iw) : T(0);

        // ---------------- the corner edges: narrow terms of two faces each
        T uZ0, vZ0, uY0, wY0, vX0, wX0, uY1, vX1;
        {
            const T ok1x = tX(kOk1, x), l1x = tX(kL1, x), i1x = tX(kInvSp, x), e1lx = tX(kEv1Lo, x), e1hx = tX(kEv1Hi, x);
            const T ok1y = tY(kOk1, y), l1y = tY(kL1, y), i1y = tY(kInvSp, y), e1ly = tY(kEv1Lo, y), e1hy = tY(kEv1Hi, y);
            const T e1lz = tZ(kEv1Lo, z), e1hz = tZ(kEv1Hi, z);
            {   // z-edge (x, y): + w omega_z ev_x(v) on the u-face, - w omega_z ev_y(u) on the v-face
                const T vl = pv[-1], vh = pv[0], ul = pu[-UW], uh = pu[0];
                const T wo = w1(ok1x, ok1y, l1x, l1y) * ((vh - vl) * i1x - (uh - ul) * i1y);
                uZ0 = wo * (e1lx * vl + e1hx * vh);
                vZ0 = -(wo * (e1ly * ul + e1hy * uh));
            }
            if (k == 0) {
                const T ok1z = tZ(kOk1, z), l1z = tZ(kL1, z), i1z = tZ(kInvSp, z);
                {   // y-edge (x, z): - w omega_y ev_x(w) on the u-face, + w omega_y ev_z(u) on the w-face
                    const T ul = pu[-UP], uh = pu[0], wl = pw[-1], wh = pw[0];
                    const T wo = w1(ok1z, ok1x, l1z, l1x) * ((uh - ul) * i1z - (wh - wl) * i1x);
                    uY0 = -(wo * (e1lx * wl + e1hx * wh));
                    wY0 = wo * (e1lz * ul + e1hz * uh);
                }
                {   // x-edge (y, z): + w omega_x ev_y(w) on the v-face, - w omega_x ev_z(v) on the w-face
                    const T wl = pw[-WW], wh = pw[0], vl = pv[-VP], vh = pv[0];
                    const T wo = w1(ok1y, ok1z, l1y, l1z) * ((wh - wl) * i1y - (vh - vl) * i1z);
                    vX0 = wo * (e1ly * wl + e1hy * wh);
                    wX0 = -(wo * (e1lz * vl + e1hz * vh));
                }
            } else {     // the previous row's edges on this cell's lower z-face
                uY0 = cyU;
                wY0 = cyWo * (e1lz * cyUl + e1hz * cyUh);
                vX0 = cxV;
                wX0 = -(cxWo * (e1lz * cxVl + e1hz * cxVh));
            }
            {   // the edges on z-face z + 1 (the next row's corner edges)
                const T ok1 = tZ(kOk1, z + 1), l1 = tZ(kL1, z + 1), i1 = tZ(kInvSp, z + 1);
                const T ul = pu[0], uh = pu[UP], wl = pw[WP - 1], wh = pw[WP];
                cyWo = w1(ok1, ok1x, l1, l1x) * ((uh - ul) * i1 - (wh - wl) * i1x);
                cyU = -(cyWo * (e1lx * wl + e1hx * wh));
                cyUl = ul;
                cyUh = uh;
                const T wl2 = pw[WP - WW], wh2 = pw[WP], vl = pv[0], vh = pv[VP];
                cxWo = w1(ok1y, ok1, l1y, l1) * ((wh2 - wl2) * i1y - (vh - vl) * i1);
                cxV = cxWo * (e1ly * wl2 + e1hy * wh2);
                cxVl = vl;
                cxVh = vh;
            }
            uY1 = cyU;
            vX1 = cxV;
        }

        // ---------------- u-face x: z-edges (b = Y, omega_z) and y-edges (b = Z, omega_y)
        {
            const int i = iu;
            if (blend) st_out(a.m0_out[X] + (i), MX[mo]);
            if (x == 0) st_out(a.out[X] + (i), T(0));
            else {
                const T ok1x = tX(kOk1, x), l1x = tX(kL1, x), l3x = tX(kL3, x), i1x = tX(kInvSp, x), i3x = tX(kInvNd3, x);
                const T e1l = tX(kEv1Lo, x), e1h = tX(kEv1Hi, x), e3l = tX(kEv3Lo, x), e3h = tX(kEv3Hi, x);
                // z-edge at y-face e (d = e - y): + w omega_z ev_x(v)
                auto pz1 = [&](int d) {
                    const int e = y + d;
                    const T vl = pv[d * VW - 1], vh = pv[d * VW], ul = pu[(d - 1) * UW], uh = pu[d * UW];
                    const T wo = w1(ok1x, tY(kOk1, e), l1x, tY(kL1, e)) * ((vh - vl) * i1x - (uh - ul) * tY(kInvSp, e));
                    return wo * (e1l * vl + e1h * vh);
                };
                auto pz3 = [&](int d) {
                    const int e = y + d;
                    const T vl = pv[d * VW - 2], vh = pv[d * VW + 1], ul = pu[(d - 2) * UW], uh = pu[(d + 1) * UW];
                    const T wo = w3(l3x, tY(kL3, e)) * ((vh - vl) * i3x - (uh - ul) * tY(kInvNd3, e));
                    return wo * (e3l * vl + e3h * vh);
                };
                // y-edge at z-face e (d = e - z): - w omega_y ev_x(w); the narrow ones are the corner edges
                auto py3 = [&](int d) {
                    const int e = z + d;
                    const T ul = pu[(d - 2) * UP], uh = pu[(d + 1) * UP], wl = pw[d * WP - 2], wh = pw[d * WP + 1];
                    const T wo = w3(tZ(kL3, e), l3x) * ((uh - ul) * tZ(kInvNd3, e) - (wh - wl) * i3x);
                    return -(wo * (e3l * wl + e3h * wh));
                };
                T L = half * (pz1(1) + uZ0) + half * (uY1 + uY0);
                if (o4) {
                    const T c3 = tX(kC3, x);
                    L = L + c3 * (pz3(2) + pz3(-1));
                    L = L + c3 * (py3(2) + py3(-1));
                }
                L = L - (kc - Kc[kidx(lane, ry + 1, rz + 1)]) * tX(kInvSp, x);
                st_out(a.out[X] + (i), viscous_rk_tile<X, T, MW, MH>(a, MX + mo, pu[0], sc, dt, lidv, x, y, z, bu, L, tX, tY, tZ));
            }
            if (x == nx - 1) {
                if (blend) st_out(a.m0_out[X] + (i + 1), MX[mo + 1]);
                st_out(a.out[X] + (i + 1), T(0));
            }
        }
        // ---------------- v-face y: z-edges (b = X, omega_z) and x-edges (b = Z, omega_x)
        {
            const int i = iv;
            if (blend) st_out(a.m0_out[Y] + (i), MY[mo]);
            if (y == 0) st_out(a.out[Y] + (i), T(0));
            else {
                const T ok1y = tY(kOk1, y), l1y = tY(kL1, y), l3y = tY(kL3, y), i1y = tY(kInvSp, y), i3y = tY(kInvNd3, y);
                const T e1l = tY(kEv1Lo, y), e1h = tY(kEv1Hi, y), e3l = tY(kEv3Lo, y), e3h = tY(kEv3Hi, y);
                // z-edge at x-face e (d = e - x): - w omega_z ev_y(u)
                auto pz1 = [&](int d) {
                    const int e = x + d;
                    const T vl = pv[d - 1], vh = pv[d], ul = pu[d - UW], uh = pu[d];
                    const T wo = w1(tX(kOk1, e), ok1y, tX(kL1, e), l1y) * ((vh - vl) * tX(kInvSp, e) - (uh - ul) * i1y);
                    return -(wo * (e1l * ul + e1h * uh));
                };
                auto pz3 = [&](int d) {
                    const int e = x + d;
                    const T vl = pv[d - 2], vh = pv[d + 1], ul = pu[d - 2 * UW], uh = pu[d + UW];
                    const T wo = w3(tX(kL3, e), l3y) * ((vh - vl) * tX(kInvNd3, e) - (uh - ul) * i3y);
                    return -(wo * (e3l * ul + e3h * uh));
                };
                // x-edge at z-face e (d = e - z): + w omega_x ev_y(w); the narrow ones are the corner edges
                auto px3 = [&](int d) {
                    const int e = z + d;
                    const T wl = pw[d * WP - 2 * WW], wh = pw[d * WP + WW], vl = pv[(d - 2) * VP], vh = pv[(d + 1) * VP];
                    const T wo = w3(l3y, tZ(kL3, e)) * ((wh - wl) * i3y - (vh - vl) * tZ(kInvNd3, e));
                    return wo * (e3l * wl + e3h * wh);
                };
                T L = half * (pz1(1) + vZ0) + half * (vX1 + vX0);
                if (o4) {
                    const T c3 = tY(kC3, y);
                    L = L + c3 * (pz3(2) + pz3(-1));
                    L = L + c3 * (px3(2) + px3(-1));
                }
                L = L - (kc - Kc[kidx(lane + 1, ry, rz + 1)]) * tY(kInvSp, y);
                st_out(a.out[Y] + (i), viscous_rk_tile<Y, T, MW, MH>(a, MY + mo, pv[0], sc, dt, lidv, x, y, z, bv, L, tX, tY, tZ));
            }
            if (y == ny - 1) {
                if (blend) st_out(a.m0_out[Y] + (i + nx), MY[mo + MW]);
                st_out(a.out[Y] + (i + nx), T(0));
            }
        }
        // ---------------- w-face z: x-edges (b = Y, omega_x) and y-edges (b = X, omega_y)
        {
            const int i = iw;
            if (blend) st_out(a.m0_out[Z] + (i), MZ[mo]);
            if (z == 0) st_out(a.out[Z] + (i), T(0));
            else {
                const T ok1z = tZ(kOk1, z), l1z = tZ(kL1, z), l3z = tZ(kL3, z), i1z = tZ(kInvSp, z), i3z = tZ(kInvNd3, z);
                const T e1l = tZ(kEv1Lo, z), e1h = tZ(kEv1Hi, z), e3l = tZ(kEv3Lo, z), e3h = tZ(kEv3Hi, z);
                // x-edge at y-face e (d = e - y): - w omega_x ev_z(v)
                auto px1 = [&](int d) {
                    const int e = y + d;
                    const T wl = pw[(d - 1) * WW], wh = pw[d * WW], vl = pv[d * VW - VP], vh = pv[d * VW];
                    const T wo = w1(tY(kOk1, e), ok1z, tY(kL1, e), l1z) * ((wh - wl) * tY(kInvSp, e) - (vh - vl) * i1z);
                    return -(wo * (e1l * vl + e1h * vh));
                };
                auto px3 = [&](int d) {
                    const int e = y + d;
                    const T wl = pw[(d - 2) * WW], wh = pw[(d + 1) * WW], vl = pv[d * VW - 2 * VP], vh = pv[d * VW + VP];
                    const T wo = w3(tY(kL3, e), l3z) * ((wh - wl) * tY(kInvNd3, e) - (vh - vl) * i3z);
                    return -(wo * (e3l * vl + e3h * vh));
                };
                // y-edge at x-face e (d = e - x): + w omega_y ev_z(u)
                auto py1 = [&](int d) {
                    const int e = x + d;
                    const T ul = pu[d - UP], uh = pu[d], wl = pw[d - 1], wh = pw[d];
                    const T wo = w1(ok1z, tX(kOk1, e), l1z, tX(kL1, e)) * ((uh - ul) * i1z - (wh - wl) * tX(kInvSp, e));
                    return wo * (e1l * ul + e1h * uh);
                };
                auto py3 = [&](int d) {
                    const int e = x + d;
                    const T ul = pu[d - 2 * UP], uh = pu[d + UP], wl = pw[d - 2], wh = pw[d + 1];
                    const T wo = w3(l3z, tX(kL3, e)) * ((uh - ul) * i3z - (wh - wl) * tX(kInvNd3, e));
                    return wo * (e3l * ul + e3h * uh);
                };
                T L = half * (px1(1) + wX0) + half * (py1(1) + wY0);
                if (o4) {
                    const T c3 = tZ(kC3, z);
                    L = L + c3 * (px3(2) + px3(-1));
                    L = L + c3 * (py3(2) + py3(-1));
                }
                L = L - (kc - Kc[kidx(lane + 1, ry + 1, rz)]) * tZ(kInvSp, z);
                st_out(a.out[Z] + (i), viscous_rk_tile<Z, T, MW, MH>(a, MZ + mo, pw[0], sc, dt, lidv, x, y, z, bw, L, tX, tY, tZ));
            }
            if (z == nz - 1) {
                if (blend) st_out(a.m0_out[Z] + (i + nx * ny), MZ[mo + MW * MH]);
                st_out(a.out[Z] + (i + nx * ny), T(0));
            }
        }
    }
}

template <class T, int TY, int TZ, int NT>
__global__ void __launch_bounds__(NT, 2) sweep_tile_kernel(MomentumArgs<T> a) {
    sweep_tile_body<T, TY, TZ, NT>(a, real_blk());
}
// a batch of cavities: grid x runs over the work list (BatchItem)
template <class T, int TY, int TZ, int NT>
__global__ void __launch_bounds__(NT, 2) sweep_tile_batched(const MomentumArgs<T>* args, const BatchItem* items,
                                                          const int* live) {
    __shared__ MomentumArgs<T> a;
    int cav;
    const Blk k = item_blk(items, live, cav);
    if (cav < 0) return;
    load_args(a, args + cav);
    sweep_tile_body<T, TY, TZ, NT>(a, k);
}

}  // namespace cavity
