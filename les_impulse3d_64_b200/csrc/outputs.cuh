// outputs.cuh - kernels behind the per-step getters and the kick: diagnostics, probes, mid-span statistics,
// centreline, mid-plane, Q criterion, and the smoothed random kick.  Same field layout as kernels.cuh.
#pragma once
#include "kernels.cuh"

namespace cavity {

enum DiagSlot : int { kSlotKE = 0, kSlotEns, kSlotDiv2, kSlotUmax0, kSlotGauge0 = kSlotUmax0 + 3,
                      kSlotGaugeIdx0 = kSlotGauge0 + 3, kSlotRms = kSlotGaugeIdx0 + 3, kNumSlots };
enum OutCounter : int { kCntDiag = 0, kCntMaxAbs, kCntGauge, kCntSumsq, kNumOutCounters };

template <class T> struct OutArgs {
    Params p;
    Geo<T> g;
    const T* u[3];
    const T* m[3];
    const double* centre_x;     // cell centres / faces (double, float-rounded) for lid shape at cells
    const double* centre_z;
    double length_x, length_z;  // (float)length as in the reference's device table
    int lid_shaped;
    double* slots;              // results
    double* partial;
    unsigned int* counters;
};

// velocity component cmp averaged to the centre of cell (x, y, z) (backend.cu:68-72)
template <class T>
__device__ __forceinline__ T centred(const OutArgs<T>& a, int cmp, int x, int y, int z) {
    const Params& p = a.p;
    if (cmp == 0) { const int i = fidx<X>(p, x, y, z); return T(0.5) * (a.u[X][i] + a.u[X][i + 1]); }
    if (cmp == 1) { const int i = fidx<Y>(p, x, y, z); return T(0.5) * (a.u[Y][i] + a.u[Y][i + p.nx]); }
    const int i = fidx<Z>(p, x, y, z);
    return T(0.5) * (a.u[Z][i] + a.u[Z][i + p.nx * p.ny]);
}

template <class T> __device__ __forceinline__ T lid_edge(T s) {                  // backend.cu:59
    const T s2 = s * s, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8, q = T(1) - s16 * s2;
    return q * q;
}
template <class T> __device__ __forceinline__ T lid_poly(T f) { const T g = f * (T(1) - f); return g * g; }
template <class T> __device__ __forceinline__ T lid_shape(int shaped, T fx, T fz) {   // backend.cu:60-63
    if (shaped == 2) return T(16) * lid_poly(fx) * lid_poly(fz);
    if (!shaped) return T(1);
    return lid_edge(T(2) * fx - T(1)) * lid_edge(T(2) * fz - T(1));
}

// g[i][j] = d u_j / d x_i at the centre of cell (x, y, z) with mirrored ghosts (backend.cu:76-96)
template <class T>
__device__ void cell_gradient(const OutArgs<T>& a, T lidv, int x, int y, int z, T g[3][3]) {
    const Params& p = a.p;
    const int q[3] = {x, y, z}, n[3] = {p.nx, p.ny, p.nz};
    T dm[3], dp[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        dm[d] = q[d] > 0 ? tab(a.g, d, kSp, q[d]) : tab(a.g, d, kW, 0);
        dp[d] = q[d] + 1 < n[d] ? tab(a.g, d, kSp, q[d] + 1) : tab(a.g, d, kW, n[d] - 1);
    }
    const T lid_cell = lid_shape<T>(a.lid_shaped, (T)a.centre_x[x] / (T)a.length_x, (T)a.centre_z[z] / (T)a.length_z);
#pragma unroll
    for (int cmp = 0; cmp < 3; cmp++) {
        const T c0 = centred(a, cmp, x, y, z);
        const T xm = x > 0 ? centred(a, cmp, x - 1, y, z) : -c0;
        const T xp = x + 1 < p.nx ? centred(a, cmp, x + 1, y, z) : -c0;
        const T ym = y > 0 ? centred(a, cmp, x, y - 1, z) : -c0;
        const T yp = y + 1 < p.ny ? centred(a, cmp, x, y + 1, z) : T(2) * (cmp == 0 ? lidv * lid_cell : T(0)) - c0;
        const T zp = z + 1 < p.nz ? centred(a, cmp, x, y, z + 1) : -c0;
        const T zm = z > 0 ? centred(a, cmp, x, y, z - 1) : -c0;
        g[0][cmp] = (xp - xm) / (dp[0] + dm[0]);
        g[1][cmp] = (yp - ym) / (dp[1] + dm[1]);
        g[2][cmp] = (zp - zm) / (dp[2] + dm[2]);
    }
    g[0][0] = (a.u[X][fidx<X>(p, x + 1, y, z)] - a.u[X][fidx<X>(p, x, y, z)]) / tab(a.g, X, kW, x);
    g[1][1] = (a.u[Y][fidx<Y>(p, x, y + 1, z)] - a.u[Y][fidx<Y>(p, x, y, z)]) / tab(a.g, Y, kW, y);
    g[2][2] = (a.u[Z][fidx<Z>(p, x, y, z + 1)] - a.u[Z][fidx<Z>(p, x, y, z)]) / tab(a.g, Z, kW, z);
}

// per cell: kinetic energy, enstrophy, divergence^2, each times the volume; summed (backend.cu:447-463)
template <class T>
__global__ void __launch_bounds__(kThreads) cell_diag_kernel(OutArgs<T> a, T lidv) {
    const Params& p = a.p;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    Vec<3> acc;
    acc.v[0] = acc.v[1] = acc.v[2] = 0.0;
    if (i < p.n_cell) {
        const int x = i % p.nx, y = (i / p.nx) % p.ny, z = i / (p.nx * p.ny);
        const double vol = a.g.dw[X][x] * a.g.dw[Y][y] * a.g.dw[Z][z];
        const double cu = centred(a, 0, x, y, z), cv = centred(a, 1, x, y, z), cw = centred(a, 2, x, y, z);
        acc.v[0] = 0.5 * (cu * cu + cv * cv + cw * cw) * vol;
        T g[3][3];
        cell_gradient(a, lidv, x, y, z, g);
        const T ox = g[1][2] - g[2][1], oy = g[2][0] - g[0][2], oz = g[0][1] - g[1][0];
        acc.v[1] = (double)(ox * ox + oy * oy + oz * oz) * vol;
        const double d = (double)(a.u[X][fidx<X>(p, x + 1, y, z)] - a.u[X][fidx<X>(p, x, y, z)]) / a.g.dw[X][x] +
                         (double)(a.u[Y][fidx<Y>(p, x, y + 1, z)] - a.u[Y][fidx<Y>(p, x, y, z)]) / a.g.dw[Y][y] +
                         (double)(a.u[Z][fidx<Z>(p, x, y, z + 1)] - a.u[Z][fidx<Z>(p, x, y, z)]) / a.g.dw[Z][z];
        acc.v[2] = d * d * vol;
    }
    const Vec<3> blk = block_reduce<3, false>(acc);
    if (publish_partials(blk, a.partial, &a.counters[kCntDiag])) {
        const Vec<3> tot = final_reduce<3, false>(a.partial);
        if (threadIdx.x == 0) {
            a.counters[kCntDiag] = 0;
            a.slots[kSlotKE] = tot.v[0];
            a.slots[kSlotEns] = tot.v[1];
            a.slots[kSlotDiv2] = tot.v[2];
        }
    }
}

// max |u_comp| (backend.cu:1106) and, for the gauge diagnostic, max |m - u| with the first index holding it
// (backend.cu:1111-1122).  One launch per component; blockIdx.y = 0: |u|, 1: |m - u|.
struct MaxIdx { double v; long long i; };
__device__ __forceinline__ MaxIdx better(MaxIdx a, MaxIdx b) {
    if (a.v != a.v) return a;
    if (b.v != b.v) return b;
    if (a.v > b.v) return a;
    if (b.v > a.v) return b;
    return a.i <= b.i ? a : b;
}
template <class T>
__global__ void __launch_bounds__(kThreads) max_abs_kernel(OutArgs<T> a, int comp, long long n, double* part2) {
    const long long i = blockIdx.x * (long long)kThreads + threadIdx.x;
    MaxIdx um{-INFINITY, 0}, gm{-INFINITY, 0};
    if (i < n) {
        um.v = (double)fabs(a.u[comp][i]);
        um.i = i;
        gm.v = (double)fabs(a.m[comp][i] - a.u[comp][i]);
        gm.i = i;
    }
    __shared__ MaxIdx sh[2][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        MaxIdx t1{__shfl_down_sync(0xffffffffu, um.v, o), __shfl_down_sync(0xffffffffu, um.i, o)};
        MaxIdx t2{__shfl_down_sync(0xffffffffu, gm.v, o), __shfl_down_sync(0xffffffffu, gm.i, o)};
        if (lane + o < 32) { um = better(um, t1); gm = better(gm, t2); }
    }
    if (lane == 0) { sh[0][warp] = um; sh[1][warp] = gm; }
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        MaxIdx bu = sh[0][0], bg = sh[1][0];
        for (int w = 1; w < kThreads / 32; w++) { bu = better(bu, sh[0][w]); bg = better(bg, sh[1][w]); }
        const unsigned int nb = gridDim.x;
        a.partial[blockIdx.x] = bu.v;
        part2[blockIdx.x] = bg.v;
        ((long long*)(a.partial + nb))[blockIdx.x] = bu.i;
        ((long long*)(part2 + nb))[blockIdx.x] = bg.i;
        __threadfence();
        last = atomicAdd(&a.counters[kCntMaxAbs], 1u) == nb - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const unsigned int nb = gridDim.x;
        MaxIdx bu{-INFINITY, 0}, bg{-INFINITY, 0};
        for (unsigned int b = 0; b < nb; b++) {
            bu = better(bu, MaxIdx{__ldcg(a.partial + b), __ldcg((const long long*)(a.partial + nb) + b)});
            bg = better(bg, MaxIdx{__ldcg(part2 + b), __ldcg((const long long*)(part2 + nb) + b)});
        }
        a.slots[kSlotUmax0 + comp] = bu.v;
        a.slots[kSlotGauge0 + comp] = bg.v;
        a.slots[kSlotGaugeIdx0 + comp] = (double)(bg.v == bg.v ? bg.i : 2147483647LL);
        a.counters[kCntMaxAbs] = 0;
    }
}

// probe values: u and v at the centre of each probe cell (backend.cu:534-540)
template <class T>
__global__ void probes_kernel(OutArgs<T> a, const int* cells, int n, float* out) {
    const int k = threadIdx.x;
    if (k >= n) return;
    const int x = cells[3 * k], y = cells[3 * k + 1], z = cells[3 * k + 2];
    out[2 * k] = (float)centred(a, 0, x, y, z);
    out[2 * k + 1] = (float)centred(a, 1, x, y, z);
}

// After a step (single cavities): the probe values and the control block into pinned, mapped host memory, so that
// the blocking per-step calls of the reference's front end (solver_step's report, solver_probes) read host memory
// after the step's one wait instead of each queueing a copy and waiting again.
template <class T>
__global__ void step_tail_kernel(OutArgs<T> a, const int* cells, int n, float* probes, const Control* c, Control* c_host) {
    const int k = threadIdx.x;
    if (k < n) {
        const int x = cells[3 * k], y = cells[3 * k + 1], z = cells[3 * k + 2];
        probes[2 * k] = (float)centred(a, 0, x, y, z);
        probes[2 * k + 1] = (float)centred(a, 1, x, y, z);
    }
    const int* src = reinterpret_cast<const int*>(c);
    int* dst = reinterpret_cast<int*>(c_host);
    for (int i = k; i < (int)(sizeof(Control) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
}

// mid-span layers: the plane z = LZ/2 lies between k1 and k2 (backend.cu:488)
__device__ __forceinline__ void midspan_layers(int nz, int& k1, int& k2) { k2 = nz / 2; k1 = (nz % 2) ? k2 : k2 - 1; }

// weighted running sums of u, v, uu, vv, ww, uv on the mid-span plane (backend.cu:507-517) and the
// centreline sample (backend.cu:519-532); threads [0, nx*ny) do the sums, the next nx the centreline.  With a
// control block `wc` the weight is the dt of the step just taken, read on the device (queued outputs), and a
// failed step adds nothing.
template <class T>
__global__ void statistics_kernel(OutArgs<T> a, double weight, const Control* wc, double* sums, double* centreline) {
    if (wc) {
        if (wc->error) return;
        weight = wc->last_dt;
    }
    const Params& p = a.p;
    const int t = blockIdx.x * kThreads + threadIdx.x;
    const int n = p.nx * p.ny;
    int k1, k2;
    midspan_layers(p.nz, k1, k2);
    auto C = [&](int c, int x, int y, int z) { return (double)centred(a, c, x, y, z); };
    if (t < n) {
        const int x = t % p.nx, y = t / p.nx;
        const double cu = 0.5 * (C(0, x, y, k1) + C(0, x, y, k2));
        const double cv = 0.5 * (C(1, x, y, k1) + C(1, x, y, k2));
        const double cw = 0.5 * (C(2, x, y, k1) + C(2, x, y, k2));
        sums[t] += weight * cu;
        sums[n + t] += weight * cv;
        sums[2 * n + t] += weight * (cu * cu);
        sums[3 * n + t] += weight * (cv * cv);
        sums[4 * n + t] += weight * (cw * cw);
        sums[5 * n + t] += weight * (cu * cv);
    } else if (t < n + p.nx) {
        const int j = t - n, mid = p.nx / 2;
        auto mean4 = [&](int c, int xa, int ya, int xb, int yb) {
            return 0.5 * (0.5 * (C(c, xa, ya, k1) + C(c, xa, ya, k2)) + 0.5 * (C(c, xb, yb, k1) + C(c, xb, yb, k2)));
        };
        const double cu = mean4(0, mid - 1, j, mid, j), cv = mean4(1, j, mid - 1, j, mid), cw = mean4(2, mid - 1, j, mid, j);
        centreline[j] = cu;
        centreline[p.nx + j] = cv;
        centreline[2 * p.nx + j] = cu * cu;
        centreline[3 * p.nx + j] = cv * cv;
        centreline[4 * p.nx + j] = cw * cw;
    }
}

// mid-span plane [u | v | w | |omega|] (backend.cu:490-505)
template <class T>
__global__ void midplane_kernel(OutArgs<T> a, T lidv, float* out) {
    const Params& p = a.p;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= p.nx * p.ny) return;
    const int x = i % p.nx, y = i / p.nx;
    int k1, k2;
    midspan_layers(p.nz, k1, k2);
    T val[2][4];
    for (int s = 0; s < 2; s++) {
        const int z = s ? k2 : k1;
        for (int c = 0; c < 3; c++) val[s][c] = centred(a, c, x, y, z);
        T g[3][3];
        cell_gradient(a, lidv, x, y, z, g);
        const T o1 = g[1][2] - g[2][1], o2 = g[2][0] - g[0][2], o3 = g[0][1] - g[1][0];
        val[s][3] = sqrt(o1 * o1 + o2 * o2 + o3 * o3);
    }
    for (int c = 0; c < 4; c++)
        out[c * p.nx * p.ny + i] = (float)((k1 == k2) ? val[1][c] : T(0.5) * (val[0][c] + val[1][c]));
}

// Q criterion (Q L^2/U^2) and a colour (w/U or |u|/U) per cell (backend.cu:474-486)
template <class T>
__global__ void __launch_bounds__(kThreads) q_kernel(OutArgs<T> a, T lidv, T qscale, T inv_U, int colour_w,
                                                     float* q, float* colour) {
    const Params& p = a.p;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= p.n_cell) return;
    const int x = i % p.nx, y = (i / p.nx) % p.ny, z = i / (p.nx * p.ny);
    T g[3][3];
    cell_gradient(a, lidv, x, y, z, g);
    T s = T(0);
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) s += g[r][c] * g[c][r];
    q[i] = (float)(T(-0.5) * s * qscale);
    const T cu = centred(a, 0, x, y, z), cv = centred(a, 1, x, y, z), cw = centred(a, 2, x, y, z);
    colour[i] = (float)(colour_w ? cw * inv_U : sqrt(cu * cu + cv * cv + cw * cw) * inv_U);
}

// ------------------------------------------------------------------------------------------ kick
// one periodic 1-2-1 smoothing pass along `axis` of an (sx, sy, sz) array (backend.cu:544-553)
__global__ void smooth_kernel(const double* in, double* out, int axis, int sx, int sy, int sz) {
    const long long i = blockIdx.x * (long long)kThreads + threadIdx.x;
    if (i >= (long long)sx * sy * sz) return;
    const int x = i % sx, y = (i / sx) % sy, z = i / ((long long)sx * sy);
    long long lo, hi;
    if (axis == 0) { lo = (x + sx - 1) % sx + sx * (y + (long long)sy * z); hi = (x + 1) % sx + sx * (y + (long long)sy * z); }
    else if (axis == 1) { lo = x + sx * ((y + sy - 1) % sy + (long long)sy * z); hi = x + sx * ((y + 1) % sy + (long long)sy * z); }
    else { lo = x + sx * (y + (long long)sy * ((z + sz - 1) % sz)); hi = x + sx * (y + (long long)sy * ((z + 1) % sz)); }
    out[i] = 0.25 * in[lo] + 0.5 * in[i] + 0.25 * in[hi];
}
// sum of squares of a double array into slots[kSlotRms] (backend.cu:969)
__global__ void __launch_bounds__(kThreads) sumsq_kernel(const double* x, long long n, double* slots, double* partial,
                                                         unsigned int* counters) {
    const long long i = blockIdx.x * (long long)kThreads + threadIdx.x;
    Vec<1> acc;
    acc.v[0] = i < n ? x[i] * x[i] : 0.0;
    const Vec<1> blk = block_reduce<1, false>(acc);
    if (publish_partials(blk, partial, &counters[kCntSumsq])) {
        const Vec<1> tot = final_reduce<1, false>(partial);
        if (threadIdx.x == 0) {
            counters[kCntSumsq] = 0;
            slots[kSlotRms] = tot.v[0];
        }
    }
}
// out = f + noise * amp*U/max(rms, 1e-30), rms from the sum of squares (backend.cu:554-557, 969-970)
template <class T>
__global__ void add_noise_kernel(const T* f, const double* noise, const double* slots, double amp_u, long long n, T* out) {
    const long long i = blockIdx.x * (long long)kThreads + threadIdx.x;
    if (i >= n) return;
    const double rms = sqrt(slots[kSlotRms] / n);
    const double s = amp_u / fmax(rms, 1e-30);
    out[i] = f[i] + (T)(noise[i] * s);
}
// m += new_u - u; u = new_u (backend.cu:973-976)
template <class T>
__global__ void kick_update_kernel(T* m, T* u, const T* new_u, long long n) {
    const long long i = blockIdx.x * (long long)kThreads + threadIdx.x;
    if (i >= n) return;
    m[i] = m[i] + (new_u[i] - u[i]);
    u[i] = new_u[i];
}

}  // namespace cavity
