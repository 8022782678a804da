// =====================================================================================================
//  cavity_oracle.cpp - TEST INFRASTRUCTURE: the parity oracle and the CPU baseline.  Not part of the product.
//
//  A CPU restatement (C++17, OpenMP) of the reference solver's setup and time step: backend.cu of
//  LES_IMPULSE3D_64 (the Eulerian-impulse lid-driven cavity).  Every function names the backend.cu lines it
//  follows.  It exports the same 18 `solver_*` C functions as backend.cu (backend.cu:980-1195), so the
//  ctypes binding that drives the B200 build drives this file too.
//
//  Build (oracle/build_oracle.py):  g++ -O2 -fopenmp -ffp-contract=off -DORACLE_REAL=double|float
//    * ORACLE_REAL=double: the FP64 oracle.  Velocity and impulse carried in double; the pressure transforms
//      use the eigenvectors in double (not rounded to float) and no rms rescaling.  The grid tables keep the
//      reference's float rounding (backend.cu:695-697) and the CFL rate and viscous rate keep its float casts
//      (backend.cu:886, 1030-1034), so dt and dt_reason take the same decisions.
//    * ORACLE_REAL=float: the same code with the fields in float, the arithmetic the reference performs on
//      the GPU (`--fmad=false` there, `-ffp-contract=off` here).  The pressure transforms, done by cuBLAS SGEMM
//      in the reference, are accumulated in double and rounded to float here.
//  Pinning: tests/golden/*.npz hold outputs of the reference's own backend.cu (built unchanged for sm_100a
//  and run on a B200 by tests/golden/make_golden.py); tests/test_oracle.py checks both builds against them.
//
//  The one addition to the reference: lid_shaped = 2 selects the polynomial lid 16 x^2(1-x)^2 z^2(1-z)^2
//  (x, z as fractions of the lid), a shape the reference does not have (backend.cu:58-63).
//
//  Arrays are [z][y][x], x fastest.  u lives on x-faces (nx+1, ny, nz), v on y-faces, w on z-faces.
// =====================================================================================================
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#ifndef ORACLE_REAL
#define ORACLE_REAL double
#endif
typedef ORACLE_REAL Real;
static const bool kFloatMode = sizeof(Real) == 4;

using std::vector;
static const int GMAX = 1024;
static const int X = 0, Y = 1, Z = 2;

// ---------------------------------------------------------------- ABI records (backend.cu:584-597)
struct Config {
    int nx, ny, nz, lid_shaped, impulse_order, adaptive_dt, dt_lag, phi_extrapolate, fdm_max_passes, grid_stretch,
        n_probes;
    double length, u_lid, nu, lz, lid_ramp_t, reinit_r, impulse_order4_ramp, grid_dx_wall, grid_max_aspect;
    double dt_fixed, dt_max, cfl_target, diffusion_limit, fdm_rtol;
    double probe_x[8], probe_y[8];
};
struct Report {
    long long steps;
    double time, dt, cfl, phi_rel;
    int dt_reason, phi_passes;
};
struct Diagnostics {
    double kinetic_energy, enstrophy, umax, div_rms, cfl_rate, gauge_ratio, gauge_x, gauge_y;
};

static void fail(const std::string& m) { throw std::runtime_error(m); }

// ---------------------------------------------------------------- deterministic reductions
// Fixed chunks summed in order, whatever the thread count (the reference reduces on the GPU in its own order,
// backend.cu:427-443, 631-640; order only changes the last bits).
template <class F> static double det_sum(long long n, F f) {
    const long long CH = 4096;
    long long nch = (n + CH - 1) / CH;
    vector<double> part(std::max(nch, 1LL), 0.0);
#pragma omp parallel for schedule(static)
    for (long long c = 0; c < nch; c++) {
        double s = 0;
        long long e = std::min(n, (c + 1) * CH);
        for (long long i = c * CH; i < e; i++) s += f(i);
        part[c] = s;
    }
    double s = 0;
    for (long long c = 0; c < nch; c++) s += part[c];
    return s;
}
// max with NaN winning (backend.cu:427-429)
static double nan_max(double a, double b) { return (a != a || a > b) ? a : b; }
template <class F> static double det_max(long long n, F f) {
    double r = -INFINITY;
    for (long long i = 0; i < n; i++) r = nan_max(r, f(i));
    return r;
}

// ---------------------------------------------------------------- grid (backend.cu:643-699)
struct Axis {
    int n;
    double length;
    vector<double> face, centre, width, spacing;
};
static vector<double> linspace(double a, double b, int count) {                  // backend.cu:643-649
    vector<double> v(count);
    double step = (b - a) / (count - 1);
    for (int i = 0; i < count; i++) v[i] = i * step + a;
    v[count - 1] = b;
    return v;
}
static vector<double> stretched_faces(int n, double length, double dx_wall) {     // backend.cu:651-666
    if (dx_wall >= length / n * (1 - 1e-12)) return linspace(0.0, length, n + 1);
    vector<double> xi = linspace(0.0, 1.0, n + 1), f(n + 1);
    auto fill = [&](double beta) {
        for (int i = 0; i <= n; i++) f[i] = length * 0.5 * (1.0 + std::tanh(beta * (2 * xi[i] - 1)) / std::tanh(beta));
    };
    double lo = 1e-8, hi = 30.0;
    for (int it = 0; it < 200; it++) {
        double mid = 0.5 * (lo + hi);
        fill(mid);
        if (f[1] - f[0] < dx_wall) hi = mid;
        else lo = mid;
    }
    fill(0.5 * (lo + hi));
    f[0] = 0.0;
    f[n] = length;
    f[n / 2] = 0.5 * length;
    return f;
}
static double largest_over_smallest(const vector<double>& f) {                    // backend.cu:667-671
    double big = 0, small = 1e300;
    for (size_t i = 1; i < f.size(); i++) {
        big = std::max(big, f[i] - f[i - 1]);
        small = std::min(small, f[i] - f[i - 1]);
    }
    return big / small;
}
static Axis make_axis(const Config& c, int n, double length) {                    // backend.cu:672-699
    vector<double> f;
    if (!c.grid_stretch) f = stretched_faces(n, length, 1e300);
    else {
        double d = std::min(c.grid_dx_wall, length / n);
        auto ratio = [&](double dw) { return largest_over_smallest(stretched_faces(n, length, dw)); };
        if (c.grid_max_aspect > 0 && ratio(d) > c.grid_max_aspect) {
            double lo = d, hi = length / n;
            for (int it = 0; it < 60; it++) {
                double mid = 0.5 * (lo + hi);
                if (ratio(mid) > c.grid_max_aspect) lo = mid;
                else hi = mid;
            }
            d = hi;
        }
        f = stretched_faces(n, length, d);
    }
    Axis a;
    a.n = n;
    a.face = f;
    a.width.resize(n);
    a.centre.resize(n);
    a.spacing.resize(n + 1);
    for (int i = 0; i < n; i++) {
        a.width[i] = f[i + 1] - f[i];
        a.centre[i] = 0.5 * (f[i + 1] + f[i]);
    }
    for (int i = 1; i < n; i++) a.spacing[i] = a.centre[i] - a.centre[i - 1];
    a.spacing[0] = 0.5 * a.width[0];
    a.spacing[n] = 0.5 * a.width[n - 1];
    a.length = f[n] - f[0];
    for (vector<double>* v : {&a.face, &a.centre, &a.width, &a.spacing})
        for (double& q : *v) q = (double)(float)q;
    return a;
}

// ---------------------------------------------------------------- FDM set-up (backend.cu:723-787)
static void jacobi_eigen(int n, vector<double>& A, vector<double>& V) {           // backend.cu:723-746
    auto a = [&](int i, int j) -> double& { return A[(size_t)i * n + j]; };
    auto v = [&](int i, int j) -> double& { return V[(size_t)i * n + j]; };
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) v(i, i) = 1.0;
    double total = 0;
    for (double q : A) total += q * q;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                if (i != j) off += a(i, j) * a(i, j);
        if (off <= 1e-28 * total) return;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) {
                if (a(p, q) == 0.0) continue;
                double theta = (a(q, q) - a(p, p)) / (2 * a(p, q));
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                double cs = 1 / std::sqrt(t * t + 1), sn = t * cs;
                for (int k = 0; k < n; k++) {
                    double x = a(k, p), y = a(k, q);
                    a(k, p) = cs * x - sn * y;
                    a(k, q) = sn * x + cs * y;
                }
                for (int k = 0; k < n; k++) {
                    double x = a(p, k), y = a(q, k);
                    a(p, k) = cs * x - sn * y;
                    a(q, k) = sn * x + cs * y;
                }
                for (int k = 0; k < n; k++) {
                    double x = v(k, p), y = v(k, q);
                    v(k, p) = cs * x - sn * y;
                    v(k, q) = sn * x + cs * y;
                }
            }
    }
    fail("pressure solver set-up: eigenvalues did not converge");
}

// ---------------------------------------------------------------- the oracle solver
struct History {
    double t, scale;
    int buf;
};

struct Oracle {
    Config c;
    int nx, ny, nz, n_cell, size[3], dims[3][3];    // dims[comp] = array extent (x, y, z) of component comp
    Axis ax[3];
    double volume;
    float viscous_rate;
    // grid tables in the field precision (values already rounded through float)
    vector<Real> FACE[3], CENTRE[3], WIDTH[3], SPACING[3];
    Real LENGTH[3];
    vector<Real> u[3], m[3], m0[3], I[3], nm[3], nu_[3], tmp[3];
    vector<double> phi, phi0, base, guess, rhs, res, phi_new, hist_buf[4], stats;
    vector<Real> S[3];                       // eigenvectors per axis, S[a][i*n+j] (float-rounded in float mode)
    vector<Real> inv_lambda;
    int probe_cell[8][3];
    double t = 0, last_dt = 0, last_cfl = 0, phi_rel = 0, prev_rates[2] = {0, 0};
    long long steps = 0;
    int dt_reason = 0, phi_passes = 0;
    bool have_prev_rates = false;
    vector<History> hist;

    double lid(double time) const {                                            // backend.cu:623-626
        if (c.lid_ramp_t > 0) return c.u_lid * std::min(1.0, std::max(time, 0.0) / c.lid_ramp_t);
        return c.u_lid;
    }
    // flat index of component comp at (x, y, z)
    long long at(int comp, int x, int y, int z) const {
        return x + (long long)dims[comp][0] * (y + (long long)dims[comp][1] * z);
    }
    long long cell(int x, int y, int z) const { return x + (long long)nx * (y + (long long)ny * z); }

    // ------------------------------------------------------------ small helpers (backend.cu:55-96)
    Real width(int a, int i) const { return WIDTH[a][i]; }
    Real spacing(int a, int i) const { return SPACING[a][i]; }
    static Real lid_edge(Real s) {                                              // backend.cu:59
        Real s2 = s * s, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8, a = Real(1) - s16 * s2;
        return a * a;
    }
    static Real lid_poly(Real f) { Real g = f * (Real(1) - f); return g * g; }
    Real lid_shape(Real fx, Real fz) const {                                    // backend.cu:60-63
        if (c.lid_shaped == 2) return Real(16) * lid_poly(fx) * lid_poly(fz);
        if (!c.lid_shaped) return Real(1);
        return lid_edge(Real(2) * fx - Real(1)) * lid_edge(Real(2) * fz - Real(1));
    }
    Real lid_at_u_face(int x, int z) const { return lid_shape(FACE[X][x] / LENGTH[X], CENTRE[Z][z] / LENGTH[Z]); }
    Real lid_at_cell(int x, int z) const { return lid_shape(CENTRE[X][x] / LENGTH[X], CENTRE[Z][z] / LENGTH[Z]); }

    // component cmp of velocity field `f` averaged to the centre of cell (x, y, z)  (backend.cu:68-72)
    Real centred(const vector<Real>* f, int cmp, int x, int y, int z) const {
        int p[3] = {x, y, z};
        long long lo = at(cmp, x, y, z);
        p[cmp]++;
        long long hi = at(cmp, p[0], p[1], p[2]);
        return Real(0.5) * (f[cmp][lo] + f[cmp][hi]);
    }
    // velocity gradient g[i][j] = d u_j / d x_i at a cell centre with mirrored ghosts (backend.cu:76-96)
    void cell_gradient(const vector<Real>* f, Real lidv, int x, int y, int z, Real g[3][3]) const {
        int p[3] = {x, y, z}, n[3] = {nx, ny, nz};
        Real dm[3], dp[3];
        for (int a = 0; a < 3; a++) {
            dm[a] = p[a] > 0 ? spacing(a, p[a]) : width(a, 0);
            dp[a] = p[a] + 1 < n[a] ? spacing(a, p[a] + 1) : width(a, n[a] - 1);
        }
        for (int cmp = 0; cmp < 3; cmp++) {
            Real q = centred(f, cmp, x, y, z);
            for (int a = 0; a < 3; a++) {
                int lo[3] = {x, y, z}, hi[3] = {x, y, z};
                lo[a]--;
                hi[a]++;
                Real vm = p[a] > 0 ? centred(f, cmp, lo[0], lo[1], lo[2]) : -q;
                Real vp;
                if (p[a] + 1 < n[a]) vp = centred(f, cmp, hi[0], hi[1], hi[2]);
                else if (a == Y) vp = Real(2) * (cmp == 0 ? lidv * lid_at_cell(x, z) : Real(0)) - q;
                else vp = -q;
                g[a][cmp] = (vp - vm) / (dp[a] + dm[a]);
            }
        }
        for (int a = 0; a < 3; a++) {
            int hi[3] = {x, y, z};
            hi[a]++;
            g[a][a] = (f[a][at(a, hi[0], hi[1], hi[2])] - f[a][at(a, x, y, z)]) / width(a, p[a]);
        }
    }

    // ------------------------------------------------------------ inviscid term I (backend.cu:102-274)
    // Written once for all three face directions.  For faces normal to axis a and a tangential axis b, the
    // Lamb vector collects (d u_b/d x_a - d u_a/d x_b) times u_b on the edges bounding the face along b; the
    // reference's six lamb_<vorticity>_<axis> functions are the six (a, b) pairs, and their signs cancel
    // (backend.cu:140-215 with 235-236, 252-253, 269-270), so the sums below are the same IEEE operations.
    static bool stencil(int e, int q, int n, int& lo, int& hi) {                // backend.cu:108-112
        lo = e - (q + 1) / 2;
        hi = e + (q - 1) / 2;
        return lo >= 0 && hi <= n - 1;
    }
    Real node_distance(int a, int e, int q, int lo, int hi) const {            // backend.cu:114-117
        if (q == 1) return spacing(a, e);
        return CENTRE[a][hi] - CENTRE[a][lo];
    }
    Real edge_value(int a, int e, int q, int lo, int hi, Real flo, Real fhi) const {   // backend.cu:119-122
        if (q == 1) return (width(a, lo) * flo + width(a, hi) * fhi) / (Real(2) * spacing(a, e));
        return (width(a, lo) * flo + width(a, hi) * fhi) / (width(a, lo) + width(a, hi));
    }
    Real edge_weight_width(int a, int e, int q, int n) const {                 // backend.cu:124-128
        int lo, hi;
        if (q == 1 || !stencil(e, q, n, lo, hi)) return spacing(a, e);
        return Real(0.5) * (width(a, lo) + width(a, hi));
    }
    static Real wall_ramp(int e, int n, Real K) {                              // backend.cu:130-133
        Real d = (Real)(e < n - e ? e : n - e) - Real(1);
        return std::min(std::max(d / K, Real(0)), Real(1));
    }
    static Real stencil_weight(int q, int o4, Real s) {                         // backend.cu:135-138
        if (q == 1) return o4 ? Real(1) + s * Real(0.125) : Real(1);
        return -s * Real(0.125);
    }
    // one Lamb edge term for faces normal to a: edge at a-face ia, b-face e, d-cell id  (backend.cu:141-215)
    Real lamb_edge(const vector<Real>* vel, int a, int b, int ia, int e, int id, int q, int o4, Real K) const {
        int n[3] = {nx, ny, nz};
        int d = 3 - a - b, al, ah, bl, bh;
        if (e < 0 || e > n[b] || !stencil(ia, q, n[a], al, ah)) return Real(0);
        Real wq = stencil_weight(q, o4, wall_ramp(e, n[b], K) * wall_ramp(ia, n[a], K));
        if (wq == Real(0)) return Real(0);
        if (!stencil(e, q, n[b], bl, bh)) return Real(0);
        int p[3];
        // u_b at a-cells al / ah on b-face e
        p[a] = al; p[b] = e; p[d] = id;
        Real ub_lo = vel[b][at(b, p[0], p[1], p[2])];
        p[a] = ah;
        Real ub_hi = vel[b][at(b, p[0], p[1], p[2])];
        // u_a at a-face ia on b-cells bl / bh
        p[a] = ia; p[b] = bl;
        Real ua_lo = vel[a][at(a, p[0], p[1], p[2])];
        p[b] = bh;
        Real ua_hi = vel[a][at(a, p[0], p[1], p[2])];
        Real o = (ub_hi - ub_lo) / node_distance(a, ia, q, al, ah) - (ua_hi - ua_lo) / node_distance(b, e, q, bl, bh);
        if (o == Real(0)) return Real(0);
        return wq * o * edge_value(a, ia, q, al, ah, ub_lo, ub_hi);
    }
    // K = u.m at a cell centre (backend.cu:218-222)
    Real K_cell(const vector<Real>* vel, const vector<Real>* imp, int x, int y, int z) const {
        long long a0 = at(0, x, y, z), b0 = at(1, x, y, z), c0 = at(2, x, y, z);
        long long a1 = at(0, x + 1, y, z), b1 = at(1, x, y + 1, z), c1 = at(2, x, y, z + 1);
        return Real(0.5) * ((vel[0][a0] * imp[0][a0] + vel[0][a1] * imp[0][a1]) +
                            (vel[1][b0] * imp[1][b0] + vel[1][b1] * imp[1][b1]) +
                            (vel[2][c0] * imp[2][c0] + vel[2][c1] * imp[2][c1]));
    }
    // I on the faces normal to a (backend.cu:225-274): tangential axes in the reference's order
    void inviscid(int a, const vector<Real>* vel, const vector<Real>* imp, int o4, Real K, vector<Real>& out) const {
        static const int order[3][2] = {{Y, Z}, {X, Z}, {Y, X}};
        int n[3] = {nx, ny, nz};
        const int* dm = dims[a];
#pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < dm[2]; z++)
            for (int y = 0; y < dm[1]; y++)
                for (int x = 0; x < dm[0]; x++) {
                    int p[3] = {x, y, z};
                    long long i = at(a, x, y, z);
                    if (p[a] == 0 || p[a] == n[a]) { out[i] = Real(0); continue; }
                    Real L = Real(0);
                    for (int q = 1; q <= (o4 ? 3 : 1); q += 2) {
                        int up = (q + 1) / 2, down = (q - 1) / 2;
                        Real cq = edge_weight_width(a, p[a], q, n[a]) / (Real(2) * spacing(a, p[a]));
                        for (int k = 0; k < 2; k++) {
                            int b = order[a][k], d = 3 - a - b;
                            L += cq * (lamb_edge(vel, a, b, p[a], p[b] + up, p[d], q, o4, K) +
                                       lamb_edge(vel, a, b, p[a], p[b] - down, p[d], q, o4, K));
                        }
                    }
                    int lo[3] = {x, y, z};
                    lo[a]--;
                    L -= (K_cell(vel, imp, x, y, z) - K_cell(vel, imp, lo[0], lo[1], lo[2])) / spacing(a, p[a]);
                    out[i] = L;
                }
    }

    // ------------------------------------------------------------ RK3 stage (backend.cu:279-330)
    void rk3_stage(int a, const vector<Real>& mm, const vector<Real>& mb, const vector<Real>& vel,
                   const vector<Real>& In, Real nu, Real lidv, Real dt, Real a0, Real b, int has_base,
                   vector<Real>& out) const {
        int n[3] = {nx, ny, nz};
        const int* dm = dims[a];
        long long stride[3] = {1, dm[0], (long long)dm[0] * dm[1]};
#pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < dm[2]; z++)
            for (int y = 0; y < dm[1]; y++)
                for (int x = 0; x < dm[0]; x++) {
                    int p[3] = {x, y, z};
                    long long i = at(a, x, y, z);
                    if (p[a] == 0 || p[a] == n[a]) { out[i] = Real(0); continue; }
                    Real cc = mm[i], wall = vel[i], lap = Real(0);
                    for (int t = 0; t < 3; t++) {
                        long long s = stride[t];
                        if (t == a) {
                            lap += ((mm[i + s] - cc) / width(t, p[t]) - (cc - mm[i - s]) / width(t, p[t] - 1)) /
                                   spacing(t, p[t]);
                            continue;
                        }
                        Real hi = p[t] < n[t] - 1 ? (mm[i + s] - cc) / spacing(t, p[t] + 1) : Real(0);
                        Real lo = p[t] > 0 ? (cc - mm[i - s]) / spacing(t, p[t]) : Real(0);
                        if (p[t] == 0) lo = wall / spacing(t, 0);
                        if (p[t] == n[t] - 1) {
                            if (t == Y) {
                                Real U = a == X ? lidv * lid_at_u_face(x, z) : Real(0);
                                hi = (U - wall) / spacing(Y, n[Y]);
                            } else {
                                hi = -wall / spacing(t, n[t]);
                            }
                        }
                        lap += (hi - lo) / width(t, p[t]);
                    }
                    Real rhs_ = nu * lap + Real(0);
                    Real q = cc + dt * (rhs_ + In[i]);
                    if (has_base) q = a0 * mb[i] + b * q;
                    out[i] = q;
                }
    }

    // ------------------------------------------------------------ projection (backend.cu:334-380)
    void divergence(const vector<Real>* f, vector<double>& out) const {         // backend.cu:334-342
#pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < nz; z++)
            for (int y = 0; y < ny; y++)
                for (int x = 0; x < nx; x++) {
                    double dx = width(X, x), dy = width(Y, y), dz = width(Z, z);
                    out[cell(x, y, z)] = ((double)f[0][at(0, x + 1, y, z)] - (double)f[0][at(0, x, y, z)]) * (dy * dz) +
                                         ((double)f[1][at(1, x, y + 1, z)] - (double)f[1][at(1, x, y, z)]) * (dx * dz) +
                                         ((double)f[2][at(2, x, y, z + 1)] - (double)f[2][at(2, x, y, z)]) * (dx * dy);
                }
    }
    void residual(const vector<double>& p, const vector<double>& b, vector<double>& r) const {   // backend.cu:345-359
        long long sy = nx, sz = (long long)nx * ny;
#pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < nz; z++)
            for (int y = 0; y < ny; y++)
                for (int x = 0; x < nx; x++) {
                    long long i = cell(x, y, z);
                    double dx = width(X, x), dy = width(Y, y), dz = width(Z, z), cc = p[i], s = 0.0;
                    if (x + 1 < nx) s += (dy * dz) * (p[i + 1] - cc) / (double)spacing(X, x + 1);
                    if (x > 0) s -= (dy * dz) * (cc - p[i - 1]) / (double)spacing(X, x);
                    if (y + 1 < ny) s += (dx * dz) * (p[i + sy] - cc) / (double)spacing(Y, y + 1);
                    if (y > 0) s -= (dx * dz) * (cc - p[i - sy]) / (double)spacing(Y, y);
                    if (z + 1 < nz) s += (dx * dy) * (p[i + sz] - cc) / (double)spacing(Z, z + 1);
                    if (z > 0) s -= (dx * dy) * (cc - p[i - sz]) / (double)spacing(Z, z);
                    r[i] = b[i] - s;
                }
    }
    void subtract_gradient(int a, const vector<Real>& mm, const vector<double>& p, vector<Real>& out) const {
        // backend.cu:361-371
        int n[3] = {nx, ny, nz};
        const int* dm = dims[a];
        long long cstride[3] = {1, nx, (long long)nx * ny};
#pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < dm[2]; z++)
            for (int y = 0; y < dm[1]; y++)
                for (int x = 0; x < dm[0]; x++) {
                    int q[3] = {x, y, z};
                    long long i = at(a, x, y, z);
                    if (q[a] == 0 || q[a] == n[a]) { out[i] = Real(0); continue; }
                    long long ci = cell(x, y, z);
                    double d = (p[ci] - p[ci - cstride[a]]) / (double)spacing(a, q[a]);
                    out[i] = mm[i] - (Real)d;
                }
    }
    void zero_walls(int a, vector<Real>& f) const {                              // backend.cu:373-380
        int n[3] = {nx, ny, nz};
        const int* dm = dims[a];
        for (int z = 0; z < dm[2]; z++)
            for (int y = 0; y < dm[1]; y++)
                for (int x = 0; x < dm[0]; x++) {
                    int q[3] = {x, y, z};
                    if (q[a] == 0 || q[a] == n[a]) f[at(a, x, y, z)] = Real(0);
                }
    }

    // ------------------------------------------------------------ pressure solve (backend.cu:750-847)
    void setup_pressure_solver() {                                              // backend.cu:750-787
        vector<double> lambda[3];
        int zero_mode[3];
        for (int a = 0; a < 3; a++) {
            const Axis& g = ax[a];
            int n = g.n;
            vector<double> A((size_t)n * n, 0.0), V;
            for (int i = 0; i < n - 1; i++) {
                double k = 1.0 / g.spacing[i + 1];
                A[i * n + i] -= k;
                A[(i + 1) * n + i + 1] -= k;
                A[i * n + i + 1] += k;
                A[(i + 1) * n + i] += k;
            }
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) A[i * n + j] /= std::sqrt(g.width[i] * g.width[j]);
            jacobi_eigen(n, A, V);
            lambda[a].resize(n);
            for (int i = 0; i < n; i++) lambda[a][i] = A[i * n + i];
            zero_mode[a] = (int)(std::max_element(lambda[a].begin(), lambda[a].end()) - lambda[a].begin());
            lambda[a][zero_mode[a]] = 0.0;
            S[a].resize((size_t)n * n);
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) S[a][i * n + j] = (Real)(V[i * n + j] / std::sqrt(g.width[i]));
        }
        inv_lambda.resize(n_cell);
        for (int z = 0; z < nz; z++)
            for (int y = 0; y < ny; y++)
                for (int x = 0; x < nx; x++) {
                    bool zero = (x == zero_mode[X] && y == zero_mode[Y] && z == zero_mode[Z]);
                    double v = 1.0 / (lambda[Z][z] + lambda[Y][y] + lambda[X][x]);
                    inv_lambda[cell(x, y, z)] = zero ? Real(0) : (Real)v;
                }
    }
    // out[.., j, ..] = sum_i M(i, j) in[.., i, ..] along axis a; M(i, j) = S[i][j] (trans = false) or S[j][i]
    void transform(int a, bool trans, const vector<Real>& in, vector<Real>& out) const {
        int n = ax[a].n;
        long long stride = a == X ? 1 : a == Y ? nx : (long long)nx * ny;
        const vector<Real>& M = S[a];
#pragma omp parallel for schedule(static)
        for (long long idx = 0; idx < n_cell; idx++) {
            long long pos = (idx / stride) % n, base_ = idx - pos * stride;
            double s = 0.0;
            for (int i = 0; i < n; i++) {
                Real mij = trans ? M[(size_t)pos * n + i] : M[(size_t)i * n + pos];
                s += (double)mij * (double)in[base_ + i * stride];
            }
            out[idx] = (Real)s;
        }
    }
    // phi += approximate solution of L phi = r (backend.cu:801-814): forward transforms with S^T, divide by
    // the eigenvalues, back with S.  Float mode scales r to rms 1 first, as the reference.
    void pressure_pass(const vector<double>& r, vector<double>& p) {
        double rms = std::sqrt(det_sum(n_cell, [&](long long i) { return r[i] * r[i]; }) / n_cell);
        if (!(rms > 0)) return;
        double scale = kFloatMode ? rms : 1.0;
        vector<Real> t1(n_cell), t2(n_cell);
        for (long long i = 0; i < n_cell; i++) t1[i] = (Real)(r[i] * (1.0 / scale));
        transform(X, false, t1, t2);
        transform(Y, false, t2, t1);
        transform(Z, false, t1, t2);
        for (long long i = 0; i < n_cell; i++) t2[i] = t2[i] * inv_lambda[i];
        transform(Z, true, t2, t1);
        transform(Y, true, t1, t2);
        transform(X, true, t2, t1);
        for (long long i = 0; i < n_cell; i++) p[i] = p[i] + (double)t1[i] * scale;
    }
    double norm(const vector<double>& v) const {
        return std::sqrt(det_sum(n_cell, [&](long long i) { return v[i] * v[i]; }));
    }
    void solve_pressure(const vector<double>& b, const vector<double>* g, vector<double>& p) {   // backend.cu:816-847
        double rhs_norm = norm(b);
        phi_passes = 0;
        if (!std::isfinite(rhs_norm)) fail("pressure solve: right-hand side is NaN/inf (the run has blown up)");
        if (rhs_norm == 0.0) { std::fill(p.begin(), p.end(), 0.0); phi_rel = 0; return; }
        const vector<double>* r = &b;
        double rel = 1.0;
        std::fill(p.begin(), p.end(), 0.0);
        if (g) {
            p = *g;
            residual(p, b, res);
            r = &res;
            rel = norm(res) / rhs_norm;
            if (rel >= 1.0) { std::fill(p.begin(), p.end(), 0.0); r = &b; rel = 1.0; }
        }
        while (rel > c.fdm_rtol && phi_passes < c.fdm_max_passes) {
            pressure_pass(*r, p);
            phi_passes++;
            residual(p, b, res);
            r = &res;
            rel = norm(res) / rhs_norm;
            if (!std::isfinite(rel)) fail("pressure solve: residual is NaN/inf");
        }
        if (rel > c.fdm_rtol) {
            char msg[200];
            std::snprintf(msg, sizeof msg, "pressure solve: residual %.2e > FDM_RTOL after %d passes", rel, phi_passes);
            fail(msg);
        }
        phi_rel = rel;
        double mean = det_sum(n_cell, [&](long long i) { return p[i]; }) / n_cell;
        for (long long i = 0; i < n_cell; i++) p[i] = p[i] - mean;
    }
    void project(vector<Real>* mm, const vector<double>* g, vector<double>& p, vector<Real>* out) {   // backend.cu:849-854
        for (int k = 0; k < 3; k++) zero_walls(k, mm[k]);
        divergence(mm, rhs);
        solve_pressure(rhs, g, p);
        for (int k = 0; k < 3; k++) subtract_gradient(k, mm[k], p, out[k]);
    }
    bool guess_phi(double tau, double scale, vector<double>& out) {             // backend.cu:857-873
        if (!c.phi_extrapolate || hist.empty()) return false;
        vector<int> order(hist.size());
        for (size_t k = 0; k < order.size(); k++) order[k] = (int)k;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            double da = std::fabs(hist[a].t - tau), db = std::fabs(hist[b].t - tau);
            return da != db ? da < db : a > b;
        });
        const History& h1 = hist[order[0]];
        const History* h2 = nullptr;
        for (size_t k = 1; k < order.size() && !h2; k++)
            if (std::fabs(hist[order[k]].t - h1.t) > 1e-12 * std::max(1.0, std::fabs(h1.t))) h2 = &hist[order[k]];
        double w2 = h2 ? (tau - h1.t) / (h2->t - h1.t) : 0.0, w1 = 1.0 - w2;
        const vector<double>& d1 = hist_buf[h1.buf];
        if (h2) {
            const vector<double>& d2 = hist_buf[h2->buf];
            double c1 = scale * w1 / h1.scale, c2 = scale * w2 / h2->scale;
            for (long long i = 0; i < n_cell; i++) out[i] = c1 * d1[i] + c2 * d2[i];
        } else {
            double c1 = scale * w1 / h1.scale;
            for (long long i = 0; i < n_cell; i++) out[i] = c1 * d1[i];
        }
        return true;
    }

    // ------------------------------------------------------------ CFL rate (backend.cu:465-472)
    // fmax as the reference's fmaxf: a NaN on one face of the pair is dropped (a single NaN face does not
    // make the rate NaN; it surfaces later as a NaN right-hand side)
    Real cfl_rate_cell(const vector<Real>* f, int x, int y, int z) const {
        return std::fmax(std::fabs(f[0][at(0, x, y, z)]), std::fabs(f[0][at(0, x + 1, y, z)])) / width(X, x) +
               std::fmax(std::fabs(f[1][at(1, x, y, z)]), std::fabs(f[1][at(1, x, y + 1, z)])) / width(Y, y) +
               std::fmax(std::fabs(f[2][at(2, x, y, z)]), std::fabs(f[2][at(2, x, y, z + 1)])) / width(Z, z);
    }
    double cfl_max(const vector<Real>* f) const {
        return det_max(n_cell, [&](long long i) {
            int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
            return (double)cfl_rate_cell(f, x, y, z);
        });
    }

    // ------------------------------------------------------------ the time step (backend.cu:877-955)
    void step() {
        long long n = n_cell;
        for (int k = 0; k < 3; k++)
            for (long long i = 0; i < size[k]; i++)
                m0[k][i] = (Real)c.reinit_r * m[k][i] + (Real)(1.0 - c.reinit_r) * u[k][i];
        for (long long i = 0; i < n; i++) phi0[i] = c.reinit_r * phi[i];

        double rates[2] = {(double)(float)cfl_max(u), (double)viscous_rate};
        double use[2] = {rates[0], rates[1]};
        if (c.dt_lag && have_prev_rates) { use[0] = prev_rates[0]; use[1] = prev_rates[1]; }
        prev_rates[0] = rates[0];
        prev_rates[1] = rates[1];
        have_prev_rates = true;
        if (!std::isfinite(use[0])) fail("velocity is NaN/inf: the solution has blown up");
        double dt;
        if (!c.adaptive_dt) { dt = c.dt_fixed; dt_reason = 0; }
        else {
            double caps[3] = {c.dt_max, c.cfl_target / std::max(use[0], 1e-300),
                              c.diffusion_limit / std::max(use[1], 1e-300)};
            int best = 0;
            for (int k = 1; k < 3; k++)
                if (caps[k] < caps[best]) best = k;
            dt = caps[best];
            dt_reason = best + 1;
        }
        if (c.dt_lag && last_dt > 0) dt = std::min(dt, 1.1 * last_dt);

        const double a0s[3] = {0.0, 0.75, 1.0 / 3.0}, bs[3] = {1.0, 0.25, 2.0 / 3.0};
        const double times[3] = {t, t + dt, t + 0.5 * dt};
        vector<Real> cur_u[3], cur_m[3];
        for (int k = 0; k < 3; k++) { cur_u[k] = u[k]; cur_m[k] = m0[k]; }
        vector<double> cur_phi = phi0;
        int o4 = c.impulse_order == 4;
        Real K = (Real)std::max(c.impulse_order4_ramp, 1.0);
        for (int stage = 0; stage < 3; stage++) {
            double a0 = a0s[stage], b = bs[stage], ts = times[stage];
            for (int k = 0; k < 3; k++) inviscid(k, cur_u, cur_m, o4, K, I[k]);
            for (int k = 0; k < 3; k++)
                rk3_stage(k, cur_m[k], m0[k], cur_u[k], I[k], (Real)c.nu, (Real)lid(ts), (Real)dt, (Real)a0, (Real)b,
                          stage > 0 ? 1 : 0, nm[k]);
            if (a0 != 0.0)
                for (long long i = 0; i < n; i++) base[i] = a0 * phi0[i] + b * cur_phi[i];
            else
                for (long long i = 0; i < n; i++) base[i] = b * cur_phi[i];
            if (guess_phi(ts, b * dt, guess))
                for (long long i = 0; i < n; i++) guess[i] = guess[i] + base[i];
            else
                guess = base;
            project(nm, &guess, phi_new, nu_);
            if (c.phi_extrapolate) {
                int buf = -1;
                for (int k = 0; k < 4 && buf < 0; k++) {
                    bool used = false;
                    for (const History& h : hist) used |= (h.buf == k);
                    if (!used) buf = k;
                }
                for (long long i = 0; i < n; i++) hist_buf[buf][i] = 1.0 * phi_new[i] + -1.0 * base[i];
                hist.push_back({ts, b * dt, buf});
                if (hist.size() > 3) hist.erase(hist.begin());
            }
            for (int k = 0; k < 3; k++) { cur_u[k] = nu_[k]; cur_m[k] = nm[k]; }
            cur_phi = phi_new;
        }
        for (int k = 0; k < 3; k++) { u[k] = cur_u[k]; m[k] = cur_m[k]; }
        phi = cur_phi;
        t += dt;
        steps++;
        last_dt = dt;
        last_cfl = dt * use[0];
    }

    // ------------------------------------------------------------ kick (backend.cu:544-561, 958-978)
    void kick(const double* const noise[3], double amp, int passes) {
        vector<Real> new_u[3];
        for (int k = 0; k < 3; k++) {
            long long n = size[k];
            int sx = dims[k][0], sy = dims[k][1], sz = dims[k][2];
            vector<double> a(noise[k], noise[k] + n), b(n);
            for (int p = 0; p < std::max(1, passes); p++)
                for (int axis = 2; axis >= 0; axis--) {
                    for (long long i = 0; i < n; i++) {
                        int x = (int)(i % sx), y = (int)((i / sx) % sy), z = (int)(i / ((long long)sx * sy));
                        long long lo, hi;
                        if (axis == 0) { lo = (x + sx - 1) % sx + sx * (y + (long long)sy * z); hi = (x + 1) % sx + sx * (y + (long long)sy * z); }
                        else if (axis == 1) { lo = x + sx * ((y + sy - 1) % sy + (long long)sy * z); hi = x + sx * ((y + 1) % sy + (long long)sy * z); }
                        else { lo = x + sx * (y + (long long)sy * ((z + sz - 1) % sz)); hi = x + sx * (y + (long long)sy * ((z + 1) % sz)); }
                        b[i] = 0.25 * a[lo] + 0.5 * a[i] + 0.25 * a[hi];
                    }
                    std::swap(a, b);
                }
            double rms = std::sqrt(det_sum(n, [&](long long i) { return a[i] * a[i]; }) / n);
            double s = amp * c.u_lid / std::max(rms, 1e-30);
            for (long long i = 0; i < n; i++) tmp[k][i] = u[k][i] + (Real)(a[i] * s);
            new_u[k].resize(n);
        }
        vector<double> scratch(n_cell);
        project(tmp, nullptr, scratch, new_u);
        for (int k = 0; k < 3; k++) {
            for (long long i = 0; i < size[k]; i++) m[k][i] = m[k][i] + (new_u[k][i] - u[k][i]);
            u[k] = new_u[k];
        }
    }
};

// =====================================================================================================
//  C ABI (backend.cu:980-1195)
// =====================================================================================================
static std::string last_error;
static Oracle* the_solver = nullptr;
template <class F> static int safely(F f) {
    try { f(); return 0; }
    catch (const std::exception& e) { last_error = e.what(); return 1; }
}
static Oracle& S() {
    if (!the_solver) fail("no solver: call solver_create first");
    return *the_solver;
}
static void fill(Report* r) {
    Oracle& s = S();
    r->steps = s.steps; r->time = s.t; r->dt = s.last_dt; r->cfl = s.last_cfl; r->phi_rel = s.phi_rel;
    r->dt_reason = s.dt_reason; r->phi_passes = s.phi_passes;
}
// midspan layers k1, k2 (backend.cu:488)
static void midspan_layers(int nz, int& k1, int& k2) { k2 = nz / 2; k1 = (nz % 2) ? k2 : k2 - 1; }

extern "C" {
int solver_destroy() {
    return safely([&] { delete the_solver; the_solver = nullptr; });
}
int solver_create(const Config* config) {                                      // backend.cu:1009-1073
    return safely([&] {
        solver_destroy();
        Oracle* p = new Oracle();
        try {
            Oracle& s = *p;
            s.c = *config;
            s.nx = s.c.nx; s.ny = s.c.ny; s.nz = s.c.nz;
            if (s.nx != s.ny || s.nx % 2 || s.nx < 6) fail("nx = ny must be even and >= 6");
            if (s.nz < 5) fail("need nz >= 5");
            if (std::max(s.nx, s.nz) > GMAX) fail("at most 1024 cells per axis");
            if (s.c.impulse_order != 2 && s.c.impulse_order != 4) fail("IMPULSE_ORDER must be 2 or 4");
            if ((double)(s.nx + 1) * s.ny * (s.nz + 1) > 2e9) fail("grid too large");
            s.n_cell = s.nx * s.ny * s.nz;
            for (int k = 0; k < 3; k++) {
                s.dims[k][0] = s.nx + (k == 0); s.dims[k][1] = s.ny + (k == 1); s.dims[k][2] = s.nz + (k == 2);
                s.size[k] = s.dims[k][0] * s.dims[k][1] * s.dims[k][2];
            }
            s.ax[X] = make_axis(s.c, s.nx, s.c.length);
            s.ax[Y] = make_axis(s.c, s.ny, s.c.length);
            s.ax[Z] = make_axis(s.c, s.nz, s.nz * (s.c.lz / s.nz));
            s.volume = s.ax[X].length * s.ax[Y].length * s.ax[Z].length;
            for (int a = 0; a < 3; a++) {
                const Axis& g = s.ax[a];
                s.FACE[a].assign(g.face.begin(), g.face.end());
                s.CENTRE[a].assign(g.centre.begin(), g.centre.end());
                s.WIDTH[a].assign(g.width.begin(), g.width.end());
                s.SPACING[a].assign(g.spacing.begin(), g.spacing.end());
                // the reference's device table holds (float)length (backend.cu:706)
                s.LENGTH[a] = (Real)(float)g.length;
            }
            float vmax = 0.0f;                                                   // backend.cu:1030-1034
            auto geo = [&](int a, int i) {
                return 4.0f / ((float)s.ax[a].width[i] * std::min((float)s.ax[a].spacing[i], (float)s.ax[a].spacing[i + 1]));
            };
            for (int z = 0; z < s.nz; z++)
                for (int y = 0; y < s.ny; y++)
                    for (int x = 0; x < s.nx; x++)
                        vmax = std::max(vmax, (float)s.c.nu * (geo(X, x) + geo(Y, y) + geo(Z, z)));
            s.viscous_rate = vmax;
            for (int k = 0; k < 3; k++)
                for (vector<Real>* v : {&s.u[k], &s.m[k], &s.m0[k], &s.I[k], &s.nm[k], &s.nu_[k], &s.tmp[k]})
                    v->assign(s.size[k], Real(0));
            for (vector<double>* v : {&s.phi, &s.phi0, &s.base, &s.guess, &s.rhs, &s.res, &s.phi_new})
                v->assign(s.n_cell, 0.0);
            for (int k = 0; k < 4; k++) s.hist_buf[k].assign(s.n_cell, 0.0);
            s.stats.assign(6LL * s.nx * s.ny, 0.0);
            s.setup_pressure_solver();
            for (int p = 0; p < s.c.n_probes; p++) {                             // backend.cu:1058-1070
                auto cell_of = [](const Axis& g, double frac) {
                    int k = (int)(std::upper_bound(g.face.begin(), g.face.end(), frac * g.length) - g.face.begin()) - 1;
                    return std::min(g.n - 1, std::max(0, k));
                };
                s.probe_cell[p][0] = cell_of(s.ax[X], s.c.probe_x[p]);
                s.probe_cell[p][1] = cell_of(s.ax[Y], s.c.probe_y[p]);
                s.probe_cell[p][2] = s.nz / 2;
            }
        } catch (...) {
            delete p;
            throw;
        }
        the_solver = p;
    });
}
int solver_initialize(const double* v_noise, const double* w_noise) {          // backend.cu:1075-1088
    return safely([&] {
        Oracle& s = S();
        const double* src[3] = {nullptr, v_noise, w_noise};
        for (int k = 0; k < 3; k++)
            for (long long i = 0; i < s.size[k]; i++) s.m[k][i] = src[k] ? (Real)(float)src[k][i] : Real(0);
        s.project(s.m, nullptr, s.phi, s.u);
        s.t = 0; s.steps = 0; s.last_dt = 0; s.hist.clear(); s.have_prev_rates = false;
    });
}
int solver_step(Report* r) { return safely([&] { S().step(); fill(r); }); }
int solver_kick(const double* nu, const double* nv, const double* nw, double amp, int passes) {
    return safely([&] { const double* n[3] = {nu, nv, nw}; S().kick(n, amp, passes); });
}
int solver_report(Report* r) { return safely([&] { fill(r); }); }
int solver_diagnostics(Diagnostics* d) {                                        // backend.cu:1096-1129, 447-463
    return safely([&] {
        Oracle& s = S();
        long long n = s.n_cell;
        Real lidv = (Real)s.lid(s.t);
        vector<double> ke(n), ens(n), div2(n);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < n; i++) {
            int x = (int)(i % s.nx), y = (int)((i / s.nx) % s.ny), z = (int)(i / ((long long)s.nx * s.ny));
            double vol = (double)s.width(X, x) * (double)s.width(Y, y) * (double)s.width(Z, z);
            double a = s.centred(s.u, 0, x, y, z), b = s.centred(s.u, 1, x, y, z), c = s.centred(s.u, 2, x, y, z);
            ke[i] = 0.5 * (a * a + b * b + c * c) * vol;
            Real g[3][3];
            s.cell_gradient(s.u, lidv, x, y, z, g);
            Real ox = g[1][2] - g[2][1], oy = g[2][0] - g[0][2], oz = g[0][1] - g[1][0];
            ens[i] = (double)(ox * ox + oy * oy + oz * oz) * vol;
            double dd = (double)(s.u[0][s.at(0, x + 1, y, z)] - s.u[0][s.at(0, x, y, z)]) / (double)s.width(X, x) +
                        (double)(s.u[1][s.at(1, x, y + 1, z)] - s.u[1][s.at(1, x, y, z)]) / (double)s.width(Y, y) +
                        (double)(s.u[2][s.at(2, x, y, z + 1)] - s.u[2][s.at(2, x, y, z)]) / (double)s.width(Z, z);
            div2[i] = dd * dd * vol;
        }
        d->kinetic_energy = det_sum(n, [&](long long i) { return ke[i]; }) / s.volume;
        d->enstrophy = 0.5 * det_sum(n, [&](long long i) { return ens[i]; }) / s.volume;
        d->div_rms = std::sqrt(det_sum(n, [&](long long i) { return div2[i]; }) / s.volume);
        double umax = 0;
        for (int k = 0; k < 3; k++)
            umax = std::max(umax, det_max(s.size[k], [&](long long i) { return std::fabs((double)s.u[k][i]); }));
        d->umax = umax;
        d->cfl_rate = s.cfl_max(s.u);
        double best = -1;
        int best_comp = 0;
        long long best_i = 0;
        for (int k = 0; k < 3; k++) {
            vector<Real> diff(s.size[k]);
            for (long long i = 0; i < s.size[k]; i++) diff[i] = std::fabs(s.m[k][i] - s.u[k][i]);
            double val = det_max(s.size[k], [&](long long i) { return (double)diff[i]; });
            if (val > best) {
                long long first = 2147483647;
                for (long long i = 0; i < s.size[k]; i++)
                    if (diff[i] == (Real)val) { first = i; break; }
                best_i = first; best = val; best_comp = k;
            }
        }
        int sx = s.nx + (best_comp == 0), sy = s.ny + (best_comp == 1);
        int ix = (int)(best_i % sx), iy = (int)((best_i / sx) % sy);
        d->gauge_ratio = best / std::max(umax, 1e-30);
        d->gauge_x = (best_comp == 0 ? s.ax[X].face[ix] : s.ax[X].centre[std::min(ix, s.nx - 1)]) / s.c.length;
        d->gauge_y = (best_comp == 1 ? s.ax[Y].face[iy] : s.ax[Y].centre[std::min(iy, s.ny - 1)]) / s.c.length;
    });
}
int solver_grid(int axis, double* faces, double* centres) {                     // backend.cu:1131-1137
    return safely([&] {
        const Axis& g = S().ax[axis];
        std::copy(g.face.begin(), g.face.end(), faces);
        std::copy(g.centre.begin(), g.centre.end(), centres);
    });
}
int solver_get_field(int field, void* out) {                                    // backend.cu:1139-1146
    return safely([&] {
        Oracle& s = S();
        if (field < 3) for (long long i = 0; i < s.size[field]; i++) ((float*)out)[i] = (float)s.u[field][i];
        else if (field < 6) for (long long i = 0; i < s.size[field - 3]; i++) ((float*)out)[i] = (float)s.m[field - 3][i];
        else std::copy(s.phi.begin(), s.phi.end(), (double*)out);
    });
}
int solver_set_field(int field, const void* in) {                               // backend.cu:1147-1155
    return safely([&] {
        Oracle& s = S();
        if (field < 3) for (long long i = 0; i < s.size[field]; i++) s.u[field][i] = (Real)((const float*)in)[i];
        else if (field < 6) for (long long i = 0; i < s.size[field - 3]; i++) s.m[field - 3][i] = (Real)((const float*)in)[i];
        else std::copy((const double*)in, (const double*)in + s.n_cell, s.phi.begin());
        s.hist.clear();
        s.have_prev_rates = false;
    });
}
int solver_set_clock(double t, long long steps, double last_dt) {
    return safely([&] { Oracle& s = S(); s.t = t; s.steps = steps; s.last_dt = last_dt; });
}
int solver_probes(float* out) {                                                 // backend.cu:1159-1166, 534-540
    return safely([&] {
        Oracle& s = S();
        for (int p = 0; p < s.c.n_probes; p++) {
            int x = s.probe_cell[p][0], y = s.probe_cell[p][1], z = s.probe_cell[p][2];
            out[2 * p] = (float)(Real(0.5) * (s.u[0][s.at(0, x, y, z)] + s.u[0][s.at(0, x + 1, y, z)]));
            out[2 * p + 1] = (float)(Real(0.5) * (s.u[1][s.at(1, x, y, z)] + s.u[1][s.at(1, x, y + 1, z)]));
        }
    });
}
int solver_add_statistics(double weight, double* centreline) {                  // backend.cu:1168-1175, 507-532
    return safely([&] {
        Oracle& s = S();
        int nx = s.nx, ny = s.ny, k1, k2;
        long long n = (long long)nx * ny;
        midspan_layers(s.nz, k1, k2);
        auto C = [&](int c, int x, int y, int z) { return (double)s.centred(s.u, c, x, y, z); };
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                long long i = x + (long long)nx * y;
                double a = 0.5 * (C(0, x, y, k1) + C(0, x, y, k2));
                double b = 0.5 * (C(1, x, y, k1) + C(1, x, y, k2));
                double c = 0.5 * (C(2, x, y, k1) + C(2, x, y, k2));
                s.stats[i] += weight * a; s.stats[n + i] += weight * b; s.stats[2 * n + i] += weight * (a * a);
                s.stats[3 * n + i] += weight * (b * b); s.stats[4 * n + i] += weight * (c * c);
                s.stats[5 * n + i] += weight * (a * b);
            }
        int mid = nx / 2;
        auto mean4 = [&](int c, int xa, int ya, int xb, int yb) {
            return 0.5 * (0.5 * (C(c, xa, ya, k1) + C(c, xa, ya, k2)) + 0.5 * (C(c, xb, yb, k1) + C(c, xb, yb, k2)));
        };
        for (int j = 0; j < nx; j++) {
            double a = mean4(0, mid - 1, j, mid, j), b = mean4(1, j, mid - 1, j, mid), c = mean4(2, mid - 1, j, mid, j);
            centreline[j] = a; centreline[nx + j] = b; centreline[2 * nx + j] = a * a;
            centreline[3 * nx + j] = b * b; centreline[4 * nx + j] = c * c;
        }
    });
}
int solver_get_statistics(double* sums) { return safely([&] { std::copy(S().stats.begin(), S().stats.end(), sums); }); }
int solver_set_statistics(const double* sums) {
    return safely([&] { Oracle& s = S(); std::copy(sums, sums + s.stats.size(), s.stats.begin()); });
}
int solver_midplane(float* out) {                                               // backend.cu:1178-1184, 490-505
    return safely([&] {
        Oracle& s = S();
        int k1, k2, nx = s.nx, ny = s.ny;
        midspan_layers(s.nz, k1, k2);
        Real lidv = (Real)s.lid(s.t);
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                Real val[2][4];
                for (int q = 0; q < 2; q++) {
                    int z = q ? k2 : k1;
                    for (int c = 0; c < 3; c++) val[q][c] = s.centred(s.u, c, x, y, z);
                    Real g[3][3];
                    s.cell_gradient(s.u, lidv, x, y, z, g);
                    Real a = g[1][2] - g[2][1], b = g[2][0] - g[0][2], c = g[0][1] - g[1][0];
                    val[q][3] = std::sqrt(a * a + b * b + c * c);
                }
                for (int c = 0; c < 4; c++)
                    out[c * nx * ny + x + nx * y] = (float)((k1 == k2) ? val[1][c] : Real(0.5) * (val[0][c] + val[1][c]));
            }
    });
}
int solver_q_volume(int colour_w, float* q, float* colour) {                    // backend.cu:1185-1194, 474-486
    return safely([&] {
        Oracle& s = S();
        double L_over_U = s.c.length / s.c.u_lid;
        Real lidv = (Real)s.lid(s.t), qscale = (Real)(L_over_U * L_over_U), inv_U = (Real)(1.0 / s.c.u_lid);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < s.n_cell; i++) {
            int x = (int)(i % s.nx), y = (int)((i / s.nx) % s.ny), z = (int)(i / ((long long)s.nx * s.ny));
            Real g[3][3];
            s.cell_gradient(s.u, lidv, x, y, z, g);
            Real sum = Real(0);
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) sum += g[a][b] * g[b][a];
            q[i] = (float)(Real(-0.5) * sum * qscale);
            Real a = s.centred(s.u, 0, x, y, z), b = s.centred(s.u, 1, x, y, z), c = s.centred(s.u, 2, x, y, z);
            colour[i] = (float)(colour_w ? c * inv_U : std::sqrt(a * a + b * b + c * c) * inv_U);
        }
    });
}
const char* solver_last_error() { return last_error.c_str(); }
// test-side addition: the fields in double (velocity and impulse are float32 in the reference ABI)
int cavity_get_field_f64(int field, double* out) {
    return safely([&] {
        Oracle& s = S();
        if (field < 3) for (long long i = 0; i < s.size[field]; i++) out[i] = (double)s.u[field][i];
        else if (field < 6) for (long long i = 0; i < s.size[field - 3]; i++) out[i] = (double)s.m[field - 3][i];
        else std::copy(s.phi.begin(), s.phi.end(), out);
    });
}
}
