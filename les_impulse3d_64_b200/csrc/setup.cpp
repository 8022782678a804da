// setup.cpp - host-side set-up of a cavity (grid, tables, pressure eigenbases, probes).
#include "setup.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <stdexcept>

#include "layout.h"

namespace cavity {

// ------------------------------------------------------------------------------------------ grid
// Faces of an axis.  Uniform: i*h on [0, length] with the last face set to length.  Stretched: two-sided tanh
// clustering length/2 (1 + tanh(beta (2 xi - 1)) / tanh(beta)), beta found by 200 bisection steps on
// [1e-8, 30] so that the first cell equals dx_wall; end and middle faces pinned (backend.cu:643-666).  The
// grid must equal the reference's to the last bit (it feeds the float-rounded tables and the probe cells),
// so the expressions keep its operation order.
static std::vector<double> axis_faces(int n, double length, double dx_wall) {
    std::vector<double> f(n + 1);
    auto uniform = [&](double a, double b, int count, std::vector<double>& v) {
        const double h = (b - a) / (count - 1);
        for (int i = 0; i < count; i++) v[i] = i * h + a;
        v[count - 1] = b;
    };
    if (dx_wall >= length / n * (1 - 1e-12)) {
        uniform(0.0, length, n + 1, f);
        return f;
    }
    std::vector<double> xi(n + 1);
    uniform(0.0, 1.0, n + 1, xi);
    auto face = [&](double beta, int i) { return length * 0.5 * (1.0 + std::tanh(beta * (2 * xi[i] - 1)) / std::tanh(beta)); };
    double lo = 1e-8, hi = 30.0;
    for (int it = 0; it < 200; it++) {
        const double beta = 0.5 * (lo + hi);
        if (face(beta, 1) - face(beta, 0) < dx_wall) hi = beta;
        else lo = beta;
    }
    const double beta = 0.5 * (lo + hi);
    for (int i = 0; i <= n; i++) f[i] = face(beta, i);
    f[0] = 0.0;
    f[n] = length;
    f[n / 2] = 0.5 * length;
    return f;
}

static double cell_ratio(const std::vector<double>& f) {                 // largest / smallest cell
    double big = 0, small = 1e300;
    for (size_t i = 1; i < f.size(); i++) {
        const double d = f[i] - f[i - 1];
        big = std::max(big, d);
        small = std::min(small, d);
    }
    return big / small;
}

AxisGrid make_axis_grid(const CavityConfig& c, int n, double length) {    // backend.cu:672-699
    std::vector<double> f;
    if (!c.grid_stretch) {
        f = axis_faces(n, length, 1e300);
    } else {
        double d = std::min(c.grid_dx_wall, length / n);
        if (c.grid_max_aspect > 0 && cell_ratio(axis_faces(n, length, d)) > c.grid_max_aspect) {
            // smallest wall cell whose stretching stays within the aspect cap: 60 bisection steps
            double lo = d, hi = length / n;
            for (int it = 0; it < 60; it++) {
                const double mid = 0.5 * (lo + hi);
                if (cell_ratio(axis_faces(n, length, mid)) > c.grid_max_aspect) lo = mid;
                else hi = mid;
            }
            d = hi;
        }
        f = axis_faces(n, length, d);
    }
    AxisGrid g;
    g.n = n;
    g.face = f;
    g.width.resize(n);
    g.centre.resize(n);
    g.spacing.resize(n + 1);
    for (int i = 0; i < n; i++) {
        g.width[i] = f[i + 1] - f[i];
        g.centre[i] = 0.5 * (f[i + 1] + f[i]);
    }
    for (int i = 1; i < n; i++) g.spacing[i] = g.centre[i] - g.centre[i - 1];
    g.spacing[0] = 0.5 * g.width[0];
    g.spacing[n] = 0.5 * g.width[n - 1];
    g.length = f[n] - f[0];
    for (std::vector<double>* v : {&g.face, &g.centre, &g.width, &g.spacing})
        for (double& q : *v) q = (double)(float)q;
    return g;
}

// ------------------------------------------------------------------------------------------ eigenbasis
// Implicit-shift QL iteration for a symmetric tridiagonal matrix with eigenvector accumulation (the tql2
// procedure of Bowdler, Martin, Reinsch and Wilkinson, Numer. Math. 11 (1968)), written for this solver:
// d = diagonal, e[i] = coupling of i and i+1; on return d holds the eigenvalues and the columns of Z
// (row-major n x n) the orthonormal eigenvectors.
static void tridiagonal_ql(int n, std::vector<double>& d, std::vector<double>& e, std::vector<double>& Z) {
    Z.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) Z[(size_t)i * n + i] = 1.0;
    e.resize(n);
    e[n - 1] = 0.0;
    const double eps = 2.220446049250313e-16;
    for (int l = 0; l < n; l++) {
        int iter = 0;
        while (true) {
            int m = l;
            for (; m < n - 1; m++) {
                const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= eps * dd) break;
            }
            if (m == l) break;
            if (++iter > 200) throw std::runtime_error("pressure solver set-up: eigenvalues did not converge");
            // Wilkinson-type shift from the leading 2x2 block
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            int i = m - 1;
            bool deflated = false;
            for (; i >= l; i--) {
                const double f = s * e[i], b = c * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {                    // underflow: split the matrix here
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    deflated = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                for (int k = 0; k < n; k++) {      // accumulate the rotation into the eigenvectors
                    double* row = &Z[(size_t)k * n];
                    const double zi = row[i], zi1 = row[i + 1];
                    row[i + 1] = s * zi + c * zi1;
                    row[i] = c * zi - s * zi1;
                }
            }
            if (deflated) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
}

void axis_tridiagonal(const AxisGrid& g, std::vector<double>& d, std::vector<double>& e) {
    const int n = g.n;
    // K: face i+1 (between cells i and i+1) couples them with 1/spacing; symmetric form W^-1/2 K W^-1/2
    d.assign(n, 0.0);
    e.assign(n, 0.0);
    for (int i = 0; i + 1 < n; i++) {
        const double k = 1.0 / g.spacing[i + 1];
        d[i] -= k;
        d[i + 1] -= k;
        e[i] = k / std::sqrt(g.width[i] * g.width[i + 1]);
    }
    for (int i = 0; i < n; i++) d[i] /= g.width[i];
}

AxisEigen axis_eigen_finish(const AxisGrid& g, std::vector<double> lambda, const std::vector<double>& Z) {
    const int n = g.n;
    AxisEigen r;
    r.lambda = std::move(lambda);
    r.zero_mode = (int)(std::max_element(r.lambda.begin(), r.lambda.end()) - r.lambda.begin());
    r.lambda[r.zero_mode] = 0.0;
    r.S.resize((size_t)n * n);
    for (int i = 0; i < n; i++) {
        const double inv = 1.0 / std::sqrt(g.width[i]);
        for (int j = 0; j < n; j++) r.S[(size_t)i * n + j] = Z[(size_t)i * n + j] * inv;
    }
    return r;
}

namespace {
// eigenbases already computed in this process, by the operator they belong to (widths and spacings of the axis,
// compared exactly) and the solver that computed them; the oldest goes first beyond kEigenCacheEntries
struct EigenEntry {
    std::vector<double> width, spacing;
    bool gpu;
    std::shared_ptr<const AxisEigen> eigen;
};
constexpr size_t kEigenCacheEntries = 16;
std::mutex g_eigen_mutex;
std::deque<EigenEntry> g_eigen_cache;
}  // namespace

AxisEigen axis_eigen_shared(const AxisGrid& g) {
    const bool gpu = eigen_on_gpu();
    {
        std::lock_guard<std::mutex> lock(g_eigen_mutex);
        for (const EigenEntry& e : g_eigen_cache)
            if (e.gpu == gpu && e.width == g.width && e.spacing == g.spacing) return *e.eigen;
    }
    auto eigen = std::make_shared<const AxisEigen>(gpu ? axis_eigen_gpu(g) : axis_eigen(g));
    std::lock_guard<std::mutex> lock(g_eigen_mutex);
    g_eigen_cache.push_back({g.width, g.spacing, gpu, eigen});
    if (g_eigen_cache.size() > kEigenCacheEntries) g_eigen_cache.pop_front();
    return *eigen;
}

bool eigen_on_gpu() {
    const char* m = std::getenv("CAVITY_EIGEN");
    return m && std::strcmp(m, "gpu") == 0;
}

AxisEigen axis_eigen(const AxisGrid& g) {
    std::vector<double> d, e, Z;
    axis_tridiagonal(g, d, e);
    tridiagonal_ql(g.n, d, e, Z);
    return axis_eigen_finish(g, std::move(d), Z);
}

// ------------------------------------------------------------------------------------------ misc
float viscous_rate(const CavityConfig& c, const AxisGrid ax[3]) {
    auto geo = [&](int a, int i) {
        return 4.0f / ((float)ax[a].width[i] * std::min((float)ax[a].spacing[i], (float)ax[a].spacing[i + 1]));
    };
    float vmax = 0.0f;
    for (int z = 0; z < ax[2].n; z++)
        for (int y = 0; y < ax[1].n; y++)
            for (int x = 0; x < ax[0].n; x++) vmax = std::max(vmax, (float)c.nu * (geo(0, x) + geo(1, y) + geo(2, z)));
    return vmax;
}

std::vector<int> probe_cells(const CavityConfig& c, const AxisGrid ax[3]) {
    std::vector<int> cells;
    auto cell_of = [](const AxisGrid& g, double frac) {
        const int k = (int)(std::upper_bound(g.face.begin(), g.face.end(), frac * g.length) - g.face.begin()) - 1;
        return std::min(g.n - 1, std::max(0, k));
    };
    for (int p = 0; p < c.n_probes; p++) {
        cells.push_back(cell_of(ax[0], c.probe_x[p]));
        cells.push_back(cell_of(ax[1], c.probe_y[p]));
        cells.push_back(ax[2].n / 2);
    }
    return cells;
}

template <class T>
std::vector<T> axis_tables(const AxisGrid& g, double ramp_cells, int stride) {
    const int n = g.n;
    std::vector<T> t((size_t)kNumTabs * stride, T(0));
    auto at = [&](int k, int i) -> T& { return t[(size_t)k * stride + i + kTabOffset]; };
    auto w = [&](int i) { return (T)g.width[i]; };
    auto sp = [&](int i) { return (T)g.spacing[i]; };
    const T K = (T)std::max(ramp_cells, 1.0);
    for (int i = 0; i < n; i++) {
        at(kW, i) = w(i);
        at(kInvW, i) = T(1) / w(i);
    }
    for (int i = 0; i <= n; i++) {
        at(kSp, i) = sp(i);
        at(kInvSp, i) = T(1) / sp(i);
        // wide (q = 3) stencil of the edge at face i: cells i-2 and i+1
        const bool wide = i - 2 >= 0 && i + 1 <= n - 1;
        at(kC3, i) = wide ? T(0.5) * (w(i - 2) + w(i + 1)) / (T(2) * sp(i)) : sp(i) / (T(2) * sp(i));
        if (wide) {
            at(kInvNd3, i) = T(1) / ((T)g.centre[i + 1] - (T)g.centre[i - 2]);
            at(kEv3Lo, i) = w(i - 2) / (w(i - 2) + w(i + 1));
            at(kEv3Hi, i) = w(i + 1) / (w(i - 2) + w(i + 1));
        }
        const bool narrow = i >= 1 && i <= n - 1;       // cells i-1 and i
        if (narrow) {
            at(kEv1Lo, i) = w(i - 1) / (T(2) * sp(i));
            at(kEv1Hi, i) = w(i) / (T(2) * sp(i));
        }
        const T d = (T)(i < n - i ? i : n - i) - T(1);     // wall ramp (backend.cu:130-133)
        at(kRamp, i) = std::min(std::max(d / K, T(0)), T(1));
        at(kOk1, i) = narrow ? T(1) : T(0);
        at(kOk3, i) = wide ? T(1) : T(0);
        at(kL1, i) = at(kOk1, i) * at(kRamp, i);
        at(kL3, i) = at(kOk3, i) * at(kRamp, i);
    }
    return t;
}
template std::vector<double> axis_tables<double>(const AxisGrid&, double, int);
template std::vector<float> axis_tables<float>(const AxisGrid&, double, int);

template <class T>
std::vector<T> lid_u_table(const CavityConfig& c, const AxisGrid ax[3]) {
    const int nx = ax[0].n, nz = ax[2].n;
    const T lx = (T)(float)ax[0].length, lz = (T)(float)ax[2].length;
    auto edge = [](T s) { const T s2 = s * s, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8, q = T(1) - s16 * s2; return q * q; };
    auto poly = [](T f) { const T g = f * (T(1) - f); return g * g; };
    std::vector<T> t((size_t)(nx + 1) * nz);
    for (int z = 0; z < nz; z++)
        for (int x = 0; x <= nx; x++) {
            const T fx = (T)ax[0].face[x] / lx, fz = (T)ax[2].centre[z] / lz;
            T s = T(1);
            if (c.lid_shaped == 2) s = T(16) * poly(fx) * poly(fz);
            else if (c.lid_shaped) s = edge(T(2) * fx - T(1)) * edge(T(2) * fz - T(1));
            t[(size_t)x + (size_t)(nx + 1) * z] = s;
        }
    return t;
}
template std::vector<double> lid_u_table<double>(const CavityConfig&, const AxisGrid[3]);
template std::vector<float> lid_u_table<float>(const CavityConfig&, const AxisGrid[3]);

std::string check_config(const CavityConfig& c) {
    if (c.nx != c.ny || c.nx % 2 || c.nx < 6) return "nx = ny must be even and >= 6";
    if (c.nz < 5) return "need nz >= 5";
    if (std::max(c.nx, c.nz) > 1024) return "at most 1024 cells per axis";
    if (c.impulse_order != 2 && c.impulse_order != 4) return "IMPULSE_ORDER must be 2 or 4";
    if ((double)(c.nx + 1) * c.ny * (c.nz + 1) > 2e9) return "grid too large";
    if (c.n_probes < 0 || c.n_probes > 8) return "at most 8 probes";
    return "";
}

}  // namespace cavity
