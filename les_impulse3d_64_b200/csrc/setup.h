// setup.h - host-side set-up of a cavity: stretched grid, coefficient tables, pressure eigenbases, probes.
#pragma once
#include <string>
#include <vector>

#include "cavity_solver.h"

namespace cavity {

// One axis of the MAC grid: n cells on [0, length].  face (n+1), centre (n), width (n), spacing (n+1,
// half a wall cell at the ends), all rounded through float once (backend.cu:689-697).
struct AxisGrid {
    int n = 0;
    double length = 0;
    std::vector<double> face, centre, width, spacing;
};

// tanh-stretched (or uniform) axis from the settings (backend.cu:651-699)
AxisGrid make_axis_grid(const CavityConfig& c, int n, double length);

// Generalised eigenbasis of the 1-D Neumann pressure operator of an axis: K S = W S diag(lambda) with
// S^T W S = I.  S is row-major n x n (eigenvector j in column j); the largest eigenvalue (the constant
// mode, ~0) is set to exactly 0 (backend.cu:750-767).  Both solvers work on the symmetric tridiagonal form
// W^-1/2 K W^-1/2 (diagonal d, coupling e[i] of i and i+1): axis_eigen by implicit-shift QL on the host,
// axis_eigen_gpu by bisection and inverse iteration on the GPU (eigen_gpu.cu).
struct AxisEigen {
    std::vector<double> S, lambda;
    int zero_mode = 0;
};
void axis_tridiagonal(const AxisGrid& g, std::vector<double>& d, std::vector<double>& e);
// eigenvalues and orthonormal eigenvectors Z (columns, row-major) of the tridiagonal form -> AxisEigen
AxisEigen axis_eigen_finish(const AxisGrid& g, std::vector<double> lambda, const std::vector<double>& Z);
AxisEigen axis_eigen(const AxisGrid& g);
AxisEigen axis_eigen_gpu(const AxisGrid& g);
// the eigensolver of the solvers' set-up: the host QL, or the GPU solver when CAVITY_EIGEN=gpu (the host QL
// measured faster at every size up to 512 cells)
bool eigen_on_gpu();
// The eigenbasis of an axis from the solver eigen_on_gpu picks, computed once per process for each operator:
// cavities of the same size and stretching (ensembles, a serving stream) share it.  Thread-safe.
AxisEigen axis_eigen_shared(const AxisGrid& g);

// Largest viscous rate over cells, nu * sum over axes 4/(width * smaller spacing), in float as
// backend.cu:1030-1034.
float viscous_rate(const CavityConfig& c, const AxisGrid ax[3]);

// Cell (x, y, nz/2) holding each probe (backend.cu:1058-1070).
std::vector<int> probe_cells(const CavityConfig& c, const AxisGrid ax[3]);

// Per-axis coefficient tables in the layout of kernels.cuh (Tab enum), `stride` entries per table.
template <class T>
std::vector<T> axis_tables(const AxisGrid& g, double ramp_cells, int stride);

// Lid shape on the top u-faces, [z][x] with nx+1 entries per row, computed in precision T.
template <class T>
std::vector<T> lid_u_table(const CavityConfig& c, const AxisGrid ax[3]);

// Validation of the settings with the reference's messages (backend.cu:1016-1020); empty if fine.
std::string check_config(const CavityConfig& c);

}  // namespace cavity
