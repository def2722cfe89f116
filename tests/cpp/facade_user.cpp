// A user program written against the C++ facade (multigrid-poisson_b200/poisson/), the way code
// written for the reference's Poisson::PoissonSolver uses it: settings by hand, init_zero, the
// right-hand side and the top boundary data written through get_rhs(0).at[idx(i,j,k)] and
// get_top_bc(0).arr.at[...], to_device, solve with verbose output and an ofile log, to_host.
// The data are dyadic rationals, so the same values come out of any compiler and of numpy.
//
// usage: facade_user <u.bin> <ofile>  -- writes u at the shape points (k fastest, float64)
#include <cstdio>
#include <cstdlib>
#include <iostream>

#include "libpoisson.h"

using namespace Poisson;

static double rhs_value(int i, int j, int k) { return ((7 * i + 3 * j + k) % 11) * 0.125 - 0.5; }
static double top_value(int i, int j) { return ((i + 2 * j) % 5) * 0.25 - 0.5; }

int main(int argc, char* argv[]) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <u.bin> <ofile>\n", argv[0]);
        return 2;
    }
    Settings settings;
    settings.dims[0] = 33;
    settings.dims[1] = 17;
    settings.dims[2] = 9;
    settings.levels = 3;
    settings.maxiter = 5;
    settings.tolerance = 0.0;
    settings.h = 1.0 / 32.0;
    settings.origin[0] = settings.origin[1] = settings.origin[2] = 0.0;
    BoundaryCondition BC{NEUMANN, NEUMANN, NEUMANN, NEUMANN, DIRICHLET, DIRICHLET};
    PoissonSolver<double_t, FullWeighting, TrilinearInterpolation, Jacobi> solver(settings, BC);
    solver.init_zero();
    DeviceArray<double_t>& f = solver.get_rhs(0);
    for (int i = 0; i < (int)f.shape[0]; i++)
        for (int j = 0; j < (int)f.shape[1]; j++)
            for (int k = 0; k < (int)f.shape[2]; k++) f.at[f.idx(i, j, k)] = rhs_value(i, j, k);
    DeviceArray<double_t>& top = solver.get_top_bc(0).arr;
    for (int i = 0; i < (int)top.shape[0]; i++)
        for (int j = 0; j < (int)top.shape[1]; j++) top.at[top.idx(i, j, 0)] = top_value(i, j);
    solver.verbose(true);
    solver.to_device();
    solver.solve("vcycle", 2, -1.0, argv[2]);
    solver.to_host();
    const DeviceArray<double_t>& u = solver.get_solution(0);
    FILE* out = std::fopen(argv[1], "wb");
    if (!out) return 1;
    for (int i = 0; i < (int)u.shape[0]; i++)
        for (int j = 0; j < (int)u.shape[1]; j++)
            for (int k = 0; k < (int)u.shape[2]; k++) {
                const double v = u.at[u.idx(i, j, k)];
                std::fwrite(&v, sizeof v, 1, out);
            }
    std::fclose(out);
    std::cout << "rel_res " << solver.relative_residual() << " iters " << solver.solve_iterations() << std::endl;
    return EXIT_SUCCESS;
}
