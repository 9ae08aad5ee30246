// example_diffusion.cpp -- a DaRe-style implicit time loop written against
// the C++ host API (include/dare_gpu.hpp), as a DaRe user would port
// test/Verification/counter_diffusion1D.cpp: Gaussian bump on the unit cube,
// Dirichlet 1 / 0 on x = 0 / 1, zero gradient elsewhere, implicit Euler with
// Jacobi-BiCGStab2 to a relative residual of 1e-10.
//
//   example_diffusion [n=32] [steps=3] [out.bin] [slabs=0]
// Prints one JSON line; writes the final ghosted field (float64) to out.bin.
// With slabs > 0 the loop runs on that many slabs of i-planes (the grid
// distributed as over ranks), gathered into the field at the end.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "dare_gpu.hpp"

int main(int argc, char** argv) {
    const int n = argc > 1 ? std::atoi(argv[1]) : 32;
    const int steps = argc > 2 ? std::atoi(argv[2]) : 3;
    const char* out = argc > 3 && argv[3][0] ? argv[3] : nullptr;
    const int num_slabs = argc > 4 ? std::atoi(argv[4]) : 0;
    try {
        dare_b200::Context ctx(0);
        dare_b200::Cartesian grid(ctx, {n, n, n}, {1., 1., 1.}, 2);
        dare_b200::Field field(grid, 2);
        std::vector<double> phi((size_t)grid.GetNumberLocalCells(), 0.);
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) {
                    const double x = (i + 0.5) / n - 0.5, y = (j + 0.5) / n - 0.5, z = (k + 0.5) / n - 0.5;
                    phi[(size_t)grid.MapInternalToLocal(i, j, k)] = std::exp(-(x * x + y * y + z * z) / (2. * 0.01));
                }
        field.Upload(phi, 0);
        field.Upload(phi, 1);

        dare_b200::Trilinos system(grid);
        system.SetBC(DARE_WEST, DARE_BC_DIRICHLET, 1.);
        system.SetBC(DARE_EAST, DARE_BC_DIRICHLET, 0.);
        for (int face = DARE_SOUTH; face <= DARE_TOP; face++) system.SetBC(face, DARE_BC_NEUMANN, 0.);

        dare_b200::Assembly functor;
        functor.dt = 1e-2;
        functor.diffusion = true;
        functor.D = 1e-3;

        dare_b200::BiCGStab2 solver({{"Convergence Tolerance", 1e-10}, {"Maximum Iterations", 5000}});
        solver.SetRelativeTolerance(true);
        std::printf("{\"n\": %d, \"steps\": %d, \"slabs\": %d, \"iters\": [", n, steps, num_slabs);
        if (num_slabs > 0) {
            dare_b200::Slabs slabs(system, num_slabs);
            slabs.Scatter(field);
            // a scalar diffusivity: every slab's functor is the grid's
            const std::vector<dare_b200::Assembly> functors((size_t)num_slabs, functor);
            for (int s = 0; s < steps; s++) {
                dare_solve_report rep{};
                if (slabs.TimeStep(solver, functors, &rep) != dare_b200::BiCGStab2::ReturnType::Converged) {
                    std::printf("]}\n");
                    std::fprintf(stderr, "solver did not converge\n");
                    return 2;
                }
                std::printf("%s%d", s ? ", " : "", rep.iters);
            }
            slabs.Gather(field);
        } else {
            for (int s = 0; s < steps; s++) {
                if (solver.TimeStep(system, field, functor) != dare_b200::BiCGStab2::ReturnType::Converged) {
                    std::printf("]}\n");
                    std::fprintf(stderr, "solver did not converge\n");
                    return 2;
                }
                std::printf("%s%d", s ? ", " : "", solver.getNumIters());
            }
        }
        const std::vector<double> result = field.Download(0);
        double sum = 0.;
        for (int64_t c = 0; c < grid.GetNumberLocalCellsInternal(); c++) {
            const int64_t i = c / ((int64_t)n * n), j = (c / n) % n, k = c % n;
            sum += result[(size_t)grid.MapInternalToLocal(i, j, k)];
        }
        std::printf("], \"sum\": %.17g}\n", sum);
        if (out) {
            FILE* f = std::fopen(out, "wb");
            if (!f) return 3;
            std::fwrite(result.data(), sizeof(double), result.size(), f);
            std::fclose(f);
        }
    } catch (const dare_b200::Error& e) {
        std::fprintf(stderr, "dare_b200 error: %s\n", e.what());
        return 1;
    }
    return 0;
}
