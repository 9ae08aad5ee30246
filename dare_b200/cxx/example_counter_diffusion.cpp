// example_counter_diffusion.cpp -- test/Verification/counter_diffusion1D.cpp
// written against the C++ host API (include/dare_gpu.hpp): two components
// on nx cells of [0, 1], the reference's functor
//     (*mblock) = ddt(field);  (*mblock) -= div(grad(*mblock));
// as a MatrixBlock of terms, component 0 with Dirichlet 1 on the west face and
// zero gradient on the east, component 1 the reverse, implicit Euler with
// dt = 1e-3 and Jacobi-BiCGStab2 to a relative residual of 1e-10.
//
//   example_counter_diffusion [nx=10] [steps=20] [out.bin]
// Prints one JSON line; writes the final ghosted field (float64, rows
// cell * 2 + c) to out.bin.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "dare_gpu.hpp"

int main(int argc, char** argv) {
    const int nx = argc > 1 ? std::atoi(argv[1]) : 10;
    const int steps = argc > 2 ? std::atoi(argv[2]) : 20;
    const char* out = argc > 3 ? argv[3] : nullptr;
    const double dt = 1e-3;
    try {
        dare_b200::Context ctx(0);
        dare_b200::Cartesian grid(ctx, {nx}, {1.}, 2);
        dare_b200::Field field(grid, 2, 2);
        std::vector<double> zero((size_t)grid.GetNumberLocalCells() * 2, 0.);   // field.SetValues(0.)
        field.Upload(zero, 0);
        field.Upload(zero, 1);

        dare_b200::Trilinos system(grid, 2);
        system.SetBC(DARE_WEST, DARE_BC_DIRICHLET, 1., 0);
        system.SetBC(DARE_EAST, DARE_BC_NEUMANN, 0., 0);
        system.SetBC(DARE_WEST, DARE_BC_NEUMANN, 0., 1);
        system.SetBC(DARE_EAST, DARE_BC_DIRICHLET, 1., 1);

        dare_b200::MatrixBlock mb;
        mb = dare_b200::DDT(dt);
        mb -= dare_b200::DivGrad();

        dare_b200::BiCGStab2 solver({{"Convergence Tolerance", 1e-10}, {"Maximum Iterations", 5000}});
        solver.SetRelativeTolerance(true);
        std::printf("{\"nx\": %d, \"steps\": %d, \"iters\": [", nx, steps);
        for (int s = 0; s < steps; s++) {
            if (solver.TimeStep(system, field, mb) != dare_b200::BiCGStab2::ReturnType::Converged) {
                std::printf("]}\n");
                std::fprintf(stderr, "solver did not converge\n");
                return 2;
            }
            std::printf("%s%d", s ? ", " : "", solver.getNumIters());
        }
        std::printf("]}\n");
        if (out) {
            const std::vector<double> result = field.Download(0);
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
