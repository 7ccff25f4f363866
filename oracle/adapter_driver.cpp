// Runs the B200 solver adapter (biofvm-b_b200/host/reference_adapter/) inside
// a reference build. Test infrastructure: built by `make -C oracle adapter`
// against the reference's own objects, with the one-line friend declaration
// the adapter documents added to a copy of BioFVM_microenvironment.h under
// oracle/_ref/patched/ (the reference tree itself is not modified).
//
//   adapter_driver [steps]
//   adapter_driver compare <steps> <x_len> <y_len> <z_len> <S> [dt_after_first]
//       Two Microenvironments are set up as examples/test_VS.cpp:218-240 does
//       (domain [0, len] per axis at dx = 20, S substrates, the reference's
//       default Dirichlet state -- every substrate active with the value 100.0
//       after resize_space -- except substrate 1, which is deactivated), with
//       the same seeded field, D and lambda. One steps through the reference's
//       LOD_3D, the other through the adapter registered in the reference's
//       diffusion_decay_solver pointer. The first step uses dt = 0.01; with
//       dt_after_first the later steps pass that dt, which both solvers must
//       ignore (their factors stay at the first call's, BioFVM_parallel.cpp:714,
//       913). The default is 5 steps on 240 x 200 x 160 with S = 3.
//       Output, one line:
//         "identical <steps>"      the fields agree bit for bit after <steps> steps
//         "differs <max |diff|>"   they do not
//         "unchanged"              the adapter's first step failed (its error is
//                                  printed above) and left the field untouched
//   adapter_driver time <edge> <S> <steps>
//       One Microenvironment of edge^3 voxels (dx = 20) and S substrates with
//       the reference's default Dirichlet state, stepped through the adapter:
//       two untimed steps, then <steps> timed ones (wall clock around
//       simulate_diffusion_decay). Output: "ms_per_step <t>".
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "BioFVM_microenvironment.h"  // the patched copy (found first), before BioFVM.h pulls in the original
#include "BioFVM.h"

namespace BioFVM {
void diffusion_decay_solver__constant_coefficients_LOD_3D_B200(Microenvironment &, double, int, int, int *, int *,
                                                                MPI_Comm);
void release_b200_solver(Microenvironment &M);
}  // namespace BioFVM

using namespace BioFVM;

static void setup(Microenvironment &M, int *dims, int *coords, double xl, double yl, double zl, int S,
                  bool deactivate_one) {
    std::mt19937_64 gen(5);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    M.set_density(0, "substrate0", "dimensionless");
    for (int d = 1; d < S; ++d) M.add_density("substrate" + std::to_string(d), "dimensionless");
    for (int d = 0; d < S; ++d) {  // D log-uniform in [1e2, 1e5], lambda in [1e-3, 1]
        M.diffusion_coefficients[d] = std::exp(std::log(1e2) + u(gen) * (std::log(1e5) - std::log(1e2)));
        M.decay_rates[d] = std::exp(std::log(1e-3) + u(gen) * (0.0 - std::log(1e-3)));
    }
    M.resize_space_uniform(0.0, xl, 0.0, yl, 0.0, zl, 20.0, dims, coords);
    for (double &x : *M.p_density_vectors) x = u(gen);
    if (deactivate_one && S > 1) M.set_substrate_dirichlet_activation(1, false);
}

static int compare(int steps, double xl, double yl, double zl, int S, double dt_later) {
    int dims[3] = {1, 1, 1}, coords[3] = {0, 0, 0};
    Microenvironment ref, gpu;
    setup(ref, dims, coords, xl, yl, zl, S, true);
    setup(gpu, dims, coords, xl, yl, zl, S, true);
    ref.diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D;
    gpu.diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D_B200;
    const std::vector<double> before = *gpu.p_density_vectors;

    gpu.simulate_diffusion_decay(0.01, 1, 0, coords, dims, MPI_COMM_WORLD);
    if (*gpu.p_density_vectors == before) {  // a failed step leaves the field as it was
        std::printf("unchanged\n");
        return 0;
    }
    for (int s = 1; s < steps; ++s) gpu.simulate_diffusion_decay(dt_later, 1, 0, coords, dims, MPI_COMM_WORLD);
    for (int s = 0; s < steps; ++s)
        ref.simulate_diffusion_decay(s == 0 ? 0.01 : dt_later, 1, 0, coords, dims, MPI_COMM_WORLD);
    double worst = 0.0;
    const std::vector<double> &a = *ref.p_density_vectors, &b = *gpu.p_density_vectors;
    for (size_t n = 0; n < a.size(); ++n) worst = std::fmax(worst, std::fabs(a[n] - b[n]));
    if (a == b) std::printf("identical %d\n", steps);
    else std::printf("differs %.3e\n", worst);
    release_b200_solver(gpu);
    return 0;
}

static int time_steps(int edge, int S, int steps) {
    int dims[3] = {1, 1, 1}, coords[3] = {0, 0, 0};
    Microenvironment M;
    setup(M, dims, coords, 20.0 * edge, 20.0 * edge, 20.0 * edge, S, false);
    M.diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D_B200;
    for (int s = 0; s < 2; ++s) M.simulate_diffusion_decay(0.01, 1, 0, coords, dims, MPI_COMM_WORLD);
    const auto t0 = std::chrono::steady_clock::now();
    for (int s = 0; s < steps; ++s) M.simulate_diffusion_decay(0.01, 1, 0, coords, dims, MPI_COMM_WORLD);
    const auto t1 = std::chrono::steady_clock::now();
    std::printf("ms_per_step %.4f\n", std::chrono::duration<double, std::milli>(t1 - t0).count() / steps);
    release_b200_solver(M);
    return 0;
}

int main(int argc, char **argv) {
    if (argc > 1 && std::strcmp(argv[1], "time") == 0) {
        if (argc < 5) return 2;
        return time_steps(std::atoi(argv[2]), std::atoi(argv[3]), std::atoi(argv[4]));
    }
    if (argc > 1 && std::strcmp(argv[1], "compare") == 0) {
        if (argc < 7) return 2;
        const double dt_later = argc > 7 ? std::atof(argv[7]) : 0.01;
        return compare(std::atoi(argv[2]), std::atof(argv[3]), std::atof(argv[4]), std::atof(argv[5]),
                       std::atoi(argv[6]), dt_later);
    }
    const int steps = argc > 1 ? std::atoi(argv[1]) : 5;
    return compare(steps, 240.0, 200.0, 160.0, 3, 0.01);
}
