// Runs the B200 solver adapter (biofvm-b_b200/host/reference_adapter/) inside
// a reference build. Test infrastructure: built by `make -C oracle adapter`
// against the reference's own objects, with the one-line friend declaration
// the adapter documents added to a copy of BioFVM_microenvironment.h under
// oracle/_ref/patched/ (the reference tree itself is not modified).
//
// Two Microenvironments are set up as examples/test_VS.cpp:218-240 does, with
// the same seeded field, D, lambda and Dirichlet state. One steps through the
// reference's LOD_3D, the other through the adapter registered in the
// reference's diffusion_decay_solver pointer. Output, one line:
//   "identical <steps>"            the fields agree bit for bit after <steps> steps
//   "differs <max |diff|>"         they do not
//   "unchanged"                    the adapter's first step failed (its error is
//                                  printed above) and left the field untouched
#include <cmath>
#include <cstdio>
#include <cstdlib>
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

static void setup(Microenvironment &M, int *dims, int *coords) {
    const double D[3] = {1e5, 3e3, 40.0}, lam[3] = {0.1, 0.01, 1.0};
    M.set_density(0, "substrate0", "dimensionless");
    M.diffusion_coefficients[0] = D[0];
    M.decay_rates[0] = lam[0];
    for (int d = 1; d < 3; ++d) {
        M.add_density("substrate" + std::to_string(d), "dimensionless");
        M.diffusion_coefficients[d] = D[d];
        M.decay_rates[d] = lam[d];
    }
    M.resize_space_uniform(0.0, 240.0, 0.0, 200.0, 0.0, 160.0, 20.0, dims, coords);
    std::mt19937_64 gen(5);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (double &x : *M.p_density_vectors) x = u(gen);
    M.set_substrate_dirichlet_activation(1, false);  // substrates 0 and 2 keep the default faces (100.0)
}

int main(int argc, char **argv) {
    const int steps = argc > 1 ? std::atoi(argv[1]) : 5;
    int dims[3] = {1, 1, 1}, coords[3] = {0, 0, 0};
    Microenvironment ref, gpu;
    setup(ref, dims, coords);
    setup(gpu, dims, coords);
    ref.diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D;
    gpu.diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D_B200;
    const std::vector<double> before = *gpu.p_density_vectors;

    gpu.simulate_diffusion_decay(0.01, 1, 0, coords, dims, MPI_COMM_WORLD);
    if (*gpu.p_density_vectors == before) {  // a failed step leaves the field as it was
        std::printf("unchanged\n");
        return 0;
    }
    for (int s = 1; s < steps; ++s) gpu.simulate_diffusion_decay(0.01, 1, 0, coords, dims, MPI_COMM_WORLD);
    for (int s = 0; s < steps; ++s) ref.simulate_diffusion_decay(0.01, 1, 0, coords, dims, MPI_COMM_WORLD);
    double worst = 0.0;
    const std::vector<double> &a = *ref.p_density_vectors, &b = *gpu.p_density_vectors;
    for (size_t n = 0; n < a.size(); ++n) worst = std::fmax(worst, std::fabs(a[n] - b[n]));
    if (a == b) std::printf("identical %d\n", steps);
    else std::printf("differs %.3e\n", worst);
    release_b200_solver(gpu);
    return 0;
}
