// facade_demo.cpp -- a driver written the way the reference's examples are
// (examples/complete_diffusion_demo.cpp: substrates, resize, Dirichlet,
// agents, then diffusion -> cells each step), compiled against the B200
// facade. Inputs come from an integer hash so that a Python test can rebuild
// them exactly and check the output field against the oracle.
//
//   facade_demo <out.bin> <precision 0=FP64|1=FP32> <host sync 0=every step|1=lazy> [steps]
//               [bulk 0=none|1=callbacks every call|2=callbacks tabulated once]
// writes the field to out.bin, its gradient vectors to out.bin.grad and the
// reference's MATLAB v4 snapshot to out.bin.mat
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "BioFVM_B200.h"

using namespace BioFVM_B200;

static double hash01(unsigned a, unsigned b) {
    unsigned h = a * 2654435761u + b * 40503u + 12345u;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    return (double)(h % 100003u) / 100003.0;
}

// time-invariant bulk source/sink callbacks (the reference's signature)
static void supply_rate(Microenvironment *M, int n, double *out) {
    for (int d = 0; d < M->number_of_densities(); ++d) out[d] = 2.0 * hash01(n, 50 + d);
}
static void supply_target(Microenvironment *M, int n, double *out) {
    for (int d = 0; d < M->number_of_densities(); ++d) out[d] = 5.0 * hash01(n, 60 + d);
}
static void uptake_rate(Microenvironment *M, int n, double *out) {
    for (int d = 0; d < M->number_of_densities(); ++d) out[d] = 0.5 * hash01(n, 70 + d);
}

int main(int argc, char **argv) {
    if (argc < 4) {
        std::printf("usage: %s <out.bin> <precision 0|1> <host sync 0|1> [steps]\n", argv[0]);
        return 2;
    }
    const int steps = argc > 4 ? std::atoi(argv[4]) : 10;
    const int bulk = argc > 5 ? std::atoi(argv[5]) : 0;
    const double dt = 0.01;
    Microenvironment M;
    M.set_precision(std::atoi(argv[2]) ? Precision::FP32 : Precision::FP64);
    M.set_host_sync(std::atoi(argv[3]) ? HostSync::Lazy : HostSync::EveryStep);
    M.set_density(0, "oxygen", "mmHg");
    M.diffusion_coefficients[0] = 1e5;
    M.decay_rates[0] = 0.1;
    M.add_density("signal", "dimensionless");
    M.diffusion_coefficients[1] = 3e3;
    M.decay_rates[1] = 0.01;
    int dims[3] = {1, 1, 1}, coords[3] = {0, 0, 0};
    M.resize_space_uniform(0, 400, 0, 360, 0, 320, 20, dims, coords);
    M.diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D_B200;

    const int S = M.number_of_densities();
    for (int n = 0; n < M.number_of_voxels(); ++n)
        for (int d = 0; d < S; ++d) (*M.p_density_vectors)[(size_t)n * S + d] = hash01(n, d);
    M.mark_host_modified();
    M.set_substrate_dirichlet_value(0, 38.0);
    M.set_substrate_dirichlet_activation(1, false);

    for (int a = 0; a < 200; ++a) {
        Basic_Agent *p = create_basic_agent();
        p->register_microenvironment(&M);
        p->assign_position(400.0 * hash01(a, 7), 360.0 * hash01(a, 8), 320.0 * hash01(a, 9), 0, dims);
        p->set_total_volume(4.0 / 3.0 * M_PI * 125.0);
        for (int d = 0; d < S; ++d) {
            (*p->secretion_rates)[d] = 10.0 * hash01(a, 20 + d);
            (*p->uptake_rates)[d] = 10.0 * hash01(a, 30 + d);
            (*p->saturation_densities)[d] = 10.0 * hash01(a, 40 + d);
        }
        p->set_internal_uptake_constants(dt);
    }

    if (bulk) {
        M.bulk_supply_rate_function = supply_rate;
        M.bulk_supply_target_densities_function = supply_target;
        M.bulk_uptake_rate_function = uptake_rate;
        M.set_bulk_tabulation(bulk == 2 ? BulkTabulation::Once : BulkTabulation::EveryCall);
    }
    for (int s = 0; s < steps; ++s) {
        if (bulk) M.simulate_bulk_sources_and_sinks(dt);
        M.simulate_diffusion_decay(dt, 1, 0, coords, dims, 0);
        M.simulate_cell_sources_and_sinks(dt);
        if (M.last_status() != BFB_OK) return 1;
    }
    M.sync_to_host();
    std::FILE *f = std::fopen(argv[1], "wb");
    if (!f) return 1;
    std::fwrite(M.p_density_vectors->data(), sizeof(double), M.p_density_vectors->size(), f);
    std::fclose(f);
    // chemotaxis-style consumer: the gradient vectors after the last step
    M.compute_all_gradient_vectors();
    std::FILE *g = std::fopen((std::string(argv[1]) + ".grad").c_str(), "wb");
    if (!g) return 1;
    for (int n = 0; n < M.number_of_voxels(); ++n)
        for (int d = 0; d < S; ++d) std::fwrite(M.gradient_vector(n)[d].data(), sizeof(double), 3, g);
    std::fclose(g);
    M.write_to_matlab(std::string(argv[1]) + ".mat");
    std::printf("facade_demo: %d x %d x %d x %d, %d steps, checksum %.17g\n", M.mesh.x_size, M.mesh.y_size,
                M.mesh.z_size, S, steps, M.checksum()[0]);
    return 0;
}
