// BioFVM_b200_solver.cpp -- the B200 LOD solver behind BioFVM-B's own plugin
// point, for a build that keeps the reference library.
//
// A BioFVM-B build adds this file to its objects, links
//   -L<repo>/biofvm-b_b200/lib -lbiofvm_b200 -Wl,-rpath,<repo>/biofvm-b_b200/lib
// and adds one line to BioFVM_microenvironment.h, next to the other solvers'
// friend declarations (:268-276), because the solver reads the private
// Dirichlet arrays as the reference's own solvers do:
//   friend void diffusion_decay_solver__constant_coefficients_LOD_3D_B200(Microenvironment &, double, int, int, int *, int *, MPI_Comm);
// A driver then registers it where the reference's drivers register theirs
// (examples/test_VS.cpp:240):
//   microenvironment.diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D_B200;
//
// The field stays in the Microenvironment's own std::vector<double>. Each call
// copies it to the device, runs one FP64 LOD step there (bit-exact with the
// reference's LOD_3D) and copies it back, so host code sees what the CPU
// solver would have produced. The device grid is created on the first call,
// where the reference computes its Thomas factors (BioFVM_parallel.cpp:714),
// and kept per Microenvironment; the factors stay at the first call's dt, D
// and lambda, as the reference's do. Errors are printed, as the reference
// prints its own (BioFVM_parallel.cpp:705-710), and leave the field unchanged.
#include <cstdint>
#include <iostream>
#include <map>
#include <vector>

#include "BioFVM_microenvironment.h"
#include "biofvm_b200.h"

namespace BioFVM {

namespace {
std::map<Microenvironment *, bfb_env> g_b200_envs;

void b200_report(const char *what) { std::cout << "B200 solver: " << what << ": " << bfb_last_error() << std::endl; }
}  // namespace

void diffusion_decay_solver__constant_coefficients_LOD_3D_B200(Microenvironment &M, double dt, int mpi_Size,
                                                                int mpi_Rank, int *mpi_Coords, int *mpi_Dims,
                                                                MPI_Comm mpi_Cart_comm) {
    (void)mpi_Rank;
    (void)mpi_Coords;
    (void)mpi_Dims;
    (void)mpi_Cart_comm;
    if (mpi_Size != 1) {
        std::cout << "B200 solver: one device-resident grid per process (mpi_Size must be 1)" << std::endl;
        return;
    }
    if (!M.mesh.uniform_mesh) {  // the reference solver's own check (BioFVM_parallel.cpp:705-710)
        std::cout << "Error: This algorithm is written for uniform Cartesian meshes. Try: other solvers!" << std::endl
                  << std::endl;
        return;
    }
    const int S = M.number_of_densities();
    auto it = g_b200_envs.find(&M);
    if (it == g_b200_envs.end()) {
        bfb_env env = nullptr;
        if (bfb_create(&env, M.mesh.x_size, M.mesh.y_size, M.mesh.z_size, S, M.mesh.dx, BFB_FP64, 0) != BFB_OK) {
            b200_report("bfb_create");
            return;
        }
        if (bfb_set_coefficients(env, M.diffusion_coefficients.data(), M.decay_rates.data()) != BFB_OK) {
            b200_report("bfb_set_coefficients");
            bfb_destroy(env);
            return;
        }
        it = g_b200_envs.emplace(&M, env).first;
    }
    std::vector<uint8_t> activation(S);
    for (int d = 0; d < S; ++d) activation[d] = M.dirichlet_activation_vector[d] ? 1 : 0;
    // all six faces follow the activation, the reference's rule (BioFVM_microenvironment.cpp:381-484)
    if (bfb_set_dirichlet(it->second, M.dirichlet_value_vectors.data(), activation.data(), nullptr) != BFB_OK) {
        b200_report("bfb_set_dirichlet");
        return;
    }
    if (bfb_step_host(it->second, M.p_density_vectors->data(), dt, 1) != BFB_OK) b200_report("bfb_step_host");
}

// Frees the device grid held for M; call it before M is destroyed if M's
// address may be reused by another Microenvironment.
void release_b200_solver(Microenvironment &M) {
    auto it = g_b200_envs.find(&M);
    if (it == g_b200_envs.end()) return;
    bfb_destroy(it->second);
    g_b200_envs.erase(it);
}

}  // namespace BioFVM
