/*
 * ref_driver.cpp -- a thin C entry layer around the UNMODIFIED reference
 * BioFVM-B library (compiled from its own sources by oracle/Makefile into
 * oracle/_ref/libbiofvm_ref.so).
 *
 * TEST INFRASTRUCTURE ONLY. It is the checker used by tests/, by the golden
 * fixture generator (tests/golden/make_golden.py) and by bench.py's CPU
 * baseline / reference arm. The product never links or calls it.
 *
 * Everything below drives the reference exactly as its own example drivers
 * do (examples/test_VS.cpp:218-291, examples/complete_diffusion_demo.cpp:
 * 223-240, 491-492): set_density/add_density, public D and lambda vectors,
 * resize_space_uniform with a 1x1x1 Cartesian topology, solver registration
 * through the diffusion_decay_solver function pointer, Dirichlet setters,
 * bulk callbacks, and Basic_Agent set-up. The one deliberate deviation is the
 * agent phase: Microenvironment::simulate_cell_sources_and_sinks runs an
 * `omp parallel for` over agents (BioFVM_microenvironment.cpp:1155-1164)
 * that races when agents share a voxel, so ref_cells_step calls
 * Basic_Agent::simulate_secretion_and_uptake serially in all_basic_agents
 * order, which is the order the reference intends.
 */
#include <cstring>
#include <map>
#include <vector>
#include <string>
#include <omp.h>
#include "BioFVM.h"

using namespace BioFVM;

namespace {

struct RefEnv {
    Microenvironment *M = nullptr;
    std::vector<double> bulk_S, bulk_T, bulk_U;   // V*S each
    std::vector<Basic_Agent *> agents;            // in creation order
    int dims[3] = {1, 1, 1};
    int coords[3] = {0, 0, 0};
};

std::map<Microenvironment *, RefEnv *> g_env;

RefEnv *env_of(Microenvironment *M) {
    auto it = g_env.find(M);
    return it == g_env.end() ? nullptr : it->second;
}

// Bulk callbacks read the tabulated arrays of the Microenvironment they are
// called for (signature BioFVM_microenvironment.h:165-167).
void bulk_S_fn(Microenvironment *M, int v, double *out) {
    RefEnv *e = env_of(M);
    int S = M->number_of_densities();
    for (int d = 0; d < S; ++d) out[d] = e->bulk_S[(size_t)v * S + d];
}
void bulk_T_fn(Microenvironment *M, int v, double *out) {
    RefEnv *e = env_of(M);
    int S = M->number_of_densities();
    for (int d = 0; d < S; ++d) out[d] = e->bulk_T[(size_t)v * S + d];
}
void bulk_U_fn(Microenvironment *M, int v, double *out) {
    RefEnv *e = env_of(M);
    int S = M->number_of_densities();
    for (int d = 0; d < S; ++d) out[d] = e->bulk_U[(size_t)v * S + d];
}

}  // namespace

extern "C" {

// Build a Microenvironment the way examples/test_VS.cpp:218-240 does.
void *ref_create(double x0, double x1, double y0, double y1, double z0, double z1,
                 double dx, int n_substrates, const double *D, const double *lambda) {
    RefEnv *e = new RefEnv();
    Microenvironment *M = new Microenvironment();
    M->set_density(0, "substrate0", "dimensionless");
    M->diffusion_coefficients[0] = D[0];
    M->decay_rates[0] = lambda[0];
    for (int i = 1; i < n_substrates; ++i) {
        M->add_density("substrate" + std::to_string(i), "dimensionless");
        M->diffusion_coefficients[i] = D[i];
        M->decay_rates[i] = lambda[i];
    }
    M->resize_space_uniform(x0, x1, y0, y1, z0, z1, dx, e->dims, e->coords);
    M->diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D;
    e->M = M;
    g_env[M] = e;
    return M;
}

void ref_destroy(void *h) {
    Microenvironment *M = (Microenvironment *)h;
    RefEnv *e = env_of(M);
    if (!e) return;
    // Agents created for this environment are removed from the global list.
    for (Basic_Agent *a : e->agents) {
        for (size_t i = 0; i < all_basic_agents.size(); ++i)
            if (all_basic_agents[i] == a) { all_basic_agents.erase(all_basic_agents.begin() + i); break; }
        delete a;
    }
    g_env.erase(M);
    delete e;
    delete M;
}

void ref_sizes(void *h, int *out4) {
    Microenvironment *M = (Microenvironment *)h;
    out4[0] = M->mesh.x_size;
    out4[1] = M->mesh.y_size;
    out4[2] = M->mesh.z_size;
    out4[3] = M->number_of_densities();
}

// 0 = scalar LOD_3D (BioFVM_parallel.cpp:693), 1 = AVX256D (BioFVM_parallel.cpp:1411)
void ref_set_solver(void *h, int which) {
    Microenvironment *M = (Microenvironment *)h;
    typedef void (*solver_fn)(Microenvironment &, double, int, int, int *, int *, MPI_Comm);
    solver_fn scalar = diffusion_decay_solver__constant_coefficients_LOD_3D;
    solver_fn avx = diffusion_decay_solver__constant_coefficients_LOD_3D_AVX256D;
    M->diffusion_decay_solver = which == 1 ? avx : scalar;
}

void ref_set_field(void *h, const double *src) {
    Microenvironment *M = (Microenvironment *)h;
    std::memcpy(M->p_density_vectors->data(), src, M->p_density_vectors->size() * sizeof(double));
}

void ref_get_field(void *h, double *dst) {
    Microenvironment *M = (Microenvironment *)h;
    std::memcpy(dst, M->p_density_vectors->data(), M->p_density_vectors->size() * sizeof(double));
}

void ref_set_dirichlet_activation(void *h, int d, int on) {
    ((Microenvironment *)h)->set_substrate_dirichlet_activation(d, on != 0);
}

void ref_set_dirichlet_value(void *h, int d, double v) {
    ((Microenvironment *)h)->set_substrate_dirichlet_value(d, v);
}

// Per-voxel Dirichlet values through add_dirichlet_node(x,y,z,values)
// (BioFVM_microenvironment.cpp:237-244). `values` is a full V*S array; only
// outer-face voxels are written, which are the only entries the LOD path reads.
void ref_set_dirichlet_face_values(void *h, const double *values) {
    Microenvironment *M = (Microenvironment *)h;
    int nx = M->mesh.x_size, ny = M->mesh.y_size, nz = M->mesh.z_size, S = M->number_of_densities();
    std::vector<double> vals(S);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                bool face = i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1;
                if (!face) continue;
                size_t base = (((size_t)i * ny + j) * nz + k) * S;
                for (int d = 0; d < S; ++d) vals[d] = values[base + d];
                M->add_dirichlet_node(i, j, k, vals);
            }
}

void ref_apply_dirichlet(void *h) {
    ((Microenvironment *)h)->apply_dirichlet_conditions(0, 1);
}

void ref_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
}

int ref_max_threads(void) { return omp_get_max_threads(); }

void ref_step(void *h, double dt, int n_steps) {
    Microenvironment *M = (Microenvironment *)h;
    RefEnv *e = env_of(M);
    for (int s = 0; s < n_steps; ++s)
        M->simulate_diffusion_decay(dt, 1, 0, e->coords, e->dims, 0);
}

// Bulk sources/sinks as three tabulated callbacks (S, T, U), V*S each.
void ref_set_bulk(void *h, const double *S_rate, const double *T_target, const double *U_rate) {
    Microenvironment *M = (Microenvironment *)h;
    RefEnv *e = env_of(M);
    size_t n = M->p_density_vectors->size();
    e->bulk_S.assign(S_rate, S_rate + n);
    e->bulk_T.assign(T_target, T_target + n);
    e->bulk_U.assign(U_rate, U_rate + n);
    M->bulk_supply_rate_function = bulk_S_fn;
    M->bulk_supply_target_densities_function = bulk_T_fn;
    M->bulk_uptake_rate_function = bulk_U_fn;
}

void ref_bulk_step(void *h, double dt) {
    ((Microenvironment *)h)->simulate_bulk_sources_and_sinks(dt);
}

// Agents the way examples/complete_diffusion_demo.cpp:223-240 makes them:
// create_basic_agent, register_microenvironment, assign_position, set the
// volume and rates, then set_internal_uptake_constants(dt). Returns the
// number of agents whose position was accepted.
int ref_add_agents(void *h, int n, const double *pos, const double *volume,
                   const double *secretion, const double *uptake, const double *saturation,
                   double dt) {
    Microenvironment *M = (Microenvironment *)h;
    RefEnv *e = env_of(M);
    int S = M->number_of_densities();
    int accepted = 0;
    for (int a = 0; a < n; ++a) {
        Basic_Agent *p = create_basic_agent();
        p->register_microenvironment(M);
        if (p->assign_position(pos[3 * a], pos[3 * a + 1], pos[3 * a + 2], 0, e->dims)) ++accepted;
        p->set_total_volume(volume[a]);
        for (int d = 0; d < S; ++d) {
            (*p->secretion_rates)[d] = secretion[(size_t)a * S + d];
            (*p->uptake_rates)[d] = uptake[(size_t)a * S + d];
            (*p->saturation_densities)[d] = saturation[(size_t)a * S + d];
        }
        p->set_internal_uptake_constants(dt);
        e->agents.push_back(p);
    }
    return accepted;
}

void ref_agent_voxels(void *h, int *out) {
    RefEnv *e = env_of((Microenvironment *)h);
    for (size_t a = 0; a < e->agents.size(); ++a) out[a] = e->agents[a]->get_current_voxel_index();
}

// Serial secretion/uptake in creation order (see the file header).
// The serial MATLAB v4 writer, Microenvironment::write_to_matlab(filename)
// (BioFVM_microenvironment.cpp:1079-1107).
void ref_write_matlab(void *h, const char *filename) {
    Microenvironment *M = (Microenvironment *)h;
    M->write_to_matlab(std::string(filename));
}

// The text dump drivers write through print_result with the
// print_voxels_densities hook (BioFVM_microenvironment.cpp:375-379,
// BioFVM_parallel.cpp:2334-2366), at rank 0 of 1; appends to filename.
void ref_print_densities(void *h, const char *filename) {
    Microenvironment *M = (Microenvironment *)h;
    int coords[3] = {0, 0, 0}, dims[3] = {1, 1, 1};
    std::string name(filename);
    M->print_voxels_densities = print_voxels_densities;
    M->print_result(0.0, 1, 0, coords, &name, dims, MPI_COMM_WORLD);
}

// compute_all_gradient_vectors (BioFVM_microenvironment.cpp:1243-1402), then
// the public accessor gradient_vector(n) per voxel: out[(n*S + q)*3 + c]. The
// jumps it uses are set by the first solver call, so call ref_step first.
void ref_gradients(void *h, double *out) {
    Microenvironment *M = (Microenvironment *)h;
    M->compute_all_gradient_vectors();
    const int V = (int)M->mesh.voxels.size(), S = M->number_of_densities();
    for (int n = 0; n < V; ++n) {
        std::vector<gradient> &g = M->gradient_vector(n);
        for (int q = 0; q < S; ++q)
            for (int c = 0; c < 3; ++c) out[((size_t)n * S + q) * 3 + c] = g[q][c];
    }
}

// The per-voxel path: reset, then gradient_vector(n) computes each voxel on
// demand with compute_gradient_vector (BioFVM_microenvironment.cpp:1404-1535).
void ref_gradients_per_voxel(void *h, double *out) {
    Microenvironment *M = (Microenvironment *)h;
    M->reset_all_gradient_vectors();
    const int V = (int)M->mesh.voxels.size(), S = M->number_of_densities();
    for (int n = 0; n < V; ++n) {
        std::vector<gradient> &g = M->gradient_vector(n);
        for (int q = 0; q < S; ++q)
            for (int c = 0; c < 3; ++c) out[((size_t)n * S + q) * 3 + c] = g[q][c];
    }
}

void ref_cells_step(void *h, double dt) {
    Microenvironment *M = (Microenvironment *)h;
    RefEnv *e = env_of(M);
    for (Basic_Agent *a : e->agents) a->simulate_secretion_and_uptake(M, dt);
}

}  // extern "C"
