// BioFVM_B200.cpp -- the reference-shaped C++ facade over the B200 C ABI.
// Compiled with -ffp-contract=off: the few host-side formulas (agent binning
// and the cached secretion/uptake constants) use explicit std::fma exactly
// where the reference build fuses, so they match it bit for bit.
#include "BioFVM_B200.h"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <iostream>

namespace BioFVM_B200 {

std::vector<Basic_Agent *> all_basic_agents;
static Microenvironment *g_default = nullptr;

Microenvironment *get_default_microenvironment() { return g_default; }
void set_default_microenvironment(Microenvironment *M) { g_default = M; }

void zero_function(Microenvironment *M, int, double *out) {
    for (int i = 0; i < M->number_of_densities(); ++i) out[i] = 0.0;
}
void one_function(Microenvironment *M, int, double *out) {
    for (int i = 0; i < M->number_of_densities(); ++i) out[i] = 1.0;
}

// ---------------------------------------------------------------------------
// Cartesian_Mesh
// ---------------------------------------------------------------------------
std::vector<int> Cartesian_Mesh::cartesian_indices(int n) const {
    std::vector<int> out(3);
    const int YZ = y_size * z_size;
    out[0] = n / YZ;
    out[1] = (n - out[0] * YZ) / z_size;
    out[2] = n - z_size * (out[1] + y_size * out[0]);
    return out;
}

bool Cartesian_Mesh::is_position_valid(double x, double y, double z) const {
    // BioFVM_mesh.cpp:204-213 (closed box)
    if (x < bounding_box[0] || x > bounding_box[3]) return false;
    if (y < bounding_box[1] || y > bounding_box[4]) return false;
    if (z < bounding_box[2] || z > bounding_box[5]) return false;
    return true;
}

// nearest_voxel_local_index at rank 0 of dims {1,1,1} (BioFVM_parallel.cpp:418-522):
// floor to a voxel per axis, clamp to the truncated global extent, then
// index with the truncated local extents.
int Cartesian_Mesh::nearest_voxel_index(const std::vector<double> &p) const {
    const double h[3] = {dx, dy, dz};
    int v[3], ext[3];
    for (int a = 0; a < 3; ++a) {
        v[a] = (int)std::floor((p[a] - bounding_box[a]) / h[a]);
        ext[a] = (int)((bounding_box[3 + a] - bounding_box[a]) / h[a]);
        if (v[a] >= ext[a]) v[a] = ext[a] - 1;
        if (v[a] < 0) v[a] = 0;
    }
    return v[0] * ext[1] * ext[2] + v[1] * ext[2] + v[2];
}

Voxel Cartesian_Mesh::voxels(int n) const {
    Voxel out;
    std::vector<int> c = cartesian_indices(n);
    out.center[0] = x_coordinates.empty() ? 0 : x_coordinates[c[0]];
    out.center[1] = y_coordinates.empty() ? 0 : y_coordinates[c[1]];
    out.center[2] = z_coordinates.empty() ? 0 : z_coordinates[c[2]];
    out.volume = dV;
    return out;
}

// ---------------------------------------------------------------------------
// Microenvironment
// ---------------------------------------------------------------------------
Microenvironment::Microenvironment() {
    // BioFVM_microenvironment.cpp:140-216, with the GPU solver registered
    density_names.assign(1, "unnamed");
    density_units.assign(1, "none");
    diffusion_coefficients.assign(1, 0.0);
    decay_rates.assign(1, 0.0);
    field_.assign(1, 0.0);
    p_density_vectors = &field_;
    dirichlet_value_vectors.assign(1, 1.0);
    dirichlet_activation_vector.assign(1, true);
    diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D_B200;
    print_voxels_densities = &BioFVM_B200::print_voxels_densities;
    bulk_supply_rate_function = zero_function;
    bulk_supply_target_densities_function = zero_function;
    bulk_uptake_rate_function = zero_function;
    mesh.x_coordinates.assign(1, 0.0);
    mesh.y_coordinates.assign(1, 0.0);
    mesh.z_coordinates.assign(1, 0.0);
    if (!g_default) g_default = this;
}

Microenvironment::~Microenvironment() {
    if (env_) bfb_destroy(env_);
    if (g_default == this) g_default = nullptr;
}

void Microenvironment::report(int st, const char *where) {
    status = st;
    if (st != BFB_OK) std::cout << "BioFVM-B200 error in " << where << ": " << bfb_last_error() << std::endl;
}

static void insert_substrate(std::vector<double> &v, int V, int S_old, double fill) {
    std::vector<double> out((size_t)V * (S_old + 1));
    for (int n = 0; n < V; ++n) {
        for (int d = 0; d < S_old; ++d) out[(size_t)n * (S_old + 1) + d] = v[(size_t)n * S_old + d];
        out[(size_t)n * (S_old + 1) + S_old] = fill;
    }
    v.swap(out);
}

void Microenvironment::add_density(const std::string &nm, const std::string &units) {
    add_density(nm, units, 0.0, 0.0);
}

void Microenvironment::add_density(const std::string &nm, const std::string &units, double D, double lambda) {
    // BioFVM_microenvironment.cpp:883-946: appends a substrate, zero-fills it,
    // and resets all Dirichlet values to 1 with activation true
    sync_to_host();
    const int S_old = number_of_densities();
    density_names.push_back(nm);
    density_units.push_back(units);
    diffusion_coefficients.push_back(D);
    decay_rates.push_back(lambda);
    insert_substrate(field_, number_of_voxels(), S_old, 0.0);
    dirichlet_value_vectors.assign((size_t)number_of_voxels() * number_of_densities(), 1.0);
    dirichlet_activation_vector.assign(number_of_densities(), true);
    face_mask_.clear();
    if (env_) {
        bfb_destroy(env_);
        env_ = nullptr;
    }
    host_newer = true;
    params_dirty = true;
}

void Microenvironment::set_density(int index, const std::string &nm, const std::string &units) {
    density_names[index] = nm;
    density_units[index] = units;
}

void Microenvironment::set_density(int index, const std::string &nm, const std::string &units, double D,
                                   double lambda) {
    density_names[index] = nm;
    density_units[index] = units;
    diffusion_coefficients[index] = D;
    decay_rates[index] = lambda;
}

int Microenvironment::find_density_index(const std::string &nm) const {
    for (size_t i = 0; i < density_names.size(); ++i)
        if (density_names[i] == nm) return (int)i;
    return -1;
}

void Microenvironment::resize_space_uniform(double x0, double x1, double y0, double y1, double z0, double z1,
                                            double dx, int *dims, int *coords) {
    resize_space(x0, x1, y0, y1, z0, z1, dx, dx, dx, dims, coords);
}

void Microenvironment::resize_space(double x0, double x1, double y0, double y1, double z0, double z1, double dx,
                                    double dy, double dz, int *dims, int *coords) {
    if (dims && (dims[0] * dims[1] * dims[2] != 1))
        std::cout << "BioFVM-B200: one device-resident grid per process; dims are ignored" << std::endl;
    (void)coords;
    // Cartesian_Mesh::resize (BioFVM_parallel.cpp:71-160) at one rank
    const double eps = 1e-16;
    mesh.x_size = (int)std::ceil(eps + (x1 - x0) / dx);
    mesh.y_size = (int)std::ceil(eps + (y1 - y0) / dy);
    mesh.z_size = (int)std::ceil(eps + (z1 - z0) / dz);
    mesh.dx = dx;
    mesh.dy = dy;
    mesh.dz = dz;
    mesh.dV = dx * dy * dz;
    const double tol = 1e-16;  // BioFVM_parallel.cpp:124-127
    mesh.uniform_mesh = !(std::fabs(dx - dy) > tol || std::fabs(dy - dz) > tol || std::fabs(dx - dz) > tol);
    mesh.bounding_box[0] = x0;
    mesh.bounding_box[1] = y0;
    mesh.bounding_box[2] = z0;
    mesh.bounding_box[3] = x1;
    mesh.bounding_box[4] = y1;
    mesh.bounding_box[5] = z1;
    mesh.x_coordinates.resize(mesh.x_size);
    mesh.y_coordinates.resize(mesh.y_size);
    mesh.z_coordinates.resize(mesh.z_size);
    for (int i = 0; i < mesh.x_size; ++i) mesh.x_coordinates[i] = x0 + (i + 0.5) * dx;
    for (int i = 0; i < mesh.y_size; ++i) mesh.y_coordinates[i] = y0 + (i + 0.5) * dy;
    for (int i = 0; i < mesh.z_size; ++i) mesh.z_coordinates[i] = z0 + (i + 0.5) * dz;
    const size_t N = (size_t)number_of_voxels() * number_of_densities();
    field_.assign(N, 0.0);
    dirichlet_value_vectors.assign(N, 100.0);  // BioFVM_parallel.cpp:56
    if (env_) {
        bfb_destroy(env_);
        env_ = nullptr;
    }
    host_newer = true;
    device_newer = false;
    params_dirty = true;
}

double *Microenvironment::density_vector(int n) {
    sync_to_host();
    host_newer = true;  // the caller may write through the pointer
    return &field_[(size_t)n * number_of_densities()];
}

double *Microenvironment::density_vector(int i, int j, int k) { return density_vector(voxel_index(i, j, k)); }

double *Microenvironment::nearest_density_vector(std::vector<double> &position) {
    return density_vector(mesh.nearest_voxel_index(position));
}

void Microenvironment::add_dirichlet_node(int voxel_index, std::vector<double> &value) {
    const int S = number_of_densities();
    for (size_t i = 0; i < value.size() && (int)i < S; ++i)
        dirichlet_value_vectors[(size_t)voxel_index * S + i] = value[i];
    params_dirty = true;
}

void Microenvironment::add_dirichlet_node(int x, int y, int z, std::vector<double> &value) {
    add_dirichlet_node(voxel_index(x, y, z), value);
}

void Microenvironment::set_substrate_dirichlet_value(int d, double v) {
    if (d < 0 || d >= number_of_densities()) {
        std::cout << "BioFVM Warning: Invalid substrate index " << d << " for Dirichlet value assignment." << std::endl;
        return;
    }
    const int S = number_of_densities();
    const size_t expected = (size_t)number_of_voxels() * S;
    if (dirichlet_value_vectors.size() != expected) dirichlet_value_vectors.resize(expected, 1.0);
    for (int n = 0; n < number_of_voxels(); ++n) dirichlet_value_vectors[(size_t)n * S + d] = v;
    params_dirty = true;
}

void Microenvironment::set_substrate_dirichlet_value(const std::string &nm, double v) {
    const int d = find_density_index(nm);
    if (d < 0) {
        std::cout << "BioFVM Warning: Invalid substrate name " << nm << " for Dirichlet value assignment." << std::endl;
        return;
    }
    set_substrate_dirichlet_value(d, v);
}

void Microenvironment::set_substrate_dirichlet_activation(int d, bool on) {
    dirichlet_activation_vector[d] = on;
    params_dirty = true;
}

double *Microenvironment::dirichlet_values(int i, int j, int k) {
    params_dirty = true;
    return &dirichlet_value_vectors[(size_t)voxel_index(i, j, k) * number_of_densities()];
}

void Microenvironment::set_dirichlet_face_mask(const std::vector<uint8_t> &mask) {
    face_mask_ = mask;
    params_dirty = true;
}

void Microenvironment::set_precision(Precision p) {
    if (p == precision_) return;
    sync_to_host();
    precision_ = p;
    if (env_) {
        bfb_destroy(env_);
        env_ = nullptr;
    }
    host_newer = true;
    params_dirty = true;
}

int Microenvironment::ensure_device() {
    if (env_) return BFB_OK;
    if (!mesh.uniform_mesh) {
        std::cout << "BioFVM-B200: the device grid needs a uniform mesh (dx = dy = dz)" << std::endl;
        return BFB_ERR_UNSUPPORTED;
    }
    const double *bb = mesh.bounding_box;
    int st = bfb_create_domain(&env_, bb[0], bb[3], bb[1], bb[4], bb[2], bb[5], mesh.dx, number_of_densities(),
                               (int)precision_, 0);
    if (st) {
        env_ = nullptr;
        return st;
    }
    host_newer = true;
    params_dirty = true;
    bulk_dirty = true;
    agents_dirty_ = true;
    D_uploaded_.clear();
    return BFB_OK;
}

bfb_env Microenvironment::device_env() {
    report(ensure_device(), "device_env");
    return env_;
}

int Microenvironment::upload_all_if_needed() {
    int st = ensure_device();
    if (st) return st;
    if (params_dirty) {
        // The reference computes its Thomas factors on the first solver call
        // and never again (BioFVM_parallel.cpp:714, 913): D and lambda are
        // sent once, before the first step.
        if (D_uploaded_.empty()) {
            st = bfb_set_coefficients(env_, diffusion_coefficients.data(), decay_rates.data());
            if (st) return st;
            D_uploaded_ = diffusion_coefficients;
            lambda_uploaded_ = decay_rates;
        }
        const int S = number_of_densities();
        std::vector<uint8_t> act(S);
        for (int d = 0; d < S; ++d) act[d] = dirichlet_activation_vector[d] ? 1 : 0;
        st = bfb_set_dirichlet(env_, dirichlet_value_vectors.data(), act.data(),
                               face_mask_.empty() ? nullptr : face_mask_.data());
        if (st) return st;
        params_dirty = false;
    }
    if (host_newer || host_sync == HostSync::EveryStep) {
        st = bfb_set_field(env_, field_.data());
        if (st) return st;
        host_newer = false;
        device_newer = false;
    }
    return BFB_OK;
}

void Microenvironment::after_device_step() {
    device_newer = true;
    if (host_sync == HostSync::EveryStep) sync_to_host();
}

void Microenvironment::sync_to_host() {
    if (!env_ || !device_newer) return;
    report(bfb_get_field(env_, field_.data()), "sync_to_host");
    device_newer = false;
}

void Microenvironment::sync_to_device() {
    report(upload_all_if_needed(), "sync_to_device");
}

// compute_all_gradient_vectors (BioFVM_microenvironment.cpp:1243-1402): all
// voxels at once on the device; the per-voxel compute_gradient_vector
// (:1404-1535) gives the same values on the uniform mesh, so a request for
// one voxel also fills every voxel.
void Microenvironment::compute_all_gradient_vectors() {
    const int V = number_of_voxels(), S = number_of_densities();
    std::vector<double> flat(3 * (size_t)V * S);
    int st = upload_all_if_needed();
    if (!st) st = bfb_get_gradients(env_, flat.data());
    report(st, "compute_all_gradient_vectors");
    if (st) return;
    gradient_vectors_.assign(V, std::vector<gradient>(S, gradient(3, 0.0)));
    for (int n = 0; n < V; ++n)
        for (int q = 0; q < S; ++q)
            for (int c = 0; c < 3; ++c) gradient_vectors_[n][q][c] = flat[((size_t)n * S + q) * 3 + c];
    gradients_valid_ = true;
}

// reset_all_gradient_vectors (BioFVM_microenvironment.cpp:1543-1553): marks
// every voxel not computed, so the next access computes again. As in the
// reference, a later step alone does not invalidate stored gradients.
void Microenvironment::reset_all_gradient_vectors() {
    gradient_vectors_.assign(number_of_voxels(), std::vector<gradient>(number_of_densities(), gradient(3, 0.0)));
    gradients_valid_ = false;
}

std::vector<Microenvironment::gradient> &Microenvironment::gradient_vector(int n) {
    if (!gradients_valid_) compute_all_gradient_vectors();
    if (gradient_vectors_.empty()) reset_all_gradient_vectors();  // a failed computation still returns storage
    return gradient_vectors_[n];
}

void Microenvironment::write_to_matlab(std::string filename) {
    int st = upload_all_if_needed();
    if (!st) st = bfb_write_matlab(env_, filename.c_str());
    report(st, "write_to_matlab");
}

std::vector<double> Microenvironment::checksum() {
    std::vector<double> out(number_of_densities(), 0.0);
    int st = upload_all_if_needed();
    if (!st) st = bfb_checksum(env_, out.data());
    report(st, "checksum");
    return out;
}

void Microenvironment::print_result(double dt, int mpi_Size, int mpi_Rank, int *mpi_Coords, std::string *file_name,
                                    int *mpi_Dims, MPI_Comm comm) {
    if (print_voxels_densities) print_voxels_densities(*this, dt, mpi_Size, mpi_Rank, mpi_Coords, file_name, mpi_Dims, comm);
}

void print_voxels_densities(Microenvironment &M, double dt, int size, int rank, int *coords, std::string *file_name,
                            int *dims, MPI_Comm comm) {
    (void)dt;
    (void)coords;
    (void)dims;
    (void)comm;
    if (size != 1) std::cout << "BioFVM-B200: one grid per process; the densities are written once" << std::endl;
    M.sync_to_host();
    const std::vector<double> &f = *M.p_density_vectors;
    const int S = M.number_of_densities();
    std::ofstream out(*file_name, std::ios::app);
    size_t index = 0;
    for (int i = 0; i < M.mesh.x_size; i++)
        for (int j = 0; j < M.mesh.y_size; j++)
            for (int k = 0; k < M.mesh.z_size; k++) {
                out << (M.mesh.x_coordinates.size() * rank) + i << " " << j << " " << k << " : ";
                for (int d = 0; d < S; ++d) out << f[index++] << " ";
                out << std::endl;
            }
    out << std::flush;
}

bool Microenvironment::compare_microenvironment(Microenvironment &reference) {
    if (mesh.x_coordinates.size() != reference.mesh.x_coordinates.size() ||
        mesh.y_coordinates.size() != reference.mesh.y_coordinates.size() ||
        mesh.z_coordinates.size() != reference.mesh.z_coordinates.size())
        return false;
    if (number_of_densities() != reference.number_of_densities()) return false;
    sync_to_host();
    reference.sync_to_host();
    for (size_t n = 0; n < field_.size(); ++n)
        if (field_[n] != reference.field_[n]) return false;
    return true;
}

void Microenvironment::apply_dirichlet_conditions(int rank, int size) {
    (void)rank;
    (void)size;
    int st = upload_all_if_needed();
    if (!st) st = bfb_apply_dirichlet(env_);
    report(st, "apply_dirichlet_conditions");
    if (!st) after_device_step();
}

void Microenvironment::simulate_diffusion_decay(double dt, int mpi_Size, int mpi_Rank, int *mpi_Coords, int *mpi_Dims,
                                                MPI_Comm comm) {
    // BioFVM_microenvironment.cpp:1018-1029
    if (diffusion_decay_solver) {
        diffusion_decay_solver(*this, dt, mpi_Size, mpi_Rank, mpi_Coords, mpi_Dims, comm);
    } else {
        std::cout << "Warning: diffusion-reaction-source/sink solver not set for Microenvironment object at " << this
                  << ". Nothing happened!" << std::endl;
    }
}

void diffusion_decay_solver__constant_coefficients_LOD_3D_B200(Microenvironment &M, double dt, int mpi_Size,
                                                                int mpi_Rank, int *, int *, MPI_Comm) {
    (void)mpi_Rank;
    if (mpi_Size != 1) {
        std::cout << "Error: the B200 solver runs one device-resident grid per process (mpi_Size must be 1)"
                  << std::endl;
        return;
    }
    if (!M.mesh.uniform_mesh || !M.mesh.Cartesian_mesh) {
        std::cout << "Error: This algorithm is written for uniform Cartesian meshes. Try: other solvers!" << std::endl
                  << std::endl;
        return;
    }
    int st = M.upload_all_if_needed();
    if (!st) st = bfb_simulate(M.device_env(), dt, 1, BFB_STEP_DIFFUSION);
    M.report(st, "diffusion_decay_solver__constant_coefficients_LOD_3D_B200");
    if (!st) M.after_device_step();
}

void Microenvironment::simulate_bulk_sources_and_sinks(double dt) {
    // BioFVM_microenvironment.cpp:1110-1153. With the default zero callbacks
    // the update is the identity (rho + dt*0)/(0*dt + 1) == rho exactly.
    if (bulk_supply_rate_function == zero_function && bulk_supply_target_densities_function == zero_function &&
        bulk_uptake_rate_function == zero_function)
        return;
    const int S = number_of_densities(), V = number_of_voxels();
    const bool same_fns = bulk_fns_used_[0] == bulk_supply_rate_function &&
                          bulk_fns_used_[1] == bulk_supply_target_densities_function &&
                          bulk_fns_used_[2] == bulk_uptake_rate_function;
    const bool tabulate = bulk_tabulation_ == BulkTabulation::EveryCall || bulk_dirty || !same_fns;
    int st = upload_all_if_needed();
    if (tabulate) {
        bulk_S_.assign((size_t)V * S, 0.0);
        bulk_T_.assign((size_t)V * S, 0.0);
        bulk_U_.assign((size_t)V * S, 0.0);
        for (int n = 0; n < V; ++n) {
            bulk_supply_rate_function(this, n, &bulk_S_[(size_t)n * S]);
            bulk_supply_target_densities_function(this, n, &bulk_T_[(size_t)n * S]);
            bulk_uptake_rate_function(this, n, &bulk_U_[(size_t)n * S]);
        }
        if (!st) st = bfb_set_bulk(env_, bulk_S_.data(), bulk_T_.data(), bulk_U_.data());
        if (!st) {
            bulk_dirty = false;
            bulk_fns_used_[0] = bulk_supply_rate_function;
            bulk_fns_used_[1] = bulk_supply_target_densities_function;
            bulk_fns_used_[2] = bulk_uptake_rate_function;
        }
    }
    if (!st) st = bfb_bulk_step(env_, dt);
    report(st, "simulate_bulk_sources_and_sinks");
    if (!st) after_device_step();
}

void Microenvironment::simulate_cell_sources_and_sinks(std::vector<Basic_Agent *> &list, double dt) {
    // BioFVM_microenvironment.cpp:1155-1164 + BioFVM_basic_agent.cpp:279-300.
    // The cached constants are refreshed where volume_is_changed, as the
    // reference does inside simulate_secretion_and_uptake; agents of other
    // microenvironments are skipped.
    const int S = number_of_densities();
    std::vector<int> vox;
    std::vector<double> t1, t2;
    std::vector<uint8_t> act;
    vox.reserve(list.size());
    for (Basic_Agent *a : list) {
        if (a->microenvironment != this) continue;
        if (a->is_active && a->volume_is_changed) a->set_internal_uptake_constants(dt);
        vox.push_back(a->current_voxel_index);
        act.push_back(a->is_active ? 1 : 0);
        for (int d = 0; d < S; ++d) {
            t1.push_back(a->cell_source_sink_solver_temp1[d]);
            t2.push_back(a->cell_source_sink_solver_temp2[d]);
        }
    }
    int st = upload_all_if_needed();
    if (!st)
        st = bfb_set_agent_constants(env_, (int)vox.size(), vox.data(), t1.data(), t2.data(), act.data());
    if (!st) st = bfb_cells_step(env_, dt);
    report(st, "simulate_cell_sources_and_sinks");
    if (!st) after_device_step();
}

void Microenvironment::simulate_cell_sources_and_sinks(double dt) { simulate_cell_sources_and_sinks(all_basic_agents, dt); }

void Microenvironment::display_information(std::ostream &os) {
    os << std::endl << "Microenvironment summary: " << name << ": " << std::endl;
    os << "Mesh: " << mesh.x_size << " x " << mesh.y_size << " x " << mesh.z_size << " voxels of " << mesh.dx << " "
       << spatial_units << " (B200 device-resident, " << (precision_ == Precision::FP64 ? "FP64" : "FP32") << ")"
       << std::endl;
    os << "Densities: (" << number_of_densities() << " total)" << std::endl;
    for (int i = 0; i < number_of_densities(); ++i) {
        os << "   " << density_names[i] << ":" << std::endl
           << "     units: " << density_units[i] << std::endl
           << "     diffusion coefficient: " << diffusion_coefficients[i] << " " << spatial_units << "^2 / "
           << time_units << std::endl
           << "     decay rate: " << decay_rates[i] << " " << time_units << "^-1" << std::endl
           << "     diffusion length scale: " << std::sqrt(diffusion_coefficients[i] / (1e-12 + decay_rates[i]))
           << " " << spatial_units << std::endl
           << std::endl;
    }
}

// ---------------------------------------------------------------------------
// Basic_Agent (BioFVM_basic_agent.cpp)
// ---------------------------------------------------------------------------
Basic_Agent::Basic_Agent() {
    static int max_id = 0;
    ID = max_id++;
    position.assign(3, 0.0);
    secretion_rates = new std::vector<double>();
    uptake_rates = new std::vector<double>();
    saturation_densities = new std::vector<double>();
    if (g_default) register_microenvironment(g_default);
}

Basic_Agent::~Basic_Agent() {
    delete secretion_rates;
    delete uptake_rates;
    delete saturation_densities;
}

void Basic_Agent::set_total_volume(double v) {
    volume = v;
    volume_is_changed = true;
}

void Basic_Agent::register_microenvironment(Microenvironment *m) {
    // BioFVM_basic_agent.cpp:178-191
    microenvironment = m;
    const int S = m->number_of_densities();
    secretion_rates->resize(S, 0.0);
    saturation_densities->resize(S, 0.0);
    uptake_rates->resize(S, 0.0);
    cell_source_sink_solver_temp1.resize(S, 0.0);
    cell_source_sink_solver_temp2.resize(S, 1.0);
}

bool Basic_Agent::assign_position(std::vector<double> p, int mpi_Rank, int *mpi_Dims) {
    return assign_position(p[0], p[1], p[2], mpi_Rank, mpi_Dims);
}

bool Basic_Agent::assign_position(double x, double y, double z, int mpi_Rank, int *mpi_Dims) {
    // BioFVM_basic_agent.cpp:112-128: a rejected position changes nothing
    if (!microenvironment->mesh.is_position_valid(x, y, z)) return false;
    position[0] = x;
    position[1] = y;
    position[2] = z;
    update_voxel_index(mpi_Rank, mpi_Dims);
    return true;
}

void Basic_Agent::update_voxel_index(int, int *) {
    // BioFVM_basic_agent.cpp:137-153
    const Cartesian_Mesh &m = microenvironment->mesh;
    if (!m.is_position_valid(position[0], position[1], position[2])) {
        current_voxel_index = -1;
        is_active = false;
        return;
    }
    int aux = m.nearest_voxel_index(position);
    const int V = microenvironment->number_of_voxels();
    if (aux < 0) aux = 0;
    if (aux >= V) aux = V - 1;
    current_voxel_index = aux;
}

void Basic_Agent::set_internal_uptake_constants(double dt) {
    // BioFVM_basic_agent.cpp:155-176 with the reference build's fused axpy
    const double c = dt * volume / microenvironment->mesh.dV;
    const size_t S = secretion_rates->size();
    cell_source_sink_solver_temp1.assign(S, 0.0);
    cell_source_sink_solver_temp2.assign(S, 1.0);
    for (size_t d = 0; d < S; ++d) {
        double t1 = 0.0;
        t1 += (*secretion_rates)[d];
        t1 *= (*saturation_densities)[d];
        t1 *= c;
        cell_source_sink_solver_temp1[d] = t1;
        double t2 = 1.0;
        t2 = std::fma(c, (*secretion_rates)[d], t2);
        t2 = std::fma(c, (*uptake_rates)[d], t2);
        cell_source_sink_solver_temp2[d] = t2;
    }
    volume_is_changed = false;
}

double *Basic_Agent::nearest_density_vector() {
    return microenvironment ? microenvironment->nearest_density_vector(current_voxel_index) : nullptr;
}

std::vector<double> &Basic_Agent::nearest_gradient(int substrate_index) {
    return microenvironment->gradient_vector(current_voxel_index)[substrate_index];
}

std::vector<std::vector<double>> &Basic_Agent::nearest_gradient_vector() {
    return microenvironment->gradient_vector(current_voxel_index);
}

void Basic_Agent::simulate_secretion_and_uptake(Microenvironment *M, double dt) {
    if (!is_active) return;
    if (volume_is_changed) set_internal_uptake_constants(dt);
    double *rho = M->density_vector(current_voxel_index);
    const int S = M->number_of_densities();
    for (int d = 0; d < S; ++d) rho[d] += cell_source_sink_solver_temp1[d];
    for (int d = 0; d < S; ++d) rho[d] /= cell_source_sink_solver_temp2[d];
}

Basic_Agent *create_basic_agent() {
    Basic_Agent *p = new Basic_Agent();
    all_basic_agents.push_back(p);
    p->index = (int)all_basic_agents.size() - 1;
    return p;
}

void delete_basic_agent(int index) {
    // BioFVM_basic_agent.cpp:210-231: move the last agent into the hole
    delete all_basic_agents[index];
    if (index == (int)all_basic_agents.size() - 1) {
        all_basic_agents.pop_back();
        return;
    }
    all_basic_agents[all_basic_agents.size() - 1]->index = index;
    all_basic_agents[index] = all_basic_agents[all_basic_agents.size() - 1];
    all_basic_agents.pop_back();
}

void delete_basic_agent(Basic_Agent *p) { delete_basic_agent(p->index); }

}  // namespace BioFVM_B200
