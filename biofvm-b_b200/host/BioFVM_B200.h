/*
 * BioFVM_B200.h -- C++ host facade with the reference's Microenvironment /
 * Basic_Agent interface for the diffusion-decay path, running on the B200
 * C ABI (include/biofvm_b200.h).
 *
 * It mirrors the names, argument meanings and defaults of
 *   BioFVM_microenvironment.h:66-292   (class Microenvironment)
 *   BioFVM_basic_agent.h:60-131        (class Basic_Agent, all_basic_agents)
 * for the members the hot path uses, so a driver written against the
 * reference (examples/test_VS.cpp, examples/complete_diffusion_demo.cpp)
 * compiles against this header with `using namespace BioFVM_B200;` and the
 * solver registration
 *     M.diffusion_decay_solver = diffusion_decay_solver__constant_coefficients_LOD_3D_B200;
 *
 * The field lives on the GPU. The host copy (*p_density_vectors, the same
 * std::vector<double>* member the reference exposes) is kept coherent by the
 * host-sync policy:
 *   HostSync::EveryStep (default) -- every simulate_* call uploads the host
 *       field before and downloads it after, exactly the reference's
 *       semantics (the field is always valid on the host);
 *   HostSync::Lazy -- the field stays on the device between calls; the
 *       accessors (density_vector, operator(), nearest_density_vector) sync
 *       on demand, and code that reads or writes *p_density_vectors directly
 *       calls sync_to_host() / mark_host_modified() around it.
 * Errors: the reference prints and returns; this facade does the same and
 * also keeps the last status in last_status().
 */
#ifndef BIOFVM_B200_FACADE_H
#define BIOFVM_B200_FACADE_H

#include <cstdint>
#include <string>
#include <vector>

#include "biofvm_b200.h"

namespace BioFVM_B200 {

// The reference's solver prototype carries an MPI communicator; the B200
// path runs one device-resident grid per process, so it is an opaque int.
typedef int MPI_Comm;

class Microenvironment;
class Basic_Agent;

enum class HostSync { EveryStep, Lazy };
// When the bulk callbacks are evaluated: on every simulate_bulk_sources_and_sinks
// call, as the reference does (BioFVM_microenvironment.cpp:1110-1153), or once
// and then reused from device memory until the callbacks change or
// mark_bulk_modified() is called (sources that do not vary in time).
enum class BulkTabulation { EveryCall, Once };
enum class Precision { FP64 = BFB_FP64, FP32 = BFB_FP32 };

struct Voxel {
    double center[3];
    double volume;
};

// Mesh facts the path needs (BioFVM_mesh.h / Cartesian_Mesh::resize).
struct Cartesian_Mesh {
    int x_size = 1, y_size = 1, z_size = 1;
    double dx = 1, dy = 1, dz = 1, dV = 1;
    double bounding_box[6] = {-0.5, -0.5, -0.5, 0.5, 0.5, 0.5};  // x0,y0,z0,x1,y1,z1
    bool uniform_mesh = true;
    bool Cartesian_mesh = true;
    std::vector<double> x_coordinates, y_coordinates, z_coordinates;
    int voxel_index(int i, int j, int k) const { return ((i * y_size) + j) * z_size + k; }
    std::vector<int> cartesian_indices(int n) const;
    bool is_position_valid(double x, double y, double z) const;
    int nearest_voxel_index(const std::vector<double> &position) const;
    Voxel voxels(int n) const;
};

class Microenvironment {
   public:
    Microenvironment();
    ~Microenvironment();
    Microenvironment(const Microenvironment &) = delete;
    Microenvironment &operator=(const Microenvironment &) = delete;

    // ---- reference public members (BioFVM_microenvironment.h:133-167)
    std::vector<double> *p_density_vectors;
    std::string timing_csv;
    unsigned granurality = 1;  // accepted and ignored: one grid, no MPI blocks
    Cartesian_Mesh mesh;
    std::string spatial_units = "none", time_units = "none", name = "unnamed";
    std::vector<std::string> density_names, density_units;
    std::vector<double> diffusion_coefficients, decay_rates;
    void (*diffusion_decay_solver)(Microenvironment &, double, int, int, int *, int *, MPI_Comm);
    void (*bulk_supply_rate_function)(Microenvironment *, int, double *);
    void (*bulk_supply_target_densities_function)(Microenvironment *, int, double *);
    void (*bulk_uptake_rate_function)(Microenvironment *, int, double *);

    // ---- sizes and substrates (BioFVM_microenvironment.cpp:709-1015)
    int number_of_densities() const { return (int)density_names.size(); }
    int number_of_voxels() const { return mesh.x_size * mesh.y_size * mesh.z_size; }
    void add_density(const std::string &name, const std::string &units);
    void add_density(const std::string &name, const std::string &units, double D, double lambda);
    void set_density(int index, const std::string &name, const std::string &units);
    void set_density(int index, const std::string &name, const std::string &units, double D, double lambda);
    int find_density_index(const std::string &name) const;

    // resize_space_uniform(..., dims, coords) at one rank (BioFVM_parallel.cpp:18-59)
    void resize_space_uniform(double x0, double x1, double y0, double y1, double z0, double z1, double dx,
                              int *dims = nullptr, int *coords = nullptr);
    // resize_space(..., dx, dy, dz, dims, coords) at one rank (BioFVM_parallel.cpp:29-59, 71-160): node
    // counts per axis from its own spacing. Spacings that differ by more than 1e-16 make the mesh
    // non-uniform, as in the reference; the LOD solver then refuses to run (it prints the reference's
    // message) and no device operation is available for that mesh.
    void resize_space(double x0, double x1, double y0, double y1, double z0, double z1, double dx, double dy,
                      double dz, int *dims = nullptr, int *coords = nullptr);
    int voxel_index(int i, int j, int k) const { return mesh.voxel_index(i, j, k); }
    std::vector<int> cartesian_indices(int n) const { return mesh.cartesian_indices(n); }
    int nearest_voxel_index(std::vector<double> &position) const { return mesh.nearest_voxel_index(position); }

    // ---- field accessors (host; sync on demand)
    double *density_vector(int n);
    double *density_vector(int i, int j, int k);
    double *operator()(int n) { return density_vector(n); }
    double *operator()(int i, int j, int k) { return density_vector(i, j, k); }
    double *operator()(int i, int j) { return density_vector(i, j, 0); }
    double *nearest_density_vector(std::vector<double> &position);
    double *nearest_density_vector(int voxel_index) { return density_vector(voxel_index); }

    // ---- Dirichlet (BioFVM_microenvironment.cpp:226-484)
    void add_dirichlet_node(int voxel_index, std::vector<double> &value);
    void add_dirichlet_node(int x, int y, int z, std::vector<double> &value);
    void update_dirichlet_node(int x, int y, int z, std::vector<double> &value) { add_dirichlet_node(x, y, z, value); }
    void set_substrate_dirichlet_value(int substrate_index, double new_value);
    void set_substrate_dirichlet_value(const std::string &substrate_name, double new_value);
    void set_substrate_dirichlet_activation(int substrate_index, bool new_value);
    double *dirichlet_values(int i, int j, int k);
    void apply_dirichlet_conditions(int rank = 0, int size = 1);
    // the reference's second version (BioFVM_microenvironment.cpp:486-...) writes the same faces with
    // the same values; examples/dirichlet_test.cpp:273-274 checks the two agree
    void apply_dirichlet_conditions_v2(int rank = 0, int size = 1) { apply_dirichlet_conditions(rank, size); }
    // compare_microenvironment (BioFVM_microenvironment.cpp:1688-1726): the same node counts and
    // substrate count, and every density equal bit for bit. The reference takes its argument by value;
    // this facade's Microenvironment owns device state and is not copyable, so it takes a reference.
    bool compare_microenvironment(Microenvironment &reference);
    // B200 extension: per-face activation mask[face*S + d] (faces x-lo, x-hi,
    // y-lo, y-hi, z-lo, z-hi), ANDed with the per-substrate activation.
    void set_dirichlet_face_mask(const std::vector<uint8_t> &mask);

    // ---- gradients (BioFVM_microenvironment.cpp:1195-1554): computed on the
    // device, held on the host in the reference's nested layout
    typedef std::vector<double> gradient;
    void compute_all_gradient_vectors();
    void compute_gradient_vector(int n) { (void)n; compute_all_gradient_vectors(); }
    void reset_all_gradient_vectors();
    std::vector<gradient> &gradient_vector(int n);
    std::vector<gradient> &gradient_vector(int i, int j, int k) { return gradient_vector(voxel_index(i, j, k)); }
    std::vector<gradient> &gradient_vector(int i, int j) { return gradient_vector(voxel_index(i, j, 0)); }
    std::vector<gradient> &nearest_gradient_vector(std::vector<double> &position) {
        return gradient_vector(nearest_voxel_index(position));
    }

    // ---- the hot path
    void simulate_diffusion_decay(double dt, int mpi_Size = 1, int mpi_Rank = 0, int *mpi_Coords = nullptr,
                                  int *mpi_Dims = nullptr, MPI_Comm comm = 0);
    void simulate_bulk_sources_and_sinks(double dt);
    void simulate_cell_sources_and_sinks(std::vector<Basic_Agent *> &basic_agent_list, double dt);
    void simulate_cell_sources_and_sinks(double dt);

    void display_information(std::ostream &os);
    // MATLAB v4 snapshot (BioFVM_microenvironment.cpp:1079-1107), packed on the device
    void write_to_matlab(std::string filename);
    // print_result (BioFVM_microenvironment.cpp:375-379) calls the print_voxels_densities hook, which
    // drivers set to the free function below (examples/test_VS.cpp:241); here it is set by default.
    void (*print_voxels_densities)(Microenvironment &, double, int, int, int *, std::string *, int *, MPI_Comm);
    void print_result(double dt, int mpi_Size, int mpi_Rank, int *mpi_Coords, std::string *file_name,
                      int *mpi_Dims, MPI_Comm comm);
    void write_to_matlab(std::string filename, int rank, int size, MPI_Comm comm) {
        (void)rank;
        (void)size;
        (void)comm;
        write_to_matlab(filename);
    }

    // ---- B200 additions
    void set_precision(Precision p);  // before the first step
    void set_host_sync(HostSync p) { host_sync = p; }
    void set_bulk_tabulation(BulkTabulation p) { bulk_tabulation_ = p; }
    void mark_bulk_modified() { bulk_dirty = true; }
    void sync_to_host();
    void sync_to_device();
    void mark_host_modified() { host_newer = true; }
    bfb_env device_env();  // creates the device env if needed
    int last_status() const { return status; }
    std::vector<double> checksum();

    // internal, used by the solver and agents
    int ensure_device();
    int upload_all_if_needed();
    void after_device_step();
    int set_bulk_on_device();
    int set_agents_on_device(std::vector<Basic_Agent *> &list, double dt);
    void report(int st, const char *where);

   private:
    std::vector<double> field_;
    std::vector<double> dirichlet_value_vectors;   // V*S, like the reference
    std::vector<bool> dirichlet_activation_vector;  // S
    std::vector<uint8_t> face_mask_;                 // 6*S or empty (all faces)
    bfb_env env_ = nullptr;
    Precision precision_ = Precision::FP64;
    HostSync host_sync = HostSync::EveryStep;
    bool host_newer = true;     // host copy changed since the last upload
    bool device_newer = false;  // device copy changed since the last download
    bool params_dirty = true;   // D, lambda, Dirichlet need uploading
    bool bulk_dirty = true;
    BulkTabulation bulk_tabulation_ = BulkTabulation::EveryCall;
    void (*bulk_fns_used_[3])(Microenvironment *, int, double *) = {nullptr, nullptr, nullptr};
    std::vector<double> bulk_S_, bulk_T_, bulk_U_;
    const void *agents_uploaded_for_ = nullptr;
    size_t agents_uploaded_n_ = 0;
    bool agents_dirty_ = true;
    int status = BFB_OK;
    std::vector<double> D_uploaded_, lambda_uploaded_;
    std::vector<std::vector<gradient>> gradient_vectors_;  // [V][S] of 3
    bool gradients_valid_ = false;
    friend class Basic_Agent;
};

// The GPU solver to register in Microenvironment::diffusion_decay_solver.
void diffusion_decay_solver__constant_coefficients_LOD_3D_B200(Microenvironment &M, double dt, int mpi_Size,
                                                                int mpi_Rank, int *mpi_Coords, int *mpi_Dims,
                                                                MPI_Comm comm);

void zero_function(Microenvironment *pMicroenvironment, int voxel_index, double *write_destination);
void one_function(Microenvironment *pMicroenvironment, int voxel_index, double *write_destination);

// ---- Basic_Agent (BioFVM_basic_agent.h:60-131)
class Basic_Agent {
   public:
    Basic_Agent();
    ~Basic_Agent();
    std::vector<double> *secretion_rates;
    std::vector<double> *saturation_densities;
    std::vector<double> *uptake_rates;
    int ID = 0;
    int index = 0;
    int type = 0;
    std::vector<double> position;

    double get_total_volume() const { return volume; }
    void set_total_volume(double v);
    void register_microenvironment(Microenvironment *m);
    Microenvironment *get_microenvironment() { return microenvironment; }
    bool assign_position(double x, double y, double z, int mpi_Rank = 0, int *mpi_Dims = nullptr);
    bool assign_position(std::vector<double> p, int mpi_Rank = 0, int *mpi_Dims = nullptr);
    void update_voxel_index(int mpi_Rank = 0, int *mpi_Dims = nullptr);
    void set_internal_uptake_constants(double dt);
    // host, single agent; the GPU path is Microenvironment::simulate_cell_sources_and_sinks
    void simulate_secretion_and_uptake(Microenvironment *M, double dt);
    int get_current_voxel_index() const { return current_voxel_index; }
    bool active() const { return is_active; }
    // BioFVM_basic_agent.cpp:250-266: the densities / gradients at the agent's voxel of its
    // microenvironment (gradients as Microenvironment::gradient_vector gives them)
    double *nearest_density_vector();
    std::vector<double> &nearest_gradient(int substrate_index);
    std::vector<std::vector<double>> &nearest_gradient_vector();
    std::vector<double> velocity;
    void update_position(double dt) { (void)dt; }  // a stub in the reference too (BioFVM_basic_agent.cpp:92-94)

   private:
    Microenvironment *microenvironment = nullptr;
    double volume = 1.0;
    bool volume_is_changed = false;
    int current_voxel_index = 0;
    bool is_active = true;
    std::vector<double> cell_source_sink_solver_temp1, cell_source_sink_solver_temp2;
    friend class Microenvironment;
};

extern std::vector<Basic_Agent *> all_basic_agents;
Basic_Agent *create_basic_agent();
void delete_basic_agent(int index);
void delete_basic_agent(Basic_Agent *p);

Microenvironment *get_default_microenvironment();
void set_default_microenvironment(Microenvironment *M);

// print_voxels_densities (BioFVM_parallel.cpp:2334-2366) at one rank: appends one line per voxel,
// "i j k : d0 d1 ... ", in (i, j, k) order with default stream formatting, to *file_name.
void print_voxels_densities(Microenvironment &M, double dt, int size, int rank, int *coords, std::string *file_name,
                            int *dims, MPI_Comm comm);

}  // namespace BioFVM_B200

#endif
