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
// solver would have produced. The vector's storage is page-locked
// (bfb_host_register) on the first call, so both copies run at the host
// link's pinned-memory speed.
//
// State per Microenvironment:
//   * the device grid, created on the first call, where the reference computes
//     its Thomas factors (BioFVM_parallel.cpp:714); the factors stay at the
//     first call's dt, D and lambda, as the reference's do (:714, 913). A grid
//     whose mesh size or substrate count no longer matches the
//     Microenvironment (after resize_space or add_density) is replaced;
//   * the Dirichlet state last sent to the device. The reference applies the
//     activation flags and the outer-face entries of dirichlet_value_vectors on
//     every call (BioFVM_microenvironment.cpp:381-484); they are compared with
//     what the device holds and sent again only when one has changed.
// Errors are printed, as the reference prints its own (BioFVM_parallel.cpp:
// 705-710), and leave the field unchanged.
#include <cstdint>
#include <cstring>
#include <iostream>
#include <map>
#include <vector>

#include "BioFVM_microenvironment.h"
#include "biofvm_b200.h"

namespace BioFVM {

namespace {

struct B200State {
    bfb_env env = nullptr;
    void *pinned = nullptr;            // the field storage page-locked for this Microenvironment
    std::vector<uint8_t> activation;   // Dirichlet activation last sent to the device
    std::vector<double> face_values;   // outer-face entries of dirichlet_value_vectors last sent
    bool dirichlet_sent = false;
};

std::map<Microenvironment *, B200State> g_b200;

void b200_report(const char *what) { std::cout << "B200 solver: " << what << ": " << bfb_last_error() << std::endl; }

void release_state(B200State &st) {
    if (st.pinned) bfb_host_unregister(st.pinned);
    if (st.env) bfb_destroy(st.env);
    st = B200State();
}

// The outer-face entries of the per-voxel Dirichlet values, in a fixed order
// (the faces x = 0, x = nx-1, y = 0, y = ny-1, z = 0, z = nz-1; edges repeat).
void face_entries(const std::vector<double> &v, int nx, int ny, int nz, int S, std::vector<double> &out) {
    out.clear();
    auto put = [&](int i, int j, int k) {
        const size_t b = (((size_t)i * ny + j) * nz + k) * S;
        out.insert(out.end(), v.begin() + b, v.begin() + b + S);
    };
    for (int i : {0, nx - 1})
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) put(i, j, k);
    for (int j : {0, ny - 1})
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nz; ++k) put(i, j, k);
    for (int k : {0, nz - 1})
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) put(i, j, k);
}

// Whether the outer-face entries of v differ, bit for bit, from `cached`
// (laid out as face_entries lays them out); compared in place, block by block.
bool faces_changed(const std::vector<double> &v, int nx, int ny, int nz, int S, const std::vector<double> &cached) {
    const size_t want = 2 * ((size_t)ny * nz + (size_t)nx * nz + (size_t)nx * ny) * S;
    if (cached.size() != want) return true;
    const double *c = cached.data();
    auto differs = [&](size_t at, size_t count) {
        const bool d = std::memcmp(v.data() + at, c, count * sizeof(double)) != 0;
        c += count;
        return d;
    };
    const size_t row = (size_t)nz * S;
    for (int i : {0, nx - 1})
        if (differs((size_t)i * ny * row, (size_t)ny * row)) return true;
    for (int j : {0, ny - 1})
        for (int i = 0; i < nx; ++i)
            if (differs(((size_t)i * ny + j) * row, row)) return true;
    for (int k : {0, nz - 1})
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                if (differs(((size_t)i * ny + j) * row + (size_t)k * S, S)) return true;
    return false;
}

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
    const int nx = M.mesh.x_size, ny = M.mesh.y_size, nz = M.mesh.z_size;
    std::vector<double> &field = *M.p_density_vectors;
    if (field.size() != (size_t)nx * ny * nz * S) {
        std::cout << "B200 solver: the density vector does not hold mesh voxels x substrates values" << std::endl;
        return;
    }
    B200State &st = g_b200[&M];
    if (st.env) {  // a grid of another size or substrate count is replaced
        int gx = 0, gy = 0, gz = 0, gs = 0;
        bfb_get_shape(st.env, &gx, &gy, &gz, &gs);
        if (gx != nx || gy != ny || gz != nz || gs != S) release_state(st);
    }
    if (!st.env) {
        if (bfb_create(&st.env, nx, ny, nz, S, M.mesh.dx, BFB_FP64, 0) != BFB_OK) {
            b200_report("bfb_create");
            st.env = nullptr;
            return;
        }
        if (bfb_set_coefficients(st.env, M.diffusion_coefficients.data(), M.decay_rates.data()) != BFB_OK) {
            b200_report("bfb_set_coefficients");
            release_state(st);
            return;
        }
    }
    if (st.pinned != field.data()) {  // the vector's storage moved: page-lock the new one
        if (st.pinned) bfb_host_unregister(st.pinned);
        st.pinned = nullptr;
        if (bfb_host_register(field.data(), field.size() * sizeof(double)) == BFB_OK) st.pinned = field.data();
        // not fatal: unregistered memory is copied at pageable speed
    }
    std::vector<uint8_t> activation(S);
    bool any = false;
    for (int d = 0; d < S; ++d) {
        activation[d] = M.dirichlet_activation_vector[d] ? 1 : 0;
        any = any || activation[d];
    }
    // the face values matter only where a substrate is active
    const bool changed = !st.dirichlet_sent || activation != st.activation ||
                         (any && faces_changed(M.dirichlet_value_vectors, nx, ny, nz, S, st.face_values));
    if (changed) {
        std::vector<double> faces;
        if (any) face_entries(M.dirichlet_value_vectors, nx, ny, nz, S, faces);
        // all six faces follow the activation, the reference's rule (BioFVM_microenvironment.cpp:381-484)
        if (bfb_set_dirichlet(st.env, any ? M.dirichlet_value_vectors.data() : nullptr, activation.data(), nullptr) !=
            BFB_OK) {
            b200_report("bfb_set_dirichlet");
            st.dirichlet_sent = false;
            return;
        }
        st.activation = activation;
        st.face_values.swap(faces);
        st.dirichlet_sent = true;
    }
    if (bfb_step_host(st.env, field.data(), dt, 1) != BFB_OK) b200_report("bfb_step_host");
}

// Frees the device grid held for M and unpins its field storage; call it
// before M is destroyed if M's address may be reused by another
// Microenvironment, and before M's density vectors are reallocated by a call
// that does not step (the solver itself notices a reallocation on its next
// call).
void release_b200_solver(Microenvironment &M) {
    auto it = g_b200.find(&M);
    if (it == g_b200.end()) return;
    release_state(it->second);
    g_b200.erase(it);
}

}  // namespace BioFVM
