// Host-only checks of the C++ facade; no device call is made, so it runs
// without a GPU. Covers the mesh resize overloads (node counts, centres,
// voxel volume, the uniform-mesh test of BioFVM_parallel.cpp:124-127),
// compare_microenvironment (BioFVM_microenvironment.cpp:1688-1726), the
// LOD solver's refusal of a non-uniform mesh and, given a file name, the
// text dump of print_result (BioFVM_parallel.cpp:2334-2366). Built and run by
// tests/test_facade_cpu.py; prints "ok" and exits 0 when every check holds.
#include <cstdio>
#include <string>
#include <vector>

#include "BioFVM_B200.h"

using namespace BioFVM_B200;

#define CHECK(c)                                                          \
    do {                                                                  \
        if (!(c)) {                                                       \
            std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);      \
            return 1;                                                     \
        }                                                                 \
    } while (0)

int main(int argc, char **argv) {
    Microenvironment a, b;
    a.set_density(0, "oxygen", "mmHg", 1e5, 0.1);
    b.set_density(0, "oxygen", "mmHg", 1e5, 0.1);
    a.resize_space_uniform(0.0, 100.0, 0.0, 80.0, -20.0, 40.0, 20.0);
    b.resize_space(0.0, 100.0, 0.0, 80.0, -20.0, 40.0, 20.0, 20.0, 20.0);
    CHECK(a.mesh.x_size == 5 && a.mesh.y_size == 4 && a.mesh.z_size == 3);
    CHECK(b.mesh.x_size == 5 && b.mesh.y_size == 4 && b.mesh.z_size == 3);
    CHECK(a.mesh.uniform_mesh && b.mesh.uniform_mesh);
    CHECK(a.mesh.dV == b.mesh.dV && a.mesh.dV == 8000.0);
    CHECK(a.mesh.z_coordinates == b.mesh.z_coordinates && b.mesh.z_coordinates[0] == -10.0);
    CHECK(a.mesh.x_coordinates == b.mesh.x_coordinates && a.mesh.y_coordinates == b.mesh.y_coordinates);

    // equal fields compare equal; one differing density breaks it until matched
    CHECK(a.compare_microenvironment(b));
    a.density_vector(7)[0] = 1.5;
    CHECK(!a.compare_microenvironment(b));
    b.density_vector(7)[0] = 1.5;
    CHECK(a.compare_microenvironment(b) && b.compare_microenvironment(a));

    // another substrate count, or other node counts, never compare equal
    Microenvironment c;
    c.resize_space_uniform(0.0, 100.0, 0.0, 80.0, -20.0, 40.0, 20.0);
    c.add_density("glucose", "mM", 1e3, 0.01);
    CHECK(!a.compare_microenvironment(c));
    Microenvironment d;
    d.resize_space_uniform(0.0, 120.0, 0.0, 80.0, -20.0, 40.0, 20.0);
    CHECK(!a.compare_microenvironment(d));

    // non-uniform spacing: per-axis node counts and volume; the solver refuses
    Microenvironment e;
    e.resize_space(0.0, 100.0, 0.0, 80.0, 0.0, 60.0, 20.0, 10.0, 20.0);
    CHECK(e.mesh.x_size == 5 && e.mesh.y_size == 8 && e.mesh.z_size == 3);
    CHECK(!e.mesh.uniform_mesh);
    CHECK(e.mesh.dV == 4000.0 && e.mesh.y_coordinates[1] == 15.0);
    e.density_vector(0)[0] = 2.0;
    e.simulate_diffusion_decay(0.01);  // prints the reference's message, computes nothing
    CHECK(e.density_vector(0)[0] == 2.0);
    CHECK(e.last_status() == 0);

    // an agent's nearest densities are its voxel's (BioFVM_basic_agent.cpp:250-253)
    {
        Basic_Agent *ag = create_basic_agent();
        ag->register_microenvironment(&a);
        ag->assign_position(45.0, 30.0, 5.0);  // voxel (2, 1, 1) of a's 5 x 4 x 3 grid
        CHECK(ag->get_current_voxel_index() == a.voxel_index(2, 1, 1));
        CHECK(ag->nearest_density_vector() == a.density_vector(a.voxel_index(2, 1, 1)));
        delete_basic_agent(ag);
    }

    // print_result's text dump of a 3 x 4 x 5 x 2 field v[n][d] = n * 0.1 + d / 7.0, appended to argv[1]
    if (argc > 1) {
        Microenvironment f;
        f.set_density(0, "a", "u", 1e3, 0.1);
        f.add_density("b", "u", 1e4, 0.2);
        f.resize_space_uniform(0.0, 60.0, 0.0, 80.0, 0.0, 100.0, 20.0);
        CHECK(f.number_of_voxels() == 60 && f.number_of_densities() == 2);
        for (int n = 0; n < 60; ++n)
            for (int d = 0; d < 2; ++d) f.density_vector(n)[d] = n * 0.1 + d / 7.0;
        std::string name(argv[1]);
        int coords[3] = {0, 0, 0}, dims[3] = {1, 1, 1};
        f.print_result(0.01, 1, 0, coords, &name, dims, 0);
    }

    std::printf("ok\n");
    return 0;
}
