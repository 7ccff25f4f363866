// Host-only checks of the C++ facade; no device call is made, so it runs
// without a GPU. Covers the mesh resize overloads (node counts, centres,
// voxel volume, the uniform-mesh test of BioFVM_parallel.cpp:124-127),
// compare_microenvironment (BioFVM_microenvironment.cpp:1688-1726) and the
// LOD solver's refusal of a non-uniform mesh. Built and run by
// tests/test_facade_cpu.py; prints "ok" and exits 0 when every check holds.
#include <cstdio>
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

int main() {
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

    std::printf("ok\n");
    return 0;
}
