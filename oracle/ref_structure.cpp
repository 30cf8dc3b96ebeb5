/* Reference structure discretisation for the oracle — TEST INFRASTRUCTURE ONLY.
 *
 * Builds the reference's own Structure object (src/structure/structure.cpp,
 * compiled unmodified from the reference tree) without its Lua host: the
 * operations a structure script would add are created directly with the
 * constructors that the script functions call (lua_structure.cpp:292-548,
 * with their argument conversions: Degree() for coating angles, x1+dx end
 * points already applied by the caller for cylinders and cones), then
 * Structure::finalize's closing loop (structure.cpp:215-220) links and
 * precomputes them, and Structure::discretize (structure.cpp:94-113) tags the
 * grid. The nominal lengths, which a script sets as Lua globals, are written
 * into the object directly. A mesh is written to a temporary OBJ file with
 * round-trip precision and read back by Add_Mesh's own loader. */
#include <lua_base.h>
#include <mesh_base.h>
#include <octree.h>
#include <Eigen/Eigen>

#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <string>
#include <unistd.h>
#include <vector>

#define private public
#include <structure.h>
#undef private
#include <phys_tools.h>

#include "../include/aefdtd.h"

extern "C" int aeref_discretize(int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                                const aefdtd_structure_op *ops, int32_t n_ops, const aefdtd_structure_desc *d,
                                uint32_t *out) {
    if (nx < 1 || ny < 1 || nz < 1 || n_ops < 0 || !d || !out) return 1;
    Structure S;
    S.set_default_material(d->default_material);
    S.set_loop(d->periodic[0], d->periodic[1], d->periodic[2]);
    S.set_flip(d->flip[0], d->flip[1], d->flip[2]);
    S.lx = d->lengths[0];
    S.ly = d->lengths[1];
    S.lz = d->lengths[2];
    std::vector<Structure_OP *> made;
    for (int q = 0; q < n_ops; q++) {
        const double *p = ops[q].p;
        const int m = ops[q].mat_index;
        Structure_OP *o = nullptr;
        switch (ops[q].kind) {
            case AEFDTD_OP_BLOCK: o = new Add_Block(p[0], p[1], p[2], p[3], p[4], p[5], m); break;
            case AEFDTD_OP_LAYER: o = new Add_Layer(int(p[0]), p[1], p[2], m); break;
            case AEFDTD_OP_SPHERE: o = new Add_Sphere(p[0], p[1], p[2], p[3], m); break;
            case AEFDTD_OP_CYLINDER: o = new Add_Cylinder(p[0], p[1], p[2], p[3], p[4], p[5], p[6], m); break;
            case AEFDTD_OP_CONE: o = new Add_Cone(p[0], p[1], p[2], p[3], p[4], p[5], p[6], m); break;
            case AEFDTD_OP_ELLIPSOID: o = new Add_Ellipsoid(p[0], p[1], p[2], p[3], p[4], p[5], m); break;
            case AEFDTD_OP_SIN_LAYER:
                o = new Add_Sin_Layer(p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], m);
                break;
            case AEFDTD_OP_VECT_BLOCK:
                o = new Add_Vect_Block(p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], p[9], p[10], p[11], m);
                break;
            case AEFDTD_OP_VECT_TRI:
                o = new Add_Vect_Tri(p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], p[9], p[10], p[11], p[12],
                                     m);
                break;
            case AEFDTD_OP_COATING:
                o = new Add_Coating(Degree(p[0]), Degree(p[1]), p[2], p[3], int(p[4]), m);
                break;
            case AEFDTD_OP_CONF_COATING: o = new Add_Conf_Coating(p[0], p[1], int(p[2]), m); break;
            case AEFDTD_OP_MESH: {
                const int mi = int(p[4]);
                if (mi < 0 || mi >= d->n_meshes) {
                    for (Structure_OP *x : made) delete x;
                    return 3;
                }
                const aefdtd_mesh &mesh = d->meshes[mi];
                char path[] = "/tmp/aeref_meshXXXXXX";
                const int fd = mkstemp(path);
                if (fd < 0) {
                    for (Structure_OP *x : made) delete x;
                    return 4;
                }
                FILE *f = fdopen(fd, "w");
                for (int v = 0; v < mesh.n_vertices; v++)
                    std::fprintf(f, "v %.17g %.17g %.17g\n", mesh.vertices[3 * v], mesh.vertices[3 * v + 1],
                                 mesh.vertices[3 * v + 2]);
                for (int t = 0; t < mesh.n_faces; t++)
                    std::fprintf(f, "f %d %d %d\n", mesh.faces[3 * t] + 1, mesh.faces[3 * t + 1] + 1, mesh.faces[3 * t + 2] + 1);
                std::fclose(f);
                o = new Add_Mesh(p[0], p[1], p[2], p[3], std::filesystem::path(path), m);
                std::remove(path);
                break;
            }
            default:
                for (Structure_OP *x : made) delete x;
                return 2;
        }
        made.push_back(o);
        S.add_operation(o);
    }
    for (std::size_t i = 0; i < S.operations.size(); i++) {
        S.operations[i]->parent = &S;
        S.operations[i]->stack_ID = int(i);
        S.operations[i]->precompute();
    }
    Grid3<unsigned int> g;
    S.discretize(g, nx, ny, nz, dx, dy, dz);
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) out[i + std::size_t(j) * nx + std::size_t(k) * nx * ny] = g(i, j, k);
    S.operations.clear();
    for (Structure_OP *x : made) delete x;
    return 0;
}

// The structure scripts' random_packing helper (phys_tools.cpp:302-426),
// called as the Lua binding does (lua_structure.cpp, random_packing).
extern "C" int aeref_random_packing(double x_max, double y_max, double r, int32_t n_part, int32_t seed, double *x,
                                    double *y) {
    if (n_part < 1 || !x || !y) return 1;
    std::vector<SeedParticle> particles(n_part);
    random_packing(particles, x_max, y_max, r, n_part, seed);
    for (int i = 0; i < n_part; i++) {
        x[i] = particles[i].x;
        y[i] = particles[i].y;
    }
    return 0;
}
