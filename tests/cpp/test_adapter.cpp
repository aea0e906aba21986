// C++ caller of the adapter (include/plato_b200.hpp), written the way the reference's
// DerivativeTests.ElastostaticResidual3D / InternalElasticEnergy3D drive
// VectorFunction and PhysicsScalarFunction (unit_tests/DerivativeTests.cpp:257-634), plus a
// Problem::solution / criterionValue / criterionGradient sequence on a small cantilever,
// and Helmholtz::Problem / VectorFunction on the same mesh.
// Prints "key: values..." lines; tests/test_gpu_adapter.py compares them with the golds.
#include <cstdio>
#include <vector>

#include "plato_b200.hpp"

using namespace plato_b200;

static void print(const char* key, const std::vector<double>& v, size_t n) {
    std::printf("%s:", key);
    for (size_t i = 0; i < n && i < v.size(); ++i) std::printf(" %.17g", v[i]);
    std::printf("\n");
}

static plato_problem_desc cube_desc(std::vector<double>& coords, std::vector<int32_t>& conn) {
    int32_t nn = 0, nc = 0;
    check(plato_box_mesh_sizes(2, 2, 2, &nn, &nc), nullptr);
    coords.resize(3 * size_t(nn));
    conn.resize(4 * size_t(nc));
    check(plato_box_mesh_tet4(2, 2, 2, 1.0, 1.0, 1.0, coords.data(), conn.data()), nullptr);
    plato_problem_desc d{};
    d.mesh = {nn, nc, coords.data(), conn.data()};
    d.material = {1.0e6, 0.3};
    d.penalty = {1.0, 0.0};
    d.solver = {1e-10, 10000, PLATO_OPERATOR_ASSEMBLED, PLATO_PRECISION_FP64, 1, 30.0, 0};
    return d;
}

int main() {
    try {
        // ---- DerivativeTests-style evaluation on the 2x2x2 TET4 cube -------------------
        std::vector<double> coords;
        std::vector<int32_t> conn;
        auto model = std::make_shared<Model>(cube_desc(coords, conn));
        const int32_t N = model->numNodes();
        std::vector<double> uh(3 * size_t(N)), zh(N, 1.0);
        double disp = 0.0;
        for (auto& v : uh) v = (disp += 0.0001);
        ScalarVector u(uh), z(zh);

        Elliptic::VectorFunction vf(model);
        print("residual", vf.value(u, z).to_host(), 81);
        print("jacobian", vf.gradient_u(u, z)->entries.to_host(), 36);
        print("gradient_z", vf.gradient_z(u, z)->entries.to_host(), 12);

        Elliptic::PhysicsScalarFunction energy(model);
        std::printf("energy: %.17g\n", energy.value(u, z));
        print("energy_gradient_u", energy.gradient_u(u, z).to_host(), 21);
        print("energy_gradient_z", energy.gradient_z(u, z).to_host(), 27);

        // ---- Problem on a 6x3x3 cantilever -----------------------------------------------
        int32_t nn = 0, nc = 0;
        check(plato_box_mesh_sizes(6, 3, 3, &nn, &nc), nullptr);
        std::vector<double> c2(3 * size_t(nn));
        std::vector<int32_t> k2(4 * size_t(nc));
        check(plato_box_mesh_tet4(6, 3, 3, 2.0, 1.0, 1.0, c2.data(), k2.data()), nullptr);
        int32_t nfix = 0, nface = 0;
        check(plato_box_nodeset(6, 3, 3, 0, nullptr, &nfix), nullptr);
        std::vector<int32_t> fixed(nfix);
        check(plato_box_nodeset(6, 3, 3, 0, fixed.data(), &nfix), nullptr);
        check(plato_box_sideset(6, 3, 3, 1, nullptr, nullptr, &nface), nullptr);
        std::vector<int32_t> fc(nface), fl(3 * size_t(nface));
        check(plato_box_sideset(6, 3, 3, 1, fc.data(), fl.data(), &nface), nullptr);
        std::vector<int32_t> bcd;
        for (int32_t n : fixed)
            for (int d = 0; d < 3; ++d) bcd.push_back(3 * n + d);
        std::vector<double> bcv(bcd.size(), 0.0);
        plato_natural_bc load{nface, fc.data(), fl.data(), {0.0, -1.0, 0.0}};
        plato_problem_desc d{};
        d.mesh = {nn, nc, c2.data(), k2.data()};
        d.material = {1.0, 0.3};
        d.penalty = {3.0, 1e-9};
        d.num_natural_bcs = 1;
        d.natural_bcs = &load;
        d.essential_bcs = {int32_t(bcd.size()), bcd.data(), bcv.data()};
        d.solver = {1e-12, 10000, PLATO_OPERATOR_ASSEMBLED, PLATO_PRECISION_FP64, 1, 30.0, 0};
        auto cant = std::make_shared<Model>(d);
        Elliptic::Problem problem(cant);
        ScalarVector zc(std::vector<double>(size_t(nn), 0.5));
        const ScalarVector& state = problem.solution(zc);
        const double f = problem.criterionValue(zc);
        std::vector<double> g = problem.criterionGradient(zc).to_host();
        std::printf("solve: iterations %d converged %d relres %.3e\n", problem.lastSolveStats().iterations,
                    problem.lastSolveStats().converged, problem.lastSolveStats().relative_residual);
        std::printf("compliance: %.17g\n", f);
        print("state", state.to_host(), 3 * size_t(nn));
        print("dcdz", g, size_t(nn));

        // ---- Helmholtz filter on the same mesh, surface term on the x = 2 side ------------
        plato_helmholtz_desc hd{};
        hd.mesh = d.mesh;
        hd.length_scale = 0.2;
        hd.surface_length_scale = 0.5;
        hd.num_surface_faces = nface;
        hd.surface_face_cells = fc.data();
        hd.surface_face_local_nodes = fl.data();
        hd.solver.tolerance = 1e-13;
        auto filter = std::make_shared<Model>(hd);
        Helmholtz::Problem hp(filter);
        std::vector<double> ctl(static_cast<size_t>(nn)), w(static_cast<size_t>(nn));
        for (int32_t i = 0; i < nn; ++i) {
            ctl[i] = 0.25 + 0.5 * ((i * 7919) % 101) / 100.0;
            w[i] = 1.0 + 0.01 * (i % 13);
        }
        ScalarVector ctl_d(ctl), w_d(w);
        print("filtered", hp.solution(ctl_d).to_host(), size_t(nn));
        print("filter_gradient", hp.criterionGradient(w_d).to_host(), size_t(nn));
        Helmholtz::VectorFunction hvf(filter);
        print("filter_jacobian", hvf.gradient_u(ctl_d, ctl_d)->entries.to_host(), size_t(filter->numBlocks()));

        // error path: an exception carries the status
        try {
            plato_problem_desc bad = d;
            bad.material.poissons_ratio = 0.5;
            Model m(bad);
            std::printf("error_path: missing\n");
        } catch (const Error& e) {
            std::printf("error_path: status %d\n", e.status);
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "FAILED: %s\n", e.what());
        return 1;
    }
    return 0;
}
