// MPMD application: the reference's Analyze_App (src/Analyze_App.hpp, src/Analyze_App.cpp)
// over the C ABI of this library.  It reads the input deck (Teuchos ParameterList XML) and
// the PlatoEngine operations file, builds the problem the deck describes (elliptic SIMP
// elastostatics or the Helmholtz filter) on the device, and runs the named operations on
// the shared data a driver imports and exports ("Topology", criterion values and gradients,
// state components).
//
// Operations (src/Analyze_App.cpp:368-446): ComputeSolution, ComputeCriterion,
// ComputeCriterionValue, ComputeCriterionGradient, ApplyHelmholtz, ApplyHelmholtzGradient,
// UpdateProblem.  Operation parameters (<Parameter> with ArgumentName, Target,
// InitialValue; :596-615, :655-683) rewrite the deck at Target and rebuild the problem
// before its next operation, as the reference does.
//
// Meshes ("Input Mesh"): an Exodus II file (exodus.cpp), or "box:NX,NY,NZ[:LX,LY,LZ]", the
// generated Kuhn-split box with node and side sets "x-", "x+", "y-", "y+", "z-", "z+".
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "deck.hpp"
#include "plato_b200.h"

using plato::deck::DeckError;
using plato::deck::ParamList;
using plato::deck::XmlNode;

namespace {

struct AppError : std::runtime_error {
    AppError(int s, const std::string& m) : std::runtime_error(m), status(s) {}
    int status;
};

void check(int rc, plato_problem* h, const char* what) {
    if (rc != PLATO_OK) {
        const char* m = plato_last_error(h);
        throw AppError(rc, std::string(what) + ": " + (m ? m : ""));
    }
}

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw AppError(PLATO_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

std::string lower(std::string s) {
    for (char& c : s) c = char(std::tolower(static_cast<unsigned char>(c)));
    return s;
}

std::string trim(const std::string& s) {
    size_t b = s.find_first_not_of(" \t\r\n"), e = s.find_last_not_of(" \t\r\n");
    return b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
}

// ---- meshes --------------------------------------------------------------------------------

struct SideSet {
    std::vector<int32_t> cells;
    std::vector<int32_t> local;  // 3 per face
};

struct MeshData {
    int32_t num_nodes = 0, num_cells = 0;
    std::vector<double> coords;
    std::vector<int32_t> conn;
    std::map<std::string, std::vector<int32_t>> node_sets;
    std::map<std::string, SideSet> side_sets;
};

std::vector<std::string> split(const std::string& s, char sep) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, sep)) out.push_back(trim(item));
    return out;
}

MeshData box_mesh(const std::string& spec) {
    const auto parts = split(spec.substr(4), ':');
    if (parts.empty() || parts.size() > 2) throw AppError(PLATO_BAD_INPUT, "mesh spec must be box:NX,NY,NZ[:LX,LY,LZ]");
    const auto n = split(parts[0], ',');
    if (n.size() != 3) throw AppError(PLATO_BAD_INPUT, "box mesh needs three cell counts");
    int32_t nx = 0, ny = 0, nz = 0;
    try {
        nx = std::stoi(n[0]);
        ny = std::stoi(n[1]);
        nz = std::stoi(n[2]);
    } catch (const std::exception&) {
        throw AppError(PLATO_BAD_INPUT, "box mesh cell counts must be integers");
    }
    double lx = 1.0, ly = 1.0, lz = 1.0;
    if (parts.size() == 2) {
        const auto l = split(parts[1], ',');
        if (l.size() != 3) throw AppError(PLATO_BAD_INPUT, "box mesh needs three lengths");
        try {
            lx = std::stod(l[0]);
            ly = std::stod(l[1]);
            lz = std::stod(l[2]);
        } catch (const std::exception&) {
            throw AppError(PLATO_BAD_INPUT, "box mesh lengths must be numbers");
        }
    }
    MeshData m;
    check(plato_box_mesh_sizes(nx, ny, nz, &m.num_nodes, &m.num_cells), nullptr, "box mesh");
    m.coords.resize(3 * size_t(m.num_nodes));
    m.conn.resize(4 * size_t(m.num_cells));
    check(plato_box_mesh_tet4(nx, ny, nz, lx, ly, lz, m.coords.data(), m.conn.data()), nullptr, "box mesh");
    static const char* names[6] = {"x-", "x+", "y-", "y+", "z-", "z+"};
    for (int f = 0; f < 6; ++f) {
        int32_t cnt = 0;
        check(plato_box_nodeset(nx, ny, nz, f, nullptr, &cnt), nullptr, "box node set");
        std::vector<int32_t> nodes(cnt);
        check(plato_box_nodeset(nx, ny, nz, f, nodes.data(), &cnt), nullptr, "box node set");
        m.node_sets[names[f]] = std::move(nodes);
        check(plato_box_sideset(nx, ny, nz, f, nullptr, nullptr, &cnt), nullptr, "box side set");
        SideSet s;
        s.cells.resize(cnt);
        s.local.resize(3 * size_t(cnt));
        check(plato_box_sideset(nx, ny, nz, f, s.cells.data(), s.local.data(), &cnt), nullptr, "box side set");
        m.side_sets[names[f]] = std::move(s);
    }
    return m;
}

MeshData exodus_mesh(const std::string& path) {
    plato_mesh_file* f = nullptr;
    if (plato_mesh_file_open(path.c_str(), &f) != PLATO_OK)
        throw AppError(PLATO_BAD_INPUT, std::string("Input Mesh: ") + plato_mesh_file_last_error());
    std::unique_ptr<plato_mesh_file, int (*)(plato_mesh_file*)> guard(f, plato_mesh_file_close);
    MeshData m;
    int32_t nns = 0, nss = 0;
    plato_mesh_file_info(f, &m.num_nodes, &m.num_cells, &nns, &nss);
    m.coords.resize(3 * size_t(m.num_nodes));
    m.conn.resize(4 * size_t(m.num_cells));
    plato_mesh_file_mesh(f, m.coords.data(), m.conn.data());
    char name[256];
    for (int32_t k = 0; k < nns; ++k) {
        int32_t cnt = 0;
        plato_mesh_file_node_set(f, k, name, sizeof(name), nullptr, &cnt);
        std::vector<int32_t> nodes(cnt);
        plato_mesh_file_node_set(f, k, name, sizeof(name), nodes.data(), &cnt);
        m.node_sets[name] = std::move(nodes);
    }
    for (int32_t k = 0; k < nss; ++k) {
        int32_t cnt = 0;
        plato_mesh_file_side_set(f, k, name, sizeof(name), nullptr, nullptr, &cnt);
        SideSet s;
        s.cells.resize(cnt);
        s.local.resize(3 * size_t(cnt));
        plato_mesh_file_side_set(f, k, name, sizeof(name), s.cells.data(), s.local.data(), &cnt);
        m.side_sets[name] = std::move(s);
    }
    return m;
}

// "Input Mesh": a generated box, or an Exodus file (relative paths from base_dir)
MeshData load_mesh(const std::string& spec, const std::string& base_dir) {
    if (spec.rfind("box:", 0) == 0) return box_mesh(spec);
    const std::string path = (spec.empty() || spec[0] == '/' || base_dir.empty()) ? spec : base_dir + "/" + spec;
    return exodus_mesh(path);
}

using FaceKey = std::array<int32_t, 3>;

FaceKey face_key(const MeshData& m, int32_t cell, const int32_t* local) {
    FaceKey k;
    for (int a = 0; a < 3; ++a) k[a] = m.conn[4 * size_t(cell) + local[a]];
    std::sort(k.begin(), k.end());
    return k;
}

// Exterior faces (in one cell only) minus those in the named side sets: the faces
// GetSideSetElementsComplement / GetSideSetLocalNodesComplement return.
SideSet exterior_complement(const MeshData& m, const std::vector<std::string>& exclude) {
    static const int32_t faces[4][3] = {{0, 1, 3}, {1, 2, 3}, {0, 3, 2}, {0, 2, 1}};
    std::vector<std::pair<FaceKey, int64_t>> keys;
    keys.reserve(4 * size_t(m.num_cells));
    for (int32_t c = 0; c < m.num_cells; ++c)
        for (int f = 0; f < 4; ++f) keys.emplace_back(face_key(m, c, faces[f]), 4 * int64_t(c) + f);
    std::sort(keys.begin(), keys.end());
    std::vector<FaceKey> excluded;
    for (const std::string& name : exclude) {
        auto it = m.side_sets.find(name);
        if (it == m.side_sets.end()) throw AppError(PLATO_BAD_INPUT, "Symmetry Plane Sides: no side set '" + name + "'");
        for (size_t f = 0; f < it->second.cells.size(); ++f)
            excluded.push_back(face_key(m, it->second.cells[f], &it->second.local[3 * f]));
    }
    std::sort(excluded.begin(), excluded.end());
    std::vector<int64_t> chosen;
    for (size_t i = 0; i < keys.size();) {
        size_t j = i;
        while (j < keys.size() && keys[j].first == keys[i].first) ++j;
        if (j - i == 1 && !std::binary_search(excluded.begin(), excluded.end(), keys[i].first))
            chosen.push_back(keys[i].second);
        i = j;
    }
    std::sort(chosen.begin(), chosen.end());
    SideSet s;
    for (int64_t id : chosen) {
        s.cells.push_back(int32_t(id / 4));
        for (int a = 0; a < 3; ++a) s.local.push_back(faces[id % 4][a]);
    }
    return s;
}

// ---- device vectors ------------------------------------------------------------------------

struct DVec {
    double* p = nullptr;
    size_t n = 0;
    DVec() = default;
    DVec(const DVec&) = delete;
    DVec& operator=(const DVec&) = delete;
    ~DVec() {
        if (p) cudaFree(p);
    }
    void resize(size_t count) {
        if (count == n) return;
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        if (count) cuda_check(cudaMalloc(&p, count * sizeof(double)), "cudaMalloc");
    }
    void fill(double v) {
        std::vector<double> h(n, v);
        upload(h.data(), n);
    }
    void upload(const double* src, size_t count) {
        if (count != n) throw AppError(PLATO_BAD_INPUT, "field size mismatch");
        if (n) cuda_check(cudaMemcpy(p, src, n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    }
    void download(double* dst, size_t count) const {
        if (count != n) throw AppError(PLATO_BAD_INPUT, "field size mismatch");
        if (n) cuda_check(cudaMemcpy(dst, p, n * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
    }
    void copy_from(const DVec& o) {
        resize(o.n);
        if (n) cuda_check(cudaMemcpy(p, o.p, n * sizeof(double), cudaMemcpyDeviceToDevice), "cudaMemcpy D2D");
    }
};

// ---- problem built from a deck --------------------------------------------------------------

enum class Physics { Elliptic, Helmholtz };

struct Criterion {
    enum Kind { Energy, Volume } kind = Energy;
    bool linear = false;
    plato_penalty penalty{3.0, 1e-9};
};

plato_penalty read_penalty(const ParamList& owner) {
    plato_penalty p{3.0, 1e-9};  // MSIMP defaults, src/Simp.hpp:48-49
    if (owner.is_sublist("Penalty Function")) {
        const ParamList& pf = owner.sublist("Penalty Function");
        const std::string type = lower(pf.get_string("Type", "SIMP"));
        if (type != "simp")
            throw AppError(PLATO_NOT_SUPPORTED, "Penalty Function type '" + pf.get_string("Type") + "': only SIMP is built");
        p.exponent = pf.get_double("Exponent", 3.0);
        p.minimum_value = pf.get_double("Minimum Value", 1e-9);
    }
    return p;
}

plato_solver_opts read_solver(const ParamList& deck) {
    plato_solver_opts o{};
    o.tolerance = 1e-10;
    o.max_iterations = 20000;
    o.operator_kind = PLATO_OPERATOR_ASSEMBLED;
    o.precision = PLATO_PRECISION_FP64;
    o.self_adjoint = deck.get_bool("Self-Adjoint", false) ? 1 : 0;  // src/elliptic/Problem.hpp:113
    o.chebyshev_ratio = 30.0;
    if (!deck.is_sublist("Linear Solver")) return o;
    const ParamList& ls = deck.sublist("Linear Solver");
    o.tolerance = ls.get_double("Tolerance", o.tolerance);  // src/alg/EpetraLinearSolver.cpp:146-149
    o.max_iterations = ls.get_int("Iterations", o.max_iterations);
    const std::string method = lower(ls.get_string("Method", "plain"));
    if (method == "plain") {
    } else if (method == "chebyshev" || method == "two-level") {
        o.precision = PLATO_PRECISION_MIXED_FP32;
        o.chebyshev_degree = ls.get_int("Chebyshev Degree", 8);
        if (method == "two-level") {
            const std::vector<double> cc = ls.get_double_array("Coarse Cells");
            if (cc.size() != 3) throw AppError(PLATO_BAD_INPUT, "Linear Solver: 'Coarse Cells' needs three counts");
            for (int d = 0; d < 3; ++d) o.coarse_cells[d] = int32_t(cc[d]);
        }
    } else if (method == "bf16") {
        o.precision = PLATO_PRECISION_MIXED_BF16;
        o.chebyshev_degree = ls.get_int("Chebyshev Degree", 16);
    } else {
        throw AppError(PLATO_BAD_INPUT, "Linear Solver: unknown Method '" + ls.get_string("Method") + "'");
    }
    o.chebyshev_ratio = ls.get_double("Chebyshev Ratio", o.chebyshev_ratio);
    o.chebyshev_kind = ls.get_int("Chebyshev Kind", 1);
    if (o.chebyshev_kind != 1 && o.chebyshev_kind != 4)
        throw AppError(PLATO_BAD_INPUT, "Linear Solver: 'Chebyshev Kind' must be 1 or 4");
    return o;
}

// Everything the deck says about one problem, resolved against the mesh on the host; the
// descriptors point into the vectors held here.
struct ProblemSpec {
    Physics physics = Physics::Elliptic;
    plato_problem_desc desc{};
    plato_helmholtz_desc helm{};
    std::vector<plato_natural_bc> nbcs;
    std::vector<int32_t> bc_dofs;
    std::vector<double> bc_values;
    SideSet faces;
    std::map<std::string, Criterion> criteria;
    std::vector<std::string> dof_names;
    int32_t num_dofs = 0;
};

struct Problem {
    Physics physics = Physics::Elliptic;
    plato_problem* h = nullptr;
    int32_t num_nodes = 0, num_dofs = 0;
    std::map<std::string, Criterion> criteria;
    std::vector<std::string> dof_names;
    ~Problem() {
        if (h) plato_destroy(h);
    }
};

// `root` is an input config: "Input Mesh" and "Spatial Dimension" at its top, the problem in
// its "Plato Problem" sublist (src/PlatoProblemFactory.hpp:439; a deck without that sublist
// is taken as the problem list itself).
std::unique_ptr<ProblemSpec> parse_problem(const MeshData& m, const ParamList& root) {
    auto P = std::make_unique<ProblemSpec>();
    const ParamList& deck = root.is_sublist("Plato Problem") ? root.sublist("Plato Problem") : root;
    const std::string physics = lower(deck.get_string("Physics", ""));
    const std::string pde = lower(deck.get_string("PDE Constraint", ""));
    plato_mesh_desc mesh{m.num_nodes, m.num_cells, m.coords.data(), m.conn.data()};

    if (physics == "helmholtz filter") {
        P->physics = Physics::Helmholtz;
        // HelmholtzResidual constructor, src/helmholtz/HelmholtzResidual.hpp:74-84
        if (!deck.is_sublist("Parameters"))
            throw AppError(PLATO_BAD_INPUT, "NO PARAMETERS SUBLIST WAS PROVIDED FOR THE HELMHOLTZ FILTER.");
        const ParamList& prm = deck.sublist("Parameters");
        plato_helmholtz_desc& d = P->helm;
        d.mesh = mesh;
        d.length_scale = prm.get_double("Length Scale", 0.5);
        d.surface_length_scale = prm.get_double("Surface Length Scale", 0.0);
        if (!(d.length_scale > 0.0)) throw AppError(PLATO_BAD_INPUT, "Helmholtz filter: 'Length Scale' must be positive");
        if (d.surface_length_scale > 0.0) {
            std::vector<std::string> sym;
            if (prm.has("Symmetry Plane Sides")) sym = prm.get_string_array("Symmetry Plane Sides");
            P->faces = exterior_complement(m, sym);
        }
        d.num_surface_faces = int32_t(P->faces.cells.size());
        d.surface_face_cells = P->faces.cells.data();
        d.surface_face_local_nodes = P->faces.local.data();
        d.solver = read_solver(deck);
        if (!deck.is_sublist("Linear Solver")) d.solver.tolerance = 1e-12;
        P->num_dofs = m.num_nodes;
        P->dof_names = {"filtered density"};
        return P;
    }
    if (physics != "mechanical")
        throw AppError(PLATO_NOT_SUPPORTED, "Physics '" + deck.get_string("Physics", "") +
                                                "': only 'Mechanical' and 'Helmholtz Filter' are built");
    if (pde != "elliptic")
        throw AppError(PLATO_NOT_SUPPORTED, "'PDE Constraint' of type '" + pde + "' is not supported.");
    if (root.get_int("Spatial Dimension", 3) != 3) throw AppError(PLATO_NOT_SUPPORTED, "only 'Spatial Dimension' 3 is built");

    // material of the (single) domain, src/IsotropicLinearElasticMaterial.cpp:86-126
    const ParamList& domains = deck.sublist("Spatial Model").sublist("Domains");
    if (domains.entries.size() != 1) throw AppError(PLATO_NOT_SUPPORTED, "one domain per problem is built");
    const ParamList& dom = *domains.entries[0].second.list;
    const std::string mat_name = dom.get_string("Material Model");
    const ParamList& mat = deck.sublist("Material Models").sublist(mat_name);
    if (!mat.is_sublist("Isotropic Linear Elastic"))
        throw AppError(PLATO_NOT_SUPPORTED, "material '" + mat_name + "': only 'Isotropic Linear Elastic' is built");
    const ParamList& ile = mat.sublist("Isotropic Linear Elastic");

    plato_problem_desc& d = P->desc;
    d.mesh = mesh;
    d.material.youngs_modulus = ile.get_double("Youngs Modulus");
    d.material.poissons_ratio = ile.get_double("Poissons Ratio");
    const plato_penalty pde_penalty = deck.is_sublist("Elliptic") ? read_penalty(deck.sublist("Elliptic"))
                                                                  : plato_penalty{3.0, 1e-9};
    d.penalty = pde_penalty;

    // natural BCs, src/NaturalBCs.hpp:110-310
    std::vector<plato_natural_bc>& nbcs = P->nbcs;
    if (deck.is_sublist("Natural Boundary Conditions")) {
        for (const auto& e : deck.sublist("Natural Boundary Conditions").entries) {
            if (!e.second.is_list()) continue;
            const ParamList& bc = *e.second.list;
            const std::string type = lower(bc.get_string("Type"));
            const std::string side = bc.get_string("Sides");
            auto it = m.side_sets.find(side);
            if (it == m.side_sets.end()) throw AppError(PLATO_BAD_INPUT, "natural BC '" + e.first + "': no side set '" + side + "'");
            plato_natural_bc nb{};
            nb.num_faces = int32_t(it->second.cells.size());
            nb.face_cells = it->second.cells.data();
            nb.face_local_nodes = it->second.local.data();
            if (type == "uniform") {
                const bool has_values = bc.has("Values"), has_value = bc.has("Value");
                if (has_values == has_value)
                    throw AppError(PLATO_BAD_INPUT, "natural BC '" + e.first + "': give 'Values' or 'Value'");
                if (has_values) {
                    const std::vector<double> v = bc.get_double_array("Values");
                    if (v.size() != 3) throw AppError(PLATO_BAD_INPUT, "natural BC '" + e.first + "': 'Values' needs 3 entries");
                    for (int k = 0; k < 3; ++k) nb.vector[k] = v[k];
                } else {
                    const double v = bc.get_double("Value");
                    for (int k = 0; k < 3; ++k) nb.vector[k] = v;
                }
            } else if (type == "uniform component") {
                const std::string comp = lower(bc.get_string("Component"));
                const int k = comp == "x" ? 0 : comp == "y" ? 1 : comp == "z" ? 2 : -1;
                if (k < 0) throw AppError(PLATO_BAD_INPUT, "natural BC '" + e.first + "': Component must be X, Y or Z");
                nb.vector[k] = bc.get_double("Value");
            } else {
                throw AppError(PLATO_NOT_SUPPORTED, "natural BC type '" + bc.get_string("Type") + "' is not built");
            }
            nbcs.push_back(nb);
        }
    }
    d.num_natural_bcs = int32_t(nbcs.size());
    d.natural_bcs = nbcs.data();

    // essential BCs, src/EssentialBCs.hpp:74-94 (later entries win on a shared dof)
    std::map<int32_t, double> fixed;
    if (deck.is_sublist("Essential Boundary Conditions")) {
        for (const auto& e : deck.sublist("Essential Boundary Conditions").entries) {
            if (!e.second.is_list()) continue;
            const ParamList& bc = *e.second.list;
            const std::string type = bc.get_string("Type");
            double value = 0.0;
            if (type == "Zero Value") value = 0.0;
            else if (type == "Fixed Value") value = bc.get_double("Value");
            else throw AppError(PLATO_BAD_INPUT, "Boundary Condition type invalid: Not 'Zero Value' or 'Fixed Value'.");
            const int index = bc.get_int("Index", 0);
            if (index < 0 || index > 2) throw AppError(PLATO_BAD_INPUT, "essential BC '" + e.first + "': Index out of range");
            const std::string side = bc.get_string("Sides");
            auto it = m.node_sets.find(side);
            if (it == m.node_sets.end()) throw AppError(PLATO_BAD_INPUT, "essential BC '" + e.first + "': no node set '" + side + "'");
            for (int32_t node : it->second) fixed[3 * node + index] = value;
        }
    }
    std::vector<int32_t>& bc_dofs = P->bc_dofs;
    std::vector<double>& bc_values = P->bc_values;
    for (const auto& kv : fixed) {
        bc_dofs.push_back(kv.first);
        bc_values.push_back(kv.second);
    }
    d.essential_bcs = {int32_t(bc_dofs.size()), bc_dofs.data(), bc_values.data()};
    d.solver = read_solver(deck);

    // criteria, src/elliptic/Problem.hpp:649-690
    if (deck.is_sublist("Criteria")) {
        for (const auto& e : deck.sublist("Criteria").entries) {
            if (!e.second.is_list()) throw AppError(PLATO_BAD_INPUT, " Parameter in Criteria block not valid.  Expect lists only.");
            const ParamList& c = *e.second.list;
            Criterion cr;
            cr.linear = c.get_bool("Linear", false);
            const std::string type = c.get_string("Scalar Function Type", "");
            if (type == "Internal Elastic Energy") {
                cr.kind = Criterion::Energy;
                const plato_penalty cp = read_penalty(c);
                if (cp.exponent != pde_penalty.exponent || cp.minimum_value != pde_penalty.minimum_value)
                    throw AppError(PLATO_NOT_SUPPORTED, "criterion '" + e.first +
                                                            "': its Penalty Function must equal the PDE's (one penalty per problem)");
            } else if (type == "Volume") {
                cr.kind = Criterion::Volume;
                cr.linear = true;
                cr.penalty = read_penalty(c);
            } else {
                throw AppError(PLATO_NOT_SUPPORTED, "criterion '" + e.first + "': Scalar Function Type '" + type + "' is not built");
            }
            P->criteria[e.first] = cr;
        }
    }
    P->num_dofs = 3 * m.num_nodes;
    P->dof_names = {"displacement X", "displacement Y", "displacement Z"};
    return P;
}

std::unique_ptr<Problem> create_problem(const MeshData& m, const ParamList& deck) {
    const std::unique_ptr<ProblemSpec> S = parse_problem(m, deck);
    auto P = std::make_unique<Problem>();
    P->physics = S->physics;
    P->num_nodes = m.num_nodes;
    P->num_dofs = S->num_dofs;
    P->criteria = S->criteria;
    P->dof_names = S->dof_names;
    if (S->physics == Physics::Helmholtz)
        check(plato_create_helmholtz(&S->helm, &P->h), nullptr, "Helmholtz filter");
    else
        check(plato_create(&S->desc, &P->h), nullptr, "elliptic problem");
    return P;
}

// ---- operations ----------------------------------------------------------------------------

struct OpParameter {
    std::string target;
    double value = 0.0;
};

struct Operation {
    std::string function, name, definition, criterion;
    double target = 0.0;
    std::string value_name, gradient_name;
    std::map<std::string, OpParameter> parameters;
};

// getArgumentName, src/Analyze_App.cpp:77-118
std::string argument_name(const XmlNode& op, const std::string& argument, bool required) {
    for (const XmlNode* out : op.children_named("Output")) {
        if (out->child_text("Argument") == argument) {
            const std::string n = out->child_text("ArgumentName");
            if (n.empty()) throw AppError(PLATO_BAD_INPUT, "operation '" + op.child_text("Name") + "': 'ArgumentName' missing");
            return n;
        }
    }
    if (required)
        throw AppError(PLATO_BAD_INPUT, "operation '" + op.child_text("Name") + "': '" + argument + "' output argument missing");
    return std::string();
}

struct Definition {
    std::shared_ptr<ParamList> params;
    bool modified = false;
};

}  // namespace

struct plato_app {
    std::string last_error;
    std::string base_dir;
    std::map<std::string, Definition> definitions;
    std::string default_definition, current_definition;
    std::map<std::string, Operation> operations;

    std::string mesh_spec;
    MeshData mesh;
    std::unique_ptr<Problem> problem;

    DVec control, state, scratch;
    std::map<std::string, double> values;        // criterion -> value minus target
    std::map<std::string, std::unique_ptr<DVec>> gradients;  // criterion -> dF/dz
    std::map<std::string, std::string> value_names, gradient_names;  // shared-data name -> criterion
    bool have_state = false;

    std::string resolve(const std::string& path) const {
        if (path.empty() || path[0] == '/' || base_dir.empty()) return path;
        return base_dir + "/" + path;
    }

    std::shared_ptr<ParamList> load_deck(const std::string& text_or_path) const {
        const std::string t = trim(text_or_path);
        if (!t.empty() && t[0] == '<') return plato::deck::parse_param_list(t);
        return plato::deck::parse_param_list(plato::deck::read_file(resolve(t)));
    }

    void build(const std::string& def_name) {
        Definition& d = definitions.at(def_name);
        const ParamList& deck = *d.params;
        if (!deck.has("Input Mesh"))
            throw AppError(PLATO_BAD_INPUT, "Analyze Application: 'Input Mesh' keyword was not defined. "
                                            "Use the 'Input Mesh' keyword to provide the name of the mesh file.");
        const std::string spec = deck.get_string("Input Mesh");
        if (spec != mesh_spec || mesh.num_nodes == 0) {
            mesh = load_mesh(spec, base_dir);
            mesh_spec = spec;
        }
        problem.reset();
        problem = create_problem(mesh, deck);
        current_definition = def_name;
        d.modified = false;
        // resetProblemMetaData: the control keeps its values while the node count holds
        if (control.n != size_t(mesh.num_nodes)) {
            control.resize(mesh.num_nodes);
            control.fill(1.0);
        }
        state.resize(problem->num_dofs);
        scratch.resize(mesh.num_nodes);
        for (auto& g : gradients) g.second->resize(mesh.num_nodes);
        have_state = false;
    }

    void solve_state() {
        plato_solve_stats st{};
        if (problem->physics == Physics::Helmholtz)
            check(plato_helmholtz_solution(problem->h, control.p, state.p, &st), problem->h, "solution");
        else
            check(plato_problem_solution(problem->h, control.p, nullptr, state.p, &st), problem->h, "solution");
        have_state = true;
    }

    const Criterion& criterion(const std::string& name) const {
        auto it = problem->criteria.find(name);
        if (it == problem->criteria.end()) throw AppError(PLATO_BAD_INPUT, "no criterion '" + name + "' in the problem");
        return it->second;
    }

    double criterion_value(const std::string& name) {
        const Criterion& c = criterion(name);
        double v = 0.0;
        if (c.kind == Criterion::Volume) {
            check(plato_volume_value(problem->h, control.p, &c.penalty, &v), problem->h, "criterion value");
        } else {
            if (!have_state) solve_state();
            check(plato_problem_criterion_value(problem->h, control.p, state.p, &v), problem->h, "criterion value");
        }
        return v;
    }

    void criterion_gradient(const std::string& name, DVec& out) {
        const Criterion& c = criterion(name);
        out.resize(mesh.num_nodes);
        if (c.kind == Criterion::Volume) {
            check(plato_volume_gradient_z(problem->h, control.p, &c.penalty, out.p), problem->h, "criterion gradient");
        } else {
            if (!have_state) solve_state();
            plato_solve_stats st{};
            check(plato_problem_criterion_gradient(problem->h, control.p, state.p, out.p, &st), problem->h,
                  "criterion gradient");
        }
    }

    void run(Operation& op) {
        // MPMD_App::compute, src/Analyze_App.cpp:566-590: rebuild when another definition is
        // needed or this one was modified by an operation parameter
        if (op.definition != current_definition || definitions.at(op.definition).modified) build(op.definition);
        const std::string& f = op.function;
        const bool elliptic = problem->physics == Physics::Elliptic;
        if (f == "ComputeSolution") {
            solve_state();
        } else if (f == "ComputeCriterion" || f == "ComputeCriterionValue" || f == "ComputeCriterionGradient") {
            if (!elliptic) throw AppError(PLATO_BAD_INPUT, f + " needs an elliptic problem");
            const Criterion& c = criterion(op.criterion);
            if (!c.linear && f != "ComputeCriterionGradient") solve_state();
            if (f != "ComputeCriterionGradient") values[op.criterion] = criterion_value(op.criterion) - op.target;
            if (f != "ComputeCriterionValue") {
                auto& g = gradients[op.criterion];
                if (!g) g = std::make_unique<DVec>();
                criterion_gradient(op.criterion, *g);
            }
        } else if (f == "ApplyHelmholtz") {
            if (elliptic) throw AppError(PLATO_BAD_INPUT, "ApplyHelmholtz needs a Helmholtz Filter problem");
            solve_state();
            control.copy_from(state);
        } else if (f == "ApplyHelmholtzGradient") {
            if (elliptic) throw AppError(PLATO_BAD_INPUT, "ApplyHelmholtzGradient needs a Helmholtz Filter problem");
            plato_solve_stats st{};
            scratch.resize(mesh.num_nodes);
            check(plato_helmholtz_criterion_gradient(problem->h, control.p, scratch.p, &st), problem->h,
                  "criterion gradient");
            control.copy_from(scratch);
        } else if (f == "UpdateProblem") {
            // continuation hooks of the penalty (src/Analyze_App.cpp UpdateProblem): MSIMP has
            // none in the elliptic path, so the problem is unchanged
        } else {
            throw AppError(PLATO_NOT_SUPPORTED, "operation function '" + f + "' is not built");
        }
    }

    void parse_operations(const XmlNode& root) {
        std::vector<const XmlNode*> ops;
        if (root.tag == "Operation") ops.push_back(&root);
        for (const XmlNode* o : root.children_named("Operation")) ops.push_back(o);
        for (const XmlNode* node : ops) {
            Operation op;
            op.function = node->child_text("Function");
            op.name = node->child_text("Name");
            if (op.function.empty() || op.name.empty())
                throw AppError(PLATO_BAD_INPUT, "an Operation needs 'Function' and 'Name'");
            if (operations.count(op.name)) throw AppError(PLATO_BAD_INPUT, "operation '" + op.name + "' defined twice");
            op.definition = node->child_text("ProblemDefinition", default_definition);
            if (!definitions.count(op.definition)) {
                Definition d;
                d.params = load_deck(op.definition);
                definitions[op.definition] = d;
            }
            for (const XmlNode* p : node->children_named("Parameter")) {
                const std::string an = p->child_text("ArgumentName");
                if (an.empty()) throw AppError(PLATO_BAD_INPUT, "operation parameter without ArgumentName");
                if (op.parameters.count(an)) throw AppError(PLATO_BAD_INPUT, "ArgumentNames must be unique.");
                OpParameter prm;
                prm.target = p->child_text("Target");
                const std::string iv = p->child_text("InitialValue", "0");
                try {
                    prm.value = std::stod(iv);
                } catch (const std::exception&) {
                    throw AppError(PLATO_BAD_INPUT, "parameter '" + an + "': InitialValue is not a number");
                }
                op.parameters[an] = prm;
            }
            const bool crit = op.function.rfind("ComputeCriterion", 0) == 0;
            if (crit) {
                op.criterion = node->child_text("Criterion");
                if (op.criterion.empty()) throw AppError(PLATO_BAD_INPUT, "Required keyword ('Criterion') missing.");
                const std::string t = node->child_text("Target", "0");
                try {
                    op.target = std::stod(t);
                } catch (const std::exception&) {
                    throw AppError(PLATO_BAD_INPUT, "operation '" + op.name + "': Target is not a number");
                }
                if (op.function != "ComputeCriterionGradient") {
                    op.value_name = argument_name(*node, "Value", false);
                    if (!op.value_name.empty()) add_unique(value_names, op.value_name, op.criterion);
                }
                if (op.function != "ComputeCriterionValue") {
                    op.gradient_name = argument_name(*node, "Gradient", false);
                    if (!op.gradient_name.empty()) add_unique(gradient_names, op.gradient_name, op.criterion);
                }
            }
            operations[op.name] = op;
        }
    }

    static void add_unique(std::map<std::string, std::string>& m, const std::string& k, const std::string& v) {
        auto it = m.find(k);
        if (it != m.end() && it->second != v)
            throw AppError(PLATO_BAD_INPUT, "shared data name '" + k + "' already belongs to criterion '" + it->second + "'");
        m[k] = v;
    }
};

namespace {

int fail(plato_app* a, int status, const std::string& msg) {
    if (a) a->last_error = msg;
    return status;
}

template <class F>
int guarded(plato_app* a, F&& f) {
    if (!a) return PLATO_BAD_INPUT;
    try {
        f();
        return PLATO_OK;
    } catch (const AppError& e) {
        return fail(a, e.status, e.what());
    } catch (const DeckError& e) {
        return fail(a, PLATO_BAD_INPUT, e.what());
    } catch (const std::bad_alloc&) {
        return fail(a, PLATO_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(a, PLATO_BAD_INPUT, e.what());
    }
}

thread_local std::string g_create_error;

}  // namespace

extern "C" {

namespace {

void setup_app(plato_app* app, const char* input_config, const char* operations) {
    app->default_definition = "__input_config__";
    Definition d;
    d.params = app->load_deck(input_config);
    app->definitions[app->default_definition] = d;
    const std::string ops = trim(operations);
    const XmlNode root =
        plato::deck::parse_xml(!ops.empty() && ops[0] == '<' ? ops : plato::deck::read_file(app->resolve(ops)));
    app->parse_operations(root);
}

void copy_message(const std::string& m, char* buf, int64_t cap) {
    if (!buf || cap <= 0) return;
    const size_t n = std::min<size_t>(m.size(), size_t(cap - 1));
    std::memcpy(buf, m.data(), n);
    buf[n] = '\0';
}

}  // namespace

int plato_app_validate(const char* input_config, const char* operations, const char* base_dir, char* message,
                       int64_t capacity) {
    copy_message("", message, capacity);
    if (!input_config || !operations) {
        copy_message("input config and operations are required", message, capacity);
        return PLATO_BAD_INPUT;
    }
    plato_app app;
    app.base_dir = base_dir ? base_dir : "";
    const int rc = guarded(&app, [&] {
        setup_app(&app, input_config, operations);
        for (const auto& kv : app.definitions) {
            const ParamList& deck = *kv.second.params;
            if (!deck.has("Input Mesh"))
                throw AppError(PLATO_BAD_INPUT, "Analyze Application: 'Input Mesh' keyword was not defined. "
                                                "Use the 'Input Mesh' keyword to provide the name of the mesh file.");
            const MeshData m = load_mesh(deck.get_string("Input Mesh"), app.base_dir);
            const auto spec = parse_problem(m, deck);
            for (const auto& op : app.operations)
                if (op.second.definition == kv.first && !op.second.criterion.empty() &&
                    !spec->criteria.count(op.second.criterion))
                    throw AppError(PLATO_BAD_INPUT, "operation '" + op.first + "': no criterion '" + op.second.criterion + "'");
        }
    });
    copy_message(app.last_error, message, capacity);
    return rc;
}

int plato_deck_to_text(const char* input_config, char* text, int64_t capacity, int64_t* needed) {
    if (!input_config || !needed) return PLATO_BAD_INPUT;
    try {
        plato_app tmp;
        const auto L = tmp.load_deck(input_config);
        std::string out;
        std::function<void(const ParamList&, const std::string&)> dump = [&](const ParamList& l, const std::string& pre) {
            for (const auto& e : l.entries) {
                if (e.second.is_list()) {
                    out += pre + e.first + ":\n";
                    dump(*e.second.list, pre + "  ");
                } else {
                    out += pre + e.first + " (" + e.second.type + ") = " + e.second.value + "\n";
                }
            }
        };
        dump(*L, "");
        *needed = int64_t(out.size()) + 1;
        if (text && capacity > 0) copy_message(out, text, capacity);
        return PLATO_OK;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        *needed = 0;
        return PLATO_BAD_INPUT;
    }
}

int plato_app_create(const char* input_config, const char* operations, const char* base_dir, plato_app** out) {
    if (!out) return PLATO_BAD_INPUT;
    *out = nullptr;
    if (!input_config || !operations) {
        g_create_error = "input config and operations are required";
        return PLATO_BAD_INPUT;
    }
    auto app = std::make_unique<plato_app>();
    app->base_dir = base_dir ? base_dir : "";
    const int rc = guarded(app.get(), [&] {
        setup_app(app.get(), input_config, operations);
        app->build(app->default_definition);
    });
    if (rc != PLATO_OK) {
        g_create_error = app->last_error;
        return rc;
    }
    *out = app.release();
    return PLATO_OK;
}

int plato_app_destroy(plato_app* a) {
    delete a;
    return PLATO_OK;
}

const char* plato_app_last_error(const plato_app* a) { return a ? a->last_error.c_str() : g_create_error.c_str(); }

int plato_app_num_nodes(const plato_app* a, int32_t* num_nodes) {
    if (!a || !num_nodes) return PLATO_BAD_INPUT;
    *num_nodes = a->mesh.num_nodes;
    return PLATO_OK;
}

int plato_app_compute(plato_app* a, const char* operation) {
    return guarded(a, [&] {
        if (!operation) throw AppError(PLATO_BAD_INPUT, "null operation name");
        auto it = a->operations.find(operation);
        if (it == a->operations.end())
            throw AppError(PLATO_BAD_INPUT, std::string("Request for operation ('") + operation + "') that doesn't exist.");
        a->run(it->second);
    });
}

int plato_app_import(plato_app* a, const char* name, int32_t layout, const char* context, const double* data,
                     int64_t count) {
    return guarded(a, [&] {
        if (!name || (!data && count)) throw AppError(PLATO_BAD_INPUT, "null argument");
        const std::string n = name;
        if (layout == PLATO_LAYOUT_SCALAR_FIELD) {
            if (n == "Topology") {
                a->control.upload(data, size_t(count));
            } else if (n == "Solution") {
                if (size_t(count) != a->state.n) throw AppError(PLATO_BAD_INPUT, "Solution size mismatch");
                a->state.upload(data, size_t(count));
                a->have_state = true;
            } else {
                throw AppError(PLATO_BAD_INPUT, "cannot import field '" + n + "'");
            }
        } else if (layout == PLATO_LAYOUT_SCALAR_PARAMETER) {
            // importScalarParameter, src/Analyze_App.hpp:231-246: the context names the operation
            if (!context) throw AppError(PLATO_BAD_INPUT, "a parameter needs the operation as its context");
            auto it = a->operations.find(context);
            if (it == a->operations.end()) throw AppError(PLATO_BAD_INPUT, std::string("no operation '") + context + "'");
            auto pit = it->second.parameters.find(n);
            if (pit == it->second.parameters.end())
                throw AppError(PLATO_BAD_INPUT, "Attempted to update a parameter ('" + n + "') that wasn't defined for this operation");
            if (count < 1) throw AppError(PLATO_BAD_INPUT, "empty parameter value");
            pit->second.value = data[0];
            if (!pit->second.target.empty()) {
                Definition& d = a->definitions.at(it->second.definition);
                d.params->set_target(pit->second.target, data[0]);  // parse_inline, src/AnalyzeAppUtils.cpp:46-120
                d.modified = true;
            }
        } else {
            throw AppError(PLATO_BAD_INPUT, "unsupported import layout");
        }
    });
}

int plato_app_export(plato_app* a, const char* name, int32_t layout, double* data, int64_t count) {
    return guarded(a, [&] {
        if (!name || (!data && count)) throw AppError(PLATO_BAD_INPUT, "null argument");
        std::string n = name;
        int index = 0;
        const size_t at = n.find('@');
        if (at != std::string::npos) {
            index = std::atoi(n.c_str() + at + 1);
            n = n.substr(0, at);
        }
        (void)index;
        if (layout == PLATO_LAYOUT_SCALAR_VALUE) {
            auto it = a->value_names.find(n);
            if (it == a->value_names.end()) throw AppError(PLATO_BAD_INPUT, "no value named '" + n + "'");
            auto v = a->values.find(it->second);
            if (v == a->values.end()) throw AppError(PLATO_BAD_INPUT, "value '" + n + "' has not been computed");
            if (count != 1) throw AppError(PLATO_BAD_INPUT, "a value has one entry");
            data[0] = v->second;
        } else if (layout == PLATO_LAYOUT_SCALAR_FIELD) {
            if (n == "Topology") {
                a->control.download(data, size_t(count));
                return;
            }
            auto g = a->gradient_names.find(n);
            if (g != a->gradient_names.end()) {
                auto it = a->gradients.find(g->second);
                if (it == a->gradients.end() || !it->second) throw AppError(PLATO_BAD_INPUT, "gradient '" + n + "' has not been computed");
                it->second->download(data, size_t(count));
                return;
            }
            const auto& names = a->problem->dof_names;
            auto d = std::find(names.begin(), names.end(), n);
            if (d == names.end()) throw AppError(PLATO_BAD_INPUT, "no field named '" + n + "'");
            if (!a->have_state) throw AppError(PLATO_BAD_INPUT, "no state has been computed");
            const size_t ncomp = names.size(), comp = size_t(d - names.begin());
            if (size_t(count) != size_t(a->mesh.num_nodes)) throw AppError(PLATO_BAD_INPUT, "field size mismatch");
            std::vector<double> all(a->state.n);
            a->state.download(all.data(), all.size());
            for (size_t i = 0; i < size_t(count); ++i) data[i] = all[ncomp * i + comp];
        } else {
            throw AppError(PLATO_BAD_INPUT, "unsupported export layout");
        }
    });
}

}  // extern "C"
