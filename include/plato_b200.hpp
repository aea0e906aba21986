// plato_b200.hpp -- header-only C++ adapter over the C ABI (plato_b200.h).
//
// Mirrors the reference's elliptic interfaces so a caller written against them maps one to
// one: Plato::Elliptic::VectorFunction (value, gradient_u, gradient_u_T, gradient_z;
// src/elliptic/VectorFunction.hpp:251-710), Plato::Elliptic::PhysicsScalarFunction
// "Internal Elastic Energy" (value, gradient_u, gradient_z;
// src/elliptic/PhysicsScalarFunction.hpp:226-495), Plato::AbstractSolver::solve
// (src/alg/PlatoAbstractSolver.hpp:38-106) and Plato::Elliptic::Problem (solution,
// criterionValue, criterionGradient; src/elliptic/Problem.hpp:237-450).
// Errors become exceptions (std::runtime_error), as ANALYZE_THROWERR does in the reference.
// Vectors and matrices live in device memory (the reference returns Kokkos device views).
#pragma once

#include <cuda_runtime_api.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "plato_b200.h"

namespace plato_b200 {

class Error : public std::runtime_error {
public:
    Error(int status, const std::string& msg) : std::runtime_error(msg), status(status) {}
    int status;
};

inline void check(int rc, const plato_problem* h) {
    if (rc != PLATO_OK) {
        const char* m = plato_last_error(h);
        throw Error(rc, std::string("plato_b200 status ") + std::to_string(rc) + ": " + (m ? m : ""));
    }
}

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(PLATO_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

// Owning device array (Kokkos::View<T*> stand-in).
template <typename T>
class DeviceArray {
public:
    DeviceArray() = default;
    explicit DeviceArray(size_t n) : n_(n) {
        if (n) cuda_check(cudaMalloc(reinterpret_cast<void**>(&p_), n * sizeof(T)), "cudaMalloc");
        if (n) cuda_check(cudaMemset(p_, 0, n * sizeof(T)), "cudaMemset");
    }
    DeviceArray(const std::vector<T>& host) : DeviceArray(host.size()) { copy_from(host); }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    DeviceArray(DeviceArray&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DeviceArray& operator=(DeviceArray&& o) noexcept {
        if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    ~DeviceArray() { release(); }

    T* data() { return p_; }
    const T* data() const { return p_; }
    size_t size() const { return n_; }
    void copy_from(const std::vector<T>& host) {
        if (host.size() != n_) throw Error(PLATO_BAD_INPUT, "DeviceArray size mismatch");
        cuda_check(cudaMemcpy(p_, host.data(), n_ * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    }
    std::vector<T> to_host() const {
        std::vector<T> h(n_);
        if (n_) cuda_check(cudaMemcpy(h.data(), p_, n_ * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
        return h;
    }

private:
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
    }
    T* p_ = nullptr;
    size_t n_ = 0;
};

using ScalarVector = DeviceArray<double>;
using OrdinalVector = DeviceArray<int32_t>;

// Block CRS matrix (Plato::CrsMatrix, src/alg/CrsMatrix.hpp:20-111).
struct CrsMatrix {
    OrdinalVector rowMap;
    OrdinalVector columnIndices;
    ScalarVector entries;
    int32_t numRowsPerBlock = 3;
    int32_t numColsPerBlock = 3;
};

// Owns the plato_problem handle: mesh, material, penalty, BCs and solver options.
class Model {
public:
    explicit Model(const plato_problem_desc& desc) {
        plato_problem* h = nullptr;
        check(plato_create(&desc, &h), nullptr);
        h_.reset(h);
        check(plato_get_sizes(h, &num_nodes_, &num_cells_, &num_blocks_), h);
    }
    // a Helmholtz density filter over the mesh (one unknown per node)
    explicit Model(const plato_helmholtz_desc& desc) {
        plato_problem* h = nullptr;
        check(plato_create_helmholtz(&desc, &h), nullptr);
        h_.reset(h);
        check(plato_get_sizes(h, &num_nodes_, &num_cells_, &num_blocks_), h);
    }
    plato_problem* handle() const { return h_.get(); }
    int32_t numNodes() const { return num_nodes_; }
    int32_t numCells() const { return num_cells_; }
    int64_t numBlocks() const { return num_blocks_; }

    std::shared_ptr<CrsMatrix> newMatrix(int32_t rows_per_block, int32_t cols_per_block) const {
        auto m = std::make_shared<CrsMatrix>();
        m->rowMap = OrdinalVector(size_t(num_nodes_) + 1);
        m->columnIndices = OrdinalVector(size_t(num_blocks_));
        m->entries = ScalarVector(size_t(num_blocks_) * rows_per_block * cols_per_block);
        m->numRowsPerBlock = rows_per_block;
        m->numColsPerBlock = cols_per_block;
        check(plato_jacobian_pattern(h_.get(), m->rowMap.data(), m->columnIndices.data()), h_.get());
        return m;
    }

private:
    struct Del {
        void operator()(plato_problem* h) const { plato_destroy(h); }
    };
    std::unique_ptr<plato_problem, Del> h_;
    int32_t num_nodes_ = 0, num_cells_ = 0;
    int64_t num_blocks_ = 0;
};

namespace Elliptic {

// Plato::Elliptic::VectorFunction<Mechanics<3>> (elastostatic residual R = K(z) u - F).
class VectorFunction {
public:
    explicit VectorFunction(std::shared_ptr<Model> m) : m_(std::move(m)) {}
    int32_t size() const { return 3 * m_->numNodes(); }

    ScalarVector value(const ScalarVector& u, const ScalarVector& z) const {
        ScalarVector R(size());
        check(plato_vf_value(m_->handle(), u.data(), z.data(), R.data()), m_->handle());
        return R;
    }
    std::shared_ptr<CrsMatrix> gradient_u(const ScalarVector& u, const ScalarVector& z) const {
        auto J = m_->newMatrix(3, 3);
        check(plato_vf_gradient_u(m_->handle(), u.data(), z.data(), J->entries.data()), m_->handle());
        return J;
    }
    std::shared_ptr<CrsMatrix> gradient_u_T(const ScalarVector& u, const ScalarVector& z) const {
        auto J = m_->newMatrix(3, 3);
        check(plato_vf_gradient_u_T(m_->handle(), u.data(), z.data(), J->entries.data()), m_->handle());
        return J;
    }
    // (dR/dz)^T, num_nodes x 3 num_nodes with 1x3 blocks
    std::shared_ptr<CrsMatrix> gradient_z(const ScalarVector& u, const ScalarVector& z) const {
        auto G = m_->newMatrix(1, 3);
        check(plato_vf_gradient_z(m_->handle(), u.data(), z.data(), G->entries.data()), m_->handle());
        return G;
    }

private:
    std::shared_ptr<Model> m_;
};

// Plato::Elliptic::PhysicsScalarFunction with "Internal Elastic Energy".
class PhysicsScalarFunction {
public:
    explicit PhysicsScalarFunction(std::shared_ptr<Model> m) : m_(std::move(m)) {}
    std::string name() const { return "Internal Elastic Energy"; }
    double value(const ScalarVector& u, const ScalarVector& z) const {
        double v = 0.0;
        check(plato_sf_value(m_->handle(), u.data(), z.data(), &v), m_->handle());
        return v;
    }
    ScalarVector gradient_u(const ScalarVector& u, const ScalarVector& z) const {
        ScalarVector g(size_t(3) * m_->numNodes());
        check(plato_sf_gradient_u(m_->handle(), u.data(), z.data(), g.data()), m_->handle());
        return g;
    }
    ScalarVector gradient_z(const ScalarVector& u, const ScalarVector& z) const {
        ScalarVector g(size_t(m_->numNodes()));
        check(plato_sf_gradient_z(m_->handle(), u.data(), z.data(), g.data()), m_->handle());
        return g;
    }

private:
    std::shared_ptr<Model> m_;
};

}  // namespace Elliptic

// Plato::AbstractSolver::solve on a constrained 3x3 block matrix.
class Solver {
public:
    explicit Solver(std::shared_ptr<Model> m) : m_(std::move(m)) {}
    plato_solve_stats solve(const CrsMatrix& A, ScalarVector& x, const ScalarVector& b) const {
        plato_solve_stats st{};
        check(plato_solver_solve(m_->handle(), A.entries.data(), x.data(), b.data(), &st), m_->handle());
        return st;
    }

private:
    std::shared_ptr<Model> m_;
};

inline void applyBlockConstraints(const Model& m, CrsMatrix& A, ScalarVector& rhs, double scale) {
    check(plato_apply_constraints(m.handle(), A.entries.data(), rhs.data(), scale), m.handle());
}

inline void MatrixTimesVectorPlusVector(const Model& m, const CrsMatrix& A, const ScalarVector& x,
                                        ScalarVector& y) {
    check(plato_matvec_plus(m.handle(), A.numRowsPerBlock, A.numColsPerBlock, A.entries.data(), x.data(),
                            y.data()),
          m.handle());
}

namespace Elliptic {

// Plato::Elliptic::Problem with the compliance criterion.
class Problem {
public:
    explicit Problem(std::shared_ptr<Model> m) : m_(std::move(m)), state_(size_t(3) * m_->numNodes()) {}

    const ScalarVector& solution(const ScalarVector& z) {
        check(plato_problem_solution(m_->handle(), z.data(), nullptr, state_.data(), &last_), m_->handle());
        return state_;
    }
    double criterionValue(const ScalarVector& z) const {
        double v = 0.0;
        check(plato_problem_criterion_value(m_->handle(), z.data(), state_.data(), &v), m_->handle());
        return v;
    }
    ScalarVector criterionGradient(const ScalarVector& z) {
        ScalarVector g(size_t(m_->numNodes()));
        plato_solve_stats st{};
        check(plato_problem_criterion_gradient(m_->handle(), z.data(), state_.data(), g.data(), &st), m_->handle());
        return g;
    }
    const plato_solve_stats& lastSolveStats() const { return last_; }

private:
    std::shared_ptr<Model> m_;
    ScalarVector state_;
    plato_solve_stats last_{};
};

}  // namespace Elliptic

namespace Helmholtz {

// Plato::Helmholtz::VectorFunction (src/helmholtz/VectorFunction.hpp) on a filter Model.
class VectorFunction {
public:
    explicit VectorFunction(std::shared_ptr<Model> m) : m_(std::move(m)) {}
    ScalarVector value(const ScalarVector& filtered, const ScalarVector& control) const {
        ScalarVector R(size_t(m_->numNodes()));
        check(plato_helmholtz_value(m_->handle(), filtered.data(), control.data(), R.data()), m_->handle());
        return R;
    }
    std::shared_ptr<CrsMatrix> gradient_u(const ScalarVector&, const ScalarVector&) const {
        auto A = m_->newMatrix(1, 1);
        check(plato_helmholtz_gradient_u(m_->handle(), A->entries.data()), m_->handle());
        return A;
    }
    std::shared_ptr<CrsMatrix> gradient_z(const ScalarVector&, const ScalarVector&) const {
        auto A = m_->newMatrix(1, 1);
        check(plato_helmholtz_gradient_z(m_->handle(), A->entries.data()), m_->handle());
        return A;
    }

private:
    std::shared_ptr<Model> m_;
};

// Plato::Helmholtz::Problem (src/helmholtz/Problem.hpp:158-208).
class Problem {
public:
    explicit Problem(std::shared_ptr<Model> m) : m_(std::move(m)), state_(size_t(m_->numNodes())) {}

    const ScalarVector& solution(const ScalarVector& control) {
        check(plato_helmholtz_solution(m_->handle(), control.data(), state_.data(), &last_), m_->handle());
        return state_;
    }
    // the reference negates its argument in place; this one leaves it unchanged
    ScalarVector criterionGradient(const ScalarVector& dfdfiltered) {
        ScalarVector g(size_t(m_->numNodes()));
        check(plato_helmholtz_criterion_gradient(m_->handle(), dfdfiltered.data(), g.data(), &last_), m_->handle());
        return g;
    }
    const plato_solve_stats& lastSolveStats() const { return last_; }

private:
    std::shared_ptr<Model> m_;
    ScalarVector state_;
    plato_solve_stats last_{};
};

}  // namespace Helmholtz
}  // namespace plato_b200
