// Minimal stand-ins for the deal.II and Trilinos types that the reference's
// headers (src/pfem2particlehandler.h, pfem2solver.h, pfem2fem.h,
// pfem2parameterhandler.h, pfem2particle.h) and the B200 adapter
// (pfem2dealii_b200/dealii/pfem2particlehandler_b200.cpp) name.  Test
// infrastructure: just enough declarations for g++ to compile the adapter
// against the unchanged reference headers; no numerics.
#pragma once

#include <array>
#include <cstddef>
#include <fstream>
#include <iostream>
#include <map>
#include <set>
#include <string>
#include <utility>
#include <vector>

using MPI_Comm = int;

namespace dealii {

namespace types {
using global_dof_index = unsigned int;
using subdomain_id = unsigned int;
}  // namespace types

template <int rank, int dim, typename Number = double>
class Tensor {
public:
    Tensor() : v_{} {}
    Number& operator[](unsigned int i) { return v_[i]; }
    const Number& operator[](unsigned int i) const { return v_[i]; }
    Tensor& operator=(const Number& x)
    {
        for (auto& e : v_) e = x;
        return *this;
    }
    Tensor& operator+=(const Tensor& o)
    {
        for (int i = 0; i < dim; ++i) v_[i] += o.v_[i];
        return *this;
    }

private:
    std::array<Number, dim> v_;
};

template <int dim, typename Number = double>
class Point : public Tensor<1, dim, Number> {
public:
    Point() = default;
};

template <int dim>
struct GeometryInfo {
    static constexpr unsigned int vertices_per_cell = 1u << dim;
    static constexpr unsigned int faces_per_cell = 2 * dim;
};

class ConditionalOStream {};

class TimerOutput {
public:
    class Scope {
    public:
        Scope(TimerOutput&, const std::string&) {}
    };
};

class IndexSet {};

namespace VectorOperation {
enum values { unknown, insert, add };
}

template <int dim, int spacedim = dim>
class Mapping {};
template <int dim, int spacedim = dim>
class MappingQ1 : public Mapping<dim, spacedim> {};

template <int dim, int spacedim = dim>
class FE_Q {
public:
    double shape_value(unsigned int, const Point<dim>&) const { return 0.0; }
};
template <int dim, int spacedim = dim>
class FEValues {};
template <int dim, int spacedim = dim>
class FEFaceValues {};
template <int dim>
class QGauss {};

// A cell as a DoFHandler's active iterator dereferences to.
template <int dim>
class CellAccessor {
public:
    Point<dim> vertex(unsigned int) const { return Point<dim>(); }
    unsigned int vertex_index(unsigned int) const { return 0; }
    types::global_dof_index vertex_dof_index(unsigned int, unsigned int) const { return 0; }
    bool is_locally_owned() const { return true; }
    unsigned int active_cell_index() const { return 0; }
    int index() const { return 0; }
    int level() const { return 0; }
};

template <int dim>
class CellIterator {
public:
    const CellAccessor<dim>* operator->() const { return &a_; }
    const CellAccessor<dim>& operator*() const { return a_; }
    CellIterator& operator++() { return *this; }
    bool operator!=(const CellIterator&) const { return false; }
    bool operator==(const CellIterator&) const { return true; }
    bool operator<(const CellIterator&) const { return false; }

private:
    CellAccessor<dim> a_;
};

// deal.II's ranges iterate over iterators: `for (const auto& cell : range)`
// gives cell iterators.
template <typename It>
class IteratorRange {
public:
    class IteratorOverIterators {
    public:
        const It& operator*() const { return it_; }
        IteratorOverIterators& operator++()
        {
            ++it_;
            return *this;
        }
        bool operator!=(const IteratorOverIterators& o) const { return it_ != o.it_; }

    private:
        It it_;
    };
    IteratorOverIterators begin() const { return {}; }
    IteratorOverIterators end() const { return {}; }
};

template <int dim, int spacedim = dim>
class Triangulation {
public:
    using cell_iterator = CellIterator<dim>;
    using active_cell_iterator = CellIterator<dim>;
    unsigned int n_active_cells() const { return 0; }
    unsigned int n_vertices() const { return 0; }
    types::subdomain_id locally_owned_subdomain() const { return 0; }
    IteratorRange<active_cell_iterator> active_cell_iterators() const { return {}; }
};

namespace parallel {
namespace distributed {
template <int dim, int spacedim = dim>
class Triangulation : public dealii::Triangulation<dim, spacedim> {};
}  // namespace distributed
}  // namespace parallel

template <int dim, int spacedim = dim>
class DoFHandler {
public:
    using cell_iterator = CellIterator<dim>;
    using active_cell_iterator = CellIterator<dim>;
    IteratorRange<active_cell_iterator> active_cell_iterators() const { return {}; }
    types::global_dof_index n_dofs() const { return 0; }
};

template <typename Number = double>
class Vector {};
template <typename Number = double>
class FullMatrix {};
template <typename Number = double>
class AffineConstraints {};
class SolverControl {};

namespace TrilinosWrappers {
class SparseMatrix {};
class SolverBase {};
class PreconditionBase {};
namespace MPI {
class Vector {
public:
    void reinit(const IndexSet&, const MPI_Comm&) {}
    Vector& operator=(double) { return *this; }
    double& operator[](types::global_dof_index) { return x_; }
    double operator[](types::global_dof_index) const { return x_; }
    double operator()(types::global_dof_index) const { return x_; }
    std::pair<types::global_dof_index, types::global_dof_index> local_range() const { return {0, 0}; }
    void compress(VectorOperation::values) {}

private:
    double x_ = 0.0;
};
}  // namespace MPI
}  // namespace TrilinosWrappers

namespace Utilities {
inline std::string int_to_string(unsigned int v, unsigned int digits = 0)
{
    std::string s = std::to_string(v);
    while (s.size() < digits) s = "0" + s;
    return s;
}
namespace MPI {
inline unsigned int this_mpi_process(const MPI_Comm&) { return 0; }
inline unsigned int n_mpi_processes(const MPI_Comm&) { return 1; }
}  // namespace MPI
}  // namespace Utilities

}  // namespace dealii
