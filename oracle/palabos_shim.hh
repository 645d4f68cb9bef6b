// palabos_shim.hh -- minimal multi-cell stand-ins for the few Palabos types and calls that the
// reference's precipitation / dissolution processors use (a lattice of D3Q7 cells addressed by
// (x, y, z), a cell's density and populations, processing-functional base classes). TEST
// INFRASTRUCTURE ONLY: it lets the reference's own processor headers be compiled and run on small
// fields so the oracle's restatement can be checked against them.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

namespace plb {
typedef long plint;
struct Box3D {
    plint x0, x1, y0, y1, z0, z1;
};
struct Dot3D {
    plint x, y, z;
};
template <typename T, int N>
struct Array {
    T v[N];
    T& operator[](int i) { return v[i]; }
    const T& operator[](int i) const { return v[i]; }
};
namespace util {
inline plint roundToInt(double x) { return (plint)(x < 0 ? x - 0.5 : x + 0.5); }
}  // namespace util
namespace BlockDomain {
enum DomainT { bulk, bulkAndEnvelope };
}
namespace modif {
enum ModifT { nothing, staticVariables, dynamicVariables, allVariables, dataStructure };
}
template <typename T>
struct D3Q7Descriptor {};

// a D3Q7 cell storing shifted populations (f_i - t_i): its density is their sum plus one
template <typename T, template <typename U> class Descriptor>
struct Cell {
    Array<T, 7> f;
    T computeDensity() const {
        T s = 0;
        for (int i = 0; i < 7; ++i) s += f[i];
        return s + (T)1;
    }
    void getPopulations(Array<T, 7>& g) const { g = f; }
    void setPopulations(const Array<T, 7>& g) { f = g; }
    // the populations of a cell at rest with density rho
    void setDensity(T rho) {
        f[0] = (rho - 1) / 4;
        for (int i = 1; i < 7; ++i) f[i] = (rho - 1) / 8;
    }
};

// dynamics objects: only declared so that processors which switch dynamics compile; the shim's
// lattices never run them
template <typename T, template <typename U> class Descriptor>
struct Dynamics {
    virtual ~Dynamics() {}
    virtual T getOmega() const { return omega; }
    T omega = 0;
};
template <typename T, template <typename U> class Descriptor>
struct BounceBack : Dynamics<T, Descriptor> {
    BounceBack() {}
};
template <typename T, template <typename U> class Descriptor>
struct AdvectionDiffusionBGKdynamics : Dynamics<T, Descriptor> {
    explicit AdvectionDiffusionBGKdynamics(T w) { this->omega = w; }
};
template <typename T, template <typename U> class Descriptor>
struct IncBGKdynamics : Dynamics<T, Descriptor> {
    explicit IncBGKdynamics(T w) { this->omega = w; }
};

template <typename T, template <typename U> class Descriptor>
struct BlockLattice3D {
    plint nx, ny, nz;
    std::vector<Cell<T, Descriptor>> cells;
    BlockLattice3D(plint nx_, plint ny_, plint nz_) : nx(nx_), ny(ny_), nz(nz_), cells((size_t)(nx_ * ny_ * nz_)) {}
    Cell<T, Descriptor>& get(plint x, plint y, plint z) { return cells[(size_t)((x * ny + y) * nz + z)]; }
    Dot3D getLocation() const { return Dot3D{0, 0, 0}; }
};

template <typename T, template <typename U> class Descriptor>
inline Dot3D computeRelativeDisplacement(const BlockLattice3D<T, Descriptor>&, const BlockLattice3D<T, Descriptor>&) {
    return Dot3D{0, 0, 0};
}

template <typename T>
struct ScalarField3D {
    plint nx, ny, nz;
    std::vector<T> v;
    T& get(plint x, plint y, plint z) { return v[(size_t)((x * ny + y) * nz + z)]; }
};

template <typename T, template <typename U> class Descriptor>
struct LatticeBoxProcessingFunctional3D {
    virtual ~LatticeBoxProcessingFunctional3D() {}
    virtual void process(Box3D, std::vector<BlockLattice3D<T, Descriptor>*>) = 0;
};

template <typename T1, template <typename U> class D1, typename T2, template <typename U> class D2>
struct BoxProcessingFunctional3D_LL {
    virtual ~BoxProcessingFunctional3D_LL() {}
};

template <typename T1, template <typename U> class Descriptor, typename T2>
struct BoxProcessingFunctional3D_LS {
    virtual ~BoxProcessingFunctional3D_LS() {}
    virtual void process(Box3D, BlockLattice3D<T1, Descriptor>&, ScalarField3D<T2>&) = 0;
};
}  // namespace plb
