// model.hpp -- host-side lattice and Hamiltonian tables.
//
// Mirrors the reference's lattice::bravais / lattice::honeycomb /
// lattice::toric_lattice and model::kitaev / model::toric (dbucher97/rbm-nqs,
// include/lattice/*.hpp, include/model/*.hpp).  Everything here is host
// precompute: the tables are uploaded once to the GPU.
#pragma once

#include <complex>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace rbmnqs {

using cplx = std::complex<double>;

struct bond {
    int a, b, type;
};

// lattice::bravais (src/lattice/bravais.cpp): unit-cell index arithmetic with
// periodic boundaries, unsigned arithmetic as in the reference.
class bravais {
   public:
    uint64_t n_uc, n_dim, n_basis, n_coordination, n_total_uc, n_total, n_uc_b, h_shift;

    bravais(uint64_t n_uc, uint64_t n_dim, uint64_t n_basis, uint64_t n_coord,
            uint64_t n_uc_b = 0, uint64_t h_shift = 0);
    virtual ~bravais() = default;

    uint64_t idx(uint64_t uc, uint64_t b) const { return uc * n_basis + b; }
    uint64_t uc_idx(uint64_t i) const { return i / n_basis; }
    uint64_t b_idx(uint64_t i) const { return i % n_basis; }
    uint64_t up(uint64_t uc, uint64_t dir = 0, uint64_t step = 1) const;
    uint64_t down(uint64_t uc, uint64_t dir = 0, uint64_t step = 1) const;

    virtual std::vector<int> nns(int site) const = 0;
    const std::vector<bond>& bonds() const { return bonds_; }

    // Symmetry permutations perm[s][i] = P_s(i) and symmetry basis for a
    // single symmetry value (0 = none).
    virtual std::vector<std::vector<int>> symmetry(double symm) const;
    virtual std::vector<int> symmetry_basis(double symm) const;

   protected:
    std::vector<bond> bonds_;
    void clean_symm(double s, uint64_t x[2]) const;
    std::vector<std::vector<uint64_t>> uc_symmetry(double s) const;
};

// lattice::honeycomb (src/lattice/honeycomb.cpp)
class honeycomb : public bravais {
   public:
    honeycomb(int n_uc, int n_uc_b = -1);
    std::vector<int> nns(int site) const override;
    std::vector<std::vector<int>> symmetry(double symm) const override;
    std::vector<int> symmetry_basis(double symm) const override;
    std::vector<std::vector<int>> hexagons() const;
};

// lattice::toric_lattice (src/lattice/toric_lattice.cpp)
class toric_lattice : public bravais {
   public:
    explicit toric_lattice(int n_uc);
    std::vector<int> nns(int site) const override;
    struct plaq {
        int idxs[4];
        int type;  // 0 plaquette, 1 star
    };
    std::vector<plaq> plaqs() const;
};

// operators::local_op as data: k sites and the dense 2^k x 2^k matrix.
struct local_op {
    int k;
    int acts_on[6];
    std::vector<cplx> mat;  // row-major
};

// model::abstract_model as data: lattice + Hamiltonian operator chain.
struct model {
    std::string kind;  // "kitaev" | "toric"
    int n_cells = 0, n_cells_b = -1;
    double symmetry = 0;
    std::vector<local_op> hamiltonian;
    std::vector<local_op> observables;  // hexagon plaquettes (evaluation)
    std::vector<bond> bonds;
    std::vector<std::vector<int>> perm;  // [S][n]
    std::vector<int> basis;
    int n = 0;
    const bravais* lat() const { return lattice_.get(); }
    std::shared_ptr<bravais> lattice_;
};

model make_kitaev(int n_cells, int n_cells_b, const double J[3], double h, double symmetry);
model make_toric(int n_cells, double J, double symmetry);
void add_hexagons(model& m);

// Pauli-string operator: kron of sigma^which[i] on bit i (first factor on the
// least-significant bit, abstract_model.cpp:28-33), scaled.
local_op pauli_string(const std::vector<int>& sites, const std::vector<int>& which, cplx scale);

// Pfaffian independent-parameter index matrix (pfaffian.cpp:31-85).
std::vector<int> pfaffian_index_matrix(int n, const std::vector<std::vector<int>>& perm,
                                       const std::vector<int>& basis, int* n_indep);

}  // namespace rbmnqs
