// model.cpp -- lattice and Hamiltonian tables (see model.hpp).
#include "model.hpp"

#include <cmath>
#include <cstdlib>
#include <memory>
#include <stdexcept>

namespace rbmnqs {

static uint64_t upow(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    for (uint64_t i = 0; i < e; i++) r *= b;
    return r;
}

// bravais.cpp:28-42
bravais::bravais(uint64_t n_uc_, uint64_t n_dim_, uint64_t n_basis_, uint64_t n_coord,
                 uint64_t n_uc_b_, uint64_t h_shift_)
    : n_uc{n_uc_},
      n_dim{n_dim_},
      n_basis{n_basis_},
      n_coordination{n_coord},
      n_total_uc{n_uc_b_ == 0 ? upow(n_uc_, n_dim_) : n_uc_ * n_uc_b_},
      n_total{0},
      n_uc_b{n_uc_b_ == 0 ? n_uc_ : n_uc_b_},
      h_shift{h_shift_} {
    n_total = n_total_uc * n_basis;
}

// bravais::up (bravais.cpp:66-85): the wrap flag drives the optional
// horizontal shift of the second direction.
uint64_t bravais::up(uint64_t uc, uint64_t dir, uint64_t step) const {
    if (step == 0) return uc;
    const uint64_t span = upow(n_uc, dir) * n_uc_b;
    const uint64_t len = dir == 0 ? n_uc_b : n_uc;
    const uint64_t block = uc / span;
    const bool wrapped = (uc + (step * span) / len) / span != 0;
    step %= len;
    uint64_t r = span * block + (uc + step * span / len) % span;
    if (wrapped && h_shift && dir == 1) r = down(r, 0, h_shift);
    return r;
}

// bravais::down (bravais.cpp:86-105)
uint64_t bravais::down(uint64_t uc, uint64_t dir, uint64_t step) const {
    if (step == 0) return uc;
    const uint64_t span = upow(n_uc, dir) * n_uc_b;
    const uint64_t len = dir == 0 ? n_uc_b : n_uc;
    const uint64_t block = uc / span;
    const bool wrapped = (uc + (len - step) * span / len) / span != 0;
    step %= len;
    uint64_t r = span * block + (uc + (len - step) * span / len) % span;
    if (!wrapped && h_shift && dir == 1) r = up(r, 0, h_shift);
    return r;
}

// bravais::clean_symms for one symmetry value (bravais.cpp:249-284)
void bravais::clean_symm(double s, uint64_t x[2]) const {
    if (s < 0) throw std::runtime_error("Negative Symmetry factors are not allowed!");
    int factor = 1;
    if (std::abs(factor * s - int(factor * s)) > 1e-14) {
        double r = factor * s - std::floor(factor * s);
        factor *= (int)(1 / r);
    }
    x[0] = (uint64_t)(int)(factor * s);
    if (x[0] == 0) x[0] = n_uc_b;
    if (n_uc_b % x[0] != 0) throw std::runtime_error("Symmetry factor invalid!");
    x[1] = x[0];
}

// bravais::construct_uc_symmetry (bravais.cpp:119-158)
std::vector<std::vector<uint64_t>> bravais::uc_symmetry(double s) const {
    uint64_t x[2];
    clean_symm(s, x);
    std::vector<std::vector<uint64_t>> out;
    for (uint64_t i1 = 0; i1 < n_uc; i1 += x[1])
        for (uint64_t i0 = 0; i0 < n_uc_b; i0 += x[0]) {
            std::vector<uint64_t> t(n_total_uc);
            for (uint64_t u = 0; u < n_total_uc; u++) t[u] = up(up(u, 0, i0), 1, i1);
            out.push_back(std::move(t));
        }
    return out;
}

// bravais::construct_symmetry (bravais.cpp:160-197)
std::vector<std::vector<int>> bravais::symmetry(double symm) const {
    std::vector<std::vector<int>> out;
    if (symm == 0) {
        std::vector<int> id(n_total);
        for (uint64_t i = 0; i < n_total; i++) id[i] = (int)i;
        out.push_back(id);
        return out;
    }
    for (auto& ucs : uc_symmetry(symm)) {
        std::vector<int> p(n_total);
        for (uint64_t i = 0; i < n_total; i++) p[i] = (int)idx(ucs[uc_idx(i)], b_idx(i));
        out.push_back(std::move(p));
    }
    return out;
}

// bravais::construct_symm_basis (bravais.cpp:199-232)
std::vector<int> bravais::symmetry_basis(double symm) const {
    std::vector<int> out;
    if (symm == 0) {
        for (uint64_t i = 0; i < n_total; i++) out.push_back((int)i);
        return out;
    }
    uint64_t x[2];
    clean_symm(symm, x);
    for (uint64_t i1 = 0; i1 < x[1]; i1++)
        for (uint64_t i0 = 0; i0 < x[0]; i0++) {
            uint64_t uc = up(up(0, 1, i1), 0, i0);
            for (uint64_t b = 0; b < n_basis; b++) out.push_back((int)idx(uc, b));
        }
    return out;
}

// ------------------------------------------------------------ honeycomb --
honeycomb::honeycomb(int n_uc_, int n_uc_b_)
    : bravais((uint64_t)n_uc_, 2, 2, 3, n_uc_b_ < 0 ? (uint64_t)n_uc_ : (uint64_t)n_uc_b_, 0) {
    // honeycomb::construct_bonds (honeycomb.cpp:47-55): x, y, z bonds of
    // every basis-0 site
    for (uint64_t u = 0; u < n_total_uc; u++) {
        auto nn = nns((int)idx(u, 0));
        for (int c = 0; c < 3; c++) bonds_.push_back({(int)idx(u, 0), nn[c], c});
    }
}

// honeycomb::nns (honeycomb.cpp:35-45), order x, y, z
std::vector<int> honeycomb::nns(int site) const {
    uint64_t uc = uc_idx(site);
    if (b_idx(site) == 0)
        return {(int)idx(uc, 1), (int)idx(down(uc), 1), (int)idx(down(uc, 1), 1)};
    return {(int)idx(uc, 0), (int)idx(up(uc), 0), (int)idx(up(uc, 1), 0)};
}

// honeycomb::construct_symmetry for symmetry 0.5 (honeycomb.cpp:69-134):
// every translation followed by its 180-degree rotation.
std::vector<std::vector<int>> honeycomb::symmetry(double symm) const {
    if (symm != 0.5) return bravais::symmetry(symm);
    std::vector<std::vector<int>> out;
    for (auto& ucs : uc_symmetry(symm)) {
        std::vector<int> t(n_total), r(n_total);
        for (uint64_t i = 0; i < n_total; i++) {
            uint64_t j = idx(ucs[uc_idx(i)], b_idx(i));
            t[i] = (int)j;
            r[i] = (int)(n_total - 1 - j);
        }
        out.push_back(std::move(t));
        out.push_back(std::move(r));
    }
    return out;
}

std::vector<int> honeycomb::symmetry_basis(double symm) const {
    if (symm == 0.5) return {0};
    return bravais::symmetry_basis(symm);
}

// honeycomb::get_hexagons (honeycomb.cpp:201-209)
std::vector<std::vector<int>> honeycomb::hexagons() const {
    std::vector<std::vector<int>> out;
    for (uint64_t uc = 0; uc < n_total_uc; uc++) {
        uint64_t r = up(uc), rd = down(r, 1);
        out.push_back({(int)idx(down(uc, 1), 1), (int)idx(uc, 0), (int)idx(uc, 1), (int)idx(r, 0),
                       (int)idx(rd, 1), (int)idx(rd, 0)});
    }
    return out;
}

// --------------------------------------------------------- toric lattice --
toric_lattice::toric_lattice(int n_uc_) : bravais((uint64_t)n_uc_, 2, 2, 4) {
    for (uint64_t u = 0; u < n_total_uc; u++) {
        auto nn = nns((int)idx(u, 0));
        for (int c = 0; c < 4; c++) bonds_.push_back({(int)idx(u, 0), nn[c], c});
    }
}

// toric_lattice::nns (toric_lattice.cpp:33-44)
std::vector<int> toric_lattice::nns(int site) const {
    uint64_t uc = uc_idx(site);
    if (b_idx(site) == 0)
        return {(int)idx(uc, 1), (int)idx(up(uc), 1), (int)idx(down(uc, 1), 1), (int)idx(up(down(uc, 1)), 1)};
    return {(int)idx(uc, 0), (int)idx(down(uc), 0), (int)idx(up(uc, 1), 0), (int)idx(down(up(uc, 1)), 0)};
}

// toric_lattice::construct_plaqs (toric_lattice.cpp:57-69)
std::vector<toric_lattice::plaq> toric_lattice::plaqs() const {
    std::vector<plaq> out;
    for (uint64_t uc = 0; uc < n_total_uc; uc++) {
        out.push_back({{(int)idx(uc, 0), (int)idx(uc, 1), (int)idx(up(uc, 1), 0), (int)idx(up(uc), 1)}, 0});
        out.push_back({{(int)idx(uc, 0), (int)idx(uc, 1), (int)idx(down(uc), 0), (int)idx(down(uc, 1), 1)}, 1});
    }
    return out;
}

// ---------------------------------------------------------------- models --
static const cplx kPauli[4][2][2] = {
    {{1, 0}, {0, 1}},
    {{0, 1}, {1, 0}},
    {{0, cplx(0, -1)}, {cplx(0, 1), 0}},
    {{1, 0}, {0, -1}},
};

local_op pauli_string(const std::vector<int>& sites, const std::vector<int>& which, cplx scale) {
    local_op op;
    op.k = (int)sites.size();
    for (int i = 0; i < 6; i++) op.acts_on[i] = i < op.k ? sites[i] : -1;
    const int d = 1 << op.k;
    op.mat.assign((size_t)d * d, 0);
    for (int r = 0; r < d; r++)
        for (int c = 0; c < d; c++) {
            cplx v = scale;
            for (int i = 0; i < op.k; i++) v *= kPauli[which[i]][(r >> i) & 1][(c >> i) & 1];
            op.mat[(size_t)r * d + c] = v;
        }
    return op;
}

// model::kitaev (kitaev.cpp:29-50)
model make_kitaev(int n_cells, int n_cells_b, const double J[3], double h, double symmetry) {
    model m;
    m.kind = "kitaev";
    m.n_cells = n_cells;
    m.n_cells_b = n_cells_b;
    m.symmetry = symmetry;
    auto lat = std::make_shared<honeycomb>(n_cells, n_cells_b);
    m.n = (int)lat->n_total;
    m.bonds = lat->bonds();
    for (auto& b : m.bonds) m.hamiltonian.push_back(pauli_string({b.a, b.b}, {b.type + 1, b.type + 1}, J[b.type]));
    if (std::abs(h) > 1e-10) {
        for (int i = 0; i < m.n; i++) {
            local_op op;
            op.k = 1;
            for (int q = 0; q < 6; q++) op.acts_on[q] = q == 0 ? i : -1;
            op.mat.resize(4);
            for (int r = 0; r < 2; r++)
                for (int c = 0; c < 2; c++) op.mat[r * 2 + c] = -h * kPauli[1][r][c] + h * kPauli[2][r][c] + h * kPauli[3][r][c];
            m.hamiltonian.push_back(op);
        }
    }
    m.perm = lat->symmetry(symmetry);
    m.basis = lat->symmetry_basis(symmetry);
    m.lattice_ = lat;
    return m;
}

// model::toric (toric.cpp:27-47): plaquettes J sz^4, stars J sx^4
model make_toric(int n_cells, double J, double symmetry) {
    model m;
    m.kind = "toric";
    m.n_cells = n_cells;
    m.symmetry = symmetry;
    auto lat = std::make_shared<toric_lattice>(n_cells);
    m.n = (int)lat->n_total;
    m.bonds = lat->bonds();
    for (auto& p : lat->plaqs()) {
        int w = p.type == 0 ? 3 : 1;
        m.hamiltonian.push_back(pauli_string({p.idxs[0], p.idxs[1], p.idxs[2], p.idxs[3]}, {w, w, w, w}, J));
    }
    m.perm = lat->symmetry(symmetry);
    m.basis = lat->symmetry_basis(symmetry);
    m.lattice_ = lat;
    return m;
}

// Hexagon plaquette observables W_p (main.cpp:645-671)
void add_hexagons(model& m) {
    auto hc = dynamic_cast<const honeycomb*>(m.lat());
    if (!hc) throw std::runtime_error("hexagon observables need a honeycomb lattice");
    for (auto& hx : hc->hexagons()) m.observables.push_back(pauli_string(hx, {1, 2, 3, 1, 2, 3}, 1.0));
}

// pfaffian::pfaffian index matrix (pfaffian.cpp:31-85); row-major bs[i*n+j].
std::vector<int> pfaffian_index_matrix(int n, const std::vector<std::vector<int>>& perm,
                                       const std::vector<int>& basis, int* n_indep) {
    std::vector<int> bs((size_t)n * n, 0);
    int offset = 0;
    for (int bi : basis) {
        for (auto& p : perm) {
            const int f = p[0] > p[1] ? -1 : 1;  // mirrored symmetry element
            for (int j = 0; j < n; j++) {
                int a = p[bi], b = p[j];
                bs[(size_t)b * n + a] = (a == b) ? 0 : f * (j + offset);
            }
        }
        offset += n;
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++) {
            int& lo = bs[(size_t)i * n + j];
            int& hi = bs[(size_t)j * n + i];
            if (std::abs(lo) <= std::abs(hi))
                hi = -lo;
            else
                lo = -hi;
        }
    auto maxv = [&]() {
        int mx = 0;
        for (int v : bs) mx = v > mx ? v : mx;
        return mx;
    };
    // close the gaps in the index set, smallest first
    for (int i = 1; i < maxv(); i++) {
        for (;;) {
            bool present = false;
            for (int v : bs) present |= v == i;
            if (present) break;
            for (int& v : bs) {
                if (v > i)
                    v -= 1;
                else if (v < -i)
                    v += 1;
            }
        }
    }
    *n_indep = maxv();
    return bs;
}

}  // namespace rbmnqs
