/*
 * orc_lattice.c -- oracle restatement of the reference's lattice and model
 * tables (TEST INFRASTRUCTURE ONLY; see orc.h).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "orc.h"

/* ------------------------------------------------------------- Philox -- */
/* Philox4x32-10 as published by Salmon et al. (SC'11): two 32x32->64
 * multiplies per round, Weyl-sequence key schedule. */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = (uint32_t)p1;
        c2 = n2;
        c3 = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

/* ------------------------------------------------------------ bravais -- */
/* lattice/bravais.cpp:28-42 */
void orc_bravais_init(orc_bravais* l, uint64_t n_uc, uint64_t n_dim,
                      uint64_t n_basis, uint64_t n_coord, uint64_t n_uc_b,
                      uint64_t h_shift) {
    l->n_uc = n_uc;
    l->n_dim = n_dim;
    l->n_basis = n_basis;
    l->n_coord = n_coord;
    uint64_t p = 1;
    for (uint64_t i = 0; i < n_dim; i++) p *= n_uc;
    l->n_total_uc = n_uc_b == 0 ? p : n_uc * n_uc_b;
    l->n_total = l->n_total_uc * n_basis;
    l->n_uc_b = n_uc_b == 0 ? n_uc : n_uc_b;
    l->h_shift = h_shift;
}

static uint64_t ipow(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    while (e--) r *= b;
    return r;
}

/* bravais::up, lattice/bravais.cpp:66-85 (unsigned arithmetic kept) */
uint64_t orc_up(const orc_bravais* l, uint64_t uc, uint64_t dir, uint64_t step) {
    if (step == 0) return uc;
    uint64_t shift = ipow(l->n_uc, dir) * l->n_uc_b;
    uint64_t offset = uc / shift;
    uint64_t n_uc2 = dir == 0 ? l->n_uc_b : l->n_uc;
    uint64_t overflow = (uc + (step * shift) / n_uc2) / shift;
    step %= n_uc2;
    uc = (uc + step * shift / n_uc2) % shift;
    uint64_t ret = shift * offset + uc;
    if (overflow && l->h_shift && dir == 1) ret = orc_down(l, ret, 0, l->h_shift);
    return ret;
}

/* bravais::down, lattice/bravais.cpp:86-105 */
uint64_t orc_down(const orc_bravais* l, uint64_t uc, uint64_t dir, uint64_t step) {
    if (step == 0) return uc;
    uint64_t shift = ipow(l->n_uc, dir) * l->n_uc_b;
    uint64_t offset = uc / shift;
    uint64_t n_uc2 = dir == 0 ? l->n_uc_b : l->n_uc;
    uint64_t overflow = (uc + (n_uc2 - step) * shift / n_uc2) / shift;
    step %= n_uc2;
    uc = (uc + (n_uc2 - step) * shift / n_uc2) % shift;
    uint64_t ret = shift * offset + uc;
    if (!overflow && l->h_shift && dir == 1) ret = orc_up(l, ret, 0, l->h_shift);
    return ret;
}

static void honeycomb_init(orc_bravais* l, int n_uc, int n_uc_b) {
    /* honeycomb.cpp:28-33: 2 dims, 2 basis sites, coordination 3 */
    orc_bravais_init(l, n_uc, 2, 2, 3, n_uc_b < 0 ? (uint64_t)n_uc : (uint64_t)n_uc_b, 0);
}

#define IDX(l, uc, b) ((uc) * (l)->n_basis + (b))

/* honeycomb::nns, honeycomb.cpp:35-45 -- order x, y, z bond */
void orc_honeycomb_nns(int n_uc, int n_uc_b, int site, int out[3]) {
    orc_bravais l;
    honeycomb_init(&l, n_uc, n_uc_b);
    uint64_t uc = site / l.n_basis;
    if (site % l.n_basis == 0) {
        out[0] = (int)IDX(&l, uc, 1);
        out[1] = (int)IDX(&l, orc_down(&l, uc, 0, 1), 1);
        out[2] = (int)IDX(&l, orc_down(&l, uc, 1, 1), 1);
    } else {
        out[0] = (int)IDX(&l, uc, 0);
        out[1] = (int)IDX(&l, orc_up(&l, uc, 0, 1), 0);
        out[2] = (int)IDX(&l, orc_up(&l, uc, 1, 1), 0);
    }
}

/* honeycomb::construct_bonds, honeycomb.cpp:47-55 */
int orc_honeycomb_bonds(int n_uc, int n_uc_b, int* out_abt) {
    orc_bravais l;
    honeycomb_init(&l, n_uc, n_uc_b);
    int c = 0;
    for (uint64_t i = 0; i < l.n_total_uc; i++) {
        int nn[3];
        orc_honeycomb_nns(n_uc, n_uc_b, (int)IDX(&l, i, 0), nn);
        for (int t = 0; t < 3; t++) {
            out_abt[3 * c + 0] = (int)IDX(&l, i, 0);
            out_abt[3 * c + 1] = nn[t];
            out_abt[3 * c + 2] = t;
            c++;
        }
    }
    return c;
}

/* honeycomb::get_hexagons, honeycomb.cpp:201-209 */
int orc_honeycomb_hexagons(int n_uc, int n_uc_b, int* out6) {
    orc_bravais l;
    honeycomb_init(&l, n_uc, n_uc_b);
    for (uint64_t uc = 0; uc < l.n_total_uc; uc++) {
        uint64_t u = orc_up(&l, uc, 0, 1);
        uint64_t du = orc_down(&l, u, 1, 1);
        int* h = out6 + 6 * uc;
        h[0] = (int)IDX(&l, orc_down(&l, uc, 1, 1), 1);
        h[1] = (int)IDX(&l, uc, 0);
        h[2] = (int)IDX(&l, uc, 1);
        h[3] = (int)IDX(&l, u, 0);
        h[4] = (int)IDX(&l, du, 1);
        h[5] = (int)IDX(&l, du, 0);
    }
    return (int)l.n_total_uc;
}

/* toric_lattice::construct_plaqs, toric_lattice.cpp:57-69 */
int orc_toric_plaqs(int n_uc, int* out5) {
    orc_bravais l;
    orc_bravais_init(&l, n_uc, 2, 2, 4, 0, 0);
    int c = 0;
    for (uint64_t uc = 0; uc < l.n_total_uc; uc++) {
        int* p = out5 + 5 * c++;
        p[0] = (int)IDX(&l, uc, 0);
        p[1] = (int)IDX(&l, uc, 1);
        p[2] = (int)IDX(&l, orc_up(&l, uc, 1, 1), 0);
        p[3] = (int)IDX(&l, orc_up(&l, uc, 0, 1), 1);
        p[4] = 0;
        p = out5 + 5 * c++;
        p[0] = (int)IDX(&l, uc, 0);
        p[1] = (int)IDX(&l, uc, 1);
        p[2] = (int)IDX(&l, orc_down(&l, uc, 0, 1), 0);
        p[3] = (int)IDX(&l, orc_down(&l, uc, 1, 1), 1);
        p[4] = 1;
    }
    return c;
}

/* bravais::clean_symms for a single symmetry value, bravais.cpp:249-284 */
static void clean_symm(const orc_bravais* l, double s, uint64_t x[2]) {
    int factor = 1;
    if (fabs(factor * s - (int)(factor * s)) > 1e-14) {
        double r = factor * s - floor(factor * s);
        factor *= (int)(1 / r);
    }
    x[0] = (uint64_t)(int)(factor * s);
    if (x[0] == 0) x[0] = l->n_uc_b;
    x[1] = x[0];
}

/* bravais::construct_uc_symmetry, bravais.cpp:119-158: translation tables
 * ucs[i][u]; returns their number. */
static int uc_symmetry(const orc_bravais* l, double s, uint64_t* ucs) {
    uint64_t x[2];
    clean_symm(l, s, x);
    int c = 0;
    for (uint64_t i1 = 0; i1 < l->n_uc; i1 += x[1]) {
        for (uint64_t i0 = 0; i0 < l->n_uc_b; i0 += x[0]) {
            for (uint64_t u = 0; u < l->n_total_uc; u++) {
                uint64_t uc = orc_up(l, u, 0, i0);
                uc = orc_up(l, uc, 1, i1);
                ucs[(uint64_t)c * l->n_total_uc + u] = uc;
            }
            c++;
        }
    }
    return c;
}

/* Symmetry permutations and basis.
 * honeycomb 0.5: honeycomb.cpp:69-134 (translations, each followed by its
 *   180-degree rotation, S = n_total, basis {0});
 * otherwise bravais::construct_symmetry / construct_symm_basis,
 *   bravais.cpp:160-247 (translations by the cleaned factor). */
int orc_symmetry(int kind, int n_uc, int n_uc_b, double symm, int* perm,
                 int* basis, int* n_vb) {
    orc_bravais l;
    if (kind == 0)
        honeycomb_init(&l, n_uc, n_uc_b);
    else
        orc_bravais_init(&l, n_uc, 2, 2, 4, 0, 0);
    uint64_t n = l.n_total;
    if (symm == 0) {
        for (uint64_t i = 0; i < n; i++) {
            perm[i] = (int)i;
            basis[i] = (int)i;
        }
        *n_vb = (int)n;
        return 1;
    }
    uint64_t* ucs = (uint64_t*)malloc(sizeof(uint64_t) * l.n_total_uc * l.n_total_uc);
    int nsym = uc_symmetry(&l, symm, ucs);
    int S;
    if (kind == 0 && symm == 0.5) {
        for (uint64_t i = 0; i < l.n_total_uc; i++) {
            for (uint64_t j = 0; j < n; j++) {
                uint64_t t = IDX(&l, ucs[i * l.n_total_uc + j / l.n_basis], j % l.n_basis);
                perm[(2 * i) * n + j] = (int)t;
                perm[(2 * i + 1) * n + j] = (int)(n - 1 - t);
            }
        }
        S = (int)n;
        basis[0] = 0;
        *n_vb = 1;
    } else {
        for (int i = 0; i < nsym; i++)
            for (uint64_t j = 0; j < n; j++)
                perm[i * n + j] = (int)IDX(&l, ucs[i * l.n_total_uc + j / l.n_basis], j % l.n_basis);
        S = nsym;
        /* construct_symm_basis: unit cells spanned by the factor x */
        uint64_t x[2];
        clean_symm(&l, symm, x);
        int c = 0;
        for (uint64_t i1 = 0; i1 < x[1]; i1++)
            for (uint64_t i0 = 0; i0 < x[0]; i0++) {
                uint64_t uc = orc_up(&l, orc_up(&l, 0, 1, i1), 0, i0);
                for (uint64_t b = 0; b < l.n_basis; b++) basis[c++] = (int)IDX(&l, uc, b);
            }
        *n_vb = c;
    }
    free(ucs);
    return S;
}

/* --------------------------------------------------------------- models -- */
/* Pauli matrices, model/abstract_model.cpp:37-58 */
static const double complex PAULI[4][2][2] = {
    {{1, 0}, {0, 1}},
    {{0, 1}, {1, 0}},
    {{0, -I}, {I, 0}},
    {{1, 0}, {0, -1}},
};

/* kron(args): the first factor sits on the least-significant bit
 * (abstract_model.cpp:28-33).  which[i] in {1,2,3} = x,y,z. */
static void dense_kron(int k, const int* which, double complex scale,
                       double* out) {
    int d = 1 << k;
    for (int r = 0; r < d; r++)
        for (int c = 0; c < d; c++) {
            double complex v = scale;
            for (int i = 0; i < k; i++) v *= PAULI[which[i]][(r >> i) & 1][(c >> i) & 1];
            out[2 * (r * d + c)] = creal(v);
            out[2 * (r * d + c) + 1] = cimag(v);
        }
}

void orc_kitaev_sizes(int n_uc, int n_uc_b, double h, int* n_ops, int* n_entries) {
    orc_bravais l;
    honeycomb_init(&l, n_uc, n_uc_b);
    int nb = (int)l.n_total_uc * 3;
    *n_ops = nb;
    *n_entries = nb * 16;
    if (fabs(h) > 1e-10) {
        *n_ops += (int)l.n_total;
        *n_entries += (int)l.n_total * 4;
    }
}

/* model::kitaev, kitaev.cpp:29-50 */
void orc_kitaev_ops(int n_uc, int n_uc_b, const double J[3], double h, int* k,
                    int* sites, int* mat_off, double* mats) {
    orc_bravais l;
    honeycomb_init(&l, n_uc, n_uc_b);
    int nb = (int)l.n_total_uc * 3;
    int* abt = (int*)malloc(sizeof(int) * 3 * nb);
    orc_honeycomb_bonds(n_uc, n_uc_b, abt);
    int off = 0;
    for (int b = 0; b < nb; b++) {
        int t = abt[3 * b + 2];
        int which[2] = {t + 1, t + 1};
        k[b] = 2;
        for (int i = 0; i < 6; i++) sites[6 * b + i] = -1;
        sites[6 * b + 0] = abt[3 * b];
        sites[6 * b + 1] = abt[3 * b + 1];
        mat_off[b] = off;
        dense_kron(2, which, J[t], mats + 2 * off);
        off += 16;
    }
    int o = nb;
    if (fabs(h) > 1e-10) {
        for (uint64_t i = 0; i < l.n_total; i++, o++) {
            k[o] = 1;
            for (int j = 0; j < 6; j++) sites[6 * o + j] = -1;
            sites[6 * o] = (int)i;
            mat_off[o] = off;
            double complex m[2][2];
            for (int r = 0; r < 2; r++)
                for (int c = 0; c < 2; c++)
                    m[r][c] = -h * PAULI[1][r][c] + h * PAULI[2][r][c] + h * PAULI[3][r][c];
            for (int r = 0; r < 2; r++)
                for (int c = 0; c < 2; c++) {
                    mats[2 * (off + r * 2 + c)] = creal(m[r][c]);
                    mats[2 * (off + r * 2 + c) + 1] = cimag(m[r][c]);
                }
            off += 4;
        }
    }
    free(abt);
}

void orc_toric_sizes(int n_uc, int* n_ops, int* n_entries) {
    *n_ops = 2 * n_uc * n_uc;
    *n_entries = *n_ops * 256;
}

/* model::toric, toric.cpp:27-47: plaquettes J sz^4, stars J sx^4 */
void orc_toric_ops(int n_uc, double J, int* k, int* sites, int* mat_off,
                   double* mats) {
    int np = 2 * n_uc * n_uc;
    int* p5 = (int*)malloc(sizeof(int) * 5 * np);
    orc_toric_plaqs(n_uc, p5);
    for (int o = 0; o < np; o++) {
        int w = p5[5 * o + 4] == 0 ? 3 : 1;
        int which[4] = {w, w, w, w};
        k[o] = 4;
        for (int i = 0; i < 6; i++) sites[6 * o + i] = i < 4 ? p5[5 * o + i] : -1;
        mat_off[o] = o * 256;
        dense_kron(4, which, J, mats + 2 * o * 256);
    }
    free(p5);
}

void orc_hexagon_sizes(int n_uc, int n_uc_b, int* n_ops, int* n_entries) {
    orc_bravais l;
    honeycomb_init(&l, n_uc, n_uc_b);
    *n_ops = (int)l.n_total_uc;
    *n_entries = *n_ops * 4096;
}

/* W_p plaquette operator kron(sx,sy,sz,sx,sy,sz), main.cpp:645-671 */
void orc_hexagon_ops(int n_uc, int n_uc_b, int* k, int* sites, int* mat_off,
                     double* mats) {
    orc_bravais l;
    honeycomb_init(&l, n_uc, n_uc_b);
    int nh = (int)l.n_total_uc;
    int* h6 = (int*)malloc(sizeof(int) * 6 * nh);
    orc_honeycomb_hexagons(n_uc, n_uc_b, h6);
    int which[6] = {1, 2, 3, 1, 2, 3};
    for (int o = 0; o < nh; o++) {
        k[o] = 6;
        for (int i = 0; i < 6; i++) sites[6 * o + i] = h6[6 * o + i];
        mat_off[o] = o * 4096;
        dense_kron(6, which, 1.0, mats + 2 * o * 4096);
    }
    free(h6);
}

/* kitaev::exact_energy and kitaev::f, kitaev.cpp:66-100 */
double orc_kitaev_exact_energy(int n_uc, int n_uc_b, const double J[3]) {
    orc_bravais l;
    honeycomb_init(&l, n_uc, n_uc_b);
    double na = (double)l.n_uc_b, nb = (double)l.n_uc;
    double smret = -1e10;
    for (int ci1 = 0; ci1 < 2; ci1++)
        for (int ci2 = 0; ci2 < 2; ci2++) {
            double ret = 0;
            double c1 = 0.5 / nb * ci1, c2 = 0.5 / na * ci2;
            for (int i = 0; i < (int)nb; i++)
                for (int j = 0; j < (int)na; j++) {
                    double p1 = i / nb + c1, p2 = j / na + c2;
                    double complex f = 2.0 * (J[0] * cexp(I * 2 * M_PI * p1) +
                                              J[1] * cexp(I * 2 * M_PI * p2) + J[2]);
                    ret += cabs(f);
                }
            if (ret > smret) smret = ret;
        }
    return -0.5 * smret / (double)l.n_total;
}
