/*
 * orc.h -- FP64 CPU oracle for the rbm-nqs VMC hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (dbucher97/rbm-nqs) used as the checker by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  It is never
 * linked into, loaded by, or called from the product library.
 *
 * Every function cites the reference file:line it restates.  Conventions:
 *   - a configuration is four uint32 words (bit i of word i/32 = site i);
 *     bit set  <=>  sigma_i = -1            (machine/spin_state.cpp:44-50)
 *   - complex numbers are C99 double complex, interleaved re/im in memory
 *   - theta has n_hidden rows and S columns, column-major: t = k + nh*s
 *     (rbm_symmetry.cpp:48-61; S = 1 for the basic RBM, rbm_base.cpp:161-172)
 *   - W is n x nh column-major: W[i + n*k]      (rbm_base.cpp:38-56, 117-143)
 *   - parameter order [v (n_vb), h (nh), W (n*nh col-major), pfaffian fs_
 *     (n_indep x 4 col-major)]                   (rbm_base.cpp:117-131)
 */
#ifndef RBMNQS_ORACLE_H
#define RBMNQS_ORACLE_H

#include <complex.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- RNG -- */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), the counter-based
 * generator both the oracle and the CUDA sampler draw from. */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ------------------------------------------------------------ lattice -- */
typedef struct {
    uint64_t n_uc, n_dim, n_basis, n_coord, n_total_uc, n_total, n_uc_b, h_shift;
} orc_bravais;

void orc_bravais_init(orc_bravais* l, uint64_t n_uc, uint64_t n_dim,
                      uint64_t n_basis, uint64_t n_coord, uint64_t n_uc_b,
                      uint64_t h_shift);
uint64_t orc_up(const orc_bravais* l, uint64_t uc, uint64_t dir, uint64_t step);
uint64_t orc_down(const orc_bravais* l, uint64_t uc, uint64_t dir, uint64_t step);

/* honeycomb (lattice/honeycomb.cpp): nearest neighbours, bonds (a,b,type) */
void orc_honeycomb_nns(int n_uc, int n_uc_b, int site, int out[3]);
int orc_honeycomb_bonds(int n_uc, int n_uc_b, int* out_abt);
int orc_honeycomb_hexagons(int n_uc, int n_uc_b, int* out6);
/* toric lattice (lattice/toric_lattice.cpp:57-69): [2L^2][5] = 4 sites + type */
int orc_toric_plaqs(int n_uc, int* out5);

/* Symmetry permutations perm[s*n + i] = P_s(i) and the symmetry basis.
 * kind: 0 = honeycomb, 1 = toric/bravais.  symm: the single symmetry value
 * (0 = none, 0.5 = honeycomb translations+rot180, 1 = translations).
 * Returns S; writes n_vb (= number of basis sites). */
int orc_symmetry(int kind, int n_uc, int n_uc_b, double symm, int* perm,
                 int* basis, int* n_vb);

/* ------------------------------------------------------------- models -- */
/* Dense local operators: op o acts on k[o] sites (<= 6), its 2^k x 2^k
 * complex matrix (row-major) starts at mats + 2*mat_off[o] doubles. */
typedef struct {
    int n_ops;
    const int* k;        /* [n_ops] */
    const int* sites;    /* [n_ops][6] */
    const int* mat_off;  /* [n_ops] offset in complex entries */
    const double* mats;  /* interleaved complex */
} orc_ops;

/* Number of ops and total matrix entries the builders will write. */
void orc_kitaev_sizes(int n_uc, int n_uc_b, double h, int* n_ops, int* n_entries);
void orc_kitaev_ops(int n_uc, int n_uc_b, const double J[3], double h, int* k,
                    int* sites, int* mat_off, double* mats);
void orc_toric_sizes(int n_uc, int* n_ops, int* n_entries);
void orc_toric_ops(int n_uc, double J, int* k, int* sites, int* mat_off,
                   double* mats);
/* Hexagon plaquette W_p = sx sy sz sx sy sz on each honeycomb hexagon
 * (main.cpp:645-671). */
void orc_hexagon_sizes(int n_uc, int n_uc_b, int* n_ops, int* n_entries);
void orc_hexagon_ops(int n_uc, int n_uc_b, int* k, int* sites, int* mat_off,
                     double* mats);
/* Analytic Kitaev ground-state energy per site (model/kitaev.cpp:66-100). */
double orc_kitaev_exact_energy(int n_uc, int n_uc_b, const double J[3]);

/* ------------------------------------------------------------ machine -- */
typedef struct {
    int n;       /* visible spins */
    int n_vb;    /* visible-bias size */
    int nh;      /* hidden rows of theta (n_alpha_ = alpha * n_vb) */
    int S;       /* symmetry columns of theta */
    int symmetric; /* 0: rbm_base, 1: rbm_symmetry */
    const int* perm;   /* [S][n] */
    const int* basis;  /* [n_vb] */
    const double complex* v;  /* [n_vb] */
    const double complex* h;  /* [nh] */
    const double complex* W;  /* [n*nh] column-major */
    /* Pfaffian pair wavefunction (machine/pfaffian.cpp), optional */
    int has_pf;
    int n_indep;
    const int* bs;            /* [n][n] row-major index matrix */
    const double complex* fs; /* [n_indep*4] column-major (i + n_indep*c) */
} orc_machine;

int orc_n_params(const orc_machine* m);
int orc_n_neural(const orc_machine* m);

/* Pfaffian index matrix bs_ (pfaffian.cpp:31-85); returns n_indep. */
int orc_pfaffian_bs(int n, int S, const int* perm, int n_basis,
                    const int* basis, int* bs);

void orc_theta(const orc_machine* m, const uint32_t* spins, double complex* theta);
double complex orc_lncosh_sum(const double complex* x, int len);
double complex orc_log_psi(const orc_machine* m, const uint32_t* spins);
double complex orc_log_psi_over_psi(const orc_machine* m, const uint32_t* spins,
                                    const int* flips, int nf);
void orc_derivative(const orc_machine* m, const uint32_t* spins,
                    double complex* O);
double complex orc_eloc(const orc_machine* m, const orc_ops* ops,
                        const uint32_t* spins);

/* Pfaffian context: X^{-1} (n x n, column-major), Pf = mant * 10^exp10. */
typedef struct {
    double complex* inv;
    double complex pf_mant;
    int pf_exp10;
    double complex update_factor;
} orc_pfctx;
void orc_pf_matrix(const orc_machine* m, const uint32_t* spins, double complex* X);
void orc_pf_context(const orc_machine* m, const uint32_t* spins, orc_pfctx* c);
void orc_pf_update(const orc_machine* m, const uint32_t* spins, const int* flips,
                   int nf, orc_pfctx* c);
/* Pfaffian of a dense antisymmetric matrix (column-major, overwritten) by
 * Parlett-Reid elimination, returned as mantissa * 10^exp10. */
double complex orc_pfaffian10(int n, double complex* A, int* exp10);

/* Batched evaluation (OpenMP over configurations). */
void orc_eval_batch(const orc_machine* m, const orc_ops* ops,
                    const uint32_t* spins, int B, double complex* logpsi,
                    double complex* eloc, double complex* O);

/* ------------------------------------------------------------ sampler -- */
typedef struct {
    int n_chains, samples_per_chain, warmup, step;
    double bond_flips;
    int n_prop_bonds;
    const int* prop_bonds; /* [n_prop_bonds][2] */
    uint64_t seed;
    int pf_refresh;
} orc_sampler_cfg;

/* Metropolis sampling of one epoch (metropolis_sampler.cpp:55-273).
 * spins_io: [n_chains][4]; if init != 0 chains start from Philox-random
 * states.  Writes E[c*spc + j], O[(c*spc + j)*P] and per-chain acceptance. */
void orc_metropolis(const orc_machine* m, const orc_ops* ops,
                    const orc_sampler_cfg* cfg, uint32_t epoch, int init,
                    uint32_t* spins_io, double complex* E, double complex* O,
                    double* acc_chain, int n_threads);

/* Exact enumeration (full_sampler.cpp:43-186): p = |psi|^2 weights.
 * Outputs p_tot (relative to the largest log|psi|), <E>, <O>, <E O*> and the
 * unbiased weighted variance of O. */
void orc_full(const orc_machine* m, const orc_ops* ops, double* p_tot,
              double complex* E_mean, double complex* d, double complex* dh,
              double* var_O, int n_threads);

/* ------------------------------------------------------------- stats  -- */
/* aggregator::aggregate/finalize (aggregator.cpp:84-239) for a scalar with
 * unit weights and n_bins bins. */
void orc_stats(const double complex* x, int N, int n_bins, double complex* mean,
               double* var, double* var_binned, double* tau, double* stddev);

/* ---------------------------------------------------------------- SR --- */
/* d = <O>, F = <E O*> - <E> conj(d), diag = unbiased var(O)
 * (stochastic_reconfiguration.cpp:81-116, aggregator.cpp:151-154). */
void orc_sr_moments(const double complex* O, const double complex* E, int N,
                    int P, double complex* d, double complex* F, double* diag);
/* Dense S = conj(O)^T-style Gram (cg_solver.cpp:274-299 CG_SINGLE form). */
void orc_sr_matrix(const double complex* O, const double complex* d, int N,
                   int P, double complex* S);
/* cg_solver::solve with the distributed CG (cg1) semantics
 * (cg_solver.cpp:119-193, 260-334).  x_io holds the warm start. */
int orc_cg_solve(const double complex* O, const double complex* d, double norm,
                 int N, int P, int n_neural, const double complex* F,
                 double complex* x_io, double r1, double r2, double rd,
                 const double* diag, int max_iterations, double rtol,
                 double* rs_out);

/* MINRES-QLP on the same operator (zminresqlpModule.f90 through
 * minresqlp_adapter.cpp:40-110): x0 = 0; rnorm, istop, Acond and the
 * number of QLP iterations through the optional pointers. */
int orc_minresqlp_solve(const double complex* O, const double complex* d, double norm,
                        int N, int P, int n_neural, const double complex* F,
                        double complex* x, double r1, double r2, double rd,
                        const double* diag, int max_iterations, double rtol,
                        double* rnorm_out, int* istop_out, double* acond_out, int* qlp_out);

/* decay_t (abstract_optimizer.cpp:27-54) */
typedef struct {
    double initial, min, decay, value;
    int min_reached;
} orc_decay;
void orc_decay_init(orc_decay* d, double initial, double min, double decay,
                    uint64_t offset);
double orc_decay_get(orc_decay* d);

#ifdef __cplusplus
}
#endif
#endif
