/*
 * rbmnqs_b200.h -- C ABI of the B200 (sm_100a) VMC hot path for rbm-nqs.
 *
 * The library replaces, for one GPU, the reference's per-epoch hot path
 *   sampler::abstract_sampler::sample()        include/sampler/abstract_sampler.hpp:74
 *   optimizer::abstract_optimizer::optimize()   src/optimizer/abstract_optimizer.cpp:80-178
 *   optimizer::abstract_solver::solve(...)      include/optimizer/abstract_solver.hpp:31-34
 * together with the machine/operators work they drive (machine/rbm_base,
 * machine/rbm_symmetry, operators/local_op, operators/aggregator).
 *
 * Conventions (all identical to the reference):
 *   - complex arrays are interleaved (re, im) doubles;
 *   - a configuration is four uint32 words, bit i of word i/32 is site i and a
 *     set bit means sigma_i = -1               (machine/spin_state.cpp:44-50);
 *   - the parameter vector is [v (n_vb), h (n_hidden), W (n x n_hidden,
 *     column-major, j + n*k), Pfaffian f (n_indep x 4, column-major)]
 *                                              (machine/rbm_base.cpp:117-131);
 *   - samples are ordered chain-major: sample c*samples_per_chain + j.
 * All functions return 0 on success or a negative RBMNQS_ERR_* code; the
 * message of the last error of the calling thread is rbmnqs_last_error().
 * No C++ exception crosses this boundary.  A handle owns one CUDA stream and
 * all its device buffers; calls on one handle must not run concurrently.
 */
#ifndef RBMNQS_B200_H
#define RBMNQS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RBMNQS_OK 0
#define RBMNQS_ERR_ARG (-1)           /* bad argument / shape */
#define RBMNQS_ERR_CUDA (-2)          /* CUDA runtime error */
#define RBMNQS_ERR_UNSUPPORTED (-3)   /* configuration not supported */
#define RBMNQS_ERR_MASSIVE_STEP (-4)  /* max|dw| > 30, abstract_optimizer.cpp:157-159 */
#define RBMNQS_ERR_NONFINITE (-5)     /* NaN/Inf in energies or update */
#define RBMNQS_ERR_NO_DEVICE (-6)     /* no CUDA device / kernels not loadable */

typedef struct rbmnqs_model rbmnqs_model;
typedef struct rbmnqs_handle rbmnqs_handle;

/* ----------------------------------------------------------- models ---- */
/* Kitaev honeycomb model: bond operators J_g sigma^g sigma^g on x/y/z bonds
 * and an optional field -h sx + h sy + h sz on every site.
 * Replaces model::kitaev (src/model/kitaev.cpp:29-50) with
 * lattice::honeycomb (src/lattice/honeycomb.cpp); `symmetry` is the
 * model.symmetry value used by rbm.type=symmetry (honeycomb.hpp:77-85). */
int rbmnqs_model_kitaev(int32_t n_cells, int32_t n_cells_b, const double J[3],
                        double h, double symmetry, rbmnqs_model** out);
/* Toric code: J sz^4 on plaquettes, J sx^4 on stars.
 * Replaces model::toric (src/model/toric.cpp:27-47) with
 * lattice::toric_lattice (src/lattice/toric_lattice.cpp:57-69). */
int rbmnqs_model_toric(int32_t n_cells, double J, double symmetry,
                       rbmnqs_model** out);
/* Adds the hexagon plaquette operators W_p (observables, main.cpp:645-671)
 * as extra, separately accumulated operators. */
int rbmnqs_model_add_hexagons(rbmnqs_model* m);
/* Sizes: spins, Hamiltonian operators, lattice bonds, observables. */
int rbmnqs_model_sizes(const rbmnqs_model* m, int32_t* n_sites,
                       int32_t* n_ops, int32_t* n_bonds, int32_t* n_observables);
/* Bond list (a, b, type) as lattice::get_bonds (bravais.hpp get_bonds). */
int rbmnqs_model_bonds(const rbmnqs_model* m, int32_t* abt);
/* Operator k, acts_on[6] (-1 padded) and its dense 2^k x 2^k row-major
 * complex matrix (operators/local_op.hpp op_), for inspection and tests. */
int rbmnqs_model_op(const rbmnqs_model* m, int32_t o, int32_t* k,
                    int32_t* acts_on, double* mat);
/* Symmetry permutations perm[s*n + i] = P_s(i) and basis (n_vb entries) used
 * by rbm.type=symmetry (bravais.cpp:160-247, honeycomb.cpp:69-134). */
int rbmnqs_model_symmetry(const rbmnqs_model* m, int32_t* S, int32_t* n_vb,
                          int32_t* perm, int32_t* basis);
/* Pfaffian pair-class matrix bs_ (pfaffian.cpp:31-85) of the model's lattice
 * for a symmetry value: bs[i*n + j] = signed 1-based class of pair (i, j)
 * (bs may be NULL) and the number of classes n_indep.  Host only. */
int rbmnqs_model_pfaffian_classes(const rbmnqs_model* m, double symmetry,
                                  int32_t* bs, int32_t* n_indep);
/* Exact diagonalisation on the GPU (n <= 28 sites): the lowest eigenvalue of
 * the model's Hamiltonian by Lanczos on the full 2^n basis, stopping when it
 * changed by at most tol (relative) over three iterations or after max_iter
 * iterations; psi (2^n complex, interleaved re, im, may be NULL) receives
 * the normalised eigenvector, indexed by the state number (bit i set <=>
 * site i down).  The reference diagonalises small systems in Python
 * (python_adapter/rbm/__init__.py:16-41, scipy); this is the same
 * Hamiltonian and basis convention.  Allocates 3 (4 with psi) device
 * vectors of 2^n x 16 bytes for the duration of the call. */
int rbmnqs_model_ground_state(const rbmnqs_model* m, int32_t max_iter, double tol, uint64_t seed,
                              double* energy, int32_t* iterations, double* psi);
void rbmnqs_model_destroy(rbmnqs_model* m);

/* ----------------------------------------------------------- config ---- */
/* Key names follow the reference's .ini options (README.md:66-173). */
typedef struct {
    int32_t rbm_type;          /* rbm.type: 0 = basic, 1 = symmetry */
    int32_t alpha;             /* rbm.alpha */
    int32_t pfaffian;          /* rbm.pfaffian (0/1) */
    double pfaffian_symmetry;  /* rbm.pfaffian.symmetry */
    int32_t n_chains;          /* sampler.metropolis.n_chains */
    int32_t samples_per_chain; /* sampler.n_samples_per_chain */
    int32_t warmup;            /* sampler.metropolis.n_warmup_steps (sweeps) */
    int32_t step;              /* sampler.metropolis.n_steps_per_sample */
    double bond_flips;         /* sampler.metropolis.bond_flips */
    int32_t pfaffian_refresh;  /* sampler.pfaffian_refresh */
    int32_t reinit_chains;     /* 1: fresh random chains every epoch (reference
                                  behaviour, metropolis_sampler.cpp:127);
                                  0: chains persist across epochs */
    uint64_t seed;             /* seed */
    double lr[3];              /* optimizer.learning_rate: initial, min, decay */
    double reg1[3];            /* optimizer.sr.reg1 */
    double reg2[3];            /* optimizer.sr.reg2 */
    double deltareg1[3];       /* optimizer.sr.deltareg1 */
    int32_t max_iterations;    /* optimizer.sr.max_iterations (0 = 2P) */
    double rtol;               /* optimizer.sr.rtol (0 = 1e-16) */
    int32_t precision;         /* 0: FP32 psi-ratio math with FP64 theta
                                     recompute, FP16x3 split-precision tensor-core Gram;
                                  1: FP64 throughout */
    int32_t n_updates;         /* rbm n_updates_ (decay_t offset on resume) */
    int32_t gram;              /* S build: 0 = by precision (FP16x3 tensor
                                  cores when precision is 0, FP64 when 1);
                                  1 = FP64 CUDA cores in either precision */
    /* Learned proposals (no reference counterpart): 0 = plain Metropolis;
     * 1 = learned_steps moves per sample after every `step` sweeps (step 0:
     * no sweeps, the chains move by learned moves alone).  A move flips one
     * entry of a dictionary of site sets: every single site and every
     * distinct off-diagonal flip set of the Hamiltonian (Kitaev x / y bonds,
     * toric-code stars; at most 256 entries).  The proposal network maps the
     * configuration s to logits over the dictionary; the move is drawn from
     * q(m|s) = 0.9 softmax(logits(s))_m + 0.1 / D and accepted by the exact
     * Metropolis-Hastings ratio |psi'/psi|^2 q(m|s') / q(m|s), q(m|s') from
     * the network at s'.  The network is trained every epoch (learned_train
     * Adam steps, learned_lr) on the first min(n_chains, 2048) chains'
     * configurations, towards targets proportional to
     * min(1, |psi(s with move m)/psi(s)|^2) (softmax cross entropy).  Not
     * with the Pfaffian factor. */
    int32_t proposal;
    int32_t learned_steps;
    int32_t learned_train;
    int32_t learned_hidden;    /* width of both hidden layers (64..256) */
    double learned_lr;
    int32_t solver;            /* optimizer.sr.method: 0 = cg (cg_solver), 1 =
                                  minresqlp (MINRES-QLP from x0 = 0; rtol
                                  then bounds the relative residual
                                  ||r|| / (||A|| ||x|| + ||b||), max_iterations
                                  defaults to 4 n_params), 2 = direct
                                  (direct_solver.cpp:31-59: multiplicative
                                  diagonal regularisation, exact solve; above
                                  2048 parameters in sample space, at most
                                  4096 samples per epoch) */
    int32_t optimizer_type;    /* optimizer.type: 0 = SR, 1 = SGD
                                  (gradient_descent.cpp:42-60) */
    double sgd_real_factor;    /* optimizer.sgd.real_factor */
    int32_t plugin;            /* optimizer.plugin: 0 none, 1 adam, 2 momentum,
                                  3 heun (plugin.cpp:29-115; heun samples
                                  and solves a second time every epoch) */
    double adam_beta1, adam_beta2, adam_eps;  /* optimizer.adam.* */
    double mom_alpha, mom_dialup;             /* optimizer.mom.* */
    double heun_eps;                          /* optimizer.heun.eps */
    int32_t sampler_type;      /* sampler.type: 0 = metropolis, 1 = full
                                  (full_sampler.cpp:43-186: all 2^n states
                                  weighted by |psi|^2; n_chains,
                                  samples_per_chain, warmup, step and
                                  bond_flips are unused; n_samples = 2^n) */
    int32_t full_parallel_bits;  /* sampler.full.n_parallel_bits: the
                                  enumeration order (blocks of the low bits,
                                  Gray code over the rest) */
} rbmnqs_config;

/* Fills the reference defaults (src/tools/ini.cpp:38-120). */
int rbmnqs_config_default(rbmnqs_config* cfg);

/* -------------------------------------------------- session lifetime ---- */
int rbmnqs_create(const rbmnqs_model* m, const rbmnqs_config* cfg,
                  rbmnqs_handle** out);
void rbmnqs_destroy(rbmnqs_handle* h);
const char* rbmnqs_last_error(void);

/* Parameter counts (abstract_machine.hpp:84-104). */
int rbmnqs_sizes(const rbmnqs_handle* h, int32_t* n_params, int32_t* n_neural,
                 int32_t* n_vb, int32_t* n_hidden, int32_t* n_symmetry);

/* Weights in the reference parameter order (rbm_base::update_weights). */
int rbmnqs_set_weights(rbmnqs_handle* h, const double* w);
int rbmnqs_get_weights(rbmnqs_handle* h, double* w);

/* ------------------------------------------------------ hot path -------- */
typedef struct {
    double energy[2];     /* <E_loc> (aggregator a_h_ result) */
    double energy_var;    /* unbiased variance of E_loc */
    double energy_stddev; /* binned standard error (aggregator::get_stddev) */
    double tau;           /* binning autocorrelation estimate */
    double acceptance;    /* mean acceptance rate over chains */
    int64_t n_samples;
    int32_t n_bins;
    int32_t status;       /* RBMNQS_OK or RBMNQS_ERR_NONFINITE */
    double learned_acceptance; /* acceptance of the learned moves (0 without) */
    double learned_loss;       /* proposal-network training loss of the epoch */
} rbmnqs_sample_stats;

/* One Metropolis epoch: sweeps, E_loc, O_k, and the reductions the
 * reference's aggregators produce (metropolis_sampler.cpp:55-116). */
int rbmnqs_sample(rbmnqs_handle* h, rbmnqs_sample_stats* out);

typedef struct {
    int32_t iterations;   /* CG iterations (cg_solver itn_) */
    int32_t status;       /* RBMNQS_OK, RBMNQS_ERR_MASSIVE_STEP, _NONFINITE */
    double residual;      /* final ||r||^2 */
    double max_dw;        /* max |x| before scaling by lr */
    double lr, reg1, reg2, deltareg1;
} rbmnqs_sr_stats;

/* SR step after rbmnqs_sample: F, S, CG solve, w -= lr * x
 * (stochastic_reconfiguration.cpp:81-116, abstract_optimizer.cpp:80-178). */
int rbmnqs_optimize(rbmnqs_handle* h, rbmnqs_sr_stats* out);

/* sample + optimize as one CUDA-graph launch (captured on first use). */
int rbmnqs_epoch(rbmnqs_handle* h, rbmnqs_sample_stats* s, rbmnqs_sr_stats* o);

/* Copies of the last epoch's per-sample data: E[N] and O[N][n_params]
 * (sample-major), both interleaved complex. */
int rbmnqs_get_samples(rbmnqs_handle* h, double* E, double* O);
/* The sampled configurations of the last epoch [N][4] (chain-major, the
 * order of E and O). */
int rbmnqs_get_sample_configs(rbmnqs_handle* h, uint32_t* configs);
/* SR moments of the last epoch: d = <O>, F, unbiased var(O), S (P x P,
 * row-major, S_kl = <conj(O_k) O_l> - conj(d_k) d_l, unregularised). */
int rbmnqs_get_sr(rbmnqs_handle* h, double* d, double* F, double* diag, double* S);

/* Chain configurations [n_chains][4]. */
int rbmnqs_get_spins(rbmnqs_handle* h, uint32_t* spins);
int rbmnqs_set_spins(rbmnqs_handle* h, const uint32_t* spins);

/* -------------------------------------------- parity / drop-in calls ---- */
/* log psi, E_loc and O_k (optional, NULL skips) of B given configurations
 * (machine::abstract_machine::psi / derivative, local_op::evaluate). */
int rbmnqs_eval_batch(rbmnqs_handle* h, const uint32_t* spins, int32_t B,
                      double* logpsi, double* eloc, double* O);
/* log(psi(sigma with flips)/psi(sigma)) for B configurations, each with
 * n_flips sites (rbm_base::log_psi_over_psi, rbm_base.cpp:306-344). */
int rbmnqs_log_psi_over_psi(rbmnqs_handle* h, const uint32_t* spins,
                            const int32_t* flips, int32_t n_flips, int32_t B,
                            double* out);
/* abstract_solver::solve on the GPU: O is N x P sample-major (the
 * reference's a_dd_ store transposed), d = <O>, norm = sum of weights, F the
 * force, x_io the warm start in / solution out, r1/r2/rd the regularisation
 * and diag = var(O) (cg_solver.cpp:260-334). */
int rbmnqs_sr_solve(rbmnqs_handle* h, const double* O, int32_t N,
                    const double* d, double norm, const double* F,
                    double* x_io, double r1, double r2, double rd,
                    const double* diag, int32_t* iterations, double* residual);
/* The last SR solve's outcome (that of rbmnqs_sr_solve or of the last
 * epoch's update), the getters of minresqlp_adapter.h (getItn, getRnorm,
 * getAcond) and the istop that minresqlp_adapter::apply returns
 * (minresqlp_adapter.cpp:104-110).  With solver = 1 (minresqlp): istop is
 * the stopping reason of MINRES-QLP (1: beta_{k+1} < eps, 2: x is an
 * eigenvector, 3: b = 0, 4/5: relative residual <= rtol / at machine
 * precision, 6/7: relative normal-equation residual <= rtol / at machine
 * precision, 8: iteration limit, 12: ||x|| reached 1e7, 13: Acond reached
 * 1e15 or 0.1/eps, 14: the least-squares problem has no further
 * solution), acond the condition estimate and qlp_iterations the number
 * of steps taken with the QLP updates (Acond above 1e7).  Other solvers
 * leave istop, acond and qlp_iterations 0.  Any output pointer may be NULL. */
int rbmnqs_solve_info(rbmnqs_handle* h, int32_t* iterations, double* residual,
                      int32_t* istop, double* acond, int32_t* qlp_iterations);
/* Exact enumeration of all 2^n configurations weighted by |psi|^2
 * (full_sampler.cpp:43-186); n <= 30.  Outputs <E>, <O>, <E O*>. */
int rbmnqs_full_sample(rbmnqs_handle* h, double* E_mean, double* d, double* dh);
/* Evaluation mode (main.cpp:640-671): expectation values of the model's
 * observables (the hexagon plaquettes W_p after rbmnqs_model_add_hexagons)
 * over the samples of the last epoch, each through the local estimator
 * sum_l' O[l, l'] psi(l') / psi(l) (local_op.cpp:31-60) with the
 * aggregator's statistics: values[4 i .. 4 i + 3] = Re <O_i>, Im <O_i>,
 * binned standard deviation of the mean, tau. */
int rbmnqs_get_observables(rbmnqs_handle* h, double* values);

/* Full enumeration only: the normalised state vector psi[2^n] (complex,
 * interleaved re, im) indexed by the state number (bit i set <=> site i
 * down) of the last sample -- full_sampler::sample(keep_state = true)
 * (full_sampler.cpp:112-159), returned instead of written to a file. */
int rbmnqs_full_state(rbmnqs_handle* h, double* psi);

/* ----------------------------------------------------------- timing ---- */
/* Device time (ms, CUDA events on the handle's stream) accumulated per stage
 * since the last reset: 0 Metropolis sweeps, 1 E_loc + O_k evaluation,
 * 2 moments + energy statistics, 3 Gram + regularisation, 4 CG, 5 update.
 * `launches` counts how often each stage ran. */
int rbmnqs_timing(rbmnqs_handle* h, double* ms, int64_t* launches, int32_t n);
int rbmnqs_timing_reset(rbmnqs_handle* h, int32_t enable);
/* Launch-shape autotuner: times the sweep kernel over `sweeps` sweeps (one
 * recorded sample) for one and (where the expanded-table path allows it)
 * two chains per warp, each with up to five warps-per-block caps, and the
 * evaluation kernel for 1..8 warps per block;
 * keeps the fastest of each (the session's chains, weights and statistics
 * are left as they were; the epoch graph is re-captured).  No reference
 * counterpart (the reference has no launch shapes).  Outputs may be NULL. */
int rbmnqs_autotune(rbmnqs_handle* h, int32_t sweeps, int32_t* sampler_warps_per_block,
                    int32_t* eval_warps_per_block, double* sampler_ms);

/* Solver-stage autotuner (no reference counterpart): on the session's
 * current O (sample first), times the tensor-core Gram for the cheapest split-K
 * counts of its cost model and keeps the fastest, and, where S is formed and
 * the cluster CG holds it, times one CG solve each with the cluster kernel
 * and the cooperative one-barrier kernel and keeps the faster.  Both CG
 * kernels follow cg1 (the same iterates up to rounding); a different split
 * count changes S only by FP32 rounding (within the 1e-5 of the FP32 path).
 * x, the chains and the weights are left as they were; the epoch graph is
 * re-captured.  Outputs (may be NULL): the split count (0 without the
 * tensor-core Gram), the CG kernel (0 cluster, 1 cooperative, -1 not tuned)
 * and the best Gram + CG milliseconds. */
int rbmnqs_autotune_sr(rbmnqs_handle* h, int32_t* gram_splits, int32_t* cg_kernel, double* sr_ms);

/* Sets the sweep launch shape: warps per block (0 = planned) and chains per
 * warp (1, or 2 for the FP32 expanded-table path with n <= 32 sites, whose
 * two-chain sweep is bit-identical to the one-chain sweep).  The epoch
 * graph is re-captured.  No reference counterpart.  RBMNQS_ERR_UNSUPPORTED
 * when two chains per warp is not available for the session. */
int rbmnqs_set_sweep_shape(rbmnqs_handle* h, int32_t warps_per_block, int32_t chains_per_warp);
/* The current sweep shape (outputs may be NULL). */
int rbmnqs_get_sweep_shape(rbmnqs_handle* h, int32_t* warps_per_block, int32_t* chains_per_warp);

/* Number of kernel launches one rbmnqs_epoch performs (kernel nodes of the
 * captured epoch graph; 0 before the first rbmnqs_epoch). */
int rbmnqs_graph_kernels(rbmnqs_handle* h, int32_t* kernel_nodes);
/* The handle's cudaStream_t, for callers that order work against it. */
void* rbmnqs_stream(rbmnqs_handle* h);

/* ------------------------------------------------------------ checkpoints */
/* The reference's .rbm file (rbm_base::save / load, rbm_base.cpp:219-288,
 * matrices as eigen_fstream.cpp:25-51: rows, cols as 8-byte size_t, then the
 * column-major complex128 data): W (n x n_hidden), h (n_hidden x 1), v (n_vb x
 * 1), n_updates (size_t), then the Pfaffian fs_ (n_indep x 4) when present.
 * `path` is the full file name.  Loading sets the weights and the update
 * count, and restarts the decay_t schedules at that count
 * (abstract_optimizer.cpp:27-54). */
int rbmnqs_save(rbmnqs_handle* h, const char* path);
int rbmnqs_load(rbmnqs_handle* h, const char* path);
/* Training log, logger.cpp:31-74: opens <name>.log, appending when the file
 * exists unless `force` (rbm.force) is set.  Every applied update (by
 * rbmnqs_epoch, rbmnqs_optimize or a batch epoch) then appends one line with
 * the values stochastic_reconfiguration.cpp:86-91 (gradient_descent.cpp:
 * 47-52 for SGD) and metropolis_sampler.cpp:275-277 log: energy per spin,
 * its standard deviation per spin and the acceptance rate (not with the
 * full sampler), as %.16g separated by ", "; the first line after opening
 * is the header "# Energy, Energy Stddev, AccetpanceRate" (the reference's
 * names, "EnergyStddev" for SGD).  A step rejected as massive or
 * non-finite writes no line, as in main.cpp:600-616.  The file is closed by
 * rbmnqs_log_close or rbmnqs_destroy. */
int rbmnqs_log_open(rbmnqs_handle* h, const char* name, int32_t force);
int rbmnqs_log_close(rbmnqs_handle* h);
/* SR updates applied so far, counting the config's n_updates offset */
int rbmnqs_n_updates(const rbmnqs_handle* h, int64_t* n_updates);

/* ---------------------------------------------- learned proposal network */
/* The proposal network n_in -> h1 -> h2 -> n_out (GELU, BF16 weights and
 * activations, FP32 accumulation; forward, backward and Adam on the GPU)
 * exposed on its own for tests and tools.  No reference counterpart.
 * Parameters are flat [W1 (h1 x n_in), b1, W2 (h2 x h1), b2, W3 (n_out x h2),
 * b3], weights row-major [out][in].  h1, h2 multiples of 64 up to 256;
 * n_in, n_out up to 256. */
typedef struct rbmnqs_mlp rbmnqs_mlp;
int rbmnqs_mlp_create(int32_t n_in, int32_t h1, int32_t h2, int32_t n_out, int32_t max_batch,
                      rbmnqs_mlp** out);
int rbmnqs_mlp_n_params(const rbmnqs_mlp* m, int64_t* n);
int rbmnqs_mlp_set_params(rbmnqs_mlp* m, const float* params);
int rbmnqs_mlp_get_params(rbmnqs_mlp* m, float* params);
/* weights N(0, std), biases zero (seeded) */
int rbmnqs_mlp_init(rbmnqs_mlp* m, float std, uint64_t seed);
/* flip logits [B][n_out] of configurations spins[B][4] (host buffers) */
int rbmnqs_mlp_forward(rbmnqs_mlp* m, const uint32_t* spins, int32_t B, float* logits);
/* loss (1/B) sum softplus(l) - t l against flip masks targets[B][4];
 * gradients in the flat parameter layout (grads may be NULL); apply != 0
 * takes one Adam step with learning rate lr. */
int rbmnqs_mlp_train_step(rbmnqs_mlp* m, const uint32_t* spins, const uint32_t* targets, int32_t B, float lr,
                          int32_t apply, float* loss, float* grads);
/* The same step on the soft-target softmax cross entropy
 * -(1/B) sum_b sum_m t[b][m] log softmax(logits[b])_m, with targets[B][n_out]
 * (rows summing to 1): the loss the learned proposals are trained with. */
int rbmnqs_mlp_train_step_soft(rbmnqs_mlp* m, const uint32_t* spins, const float* targets, int32_t B, float lr,
                               int32_t apply, float* loss, float* grads);
/* tensor of the last pass for tests: 0 a1, 1 a2, 2 z1, 3 z2, 4 g1, 5 g2,
 * 6 g3 (dL/dlogits); [B][cols] as float (out may be NULL to query cols) */
int rbmnqs_mlp_intermediate(rbmnqs_mlp* m, int32_t which, int32_t B, float* out, int32_t* cols);
void rbmnqs_mlp_destroy(rbmnqs_mlp* m);

/* ------------------------------------------- batched independent trainings */
/* Several sessions (different lattices, machines and sizes allowed) advanced
 * together: one CUDA-graph launch runs the whole sample + SR epoch of every
 * session, each on its own branch of the graph so their kernels overlap.
 * The sessions stay owned by the caller and must outlive the batch; while a
 * batch exists, do not run their own epochs concurrently with it.  No
 * reference counterpart (the reference trains one model per process). */
typedef struct rbmnqs_batch rbmnqs_batch;
int rbmnqs_batch_create(rbmnqs_handle* const* sessions, int32_t n, rbmnqs_batch** out);
/* s, o: arrays of n entries (may be NULL). */
int rbmnqs_batch_epoch(rbmnqs_batch* b, rbmnqs_sample_stats* s, rbmnqs_sr_stats* o);
/* kernel nodes of the batch graph (0 before the first epoch) */
int rbmnqs_batch_graph_kernels(rbmnqs_batch* b, int32_t* kernel_nodes);
void* rbmnqs_batch_stream(rbmnqs_batch* b);
void rbmnqs_batch_destroy(rbmnqs_batch* b);
/* Measured special-function (MUFU: ex2/lg2/sin/cos) throughput of the current
 * device in operations per second, from a dependent-chain probe kernel on
 * every SM; the denominator of the sampler kernel's roofline.  No
 * counterpart in the reference (measurement helper). */
int rbmnqs_probe_mufu(int32_t iters, double* ops_per_second);

/* Test hook for failure detection (no reference counterpart; the
 * reference's failure handling is the max|dw| guard and exceptions,
 * abstract_optimizer.cpp:157-159, main.cpp:610-615).  Process-wide:
 *   0  off;
 *   1  the grid barriers of the cooperative solvers (matrix-free CG, the
 *      formed-S cooperative CG and MINRES, the direct solver) wait for one
 *      arrival more than the grid makes and give up after a short bounded
 *      wait: the solve reports status RBMNQS_ERR_CUDA (rbmnqs_sr_stats) and
 *      leaves the weights unchanged;
 *   2  the proposal network's GEMM issues no copies and its bounded wait for
 *      them runs out: calls that run the network fail with RBMNQS_ERR_CUDA.
 * No copy is in flight when a wait gives up and no GPU fault is raised; the
 * context stays usable once the hook is off again.  Captured epoch graphs
 * keep the setting they were captured with. */
int rbmnqs_test_fault(int32_t kind);

/* ------------------------------------------ allocation-free SR solve ---- */
/* No counterpart in the reference.  The same solve as rbmnqs_sr_solve for
 * callers that cannot allocate device memory: code inside a runtime that
 * owns all device memory through its own pool and forbids raw
 * cudaMalloc/cudaFree, and latency-critical loops that cannot take the
 * implicit device-wide synchronisation of cudaMalloc/cudaFree.
 * All buffers are the caller's DEVICE pointers (interleaved complex):
 * O (N x n_params, sample-major), d, F, x (warm start in, solution out,
 * n_params each) and diag (n_params doubles); the work is queued on
 * `stream` (a cudaStream_t, NULL = default stream).  Working memory is one
 * fixed array of (2 + 2) * 256^2 * 16 + 256 bytes (4 MiB + 256 B) that every
 * GPU loading this library holds until the process exits; n_params above
 * RBMNQS_NOALLOC_MAX_PARAMS is rejected with RBMNQS_ERR_ARG.  The first call
 * on a device resolves the array's device address (cudaGetSymbolAddress with
 * that device current), so make that first call before any stream capture.
 * Every call shares the array: calls that overlap on the GPU (other streams,
 * other threads) race and must be serialised by the caller.  When
 * `iterations` or `residual` is non-NULL the call waits for `stream` to read
 * them back.  max_iterations 0 means 2 n_params, a negative value is
 * rejected with RBMNQS_ERR_ARG; rtol 0 means 1e-16.  The array's address is
 * resolved once per device and kept, so the library must not outlive a
 * cudaDeviceReset (or a release of the primary context) of a device it has
 * solved on.  Allocates nothing: no cudaMalloc, cudaFree or allocating
 * library routine. */
#define RBMNQS_NOALLOC_MAX_PARAMS 256
int rbmnqs_sr_solve_noalloc(const double* O, int32_t N, int32_t n_params,
                            int32_t n_neural, const double* d, double norm,
                            const double* F, double* x, double r1, double r2,
                            double rd, const double* diag,
                            int32_t max_iterations, double rtol, void* stream,
                            int32_t* iterations, double* residual);

#ifdef __cplusplus
}
#endif
#endif
