// sr.cuh -- device-side state blocks and launchers of the SR kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <string>

namespace rbmnqs {

// Message returned by rbmnqs_last_error() on the calling thread.
void set_last_error(const std::string& msg);

// Per-epoch statistics written on the device, read back once per epoch.
struct EpochStatsDev {
    double2 energy;
    double var, var_binned, tau, stddev, acceptance;
    int finite;
};

// decay_t state of lr, reg1, reg2, deltareg1 (indices 0..3).
struct ScheduleDev {
    double value[4], min[4], decay[4];
    int min_reached[4];
};

struct CgResultDev {
    int iterations;
    int status;
    double residual;
    double max_dw;
    // MINRES-QLP: stopping reason (istop 1-14 of zminresqlpModule.f90), the
    // condition estimate Acond and the number of QLP iterations
    int istop;
    int qlp_iterations;
    double acond;
};

// w: optional per-sample weights, wsum: their total (device scalar)
cudaError_t launch_moments(const void* O, int fp64, const double2* E, int N, int P, int nblk, double2* pd,
                           double2* pf, double2* pe, double2* d, double2* F, double2* emean, cudaStream_t st,
                           const double* w = nullptr, const double* wsum = nullptr);
// E_loc statistics (one block per bin; n_bins <= kMaxBins and divides N).
// scratch: energy_stats_scratch_doubles(n_bins) doubles, zero before the
// first launch (each launch leaves it zero).
constexpr int kMaxBins = 64;
inline size_t energy_stats_scratch_doubles(int n_bins) { return 4 * (size_t)n_bins + 1; }
cudaError_t launch_energy_stats(const double2* E, int N, int n_bins, const double2* emean, const uint32_t* nacc,
                                const uint32_t* nprop, int n_chains, double* scratch, EpochStatsDev* out,
                                cudaStream_t st);
cudaError_t launch_mean(const double2* E, int N, double2* mu, cudaStream_t st);
int gram_splits(int N, int P);
cudaError_t launch_gram_fp64(const void* O, int fp64, const double2* d, int N, int P, int nks, double2* part,
                             double2* S, cudaStream_t st);
// direct != 0: the direct solver's regularisation (direct_solver.cpp:42-49),
// the diagonal scaled by (1 + r1) ((1 + r1) + rd) instead of adding r1 diag
cudaError_t launch_solve_prep(const double2* G, int N, double norm, const double2* d, const double* diag, int P,
                              int n_neural, double r1, double r2, double rd, double2* Sreg, cudaStream_t st,
                              int direct = 0);
cudaError_t launch_schedule(ScheduleDev* s, cudaStream_t st);
// vfac: optional device scalar replacing the N / (N - 1) variance factor
cudaError_t launch_regularize(const double2* S, int P, int n_neural, int N, const ScheduleDev* sch, double* diag,
                              double2* Sreg, double* max_diag, cudaStream_t st, int direct = 0,
                              const double* vfac = nullptr);
cudaError_t launch_cg(const double2* A, const double2* b, double2* x, int P, int max_it, double rtol,
                      CgResultDev* res, cudaStream_t st);
// Update-step plugins (optimizer/plugin.cpp:29-115): state on the device.
struct PluginDev {
    int type;            // 0 none, 1 adam, 2 momentum, 3 heun
    double beta1, beta2, eps;  // adam
    double alpha, dialup;      // momentum
    double dup;                // momentum dial-up factor state
    int t;                     // adam step counter (starts at 1)
    double2* m;                // [P] first moment / momentum / heun delta
    double* wr;                // [P] adam second moment, real parts
    double* wi;                // [P] adam second moment, imaginary parts
    // heun
    double heps;               // optimizer.heun.eps
    int gstat;                 // guard status of the first step
    double gmax;               // its max |dw|
    double2 dd;                // d^T delta
    double nrm2;               // |delta|^2
    double* part;              // [kHeunBlocks] partial sums of |O delta - d^T delta|^2
};
constexpr int kHeunBlocks = 296;
// heun_plugin::apply (plugin.cpp:87-115) around a second sample + solve:
// begin: guard on x1, delta = lr/2 x1, w -= delta;
// finish: delta = (delta - lr/2 x2) / 6, err from O (metric, SR) or |delta|
// (SGD), x = x2 (cbrt(eps / err) - 1/2) lr, w -= x.
cudaError_t launch_heun_begin(double2* params, const double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                              PluginDev* plug, cudaStream_t st);
cudaError_t launch_heun_finish(double2* params, double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                               PluginDev* plug, const void* O, int fp64, const double2* d, int N, int metric,
                               cudaStream_t st);
// decay the regularisation schedules only (a second gradient() call)
cudaError_t launch_schedule_regs(ScheduleDev* s, cudaStream_t st);
// SGD direction (gradient_descent.cpp:42-60): x = F with Re(x) / real_factor
cudaError_t launch_sgd_direction(const double2* F, double2* x, int P, double real_factor, CgResultDev* res,
                                 cudaStream_t st);
cudaError_t launch_update(double2* params, double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                          PluginDev* plug, cudaStream_t st);
cudaError_t launch_update(double2* params, double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                          cudaStream_t st);
// Matrix-free CG (cg_mfree.cu) for parameter counts without a formed S.
struct MfreeSync {
    uint32_t count, gen;  // count: arrivals so far (grows by the grid's blocks per barrier); gen unused
    int bad;
    uint32_t extra;     // arrivals beyond the grid's blocks a barrier waits for (0; 1 under test fault 1)
    uint32_t spin_cap;  // polls before a waiting block gives up (0: kBarrierSpin)
};
// Barrier state for a cooperative launch: zero, or under test fault 1 an
// extra arrival that never comes and a short wait limit.
cudaError_t launch_init_sync(MfreeSync* sync, cudaStream_t st);
// Process-wide test hook (rbmnqs_test_fault): 0 none, 1 cooperative-solve
// barriers never complete, 2 the proposal network's GEMM copies are never
// issued; the bounded waits then run out and the calls report an error.
int test_fault();
// Direct solve (direct.cu, direct_solver.cpp:31-59) of the regularised
// Hermitian positive definite Sreg (P x P, overwritten by its Cholesky
// factor): x = Sreg^-1 F.  work: P entries; sync: barrier state.
cudaError_t launch_direct_solve(double2* Sreg, const double2* F, double2* x, int P, double2* work, MfreeSync* sync,
                                CgResultDev* res, cudaStream_t st);
// Full enumeration (full_sampler.cpp:43-186): every state once, weighted by
// p = |psi|^2 (scaled by exp(-max 2 Re log psi), which the normalisation
// removes).  full.cu.
struct FullStatsDev {
    double mx;    // max over states of 2 Re log psi
    double W;     // sum p
    double W2;    // sum p^2
    double vfac;  // W / (W - W2 / W): the weighted unbiased-variance factor
};
// samples[k] = state k of the enumeration order: blocks b < 2^bits of the
// low bits, Gray code over the high n - bits bits within each block
cudaError_t launch_full_states(uint32_t* samples, int n, int bits, cudaStream_t st);
// p[k] from log psi, and the totals; part: 2 * kFullBlocks doubles
constexpr int kFullBlocks = 296;
cudaError_t launch_full_weights(const double2* logpsi, int64_t N, double* p, double* part, FullStatsDev* fs,
                                cudaStream_t st);
// O[k] <- sqrt(N p_k / W) (O[k] - d): the weighted, centred samples whose
// plain Gram (1/N) O^H O is S
cudaError_t launch_full_center(void* O, int fp64, const double* p, const FullStatsDev* fs, const double2* d,
                               int64_t N, int P, cudaStream_t st);
// energy aggregator with weights (aggregator.cpp:190-239): mean, weighted
// unbiased variance, binned variance over n_bins consecutive blocks, tau
cudaError_t launch_energy_stats_weighted(const double2* E, const double* p, int64_t N, int n_bins,
                                         const double2* emean, const FullStatsDev* fs, EpochStatsDev* out,
                                         cudaStream_t st);
// weighted mean sum p E / W into *mu
cudaError_t launch_wmean(const double2* E, const double* p, int64_t N, const FullStatsDev* fs, double2* mu,
                         cudaStream_t st);
// normalised state vector psi[num(state k)] = exp(log psi_k - mx / 2) / sqrt(W)
cudaError_t launch_full_state_vector(const double2* logpsi, const uint32_t* samples, int64_t N,
                                     const FullStatsDev* fs, double2* psi, cudaStream_t st);
struct MfreePlan {
    int blocks, nseg, lseg, diag_blocks;
};
struct MfreeWork {
    const double2* S;  // formed regularised S (dense cooperative mode) or null
    int minres;        // 0: CG (cg1), 1: MINRES-QLP from x0 = 0 (rtol bounds the relative residual)
    double2 *r, *p, *Ap, *tmpN, *partA, *zpart;
    double2 *R1, *R2, *w1, *w2, *v;  // MINRES vectors
    double *dpart, *maxpart;
    MfreeSync* sync;
    int nseg, lseg;
};
// Several matrix-free CG systems (cg1 semantics) in one cooperative launch
// (cg_multi.cu).  One descriptor per system; O is float2 or double2 (one
// precision per launch); r, p0, p1, Ap hold P entries, v N entries.
constexpr int kCgMultiMax = 64;
struct CgMultiProb {
    const void* O;
    const double2* d;
    const double2* F;
    double2* x;
    const double* diag;
    const double* max_diag;
    const ScheduleDev* sch;
    CgResultDev* res;
    double2 *r, *p0, *p1, *Ap, *v;
    double norm, rtol;
    int N, P, n_neural, max_it;
    // filled by cg_multi_units: first unit costs and first tile of the system
    long long row_cost0, tile_cost0;
    int tile0, pad;
};
// per-tile partial sums (d . b, p^H A p, ||r||^2) of all systems and the
// barrier state; row_cost / tile_cost from cg_multi_units
struct CgMultiScratch {
    double2* tdb;
    double2* tpap;
    double* trs;
    MfreeSync* sync;
    long long row_cost, tile_cost;
};
// Fills the unit offsets of the descriptors; returns the total tile count
// (the length of each partial-sum array).
int cg_multi_units(CgMultiProb* probs, int nprob, long long* row_cost, long long* tile_cost);
// cooperative grid size of the multi-system kernel on this device
cudaError_t cg_multi_blocks(int* blocks);
cudaError_t launch_cg_multi(const CgMultiProb* probs_dev, int nprob, int fp64, const CgMultiScratch& s, int blocks,
                            cudaStream_t st);
// The direct solver above the formed-S sizes (woodbury.cu): S_reg x = F
// through the N x N system K = N I + Abar Lambda^-1 Abar^H of the Woodbury
// identity, K factored by launch_direct_solve.
struct WoodburyWork {
    double2* K;  // [N][N]
    double2 *y, *u, *z, *work;
    double *winv, *spp;
    MfreeSync* sync;
};
constexpr int kWoodburyMaxN = 4096;
size_t woodbury_work_bytes(int N, int P);
WoodburyWork woodbury_carve(void* base, int N, int P);
// x = S_reg^-1 F; the regularisation from sch (device schedules) or, when
// sch is null, r1, r2, rd; S_pp from O itself, the r2 shift from max_diag
// (the maximum of the variance diagonal)
cudaError_t launch_woodbury_solve(const void* O, int fp64, const double2* d, int N, int P, int n_neural,
                                  double norm, const double2* F, double2* x, const double* max_diag,
                                  const ScheduleDev* sch, double r1, double r2, double rd, const WoodburyWork& w,
                                  CgResultDev* res, cudaStream_t st);
cudaError_t mfree_plan(int N, int P, MfreePlan* pl);
size_t mfree_work_bytes(int N, int P, const MfreePlan& pl);
MfreeWork mfree_carve(void* base, int N, int P, const MfreePlan& pl);
// diag = unbiased var(O) per parameter and its maximum (device scalar)
// vfac: optional device scalar: diag = (sum |O - d|^2 / N) vfac instead of / (N - 1)
cudaError_t launch_var_diag(const void* O, int fp64, const double2* d, int N, int P, const MfreePlan& pl,
                            const MfreeWork& w, double* diag, double* max_diag, cudaStream_t st,
                            const double* vfac = nullptr);
// CG on a formed regularised S (P x P) with the cooperative kernel: for P
// whose S does not fit the shared-memory cluster solve.  Work from
// mfree_plan(1, P) / mfree_carve.
cudaError_t launch_cg_dense_coop(const double2* A, const double2* b, double2* x, int P, int max_it, double rtol,
                                 const MfreePlan& pl, const MfreeWork& w, CgResultDev* res, cudaStream_t st);
// whether the 8-CTA shared-memory CG holds S for this P
bool cg_cluster_fits(int P);
// max of a given diag (explicit-solve entry)
cudaError_t launch_max_diag(const double* diag, int P, double* max_diag, cudaStream_t st);
// r1 / r2 / rd from sch when non-null, else the explicit values
cudaError_t launch_cg_mfree(const void* O, int fp64, const double2* d, double norm, int N, int P, int n_neural,
                            const double2* F, double2* x, const double* diag, const double* max_diag,
                            const ScheduleDev* sch, double r1, double r2, double rd, int max_it, double rtol,
                            const MfreePlan& pl, const MfreeWork& w, CgResultDev* res, cudaStream_t st);
cudaError_t launch_unpack(const double2* params, int n, int n_vb, int nh, double2* vb, double2* hb, double2* W64,
                          float2* W32, cudaStream_t st);

}  // namespace rbmnqs
