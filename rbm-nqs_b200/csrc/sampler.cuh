// sampler.cuh -- argument block of the fused Metropolis/E_loc/O_k kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pfaffian.cuh"

namespace rbmnqs {

// One local operator of the Hamiltonian (operators::local_op): k sites and a
// CSR view of its 2^k x 2^k matrix; the nonzeros of row `loc` are
// ent[rowptr[rp + loc] .. rowptr[rp + loc + 1]), each stored as the flip
// mask loc ^ col (0 = diagonal) and the complex matrix element.
struct OpDev {
    int k;
    int sites[6];
    int rp;
};

struct MachineDev {
    int n, n_vb, nh, S, T, P, P_neural;
    int symmetric;
    const double2* W64;    // [n][nh] site-major: W64[i*nh + k] = W(i, k)
    const float2* W32;     // FP32 copy of W64
    const double2* hb;     // [nh]
    const double2* vb;     // [n_vb]
    const uint8_t* perm;   // [n][S] perm[f*S + s] = P_s(f)      (symmetric)
    const uint8_t* inv;    // [S][n] inv[s*n + j] = P_s^{-1}(j)  (symmetric)
    const uint8_t* orbit;  // [n_vb][S] orbit[i*S + s] = P_s(basis_i)
    PfDev pf;              // Pfaffian factor (pf.n == 0: none)
};

struct HamDev {
    int n_ops;
    const OpDev* ops;
    const int* rowptr;
    const uint32_t* ent_mask;
    const double2* ent_val;
    int n_rows, n_ents;  // lengths of rowptr and of the entry arrays
};
// Bytes of a HamDev's tables staged in shared memory (0: too large to stage).
int ham_stage_bytes(const HamDev& H);

// Which tables live in shared memory (decided on the host from their sizes).
struct SmemPlan {
    int use_u;  // expanded FP32 flip table U[n+1][TP] (row n all zero)
    int w32;    // FP32 W
    int w64;    // FP64 W
    int u64;    // expanded FP64 table U64[n][TP] for the theta recompute
    int bonds;  // proposal bond list
    int gather; // FP32 sweep with gathered flip rows (the expanded table does not fit)
    int wg;     // gather path: W32 with its zero pad row in shared memory
    int lane_rows;  // gather path, symmetric, nh | 32, T = 32 E (E >= 4): the symmetry
                    // table in lane order (one E-byte load gives a lane its rows)
    int pair;   // table path with two chains per warp
    int ham;    // evaluation: bytes of the Hamiltonian tables staged in shared memory (0: read from L2)
};

struct SamplerArgs {
    MachineDev m;
    HamDev H;
    const MachineDev* md;  // device copies of m and H for the out-of-line
    const HamDev* hd;      // per-sample evaluation
    // proposals (metropolis_sampler.cpp:145-219)
    int n_prop_bonds;
    const int2* prop_bonds;
    uint32_t bond_thr24;  // bond proposal iff (r >> 8) < bond_thr24, i.e.
                          // unit24(r) < bond_flips (0 disables bonds)
    // schedule
    int n_chains, spc, warmup, step;
    const uint32_t* ctl;  // device {epoch, init}: advanced in-stream so a
                          // captured graph can be replayed epoch after epoch
    uint64_t seed;
    // state
    uint32_t* spins;  // [n_chains][4]
    // outputs
    uint32_t* samples;  // [n_chains*spc][4] sampled configurations, evaluated
                        // afterwards by the batched E_loc / O_k kernel
    uint32_t* n_acc;  // [n_chains]
    uint32_t* n_prop; // [n_chains]
    SmemPlan plan;
    // a launch may run a segment of the epoch's sweeps (learned proposals
    // run between segments): sweeps [sweep0, sweep0 + nsweeps) (nsweeps 0 =
    // all), recording samples only when record != 0; chains start fresh only
    // in the segment at sweep 0, and the counters accumulate over segments
    int sweep0 = 0, nsweeps = 0, record = 1;
    // [n_chains][padded T] FP32 theta of each chain's final configuration
    // (after the launch's last FP64 recompute), entry t of chain c at
    // c * padded T + t; written only by the FP32 table and gather paths
    // (sampler_writes_theta), null: not written
    float2* theta_out = nullptr;
    // the same layout read at chain start instead of the FP64 theta
    // recompute, when the caller keeps it current for the configurations
    // (learned moves between sweep launches); used by the lane-ordered
    // gather path, the others recompute; null: recomputed
    const float2* theta_in = nullptr;
};

// The Hamiltonian regrouped by transition for the FP32 evaluation kernel
// (local_op.cpp:31-60): every (operator, flip mask) pair that appears in some
// row of an operator's matrix is one term.  Its value for a configuration is
// vals[voff + loc] (loc = the operator's local bits, bit i = site i of the
// operator), zero where the row has no entry with that mask.  Diagonal
// entries (mask 0) form one term per operator in `diag`.  Sites and flips
// are packed one byte each.
struct TermDev {
    uint32_t flip0;  // flipped sites 0..3
    uint32_t flip1;  // flipped sites 4..5, then nf, k
    uint32_t site0;  // operator sites 0..3
    uint32_t site1;  // operator sites 4..5
    int voff;        // offset of the 2^k values in vals
    int pad[3];
};
struct TermTable {
    int n_terms = 0, n_diag = 0, nf_max = 0, n_vals = 0;
    const TermDev* terms = nullptr;
    const TermDev* diag = nullptr;
    const double2* vals = nullptr;
};

struct EvalArgs {
    MachineDev m;
    HamDev H;
    const MachineDev* md;
    const HamDev* hd;
    const uint32_t* spins;  // [B][4]
    int B;
    double2* logpsi;        // may be null
    double2* eloc;          // may be null
    void* O;                // may be null; float2 or double2 per precision
    const int* flips;       // ratio mode: [B][n_flips]
    int n_flips;
    double2* ratio;         // ratio mode output (log psi'/psi)
    SmemPlan plan;
    TermTable tt;           // terms of H for the FP32 evaluation kernel (n_terms 0 with terms null: none)
    const uint8_t* wrank;   // symmetric machines: row order of W in that kernel's shared memory (null: identity)
};

// Learned-proposal move for every chain (dictionary moves): propose draws a
// move m of the dictionary from q(.|s) = (1 - eps) softmax(logits(s)) +
// eps / D and records log q(m|s) and s' = s with m's sites flipped; accept
// takes the logits at s' for log q(m|s'), forms log|psi(s')/psi(s)| and
// applies the Metropolis-Hastings test.  targets writes the network's
// training targets at configurations spins[0..B).
struct LearnedArgs {
    MachineDev m;
    int n_chains;
    uint32_t* spins;        // [n_chains][4] current configurations
    uint32_t* prop;         // [n_chains][4] proposed configurations
    int* mv;                // [n_chains] proposed move
    float* qfw;             // [n_chains] log q(m|s)
    const float* logits;    // [rows][ldl] network output
    int ldl;
    int n_moves;            // D (<= 256)
    const uint32_t* mmask;  // [D][4] flip masks
    const uint32_t* mflip;  // [D][2] flipped sites (bytes 0..5) and their count (byte 6)
    const uint32_t* ctl;    // {epoch, init}
    uint64_t seed;
    uint32_t move;          // move index within the epoch (Philox counter)
    uint32_t* n_acc;        // [n_chains] accepted learned moves (epoch)
    uint32_t* n_try;        // [n_chains] learned moves tried (epoch)
    float eps;              // uniform part of the proposal
    float* targets;         // [B][D] training targets (targets kernel)
    int B;
    // [n_chains][padded T] FP32 theta of spins, kept current by accept (an
    // accepted move stores its theta'); null: accept recomputes theta from
    // the configuration in FP64
    float2* theta = nullptr;
};
cudaError_t launch_learned_propose(const LearnedArgs& a, cudaStream_t st);
cudaError_t launch_learned_accept(const LearnedArgs& a, cudaStream_t st);
cudaError_t launch_learned_targets(const LearnedArgs& a, cudaStream_t st);
// a.theta <- FP32 theta of a.spins (FP64 recompute from the configuration)
cudaError_t launch_learned_theta(const LearnedArgs& a, cudaStream_t st);
// chains from Philox stream 1 (as the sweep kernel's fresh start) when ctl[1] is set
cudaError_t launch_init_chains(uint32_t* spins, int n, int n_chains, const uint32_t* ctl, uint64_t seed,
                               cudaStream_t st);
// samples[c * spc + j] = spins[c]
cudaError_t launch_record(const uint32_t* spins, int n_chains, int spc, int j, uint32_t* samples, cudaStream_t st);
// acceptance of the learned moves -> *out (device)
cudaError_t launch_learned_rate(const uint32_t* n_acc, const uint32_t* n_try, int n_chains, double* out,
                                cudaStream_t st);

// Launch helpers implemented in sampler.cu
int sampler_smem_bytes(const MachineDev& m, int fp64, int warps, const SmemPlan& plan, int n_bonds);
int eval_smem_bytes(const MachineDev& m, int fp64, int warps, const SmemPlan& plan);
// Plan + launch shape of the sampler for this machine and chain count:
// one persistent block per SM with enough warps to hold every chain when
// registers allow.
struct SamplerShape {
    SmemPlan plan;
    int warps_per_block;
    int blocks;
    int smem;
};
// max_wpb > 0 caps the warps per block (launch-shape autotuning); pair_mode
// 1 asks for two chains per warp where the table path allows it (else, and
// by default, one chain per warp).
cudaError_t plan_sampler(const MachineDev& m, int fp64, int n_chains, int n_bonds, SamplerShape* out,
                         int max_wpb = 0, int pair_mode = -1);
cudaError_t launch_sampler(const SamplerArgs& a, int fp64, const SamplerShape& shape, cudaStream_t st);
// The sweeps of several sessions in one launch per entries-per-lane class
// (a batch): one descriptor per session, its blocks [block0, block0 +
// blocks) of the launch.
constexpr int kBatchSweepWarps = 8;
struct BatchSweepDesc {
    SamplerArgs a;  // the session's arguments with its plan for kBatchSweepWarps warps
    int block0, blocks;
    int E;          // entries per lane
    int path;       // 0 expanded flip table, 1 gathered rows
};
// Fills d->a.plan, E, path and blocks (d->a must hold the session's other
// arguments) and the shared-memory bytes; false when the session's sweep
// cannot run in the batch launch (FP64, Pfaffian, more than 8 entries per
// lane, or tables that do not fit with kBatchSweepWarps warps).
bool sampler_batch_plan(const MachineDev& m, int fp64, int n_chains, int n_bonds, BatchSweepDesc* d, int* smem);
cudaError_t launch_sampler_batch(int E, const BatchSweepDesc* desc_dev, int nprob, int blocks, int smem,
                                 cudaStream_t st);
// whether the sweep path of this shape writes SamplerArgs::theta_out
bool sampler_writes_theta(const MachineDev& m, int fp64, const SamplerShape& shape);
cudaError_t launch_eval(const EvalArgs& a, int fp64, int warps_per_block, cudaStream_t st);
// The FP32 evaluation kernel (E_loc and O_k from the term table, no Pfaffian
// factor).  cudaErrorNotSupported when the machine or the table does not fit
// it; launch_eval then runs eval_kernel.
cudaError_t launch_eloc_fast(const EvalArgs& a, cudaStream_t st);
int elements_per_lane(int T);
cudaError_t launch_advance(uint32_t* ctl, int reinit, cudaStream_t st);
cudaError_t launch_mufu_probe(float* out, int iters, int blocks, cudaStream_t st);

}  // namespace rbmnqs
