// capi.cu -- the C ABI (include/rbmnqs_b200.h): models, the GPU session that
// plays the role of the reference's metropolis_sampler + stochastic_
// reconfiguration + cg_solver for one GPU, and the parity entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../host/model.hpp"
#include "ed.cuh"
#include "rbmnqs_b200.h"
#include "gram_tc.cuh"
#include "mlp.cuh"
#include "sampler.cuh"
#include "sr.cuh"

using rbmnqs::cplx;

struct rbmnqs_model {
    rbmnqs::model m;
};

// Largest parameter count with a formed P x P matrix S (dense Gram + CG in
// shared memory); above it the matrix-free operator is used.
constexpr int kDenseMax = 2048;

namespace {

thread_local std::string g_err;

struct Fail {
    int code;
    std::string msg;
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Fail{RBMNQS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

template <typename F> int guard(F&& f) {
    try {
        f();
        return RBMNQS_OK;
    } catch (const Fail& e) {
        g_err = e.msg;
        return e.code;
    } catch (const std::exception& e) {
        g_err = e.what();
        return RBMNQS_ERR_ARG;
    }
}

void require(bool c, const std::string& msg, int code = RBMNQS_ERR_ARG) {
    if (!c) throw Fail{code, msg};
}

template <typename T> struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        release();
        n = count;
        if (count) ck(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
};

// Hamiltonian operators in the device CSR form (see OpDev).
struct HamHost {
    std::vector<rbmnqs::OpDev> ops;
    std::vector<int> rowptr;
    std::vector<uint32_t> mask;
    std::vector<double2> val;
};

HamHost build_ham(const std::vector<rbmnqs::local_op>& ops) {
    HamHost h;
    for (auto& op : ops) {
        rbmnqs::OpDev d;
        d.k = op.k;
        for (int i = 0; i < 6; i++) d.sites[i] = op.acts_on[i];
        d.rp = (int)h.rowptr.size();
        const int dim = 1 << op.k;
        for (int r = 0; r < dim; r++) {
            h.rowptr.push_back((int)h.mask.size());
            for (int c = 0; c < dim; c++) {
                const cplx v = op.mat[(size_t)r * dim + c];
                if (v == cplx(0, 0)) continue;
                h.mask.push_back((uint32_t)(r ^ c));
                h.val.push_back(make_double2(v.real(), v.imag()));
            }
        }
        h.rowptr.push_back((int)h.mask.size());
        h.ops.push_back(d);
    }
    return h;
}

// The operators regrouped by transition for the FP32 evaluation kernel
// (TermDev): one term per (operator, nonzero flip mask), with the matrix
// element of every local configuration (zero where the row lacks the mask),
// and one diagonal term per operator with diagonal entries.
struct TermHost {
    std::vector<rbmnqs::TermDev> terms, diag;
    std::vector<double2> vals;
    int nf_max = 0;
};

TermHost build_terms(const std::vector<rbmnqs::local_op>& ops) {
    TermHost t;
    auto pack4 = [](const int* v, int cnt) {
        uint32_t w = 0;
        for (int i = 0; i < cnt && i < 4; i++) w |= (uint32_t)(v[i] & 0xff) << (8 * i);
        return w;
    };
    for (const auto& op : ops) {
        const int dim = 1 << op.k;
        int sites[6] = {0, 0, 0, 0, 0, 0};
        for (int i = 0; i < op.k; i++) sites[i] = op.acts_on[i];
        std::vector<uint32_t> masks;  // distinct masks in increasing order
        for (int r = 0; r < dim; r++)
            for (int c = 0; c < dim; c++)
                if (op.mat[(size_t)r * dim + c] != cplx(0, 0)) masks.push_back((uint32_t)(r ^ c));
        std::sort(masks.begin(), masks.end());
        masks.erase(std::unique(masks.begin(), masks.end()), masks.end());
        for (uint32_t mk : masks) {
            rbmnqs::TermDev d{};
            int fl[6] = {0, 0, 0, 0, 0, 0}, nf = 0;
            for (int i = 0; i < op.k; i++)
                if ((mk >> i) & 1u) fl[nf++] = sites[i];
            d.flip0 = pack4(fl, 4);
            d.flip1 = (uint32_t)(fl[4] & 0xff) | ((uint32_t)(fl[5] & 0xff) << 8) | ((uint32_t)nf << 16) |
                      ((uint32_t)op.k << 24);
            d.site0 = pack4(sites, 4);
            d.site1 = (uint32_t)(sites[4] & 0xff) | ((uint32_t)(sites[5] & 0xff) << 8);
            d.voff = (int)t.vals.size();
            for (int r = 0; r < dim; r++) {
                const cplx v = op.mat[(size_t)r * dim + (r ^ (int)mk)];
                t.vals.push_back(make_double2(v.real(), v.imag()));
            }
            if (mk == 0) {
                t.diag.push_back(d);
            } else {
                t.terms.push_back(d);
                t.nf_max = std::max(t.nf_max, nf);
            }
        }
    }
    return t;
}

// Row order of W in the shared memory of the FP32 evaluation kernel
// (symmetric machines).  The kernel reads 16-byte pieces of row P_s(f) for
// the symmetry indices s of eight consecutive lanes at a time; a row of rank
// q starts at 16-byte unit q u (u odd), i.e. in bank group (q u) mod 8.  Two
// orders are scored by the number of load wavefronts they cost over every
// flipped site (the ideal is one per eight lanes): the identity, and the
// order in which the symmetry orbits of the sites enumerate the rows
// (rank(P_s(rep)) consecutive in s), which for translation groups gives
// consecutive lanes consecutive ranks.  The cheaper one is returned.
std::vector<uint8_t> eval_row_order(const std::vector<std::vector<int>>& perm, int n, int nh) {
    const int S = (int)perm.size();
    std::vector<uint8_t> ident(n);
    for (int r = 0; r < n; r++) ident[r] = (uint8_t)r;
    const int kb = nh % 4 == 0 ? 4 : (nh % 2 == 0 ? 2 : 1);
    if (kb == 1 || S == 0) return ident;
    int u = (8 * nh + 15) / 16;
    if ((u & 1) == 0) u++;
    const int G = nh * S / kb, NGK = nh / kb, loads = kb == 4 ? 2 : 1;
    auto cost = [&](const std::vector<uint8_t>& rank) {
        long c = 0;
        for (int f = 0; f < n; f++)
            for (int g0 = 0; g0 < G; g0 += 8)
                for (int h = 0; h < loads; h++) {
                    int cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0}, mx = 0;
                    for (int g = g0; g < std::min(G, g0 + 8); g++) {
                        const int sidx = g / NGK, k0 = (g % NGK) * kb;
                        const int unit = rank[perm[sidx][f]] * u + (8 * k0) / 16 + h;
                        mx = std::max(mx, ++cnt[unit & 7]);
                    }
                    c += mx;
                }
        return c;
    };
    std::vector<uint8_t> orb(n, 0);
    std::vector<char> used(n, 0);
    int next = 0;
    for (int rep = 0; rep < n && next < n; rep++) {
        if (used[rep]) continue;
        for (int sidx = 0; sidx < S; sidx++) {
            const int r = perm[sidx][rep];
            if (!used[r]) {
                used[r] = 1;
                orb[r] = (uint8_t)next++;
            }
        }
    }
    return cost(orb) < cost(ident) ? orb : ident;
}

}  // namespace

void rbmnqs::set_last_error(const std::string& msg) { g_err = msg; }

namespace {
std::atomic<int> g_test_fault{0};
}
int rbmnqs::test_fault() { return g_test_fault.load(std::memory_order_relaxed); }

// Device copy of a TermHost and its view for the evaluation kernel.
struct TermBufs {
    DevBuf<rbmnqs::TermDev> terms, diag;
    DevBuf<double2> vals;
    rbmnqs::TermTable tt{};
    void upload(const TermHost& t) {
        terms.alloc(std::max<size_t>(1, t.terms.size()));
        diag.alloc(std::max<size_t>(1, t.diag.size()));
        vals.alloc(std::max<size_t>(1, t.vals.size()));
        if (!t.terms.empty())
            ck(cudaMemcpy(terms.p, t.terms.data(), t.terms.size() * sizeof(rbmnqs::TermDev), cudaMemcpyHostToDevice),
               "c");
        if (!t.diag.empty())
            ck(cudaMemcpy(diag.p, t.diag.data(), t.diag.size() * sizeof(rbmnqs::TermDev), cudaMemcpyHostToDevice),
               "c");
        if (!t.vals.empty())
            ck(cudaMemcpy(vals.p, t.vals.data(), t.vals.size() * sizeof(double2), cudaMemcpyHostToDevice), "c");
        tt.n_terms = (int)t.terms.size();
        tt.n_diag = (int)t.diag.size();
        tt.nf_max = t.nf_max;
        tt.n_vals = (int)t.vals.size();
        tt.terms = terms.p;
        tt.diag = diag.p;
        tt.vals = vals.p;
    }
};

// One observable (evaluation mode) as a one-operator Hamiltonian table.
struct ObsDev {
    DevBuf<rbmnqs::OpDev> ops;
    DevBuf<int> rowptr;
    DevBuf<uint32_t> mask;
    DevBuf<double2> val;
    DevBuf<rbmnqs::HamDev> hd;
    rbmnqs::HamDev H{};
    TermBufs terms;
};

struct rbmnqs_handle {
    rbmnqs_config cfg{};
    rbmnqs::model model;
    int n = 0, n_vb = 0, nh = 0, S = 0, T = 0, P = 0, P_neural = 0, N = 0, n_bins = 1;
    int fp64 = 0, wpb = 8, w_in_smem = 1;
    rbmnqs::SamplerShape shape{};
    uint32_t bond_thr24 = 0;
    int gram_ks = 1, mom_blocks = 1;
    cudaStream_t st = nullptr;

    DevBuf<double2> params, vb, hb, W64, x;
    DevBuf<float2> W32;
    DevBuf<uint8_t> perm, inv, orbit;
    DevBuf<uint8_t> wrank;  // row order of W in the FP32 evaluation kernel (symmetric machines)
    DevBuf<rbmnqs::OpDev> ops;
    DevBuf<int> rowptr;
    DevBuf<uint32_t> emask;
    DevBuf<double2> eval;
    DevBuf<int2> bonds;
    DevBuf<uint32_t> spins, nacc, nprop, ctl, samples;
    DevBuf<double2> E;
    DevBuf<unsigned char> O;
    DevBuf<double2> pd, pf, pe, d, F, emean, part, Sm, Sreg;
    DevBuf<double> diag, maxdiag;
    DevBuf<rbmnqs::ScheduleDev> sched;
    DevBuf<rbmnqs::MachineDev> mdev;
    DevBuf<rbmnqs::HamDev> hdev;
    TermBufs terms;  // the Hamiltonian as terms (FP32 evaluation kernel)
    DevBuf<rbmnqs::CgResultDev> cgres;
    // update plugin (adam / momentum) state
    DevBuf<rbmnqs::PluginDev> plug;
    DevBuf<double2> plug_m;
    DevBuf<double> plug_wr, plug_wi, plug_part;
    DevBuf<rbmnqs::EpochStatsDev> stats_first;
    // full enumeration: log psi, weights p, reduction partials, totals, a zero d
    bool full = false;
    DevBuf<double2> lpsi, dzero;
    DevBuf<double> pw, fpart;
    DevBuf<rbmnqs::FullStatsDev> fstat;
    const double* fstat_W() const {
        return reinterpret_cast<const double*>(reinterpret_cast<const char*>(fstat.p) +
                                               offsetof(rbmnqs::FullStatsDev, W));
    }
    const double* fstat_vfac() const {
        return reinterpret_cast<const double*>(reinterpret_cast<const char*>(fstat.p) +
                                               offsetof(rbmnqs::FullStatsDev, vfac));
    }
    // direct solver: barrier state and triangular-solve work vector
    DevBuf<rbmnqs::MfreeSync> dsync;
    DevBuf<double2> dwork;
    DevBuf<rbmnqs::EpochStatsDev> stats;
    DevBuf<double> estat;  // per-bin partials and ticket of the energy statistics
    // matrix-free SR (n_params above the dense limit): no S is formed
    bool mfree = false;
    bool coop_dense = false;  // formed S too large for the cluster CG: cooperative grid CG
    rbmnqs::MfreePlan mfp{};
    rbmnqs::MfreeWork mfw{};
    // matrix-free CG (solver 0) by the multi-system kernel: this session's
    // descriptor, its tile partial sums and grid size; a batch merges the
    // descriptors of its sessions into one launch
    bool multi_cg = false;
    // set while a batch captures its graph: this session's sweep runs in the
    // batch's sweep launch, enqueue_sample skips its own
    bool batch_swept = false;
    DevBuf<rbmnqs::CgMultiProb> cgm;
    DevBuf<double2> cgm_t2;
    DevBuf<double> cgm_t1;
    rbmnqs::CgMultiScratch cgms{};
    int cgm_blocks = 0;
    DevBuf<unsigned char> mfbuf;
    // direct solver above the formed-S sizes: the sample-space (Woodbury) work
    DevBuf<unsigned char> wbbuf;
    rbmnqs::WoodburyWork wbw{};
    // evaluation-mode observables, their per-sample values and statistics
    std::vector<std::unique_ptr<ObsDev>> obs;
    DevBuf<double2> obsE, obsMean;
    DevBuf<rbmnqs::EpochStatsDev> obsStats;
    // learned proposals: network, proposed configurations, masks, counters
    std::unique_ptr<rbmnqs::Mlp> net;
    DevBuf<uint32_t> lprop, lacc, ltry;
    DevBuf<int> lmv;
    DevBuf<float> lqfw, lloss, ltgt;
    DevBuf<double> lrate;
    // FP32 theta of each chain [n_chains][padded T]: handed from the sweep
    // kernel (or the theta kernel) to the learned moves
    DevBuf<float2> lth;
    // move dictionary: flip masks [D][4], flip lists [D][2]; training batch
    int n_moves = 0, train_batch = 0;
    DevBuf<uint32_t> dmask, dflip;
    // Pfaffian factor: class matrix, derivative pairs, unscramble buffers
    int pf_n = 0, pf_indep = 0;
    DevBuf<int16_t> pf_bs;
    DevBuf<int> pf_ptr;
    DevBuf<uint32_t> pf_pairs;
    DevBuf<double2> pf_scratch;
    // tensor-core Gram (mixed precision): FP16 hi / lo planes, FP32 split-K
    // partial tiles, pipeline error flag
    bool gram_tc = false;
    rbmnqs::GramTC gtc;
    DevBuf<float> gplanes, gpart;
    DevBuf<int> gerr;
    int n_ops = 0, n_prop_bonds = 0;
    uint32_t epoch = 0;
    bool sampled = false;
    int64_t n_updates = 0;  // rbm_base::n_updates_ (offset + applied SR updates)
    rbmnqs::CgResultDev last_solve{};  // the last SR solve's result (rbmnqs_solve_info)
    // training log <name>.log (rbmnqs_log_open): one line per applied update
    struct LogFile {
        FILE* f = nullptr;
        bool first = true;  // the header line precedes the first line written
        ~LogFile() {
            if (f) fclose(f);
        }
    } log;

    cudaGraphExec_t graph = nullptr;
    int graph_kernels = 0;
    static constexpr int kStages = 6;  // sampler, eval, moments+stats, gram+reg, cg, update
    cudaEvent_t ev[kStages + 1] = {};
    bool timing = false;
    double stage_ms[kStages] = {};
    int64_t stage_launches[kStages] = {};

    // pinned host copies of the per-epoch results, read back with one
    // stream synchronisation
    struct Readback {
        rbmnqs::EpochStatsDev stats;
        rbmnqs::CgResultDev cg;
        rbmnqs::ScheduleDev sched;
        int gerr;
        double lrate;
        float lloss;
        int nerr;  // proposal network pipeline error flag
    };
    Readback* rb = nullptr;
    ~rbmnqs_handle() {
        if (rb) cudaFreeHost(rb);
        if (graph) cudaGraphExecDestroy(graph);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (st) cudaStreamDestroy(st);
    }

    rbmnqs::MachineDev machine() const {
        rbmnqs::MachineDev m{};
        m.n = n;
        m.n_vb = n_vb;
        m.nh = nh;
        m.S = S;
        m.T = T;
        m.P = P;
        m.P_neural = P_neural;
        m.symmetric = cfg.rbm_type == 1;
        m.W64 = W64.p;
        m.W32 = W32.p;
        m.hb = hb.p;
        m.vb = vb.p;
        m.perm = perm.p;
        m.inv = inv.p;
        m.orbit = orbit.p;
        if (pf_n) {
            m.pf.n = pf_n;
            m.pf.n_indep = pf_indep;
            m.pf.refresh = cfg.pfaffian_refresh;
            m.pf.bs = pf_bs.p;
            m.pf.fs = params.p + P_neural;
            m.pf.pair_ptr = pf_ptr.p;
            m.pf.pairs = pf_pairs.p;
            m.pf.scratch = pf_scratch.p;
        }
        return m;
    }
    rbmnqs::HamDev ham() const {
        rbmnqs::HamDev H{};
        H.n_ops = n_ops;
        H.ops = ops.p;
        H.rowptr = rowptr.p;
        H.ent_mask = emask.p;
        H.ent_val = eval.p;
        H.n_rows = (int)rowptr.n;
        H.n_ents = (int)emask.n;
        return H;
    }
    size_t osize() const { return fp64 ? sizeof(double2) : sizeof(float2); }

    // stage timing event: an external event node inside a graph capture, a
    // plain record on the stream otherwise
    void mark(int i) {
        if (!timing) return;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        ck(cudaStreamIsCapturing(st, &cs), "capture status");
        if (cs == cudaStreamCaptureStatusActive)
            ck(cudaEventRecordWithFlags(ev[i], st, cudaEventRecordExternal), "event");
        else
            ck(cudaEventRecord(ev[i], st), "event");
    }

    // --- the epoch pieces -------------------------------------------------
    rbmnqs::SamplerArgs sampler_args() const {
        rbmnqs::SamplerArgs a{};
        a.m = machine();
        a.H = ham();
        a.md = mdev.p;
        a.hd = hdev.p;
        a.n_prop_bonds = n_prop_bonds;
        a.prop_bonds = bonds.p;
        a.bond_thr24 = bond_thr24;
        a.n_chains = cfg.n_chains;
        a.spc = cfg.samples_per_chain;
        a.warmup = cfg.warmup;
        a.step = cfg.step;
        a.ctl = ctl.p;
        a.seed = cfg.seed;
        a.spins = spins.p;
        a.samples = samples.p;
        a.n_acc = nacc.p;
        a.n_prop = nprop.p;
        return a;
    }
    // evaluation tables: W in shared memory when it fits, the operator
    // tables staged in shared memory when they fit
    rbmnqs::SmemPlan eval_plan() const {
        rbmnqs::SmemPlan p{};
        p.w32 = w_in_smem;
        p.ham = rbmnqs::ham_stage_bytes(ham());
        return p;
    }
    rbmnqs::EvalArgs eval_args() const {
        rbmnqs::EvalArgs ea{};
        ea.m = machine();
        ea.H = ham();
        ea.md = mdev.p;
        ea.hd = hdev.p;
        ea.spins = samples.p;
        ea.B = N;
        ea.eloc = E.p;
        ea.O = O.p;
        ea.plan = eval_plan();
        ea.tt = terms.tt;
        ea.wrank = wrank.p;
        return ea;
    }
    rbmnqs::LearnedArgs learned_args() const {
        rbmnqs::LearnedArgs l{};
        l.m = machine();
        l.n_chains = cfg.n_chains;
        l.spins = spins.p;
        l.prop = lprop.p;
        l.mv = lmv.p;
        l.qfw = lqfw.p;
        l.logits = net->logits();
        l.ldl = net->dims().out_p;
        l.n_moves = n_moves;
        l.mmask = dmask.p;
        l.mflip = dflip.p;
        l.ctl = ctl.p;
        l.seed = cfg.seed ^ 0x5DEECE66DULL;
        l.n_acc = lacc.p;
        l.n_try = ltry.p;
        l.eps = 0.1f;
        l.targets = ltgt.p;
        l.B = train_batch;
        return l;
    }
    // sweeps in segments (step sweeps per sample, none when step is 0),
    // learned moves after them, samples recorded after the moves
    void enqueue_learned_sampling() {
        rbmnqs::SamplerArgs a = sampler_args();
        a.record = 0;
        ck(cudaMemsetAsync(lacc.p, 0, lacc.n * sizeof(uint32_t), st), "memset");
        ck(cudaMemsetAsync(ltry.p, 0, ltry.n * sizeof(uint32_t), st), "memset");
        // fresh chains when this epoch starts them (the sweep kernel would
        // draw the same configurations at its first sweep)
        ck(rbmnqs::launch_init_chains(spins.p, n, cfg.n_chains, ctl.p, cfg.seed, st), "init chains");
        if (cfg.warmup > 0) {
            a.sweep0 = 0;
            a.nsweeps = cfg.warmup;
            ck(rbmnqs::launch_sampler(a, fp64, shape, st), "sampler kernel");
        }
        rbmnqs::LearnedArgs l = learned_args();
        // theta of the current configurations for the moves: from the sweep
        // kernel when its path writes it, else (no sweeps) from the theta
        // kernel once per sample; the moves keep it current
        const bool sweep_theta = cfg.step > 0 && rbmnqs::sampler_writes_theta(machine(), fp64, shape);
        if (!fp64 && (sweep_theta || cfg.step == 0)) {
            a.theta_out = lth.p;
            l.theta = lth.p;
        }
        for (int j = 0; j < cfg.samples_per_chain; j++) {
            if (cfg.step > 0) {
                a.sweep0 = cfg.warmup + j * cfg.step;
                a.nsweeps = cfg.step;
                // after the sample loop's first sweep launch theta is current
                // for every chain (written by that launch, kept by the moves)
                a.theta_in = (sweep_theta && j > 0) ? lth.p : nullptr;
                ck(rbmnqs::launch_sampler(a, fp64, shape, st), "sampler kernel");
            } else if (l.theta && cfg.learned_steps > 0) {
                ck(rbmnqs::launch_learned_theta(l, st), "learned theta");
            }
            for (int k = 0; k < cfg.learned_steps; k++) {
                l.move = (uint32_t)(j * cfg.learned_steps + k);
                ck(net->forward(spins.p, cfg.n_chains, st), "proposal network");
                ck(rbmnqs::launch_learned_propose(l, st), "learned propose");
                ck(net->forward(lprop.p, cfg.n_chains, st), "proposal network");
                ck(rbmnqs::launch_learned_accept(l, st), "learned accept");
            }
            ck(rbmnqs::launch_record(spins.p, cfg.n_chains, cfg.samples_per_chain, j, samples.p, st), "record");
        }
        ck(rbmnqs::launch_learned_rate(lacc.p, ltry.p, cfg.n_chains, lrate.p, st), "learned rate");
    }
    // the network is trained on the chains' current configurations (the
    // first train_batch of them) towards t_m proportional to min(1,
    // |psi(s with move m)/psi(s)|^2)
    void enqueue_learned_training() {
        if (cfg.learned_train <= 0) return;
        ck(rbmnqs::launch_learned_targets(learned_args(), st), "learned targets");
        for (int t = 0; t < cfg.learned_train; t++)
            ck(net->train_step_soft(spins.p, ltgt.p, train_batch, (float)cfg.learned_lr, st, lloss.p, true),
               "proposal training");
    }
    // tm: record the stage timing events (off for the second sample of a
    // Heun step, which runs inside the optimisation stage)
    // full_sampler::sample: every state (the list is fixed at creation),
    // weights p = |psi|^2, weighted aggregators
    void enqueue_full_sample(bool tm) {
        if (tm) mark(0);
        if (tm) mark(1);
        rbmnqs::EvalArgs ea = eval_args();
        ea.logpsi = lpsi.p;
        ck(rbmnqs::launch_eval(ea, fp64, wpb, st), "eval kernel");
        if (tm) mark(2);
        ck(rbmnqs::launch_full_weights(lpsi.p, N, pw.p, fpart.p, fstat.p, st), "full weights");
        ck(rbmnqs::launch_moments(O.p, fp64, E.p, N, P, mom_blocks, pd.p, pf.p, pe.p, d.p, F.p, emean.p, st, pw.p,
                                  fstat_W()),
           "moments");
        ck(rbmnqs::launch_energy_stats_weighted(E.p, pw.p, N, n_bins, emean.p, fstat.p, stats.p, st), "energy stats");
        if (tm) mark(3);
    }
    void enqueue_sample(bool tm = true) {
        if (full) {
            enqueue_full_sample(tm);
            return;
        }
        const rbmnqs::SamplerArgs a = sampler_args();
        if (tm) mark(0);
        if (net)
            enqueue_learned_sampling();
        else if (!batch_swept)
            ck(rbmnqs::launch_sampler(a, fp64, shape, st), "sampler kernel");
        if (tm) mark(1);
        // E_loc and O_k of every sample (local_op::evaluate, derivative)
        ck(rbmnqs::launch_eval(eval_args(), fp64, wpb, st), "eval kernel");
        if (tm) mark(2);
        ck(rbmnqs::launch_moments(O.p, fp64, E.p, N, P, mom_blocks, pd.p, pf.p, pe.p, d.p, F.p, emean.p, st),
           "moments");
        ck(rbmnqs::launch_energy_stats(E.p, N, n_bins, emean.p, nacc.p, nprop.p, cfg.n_chains, estat.p, stats.p, st),
           "energy stats");
        if (net) enqueue_learned_training();
        ck(rbmnqs::launch_advance(ctl.p, cfg.reinit_chains, st), "advance");
        if (tm) mark(3);
    }
    // cg_after / cg_done: optional events ordering the matrix-free CG (a
    // cooperative launch) after another session's, so that two grid-wide
    // solves never compete for residency inside one batch graph.
    void enqueue_optimize(cudaEvent_t cg_after = nullptr, cudaEvent_t cg_done = nullptr) {
        ck(rbmnqs::launch_schedule(sched.p, st), "schedule");
        if (cfg.plugin != 3) {
            enqueue_solve(cg_after, cg_done, true);
            ck(rbmnqs::launch_update(params.p, x.p, P, sched.p, cgres.p, plug.p, st), "update");
        } else {
            // heun_plugin::apply (plugin.cpp:87-115): half step, second
            // sample and gradient() (the regularisation schedules decay
            // again, the learning rate does not), then the combined step.
            // The sample statistics reported are the first sample's.
            enqueue_solve(cg_after, nullptr, true);
            ck(rbmnqs::launch_heun_begin(params.p, x.p, P, sched.p, cgres.p, plug.p, st), "heun");
            ck(rbmnqs::launch_unpack(params.p, n, n_vb, nh, vb.p, hb.p, W64.p, W32.p, st), "unpack");
            ck(cudaMemcpyAsync(stats_first.p, stats.p, sizeof(rbmnqs::EpochStatsDev), cudaMemcpyDeviceToDevice, st),
               "copy");
            enqueue_sample(false);
            ck(cudaMemcpyAsync(stats.p, stats_first.p, sizeof(rbmnqs::EpochStatsDev), cudaMemcpyDeviceToDevice, st),
               "copy");
            if (cfg.optimizer_type == 0) ck(rbmnqs::launch_schedule_regs(sched.p, st), "schedule");
            enqueue_solve(nullptr, cg_done, false);
            ck(rbmnqs::launch_heun_finish(params.p, x.p, P, sched.p, cgres.p, plug.p, O.p, fp64, d.p, N,
                                          cfg.optimizer_type == 0, st),
               "heun");
        }
        ck(rbmnqs::launch_unpack(params.p, n, n_vb, nh, vb.p, hb.p, W64.p, W32.p, st), "unpack");
        mark(6);
    }
    // the CG limits of cg_solver.cpp:260-334 (cg1)
    int cg_max_it() const {
        const int m = std::min(2 * P, cfg.max_iterations);
        return m == 0 ? 2 * P : m;
    }
    double cg_rtol() const { return cfg.rtol == 0 ? 1e-16 : cfg.rtol; }
    // this session's system for the multi-system matrix-free CG
    rbmnqs::CgMultiProb cg_prob() const {
        rbmnqs::CgMultiProb p{};
        p.O = O.p;
        p.d = full ? dzero.p : d.p;
        p.F = F.p;
        p.x = x.p;
        p.diag = diag.p;
        p.max_diag = maxdiag.p;
        p.sch = sched.p;
        p.res = cgres.p;
        p.r = mfw.r;
        p.p0 = mfw.p;
        p.p1 = mfw.R1;
        p.Ap = mfw.Ap;
        p.v = mfw.tmpN;
        p.norm = (double)N;
        p.rtol = cg_rtol();
        p.N = N;
        p.P = P;
        p.n_neural = P_neural;
        p.max_it = cg_max_it();
        return p;
    }
    // a batch solves this session's system in its merged launch: the SR
    // step (not SGD, not the two solves of Heun) by matrix-free CG
    bool batch_cg() const { return multi_cg && cfg.plugin != 3 && cfg.optimizer_type == 0 && !full; }
    // the SR step around a solve that the batch launches: schedules and
    // var(O) before it, the update after it
    void enqueue_optimize_pre() {
        ck(rbmnqs::launch_schedule(sched.p, st), "schedule");
        ck(rbmnqs::launch_var_diag(O.p, fp64, d.p, N, P, mfp, mfw, diag.p, maxdiag.p, st, nullptr), "var diag");
        mark(4);
    }
    void enqueue_optimize_post() {
        mark(5);
        ck(rbmnqs::launch_update(params.p, x.p, P, sched.p, cgres.p, plug.p, st), "update");
        ck(rbmnqs::launch_unpack(params.p, n, n_vb, nh, vb.p, hb.p, W64.p, W32.p, st), "unpack");
        mark(6);
    }
    // solves that are cooperative launches (ordered one after another in a batch graph)
    bool coop_solve() const { return mfree || coop_dense || cfg.solver == 2; }
    // the step direction x: SR solve (warm start x) or the SGD gradient
    void enqueue_solve(cudaEvent_t cg_after, cudaEvent_t cg_done, bool tm) {
        int max_it = std::min(2 * P, cfg.max_iterations);
        if (max_it == 0) max_it = 2 * P;
        double rtol = cfg.rtol == 0 ? 1e-16 : cfg.rtol;
        if (cfg.solver == 1) {  // minresqlp semantics (minresqlp_adapter.cpp:86-112)
            max_it = cfg.max_iterations > 0 ? cfg.max_iterations : 4 * P;
            rtol = cfg.rtol > 0 ? cfg.rtol : 1e-16;
        }
        auto mk = [&](int i) {
            if (tm) mark(i);
        };
        // full enumeration: O becomes sqrt(N p / W) (O - d), whose plain Gram
        // is S = sum p conj(O - d)(O - d)^T / W (the reference's sqrt(p) O
        // store with norm W, aggregator.cpp:274-289); d is then zero for the
        // solve and the variance factor is W / (W - W2 / W)
        const double2* dS = full ? dzero.p : d.p;
        const double* vf = full ? fstat_vfac() : nullptr;
        if (cfg.optimizer_type != 1 && full)
            ck(rbmnqs::launch_full_center(O.p, fp64, pw.p, fstat.p, d.p, N, P, st), "full centring");
        if (cfg.optimizer_type == 1) {
            // SGD: the gradient itself is the step direction
            mk(4);
            ck(rbmnqs::launch_sgd_direction(F.p, x.p, P, cfg.sgd_real_factor, cgres.p, st), "sgd direction");
            mk(5);
        } else if (mfree) {
            // diag = var(O) straight from O; CG on the operator (cg_solver.cpp aprod)
            ck(rbmnqs::launch_var_diag(O.p, fp64, dS, N, P, mfp, mfw, diag.p, maxdiag.p, st, vf), "var diag");
            mk(4);
            if (cg_after) ck(cudaStreamWaitEvent(st, cg_after, 0), "cg order");
            if (cfg.solver == 2)
                ck(rbmnqs::launch_woodbury_solve(O.p, fp64, dS, N, P, P_neural, (double)N, F.p, x.p, maxdiag.p,
                                                 sched.p, 0, 0, 0, wbw, cgres.p, st),
                   "direct solve (sample space)");
            else if (multi_cg)
                ck(rbmnqs::launch_cg_multi(cgm.p, 1, fp64, cgms, cgm_blocks, st), "matrix-free cg");
            else
                ck(rbmnqs::launch_cg_mfree(O.p, fp64, dS, (double)N, N, P, P_neural, F.p, x.p, diag.p, maxdiag.p,
                                           sched.p, 0, 0, 0, max_it, rtol, mfp, mfw, cgres.p, st),
                   "matrix-free cg");
            if (cg_done) ck(cudaEventRecord(cg_done, st), "cg order");
            mk(5);
        } else {
            if (gram_tc)
                ck(rbmnqs::launch_gram_tc(gtc, O.p, fp64, dS, gpart.p, gerr.p, Sm.p, st), "tensor-core gram");
            else
                ck(rbmnqs::launch_gram_fp64(O.p, fp64, dS, N, P, gram_ks, part.p, Sm.p, st), "gram");
            ck(rbmnqs::launch_regularize(Sm.p, P, P_neural, N, sched.p, diag.p, Sreg.p, maxdiag.p, st,
                                         cfg.solver == 2, vf),
               "regularize");
            mk(4);
            const bool coop = coop_solve();
            if (coop && cg_after) ck(cudaStreamWaitEvent(st, cg_after, 0), "cg order");
            if (cfg.solver == 2)
                ck(rbmnqs::launch_direct_solve(Sreg.p, F.p, x.p, P, dwork.p, dsync.p, cgres.p, st), "direct solve");
            else if (coop_dense || cfg.solver == 1)
                ck(rbmnqs::launch_cg_dense_coop(Sreg.p, F.p, x.p, P, max_it, rtol, mfp, mfw, cgres.p, st),
                   "cooperative solve");
            else
                ck(rbmnqs::launch_cg(Sreg.p, F.p, x.p, P, max_it, rtol, cgres.p, st), "cg");
            if (coop && cg_done) ck(cudaEventRecord(cg_done, st), "cg order");
            mk(5);
        }
    }
    void collect_timing(int first, int last) {
        if (!timing) return;
        ck(cudaEventSynchronize(ev[last]), "event sync");
        for (int i = first; i < last; i++) {
            float ms = 0;
            ck(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]), "elapsed");
            stage_ms[i] += ms;
            stage_launches[i] += 1;
        }
    }
};

// ---------------------------------------------------------------------------
extern "C" {

static void set_schedules(rbmnqs_handle* h, int64_t n_updates);

const char* rbmnqs_last_error(void) { return g_err.c_str(); }

int rbmnqs_model_kitaev(int32_t n_cells, int32_t n_cells_b, const double J[3], double h, double symmetry,
                        rbmnqs_model** out) {
    return guard([&] {
        require(out && J && n_cells >= 1, "rbmnqs_model_kitaev: bad arguments");
        auto m = std::make_unique<rbmnqs_model>();
        m->m = rbmnqs::make_kitaev(n_cells, n_cells_b, J, h, symmetry);
        require(m->m.n <= 128, "rbmnqs_model_kitaev: more than 128 sites (MAX_SPIN_SITES)");
        *out = m.release();
    });
}

int rbmnqs_model_toric(int32_t n_cells, double J, double symmetry, rbmnqs_model** out) {
    return guard([&] {
        require(out && n_cells >= 1, "rbmnqs_model_toric: bad arguments");
        auto m = std::make_unique<rbmnqs_model>();
        m->m = rbmnqs::make_toric(n_cells, J, symmetry);
        require(m->m.n <= 128, "rbmnqs_model_toric: more than 128 sites (MAX_SPIN_SITES)");
        *out = m.release();
    });
}

int rbmnqs_model_add_hexagons(rbmnqs_model* m) {
    return guard([&] {
        require(m != nullptr, "null model");
        rbmnqs::add_hexagons(m->m);
    });
}

int rbmnqs_model_sizes(const rbmnqs_model* m, int32_t* n_sites, int32_t* n_ops, int32_t* n_bonds,
                       int32_t* n_obs) {
    return guard([&] {
        require(m != nullptr, "null model");
        if (n_sites) *n_sites = m->m.n;
        if (n_ops) *n_ops = (int32_t)m->m.hamiltonian.size();
        if (n_bonds) *n_bonds = (int32_t)m->m.bonds.size();
        if (n_obs) *n_obs = (int32_t)m->m.observables.size();
    });
}

int rbmnqs_model_bonds(const rbmnqs_model* m, int32_t* abt) {
    return guard([&] {
        require(m && abt, "null argument");
        for (size_t i = 0; i < m->m.bonds.size(); i++) {
            abt[3 * i] = m->m.bonds[i].a;
            abt[3 * i + 1] = m->m.bonds[i].b;
            abt[3 * i + 2] = m->m.bonds[i].type;
        }
    });
}

int rbmnqs_model_op(const rbmnqs_model* m, int32_t o, int32_t* k, int32_t* acts_on, double* mat) {
    return guard([&] {
        require(m != nullptr, "null model");
        const int nh = (int)m->m.hamiltonian.size();
        require(o >= 0 && o < nh + (int)m->m.observables.size(), "operator index out of range");
        const auto& op = o < nh ? m->m.hamiltonian[o] : m->m.observables[o - nh];
        if (k) *k = op.k;
        if (acts_on)
            for (int i = 0; i < 6; i++) acts_on[i] = op.acts_on[i];
        if (mat)
            for (size_t i = 0; i < op.mat.size(); i++) {
                mat[2 * i] = op.mat[i].real();
                mat[2 * i + 1] = op.mat[i].imag();
            }
    });
}

int rbmnqs_model_symmetry(const rbmnqs_model* m, int32_t* S, int32_t* n_vb, int32_t* perm, int32_t* basis) {
    return guard([&] {
        require(m != nullptr, "null model");
        if (S) *S = (int32_t)m->m.perm.size();
        if (n_vb) *n_vb = (int32_t)m->m.basis.size();
        if (perm)
            for (size_t s = 0; s < m->m.perm.size(); s++)
                for (int i = 0; i < m->m.n; i++) perm[s * m->m.n + i] = m->m.perm[s][i];
        if (basis)
            for (size_t i = 0; i < m->m.basis.size(); i++) basis[i] = m->m.basis[i];
    });
}

int rbmnqs_model_ground_state(const rbmnqs_model* m, int32_t max_iter, double tol, uint64_t seed, double* energy,
                              int32_t* iterations, double* psi) {
    return guard([&] {
        require(m && energy && max_iter >= 1 && tol >= 0, "rbmnqs_model_ground_state: bad arguments");
        const int n = m->m.n;
        require(n >= 1 && n <= 28, "exact diagonalisation needs 1 <= n <= 28 sites", RBMNQS_ERR_UNSUPPORTED);
        HamHost hh = build_ham(m->m.hamiltonian);
        DevBuf<rbmnqs::OpDev> ops;
        DevBuf<int> rowptr;
        DevBuf<uint32_t> mask;
        DevBuf<double2> val;
        ops.alloc(hh.ops.size());
        rowptr.alloc(hh.rowptr.size());
        mask.alloc(std::max<size_t>(1, hh.mask.size()));
        val.alloc(std::max<size_t>(1, hh.val.size()));
        ck(cudaMemcpy(ops.p, hh.ops.data(), hh.ops.size() * sizeof(rbmnqs::OpDev), cudaMemcpyHostToDevice), "c");
        ck(cudaMemcpy(rowptr.p, hh.rowptr.data(), hh.rowptr.size() * sizeof(int), cudaMemcpyHostToDevice), "c");
        if (!hh.mask.empty()) {
            ck(cudaMemcpy(mask.p, hh.mask.data(), hh.mask.size() * sizeof(uint32_t), cudaMemcpyHostToDevice), "c");
            ck(cudaMemcpy(val.p, hh.val.data(), hh.val.size() * sizeof(double2), cudaMemcpyHostToDevice), "c");
        }
        rbmnqs::HamDev H{};
        H.n_ops = (int)hh.ops.size();
        H.ops = ops.p;
        H.rowptr = rowptr.p;
        H.ent_mask = mask.p;
        H.ent_val = val.p;
        cudaStream_t st;
        ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
        int it = 0;
        const cudaError_t e =
            rbmnqs::ed_ground_state(H, n, max_iter, tol, seed, st, energy, &it, reinterpret_cast<double2*>(psi));
        cudaStreamDestroy(st);
        ck(e, "exact diagonalisation");
        if (iterations) *iterations = it;
    });
}

int rbmnqs_model_pfaffian_classes(const rbmnqs_model* m, double symmetry, int32_t* bs, int32_t* n_indep) {
    return guard([&] {
        require(m != nullptr && m->m.lat() != nullptr, "null model");
        const auto* lat = m->m.lat();
        int ni = 0;
        auto v = rbmnqs::pfaffian_index_matrix(m->m.n, lat->symmetry(symmetry), lat->symmetry_basis(symmetry), &ni);
        if (bs)
            for (size_t i = 0; i < v.size(); i++) bs[i] = v[i];
        if (n_indep) *n_indep = ni;
    });
}

void rbmnqs_model_destroy(rbmnqs_model* m) { delete m; }

int rbmnqs_config_default(rbmnqs_config* c) {
    return guard([&] {
        require(c != nullptr, "null config");
        std::memset(c, 0, sizeof(*c));
        // src/tools/ini.cpp:38-120
        c->rbm_type = 0;
        c->alpha = 1;
        c->pfaffian = 0;
        c->pfaffian_symmetry = 0.5;
        c->n_chains = 4;
        c->samples_per_chain = 250;  // sampler.n_samples 1000 / 4 chains
        c->warmup = 100;
        c->step = 1;
        c->bond_flips = 0.5;
        c->pfaffian_refresh = 0;
        c->reinit_chains = 1;
        c->seed = 421390484ULL;
        const double lr[3] = {1e-2, 1e-2, 1.0}, r1[3] = {1, 1e-4, 0.9}, r2[3] = {1e-3, 1e-6, 0.9},
                     rd[3] = {1e-2, 1e-2, 1.0};
        std::memcpy(c->lr, lr, sizeof(lr));
        std::memcpy(c->reg1, r1, sizeof(r1));
        std::memcpy(c->reg2, r2, sizeof(r2));
        std::memcpy(c->deltareg1, rd, sizeof(rd));
        c->max_iterations = 0;
        c->rtol = 0;
        c->precision = 0;
        c->n_updates = 0;
        c->gram = 0;
        c->proposal = 0;
        c->learned_steps = 1;
        c->learned_train = 1;
        c->learned_hidden = 256;
        c->learned_lr = 1e-3;
        c->solver = 0;
        c->optimizer_type = 0;
        c->sgd_real_factor = 1.0;
        c->plugin = 0;
        c->adam_beta1 = 0.9;
        c->adam_beta2 = 0.999;
        c->adam_eps = 1e-8;
        c->mom_alpha = 0.9;
        c->mom_dialup = 1.0;
        c->heun_eps = 1e-3;
        c->sampler_type = 0;
        c->full_parallel_bits = 2;
    });
}

int rbmnqs_create(const rbmnqs_model* mdl, const rbmnqs_config* cfg, rbmnqs_handle** out) {
    return guard([&] {
        require(mdl && cfg && out, "rbmnqs_create: null argument");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            throw Fail{RBMNQS_ERR_NO_DEVICE, "no CUDA device available"};
        require(cfg->rbm_type == 0 || cfg->rbm_type == 1, "rbm.type must be basic (0) or symmetry (1)");
        require(!cfg->pfaffian || mdl->m.n <= rbmnqs::kPfMaxSites,
                "the Pfaffian factor supports at most 32 sites", RBMNQS_ERR_UNSUPPORTED);
        require(cfg->pfaffian_refresh >= 0, "sampler.pfaffian_refresh must be >= 0");
        require(cfg->proposal == 0 || cfg->proposal == 1, "proposal must be 0 (plain) or 1 (learned)");
        require(cfg->proposal == 0 || (!cfg->pfaffian && mdl->m.n <= 256 && cfg->learned_steps >= 0 &&
                                       cfg->learned_train >= 0 && cfg->learned_hidden % 64 == 0 &&
                                       cfg->learned_hidden >= 64 && cfg->learned_hidden <= 256),
                "learned proposals: no Pfaffian factor, <= 256 sites, hidden width 64..256 (multiple of 64)",
                RBMNQS_ERR_UNSUPPORTED);
        require(cfg->alpha >= 1 && cfg->n_chains >= 1 && cfg->samples_per_chain >= 1 && cfg->warmup >= 0 &&
                    (cfg->step >= 1 || (cfg->proposal == 1 && cfg->step == 0 && cfg->learned_steps >= 1)),
                "bad sampler/machine sizes (step 0 needs learned proposals)");
        auto h = std::make_unique<rbmnqs_handle>();
        h->cfg = *cfg;
        h->model = mdl->m;
        const auto& m = h->model;
        h->n = m.n;
        if (cfg->rbm_type == 1) {
            h->S = (int)m.perm.size();
            h->n_vb = (int)m.basis.size();
            require(h->n % h->S == 0 || true, "");
        } else {
            h->S = 1;
            h->n_vb = h->n;
        }
        h->nh = cfg->alpha * h->n_vb;
        h->T = h->nh * h->S;
        h->P_neural = h->n_vb + h->nh + h->n * h->nh;
        h->P = h->P_neural;
        std::vector<int> pf_bs_host;
        if (cfg->pfaffian) {
            // pfaffian::pfaffian (pfaffian.cpp:31-85) with its own symmetry
            const auto* lat = m.lat();
            require(lat != nullptr, "model has no lattice");
            const double ps = cfg->pfaffian_symmetry;
            auto pperm = lat->symmetry(ps);
            auto pbasis = lat->symmetry_basis(ps);
            pf_bs_host = rbmnqs::pfaffian_index_matrix(h->n, pperm, pbasis, &h->pf_indep);
            h->pf_n = h->n;
            h->P += 4 * h->pf_indep;
        }
        require(rbmnqs::elements_per_lane(h->T) > 0, "theta table larger than 512 entries per chain",
                RBMNQS_ERR_UNSUPPORTED);
        // dense S up to kDenseMax parameters, the matrix-free operator above
        h->mfree = h->P > kDenseMax;
        require(cfg->sampler_type == 0 || cfg->sampler_type == 1, "sampler_type must be 0 (metropolis) or 1 (full)");
        h->full = cfg->sampler_type == 1;
        if (h->full) {
            // full_sampler.cpp:36-41: every state once (the device holds N x P
            // derivatives, so n is bounded by memory, not by 64)
            require(h->n <= 30 && cfg->full_parallel_bits >= 0 && cfg->full_parallel_bits <= h->n,
                    "full enumeration needs n <= 30 and 0 <= full_parallel_bits <= n", RBMNQS_ERR_UNSUPPORTED);
            require((double)(int64_t(1) << h->n) * h->P * (cfg->precision == 1 ? 16 : 8) <= 64.0 * (1ull << 30),
                    "full enumeration: 2^n x n_params derivatives exceed 64 GiB", RBMNQS_ERR_UNSUPPORTED);
            require(cfg->proposal == 0, "full enumeration has no proposals", RBMNQS_ERR_UNSUPPORTED);
            require(cfg->plugin != 3, "the heun plugin is not supported with full enumeration",
                    RBMNQS_ERR_UNSUPPORTED);
            h->N = 1 << h->n;
        } else {
            h->N = cfg->n_chains * cfg->samples_per_chain;
        }
        require(h->N >= 2, "need at least two samples");
        int k = 50;
        while (h->N % k) k--;
        h->n_bins = k;
        h->fp64 = cfg->precision == 1;

        ck(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking), "stream");
        for (auto& e : h->ev) ck(cudaEventCreate(&e), "event");

        // machine tables
        const int n = h->n, S = h->S, nh = h->nh;
        h->params.alloc(h->P);
        h->vb.alloc(h->n_vb);
        h->hb.alloc(nh);
        h->W64.alloc((size_t)n * nh);
        h->W32.alloc((size_t)(n + 1) * nh);  // row n: zero pad row of the gather sweep
        ck(cudaMemsetAsync(h->W32.p, 0, (size_t)(n + 1) * nh * sizeof(float2), h->st), "memset");
        h->x.alloc(h->P);
        ck(cudaMemsetAsync(h->params.p, 0, h->P * sizeof(double2), h->st), "memset");
        ck(cudaMemsetAsync(h->x.p, 0, h->P * sizeof(double2), h->st), "memset");
        if (cfg->rbm_type == 1) {
            std::vector<uint8_t> perm((size_t)n * S), inv((size_t)S * n), orbit((size_t)h->n_vb * S);
            for (int s = 0; s < S; s++)
                for (int i = 0; i < n; i++) {
                    perm[(size_t)i * S + s] = (uint8_t)m.perm[s][i];
                    inv[(size_t)s * n + m.perm[s][i]] = (uint8_t)i;
                }
            for (int i = 0; i < h->n_vb; i++)
                for (int s = 0; s < S; s++) orbit[(size_t)i * S + s] = (uint8_t)m.perm[s][m.basis[i]];
            h->perm.alloc(perm.size());
            h->inv.alloc(inv.size());
            h->orbit.alloc(orbit.size());
            ck(cudaMemcpy(h->perm.p, perm.data(), perm.size(), cudaMemcpyHostToDevice), "copy");
            ck(cudaMemcpy(h->inv.p, inv.data(), inv.size(), cudaMemcpyHostToDevice), "copy");
            ck(cudaMemcpy(h->orbit.p, orbit.data(), orbit.size(), cudaMemcpyHostToDevice), "copy");
            if (n < 255) {
                const std::vector<uint8_t> wr = eval_row_order(m.perm, n, nh);
                h->wrank.alloc(n);
                ck(cudaMemcpy(h->wrank.p, wr.data(), n, cudaMemcpyHostToDevice), "copy");
            }
        }
        if (h->pf_n) {
            const int pn = h->pf_n;
            std::vector<int16_t> b16(pf_bs_host.begin(), pf_bs_host.end());
            // derivative gather lists: pairs (i > j) of each class
            std::vector<std::vector<uint32_t>> cls(h->pf_indep);
            for (int i = 0; i < pn; i++)
                for (int j = 0; j < i; j++) {
                    const int b = pf_bs_host[(size_t)i * pn + j];
                    require(b != 0, "Pfaffian class matrix has a zero off-diagonal entry");
                    cls[std::abs(b) - 1].push_back(((uint32_t)i << 16) | ((uint32_t)j << 8) | (b > 0 ? 1u : 0u));
                }
            std::vector<int> ptr(1, 0);
            std::vector<uint32_t> pairs;
            for (auto& c : cls) {
                pairs.insert(pairs.end(), c.begin(), c.end());
                ptr.push_back((int)pairs.size());
            }
            h->pf_bs.alloc(b16.size());
            h->pf_ptr.alloc(ptr.size());
            h->pf_pairs.alloc(pairs.size());
            ck(cudaMemcpy(h->pf_bs.p, b16.data(), b16.size() * sizeof(int16_t), cudaMemcpyHostToDevice), "c");
            ck(cudaMemcpy(h->pf_ptr.p, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice), "c");
            ck(cudaMemcpy(h->pf_pairs.p, pairs.data(), pairs.size() * sizeof(uint32_t), cudaMemcpyHostToDevice), "c");
        }
        // Hamiltonian
        HamHost hh = build_ham(m.hamiltonian);
        h->n_ops = (int)hh.ops.size();
        h->ops.alloc(hh.ops.size());
        h->rowptr.alloc(hh.rowptr.size());
        h->emask.alloc(hh.mask.size());
        h->eval.alloc(hh.val.size());
        ck(cudaMemcpy(h->ops.p, hh.ops.data(), hh.ops.size() * sizeof(rbmnqs::OpDev), cudaMemcpyHostToDevice), "c");
        ck(cudaMemcpy(h->rowptr.p, hh.rowptr.data(), hh.rowptr.size() * sizeof(int), cudaMemcpyHostToDevice), "c");
        ck(cudaMemcpy(h->emask.p, hh.mask.data(), hh.mask.size() * sizeof(uint32_t), cudaMemcpyHostToDevice), "c");
        ck(cudaMemcpy(h->eval.p, hh.val.data(), hh.val.size() * sizeof(double2), cudaMemcpyHostToDevice), "c");
        h->terms.upload(build_terms(m.hamiltonian));
        // observables (evaluation mode), one table each
        for (const auto& op : m.observables) {
            auto od = std::make_unique<ObsDev>();
            HamHost oh = build_ham({op});
            od->ops.alloc(oh.ops.size());
            od->rowptr.alloc(oh.rowptr.size());
            od->mask.alloc(oh.mask.size());
            od->val.alloc(oh.val.size());
            ck(cudaMemcpy(od->ops.p, oh.ops.data(), oh.ops.size() * sizeof(rbmnqs::OpDev), cudaMemcpyHostToDevice), "c");
            ck(cudaMemcpy(od->rowptr.p, oh.rowptr.data(), oh.rowptr.size() * sizeof(int), cudaMemcpyHostToDevice), "c");
            ck(cudaMemcpy(od->mask.p, oh.mask.data(), oh.mask.size() * sizeof(uint32_t), cudaMemcpyHostToDevice), "c");
            ck(cudaMemcpy(od->val.p, oh.val.data(), oh.val.size() * sizeof(double2), cudaMemcpyHostToDevice), "c");
            od->H.n_ops = 1;
            od->H.ops = od->ops.p;
            od->H.rowptr = od->rowptr.p;
            od->H.ent_mask = od->mask.p;
            od->H.ent_val = od->val.p;
            od->H.n_rows = (int)oh.rowptr.size();
            od->H.n_ents = (int)oh.mask.size();
            od->hd.alloc(1);
            ck(cudaMemcpy(od->hd.p, &od->H, sizeof(od->H), cudaMemcpyHostToDevice), "c");
            od->terms.upload(build_terms({op}));
            h->obs.push_back(std::move(od));
        }
        // bond proposals: bonds of type != 2 (metropolis_sampler.cpp:145-166)
        std::vector<int2> pb;
        if (m.kind == "kitaev")
            for (auto& b : m.bonds)
                if (b.type != 2) pb.push_back(make_int2(b.a, b.b));
        h->n_prop_bonds = (int)pb.size();
        if (!pb.empty()) {
            h->bonds.alloc(pb.size());
            ck(cudaMemcpy(h->bonds.p, pb.data(), pb.size() * sizeof(int2), cudaMemcpyHostToDevice), "c");
        }
        // sampler state and outputs
        h->spins.alloc((size_t)cfg->n_chains * 4);
        ck(cudaMemsetAsync(h->spins.p, 0, (size_t)cfg->n_chains * 16, h->st), "memset");
        h->nacc.alloc(cfg->n_chains);
        h->nprop.alloc(cfg->n_chains);
        h->ctl.alloc(2);
        const uint32_t ctl0[2] = {0, 1};
        ck(cudaMemcpy(h->ctl.p, ctl0, sizeof(ctl0), cudaMemcpyHostToDevice), "c");
        h->E.alloc(h->N);
        h->samples.alloc((size_t)h->N * 4);
        h->O.alloc((size_t)h->N * h->P * h->osize());
        h->mom_blocks = std::max(1, std::min(296, h->N / 64));
        h->pd.alloc((size_t)h->mom_blocks * h->P);
        h->pf.alloc((size_t)h->mom_blocks * h->P);
        h->pe.alloc(h->mom_blocks);
        h->d.alloc(h->P);
        h->F.alloc(h->P);
        h->emean.alloc(1);
        if (h->full) {
            h->lpsi.alloc(h->N);
            h->pw.alloc(h->N);
            h->fpart.alloc(3 * rbmnqs::kFullBlocks);
            h->fstat.alloc(1);
            h->dzero.alloc(h->P);
            ck(cudaMemsetAsync(h->dzero.p, 0, h->P * sizeof(double2), h->st), "memset");
            ck(rbmnqs::launch_full_states(h->samples.p, h->n, cfg->full_parallel_bits, h->st), "full states");
        }
        h->gram_tc = !h->fp64 && cfg->gram == 0 && !h->mfree;
        require(cfg->solver >= 0 && cfg->solver <= 2, "solver must be 0 (cg), 1 (minresqlp) or 2 (direct)");
        require(cfg->solver != 2 || !h->mfree || h->N <= rbmnqs::kWoodburyMaxN,
                "the direct solver above " + std::to_string(kDenseMax) + " parameters solves in sample space: at most " +
                    std::to_string(rbmnqs::kWoodburyMaxN) + " samples per epoch",
                RBMNQS_ERR_UNSUPPORTED);
        if (cfg->solver == 2 && h->mfree) {
            h->wbbuf.alloc(rbmnqs::woodbury_work_bytes(h->N, h->P));
            h->wbw = rbmnqs::woodbury_carve(h->wbbuf.p, h->N, h->P);
        }
        h->coop_dense = !h->mfree && cfg->solver != 2 && (!rbmnqs::cg_cluster_fits(h->P) || cfg->solver == 1);
        if (cfg->solver == 2) {
            h->dsync.alloc(1);
            h->dwork.alloc(h->P);
        }
        if (h->mfree || h->coop_dense) {
            const int nn = h->mfree ? h->N : 1;
            ck(rbmnqs::mfree_plan(nn, h->P, &h->mfp), "cooperative CG plan");
            h->mfbuf.alloc(rbmnqs::mfree_work_bytes(nn, h->P, h->mfp));
            h->mfw = rbmnqs::mfree_carve(h->mfbuf.p, nn, h->P, h->mfp);
            h->mfw.minres = cfg->solver == 1;
        }
        if (h->mfree) {
        } else if (h->gram_tc) {
            ck(rbmnqs::gram_tc_plan(h->N, h->P, &h->gtc), "gram plan");
            const size_t gb = h->gtc.buffer_bytes();
            h->gplanes.alloc((gb + 3) / 4);
            ck(cudaMemsetAsync(h->gplanes.p, 0, gb, h->st), "memset");  // padding stays 0
            h->gpart.alloc(h->gtc.partial_bytes() / sizeof(float));
            h->gerr.alloc(1);
            ck(cudaMemsetAsync(h->gerr.p, 0, sizeof(int), h->st), "memset");
            ck(rbmnqs::gram_tc_maps(&h->gtc, h->gplanes.p), "tensor map");
        } else {
            h->gram_ks = rbmnqs::gram_splits(h->N, h->P);
            h->part.alloc((size_t)h->gram_ks * h->P * h->P);
        }
        if (!h->mfree) {
            h->Sm.alloc((size_t)h->P * h->P);
            h->Sreg.alloc((size_t)h->P * h->P);
        }
        h->diag.alloc(h->P);
        h->maxdiag.alloc(1);
        h->sched.alloc(1);
        h->cgres.alloc(1);
        h->multi_cg = h->mfree && cfg->solver == 0;
        {
            require(cfg->optimizer_type == 0 || cfg->optimizer_type == 1, "optimizer.type must be 0 (SR) or 1 (SGD)");
            require(cfg->plugin >= 0 && cfg->plugin <= 3,
                    "optimizer.plugin must be 0, 1 (adam), 2 (momentum) or 3 (heun)");
            require(cfg->plugin != 3 || cfg->heun_eps > 0, "optimizer.heun.eps must be positive");
            require(cfg->sgd_real_factor != 0, "optimizer.sgd.real_factor must be nonzero");
            rbmnqs::PluginDev pd{};
            pd.type = cfg->plugin;
            pd.beta1 = cfg->adam_beta1;
            pd.beta2 = cfg->adam_beta2;
            pd.eps = cfg->adam_eps;
            pd.alpha = cfg->mom_alpha;
            pd.dialup = cfg->mom_dialup;
            pd.dup = cfg->mom_dialup == 1.0 ? 1.0 : 1e-3;  // plugin.cpp:64
            pd.t = 1;
            pd.heps = cfg->heun_eps;
            if (cfg->plugin == 3) {
                h->plug_part.alloc(rbmnqs::kHeunBlocks);
                h->stats_first.alloc(1);
                pd.part = h->plug_part.p;
            }
            if (cfg->plugin) {
                h->plug_m.alloc(h->P);
                h->plug_wr.alloc(h->P);
                h->plug_wi.alloc(h->P);
                ck(cudaMemsetAsync(h->plug_m.p, 0, h->P * sizeof(double2), h->st), "memset");
                ck(cudaMemsetAsync(h->plug_wr.p, 0, h->P * sizeof(double), h->st), "memset");
                ck(cudaMemsetAsync(h->plug_wi.p, 0, h->P * sizeof(double), h->st), "memset");
                pd.m = h->plug_m.p;
                pd.wr = h->plug_wr.p;
                pd.wi = h->plug_wi.p;
            }
            h->plug.alloc(1);
            ck(cudaMemcpyAsync(h->plug.p, &pd, sizeof(pd), cudaMemcpyHostToDevice, h->st), "copy");
        }
        h->stats.alloc(1);
        h->estat.alloc(rbmnqs::energy_stats_scratch_doubles(h->n_bins));
        ck(cudaMemsetAsync(h->estat.p, 0, h->estat.n * sizeof(double), h->st), "memset");
        // decay_t schedules with the n_updates offset
        h->n_updates = cfg->n_updates;
        set_schedules(h.get(), h->n_updates);
        // device copies of the machine / Hamiltonian descriptors
        h->mdev.alloc(1);
        h->hdev.alloc(1);
        {
            const rbmnqs::MachineDev md = h->machine();
            const rbmnqs::HamDev hd = h->ham();
            ck(cudaMemcpy(h->mdev.p, &md, sizeof(md), cudaMemcpyHostToDevice), "c");
            ck(cudaMemcpy(h->hdev.p, &hd, sizeof(hd), cudaMemcpyHostToDevice), "c");
        }
        // launch shapes: persistent sampler blocks; evaluation kernels with
        // FP32 W in shared memory when it fits
        ck(rbmnqs::plan_sampler(h->machine(), h->fp64, cfg->n_chains, h->n_prop_bonds, &h->shape), "sampler plan");
        if (cfg->proposal == 1) {
            // move dictionary: every site, then the Hamiltonian's distinct
            // off-diagonal flip sets of two or more sites
            std::vector<std::vector<int>> moves;
            for (int i = 0; i < n; i++) moves.push_back({i});
            {
                std::vector<std::vector<int>> seen;
                for (const auto& t : build_terms(m.hamiltonian).terms) {
                    const int nf = (t.flip1 >> 16) & 0xff;
                    std::vector<int> fs;
                    for (int q = 0; q < nf; q++)
                        fs.push_back(q < 4 ? (t.flip0 >> (8 * q)) & 0xff : (t.flip1 >> (8 * (q - 4))) & 0xff);
                    std::sort(fs.begin(), fs.end());
                    if (fs.size() < 2 || std::find(seen.begin(), seen.end(), fs) != seen.end()) continue;
                    seen.push_back(fs);
                    moves.push_back(fs);
                }
            }
            require(moves.size() <= 256,
                    "learned proposals: the move dictionary (sites + off-diagonal flip sets) exceeds 256 moves",
                    RBMNQS_ERR_UNSUPPORTED);
            h->n_moves = (int)moves.size();
            std::vector<uint32_t> mk((size_t)h->n_moves * 4, 0u), fl((size_t)h->n_moves * 2, 0u);
            for (int d = 0; d < h->n_moves; d++) {
                const auto& fs = moves[d];
                for (size_t q = 0; q < fs.size(); q++) {
                    mk[4 * d + fs[q] / 32] |= 1u << (fs[q] % 32);
                    const uint32_t b = (uint32_t)fs[q] & 0xff;
                    if (q < 4)
                        fl[2 * d] |= b << (8 * q);
                    else
                        fl[2 * d + 1] |= b << (8 * (q - 4));
                }
                fl[2 * d + 1] |= (uint32_t)fs.size() << 16;
            }
            h->dmask.alloc(mk.size());
            h->dflip.alloc(fl.size());
            ck(cudaMemcpy(h->dmask.p, mk.data(), mk.size() * 4, cudaMemcpyHostToDevice), "copy");
            ck(cudaMemcpy(h->dflip.p, fl.data(), fl.size() * 4, cudaMemcpyHostToDevice), "copy");
            h->train_batch = std::min(cfg->n_chains, 2048);
            rbmnqs::MlpDims md;
            md.n_in = n;
            md.n_out = h->n_moves;
            md.h1 = md.h2 = cfg->learned_hidden;
            try {
                h->net = std::make_unique<rbmnqs::Mlp>(md, std::max(cfg->n_chains, h->train_batch), h->st);
            } catch (cudaError_t e) {
                ck(e, "proposal network");
            }
            ck(h->net->init_random(0.02f, cfg->seed), "proposal network init");
            h->lprop.alloc((size_t)cfg->n_chains * 4);
            h->lmv.alloc(cfg->n_chains);
            h->lqfw.alloc(cfg->n_chains);
            h->lacc.alloc(cfg->n_chains);
            h->ltry.alloc(cfg->n_chains);
            h->ltgt.alloc((size_t)h->train_batch * h->n_moves);
            h->lth.alloc((size_t)cfg->n_chains * 32 * rbmnqs::elements_per_lane(h->T));
            h->lloss.alloc(1);
            h->lrate.alloc(1);
            ck(cudaMemsetAsync(h->lloss.p, 0, sizeof(float), h->st), "memset");
            ck(cudaMemsetAsync(h->lrate.p, 0, sizeof(double), h->st), "memset");
        }
        if (h->pf_n)  // one X^{-1} unscramble buffer per sampler warp
            h->pf_scratch.alloc((size_t)h->shape.blocks * h->shape.warps_per_block * rbmnqs::kPfMaxSites *
                                rbmnqs::kPfMaxSites);
        if (h->n_prop_bonds > 0 && cfg->bond_flips > 0) {
            const double thr = std::ceil(cfg->bond_flips * 16777216.0);
            h->bond_thr24 = (uint32_t)std::min(thr, 16777216.0);
        }
        h->w_in_smem = (size_t)n * nh * 8 <= 64 * 1024 ? 1 : 0;
        h->wpb = 8;
        {
            const rbmnqs::SmemPlan pl = h->eval_plan();
            while (h->wpb > 1 && rbmnqs::eval_smem_bytes(h->machine(), h->fp64, h->wpb, pl) > 200 * 1024)
                h->wpb >>= 1;
        }
        if (h->multi_cg) {
            rbmnqs::CgMultiProb pr = h->cg_prob();
            long long rc = 0, tc = 0;
            const int tiles = rbmnqs::cg_multi_units(&pr, 1, &rc, &tc);
            h->cgm.alloc(1);
            h->cgm_t2.alloc(2 * (size_t)tiles);
            h->cgm_t1.alloc(tiles);
            ck(cudaMemcpyAsync(h->cgm.p, &pr, sizeof(pr), cudaMemcpyHostToDevice, h->st), "copy");
            h->cgms.tdb = h->cgm_t2.p;
            h->cgms.tpap = h->cgm_t2.p + tiles;
            h->cgms.trs = h->cgm_t1.p;
            h->cgms.sync = h->mfw.sync;
            h->cgms.row_cost = rc;
            h->cgms.tile_cost = tc;
            ck(rbmnqs::cg_multi_blocks(&h->cgm_blocks), "multi-system CG plan");
        }
        ck(cudaStreamSynchronize(h->st), "sync");
        *out = h.release();
    });
}

void rbmnqs_destroy(rbmnqs_handle* h) { delete h; }

int rbmnqs_sizes(const rbmnqs_handle* h, int32_t* n_params, int32_t* n_neural, int32_t* n_vb, int32_t* n_hidden,
                 int32_t* n_symm) {
    return guard([&] {
        require(h != nullptr, "null handle");
        if (n_params) *n_params = h->P;
        if (n_neural) *n_neural = h->P_neural;
        if (n_vb) *n_vb = h->n_vb;
        if (n_hidden) *n_hidden = h->nh;
        if (n_symm) *n_symm = h->S;
    });
}

int rbmnqs_set_weights(rbmnqs_handle* h, const double* w) {
    return guard([&] {
        require(h && w, "null argument");
        ck(cudaMemcpyAsync(h->params.p, w, h->P * sizeof(double2), cudaMemcpyHostToDevice, h->st), "copy");
        ck(rbmnqs::launch_unpack(h->params.p, h->n, h->n_vb, h->nh, h->vb.p, h->hb.p, h->W64.p, h->W32.p, h->st),
           "unpack");
        // a pageable host buffer is free once the copy call returns (the unpack
        // is ordered before any later work on the stream); a pinned or
        // device-visible one only after the copy completes
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, w) != cudaSuccess || pa.type != cudaMemoryTypeUnregistered)
            ck(cudaStreamSynchronize(h->st), "sync");
        cudaGetLastError();  // clear a failed attribute query
    });
}

int rbmnqs_get_weights(rbmnqs_handle* h, double* w) {
    return guard([&] {
        require(h && w, "null argument");
        ck(cudaMemcpyAsync(w, h->params.p, h->P * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "copy");
        ck(cudaStreamSynchronize(h->st), "sync");
    });
}

// decay_t (abstract_optimizer.cpp:27-54) for lr, reg1, reg2, deltareg1,
// constructed with an update offset
static void set_schedules(rbmnqs_handle* h, int64_t n_updates) {
    rbmnqs::ScheduleDev sd{};
    const auto& c = h->cfg;
    const double* src[4] = {c.lr, c.reg1, c.reg2, c.deltareg1};
    for (int i = 0; i < 4; i++) {
        sd.value[i] = std::pow(src[i][2], (double)n_updates) * src[i][0];
        sd.min[i] = src[i][1];
        sd.decay[i] = src[i][2];
        sd.min_reached[i] = src[i][2] == 1.0;
    }
    ck(cudaMemcpyAsync(h->sched.p, &sd, sizeof(sd), cudaMemcpyHostToDevice, h->st), "copy");
    ck(cudaStreamSynchronize(h->st), "sync");
}

static int count_kernel_nodes(cudaGraph_t g) {
    size_t nn = 0;
    ck(cudaGraphGetNodes(g, nullptr, &nn), "graph nodes");
    std::vector<cudaGraphNode_t> nodes(nn);
    ck(cudaGraphGetNodes(g, nodes.data(), &nn), "graph nodes");
    int k = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        ck(cudaGraphNodeGetType(nd, &t), "node type");
        k += t == cudaGraphNodeTypeKernel;
    }
    return k;
}

// One line of the training log (logger.cpp:53-74 with the values that
// stochastic_reconfiguration.cpp:86-91 / gradient_descent.cpp:47-52 and
// metropolis_sampler.cpp:275-277 log): energy per spin, its standard
// deviation per spin and, for Metropolis sampling, the acceptance rate,
// written as %.16g (ostream precision 16) separated by ", ", after a header
// "# <names>" on the first line a handle writes.
static void write_log_line(rbmnqs_handle* h, const rbmnqs::EpochStatsDev& s) {
    FILE* f = h->log.f;
    const bool sgd = h->cfg.optimizer_type == 1;
    if (h->log.first) {
        std::fprintf(f, "# Energy, %s%s\n", sgd ? "EnergyStddev" : "Energy Stddev", h->full ? "" : ", AccetpanceRate");
        h->log.first = false;
    }
    const double n = h->n;
    std::fprintf(f, "%.16g, %.16g", s.energy.x / n, s.stddev / n);
    if (!h->full) std::fprintf(f, ", %.16g", s.acceptance);
    std::fprintf(f, "\n");
    std::fflush(f);
}

// Sample statistics (s) and SR statistics (o) of the last sample / optimize
// step: the device results are copied into pinned host memory and read after
// one stream synchronisation.  With sr, a successful step counts as an update.
static void readback(rbmnqs_handle* h, bool sample, rbmnqs_sample_stats* out, bool sr, rbmnqs_sr_stats* o) {
    if (!h->rb) ck(cudaMallocHost(&h->rb, sizeof(*h->rb)), "cudaMallocHost");
    auto* rb = h->rb;
    if (sample) {
        ck(cudaMemcpyAsync(&rb->stats, h->stats.p, sizeof(rb->stats), cudaMemcpyDeviceToHost, h->st), "copy");
        if (h->net) {
            ck(cudaMemcpyAsync(&rb->lrate, h->lrate.p, sizeof(double), cudaMemcpyDeviceToHost, h->st), "copy");
            ck(cudaMemcpyAsync(&rb->lloss, h->lloss.p, sizeof(float), cudaMemcpyDeviceToHost, h->st), "copy");
        }
    }
    rb->gerr = 0;
    if (sr) {
        ck(cudaMemcpyAsync(&rb->cg, h->cgres.p, sizeof(rb->cg), cudaMemcpyDeviceToHost, h->st), "copy");
        ck(cudaMemcpyAsync(&rb->sched, h->sched.p, sizeof(rb->sched), cudaMemcpyDeviceToHost, h->st), "copy");
        if (h->gram_tc) ck(cudaMemcpyAsync(&rb->gerr, h->gerr.p, sizeof(int), cudaMemcpyDeviceToHost, h->st), "copy");
    }
    rb->nerr = 0;
    if (h->net) ck(cudaMemcpyAsync(&rb->nerr, h->net->error_flag(), sizeof(int), cudaMemcpyDeviceToHost, h->st), "copy");
    ck(cudaStreamSynchronize(h->st), "sync");
    if (rb->nerr) {
        const int ne = rb->nerr;
        ck(h->net->clear_error(h->st), "memset");
        throw Fail{RBMNQS_ERR_CUDA, "proposal network GEMM: pipeline wait timed out (code " + std::to_string(ne) + ")"};
    }
    if (sample && out) {
        const auto& s = rb->stats;
        out->energy[0] = s.energy.x;
        out->energy[1] = s.energy.y;
        out->energy_var = s.var;
        out->energy_stddev = s.stddev;
        out->tau = s.tau;
        out->acceptance = s.acceptance;
        out->n_samples = h->N;
        out->n_bins = h->n_bins;
        out->status = s.finite ? RBMNQS_OK : RBMNQS_ERR_NONFINITE;
        out->learned_acceptance = h->net ? rb->lrate : 0;
        out->learned_loss = h->net ? rb->lloss : 0;
    }
    if (sr) {
        if (rb->gerr)
            throw Fail{RBMNQS_ERR_CUDA,
                       "tensor-core Gram: pipeline wait timed out (code " + std::to_string(rb->gerr) + ")"};
        const auto& r = rb->cg;
        h->last_solve = r;
        if (r.status == 0) h->n_updates++;
        if (r.status == 0 && h->log.f) write_log_line(h, rb->stats);
        if (o) {
            o->iterations = r.iterations;
            o->status = r.status;
            o->residual = r.residual;
            o->max_dw = r.max_dw;
            o->lr = rb->sched.value[0];
            o->reg1 = rb->sched.value[1];
            o->reg2 = rb->sched.value[2];
            o->deltareg1 = rb->sched.value[3];
        }
    }
}

int rbmnqs_sample(rbmnqs_handle* h, rbmnqs_sample_stats* out) {
    return guard([&] {
        require(h != nullptr, "null handle");
        h->enqueue_sample();
        h->collect_timing(0, 3);
        readback(h, true, out, false, nullptr);
        h->sampled = true;
    });
}

int rbmnqs_optimize(rbmnqs_handle* h, rbmnqs_sr_stats* out) {
    return guard([&] {
        require(h != nullptr, "null handle");
        require(h->sampled, "rbmnqs_optimize needs a preceding rbmnqs_sample");
        h->mark(3);
        h->enqueue_optimize();
        h->collect_timing(3, 6);
        readback(h, false, nullptr, true, out);
    });
}

int rbmnqs_epoch(rbmnqs_handle* h, rbmnqs_sample_stats* s, rbmnqs_sr_stats* o) {
    return guard([&] {
        require(h != nullptr, "null handle");
        if (!h->graph) {
            cudaGraph_t g;
            ck(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal), "capture");
            try {
                h->enqueue_sample();
                h->enqueue_optimize();
            } catch (...) {
                cudaStreamEndCapture(h->st, &g);
                throw;
            }
            ck(cudaStreamEndCapture(h->st, &g), "end capture");
            h->graph_kernels = count_kernel_nodes(g);
            ck(cudaGraphInstantiate(&h->graph, g, 0), "instantiate");
            cudaGraphDestroy(g);
        }
        ck(cudaGraphLaunch(h->graph, h->st), "graph launch");
        h->collect_timing(0, 6);
        readback(h, true, s, true, o);
        h->sampled = true;
    });
}

int rbmnqs_get_samples(rbmnqs_handle* h, double* E, double* O) {
    return guard([&] {
        require(h != nullptr, "null handle");
        if (E) ck(cudaMemcpyAsync(E, h->E.p, (size_t)h->N * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "c");
        if (O) {
            const size_t cnt = (size_t)h->N * h->P;
            if (h->fp64) {
                ck(cudaMemcpyAsync(O, h->O.p, cnt * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "c");
            } else {
                std::vector<float2> tmp(cnt);
                ck(cudaMemcpyAsync(tmp.data(), h->O.p, cnt * sizeof(float2), cudaMemcpyDeviceToHost, h->st), "c");
                ck(cudaStreamSynchronize(h->st), "sync");
                for (size_t i = 0; i < cnt; i++) {
                    O[2 * i] = tmp[i].x;
                    O[2 * i + 1] = tmp[i].y;
                }
            }
        }
        ck(cudaStreamSynchronize(h->st), "sync");
    });
}

int rbmnqs_get_sr(rbmnqs_handle* h, double* d, double* F, double* diag, double* S) {
    return guard([&] {
        require(h != nullptr, "null handle");
        const size_t P = h->P;
        if (d) ck(cudaMemcpyAsync(d, h->d.p, P * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "c");
        if (F) ck(cudaMemcpyAsync(F, h->F.p, P * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "c");
        if (diag) ck(cudaMemcpyAsync(diag, h->diag.p, P * sizeof(double), cudaMemcpyDeviceToHost, h->st), "c");
        if (S) {
            require(!h->mfree, "S is not formed above " + std::to_string(kDenseMax) +
                                   " parameters (matrix-free CG)", RBMNQS_ERR_UNSUPPORTED);
            ck(cudaMemcpyAsync(S, h->Sm.p, P * P * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "c");
        }
        ck(cudaStreamSynchronize(h->st), "sync");
    });
}

int rbmnqs_get_sample_configs(rbmnqs_handle* h, uint32_t* configs) {
    return guard([&] {
        require(h && configs, "null argument");
        ck(cudaMemcpyAsync(configs, h->samples.p, (size_t)h->N * 16, cudaMemcpyDeviceToHost, h->st), "c");
        ck(cudaStreamSynchronize(h->st), "sync");
    });
}

int rbmnqs_get_spins(rbmnqs_handle* h, uint32_t* spins) {
    return guard([&] {
        require(h && spins, "null argument");
        ck(cudaMemcpyAsync(spins, h->spins.p, (size_t)h->cfg.n_chains * 16, cudaMemcpyDeviceToHost, h->st), "c");
        ck(cudaStreamSynchronize(h->st), "sync");
    });
}

int rbmnqs_set_spins(rbmnqs_handle* h, const uint32_t* spins) {
    return guard([&] {
        require(h && spins, "null argument");
        ck(cudaMemcpyAsync(h->spins.p, spins, (size_t)h->cfg.n_chains * 16, cudaMemcpyHostToDevice, h->st), "c");
        const uint32_t zero = 0;
        ck(cudaMemcpyAsync(h->ctl.p + 1, &zero, sizeof(zero), cudaMemcpyHostToDevice, h->st), "c");
        ck(cudaStreamSynchronize(h->st), "sync");
    });
}

static void eval_common(rbmnqs_handle* h, const uint32_t* spins, int B, double* logpsi, double* eloc, double* O,
                        const int32_t* flips, int nflips, double* ratio) {
    require(h && spins && B >= 0, "bad arguments");
    if (B == 0) return;
    DevBuf<uint32_t> ds;
    DevBuf<double2> dl, de, dr;
    DevBuf<unsigned char> dO;
    DevBuf<int> df;
    ds.alloc((size_t)B * 4);
    ck(cudaMemcpyAsync(ds.p, spins, (size_t)B * 16, cudaMemcpyHostToDevice, h->st), "c");
    rbmnqs::EvalArgs a{};
    a.m = h->machine();
    a.H = h->ham();
    a.md = h->mdev.p;
    a.hd = h->hdev.p;
    a.spins = ds.p;
    a.B = B;
    a.plan = rbmnqs::SmemPlan{0, h->w_in_smem, 0, 0, 0};
    a.tt = h->terms.tt;
    a.wrank = h->wrank.p;
    if (logpsi) {
        dl.alloc(B);
        a.logpsi = dl.p;
    }
    if (eloc) {
        de.alloc(B);
        a.eloc = de.p;
    }
    if (O) {
        dO.alloc((size_t)B * h->P * h->osize());
        a.O = dO.p;
    }
    if (ratio) {
        require(flips && nflips >= 1 && nflips <= 6, "1..6 flips per configuration");
        df.alloc((size_t)B * nflips);
        dr.alloc(B);
        ck(cudaMemcpyAsync(df.p, flips, (size_t)B * nflips * sizeof(int), cudaMemcpyHostToDevice, h->st), "c");
        a.flips = df.p;
        a.n_flips = nflips;
        a.ratio = dr.p;
    }
    ck(rbmnqs::launch_eval(a, h->fp64, h->wpb, h->st), "eval kernel");
    if (logpsi) ck(cudaMemcpyAsync(logpsi, dl.p, B * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "c");
    if (eloc) ck(cudaMemcpyAsync(eloc, de.p, B * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "c");
    if (ratio) ck(cudaMemcpyAsync(ratio, dr.p, B * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "c");
    if (O) {
        const size_t cnt = (size_t)B * h->P;
        if (h->fp64) {
            ck(cudaMemcpyAsync(O, dO.p, cnt * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "c");
        } else {
            std::vector<float2> tmp(cnt);
            ck(cudaMemcpyAsync(tmp.data(), dO.p, cnt * sizeof(float2), cudaMemcpyDeviceToHost, h->st), "c");
            ck(cudaStreamSynchronize(h->st), "sync");
            for (size_t i = 0; i < cnt; i++) {
                O[2 * i] = tmp[i].x;
                O[2 * i + 1] = tmp[i].y;
            }
        }
    }
    ck(cudaStreamSynchronize(h->st), "sync");
}

int rbmnqs_eval_batch(rbmnqs_handle* h, const uint32_t* spins, int32_t B, double* logpsi, double* eloc, double* O) {
    return guard([&] { eval_common(h, spins, B, logpsi, eloc, O, nullptr, 0, nullptr); });
}

int rbmnqs_log_psi_over_psi(rbmnqs_handle* h, const uint32_t* spins, const int32_t* flips, int32_t n_flips,
                            int32_t B, double* out) {
    return guard([&] {
        require(out != nullptr, "null output");
        eval_common(h, spins, B, nullptr, nullptr, nullptr, flips, n_flips, out);
    });
}

int rbmnqs_sr_solve(rbmnqs_handle* h, const double* O, int32_t N, const double* d, double norm, const double* F,
                    double* x_io, double r1, double r2, double rd, const double* diag, int32_t* iterations,
                    double* residual) {
    return guard([&] {
        require(h && O && d && F && x_io && diag && N >= 1 && norm > 0, "bad arguments");
        const int P = h->P;
        DevBuf<double2> dO, dd, dF, dx, part, G, Sreg;
        DevBuf<double> ddiag, dmax;
        DevBuf<rbmnqs::CgResultDev> res;
        dO.alloc((size_t)N * P);
        dd.alloc(P);
        dF.alloc(P);
        dx.alloc(P);
        ddiag.alloc(P);
        res.alloc(1);
        ck(cudaMemcpyAsync(dO.p, O, (size_t)N * P * sizeof(double2), cudaMemcpyHostToDevice, h->st), "c");
        ck(cudaMemcpyAsync(dd.p, d, P * sizeof(double2), cudaMemcpyHostToDevice, h->st), "c");
        ck(cudaMemcpyAsync(dF.p, F, P * sizeof(double2), cudaMemcpyHostToDevice, h->st), "c");
        ck(cudaMemcpyAsync(dx.p, x_io, P * sizeof(double2), cudaMemcpyHostToDevice, h->st), "c");
        ck(cudaMemcpyAsync(ddiag.p, diag, P * sizeof(double), cudaMemcpyHostToDevice, h->st), "c");
        int max_it = std::min(2 * P, h->cfg.max_iterations);
        if (max_it == 0) max_it = 2 * P;
        double rtol = h->cfg.rtol == 0 ? 1e-16 : h->cfg.rtol;
        const bool minres = h->cfg.solver == 1;
        const bool direct = h->cfg.solver == 2;
        if (minres) {
            max_it = h->cfg.max_iterations > 0 ? h->cfg.max_iterations : 4 * P;
            rtol = h->cfg.rtol > 0 ? h->cfg.rtol : 1e-16;
        }
        require(!direct || P <= kDenseMax || N <= rbmnqs::kWoodburyMaxN,
                "the direct solver above " + std::to_string(kDenseMax) + " parameters solves in sample space: at most " +
                    std::to_string(rbmnqs::kWoodburyMaxN) + " samples",
                RBMNQS_ERR_UNSUPPORTED);
        if (P > kDenseMax && direct) {
            // the sample-space form of the direct solve (woodbury.cu)
            DevBuf<unsigned char> wb;
            wb.alloc(rbmnqs::woodbury_work_bytes(N, P));
            const rbmnqs::WoodburyWork ww = rbmnqs::woodbury_carve(wb.p, N, P);
            dmax.alloc(1);
            ck(rbmnqs::launch_max_diag(ddiag.p, P, dmax.p, h->st), "max diag");
            ck(rbmnqs::launch_woodbury_solve(dO.p, 1, dd.p, N, P, h->P_neural, norm, dF.p, dx.p, dmax.p, nullptr, r1,
                                             r2, rd, ww, res.p, h->st),
               "direct solve (sample space)");
            ck(cudaStreamSynchronize(h->st), "sync");  // before wb goes out of scope
        } else if (P > kDenseMax) {
            // the operator form (cg_solver.cpp aprod) on the given O, d, norm
            rbmnqs::MfreePlan pl{};
            ck(rbmnqs::mfree_plan(N, P, &pl), "matrix-free plan");
            DevBuf<unsigned char> wb;
            wb.alloc(rbmnqs::mfree_work_bytes(N, P, pl));
            rbmnqs::MfreeWork wk = rbmnqs::mfree_carve(wb.p, N, P, pl);
            wk.minres = minres;
            dmax.alloc(1);
            ck(rbmnqs::launch_max_diag(ddiag.p, P, dmax.p, h->st), "max diag");
            ck(rbmnqs::launch_cg_mfree(dO.p, 1, dd.p, norm, N, P, h->P_neural, dF.p, dx.p, ddiag.p, dmax.p, nullptr,
                                       r1, r2, rd, max_it, rtol, pl, wk, res.p, h->st),
               "matrix-free cg");
            ck(cudaStreamSynchronize(h->st), "sync");  // before wb goes out of scope
        } else {
            G.alloc((size_t)P * P);
            Sreg.alloc((size_t)P * P);
            const int ks = rbmnqs::gram_splits(N, P);
            part.alloc((size_t)ks * P * P);
            ck(rbmnqs::launch_gram_fp64(dO.p, 1, nullptr, N, P, ks, part.p, G.p, h->st), "gram");
            ck(rbmnqs::launch_solve_prep(G.p, N, norm, dd.p, ddiag.p, P, h->P_neural, r1, r2, rd, Sreg.p, h->st,
                                         direct),
               "prep");
            if (direct) {
                DevBuf<double2> wk;
                DevBuf<rbmnqs::MfreeSync> sy;
                wk.alloc(P);
                sy.alloc(1);
                ck(rbmnqs::launch_direct_solve(Sreg.p, dF.p, dx.p, P, wk.p, sy.p, res.p, h->st), "direct solve");
                ck(cudaStreamSynchronize(h->st), "sync");  // before wk, sy go out of scope
            } else if (minres) {
                rbmnqs::MfreePlan pl{};
                ck(rbmnqs::mfree_plan(1, P, &pl), "cooperative plan");
                DevBuf<unsigned char> wb;
                wb.alloc(rbmnqs::mfree_work_bytes(1, P, pl));
                rbmnqs::MfreeWork wk = rbmnqs::mfree_carve(wb.p, 1, P, pl);
                wk.minres = 1;
                ck(rbmnqs::launch_cg_dense_coop(Sreg.p, dF.p, dx.p, P, max_it, rtol, pl, wk, res.p, h->st),
                   "minres");
                ck(cudaStreamSynchronize(h->st), "sync");  // before wb goes out of scope
            } else {
                ck(rbmnqs::launch_cg(Sreg.p, dF.p, dx.p, P, max_it, rtol, res.p, h->st), "cg");
            }
        }
        rbmnqs::CgResultDev r{};
        ck(cudaMemcpyAsync(x_io, dx.p, P * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "c");
        ck(cudaMemcpyAsync(&r, res.p, sizeof(r), cudaMemcpyDeviceToHost, h->st), "c");
        ck(cudaStreamSynchronize(h->st), "sync");
        h->last_solve = r;
        if (iterations) *iterations = r.iterations;
        if (residual) *residual = r.residual;
    });
}

int rbmnqs_log_open(rbmnqs_handle* h, const char* name, int32_t force) {
    return guard([&] {
        require(h != nullptr && name != nullptr && name[0] != 0, "null handle or empty name");
        if (h->log.f) fclose(h->log.f);
        h->log.f = nullptr;
        const std::string fn = std::string(name) + ".log";
        FILE* probe = std::fopen(fn.c_str(), "r");
        const bool exists = probe != nullptr;
        if (probe) fclose(probe);
        h->log.f = std::fopen(fn.c_str(), exists && !force ? "a" : "w");
        require(h->log.f != nullptr, "cannot open " + fn);
        h->log.first = true;
    });
}

int rbmnqs_log_close(rbmnqs_handle* h) {
    return guard([&] {
        require(h != nullptr, "null handle");
        if (h->log.f) fclose(h->log.f);
        h->log.f = nullptr;
    });
}

int rbmnqs_solve_info(rbmnqs_handle* h, int32_t* iterations, double* residual, int32_t* istop, double* acond,
                      int32_t* qlp_iterations) {
    return guard([&] {
        require(h != nullptr, "null handle");
        const auto& r = h->last_solve;
        const bool mq = h->cfg.solver == 1;
        if (iterations) *iterations = r.iterations;
        if (residual) *residual = r.residual;
        if (istop) *istop = mq ? r.istop : 0;
        if (acond) *acond = mq ? r.acond : 0.0;
        if (qlp_iterations) *qlp_iterations = mq ? r.qlp_iterations : 0;
    });
}

int rbmnqs_full_sample(rbmnqs_handle* h, double* E_mean, double* dm, double* dh) {
    return guard([&] {
        require(h && E_mean, "bad arguments");
        require(h->n <= 30, "full enumeration needs n <= 30 (full_sampler.cpp:38-40 allows 64)",
                RBMNQS_ERR_UNSUPPORTED);
        const int64_t NS = int64_t(1) << h->n;
        const int P = h->P;
        const int64_t chunk = 1 << 16;
        std::vector<uint32_t> sp;
        std::vector<double> lp, el, Ob;
        // pass 1: max log|psi|
        double mx = -1e300;
        for (int64_t s0 = 0; s0 < NS; s0 += chunk) {
            const int B = (int)std::min(chunk, NS - s0);
            sp.assign((size_t)B * 4, 0);
            for (int b = 0; b < B; b++) sp[4 * b] = (uint32_t)(s0 + b);
            lp.resize(2 * B);
            eval_common(h, sp.data(), B, lp.data(), nullptr, nullptr, nullptr, 0, nullptr);
            for (int b = 0; b < B; b++) mx = std::max(mx, 2 * lp[2 * b]);
        }
        // pass 2: weighted sums (full_sampler.cpp:93-139)
        double pt = 0;
        cplx em = 0;
        std::vector<cplx> sd(dm ? P : 0), sh(dh ? P : 0);
        for (int64_t s0 = 0; s0 < NS; s0 += chunk) {
            const int B = (int)std::min(chunk, NS - s0);
            sp.assign((size_t)B * 4, 0);
            for (int b = 0; b < B; b++) sp[4 * b] = (uint32_t)(s0 + b);
            lp.resize(2 * B);
            el.resize(2 * B);
            if (dm || dh) Ob.resize((size_t)2 * B * P);
            eval_common(h, sp.data(), B, lp.data(), el.data(), (dm || dh) ? Ob.data() : nullptr, nullptr, 0,
                        nullptr);
            for (int b = 0; b < B; b++) {
                const double p = std::exp(2 * lp[2 * b] - mx);
                const cplx e(el[2 * b], el[2 * b + 1]);
                pt += p;
                em += p * e;
                if (dm || dh)
                    for (int k = 0; k < P; k++) {
                        const cplx o(Ob[(size_t)2 * (b * (size_t)P + k)], Ob[(size_t)2 * (b * (size_t)P + k) + 1]);
                        if (dm) sd[k] += p * o;
                        if (dh) sh[k] += p * e * std::conj(o);
                    }
            }
        }
        E_mean[0] = (em / pt).real();
        E_mean[1] = (em / pt).imag();
        for (int k = 0; dm && k < P; k++) {
            dm[2 * k] = (sd[k] / pt).real();
            dm[2 * k + 1] = (sd[k] / pt).imag();
        }
        for (int k = 0; dh && k < P; k++) {
            dh[2 * k] = (sh[k] / pt).real();
            dh[2 * k + 1] = (sh[k] / pt).imag();
        }
    });
}

int rbmnqs_full_state(rbmnqs_handle* h, double* psi) {
    return guard([&] {
        require(h && psi, "null argument");
        require(h->full, "rbmnqs_full_state needs sampler_type 1 (full enumeration)", RBMNQS_ERR_UNSUPPORTED);
        require(h->sampled, "rbmnqs_full_state needs a preceding sample or epoch");
        DevBuf<double2> v;
        v.alloc(h->N);
        ck(rbmnqs::launch_full_state_vector(h->lpsi.p, h->samples.p, h->N, h->fstat.p, v.p, h->st), "state vector");
        ck(cudaMemcpyAsync(psi, v.p, (size_t)h->N * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "copy");
        ck(cudaStreamSynchronize(h->st), "sync");
    });
}

int rbmnqs_get_observables(rbmnqs_handle* h, double* values) {
    return guard([&] {
        require(h && values, "null argument");
        require(!h->obs.empty(), "the model has no observables (rbmnqs_model_add_hexagons)");
        require(h->sampled, "rbmnqs_get_observables needs a preceding sample or epoch");
        const int no = (int)h->obs.size();
        if (!h->obsE.p) {
            h->obsE.alloc(h->N);
            h->obsMean.alloc(no);
            h->obsStats.alloc(no);
        }
        for (int i = 0; i < no; i++) {
            rbmnqs::EvalArgs ea = h->eval_args();
            ea.H = h->obs[i]->H;
            ea.plan.ham = rbmnqs::ham_stage_bytes(ea.H);
            ea.hd = h->obs[i]->hd.p;
            ea.tt = h->obs[i]->terms.tt;
            ea.O = nullptr;
            ea.eloc = h->obsE.p;
            ck(rbmnqs::launch_eval(ea, h->fp64, h->wpb, h->st), "observable evaluation");
            if (h->full) {
                ck(rbmnqs::launch_wmean(h->obsE.p, h->pw.p, h->N, h->fstat.p, h->obsMean.p + i, h->st),
                   "observable mean");
                ck(rbmnqs::launch_energy_stats_weighted(h->obsE.p, h->pw.p, h->N, h->n_bins, h->obsMean.p + i,
                                                        h->fstat.p, h->obsStats.p + i, h->st),
                   "observable statistics");
                continue;
            }
            ck(rbmnqs::launch_mean(h->obsE.p, h->N, h->obsMean.p + i, h->st), "observable mean");
            ck(rbmnqs::launch_energy_stats(h->obsE.p, h->N, h->n_bins, h->obsMean.p + i, h->nacc.p, h->nprop.p,
                                           h->cfg.n_chains, h->estat.p, h->obsStats.p + i, h->st),
               "observable statistics");
        }
        std::vector<rbmnqs::EpochStatsDev> st(no);
        ck(cudaMemcpyAsync(st.data(), h->obsStats.p, no * sizeof(st[0]), cudaMemcpyDeviceToHost, h->st), "copy");
        ck(cudaStreamSynchronize(h->st), "sync");
        for (int i = 0; i < no; i++) {
            values[4 * i] = st[i].energy.x;
            values[4 * i + 1] = st[i].energy.y;
            values[4 * i + 2] = st[i].stddev;
            values[4 * i + 3] = st[i].tau;
        }
    });
}

int rbmnqs_timing(rbmnqs_handle* h, double* ms, int64_t* launches, int32_t n) {
    return guard([&] {
        require(h != nullptr, "null handle");
        for (int i = 0; i < n && i < rbmnqs_handle::kStages; i++) {
            if (ms) ms[i] = h->stage_ms[i];
            if (launches) launches[i] = h->stage_launches[i];
        }
    });
}

int rbmnqs_timing_reset(rbmnqs_handle* h, int32_t enable) {
    return guard([&] {
        require(h != nullptr, "null handle");
        const bool en = enable != 0;
        if (en != h->timing && h->graph) {
            cudaGraphExecDestroy(h->graph);  // re-capture with/without event nodes
            h->graph = nullptr;
        }
        h->timing = en;
        for (int i = 0; i < rbmnqs_handle::kStages; i++) {
            h->stage_ms[i] = 0;
            h->stage_launches[i] = 0;
        }
    });
}

void* rbmnqs_stream(rbmnqs_handle* h) { return h ? (void*)h->st : nullptr; }

int rbmnqs_graph_kernels(rbmnqs_handle* h, int32_t* kernel_nodes) {
    return guard([&] {
        require(h && kernel_nodes, "null argument");
        *kernel_nodes = h->graph_kernels;
    });
}

int rbmnqs_test_fault(int32_t kind) {
    return guard([&] {
        require(kind >= 0 && kind <= 2, "rbmnqs_test_fault: kind must be 0, 1 or 2");
        g_test_fault.store(kind);
    });
}

int rbmnqs_probe_mufu(int32_t iters, double* ops_per_second) {
    return guard([&] {
        require(ops_per_second && iters > 0, "bad arguments");
        int dev = 0, sms = 0;
        ck(cudaGetDevice(&dev), "device");
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attr");
        cudaStream_t st;
        ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
        DevBuf<float> out;
        out.alloc(1);
        cudaEvent_t a, b;
        ck(cudaEventCreate(&a), "event");
        ck(cudaEventCreate(&b), "event");
        const int blocks = sms * 8;  // 2048 threads per SM
        ck(rbmnqs::launch_mufu_probe(out.p, iters, blocks, st), "probe");  // warm-up
        ck(cudaEventRecord(a, st), "event");
        ck(rbmnqs::launch_mufu_probe(out.p, iters, blocks, st), "probe");
        ck(cudaEventRecord(b, st), "event");
        ck(cudaEventSynchronize(b), "sync");
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, a, b), "elapsed");
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaStreamDestroy(st);
        *ops_per_second = 4.0 * iters * (double)blocks * 256.0 / (ms * 1e-3);
    });
}

int rbmnqs_autotune(rbmnqs_handle* h, int32_t sweeps, int32_t* sampler_wpb, int32_t* eval_wpb, double* sampler_ms) {
    return guard([&] {
        require(h != nullptr && sweeps >= 1, "rbmnqs_autotune: bad arguments");
        cudaEvent_t a, b;
        ck(cudaEventCreate(&a), "event");
        ck(cudaEventCreate(&b), "event");
        auto timed = [&](auto&& launch) {
            launch();  // warm-up
            ck(cudaEventRecord(a, h->st), "event");
            launch();
            ck(cudaEventRecord(b, h->st), "event");
            ck(cudaEventSynchronize(b), "sync");
            float ms = 0;
            ck(cudaEventElapsedTime(&ms, a, b), "elapsed");
            return (double)ms;
        };
        // chains restart from the same configurations in every trial and
        // get them back at the end
        const size_t sb = (size_t)h->cfg.n_chains * 16;
        DevBuf<uint32_t> saved;
        saved.alloc((size_t)h->cfg.n_chains * 4);
        ck(cudaMemcpyAsync(saved.p, h->spins.p, sb, cudaMemcpyDeviceToDevice, h->st), "save chains");
        double best_ms = 0;
        rbmnqs::SamplerArgs args = h->sampler_args();
        args.spc = 1;
        args.step = 1;
        args.warmup = sweeps - 1;
        if (!h->pf_n) {  // the Pfaffian buffers are sized for the planned shape
            rbmnqs::SamplerShape best = h->shape;
            best_ms = -1;
            // one or two chains per warp, then the warps per block
            for (int pm = 0; pm <= 1; pm++) {
                std::vector<int> tried;
                const int top = std::max(h->shape.warps_per_block, 32);
                for (int cap = top; cap >= 1; cap /= 2) {
                    rbmnqs::SamplerShape sh{};
                    ck(rbmnqs::plan_sampler(h->machine(), h->fp64, h->cfg.n_chains, h->n_prop_bonds, &sh, cap, pm),
                       "sampler plan");
                    if (sh.plan.pair != pm) break;  // two chains per warp not possible here
                    if (std::find(tried.begin(), tried.end(), sh.warps_per_block) != tried.end()) continue;
                    tried.push_back(sh.warps_per_block);
                    const double ms = timed([&] {
                        ck(cudaMemcpyAsync(h->spins.p, saved.p, sb, cudaMemcpyDeviceToDevice, h->st), "restore");
                        ck(rbmnqs::launch_sampler(args, h->fp64, sh, h->st), "sampler kernel");
                    });
                    if (best_ms < 0 || ms < best_ms) {
                        best_ms = ms;
                        best = sh;
                    }
                    if (tried.size() >= 5) break;
                }
            }
            rbmnqs::SamplerShape chk{};
            ck(rbmnqs::plan_sampler(h->machine(), h->fp64, h->cfg.n_chains, h->n_prop_bonds, &chk,
                                    best.warps_per_block, best.plan.pair),
               "sampler plan");
            h->shape = chk;
        }
        // evaluation kernel: 1..8 warps per block within the smem budget
        {
            rbmnqs::EvalArgs ea = h->eval_args();
            const rbmnqs::SmemPlan pl = h->eval_plan();
            double best = -1;
            int bw = h->wpb;
            for (int w = 1; w <= 8; w *= 2) {
                if (rbmnqs::eval_smem_bytes(h->machine(), h->fp64, w, pl) > 200 * 1024) break;
                const double ms = timed([&] { ck(rbmnqs::launch_eval(ea, h->fp64, w, h->st), "eval kernel"); });
                if (best < 0 || ms < best) {
                    best = ms;
                    bw = w;
                }
            }
            h->wpb = bw;
        }
        ck(cudaMemcpyAsync(h->spins.p, saved.p, sb, cudaMemcpyDeviceToDevice, h->st), "restore chains");
        ck(cudaStreamSynchronize(h->st), "sync");
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (h->graph) {  // re-capture with the new shapes
            cudaGraphExecDestroy(h->graph);
            h->graph = nullptr;
        }
        if (sampler_wpb) *sampler_wpb = h->shape.warps_per_block;
        if (eval_wpb) *eval_wpb = h->wpb;
        if (sampler_ms) *sampler_ms = best_ms;
    });
}

int rbmnqs_autotune_sr(rbmnqs_handle* h, int32_t* gram_splits, int32_t* cg_kernel, double* sr_ms) {
    return guard([&] {
        require(h != nullptr, "rbmnqs_autotune_sr: null handle");
        cudaEvent_t a, b;
        ck(cudaEventCreate(&a), "event");
        ck(cudaEventCreate(&b), "event");
        auto timed = [&](auto&& launch) {
            launch();  // warm-up
            ck(cudaEventRecord(a, h->st), "event");
            launch();
            ck(cudaEventRecord(b, h->st), "event");
            ck(cudaEventSynchronize(b), "sync");
            float ms = 0;
            ck(cudaEventElapsedTime(&ms, a, b), "elapsed");
            return (double)ms;
        };
        const double2* dS = h->full ? h->dzero.p : h->d.p;
        double total = 0;
        int32_t splits = 0, kernel = -1;
        // split-K count of the tensor-core Gram
        if (h->gram_tc) {
            int cand[6];
            const int nc = rbmnqs::gram_tc_split_candidates(h->gtc, cand, 6);
            double best = -1;
            int bs = h->gtc.nsplit;
            for (int i = 0; i < nc; i++) {
                ck(rbmnqs::gram_tc_set_splits(&h->gtc, cand[i]), "gram splits");
                const double ms = timed([&] {
                    ck(rbmnqs::launch_gram_tc(h->gtc, h->O.p, h->fp64, dS, h->gpart.p, h->gerr.p, h->Sm.p, h->st),
                       "tensor-core gram");
                });
                if (best < 0 || ms < best) {
                    best = ms;
                    bs = cand[i];
                }
            }
            ck(rbmnqs::gram_tc_set_splits(&h->gtc, bs), "gram splits");
            splits = bs;
            total += best;
        }
        // CG kernel on the formed S: the cluster CG against the cooperative
        // one-barrier CG (x restored after each trial)
        if (!h->mfree && h->cfg.solver == 0 && h->cfg.optimizer_type == 0 && rbmnqs::cg_cluster_fits(h->P)) {
            if (!h->mfbuf.p) {
                ck(rbmnqs::mfree_plan(1, h->P, &h->mfp), "cooperative CG plan");
                h->mfbuf.alloc(rbmnqs::mfree_work_bytes(1, h->P, h->mfp));
                h->mfw = rbmnqs::mfree_carve(h->mfbuf.p, 1, h->P, h->mfp);
                h->mfw.minres = 0;
            }
            if (h->gram_tc)
                ck(rbmnqs::launch_gram_tc(h->gtc, h->O.p, h->fp64, dS, h->gpart.p, h->gerr.p, h->Sm.p, h->st),
                   "tensor-core gram");
            else
                ck(rbmnqs::launch_gram_fp64(h->O.p, h->fp64, dS, h->N, h->P, h->gram_ks, h->part.p, h->Sm.p, h->st),
                   "gram");
            ck(rbmnqs::launch_regularize(h->Sm.p, h->P, h->P_neural, h->N, h->sched.p, h->diag.p, h->Sreg.p,
                                         h->maxdiag.p, h->st, 0, h->full ? h->fstat_vfac() : nullptr),
               "regularize");
            DevBuf<double2> x0;
            x0.alloc(h->P);
            ck(cudaMemcpyAsync(x0.p, h->x.p, h->P * sizeof(double2), cudaMemcpyDeviceToDevice, h->st), "save x");
            const int max_it = h->cg_max_it();
            const double rtol = h->cg_rtol();
            double ms[2];
            for (int k = 0; k < 2; k++)
                ms[k] = timed([&] {
                    ck(cudaMemcpyAsync(h->x.p, x0.p, h->P * sizeof(double2), cudaMemcpyDeviceToDevice, h->st),
                       "restore x");
                    if (k == 0)
                        ck(rbmnqs::launch_cg(h->Sreg.p, h->F.p, h->x.p, h->P, max_it, rtol, h->cgres.p, h->st), "cg");
                    else
                        ck(rbmnqs::launch_cg_dense_coop(h->Sreg.p, h->F.p, h->x.p, h->P, max_it, rtol, h->mfp, h->mfw,
                                                        h->cgres.p, h->st),
                           "cooperative solve");
                });
            ck(cudaMemcpyAsync(h->x.p, x0.p, h->P * sizeof(double2), cudaMemcpyDeviceToDevice, h->st), "restore x");
            kernel = ms[1] < ms[0] ? 1 : 0;
            h->coop_dense = kernel == 1;
            total += std::min(ms[0], ms[1]);
        }
        ck(cudaStreamSynchronize(h->st), "sync");
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (h->graph) {  // re-capture with the new choices
            cudaGraphExecDestroy(h->graph);
            h->graph = nullptr;
        }
        if (gram_splits) *gram_splits = splits;
        if (cg_kernel) *cg_kernel = kernel;
        if (sr_ms) *sr_ms = total;
    });
}

int rbmnqs_set_sweep_shape(rbmnqs_handle* h, int32_t warps_per_block, int32_t chains_per_warp) {
    return guard([&] {
        require(h && warps_per_block >= 0 && (chains_per_warp == 1 || chains_per_warp == 2), "bad arguments");
        require(!h->pf_n, "the Pfaffian buffers are sized for the planned shape", RBMNQS_ERR_UNSUPPORTED);
        rbmnqs::SamplerShape sh{};
        ck(rbmnqs::plan_sampler(h->machine(), h->fp64, h->cfg.n_chains, h->n_prop_bonds, &sh, warps_per_block,
                                chains_per_warp == 2 ? 1 : 0),
           "sampler plan");
        require(sh.plan.pair == (chains_per_warp == 2),
                "two chains per warp needs the FP32 expanded-table sweep with n <= 32", RBMNQS_ERR_UNSUPPORTED);
        h->shape = sh;
        if (h->graph) {
            cudaGraphExecDestroy(h->graph);
            h->graph = nullptr;
        }
    });
}

int rbmnqs_get_sweep_shape(rbmnqs_handle* h, int32_t* warps_per_block, int32_t* chains_per_warp) {
    return guard([&] {
        require(h != nullptr, "null handle");
        if (warps_per_block) *warps_per_block = h->shape.warps_per_block;
        if (chains_per_warp) *chains_per_warp = h->shape.plan.pair ? 2 : 1;
    });
}

}  // extern "C"

struct rbmnqs_batch {
    std::vector<rbmnqs_handle*> hs;
    cudaStream_t st = nullptr;
    cudaEvent_t fork = nullptr, solved = nullptr;
    std::vector<cudaEvent_t> joins, cg_done, joins2;
    cudaGraphExec_t graph = nullptr;
    int graph_kernels = 0;
    // sessions whose matrix-free CG runs in the merged multi-system launches
    // (one launch per precision and per kCgMultiMax systems)
    std::vector<char> merged;
    struct Group {
        int fp64, nprob;
        DevBuf<rbmnqs::CgMultiProb> probs;
        DevBuf<double2> t2;
        DevBuf<double> t1;
        DevBuf<rbmnqs::MfreeSync> sync;
        rbmnqs::CgMultiScratch sc{};
    };
    std::vector<std::unique_ptr<Group>> groups;
    int cg_blocks = 0;
    // sessions whose sweeps run in the batch's sweep launches (one per
    // entries-per-lane class with at least two sessions)
    std::vector<char> swept;
    struct SweepGroup {
        int E, nprob, blocks, smem;
        int first;  // the group's first session: its stream runs the launch
        cudaEvent_t done = nullptr;
        DevBuf<rbmnqs::BatchSweepDesc> desc;
        ~SweepGroup() {
            if (done) cudaEventDestroy(done);
        }
    };
    std::vector<int> sweep_group;  // per session: its sweep group, -1 none
    std::vector<std::unique_ptr<SweepGroup>> sweeps;
    ~rbmnqs_batch() {
        if (graph) cudaGraphExecDestroy(graph);
        for (auto* v : {&joins, &cg_done, &joins2})
            for (auto e : *v)
                if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (solved) cudaEventDestroy(solved);
        if (st) cudaStreamDestroy(st);
    }
};

extern "C" {

int rbmnqs_batch_create(rbmnqs_handle* const* sessions, int32_t n, rbmnqs_batch** out) {
    return guard([&] {
        require(sessions && out && n >= 1, "rbmnqs_batch_create: bad arguments");
        auto b = std::make_unique<rbmnqs_batch>();
        for (int i = 0; i < n; i++) {
            require(sessions[i] != nullptr, "rbmnqs_batch_create: null session");
            require(std::find(b->hs.begin(), b->hs.end(), sessions[i]) == b->hs.end(),
                    "rbmnqs_batch_create: a session appears twice");
            b->hs.push_back(sessions[i]);
        }
        ck(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking), "stream");
        ck(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "event");
        ck(cudaEventCreateWithFlags(&b->solved, cudaEventDisableTiming), "event");
        b->joins.resize(n, nullptr);
        b->cg_done.resize(n, nullptr);
        b->joins2.resize(n, nullptr);
        for (auto& e : b->joins) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        for (auto& e : b->cg_done) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        for (auto& e : b->joins2) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        // matrix-free CG systems of the same precision share launches when
        // there are at least two of them
        b->merged.assign(n, 0);
        for (int fp = 0; fp < 2; fp++) {
            std::vector<int> idx;
            for (int i = 0; i < n; i++)
                if (b->hs[i]->batch_cg() && b->hs[i]->fp64 == fp) idx.push_back(i);
            if (idx.size() < 2) continue;
            for (size_t g0 = 0; g0 < idx.size(); g0 += rbmnqs::kCgMultiMax) {
                auto g = std::make_unique<rbmnqs_batch::Group>();
                std::vector<rbmnqs::CgMultiProb> pr;
                for (size_t k = g0; k < std::min(idx.size(), g0 + rbmnqs::kCgMultiMax); k++) {
                    pr.push_back(b->hs[idx[k]]->cg_prob());
                    b->merged[idx[k]] = 1;
                }
                g->fp64 = fp;
                g->nprob = (int)pr.size();
                long long rc = 0, tc = 0;
                const int tiles = rbmnqs::cg_multi_units(pr.data(), g->nprob, &rc, &tc);
                g->probs.alloc(pr.size());
                g->t2.alloc(2 * (size_t)tiles);
                g->t1.alloc(tiles);
                g->sync.alloc(1);
                ck(cudaMemcpyAsync(g->probs.p, pr.data(), pr.size() * sizeof(rbmnqs::CgMultiProb),
                                   cudaMemcpyHostToDevice, b->st),
                   "copy");
                g->sc.tdb = g->t2.p;
                g->sc.tpap = g->t2.p + tiles;
                g->sc.trs = g->t1.p;
                g->sc.sync = g->sync.p;
                g->sc.row_cost = rc;
                g->sc.tile_cost = tc;
                b->groups.push_back(std::move(g));
            }
        }
        if (!b->groups.empty()) ck(rbmnqs::cg_multi_blocks(&b->cg_blocks), "multi-system CG plan");
        // sweeps: the plain FP32 Metropolis sessions grouped by entries per lane
        b->swept.assign(n, 0);
        b->sweep_group.assign(n, -1);
        for (int E = 1; E <= 8; E *= 2) {
            std::vector<rbmnqs::BatchSweepDesc> ds;
            std::vector<int> idx;
            int smem = 0, blocks = 0;
            for (int i = 0; i < n; i++) {
                rbmnqs_handle* h = b->hs[i];
                if (h->fp64 || h->pf_n || h->net || h->full || rbmnqs::elements_per_lane(h->T) != E) continue;
                rbmnqs::BatchSweepDesc d{};
                d.a = h->sampler_args();
                int sm = 0;
                if (!rbmnqs::sampler_batch_plan(h->machine(), 0, h->cfg.n_chains, h->n_prop_bonds, &d, &sm)) continue;
                d.block0 = blocks;
                blocks += d.blocks;
                smem = std::max(smem, sm);
                ds.push_back(d);
                idx.push_back(i);
            }
            if (ds.size() < 2) continue;
            auto g = std::make_unique<rbmnqs_batch::SweepGroup>();
            g->E = E;
            g->nprob = (int)ds.size();
            g->blocks = blocks;
            g->smem = smem;
            g->desc.alloc(ds.size());
            ck(cudaMemcpyAsync(g->desc.p, ds.data(), ds.size() * sizeof(rbmnqs::BatchSweepDesc),
                               cudaMemcpyHostToDevice, b->st),
               "copy");
            g->first = idx[0];
            ck(cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming), "event");
            for (int i : idx) {
                b->swept[i] = 1;
                b->sweep_group[i] = (int)b->sweeps.size();
            }
            b->sweeps.push_back(std::move(g));
        }
        ck(cudaStreamSynchronize(b->st), "sync");
        *out = b.release();
    });
}

int rbmnqs_batch_epoch(rbmnqs_batch* b, rbmnqs_sample_stats* s, rbmnqs_sr_stats* o) {
    return guard([&] {
        require(b != nullptr, "null batch");
        if (!b->graph) {
            // fork: every session's epoch on its own stream, joined back
            cudaGraph_t g;
            ck(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal), "capture");
            try {
                ck(cudaEventRecord(b->fork, b->st), "fork");
                // the batched sweeps, each class on the stream of its first
                // session, concurrently; the sessions of a class continue
                // after its launch
                for (auto& g : b->sweeps) {
                    cudaStream_t gs = b->hs[g->first]->st;
                    ck(cudaStreamWaitEvent(gs, b->fork, 0), "fork wait");
                    ck(rbmnqs::launch_sampler_batch(g->E, g->desc.p, g->nprob, g->blocks, g->smem, gs), "batch sweep");
                    ck(cudaEventRecord(g->done, gs), "swept");
                }
                cudaEvent_t prev_cg = nullptr;  // cooperative solves run one after another
                for (size_t i = 0; i < b->hs.size(); i++) {
                    rbmnqs_handle* h = b->hs[i];
                    ck(cudaStreamWaitEvent(h->st, b->fork, 0), "fork wait");
                    if (b->sweep_group[i] >= 0) ck(cudaStreamWaitEvent(h->st, b->sweeps[b->sweep_group[i]]->done, 0), "swept wait");
                    h->batch_swept = b->swept[i] != 0;
                    h->enqueue_sample();
                    h->batch_swept = false;
                    if (b->merged[i]) {
                        h->enqueue_optimize_pre();
                    } else if (h->coop_solve()) {
                        h->enqueue_optimize(prev_cg, b->cg_done[i]);
                        prev_cg = b->cg_done[i];
                    } else {
                        h->enqueue_optimize();
                    }
                    ck(cudaEventRecord(b->joins[i], h->st), "join");
                    ck(cudaStreamWaitEvent(b->st, b->joins[i], 0), "join wait");
                }
                if (!b->groups.empty()) {
                    // the merged matrix-free solves, after every session's
                    // sample and var(O) (and after the other cooperative
                    // solves), then each merged session's update
                    for (auto& g : b->groups)
                        ck(rbmnqs::launch_cg_multi(g->probs.p, g->nprob, g->fp64, g->sc, b->cg_blocks, b->st),
                           "matrix-free cg");
                    ck(cudaEventRecord(b->solved, b->st), "solved");
                    for (size_t i = 0; i < b->hs.size(); i++) {
                        if (!b->merged[i]) continue;
                        rbmnqs_handle* h = b->hs[i];
                        ck(cudaStreamWaitEvent(h->st, b->solved, 0), "solved wait");
                        h->enqueue_optimize_post();
                        ck(cudaEventRecord(b->joins2[i], h->st), "join");
                        ck(cudaStreamWaitEvent(b->st, b->joins2[i], 0), "join wait");
                    }
                }
            } catch (...) {
                for (auto* h : b->hs) h->batch_swept = false;
                cudaStreamEndCapture(b->st, &g);
                throw;
            }
            ck(cudaStreamEndCapture(b->st, &g), "end capture");
            b->graph_kernels = count_kernel_nodes(g);
            ck(cudaGraphInstantiate(&b->graph, g, 0), "instantiate");
            cudaGraphDestroy(g);
        }
        ck(cudaGraphLaunch(b->graph, b->st), "graph launch");
        ck(cudaStreamSynchronize(b->st), "sync");
        for (size_t i = 0; i < b->hs.size(); i++) {
            readback(b->hs[i], true, s ? s + i : nullptr, true, o ? o + i : nullptr);
            b->hs[i]->sampled = true;
        }
    });
}

int rbmnqs_batch_graph_kernels(rbmnqs_batch* b, int32_t* kernel_nodes) {
    return guard([&] {
        require(b && kernel_nodes, "null argument");
        *kernel_nodes = b->graph_kernels;
    });
}

void* rbmnqs_batch_stream(rbmnqs_batch* b) { return b ? (void*)b->st : nullptr; }

void rbmnqs_batch_destroy(rbmnqs_batch* b) { delete b; }

}  // extern "C"

struct rbmnqs_mlp {
    cudaStream_t st = nullptr;
    std::unique_ptr<rbmnqs::Mlp> net;
    DevBuf<uint32_t> spins, targets;
    DevBuf<float> loss, soft;  // soft: [max_batch][n_out] targets of the softmax loss
    ~rbmnqs_mlp() {
        net.reset();
        if (st) cudaStreamDestroy(st);
    }
};

namespace {
void mlp_upload(rbmnqs_mlp* m, const uint32_t* spins, const uint32_t* targets, int B) {
    require(B >= 1 && B <= m->net->max_batch(), "batch larger than max_batch");
    ck(cudaMemcpyAsync(m->spins.p, spins, (size_t)B * 16, cudaMemcpyHostToDevice, m->st), "copy");
    if (targets) ck(cudaMemcpyAsync(m->targets.p, targets, (size_t)B * 16, cudaMemcpyHostToDevice, m->st), "copy");
}
void mlp_check(rbmnqs_mlp* m) {
    ck(cudaStreamSynchronize(m->st), "sync");
    const int e = m->net->error_flag_host();
    if (e) {
        ck(m->net->clear_error(m->st), "memset");
        ck(cudaStreamSynchronize(m->st), "sync");
        throw Fail{RBMNQS_ERR_CUDA, "proposal network GEMM: pipeline wait timed out (code " + std::to_string(e) + ")"};
    }
}
}  // namespace

extern "C" {

int rbmnqs_mlp_create(int32_t n_in, int32_t h1, int32_t h2, int32_t n_out, int32_t max_batch, rbmnqs_mlp** out) {
    return guard([&] {
        require(out && n_in >= 1 && n_in <= 256 && n_out >= 1 && n_out <= 256 && h1 % 64 == 0 && h2 % 64 == 0 &&
                    h1 >= 64 && h1 <= 256 && h2 >= 64 && h2 <= 256 && max_batch >= 1,
                "rbmnqs_mlp_create: unsupported sizes");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            throw Fail{RBMNQS_ERR_NO_DEVICE, "no CUDA device available"};
        auto m = std::make_unique<rbmnqs_mlp>();
        ck(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking), "stream");
        rbmnqs::MlpDims d;
        d.n_in = n_in;
        d.h1 = h1;
        d.h2 = h2;
        d.n_out = n_out;
        try {
            m->net = std::make_unique<rbmnqs::Mlp>(d, max_batch, m->st);
        } catch (cudaError_t e) {
            ck(e, "proposal network");
        }
        const int bm = m->net->max_batch();
        m->spins.alloc((size_t)bm * 4);
        m->targets.alloc((size_t)bm * 4);
        m->loss.alloc(1);
        ck(cudaStreamSynchronize(m->st), "sync");
        *out = m.release();
    });
}

int rbmnqs_mlp_n_params(const rbmnqs_mlp* m, int64_t* n) {
    return guard([&] {
        require(m && n, "null argument");
        const auto& d = m->net->dims();
        *n = (int64_t)d.h1 * d.n_in + d.h1 + (int64_t)d.h2 * d.h1 + d.h2 + (int64_t)d.n_out * d.h2 + d.n_out;
    });
}

int rbmnqs_mlp_set_params(rbmnqs_mlp* m, const float* params) {
    return guard([&] {
        require(m && params, "null argument");
        ck(m->net->set_params(params), "set params");
        mlp_check(m);
    });
}

int rbmnqs_mlp_get_params(rbmnqs_mlp* m, float* params) {
    return guard([&] {
        require(m && params, "null argument");
        ck(m->net->get_params(params), "get params");
    });
}

int rbmnqs_mlp_init(rbmnqs_mlp* m, float std, uint64_t seed) {
    return guard([&] {
        require(m != nullptr, "null argument");
        ck(m->net->init_random(std, seed), "init");
        mlp_check(m);
    });
}

int rbmnqs_mlp_forward(rbmnqs_mlp* m, const uint32_t* spins, int32_t B, float* logits) {
    return guard([&] {
        require(m && spins, "null argument");
        mlp_upload(m, spins, nullptr, B);
        ck(m->net->forward(m->spins.p, B, m->st), "forward");
        if (logits) {
            const auto& d = m->net->dims();
            std::vector<float> t((size_t)B * d.out_p);
            ck(cudaMemcpyAsync(t.data(), m->net->logits(), t.size() * 4, cudaMemcpyDeviceToHost, m->st), "copy");
            mlp_check(m);
            for (int b = 0; b < B; b++)
                for (int o = 0; o < d.n_out; o++) logits[(size_t)b * d.n_out + o] = t[(size_t)b * d.out_p + o];
        } else {
            mlp_check(m);
        }
    });
}

namespace {
// loss and gradients of the last training step, gradients in the logical
// flat parameter layout
void mlp_results(rbmnqs_mlp* m, float* loss, float* grads);
}  // namespace

int rbmnqs_mlp_train_step(rbmnqs_mlp* m, const uint32_t* spins, const uint32_t* targets, int32_t B, float lr,
                          int32_t apply, float* loss, float* grads) {
    return guard([&] {
        require(m && spins && targets, "null argument");
        mlp_upload(m, spins, targets, B);
        ck(m->net->train_step(m->spins.p, m->targets.p, B, lr, m->st, m->loss.p, apply != 0), "train step");
        mlp_results(m, loss, grads);
    });
}

int rbmnqs_mlp_train_step_soft(rbmnqs_mlp* m, const uint32_t* spins, const float* targets, int32_t B, float lr,
                               int32_t apply, float* loss, float* grads) {
    return guard([&] {
        require(m && spins && targets, "null argument");
        mlp_upload(m, spins, nullptr, B);
        const size_t cnt = (size_t)B * m->net->dims().n_out;
        if (m->soft.n < cnt) m->soft.alloc((size_t)m->net->max_batch() * m->net->dims().n_out);
        ck(cudaMemcpyAsync(m->soft.p, targets, cnt * 4, cudaMemcpyHostToDevice, m->st), "copy");
        ck(m->net->train_step_soft(m->spins.p, m->soft.p, B, lr, m->st, m->loss.p, apply != 0), "train step");
        mlp_results(m, loss, grads);
    });
}

}  // extern "C"

namespace {
void mlp_results(rbmnqs_mlp* m, float* loss, float* grads) {
    {
        float l = 0;
        ck(cudaMemcpyAsync(&l, m->loss.p, 4, cudaMemcpyDeviceToHost, m->st), "copy");
        std::vector<float> g;
        if (grads) {
            g.resize(m->net->n_params());
            ck(cudaMemcpyAsync(g.data(), m->net->grads(), g.size() * 4, cudaMemcpyDeviceToHost, m->st), "copy");
        }
        mlp_check(m);
        if (loss) *loss = l;
        if (grads) {
            // padded -> logical layout
            const auto& d = m->net->dims();
            const int rows[3] = {d.h1, d.h2, d.n_out}, cols[3] = {d.n_in, d.h1, d.h2};
            const int prow[3] = {d.h1, d.h2, d.out_p}, pcol[3] = {d.in_p, d.h1, d.h2};
            size_t src = 0, dst = 0;
            for (int l2 = 0; l2 < 3; l2++) {
                for (int r = 0; r < rows[l2]; r++)
                    for (int c = 0; c < cols[l2]; c++) grads[dst++] = g[src + (size_t)r * pcol[l2] + c];
                src += (size_t)prow[l2] * pcol[l2];
                for (int r = 0; r < rows[l2]; r++) grads[dst++] = g[src + r];
                src += prow[l2];
            }
        }
    }
}
}  // namespace

extern "C" {

int rbmnqs_mlp_intermediate(rbmnqs_mlp* m, int32_t which, int32_t B, float* out, int32_t* cols) {
    return guard([&] {
        require(m != nullptr && B >= 1 && B <= m->net->max_batch(), "bad arguments");
        int c = 0;
        ck(m->net->intermediate(which, B, out, &c), "intermediate");
        if (cols) *cols = c;
    });
}

void rbmnqs_mlp_destroy(rbmnqs_mlp* m) { delete m; }

}  // extern "C"

// ----------------------------------------------------------- checkpoints --
namespace {
void write_mat(std::FILE* f, const cplx* data, uint64_t rows, uint64_t cols) {
    require(std::fwrite(&rows, 8, 1, f) == 1 && std::fwrite(&cols, 8, 1, f) == 1 &&
                std::fwrite(data, sizeof(cplx), rows * cols, f) == rows * cols,
            "checkpoint write failed");
}
void read_mat(std::FILE* f, cplx* data, uint64_t rows, uint64_t cols) {
    uint64_t r = 0, c = 0;
    require(std::fread(&r, 8, 1, f) == 1 && std::fread(&c, 8, 1, f) == 1, "checkpoint truncated");
    require(r == rows && c == cols, "checkpoint dimension mismatch: file " + std::to_string(r) + " x " +
                                        std::to_string(c) + ", machine " + std::to_string(rows) + " x " +
                                        std::to_string(cols));
    require(std::fread(data, sizeof(cplx), rows * cols, f) == rows * cols, "checkpoint truncated");
}
}  // namespace

extern "C" {

int rbmnqs_save(rbmnqs_handle* h, const char* path) {
    return guard([&] {
        require(h && path, "null argument");
        std::vector<cplx> w(h->P);
        ck(cudaMemcpyAsync(w.data(), h->params.p, h->P * sizeof(double2), cudaMemcpyDeviceToHost, h->st), "copy");
        ck(cudaStreamSynchronize(h->st), "sync");
        std::FILE* f = std::fopen(path, "wb");
        require(f != nullptr, std::string("cannot open ") + path);
        try {
            const int nvb = h->n_vb, nh = h->nh, n = h->n;
            // rbm_base::save order: weights_, h_bias_, v_bias_, n_updates_, pfaffian fs_
            write_mat(f, w.data() + nvb + nh, n, nh);
            write_mat(f, w.data() + nvb, nh, 1);
            write_mat(f, w.data(), nvb, 1);
            const uint64_t nu = (uint64_t)h->n_updates;
            require(std::fwrite(&nu, 8, 1, f) == 1, "checkpoint write failed");
            if (h->pf_n) write_mat(f, w.data() + h->P_neural, h->pf_indep, 4);
        } catch (...) {
            std::fclose(f);
            throw;
        }
        require(std::fclose(f) == 0, "checkpoint write failed");
    });
}

int rbmnqs_load(rbmnqs_handle* h, const char* path) {
    return guard([&] {
        require(h && path, "null argument");
        std::vector<cplx> w(h->P);
        std::FILE* f = std::fopen(path, "rb");
        require(f != nullptr, std::string("cannot open ") + path);
        uint64_t nu = 0;
        try {
            const int nvb = h->n_vb, nh = h->nh, n = h->n;
            read_mat(f, w.data() + nvb + nh, n, nh);
            read_mat(f, w.data() + nvb, nh, 1);
            read_mat(f, w.data(), nvb, 1);
            require(std::fread(&nu, 8, 1, f) == 1, "checkpoint truncated");
            if (h->pf_n) read_mat(f, w.data() + h->P_neural, h->pf_indep, 4);
        } catch (...) {
            std::fclose(f);
            throw;
        }
        std::fclose(f);
        ck(cudaMemcpyAsync(h->params.p, w.data(), h->P * sizeof(double2), cudaMemcpyHostToDevice, h->st), "copy");
        ck(rbmnqs::launch_unpack(h->params.p, h->n, h->n_vb, h->nh, h->vb.p, h->hb.p, h->W64.p, h->W32.p, h->st),
           "unpack");
        h->n_updates = (int64_t)nu;
        set_schedules(h, h->n_updates);
    });
}

int rbmnqs_n_updates(const rbmnqs_handle* h, int64_t* n_updates) {
    return guard([&] {
        require(h && n_updates, "null argument");
        *n_updates = h->n_updates;
    });
}

}  // extern "C"
