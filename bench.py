"""Benchmark of the VMC hot path (one SR epoch per step) on B200.

Default workload (the config the headline metric is quoted on): Kitaev
honeycomb n_cells=8 (128 spins), J=-1, h=0; symmetric RBM (symmetry 0.5),
alpha=4 -> 517 parameters; 16384 chains, 16 samples per chain one sweep
apart (persistent chains), single-spin-flip sweeps; SR with CG.

The metric compares forms of the method on the same trained wavefunction:
a checkpoint is trained first (plain FP32 SR from seeded complex Gaussian
weights of std 1e-4, 600 epochs of 4096 chains; saved with rbmnqs_save and
loaded by every form), then each form runs its epochs from it:
  * learned  -- the headline `value`: mixed precision (FP32 psi ratios,
    FP64 theta recompute, FP16x3 split-precision tensor-core Gram, FP64 CG), the whole epoch
    as one CUDA graph, one learned move per sample after each sweep (the
    proposal network trained every epoch);
  * plain_fp32 -- the same without the learned moves;
  * plain_fp64 -- plain GPU Metropolis in the reference's arithmetic (FP64
    throughout), launched stage by stage.
Uncorrelated samples/s = N / (1 + 2 tau) per epoch time, tau the
reference's binning estimate of the E_loc autocorrelation along the chains;
SR epochs/s, E/site and their differences are reported beside it.
`--impl reference` times the reference algorithm's CPU restatement (the
FP64 oracle; the reference itself cannot be built here) on all host cores on
a bounded sample of the same workload.

Multi-GPU: the path does not shard (one GPU, no collective); --gpus N runs N
independent replicas, one process per GPU under torchrun, timed as the max
over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rbm-nqs_b200"))

import numpy as np  # noqa: E402

# Workloads (seeded synthetic inputs of the benchmark shapes).  The metric
# line is quoted on kitaev128_forms; the others measure the 32-spin lattice,
# the Pfaffian path and the batched toric problems with the same harness.
WORKLOADS = {
    # the metric's config: the 128-spin Kitaev lattice, forms compared on a
    # trained checkpoint (see the module docstring)
    "kitaev128_forms": dict(model="kitaev", n_cells=8, rbm_type=1, alpha=4, symmetry=0.5, n_chains=16384,
                            samples_per_chain=16, warmup=0, step=1, bond_flips=0.0, std=1e-4,
                            reg2=(1e-4, 1e-4, 1.0), precision=0, gram=0, forms=True,
                            train=dict(n_chains=4096, warmup=15, bond_flips=0.5, epochs=600),
                            learned=dict(proposal=1, learned_steps=1, learned_train=2, learned_lr=1e-3)),
    # Kitaev 32 spins, symmetric RBM alpha=4, 4096 chains x 64 sweeps,
    # FP32 sweep / FP64 theta recompute, FP16x3 split-precision tensor-core Gram, FP64 CG
    "kitaev32_symm_a4": dict(model="kitaev", n_cells=4, rbm_type=1, alpha=4, symmetry=0.5, n_chains=4096,
                             samples_per_chain=1, warmup=63, step=1, bond_flips=0.5, std=1e-4,
                             reg2=(1e-4, 1e-4, 1.0), precision=0, gram=0),
    # RBM alpha=2 + Pfaffian (pair classes of symmetry 0.5, std 1e-2), 2048
    # chains, X^{-1} rebuilt every 32 accepted moves, FP64 Gram and CG
    "kitaev32_pf_symm_a2": dict(model="kitaev", n_cells=4, rbm_type=1, alpha=2, symmetry=0.5, n_chains=2048,
                                samples_per_chain=1, warmup=63, step=1, bond_flips=0.5, std=1e-4,
                                reg2=(1e-4, 1e-4, 1.0), precision=0, gram=1, pfaffian=1, pf_symmetry=0.5,
                                pf_std=1e-2, pf_refresh=32),
    # Kitaev 128 spins, symmetric RBM alpha=4, 16384 chains, plain
    # single-spin/bond Metropolis
    "kitaev128_symm_a4": dict(model="kitaev", n_cells=8, rbm_type=1, alpha=4, symmetry=0.5, n_chains=16384,
                              samples_per_chain=1, warmup=63, step=1, bond_flips=0.5, std=1e-4,
                              reg2=(1e-4, 1e-4, 1.0), precision=0, gram=0),
    # the 128-spin lattice as a time series (persistent chains, 16 samples per
    # chain, 4 sweeps apart), seeded weights (profiling)
    "kitaev128_plain_ts": dict(model="kitaev", n_cells=8, rbm_type=1, alpha=4, symmetry=0.5, n_chains=16384,
                               samples_per_chain=16, warmup=0, step=4, bond_flips=0.5, std=1e-4,
                               reg2=(1e-4, 1e-4, 1.0), precision=0, gram=0),
    # 48 independent toric-code trainings (L = 3..8, 8 each, basic RBM
    # alpha=2, 1024 chains each) advanced by one CUDA-graph launch per epoch;
    # launch shapes autotuned per L; matrix-free CG capped at 100 iterations
    "toric_batch48": dict(model="toric", batch_L=(3, 4, 5, 6, 7, 8), batch_copies=8, rbm_type=0, alpha=2,
                          symmetry=1.0, n_chains=1024, samples_per_chain=1, warmup=63, step=1, bond_flips=0.0,
                          std=1e-4, reg2=(1e-4, 1e-4, 1.0), precision=0, gram=0, max_iterations=100),
}
METRIC = "uncorrelated samples/s (SR epoch, E_loc binning tau)"
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes per sampler launch from an ncu capture of the same workload: the
# theta tables, flip tables and chains live in shared memory and registers
SAMPLER_DRAM_BYTES = {"kitaev32_symm_a4": 136704.0}
# DRAM bytes per launch of the evaluation kernel: the O store written (N x P
# FP32 complex); the capture of 32768 samples wrote 78.9 MB (the rest of its
# 135.5 MB still in L2 when the kernel ended), scaled by 8 to the 262144
# samples of one launch
ELOC_DRAM_BYTES = {"kitaev128_forms": 8 * 79.5e6}
ELOC_TRAFFIC_SOURCE = ("dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of 32768 samples "
                       "(profiles/eloc_kernel_kitaev128_symm_a4.md), scaled to 262144 samples")
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="kitaev128_forms", choices=list(WORKLOADS))
    ap.add_argument("--train-epochs", type=int, default=0, help="override the checkpoint's training epochs")
    ap.add_argument("--cpu-baseline", type=int, default=1, help="time the CPU restatement beside our arm")
    ap.add_argument("--chains", type=int, default=0, help="override the workload's chain count (profiling)")
    ap.add_argument("--sweeps", type=int, default=0, help="override the sweeps per epoch (profiling)")
    ap.add_argument("--pf-refresh", type=int, default=-1,
                    help="override the Pfaffian workloads' refresh period in accepted moves (0: never; profiling)")
    ap.add_argument("--forms", default="learned,plain_fp32,plain_fp64",
                    help="forms of the 128-spin workload to run (profiling runs a subset; the metric line needs all)")
    ap.add_argument("--profile-region", type=int, default=0,
                    help="bracket each form's timed epochs with cudaProfilerStart/Stop (ncu --profile-from-start off)")
    return ap.parse_args()


def workload(args):
    wl = dict(WORKLOADS[args.workload])
    if args.chains:
        wl["n_chains"] = args.chains
    if args.sweeps:
        wl["warmup"] = args.sweeps - wl["samples_per_chain"] * wl["step"]
    if args.pf_refresh >= 0 and wl.get("pfaffian"):
        wl["pf_refresh"] = args.pf_refresh
    return wl


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world, backend):
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        import datetime
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(values, world, device="cuda"):
    """Device times of every rank reduced to their maximum (the job's time
    is the slowest replica's); unchanged with one rank."""
    if world <= 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def make_weights(P, std, seed, n_neural=None, pf_std=None):
    """complex Gaussian weights; pair parameters (index >= n_neural) with pf_std"""
    rng = np.random.default_rng(seed)
    w = rng.normal(0, std, P) + 1j * rng.normal(0, std, P)
    if n_neural is not None and pf_std is not None and n_neural < P:
        m = P - n_neural
        w[n_neural:] = rng.normal(0, pf_std, m) + 1j * rng.normal(0, pf_std, m)
    return w


def describe(wl, P):
    kind = "symmetric RBM" if wl["rbm_type"] == 1 else "RBM"
    d = {"model": f"kitaev honeycomb n_cells={wl['n_cells']} ({2 * wl['n_cells'] ** 2} spins) J=-1",
         "machine": f"{kind} alpha={wl['alpha']}" + (" + Pfaffian (pair symmetry %g)" % wl["pf_symmetry"]
                                                      if wl.get("pfaffian") else "") + f", {P} params",
         "n_chains": wl["n_chains"], "sweeps_per_epoch": wl["warmup"] + wl["samples_per_chain"] * wl["step"],
         "samples_per_epoch": wl["n_chains"] * wl["samples_per_chain"], "bond_flips": wl["bond_flips"],
         "gram": "FP16x3 split-precision tcgen05" if wl["gram"] == 0 and wl["precision"] == 0 else "FP64",
         "sr": "CG reg2=1e-4 reg1=(1,1e-4,0.9) lr=1e-2"}
    if wl.get("pfaffian"):
        d["pfaffian_refresh"] = wl["pf_refresh"]
    if wl.get("proposal"):
        d["proposal"] = "learned (MLP %d-256-256-%d, BF16), %d move(s) per sample, %d Adam step(s) per epoch" % (
            2 * wl["n_cells"] ** 2, 2 * wl["n_cells"] ** 2, wl["learned_steps"], wl["learned_train"])
    return d


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------- ours --
def run_ours(args, rank, world, local):
    import torch
    import rbmnqs

    dist = init_dist(world, "nccl")
    torch.cuda.set_device(local)
    wl = workload(args)
    model = rbmnqs.Model.kitaev(wl["n_cells"], symmetry=wl["symmetry"])
    cfg = rbmnqs.default_config(rbm_type=wl["rbm_type"], alpha=wl["alpha"], n_chains=wl["n_chains"],
                                samples_per_chain=wl["samples_per_chain"], warmup=wl["warmup"], step=wl["step"],
                                bond_flips=wl["bond_flips"], seed=1234 + rank, precision=wl["precision"],
                                gram=wl["gram"], reinit_chains=0, reg2=wl["reg2"],
                                pfaffian=wl.get("pfaffian", 0), pfaffian_symmetry=wl.get("pf_symmetry", 0.5),
                                pfaffian_refresh=wl.get("pf_refresh", 0), proposal=wl.get("proposal", 0),
                                learned_steps=wl.get("learned_steps", 1), learned_train=wl.get("learned_train", 1),
                                learned_lr=wl.get("learned_lr", 1e-3))
    sess = rbmnqs.Session(model, cfg)
    P, N = sess.n_params, sess.N
    w0 = make_weights(P, wl["std"], 99 + rank, sess.n_neural, wl.get("pf_std"))
    sess.set_weights(w0)
    stream = torch.cuda.ExternalStream(sess.stream())
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def l2_flush():
        with torch.cuda.stream(stream):
            flush.zero_()

    for _ in range(max(3, args.warmup)):
        sess.epoch()
    sess.timing_reset(True)
    sess.epoch()  # re-capture with event nodes; not timed
    sess.timing_reset(True)
    kern_per_epoch = sess.graph_kernels()

    # ---- device-timed region: K epochs, each bracketed by events on the
    # library's stream, L2 flushed between epochs (outside the events)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    taus, energies, accs, its, errs, laccs = [], [], [], [], [], []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if args.profile_region:
        torch.cuda.profiler.start()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            l2_flush()
            ev[k][0].record(stream)
            st, sr = sess.epoch()
            ev[k][1].record(stream)
            taus.append(st["tau"])
            energies.append(st["energy"].real)
            accs.append(st["acceptance"])
            errs.append(st["stddev"])
            if wl.get("proposal"):
                laccs.append(st["learned_acceptance"])
            its.append(sr["iterations"])
        torch.cuda.synchronize()
    if args.profile_region:
        torch.cuda.profiler.stop()
    if world > 1:
        dist.barrier()
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    stage_ms, stage_cnt = sess.timing()
    clocks = clk.summary()

    # ---- end to end through the C ABI with host buffers: weights in,
    # epoch, weights + stats out, every step
    w = sess.get_weights()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for k in range(args.steps):
        l2_flush()
        ev2[k][0].record(stream)
        sess.set_weights(w)
        sess.epoch()
        w = sess.get_weights()
        ev2[k][1].record(stream)
    torch.cuda.synchronize()
    t2_ms = sum(a.elapsed_time(b) for a, b in ev2)

    t_ms, t2_ms = max_over_ranks([t_ms, t2_ms], world)
    tau = float(np.mean(taus))
    neff_epoch = N / (1.0 + 2.0 * tau)
    value = world * args.steps * neff_epoch / (t_ms * 1e-3)
    e2e = world * args.steps * neff_epoch / (t2_ms * 1e-3)
    result = None
    if rank == 0:
        ms_step = t_ms / args.steps
        mufu = rbmnqs.probe_mufu()
        sampler_ms = stage_ms[0] / max(1, stage_cnt[0])
        # algorithmic special-function work of one sweep-kernel launch: every
        # proposal evaluates ln|cosh| of all T theta entries (one exp, one cos,
        # one log each) and the FP64 theta recompute after every sweep
        # re-evaluates the T entries; proposals per sweep = n / (1 + p_bond)
        T = sess.n_hidden * sess.n_symm
        acc = float(np.mean(accs))
        sweeps = wl["warmup"] + wl["samples_per_chain"] * wl["step"]
        props_per_sweep = model.n / (1 + wl["bond_flips"])
        per_chain = sweeps * (props_per_sweep * T * 3 + T * 3)
        mufu_ops = per_chain * wl["n_chains"]
        achieved = mufu_ops / (sampler_ms * 1e-3)
        result = {
            "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 ratios / fp64 theta+CG",
            "data": "synthetic (seeded complex Gaussian weights std 1e-4, Philox chains)",
            "config": dict(workload=args.workload, **describe(wl, P), parallelism=f"replicas x{world}",
                           l2="256 MiB L2 flush between timed epochs (outside the event pairs)"),
            "sr_epochs_per_s": world * args.steps / (t_ms * 1e-3),
            "tau": tau, "energy_per_site": float(np.mean(energies)) / model.n, "acceptance": acc,
            "energy_per_site_stderr": float(np.sqrt(np.mean(np.square(errs))) / np.sqrt(len(errs))) / model.n,
            "learned_acceptance": float(np.mean(laccs)) if laccs else None,
            "cg_iterations": float(np.mean(its)),
            "stage_ms_per_epoch": {nm: stage_ms[i] / max(1, stage_cnt[i]) for i, nm in
                                   enumerate(["sampler", "eval", "moments+stats", "gram+regularise", "cg",
                                              "update"])},
            "roofline": {"bound": "mufu", "kernel": "sampler_kernel", "achieved": achieved / 1e9,
                         "peak": mufu / 1e9, "unit": "Gop/s (MUFU)", "frac": achieved / mufu,
                         "peak_source": "measured in this run by rbmnqs_probe_mufu (no MUFU figure in "
                                        "MEASURED_PEAKS.json)",
                         "algorithmic_ops_per_launch": mufu_ops,
                         "traffic": SAMPLER_DRAM_BYTES.get(args.workload),
                         "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture "
                                           "(profiles/sampler_kernel_kitaev32_symm_a4.md)"},
            "e2e": {"value": e2e, "unit": "samples/s", "h2d_bytes_per_step": P * 16,
                    "d2h_bytes_per_step": P * 16 + 96},
            "gpu_launches": kern_per_epoch * args.steps,
            "clocks": clocks,
        }
    return result


def run_batch(args, rank, world, local):
    """The batched toric workload: all problems' epochs in one graph launch."""
    import torch
    import rbmnqs

    dist = init_dist(world, "nccl")
    torch.cuda.set_device(local)
    wl = workload(args)
    sessions, Ls = [], []
    for L in wl["batch_L"]:
        model = rbmnqs.Model.toric(L, symmetry=wl["symmetry"])
        for c in range(wl["batch_copies"]):
            cfg = rbmnqs.default_config(rbm_type=wl["rbm_type"], alpha=wl["alpha"], n_chains=wl["n_chains"],
                                        samples_per_chain=wl["samples_per_chain"], warmup=wl["warmup"],
                                        step=wl["step"], bond_flips=0.0, seed=1000 * L + c + 77 * rank,
                                        precision=wl["precision"], gram=wl["gram"], reinit_chains=0,
                                        reg2=wl["reg2"], max_iterations=wl["max_iterations"])
            s = rbmnqs.Session(model, cfg)
            s.set_weights(make_weights(s.n_params, wl["std"], 7 * L + c + rank))
            sessions.append(s)
            Ls.append(L)
    tuned = {}  # launch shapes chosen by the autotuner, per L
    for s, L in zip(sessions, Ls):
        shape = s.autotune(sweeps=4)[:2]
        tuned.setdefault(L, shape)
    batch = rbmnqs.Batch(sessions)
    stream = torch.cuda.ExternalStream(batch.stream())
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    for _ in range(max(3, args.warmup)):
        batch.epoch()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    neff = 0.0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if args.profile_region:
        torch.cuda.profiler.start()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            ev[k][0].record(stream)
            st, sr = batch.epoch()
            ev[k][1].record(stream)
            neff += sum(s.N / (1.0 + 2.0 * x["tau"]) for s, x in zip(sessions, st))
        torch.cuda.synchronize()
    if args.profile_region:
        torch.cuda.profiler.stop()
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    # end to end: every session's weights in and out through the C ABI, each step
    ws = [s.get_weights() for s in sessions]
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for k in range(args.steps):
        ev2[k][0].record(stream)
        for s, w in zip(sessions, ws):
            s.set_weights(w)
        batch.epoch()
        ws = [s.get_weights() for s in sessions]
        ev2[k][1].record(stream)
    torch.cuda.synchronize()
    t2_ms = sum(a.elapsed_time(b) for a, b in ev2)
    t_ms, t2_ms = max_over_ranks([t_ms, t2_ms], world)
    its = [x["iterations"] for x in sr]
    Pmax = max(s.n_params for s in sessions)
    hb = sum(s.n_params for s in sessions) * 16
    res = {
        "metric": METRIC, "value": world * neff / (t_ms * 1e-3), "unit": "samples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 ratios / fp64 theta+CG",
        "data": "synthetic (seeded complex Gaussian weights std 1e-4, Philox chains)",
        "config": {"workload": args.workload, "problems": len(sessions),
                   "model": "toric code L x L (2 L^2 spins), L in %s, %d each" % (list(wl["batch_L"]),
                                                                              wl["batch_copies"]),
                   "machine": f"RBM alpha={wl['alpha']}, up to {Pmax} params (matrix-free CG above 2048)",
                   "n_chains_each": wl["n_chains"], "sweeps_per_epoch": wl["warmup"] + 1,
                   "max_cg_iterations": wl["max_iterations"], "launch_shapes": {str(k): v for k, v in tuned.items()},
                   "parallelism": f"replicas x{world}", "l2": "256 MiB L2 flush between timed epochs"},
        "sr_epochs_per_s": world * args.steps / (t_ms * 1e-3), "batch_graph_kernels": batch.graph_kernels(),
        "cg_iterations_mean": float(np.mean(its)),
        "e2e": {"value": world * neff / (t2_ms * 1e-3), "unit": "samples/s", "h2d_bytes_per_step": hb,
                "d2h_bytes_per_step": hb},
        "gpu_launches": batch.graph_kernels() * args.steps, "clocks": clk.summary(),
    }
    if world > 1:
        dist.destroy_process_group()
    return res if rank == 0 else None


# ------------------------------------------------------- forms (C5) --
def forms_config(wl, seed, form):
    """Session config of one form of the 128-spin workload."""
    import rbmnqs
    kw = dict(rbm_type=wl["rbm_type"], alpha=wl["alpha"], n_chains=wl["n_chains"],
              samples_per_chain=wl["samples_per_chain"], warmup=wl["warmup"], step=wl["step"],
              bond_flips=wl["bond_flips"], seed=seed, precision=0, gram=0, reinit_chains=0, reg2=wl["reg2"])
    if form == "learned":
        kw.update(wl["learned"])
    elif form == "plain_fp64":
        kw["precision"] = 1
    return rbmnqs.default_config(**kw)


def train_checkpoint(wl, model, epochs, seed, path):
    """Plain FP32 SR from seeded std-1e-4 weights; saved as a .rbm file."""
    import rbmnqs
    t = wl["train"]
    cfg = rbmnqs.default_config(rbm_type=wl["rbm_type"], alpha=wl["alpha"], n_chains=t["n_chains"],
                                samples_per_chain=1, warmup=t["warmup"], step=1, bond_flips=t["bond_flips"],
                                seed=seed, precision=0, gram=0, reinit_chains=0, reg2=wl["reg2"])
    s = rbmnqs.Session(model, cfg)
    s.set_weights(make_weights(s.n_params, wl["std"], 99))
    t0 = time.perf_counter()
    es = []
    for _ in range(epochs):
        st, _ = s.epoch()
        es.append(st["energy"].real / model.n)
    s.save(path)
    return {"epochs": epochs, "n_chains": t["n_chains"], "sweeps_per_epoch": t["warmup"] + 1,
            "energy_per_site_last50": float(np.mean(es[-50:])), "seconds": time.perf_counter() - t0}


def time_form(sess, graph, steps, warmup, l2_flush, stream, clk=None, profile=False):
    """Warm-up epochs, then `steps` epochs timed with CUDA events on the
    session's stream (L2 flushed between epochs, outside the events);
    `profile` brackets the timed epochs with cudaProfilerStart/Stop."""
    import torch
    tuned = None
    if graph:
        # the solver-stage choices (Gram split count, CG kernel) tuned on
        # the form's own O
        sess.epoch()
        tuned = sess.autotune_sr()
    for _ in range(max(1, warmup)):
        sess.epoch() if graph else (sess.sample(), sess.optimize())
    sess.timing_reset(True)
    if graph:
        sess.epoch()  # re-capture with the stage-timing event nodes; not timed
        sess.timing_reset(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    stats = []
    torch.cuda.synchronize()
    ctx = clk if clk is not None else _Null()
    if profile:
        torch.cuda.profiler.start()
    with ctx:
        for k in range(steps):
            l2_flush()
            ev[k][0].record(stream)
            if graph:
                st, sr = sess.epoch()
            else:
                st = sess.sample()
                sr = sess.optimize()
            ev[k][1].record(stream)
            stats.append((st, sr))
        torch.cuda.synchronize()
    if profile:
        torch.cuda.profiler.stop()
    t_ms = [a.elapsed_time(b) for a, b in ev]
    ms, cnt = sess.timing()
    if tuned is not None:
        stats[0][1]["sr_tuning"] = {"gram_splits": tuned[0], "cg_kernel": ["cluster", "cooperative"][tuned[1]]
                                    if tuned[1] >= 0 else None, "ms": tuned[2]}
    return t_ms, stats, [float(m / max(1, c)) for m, c in zip(ms, cnt)]


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass


def form_summary(N, n, t_ms, stats, stage_ms):
    taus = [st["tau"] for st, _ in stats]
    es = [st["energy"].real / n for st, _ in stats]
    errs = [st["stddev"] / n for st, _ in stats]
    tau = float(np.mean(taus))
    t = float(np.sum(t_ms)) * 1e-3
    neff = len(stats) * N / (1.0 + 2.0 * tau)
    d = {"uncorrelated_samples_per_s": neff / t, "ms_per_epoch": 1e3 * t / len(stats),
         "sr_epochs_per_s": len(stats) / t, "tau": tau, "energy_per_site": float(np.mean(es)),
         "energy_per_site_stderr": float(np.sqrt(np.sum(np.square(errs)))) / len(errs),
         "acceptance": float(np.mean([st["acceptance"] for st, _ in stats])),
         "cg_iterations": float(np.mean([sr["iterations"] for _, sr in stats])),
         "epochs_timed": len(stats),
         "stage_ms_per_epoch": {nm: stage_ms[i] for i, nm in enumerate(
             ["sampler", "eval", "moments+stats", "gram+regularise", "cg", "update"])}}
    if "sr_tuning" in stats[0][1]:
        d["sr_tuning"] = stats[0][1]["sr_tuning"]
    if any(st["learned_acceptance"] for st, _ in stats):
        d["learned_acceptance"] = float(np.mean([st["learned_acceptance"] for st, _ in stats]))
    return d


def run_forms(args, rank, world, local):
    import tempfile

    import torch
    import rbmnqs

    dist = init_dist(world, "nccl")
    torch.cuda.set_device(local)
    wl = workload(args)
    model = rbmnqs.Model.kitaev(wl["n_cells"], symmetry=wl["symmetry"])
    n = model.n
    tmp = tempfile.mkdtemp(prefix="rbmnqs_bench_")
    ckpt = os.path.join(tmp, "kitaev128_trained.rbm")
    train = train_checkpoint(wl, model, args.train_epochs or wl["train"]["epochs"], 77 + rank, ckpt)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def session(form):
        s = rbmnqs.Session(model, forms_config(wl, 1234 + rank, form))
        s.load(ckpt)
        return s

    def flush_on(stream):
        def f():
            with torch.cuda.stream(stream):
                flush.zero_()
        return f

    out = {}
    forms = [f for f in args.forms.split(",") if f]
    if sorted(forms) != sorted(["learned", "plain_fp32", "plain_fp64"]):
        # a subset of the forms (profiling): each timed alone, no metric line
        for form in forms:
            s = session(form)
            st = torch.cuda.ExternalStream(s.stream())
            graph = form != "plain_fp64"
            t_ms, stats, stage = time_form(s, graph, args.steps, args.warmup, flush_on(st), st,
                                           profile=bool(args.profile_region))
            out[form] = form_summary(s.N, n, t_ms, stats, stage)
            out[form]["graph_kernels"] = s.graph_kernels() if graph else None
            del s
        return {"workload": args.workload, "forms_only": out, "checkpoint": train} if rank == 0 else None
    # learned form: the headline number, clocks sampled in its timed region
    learned = session("learned")
    lstream = torch.cuda.ExternalStream(learned.stream())

    if world > 1:
        dist.barrier()
    clk = ClockSampler(local)
    t_ms, stats, stage = time_form(learned, True, args.steps, args.warmup, flush_on(lstream), lstream, clk,
                                   profile=bool(args.profile_region))
    clocks = clk.summary()
    t_learned_ms = float(np.sum(t_ms))
    out["learned"] = form_summary(learned.N, n, t_ms, stats, stage)
    kern_per_epoch = learned.graph_kernels()
    # end to end through the C ABI with host buffers: weights in, epoch,
    # weights and statistics out, every step
    w = learned.get_weights()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    taus2 = []
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush_on(lstream)()
        ev2[k][0].record(lstream)
        learned.set_weights(w)
        st, _ = learned.epoch()
        w = learned.get_weights()
        ev2[k][1].record(lstream)
        taus2.append(st["tau"])
    torch.cuda.synchronize()
    t2_ms = sum(a.elapsed_time(b) for a, b in ev2)
    mufu = rbmnqs.probe_mufu() if rank == 0 else 0.0
    T = learned.n_hidden * learned.n_symm
    P = learned.n_params
    del learned
    # plain forms
    p32 = session("plain_fp32")
    s32 = torch.cuda.ExternalStream(p32.stream())
    t_ms, stats, stage = time_form(p32, True, args.steps, args.warmup, flush_on(s32), s32,
                                   profile=bool(args.profile_region))
    out["plain_fp32"] = form_summary(p32.N, n, t_ms, stats, stage)
    del p32
    p64 = session("plain_fp64")
    s64 = torch.cuda.ExternalStream(p64.stream())
    steps64 = max(2, min(args.steps, 3))
    t_ms, stats, stage = time_form(p64, False, steps64, 1, flush_on(s64), s64)
    out["plain_fp64"] = form_summary(p64.N, n, t_ms, stats, stage)
    del p64

    t_learned_ms, t2_ms = max_over_ranks([t_learned_ms, t2_ms], world)
    if rank != 0:
        return None
    L = out["learned"]
    N = wl["n_chains"] * wl["samples_per_chain"]
    value = world * args.steps * N / (1.0 + 2.0 * L["tau"]) / (t_learned_ms * 1e-3)
    e2e = world * args.steps * N / (1.0 + 2.0 * float(np.mean(taus2))) / (t2_ms * 1e-3)
    # roofline of the dominant kernel (the E_loc / O_k evaluation): every
    # off-diagonal term (the x and y bonds, n / 2 each) evaluates ln cosh of
    # all T theta entries of theta', each one ex2, one sin and one cos (the
    # per-four lg2 and rsqrt not counted)
    terms = n
    ops = float(N) * terms * T * 3.0
    eval_ms = L["stage_ms_per_epoch"]["eval"]
    achieved = ops / (eval_ms * 1e-3)
    sweep_ms = L["stage_ms_per_epoch"]["sampler"]
    dE = L["energy_per_site"] - out["plain_fp32"]["energy_per_site"]
    dE_err = float(np.hypot(L["energy_per_site_stderr"], out["plain_fp32"]["energy_per_site_stderr"]))
    res = {
        "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_learned_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 psi ratios / fp64 theta+CG / fp16x3 split-precision Gram",
        "data": "synthetic (checkpoint trained here from seeded complex Gaussian weights std 1e-4, Philox chains)",
        "config": {"workload": args.workload, "model": f"kitaev honeycomb n_cells={wl['n_cells']} ({n} spins) J=-1",
                   "machine": f"symmetric RBM alpha={wl['alpha']}, {P} params",
                   "n_chains": wl["n_chains"], "samples_per_chain": wl["samples_per_chain"],
                   "sweeps_between_samples": wl["step"], "proposals": "single-spin flips",
                   "learned": "1 learned move per sample (dictionary of 128 sites + 128 x/y bonds, MLP "
                              "128-256-256-256 BF16), 2 Adam steps per epoch",
                   "sr": "CG reg2=1e-4 reg1=(1,1e-4,0.9) lr=1e-2", "checkpoint": train,
                   "parallelism": f"replicas x{world}",
                   "l2": "256 MiB L2 flush between timed epochs (outside the event pairs)"},
        "sr_epochs_per_s": world * args.steps / (t_learned_ms * 1e-3),
        "tau": L["tau"], "energy_per_site": L["energy_per_site"],
        "energy_per_site_stderr": L["energy_per_site_stderr"],
        "forms": out,
        "vs_plain_fp64": value / (world * out["plain_fp64"]["uncorrelated_samples_per_s"]),
        "vs_plain_fp32": value / (world * out["plain_fp32"]["uncorrelated_samples_per_s"]),
        "sr_epochs_vs_plain_fp64": L["sr_epochs_per_s"] / out["plain_fp64"]["sr_epochs_per_s"],
        "delta_energy_per_site_learned_vs_plain_fp32": {"value": dE, "stderr": dE_err},
        "delta_energy_per_site_learned_vs_plain_fp64": {
            "value": L["energy_per_site"] - out["plain_fp64"]["energy_per_site"],
            "stderr": float(np.hypot(L["energy_per_site_stderr"], out["plain_fp64"]["energy_per_site_stderr"]))},
        "roofline": {"bound": "mufu", "kernel": "eloc_kernel", "achieved": achieved / 1e9, "peak": mufu / 1e9,
                     "unit": "Gop/s (MUFU)", "frac": achieved / mufu,
                     "peak_source": "measured in this run by rbmnqs_probe_mufu (no MUFU figure in "
                                    "MEASURED_PEAKS.json)",
                     "algorithmic_ops_per_launch": ops,
                     "ops_per_unit": "3 MUFU (ex2, sin, cos) per theta entry per off-diagonal term per sample: "
                                     f"{N} samples x {terms} terms x {T} entries",
                     "traffic": ELOC_DRAM_BYTES.get(args.workload),
                     "traffic_source": ELOC_TRAFFIC_SOURCE,
                     "sweep_kernel": {"ms_per_epoch": sweep_ms}},
        "e2e": {"value": e2e, "unit": "samples/s", "h2d_bytes_per_step": P * 16,
                "d2h_bytes_per_step": P * 16 + 96},
        "gpu_launches": kern_per_epoch * args.steps,
        "clocks": clocks,
    }
    return res


# ------------------------------------------------------------ CPU arm --
def cpu_epoch(wl, chains, seed, threads):
    """One bounded epoch of the workload on the FP64 CPU restatement:
    `chains` Metropolis chains (same sweeps, same Philox streams) and the
    reference's matrix-free CG on their samples.  Returns (seconds, tau,
    samples)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    om = O.Model.kitaev(wl["n_cells"])
    mach = O.Machine(om, "symmetry" if wl["rbm_type"] == 1 else "basic", wl["alpha"], symm=wl["symmetry"],
                     pfaffian=bool(wl.get("pfaffian")), pf_symm=wl.get("pf_symmetry", 0.5))
    mach.set_params(make_weights(mach.n_params, wl["std"], 99, mach.n_neural, wl.get("pf_std")))
    t0 = time.perf_counter()
    E, Om, acc, _ = O.metropolis(mach, om, chains, wl["samples_per_chain"], warmup=wl["warmup"],
                                 step=wl["step"], bond_flips=wl["bond_flips"], seed=seed, threads=threads,
                                 pf_refresh=wl.get("pf_refresh", 0))
    d, F, diag = O.sr_moments(Om, E)
    O.cg_solve(Om, d, F, np.zeros(mach.n_params), 0.9, wl["reg2"][0], 1e-2, diag, n_neural=mach.n_neural)
    dt = time.perf_counter() - t0
    return dt, O.stats(E)["tau"], len(E)


def cpu_forms_epoch(wl, chains, seed, threads):
    """One bounded epoch of the 128-spin workload on the FP64 CPU
    restatement, the reference's sampler structure: `chains` fresh chains,
    warm-up sweeps, samples_per_chain samples one sweep apart, then the
    matrix-free CG on their samples; seeded weights of std 1e-4 (the
    configuration's initial weights).  Returns (seconds, tau, samples)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    om = O.Model.kitaev(wl["n_cells"])
    mach = O.Machine(om, "symmetry", wl["alpha"], symm=wl["symmetry"])
    mach.set_params(make_weights(mach.n_params, wl["std"], 99))
    t0 = time.perf_counter()
    E, Om, acc, _ = O.metropolis(mach, om, chains, wl["samples_per_chain"], warmup=wl["train"]["warmup"],
                                 step=wl["step"], bond_flips=wl["bond_flips"], seed=seed, threads=threads)
    d, F, diag = O.sr_moments(Om, E)
    O.cg_solve(Om, d, F, np.zeros(mach.n_params), 0.9, wl["reg2"][0], 1e-2, diag)
    dt = time.perf_counter() - t0
    return dt, O.stats(E)["tau"], len(E)


def cpu_arm(wl, steps, warmup, chains=256):
    threads = os.cpu_count() or 1
    times = []
    for k in range(warmup + steps):
        dt, tau, n = cpu_epoch(wl, chains, 1234 + k, threads)
        if k >= warmup:
            times.append(dt)
    # samples scale linearly in chains; the bounded sample runs `chains` of
    # the workload's chains at the same sweeps per epoch
    t = float(np.mean(times))
    per_sample = t / n
    return 1.0 / per_sample, threads, t, n


def main():
    args = parse()
    rank, world, local = dist_env()
    wl = workload(args)
    if args.impl == "reference" and wl.get("forms"):
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        chains = 64
        ts, taus, n = [], [], 0
        for k in range(args.warmup + args.steps):
            dt, tau, n = cpu_forms_epoch(wl, chains, 1234 + k, threads)
            if k >= args.warmup:
                ts.append(dt)
                taus.append(tau)
        t = float(np.mean(ts))
        v = n / (1.0 + 2.0 * float(np.mean(taus))) / t
        line = {"metric": METRIC, "value": v, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "fp64", "data": "synthetic", "impl": "reference",
                "tau": float(np.mean(taus)),
                "config": {"workload": args.workload, "parallelism": "host cores",
                           "sample": f"{chains} of {wl['n_chains']} chains x ({wl['train']['warmup']} warm-up + "
                                     f"{wl['samples_per_chain']}) sweeps, one sample per sweep, + CG on their "
                                     f"samples, per step; weights std 1e-4"},
                "cpu_baseline": {"value": v, "unit": "samples/s", "cores": threads, "kind": "port",
                                 "sample": f"{n} samples of {chains} chains per step"},
                "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if args.impl == "reference":
        if rank != 0:
            return
        v_raw, cores, t, n = cpu_arm(wl, args.steps, args.warmup)
        # one sample per chain after 63 warm-up sweeps: successive samples of
        # a chain are 64 sweeps apart, tau ~ 0 in the binning estimator
        line = {"metric": METRIC, "value": v_raw, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "fp64", "data": "synthetic", "impl": "reference",
                "config": {"workload": args.workload, "parallelism": "host cores"},
                "cpu_baseline": {"value": v_raw, "unit": "samples/s", "cores": cores, "kind": "port",
                                 "sample": f"{n} of {wl['n_chains']} chains x {wl['warmup'] + 1} sweeps + CG "
                                           f"on their samples, per step"},
                "e2e": {"value": v_raw, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if "batch_L" in wl:
        res = run_batch(args, rank, world, local)
        if rank == 0:
            print(json.dumps(res))
        return
    if wl.get("forms"):
        res = run_forms(args, rank, world, local)
        if rank == 0:
            if args.cpu_baseline and world == 1:
                threads = os.cpu_count() or 1
                dt, tau, n = cpu_forms_epoch(wl, 128, 4321, threads)
                res["cpu_baseline"] = {"value": n / (1.0 + 2.0 * tau) / dt, "unit": "samples/s", "cores": threads,
                                       "kind": "port",
                                       "sample": f"128 of {wl['n_chains']} chains x ({wl['train']['warmup']} "
                                                 f"warm-up + {wl['samples_per_chain']}) sweeps + CG on their "
                                                 f"{n} samples ({dt:.1f} s), weights std 1e-4, tau {tau:.3f}"}
            print(json.dumps(res))
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    res = run_ours(args, rank, world, local)
    if rank == 0:
        if args.cpu_baseline and world == 1:
            v_raw, cores, t, n = cpu_arm(wl, 1, 0, chains=2048)
            res["cpu_baseline"] = {"value": v_raw / (1 + 2 * res["tau"]), "unit": "samples/s", "cores": cores,
                                   "kind": "port",
                                   "sample": f"{n} of {wl['n_chains']} chains x {wl['warmup'] + 1} sweeps + "
                                             f"CG on their samples (one epoch, {t:.1f} s), tau of the GPU run"}
        print(json.dumps(res))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
