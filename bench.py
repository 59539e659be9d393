"""Benchmark of the VMC hot path (one SR epoch per step) on B200.

Workload (default, the config the headline metric is quoted on):
  Kitaev honeycomb, n_cells=4 (32 spins), J=-1, h=0; symmetric RBM
  (translations + 180-degree rotation, symmetry 0.5), alpha=4 -> 133
  parameters; weights complex Gaussian std 1e-4 (seeded synthetic);
  4096 Metropolis chains x 64 sweeps per epoch (63 warm-up sweeps + 1
  sampled sweep, one sample per chain -> O is 4096 x 133), bond flips with
  probability 0.5, persistent chains; FP32 psi-ratio math with an FP64
  theta recompute after every sweep; SR with S from the 4096 x 133 O matrix,
  FP64 CG with diagonal shift reg2 = 1e-4, reg1 = (1, 1e-4, 0.9), lr = 1e-2.

One step = one SR epoch: sweeps -> E_loc -> O_k -> moments/stats -> Gram S
-> regularise -> CG -> weight update, launched as one CUDA graph.

Metric: uncorrelated samples/s = N / (1 + 2 tau) per epoch time, tau the
reference's binning estimate of the E_loc autocorrelation; SR epochs/s is
reported beside it.  `--impl reference` times the reference algorithm's CPU
restatement (the FP64 oracle; the reference itself cannot be built here) on
all host cores on a bounded sample of the same workload.

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
# line is quoted on kitaev32_symm_a4; the others measure the Pfaffian path and
# the 128-spin lattice with the same harness.
WORKLOADS = {
    # Kitaev 32 spins, symmetric RBM alpha=4, 4096 chains x 64 sweeps,
    # FP32 sweep / FP64 theta recompute, TF32x3 tensor-core Gram, FP64 CG
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
    # chain, 4 sweeps apart) for tau_int of E_loc: plain single-spin / bond
    # Metropolis against the learned multi-spin proposals at 1 sweep + 1
    # learned move per sample (network trained on the chains' own samples)
    "kitaev128_plain_ts": dict(model="kitaev", n_cells=8, rbm_type=1, alpha=4, symmetry=0.5, n_chains=16384,
                               samples_per_chain=16, warmup=0, step=4, bond_flips=0.5, std=1e-4,
                               reg2=(1e-4, 1e-4, 1.0), precision=0, gram=0),
    "kitaev128_learned_ts": dict(model="kitaev", n_cells=8, rbm_type=1, alpha=4, symmetry=0.5, n_chains=16384,
                                 samples_per_chain=16, warmup=0, step=1, bond_flips=0.5, std=1e-4,
                                 reg2=(1e-4, 1e-4, 1.0), precision=0, gram=0, proposal=1, learned_steps=1,
                                 learned_train=2, learned_lr=1e-3),
    # 48 independent toric-code trainings (L = 3..8, 8 each, basic RBM
    # alpha=2, 1024 chains each) advanced by one CUDA-graph launch per epoch;
    # launch shapes autotuned per L; matrix-free CG capped at 100 iterations
    "toric_batch48": dict(model="toric", batch_L=(3, 4, 5, 6, 7, 8), batch_copies=8, rbm_type=0, alpha=2,
                          symmetry=1.0, n_chains=1024, samples_per_chain=1, warmup=63, step=1, bond_flips=0.0,
                          std=1e-4, reg2=(1e-4, 1e-4, 1.0), precision=0, gram=0, max_iterations=100),
}
METRIC = "uncorrelated samples/s (SR epoch, E_loc binning tau)"
# DRAM bytes per sampler launch from an ncu capture of the same workload: the
# theta tables, flip tables and chains live in shared memory and registers
SAMPLER_DRAM_BYTES = {"kitaev32_symm_a4": 136704.0}
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="kitaev32_symm_a4", choices=list(WORKLOADS))
    ap.add_argument("--cpu-baseline", type=int, default=1, help="time the CPU restatement beside our arm")
    ap.add_argument("--chains", type=int, default=0, help="override the workload's chain count (profiling)")
    ap.add_argument("--sweeps", type=int, default=0, help="override the sweeps per epoch (profiling)")
    return ap.parse_args()


def workload(args):
    wl = dict(WORKLOADS[args.workload])
    if args.chains:
        wl["n_chains"] = args.chains
    if args.sweeps:
        wl["warmup"] = args.sweeps - wl["samples_per_chain"] * wl["step"]
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
         "gram": "TF32x3 tcgen05" if wl["gram"] == 0 and wl["precision"] == 0 else "FP64",
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

    if world > 1:
        t = torch.tensor([t_ms, t2_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms, t2_ms = t.tolist()
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
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            ev[k][0].record(stream)
            st, sr = batch.epoch()
            ev[k][1].record(stream)
            neff += sum(s.N / (1.0 + 2.0 * x["tau"]) for s, x in zip(sessions, st))
        torch.cuda.synchronize()
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
    if world > 1:
        t = torch.tensor([t_ms, t2_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms, t2_ms = t.tolist()
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
