#!/usr/bin/env python
"""Benchmark: forward+reverse atom-steps/s of the reversible-simulation gradient.

Workload (default): 3,000 flexible 3-site waters (9,000 atoms) in a 4.5 nm periodic box,
mixed precision (FP32 pair/bonded arithmetic, FP64 state, reconstruction and gradient
sum), LJ + reaction-field Coulomb, dt = 1 fs, velocity Verlet (gamma = 0), 5,000 steps
forward then 5,000 reverse; loss = squared error of the smoothed O-O RDF (200 bins,
0-1 nm) every 1,000 steps against a target from the same code with sigma x 1.02,
eps x 0.95; gradient w.r.t. the 7 parameters.  One bench "step" = one full gradient
(forward_sim + reverse_sim).  One atom-step = one atom advanced one step forward and
one step back.  Seeded synthetic input (jittered lattice, random orientations,
Maxwell-Boltzmann velocities, equilibrated on the GPU before timing).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the CPU restatement of the reference (the FP64 oracle, OpenMP on
all host cores; the Julia reference cannot run on these machines) on bounded samples of
the same workload.  N > 1 (torchrun): independent replicas, one per GPU, no collective
on the data path (weak scaling); timing is the max over ranks.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "rev-sim_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "fwd+rev atom-steps/s"
UNIT = "atom-steps/s"
# Algorithmic work per interacting pair (r <= 1.0 nm, unordered), counted from the
# reference expressions (add/mul = 1, FMA = 2, sqrt/div/exp = 1): forward 40 (+15 for
# an O-O LJ pair), reverse 170 (force + 3x3 VJP with mass scaling + dF/dtheta).
FLOPS_FWD_IPAIR, FLOPS_FWD_OO_EXTRA, FLOPS_REV_IPAIR = 40, 15, 170
# DRAM traffic per reverse-step launch of the default workload: dram__bytes_read.sum +
# dram__bytes_write.sum of one ncu capture of that kernel on the same 9,000-atom system
# (5.546 MB read, 0 written).
REV_STEP_DRAM_BYTES = 5.546e6
# DRAM traffic per forward-step launch of the gas-in-water engine (2,675 atoms), from one ncu
# capture with cold caches (8.11 MB read, 0.11 MB written).
GAS_FWD_STEP_DRAM_BYTES = 8.22e6
GAS_REV_STEP_DRAM_BYTES = 8.97e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-mol", type=int, default=3000)
    ap.add_argument("--box", type=float, default=4.5)
    ap.add_argument("--n-steps", type=int, default=5000)
    ap.add_argument("--n-steps-loss", type=int, default=1000)
    ap.add_argument("--gamma", type=float, default=0.0)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--form", default="lj")
    ap.add_argument("--loss", default="rdf", choices=["rdf", "enth_vap", "both"],
                    help="water: loss_type of loss_fn (water.jl:757-769)")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64-GPU comparison run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-steps", type=int, default=10)
    ap.add_argument("--equil-ps", type=int, default=3, help="ps of Langevin equilibration")
    ap.add_argument("--n-replicas", type=int, default=64, help="replicas workload: boxes")
    ap.add_argument("--rep-steps", type=int, default=2000, help="replicas workload: steps")
    ap.add_argument("--integrator", default="exact", choices=["exact", "reference"],
                    help="water: the exactly reversible integrator (grid increments) or the "
                         "reference's FP64 step arithmetic")
    ap.add_argument("--pair-mode", default="both_sides", choices=["both_sides", "half_shell"],
                    help="water, mixed precision: each molecule pair evaluated from both sides in "
                         "one fused kernel, or once by its owner with a gather kernel")
    ap.add_argument("--cfg1-replicas", type=int, default=16,
                    help="895-water target configuration: replicas batched in one handle")
    ap.add_argument("--no-target", action="store_true",
                    help="water: skip the 895-water target configuration in the headline line")
    ap.add_argument("--workload", default="water", choices=["water", "diamond", "mlp", "replicas", "equil", "reweight",
                             "diffusion", "cfg1"],
                    help="water: 3,000-molecule box (the headline); diamond: Stillinger-Weber "
                         "carbon, 16 replicas of 8,000 atoms; mlp: 895 waters with the learned "
                         "pair correction, gradient throughput and a training comparison; "
                         "replicas: 64 water boxes of 300-3,000 molecules at 280-320 K in one launch; "
                         "equil: barostatted forward equilibration of the water box; "
                         "reweight: the reweighting gradient estimator on the water box; "
                         "diffusion: O2 in water, the diffusion-coefficient gradient")
    ap.add_argument("--gas-water", type=int, default=885, help="diffusion: waters")
    ap.add_argument("--gas-n", type=int, default=10, help="diffusion: O2 molecules")
    ap.add_argument("--gas-box", type=float, default=3.0)
    ap.add_argument("--gas-steps", type=int, default=50000)
    ap.add_argument("--gas-steps-loss", type=int, default=500)
    ap.add_argument("--gas-trunc", type=int, default=200)
    ap.add_argument("--gas-loss", default="diff_rdf_ev", choices=["diff", "diff_ev", "diff_rdf_ev"])
    ap.add_argument("--gas-precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--updates", type=int, default=150, help="mlp: classical training updates "
                    "per seed (the MLP arm trains for the same wall-clock time)")
    ap.add_argument("--mlp-precision", default="bf16_tc", choices=["bf16_tc", "fp64"],
                    help="mlp: the network arithmetic (split-BF16 tensor cores or FP64 CUDA cores)")
    ap.add_argument("--replicas", type=int, default=16, help="diamond replicas")
    ap.add_argument("--cells", type=int, default=10, help="diamond conventional cells per side")
    ap.add_argument("--sw-steps", type=int, default=2000)
    ap.add_argument("--sw-steps-loss", type=int, default=500)
    ap.add_argument("--sw-plain", action="store_true",
                    help="diamond without the learned radial term (SW alone)")
    ap.add_argument("--profile", action="store_true",
                    help="one untimed gradient and exit (the command profiled under ncu)")
    ap.add_argument("--profile-shape", default="16,24,1/16,24,2",
                    help="water --profile: reverse/forward launch shapes (lanes,mols_per_cta,unroll)")
    return ap.parse_args()


def workload_name(a):
    loss = "" if a.loss == "rdf" else f"_loss-{a.loss}"
    return (f"water_{a.n_mol}mol_{a.box:g}nm_{a.form}_{a.precision}_"
            f"{a.n_steps}fwd+{a.n_steps}rev{loss}")


LOSS_TEXT = {
    "rdf": "O-O smoothed RDF, 200 bins 0-1 nm, squared error vs sigma x1.02 / eps x0.95 target",
    "enth_vap": "enthalpy of vaporisation (loss_enth_vap, water.jl:738-755): "
                "(3.69 - U/n + 2.45 - 46.92)^2 per loss point, direct dl/dtheta included",
    "both": "O-O smoothed RDF (as rdf) plus the enthalpy-of-vaporisation term (as enth_vap)",
}


def integ(e, a):
    """The integrator arithmetic of a timed water engine (revsim_set_integrator) and, for
    mixed precision, its pair evaluation (revsim_set_pair_mode)."""
    e.set_integrator(a.integrator)
    if e.precision == "mixed":
        e.set_pair_mode(a.pair_mode)
    return e


def apply_loss(e, a, target):
    """loss_type: the RDF term, the enthalpy term or both on an engine."""
    from revsim import oo_l2_term
    e.set_loss([oo_l2_term(target)] if a.loss in ("rdf", "both") else [])
    e.set_enth_vap(a.loss in ("enth_vap", "both"))


def oracle_loss(a, target):
    from oracle import orc
    t = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)
    return orc.Loss([t] if a.loss in ("rdf", "both") else [], enth_vap=a.loss in ("enth_vap", "both"))


def config(a, extra=None):
    c = {"workload": workload_name(a), "n_atoms": 3 * a.n_mol, "box_nm": a.box,
         "n_steps": a.n_steps, "n_steps_loss": a.n_steps_loss, "n_steps_trunc": a.n_steps_loss,
         "n_steps_log": 1000, "dt_ps": 0.001, "gamma_per_ps": a.gamma, "pair_form": a.form,
         "precision": a.precision,
         "loss": LOSS_TEXT[a.loss],
         "l2": "flushed (256 MiB write) between timed steps", "integrator": a.integrator,
         "pair_mode": a.pair_mode}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------ system set-up
def prepare(a, device, equil_ps=3):
    """Equilibrated start state and RDF target, both made on the GPU by the engine."""
    from revsim import Engine, constants as C, oo_l2_term, systems
    x = systems.water_coords(a.n_mol, a.box, seed=0)
    v = systems.mb_velocities(a.n_mol, seed=1)
    p = np.array(C.default_params(a.form))
    eq = Engine(a.n_mol, a.box, inter_type=a.form, precision="mixed", device=device)
    eq.set_params(p)
    eq.set_state(x, v)
    for blk in range(equil_ps):   # Langevin dynamics (gamma = 5/ps) from the lattice
        eq.forward(systems.noise_seeds(1000, seed=10 + blk), 5.0, 1000, 1000, 0.001, calc_loss=False)
    x0, v0 = eq.get_state()
    # target: the same code with sigma x 1.02, eps x 0.95
    pt = p.copy()
    pt[0] *= 1.02
    pt[1] *= 0.95
    eq.set_params(pt)
    eq.forward(systems.noise_seeds(1000, seed=20), 5.0, 1000, 1000, 0.001, calc_loss=False)
    eq.set_loss([oo_l2_term(np.zeros(200))])
    target = eq.rdf(0, 0)
    eq.close()
    return x0, v0, p, target


def count_ipairs(x, box, pairs, cutoff=1.0):
    d = x[pairs[:, 1]] - x[pairs[:, 0]]
    d -= box * np.round(d / box)
    r2 = (d * d).sum(1)
    inter = r2 <= cutoff * cutoff
    oo = inter & (pairs[:, 0] % 3 == 0) & (pairs[:, 1] % 3 == 0)
    return int(inter.sum()), int(oo.sum())


# ------------------------------------------------------------------- clocks
class Clocks:
    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.f:
            return None
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [t.strip() for t in line.split(",")]
                if len(parts) == 7:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ CPU baseline
def cpu_sample(a, x0, v0, p, target, n_s):
    """The FP64 oracle on n_s forward + n_s reverse steps of the same system (all host
    threads).  Returns (atom-steps/s, threads, description)."""
    from oracle import orc
    from revsim import systems
    s = orc.make_system(a.n_mol, a.box, a.form)
    loss = oracle_loss(a, target)
    seeds = systems.noise_seeds(n_s, seed=99)
    t0 = time.perf_counter()
    xf, vf, _, sx, sv = orc.forward_sim(s, p, x0, v0, seeds, a.gamma, n_s, n_s, 0.001, loss, False)
    t1 = time.perf_counter()
    orc.reverse_sim(s, p, xf, vf, seeds, a.gamma, n_s, n_s, n_s, 0.001, sx, sv, loss)
    t2 = time.perf_counter()
    orc.loss_and_grads(s, p, loss, xf)
    t3 = time.perf_counter()
    t_loss = t3 - t2
    # steps only, plus the loss amortised at one evaluation per n_steps_loss in each pass
    t_steps = (t1 - t0) + (t2 - t1 - t_loss) + 2 * t_loss * n_s / a.n_steps_loss
    return 3 * a.n_mol * n_s / t_steps, orc.num_threads(), (
        f"{n_s} forward + {n_s} reverse steps of the {3 * a.n_mol}-atom box, FP64 oracle, "
        f"loss cost amortised at one evaluation per {a.n_steps_loss} steps")


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import orc
    from revsim import constants as C, systems
    orc.build()
    # same seeded start as the GPU arm, relaxed on the CPU (the arm is CPU-only)
    x = systems.water_coords(a.n_mol, a.box, seed=0)
    v = systems.mb_velocities(a.n_mol, seed=1)
    p = np.array(C.default_params(a.form))
    s = orc.make_system(a.n_mol, a.box, a.form)
    x, v, _, _, _ = orc.forward_sim(s, p, x, v, systems.noise_seeds(50, seed=10), 5.0, 50, 50,
                                    0.001, None, False)
    t = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    target = orc.rdf(s, t, x)
    vals = []
    for i in range(a.warmup + a.steps):
        val, cores, desc = cpu_sample(a, x, v, p, target, a.cpu_sample_steps)
        if i >= a.warmup:
            vals.append(val)
    value = statistics.mean(vals)
    ms = 1e3 * 3 * a.n_mol * a.n_steps / value
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
           "config": config(a, {"precision": "fp64"}),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                            "sample": desc},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "note": "the reference is Julia (Molly/Enzyme); no Julia toolchain exists on these "
                   "machines, so this arm times the FP64 C restatement of its algorithm"}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------- GPU arm
def run_ours(a):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    import build as _build
    _build.build()
    from revsim import Engine, _lib, oo_l2_term, systems

    x0, v0, p, target = prepare(a, local, a.equil_ps)
    eng = integ(Engine(a.n_mol, a.box, inter_type=a.form, precision=a.precision, device=local), a)
    eng.set_params(p)
    apply_loss(eng, a, target)
    eng.set_state(x0, v0)
    seeds = systems.noise_seeds(a.n_steps, seed=100 + rank)
    if a.profile:
        # the launch shapes the bench's autotuner picks on this box (fixed here: timings
        # under the profiler would steer the tuner), then one gradient between
        # cudaProfilerStart/Stop (ncu --profile-from-start off captures only that gradient)
        (rg, rm, ru), (fg, fm, fu) = [tuple(int(t) for t in q.split(",")) for q in a.profile_shape.split("/")]
        eng.set_launch_shape(rg, rm, ru, which=0)
        eng.set_launch_shape(fg, fm, fu, which=1)
        eng.set_state(x0, v0)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        eng.forward(seeds, a.gamma, a.n_steps, a.n_steps_loss, 0.001)
        eng.reverse(seeds, a.gamma, a.n_steps, a.n_steps_loss, a.n_steps_loss, 0.001)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"profiled_shape": eng.launch_shape(0), "forward_shape": eng.launch_shape(1)}))
        eng.close()
        return
    shape = eng.autotune()
    eng.set_state(x0, v0)
    stream = torch.cuda.ExternalStream(eng.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def gradient():
        lf = eng.forward(seeds, a.gamma, a.n_steps, a.n_steps_loss, 0.001)
        lr, g = eng.reverse(seeds, a.gamma, a.n_steps, a.n_steps_loss, a.n_steps_loss, 0.001)
        return lf, lr, g

    for _ in range(a.warmup):
        gradient()
    n0 = eng.launch_count()
    times = []
    with Clocks(local) as clk:
        for _ in range(a.steps):
            flush.zero_()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            lf, lr, g = gradient()
            e1.record(stream)
            barrier()
            times.append(e0.elapsed_time(e1))
    launches = (eng.launch_count() - n0) // a.steps
    clocks = clk.summary()
    total_ms = sum(times)
    if dist is not None:
        t = torch.tensor([total_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_step = total_ms / a.steps
    n_atoms = 3 * a.n_mol
    value = world * n_atoms * a.n_steps / (ms_step * 1e-3)

    # end to end through the public API from pinned host buffers
    xh = torch.from_numpy(x0.copy()).pin_memory()
    vh = torch.from_numpy(v0.copy()).pin_memory()
    e2e_ms = []
    for _ in range(a.steps):
        flush.zero_()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.set_state(xh.numpy(), vh.numpy())
        gradient()
        e1.record(stream)
        barrier()
        e2e_ms.append(e0.elapsed_time(e1))
    e2e_total = sum(e2e_ms)
    if dist is not None:
        t = torch.tensor([e2e_total], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * n_atoms * a.n_steps / (e2e_total / a.steps * 1e-3)
    h2d = 2 * 3 * n_atoms * 8 + 2 * a.n_steps * 8
    d2h = 8 + 8 + 8 * eng.n_params

    # roofline of the dominant kernel (the fused reverse step), timed per launch
    eng.set_state(x0, v0)
    eng.set_kernel_timing(True)
    eng.forward(seeds, a.gamma, a.n_steps, a.n_steps_loss, 0.001)
    eng.reverse(seeds, a.gamma, a.n_steps, a.n_steps_loss, a.n_steps_loss, 0.001)
    kt_ms, kt_n = eng.kernel_time(0)
    ft_ms, ft_n = eng.kernel_time(1)
    eng.set_kernel_timing(False)
    launch_ms = kt_ms / max(kt_n, 1)
    xs, _ = eng.get_state()
    # the reverse pass ends at the start state, rebuilt over the first snapshot block
    recon = {"mixed" if a.precision == "mixed" else "fp64": recon_error(xs, x0, a.box),
             "steps_reconstructed": 1000, "integrator": a.integrator}
    if a.integrator == "exact" and rank == 0:
        # the same gradient with the reference's step arithmetic, for its reconstruction
        recon["reference_arithmetic"] = {}
        for prec in ("mixed", "fp64"):
            er = Engine(a.n_mol, a.box, inter_type=a.form, precision=prec, device=local)
            er.set_params(p)
            apply_loss(er, a, target)
            er.set_state(x0, v0)
            er.forward(seeds, a.gamma, a.n_steps, a.n_steps_loss, 0.001)
            er.reverse(seeds, a.gamma, a.n_steps, a.n_steps_loss, a.n_steps_loss, 0.001)
            recon["reference_arithmetic"][prec] = recon_error(er.get_state()[0], x0, a.box)
            er.close()
    pairs = eng.neighbor_pairs(0)
    ipairs, oo = count_ipairs(xs, a.box, pairs)
    flops_launch = FLOPS_REV_IPAIR * ipairs
    achieved = flops_launch / (launch_ms * 1e-3) / 1e12
    import ctypes
    peak = ctypes.c_double()
    _lib.load().revsim_probe_fp32_tflops(local, ctypes.byref(peak))
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": achieved / peak.value if peak.value else None,
                "traffic": REV_STEP_DRAM_BYTES,
                "traffic_source": "ncu constant: dram__bytes_read.sum + dram__bytes_write.sum of one "
                                  "capture of this kernel on this system, not measured in this run",
                "kernel": "k_water_step<float, LJ, reverse> (fused reverse step)",
                "launch_ms": launch_ms, "launches_timed": kt_n, "ipairs": ipairs,
                "flops_per_launch": flops_launch,
                "peak_source": "measured FP32 FFMA throughput of this GPU (revsim_probe_fp32_tflops); "
                               "the step kernels are scalar FP32 work, neither HBM- nor tensor-bound",
                "shape": {"reverse": dict(zip(("lanes_per_mol", "mols_per_cta", "unroll"), shape[0])),
                          "forward": dict(zip(("lanes_per_mol", "mols_per_cta", "unroll"), shape[1]))},
                "forward_step_launch_ms": ft_ms / max(ft_n, 1),
                "step_kernels_share_of_gradient": (kt_ms + ft_ms) / ms_step,
                "launch_ms_note": "per-launch times come from a pass with events between the "
                                  "launches, which breaks the launch chaining of the timed "
                                  "gradient, so they include the launch gap the chain hides"}

    extra = {}
    if not a.no_compare and rank == 0:
        # the same gradient in plain FP64 on the GPU: throughput and gradient difference
        e64 = integ(Engine(a.n_mol, a.box, inter_type=a.form, precision="fp64", device=local), a)
        e64.set_params(p)
        apply_loss(e64, a, target)
        e64.set_state(x0, v0)
        e64.autotune()
        e64.set_state(x0, v0)
        e64.forward(seeds, a.gamma, a.n_steps, a.n_steps_loss, 0.001)
        e64.reverse(seeds, a.gamma, a.n_steps, a.n_steps_loss, a.n_steps_loss, 0.001)
        torch.cuda.synchronize()
        s64 = torch.cuda.ExternalStream(e64.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e64.set_state(x0, v0)
        e0.record(s64)
        e64.forward(seeds, a.gamma, a.n_steps, a.n_steps_loss, 0.001)
        _, g64 = e64.reverse(seeds, a.gamma, a.n_steps, a.n_steps_loss, a.n_steps_loss, 0.001)
        e1.record(s64)
        torch.cuda.synchronize()
        ms64 = e0.elapsed_time(e1)
        recon["fp64"] = recon_error(e64.get_state()[0], x0, a.box)
        eng.set_state(x0, v0)
        eng.forward(seeds, a.gamma, a.n_steps, a.n_steps_loss, 0.001)
        _, gm = eng.reverse(seeds, a.gamma, a.n_steps, a.n_steps_loss, a.n_steps_loss, 0.001)
        # short window: the same comparison over the first 100 steps (before chaos
        # amplifies the FP32 rounding of the trajectory)
        short = {}
        for eng_, key in ((eng, "mixed"), (e64, "fp64")):
            eng_.set_state(x0, v0)
            eng_.forward(seeds[:100], a.gamma, 100, 100, 0.001)
            short[key] = eng_.reverse(seeds[:100], a.gamma, 100, 100, 100, 0.001)[1][0]
        e64.close()

        def make(prec):
            e = integ(Engine(a.n_mol, a.box, inter_type=a.form, precision=prec, device=local), a)
            e.set_params(p)
            apply_loss(e, a, target)
            return e
        extra = {"fp64_gpu": {"value": n_atoms * a.n_steps / (ms64 * 1e-3), "ms_per_step": ms64,
                              "speedup_mixed_over_fp64": (ms64 / ms_step)},
                 "grad_rel_err_vs_fp64": {
                     "full_workload": grad_rel_err(gm[0], g64[0], p),
                     "full_workload_note": "one mixed / FP64 pair over 1,000-step untruncated blocks "
                                           "at gamma = 0: the trajectories part ways within a block "
                                           "(chaos), so this is not a precision bound",
                     "first_100_steps": grad_rel_err(short["mixed"], short["fp64"], p),
                     "train_schedule_windows": train_window_errors(make, x0, v0, p),
                     "definition": GRAD_ERR_DEFINITION}}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        val, cores, desc = cpu_sample(a, x0, v0, p, target, a.cpu_sample_steps)
        cpu = {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}
    if rank == 0 and world == 1 and not a.no_target and a.form == "lj" and a.loss == "rdf":
        extra["target_config"] = run_target_cfg1(a, local, with_cpu=not a.no_cpu_baseline)

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None,
               "dtype": "f32+f64" if a.precision == "mixed" else "f64", "data": "synthetic",
               "config": config(a, {"parallelism": f"replicas{world}" if world > 1 else "single"}),
               "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": d2h},
               "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
               "clocks": clocks, "loss": {"forward": float(lf[0]), "reverse": float(lr[0])},
               "recon": recon}
        out.update(extra)
        print(json.dumps(out), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------ accuracy of a result
GRAD_ERR_DEFINITION = ("max over parameters of |g - g_fp64| * |theta| / max(|g_fp64 * theta|, "
                       "0.01 max_k |g_fp64,k * theta_k|)")


def grad_rel_err(gx, gref, p):
    """Classical parameters in units of dL/dlog(theta), floored at 1 % of the largest; the
    MLP's (when present) relative to the largest MLP entry."""
    p = np.asarray(p)
    nc = min(len(p), 9)
    q = p[:nc]
    sc = np.abs(gref[:nc] * q)
    e = float(np.max(np.abs((gx[:nc] - gref[:nc]) * q) / np.maximum(sc, 0.01 * sc.max())))
    if len(p) > nc:
        e = max(e, float(np.abs(gx[nc:] - gref[nc:]).max() / np.abs(gref[nc:]).max()))
    return e


def recon_error(x_rec, x0, box):
    """How well a reverse pass rebuilt the start state: minimum-image RMSD and largest
    component error over the atoms, nm.  ``box``: a side or one side per atom."""
    b = np.asarray(box, dtype=np.float64)
    b = b if b.ndim == 0 else b[:, None]
    d = np.asarray(x_rec) - np.asarray(x0)
    d -= b * np.round(d / b)
    return {"rmsd_nm": float(np.sqrt((d * d).sum(1).mean())), "max_nm": float(np.abs(d).max())}


def train_window_errors(make, x0, v0, p, gamma=1.0, n_windows=5, n_loss=2000, n_trunc=200, seed=500):
    """Mixed-precision gradient error under train()'s schedule (water.jl:1624-1631, 1666-1669:
    gamma = 1/ps, a loss point every 2,000 steps, each reverse window truncated at 200 steps).
    That gradient is a sum over loss points of 200-step window gradients; the forward run only
    samples the windows' start states, and any two runs of it (FP32 or FP64 rounding alike)
    part ways within a few ps.  So a mixed-precision sampler runs the schedule, and at each of
    n_windows loss points the window gradient is computed from the same start state in mixed
    precision and in FP64; returns the per-window errors and the windows' reconstruction."""
    from revsim import systems
    sampler, em, e64 = make("mixed"), make("mixed"), make("fp64")
    sampler.set_state(x0, v0)
    seeds = systems.noise_seeds(n_windows * n_loss, seed=seed)
    errs, recon = [], {"mixed": 0.0, "fp64": 0.0}
    for w in range(n_windows):
        s0 = w * n_loss
        sampler.forward(seeds[s0:s0 + n_loss - n_trunc], gamma, n_loss - n_trunc, n_loss, 0.001,
                        calc_loss=False)
        xs, vs = sampler.get_state()
        sw = seeds[s0 + n_loss - n_trunc:s0 + n_loss]
        gw = {}
        for key, e in (("mixed", em), ("fp64", e64)):
            e.set_state(xs, vs)
            e.forward(sw, gamma, n_trunc, n_trunc, 0.001, calc_loss=False)
            gw[key] = e.reverse(sw, gamma, n_trunc, n_trunc, n_trunc, 0.001)[1][0]
            xr, _ = e.get_state()
            recon[key] = max(recon[key], recon_error(xr, xs, e.box[0] if e.R == 1 else
                                                     np.repeat(e.box, 3 * e.n_mol))["max_nm"])
        errs.append(grad_rel_err(gw["mixed"], gw["fp64"], p))
        sampler.forward(sw, gamma, n_trunc, n_trunc, 0.001, calc_loss=False)
    for e in (sampler, em, e64):
        e.close()
    return {"schedule": f"gamma {gamma:g}/ps, loss every {n_loss} steps, reverse truncated at "
                        f"{n_trunc} steps (train(), water.jl:1624-1631)",
            "windows": n_windows, "max": float(max(errs)), "mean": float(np.mean(errs)),
            "per_window": [float(t) for t in errs],
            "window_recon_max_nm": {k: float(v) for k, v in recon.items()},
            "method": "each window's gradient from the same start state (a mixed-precision run's "
                      "state 200 steps before the loss point) in mixed precision and in FP64"}


def seed_ensemble(make, x0, n_mol, p, n_seeds=8, n_steps=1000, gamma=0.0):
    """Untruncated n_steps-step gradients from n_seeds start states (the same positions,
    Maxwell-Boltzmann velocities from n_seeds seeds) in both precisions.  One mixed / FP64
    pair from one state is a chaotic pair (the trajectories part ways within the block); the
    ensemble means are compared against their standard error instead."""
    from revsim import systems
    em, e64 = make("mixed"), make("fp64")
    G = {"mixed": [], "fp64": []}
    for k in range(n_seeds):
        v = systems.mb_velocities(n_mol, seed=1000 + k)
        seeds = systems.noise_seeds(n_steps, seed=2000 + k)
        for key, e in (("mixed", em), ("fp64", e64)):
            e.set_state(x0, v)
            e.forward(seeds, gamma, n_steps, n_steps, 0.001)
            G[key].append(e.reverse(seeds, gamma, n_steps, n_steps, n_steps, 0.001)[1][0])
    em.close()
    e64.close()
    gm, g64 = np.array(G["mixed"]), np.array(G["fp64"])
    diff = gm.mean(0) - g64.mean(0)
    se = np.sqrt(gm.var(0, ddof=1) / n_seeds + g64.var(0, ddof=1) / n_seeds)
    z = diff / np.where(se > 0, se, np.inf)
    paired = [grad_rel_err(gm[k], g64[k], p) for k in range(n_seeds)]
    return {"n_seeds": n_seeds, "n_steps": n_steps, "gamma_per_ps": gamma,
            "max_abs_z_of_mean_difference": float(np.max(np.abs(z))),
            "z_per_parameter": [float(t) for t in z],
            "rel_err_of_means": grad_rel_err(gm.mean(0), g64.mean(0), p),
            "rel_err_of_one_seed_pairs": {"median": float(np.median(paired)), "max": float(max(paired))},
            "reading": "|z| below ~3 for every parameter: the mixed and FP64 ensemble means agree "
                       "within their standard error"}


def time_gradients(eng, x0, v0, seeds, gamma, n_steps, n_steps_loss, reps, flush=None):
    """Device time (ms) of `reps` gradients (forward + reverse from x0, v0), each bracketed by
    CUDA events on the engine's stream, the L2 flushed in between; returns (mean ms, last
    gradient, launches per gradient)."""
    import torch
    st = torch.cuda.ExternalStream(eng.stream())
    ms, g, n0 = [], None, eng.launch_count()
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        eng.set_state(x0, v0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        eng.forward(seeds, gamma, n_steps, n_steps_loss, 0.001)
        _, g = eng.reverse(seeds, gamma, n_steps, n_steps_loss, n_steps_loss, 0.001)
        e1.record(st)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(np.mean(ms)), g, (eng.launch_count() - n0) // max(reps, 1)


# ------------------------------------------------------- the 895-water target configuration
TIP3P_FIXTURE = os.path.join(ROOT, "tests", "golden", "reference_inputs.npz")


def cfg1_start(R, device):
    """R replicas of the reference's own input box (water/tip3p.pdb: 895 waters, 3.0 nm, read
    from the committed fixture), Maxwell-Boltzmann velocities at 295.15 K from seeds 0..R-1,
    1 ps of Langevin equilibration (gamma = 5/ps) on the GPU; the target is the replica-mean
    O-O RDF of a 0.5 ps run of the same code with sigma x 1.02, eps x 0.95.  Returns
    (x [R * 2685, 3], v, params, target)."""
    from revsim import Engine, constants as C, oo_l2_term, systems
    d = np.load(TIP3P_FIXTURE)
    x1, box = d["x_tip3p"], float(d["box_tip3p"])
    x = np.concatenate([x1] * R)
    v = np.concatenate([systems.mb_velocities(895, seed=r) for r in range(R)])
    p = np.array(C.default_params("lj"))
    eq = Engine([895] * R, [box] * R, precision="mixed", device=device)
    eq.set_params(p)
    eq.set_state(x, v)
    eq.forward(systems.noise_seeds(1000 * R, seed=40).reshape(1000, R), 5.0, 1000, 1000, 0.001,
               calc_loss=False)
    x0, v0 = eq.get_state()
    pt = p.copy()
    pt[0] *= 1.02
    pt[1] *= 0.95
    eq.set_params(pt)
    eq.forward(systems.noise_seeds(500 * R, seed=41).reshape(500, R), 5.0, 500, 500, 0.001,
               calc_loss=False)
    eq.set_loss([oo_l2_term(np.zeros(200))])
    target = np.mean([eq.rdf(0, r) for r in range(R)], axis=0)
    eq.close()
    return x0, v0, p, target, box


def cfg1_cpu_sample(x0, v0, p, target, box, n_s=10):
    """The FP64 oracle on n_s forward + n_s reverse steps of one 895-water box (all host
    threads), the loss amortised at one evaluation per 1,000 steps."""
    from oracle import orc
    from revsim import systems
    s = orc.make_system(895, box)
    t = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)
    loss = orc.Loss([t])
    seeds = systems.noise_seeds(n_s, seed=99)
    t0 = time.perf_counter()
    xf, vf, _, sx, sv = orc.forward_sim(s, p, x0, v0, seeds, 0.0, n_s, n_s, 0.001, loss, False)
    t1 = time.perf_counter()
    orc.reverse_sim(s, p, xf, vf, seeds, 0.0, n_s, n_s, n_s, 0.001, sx, sv, loss)
    t2 = time.perf_counter()
    orc.loss_and_grads(s, p, loss, xf)
    t3 = time.perf_counter()
    t_loss = t3 - t2
    t_steps = (t1 - t0) + (t2 - t1 - t_loss) + 2 * t_loss * n_s / 1000
    return 2685 * n_s / t_steps, orc.num_threads(), (
        f"{n_s} forward + {n_s} reverse steps of one 895-water box, FP64 oracle, loss amortised "
        f"at one evaluation per 1,000 steps")


def run_target_cfg1(a, device, reps=3, with_cpu=True):
    """The target configuration of the engine: the 895-water box, 1,000 steps forward
    + 1,000 reverse (velocity Verlet, gamma = 0), loss = O-O RDF L2 (200 bins, 0-1 nm) against
    the sigma x 1.02 / eps x 0.95 target; R replicas of it batched in one handle (one launch
    per step), mixed precision against the same engine in FP64 and against the FP64 oracle on
    the host cores, with the gradient's accuracy (train()'s window schedule, a seed ensemble)
    and the reconstruction of the start state in both precisions."""
    import torch
    from revsim import Engine, oo_l2_term, systems
    R = a.cfg1_replicas
    n, nl = 1000, 1000
    x0, v0, p, target, box = cfg1_start(R, device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")
    seeds = systems.noise_seeds(n * R, seed=42).reshape(n, R)
    n_atoms = 2685 * R
    out = {"workload": f"water_895mol_3nm_tip3p_x{R}replicas_lj_1000fwd+1000rev",
           "start": "water/tip3p.pdb positions (committed fixture), MB velocities at 295.15 K, 1 ps "
                    "Langevin equilibration on the GPU", "replicas": R, "n_atoms": n_atoms,
           "n_steps": n, "gamma_per_ps": 0.0, "dt_ps": 0.001, "integrator": a.integrator}
    res = {}
    for prec in ("mixed", "fp64"):
        e = integ(Engine([895] * R, [box] * R, precision=prec, device=device), a)
        e.set_params(p)
        e.set_loss([oo_l2_term(target)])
        e.set_state(x0, v0)
        shape = e.autotune()
        time_gradients(e, x0, v0, seeds, 0.0, n, nl, 2, flush)          # warm-up
        ms, g, launches = time_gradients(e, x0, v0, seeds, 0.0, n, nl, reps, flush)
        xr, _ = e.get_state()
        e.set_graph_mode(True)
        time_gradients(e, x0, v0, seeds, 0.0, n, nl, 2, flush)
        msg, _, _ = time_gradients(e, x0, v0, seeds, 0.0, n, nl, reps, flush)
        e.set_graph_mode(False)
        res[prec] = {"value": n_atoms * n / (ms * 1e-3), "ms_per_gradient": ms, "gpu_launches": launches,
                     "cuda_graph": {"value": n_atoms * n / (msg * 1e-3), "ms_per_gradient": msg},
                     "shape": {"reverse": list(shape[0]), "forward": list(shape[1])},
                     "recon_1000_steps": recon_error(xr, x0, box), "grad": g}
        # one replica alone (the unbatched form) for the same comparison
        e.close()
        e1 = integ(Engine(895, box, precision=prec, device=device), a)
        e1.set_params(p)
        e1.set_loss([oo_l2_term(target)])
        e1.set_state(x0[:2685], v0[:2685])
        e1.autotune()
        time_gradients(e1, x0[:2685], v0[:2685], seeds[:, 0], 0.0, n, nl, 2, flush)
        ms1, _, _ = time_gradients(e1, x0[:2685], v0[:2685], seeds[:, 0], 0.0, n, nl, reps, flush)
        res[prec]["single_replica"] = {"value": 2685 * n / (ms1 * 1e-3), "ms_per_gradient": ms1}
        # the same passes captured in CUDA graphs (revsim_set_graph_mode), against chained launches
        e1.set_graph_mode(True)
        time_gradients(e1, x0[:2685], v0[:2685], seeds[:, 0], 0.0, n, nl, 2, flush)
        msg, _, _ = time_gradients(e1, x0[:2685], v0[:2685], seeds[:, 0], 0.0, n, nl, reps, flush)
        res[prec]["single_replica"]["cuda_graph"] = {"value": 2685 * n / (msg * 1e-3), "ms_per_gradient": msg,
                                                     "captures_replays": list(e1.graph_stats())}
        e1.close()
    gm, g64 = res["mixed"].pop("grad"), res["fp64"].pop("grad")
    out["mixed"], out["fp64"] = res["mixed"], res["fp64"]
    out["speedup_mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
    out["speedup_mixed_over_fp64_single_replica"] = (res["mixed"]["single_replica"]["value"] /
                                                     res["fp64"]["single_replica"]["value"])

    def make(prec):
        e = integ(Engine(895, box, precision=prec, device=device), a)
        e.set_params(p)
        e.set_loss([oo_l2_term(target)])
        return e
    # the same comparison over the first 100 steps of each box (before the dynamics amplify
    # the FP32 rounding of the trajectory), gamma = 0, one untruncated block
    short = {}
    for prec in ("mixed", "fp64"):
        e = make(prec)
        e.set_state(x0[:2685], v0[:2685])
        s100 = systems.noise_seeds(100, seed=45)
        e.forward(s100, 0.0, 100, 100, 0.001)
        short[prec] = e.reverse(s100, 0.0, 100, 100, 100, 0.001)[1][0]
        e.close()
    out["grad_rel_err_vs_fp64"] = {
        "first_100_steps": grad_rel_err(short["mixed"], short["fp64"], p),
        "same_start_1000_steps": float(np.median([grad_rel_err(gm[r], g64[r], p) for r in range(R)])),
        "same_start_note": "median over the replicas of one mixed / FP64 pair each: a chaotic pair "
                           "over 1,000 untruncated steps, not a precision bound",
        "train_schedule_windows": train_window_errors(make, x0[:2685], v0[:2685], p),
        "seed_ensemble": seed_ensemble(make, x0[:2685], 895, p),
        "definition": GRAD_ERR_DEFINITION}
    if with_cpu:
        val, cores, desc = cfg1_cpu_sample(x0[:2685], v0[:2685], p, target, box)
        out["cpu_baseline"] = {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}
        out["speedup_mixed_over_cpu"] = res["mixed"]["value"] / val
    return out


def run_ours_cfg1(a):
    """--workload cfg1: the target configuration as its own bench line."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    import build as _build
    _build.build()
    if a.profile:
        # one batched gradient between cudaProfilerStart/Stop at the launch shapes the
        # autotuner picks for it (8 lanes x 16 molecules per CTA for both step kernels)
        from revsim import Engine, oo_l2_term, systems
        R = a.cfg1_replicas
        x0, v0, p, target, box = cfg1_start(R, local)
        e = integ(Engine([895] * R, [box] * R, precision="mixed", device=local), a)
        e.set_params(p)
        e.set_loss([oo_l2_term(target)])
        e.set_launch_shape(8, 16, 1, which=-1)
        e.set_state(x0, v0)
        seeds = systems.noise_seeds(1000 * R, seed=42).reshape(1000, R)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        e.forward(seeds, 0.0, 1000, 1000, 0.001)
        e.reverse(seeds, 0.0, 1000, 1000, 1000, 0.001)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"profiled_shape": e.launch_shape(0), "forward_shape": e.launch_shape(1)}))
        e.close()
        return
    with Clocks(local) as clk:
        t = run_target_cfg1(a, local, reps=max(a.steps, 1))
    if rank != 0:
        return
    m = t["mixed"]
    out = {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": 1, "steps": a.steps,
           "warmup": 2, "ms_per_step": m["ms_per_gradient"], "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
           "config": {"workload": t["workload"], "replicas": t["replicas"], "n_atoms": t["n_atoms"],
                      "l2": "flushed (256 MiB write) between timed gradients",
                      "start": t["start"]},
           "e2e": {"value": m["value"], "unit": UNIT,
                   "h2d_bytes_per_step": 2 * 3 * t["n_atoms"] * 8 + 2 * 1000 * t["replicas"] * 8,
                   "d2h_bytes_per_step": 2 * t["replicas"] * 8 + t["replicas"] * 7 * 8},
           "gpu_launches": m["gpu_launches"], "cpu_baseline": t.get("cpu_baseline"),
           "clocks": clk.summary(), "target": t,
           "e2e_note": "every timed gradient starts from host arrays (set_state), so value is end to end"}
    print(json.dumps(out), flush=True)


# --------------------------------------------------------- equilibration workload
EQUIL_METRIC = "forward atom-steps/s (barostatted Langevin equilibration)"


def equil_config(a, extra=None):
    c = {"workload": f"water_{a.n_mol}mol_{a.box:g}nm_{a.form}_{a.precision}_equil_npt_{a.n_steps}fwd",
         "n_atoms": 3 * a.n_mol, "box_nm": a.box, "n_steps": a.n_steps, "dt_ps": 0.001,
         "gamma_per_ps": 1.0, "pair_form": a.form, "precision": a.precision,
         "barostat": "Monte-Carlo, 1 bar, a volume move every 30 steps (water.jl:789-865, "
                     "use_barostat of the train() equilibration, water.jl:1642-1645)",
         "l2": "flushed (256 MiB write) between timed steps"}
    if extra:
        c.update(extra)
    return c


def equil_cpu_sample(a, x0, v0, p, n_s=60):
    """The FP64 oracle's barostatted forward run on n_s steps (two volume moves)."""
    from oracle import orc
    from revsim import systems
    s = orc.make_system(a.n_mol, a.box, a.form)
    b = orc.make_barostat(a.box, seed=5)
    seeds = systems.noise_seeds(n_s, seed=97)
    t0 = time.perf_counter()
    orc.forward_sim_barostat(s, p, x0, v0, seeds, 1.0, n_s, 0.001, b)
    dt = time.perf_counter() - t0
    return 3 * a.n_mol * n_s / dt, orc.num_threads(), (
        f"{n_s} barostatted forward steps ({n_s // 30} volume moves) of the {3 * a.n_mol}-atom box, "
        f"FP64 oracle")


def run_reference_equil(a):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import orc
    from revsim import constants as C, systems
    orc.build()
    x = systems.water_coords(a.n_mol, a.box, seed=0)
    v = systems.mb_velocities(a.n_mol, seed=1)
    p = np.array(C.default_params(a.form))
    s = orc.make_system(a.n_mol, a.box, a.form)
    x, v, _, _, _ = orc.forward_sim(s, p, x, v, systems.noise_seeds(50, seed=10), 5.0, 50, 50,
                                    0.001, None, False)
    vals = []
    for i in range(a.warmup + a.steps):
        val, cores, desc = equil_cpu_sample(a, x, v, p)
        if i >= a.warmup:
            vals.append(val)
    value = statistics.mean(vals)
    out = {"metric": EQUIL_METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": 1e3 * 3 * a.n_mol * a.n_steps / value,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "impl": "reference", "config": equil_config(a, {"precision": "fp64"}),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_ours_equil(a):
    """Throughput of the barostatted equilibration (forward steps with a Monte-Carlo volume
    move every 30 steps) of the water box, on one GPU per rank (independent replicas)."""
    import ctypes
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import build as _build
    _build.build()
    from revsim import Engine, _lib, systems
    x0, v0, p, _ = prepare(a, local, a.equil_ps)
    eng = Engine(a.n_mol, a.box, inter_type=a.form, precision=a.precision, device=local)
    eng.set_params(p)
    eng.set_state(x0, v0)
    eng.autotune()
    seeds = systems.noise_seeds(a.n_steps, seed=500 + rank)
    stream = torch.cuda.ExternalStream(eng.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def run(xs=x0, vs=v0):
        eng.set_box(a.box)
        eng.set_state(xs, vs)
        eng.set_barostat(True, seed=7 + rank)
        eng.forward(seeds, 1.0, a.n_steps, a.n_steps, 0.001, calc_loss=False)
        eng.set_barostat(False)

    for _ in range(a.warmup):
        run()
    n0 = eng.launch_count()
    times = []
    with Clocks(local) as clk:
        for _ in range(a.steps):
            flush.zero_()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run()
            e1.record(stream)
            barrier()
            times.append(e0.elapsed_time(e1))
    launches = (eng.launch_count() - n0) // a.steps
    box, vs, na, nacc = eng.barostat_state()
    total = sum(times)
    if dist is not None:
        t = torch.tensor([total], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    ms = total / a.steps
    n_atoms = 3 * a.n_mol
    value = world * n_atoms * a.n_steps / (ms * 1e-3)
    # end to end: the state from pinned host buffers, the final state and box read back
    xh = torch.from_numpy(x0.copy()).pin_memory()
    vh = torch.from_numpy(v0.copy()).pin_memory()
    e2e = []
    for _ in range(a.steps):
        flush.zero_()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run(xh.numpy(), vh.numpy())
        eng.get_state()
        eng.barostat_state()
        e1.record(stream)
        barrier()
        e2e.append(e0.elapsed_time(e1))
    e2e_value = world * n_atoms * a.n_steps / (sum(e2e) / a.steps * 1e-3)
    # roofline of the dominant kernel (the fused forward step)
    eng.set_kernel_timing(True)
    run()
    ft_ms, ft_n = eng.kernel_time(1)
    eng.set_kernel_timing(False)
    launch_ms = ft_ms / max(ft_n, 1)
    xs, _ = eng.get_state()
    box_now = eng.barostat_state()[0][0]
    ipairs, oo = count_ipairs(xs, box_now, eng.neighbor_pairs(0))
    flops_launch = FLOPS_FWD_IPAIR * ipairs + FLOPS_FWD_OO_EXTRA * oo
    peak = ctypes.c_double()
    _lib.load().revsim_probe_fp32_tflops(local, ctypes.byref(peak))
    achieved = flops_launch / (launch_ms * 1e-3) / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": achieved / peak.value if peak.value else None, "traffic": None,
                "kernel": "k_water_step<float, LJ, forward> (fused forward step)",
                "launch_ms": launch_ms, "launches_timed": ft_n, "ipairs": ipairs,
                "flops_per_launch": flops_launch,
                "peak_source": "measured FP32 FFMA throughput of this GPU (revsim_probe_fp32_tflops)",
                "step_kernel_share": ft_ms / ms}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        val, cores, desc = equil_cpu_sample(a, x0, v0, p)
        cpu = {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}
    if rank == 0:
        out = {"metric": EQUIL_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32+f64" if a.precision == "mixed" else "f64",
               "data": "synthetic", "config": equil_config(a),
               "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * 3 * n_atoms * 8 + a.n_steps * 8,
                       "d2h_bytes_per_step": 2 * 3 * n_atoms * 8 + 32},
               "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(),
               "barostat": {"final_box_nm": float(box[0]), "volume_moves": int(na[0]),
                            "accepted": int(nacc[0]), "volume_scale_nm3": float(vs[0])}}
        print(json.dumps(out), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------------- reweighting workload
REWEIGHT_METRIC = "forward atom-steps/s (reweighting gradient estimator)"


def reweight_config(a, extra=None):
    c = {"workload": f"water_{a.n_mol}mol_{a.box:g}nm_{a.form}_{a.precision}_reweight_{a.n_steps}fwd",
         "n_atoms": 3 * a.n_mol, "box_nm": a.box, "n_steps": a.n_steps, "n_steps_loss": a.n_steps_loss,
         "dt_ps": 0.001, "gamma_per_ps": 1.0, "pair_form": a.form, "precision": a.precision,
         "estimator": "reweighting_sim (water.jl:1107-1210): at every loss point the loss, its "
                      "direct gradient and dE/dtheta (FP64 energy kernel); "
                      "<dl/dtheta> - beta (<L dE/dtheta> - <L><dE/dtheta>) on the host",
         "loss": LOSS_TEXT[a.loss], "l2": "flushed (256 MiB write) between timed steps"}
    if extra:
        c.update(extra)
    return c


def reweight_cpu_sample(a, x0, v0, p, target, n_s=20):
    """The FP64 oracle: n_s forward steps, then the loss, its gradient and dE/dtheta once."""
    from oracle import orc
    from revsim import systems
    s = orc.make_system(a.n_mol, a.box, a.form)
    loss = oracle_loss(a, target)
    seeds = systems.noise_seeds(n_s, seed=96)
    t0 = time.perf_counter()
    xf, _, _, _, _ = orc.forward_sim(s, p, x0, v0, seeds, 1.0, n_s, n_s, 0.001, loss, False)
    t1 = time.perf_counter()
    orc.loss_and_grads(s, p, loss, xf)
    orc.energy_grads(s, p, xf, orc.neighbor_pairs(s, xf))
    t2 = time.perf_counter()
    per_step = (t1 - t0) / n_s + (t2 - t1) / a.n_steps_loss
    return 3 * a.n_mol / per_step, orc.num_threads(), (
        f"{n_s} forward steps of the {3 * a.n_mol}-atom box plus one loss point (loss, gradient, "
        f"dE/dtheta) amortised over {a.n_steps_loss} steps, FP64 oracle")


def run_reference_reweight(a):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import orc
    from revsim import constants as C, systems
    orc.build()
    x = systems.water_coords(a.n_mol, a.box, seed=0)
    v = systems.mb_velocities(a.n_mol, seed=1)
    p = np.array(C.default_params(a.form))
    s = orc.make_system(a.n_mol, a.box, a.form)
    x, v, _, _, _ = orc.forward_sim(s, p, x, v, systems.noise_seeds(50, seed=10), 5.0, 50, 50,
                                    0.001, None, False)
    target = np.zeros(200)
    vals = []
    for i in range(a.warmup + a.steps):
        val, cores, desc = reweight_cpu_sample(a, x, v, p, target)
        if i >= a.warmup:
            vals.append(val)
    value = statistics.mean(vals)
    out = {"metric": REWEIGHT_METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": 1e3 * 3 * a.n_mol * a.n_steps / value,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "impl": "reference", "config": reweight_config(a, {"precision": "fp64"}),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_ours_reweight(a):
    import ctypes
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import build as _build
    _build.build()
    from revsim import Engine, _lib, systems
    from revsim.water import reweighting_sim
    x0, v0, p, target = prepare(a, local, a.equil_ps)
    eng = Engine(a.n_mol, a.box, inter_type=a.form, precision=a.precision, device=local)
    eng.set_params(p)
    eng.set_state(x0, v0)
    eng.autotune()
    seeds = systems.noise_seeds(a.n_steps, seed=600 + rank)
    from revsim import oo_l2_term
    terms = [oo_l2_term(target)] if a.loss in ("rdf", "both") else []
    stream = torch.cuda.ExternalStream(eng.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def run(xs=x0, vs=v0):
        return reweighting_sim(xs, vs, None, seeds, 1.0, a.n_steps, a.n_steps_loss, p, 0.001, 1,
                               a.form, a.loss, loss_terms=terms, engine=eng)

    for _ in range(a.warmup):
        run()
    n0 = eng.launch_count()
    times = []
    with Clocks(local) as clk:
        for _ in range(a.steps):
            flush.zero_()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = run()
            e1.record(stream)
            barrier()
            times.append(e0.elapsed_time(e1))
    launches = (eng.launch_count() - n0) // a.steps
    total = sum(times)
    if dist is not None:
        t = torch.tensor([total], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    ms = total / a.steps
    n_atoms = 3 * a.n_mol
    value = world * n_atoms * a.n_steps / (ms * 1e-3)
    eng.set_kernel_timing(True)
    run()
    ft_ms, ft_n = eng.kernel_time(1)
    eng.set_kernel_timing(False)
    launch_ms = ft_ms / max(ft_n, 1)
    xs, _ = eng.get_state()
    ipairs, oo = count_ipairs(xs, a.box, eng.neighbor_pairs(0))
    flops_launch = FLOPS_FWD_IPAIR * ipairs + FLOPS_FWD_OO_EXTRA * oo
    peak = ctypes.c_double()
    _lib.load().revsim_probe_fp32_tflops(local, ctypes.byref(peak))
    achieved = flops_launch / (launch_ms * 1e-3) / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": achieved / peak.value if peak.value else None, "traffic": None,
                "kernel": "k_water_step<float, LJ, forward> (fused forward step)",
                "launch_ms": launch_ms, "ipairs": ipairs, "flops_per_launch": flops_launch,
                "peak_source": "measured FP32 FFMA throughput of this GPU (revsim_probe_fp32_tflops)",
                "step_kernel_share": ft_ms / ms}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        val, cores, desc = reweight_cpu_sample(a, x0, v0, p, target)
        cpu = {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}
    if rank == 0:
        _, loss, grads, l_rdf, l_ev = out
        res = {"metric": REWEIGHT_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32+f64" if a.precision == "mixed" else "f64",
               "data": "synthetic", "config": reweight_config(a),
               "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 2 * 3 * n_atoms * 8 + a.n_steps * 8,
                       "d2h_bytes_per_step": 2 * 3 * n_atoms * 8 + 8 * (3 + 2 * len(p)) * (a.n_steps // a.n_steps_loss)},
               "e2e_note": "every timed run starts from host arrays (reweighting_sim sets the state)",
               "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(),
               "loss": float(loss), "l_rdf": float(l_rdf), "l_ev": float(l_ev),
               "gradient": [float(g) for g in grads]}
        print(json.dumps(res), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------ diffusion workload
DIFF_METRIC = "gas-in-water gradient atom-steps/s (forward steps of forward + truncated reverse)"


def diffusion_config(a, extra=None):
    c = {"workload": (f"gas_{a.gas_water}w+{a.gas_n}O2_{a.gas_box:g}nm_{a.form}_{a.gas_precision}_"
                      f"{a.gas_steps}fwd_loss{a.gas_steps_loss}_trunc{a.gas_trunc}_{a.gas_loss}"),
         "n_atoms": 3 * a.gas_water + 2 * a.gas_n, "n_water": a.gas_water, "n_gas": a.gas_n,
         "box_nm": a.gas_box, "n_steps": a.gas_steps, "n_steps_loss": a.gas_steps_loss,
         "n_steps_trunc": a.gas_trunc,
         "reverse_steps": (a.gas_steps // a.gas_steps_loss) * min(a.gas_trunc, a.gas_steps_loss),
         "dt_ps": 0.001, "gamma_per_ps": 1.0, "pair_form": a.form, "precision": a.gas_precision,
         "loss": {"diff": "diffusion coefficient of the O2 centres (calculate_D, diffusion.jl:861-911)",
                  "diff_ev": "diffusion coefficient plus the enthalpy-of-vaporisation term "
                             "(diffusion.jl:799-815, 861-911)",
                  "diff_rdf_ev": "train()'s :diff_rdf_ev: diffusion coefficient, the O-O and O-H "
                                 "L1 RDF terms of the water atoms on the reference grid and "
                                 "slices against flat synthetic targets (g = 1; the Soper data "
                                 "is not on the box), and the enthalpy term "
                                 "(diffusion.jl:759-815, 861-911)"}[a.gas_loss],
         "source": "train() of diffusion.jl:1683-1700 (50 ps forward, loss every 500 fs, "
                   "reverse truncated at 200 steps per loss point)",
         "l2": "flushed (256 MiB write) between timed steps"}
    if extra:
        c.update(extra)
    return c


def gas_prepare(a, device):
    """Seeded gas-in-water box equilibrated on the GPU (a.equil_ps ps of Langevin, gamma 1/ps)."""
    from revsim import constants as C, systems
    from revsim.gas import GasEngine
    x = systems.gas_water_coords(a.gas_water, a.gas_n, a.gas_box, seed=0)
    v = systems.gas_water_velocities(a.gas_water, a.gas_n, seed=1)
    p = np.array(C.gas_default_params(a.form))
    eq = GasEngine(a.gas_water, a.gas_n, a.gas_box, a.form, device=device)
    eq.set_params(p)
    eq.set_state(x, v)
    n = 1000 * a.equil_ps
    eq.forward(systems.noise_seeds(n, seed=30), 1.0, n, n, 0.001, "diff", calc_loss=False)
    x0, v0 = eq.get_state()
    eq.close()
    return x0, v0, p


def gas_count_ipairs(x, a, cutoff=1.0):
    """Unordered pairs within the cutoff that carry a term (water-water, and pairs of non-H
    sites), and how many of them carry the pair form."""
    n = len(x)
    nw3 = 3 * a.gas_water
    kind = np.array([(0 if i % 3 == 0 else 1) if i < nw3 else 2 for i in range(n)])
    mol = np.array([i // 3 if i < nw3 else a.gas_water + (i - nw3) // 2 for i in range(n)])
    total = form = 0
    for i0 in range(0, n, 512):
        d = x[None, :, :] - x[i0:i0 + 512, None, :]
        d -= a.gas_box * np.round(d / a.gas_box)
        r2 = (d * d).sum(-1)
        ii = np.arange(i0, min(i0 + 512, n))[:, None]
        jj = np.arange(n)[None, :]
        ki, kj = kind[ii], kind[jj]
        ok = (jj > ii) & (mol[ii] != mol[jj]) & (r2 <= cutoff * cutoff)
        coul = (ki != 2) & (kj != 2)
        pf = (ki != 1) & (kj != 1)
        total += int((ok & (coul | pf)).sum())
        form += int((ok & pf).sum())
    return total, form


def gas_rdf_terms(a):
    """The RDF terms of the diffusion workload: loss_rdf's O-O and O-H L1 terms on the
    reference grid and slices (diffusion.jl:759-774) against flat targets (g = 1)."""
    from revsim.loss import reference_rdf_terms
    return reference_rdf_terms(np.ones(248), np.ones(281)) if "rdf" in a.gas_loss else None


def gas_oracle_rdf(a):
    from oracle import orc
    terms = gas_rdf_terms(a)
    if terms is None:
        return None
    return orc.Loss([orc.RdfTerm(t.sel1, t.sel2, t.x_min, t.step, t.width, t.exp_cutoff, t.n_grid,
                                 t.slice_start, t.slice_stride, t.target, t.norm, t.weight)
                     for t in terms])


def gas_cpu_sample(a, x0, v0, p):
    """The FP64 oracle on a bounded sample, scaled to the workload: 10 forward steps, the 4
    reverse steps of two truncated blocks (diffusion loss only), and one loss point of the RDF
    and enthalpy terms (value and gradient), counted twice per loss point (forward value,
    reverse gradient)."""
    from oracle import orc
    from revsim import systems
    s = orc.make_gas_system(a.gas_water, a.gas_n, a.gas_box, a.form)
    rdf = gas_oracle_rdf(a)
    seeds = systems.noise_seeds(10, seed=98)
    t0 = time.perf_counter()
    xf, vf, _, sx, sv, gc, _ = orc.gas_forward_sim(s, p, x0, v0, seeds, 1.0, 10, 5, 0.001, "diff")
    t1 = time.perf_counter()
    orc.gas_reverse_sim(s, p, xf, vf, seeds, 1.0, 10, 5, 2, 0.001, sx, sv, gc, "diff")
    t2 = time.perf_counter()
    if rdf is not None:
        orc.loss_grad(orc.make_system(a.gas_water, a.gas_box), rdf, xf[:3 * a.gas_water])
    if "ev" in a.gas_loss:
        orc.gas_ev_point(s, p, xf, 1)
    t3 = time.perf_counter()
    nb = a.gas_steps // a.gas_steps_loss
    n_rev = nb * min(a.gas_trunc, a.gas_steps_loss)
    per_grad = (t1 - t0) / 10 * a.gas_steps + (t2 - t1) / 4 * n_rev + 2 * nb * (t3 - t2)
    n_atoms = 3 * a.gas_water + 2 * a.gas_n
    return n_atoms * a.gas_steps / per_grad, orc.num_threads(), (
        f"10 forward and 4 reverse steps of the {n_atoms}-atom box and one loss point of the "
        f"RDF / enthalpy terms, FP64 oracle; scaled to {a.gas_steps} forward + {n_rev} reverse "
        f"steps and {nb} loss points (each counted twice)")


def run_reference_diffusion(a):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import orc
    from revsim import constants as C, systems
    orc.build()
    s = orc.make_gas_system(a.gas_water, a.gas_n, a.gas_box, a.form)
    x = systems.gas_water_coords(a.gas_water, a.gas_n, a.gas_box, seed=0)
    v = systems.gas_water_velocities(a.gas_water, a.gas_n, seed=1)
    p = np.array(C.gas_default_params(a.form))
    x, v, *_ = orc.gas_forward_sim(s, p, x, v, systems.noise_seeds(40, seed=30), 1.0, 40, 40, 0.001,
                                   "diff", calc_loss=False)
    vals = []
    for i in range(a.warmup + a.steps):
        val, cores, desc = gas_cpu_sample(a, x, v, p)
        if i >= a.warmup:
            vals.append(val)
    value = statistics.mean(vals)
    n_atoms = 3 * a.gas_water + 2 * a.gas_n
    out = {"metric": DIFF_METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": 1e3 * n_atoms * a.gas_steps / value,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "impl": "reference", "config": diffusion_config(a),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_ours_diffusion(a):
    """One gradient of the gas-in-water system per step: forward_sim then reverse_sim through
    the host API, from host arrays, on one GPU per rank (independent replicas)."""
    import ctypes
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import build as _build
    _build.build()
    from revsim import _lib, systems
    from revsim.gas import GasEngine, forward_sim, reverse_sim
    x0, v0, p = gas_prepare(a, local)
    eng = GasEngine(a.gas_water, a.gas_n, a.gas_box, a.form, device=local, precision=a.gas_precision)
    if "rdf" in a.gas_loss:
        eng.set_rdf(gas_rdf_terms(a))
    seeds = systems.noise_seeds(a.gas_steps, seed=700 + rank)
    stream = torch.cuda.ExternalStream(eng.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def run():
        sys_f, loss_f, acc, _ = forward_sim(x0, v0, seeds, 1.0, a.gas_steps, a.gas_steps_loss, p,
                                            0.001, 1, a.form, a.gas_loss, engine=eng)
        out = reverse_sim(sys_f.coords, sys_f.velocities, seeds, 1.0, a.gas_steps, a.gas_steps_loss,
                          a.gas_trunc, p, 0.001, 1, sys_f.loggers, acc, a.form, a.gas_loss)
        return loss_f, out

    for _ in range(a.warmup):
        run()
    n0 = eng.launch_count()
    times = []
    with Clocks(local) as clk:
        for _ in range(a.steps):
            flush.zero_()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            loss_f, out = run()
            e1.record(stream)
            barrier()
            times.append(e0.elapsed_time(e1))
    launches = (eng.launch_count() - n0) // a.steps
    total = sum(times)
    if dist is not None:
        t = torch.tensor([total], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    ms = total / a.steps
    n_atoms = 3 * a.gas_water + 2 * a.gas_n
    value = world * n_atoms * a.gas_steps / (ms * 1e-3)
    eng.set_kernel_timing(True)
    run()
    rev_ms, rev_n = eng.kernel_time(0)
    fwd_ms, fwd_n = eng.kernel_time(1)
    eng.set_kernel_timing(False)
    ipairs, form_pairs = gas_count_ipairs(x0, a)
    peak = ctypes.c_double()
    mixed = a.gas_precision == "mixed"
    (_lib.load().revsim_probe_fp32_tflops if mixed else _lib.load().revsim_probe_fp64_tflops)(
        local, ctypes.byref(peak))
    fl_fwd = FLOPS_FWD_IPAIR * ipairs + FLOPS_FWD_OO_EXTRA * form_pairs
    fl_rev = FLOPS_REV_IPAIR * ipairs
    k_rev, k_fwd = rev_ms / max(rev_n, 1), fwd_ms / max(fwd_n, 1)
    rev_dominant = rev_ms >= fwd_ms
    launch_ms = k_rev if rev_dominant else k_fwd
    flops_launch = fl_rev if rev_dominant else fl_fwd
    achieved = flops_launch / (launch_ms * 1e-3) / 1e12
    roofline = {"bound": "fp32" if mixed else "fp64", "achieved": achieved, "peak": peak.value,
                "unit": "TFLOP/s", "frac": achieved / peak.value if peak.value else None,
                "traffic": GAS_REV_STEP_DRAM_BYTES if rev_dominant else GAS_FWD_STEP_DRAM_BYTES,
                "traffic_source": "ncu constant from one capture of this kernel on this system",
                "traffic_note": "ncu, cold caches (rows and positions are L2-resident live)",
                "kernel": ("k_gas_step<LJ, reverse>" if rev_dominant else "k_gas_step<LJ, forward>"),
                "launch_ms": launch_ms, "ipairs": ipairs, "pair_form_ipairs": form_pairs,
                "flops_per_launch": flops_launch,
                "peak_source": ("measured FP32 FMA throughput of this GPU (revsim_probe_fp32_tflops)" if mixed
                                else "measured FP64 FMA throughput of this GPU (revsim_probe_fp64_tflops)"),
                "reverse_step_ms": k_rev, "forward_step_ms": k_fwd,
                "reverse_share": rev_ms / ms, "forward_share": fwd_ms / ms}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        val, cores, desc = gas_cpu_sample(a, x0, v0, p)
        cpu = {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}
    if rank == 0:
        sys_r, loss_r, dl_dp, D, l_diff, l_rdf, l_ev = out
        nb = a.gas_steps // a.gas_steps_loss
        res = {"metric": DIFF_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64" if a.gas_precision == "fp64" else "f32+f64",
               "data": "synthetic",
               "config": diffusion_config(a, {"parallelism": f"replicas{world}" if world > 1 else "single"}),
               "e2e": {"value": value, "unit": UNIT,
                       "h2d_bytes_per_step": 2 * 3 * n_atoms * 8 + nb * 6 * a.gas_n * 8,
                       "d2h_bytes_per_step": 4 * 3 * n_atoms * 8 + nb * 6 * a.gas_n * 8 + n_atoms * len(p) * 8},
               "e2e_note": "every timed step runs forward_sim and reverse_sim of revsim.gas from host arrays",
               "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
               "clocks": clk.summary(), "loss_fwd": float(loss_f), "loss_rev": float(loss_r),
               "D_m2_per_s": D, "l_diff": l_diff, "l_ev": l_ev,
               "gradient": [float(g) for g in dl_dp]}
        print(json.dumps(res), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------ diamond workload
# Algorithmic work of the Stillinger-Weber reverse terms kernel, counted from its
# arithmetic (add/mul = 1, FMA = 2, div/exp = 1) with 4 tangents (the position direction
# and a, gamma, sigma): per ordered pair of active neighbours (q, q') of a centre 97 flops
# (the 3-body gradient with respect to d_q: 18 for the value, 79 for the tangents), per
# active neighbour 440 flops (unit vector, radial factors, 2-body term, slot assembly,
# parameter contraction).  Forward kernel (values only): 18 and 40.
SW_FLOPS_REV_PAIR, SW_FLOPS_REV_SLOT = 97, 440
SW_FLOPS_FWD_PAIR, SW_FLOPS_FWD_SLOT = 18, 40
# The learned radial term per active slot within its 0.25 nm cutoff: reverse 25 flops
# (interval, u'/2 and its tangent, the coefficient-adjoint weights), forward 10.
SW_FLOPS_REV_MLP, SW_FLOPS_FWD_MLP = 25, 10
SW_DT, SW_GAMMA, SW_NOISE = 0.0005, 4.0, 0.005


def diamond_name(a):
    return (f"diamond_sw{'' if a.sw_plain else '+mlp'}_{a.replicas}x{8 * a.cells ** 3}atoms_"
            f"{a.precision}_{a.sw_steps}fwd+{a.sw_steps}rev")


def diamond_params(a):
    """SW parameters of diamond.jl:53, then (with the learned term) its seeded MLP."""
    from revsim import diamond as D
    p = D.default_params()
    return p if a.sw_plain else np.concatenate([p, D.init_mlp_params(3)])


def diamond_config(a, extra=None):
    from revsim import diamond as D
    c = {"workload": diamond_name(a), "replicas": a.replicas, "n_atoms_per_replica": 8 * a.cells ** 3,
         "box_nm": a.cells * D.LATTICE_A, "lattice_nm": D.LATTICE_A, "noise_nm": SW_NOISE,
         "temp_K": 300.0, "n_steps": a.sw_steps, "n_steps_loss": a.sw_steps_loss,
         "n_steps_trunc": a.sw_steps_loss, "dt_ps": SW_DT, "gamma_per_ps": SW_GAMMA,
         "precision": a.precision,
         "loss": "stress tensor squared error (weight 5e-8) vs the mean stress of a run with "
                 "A x1.05, lambda x0.95",
         "learned_term": None if a.sw_plain else (
             "one MLP pair function on the SW 2-body term: 16 RBF (0-0.25 nm, width 0.0125 nm) "
             "-> 64 -> 64 SiLU -> 1, cosine cutoff, 5,313 parameters, seeded Xavier init; "
             "tabulated on 1,024 intervals, cubic Hermite per active pair within 0.25 nm"),
         "equilibration": "1 ps Langevin (gamma 4/ps) from the noisy lattice, untimed",
         "l2": "flushed (256 MiB write) between timed steps"}
    if extra:
        c.update(extra)
    return c


def diamond_prepare(a, device):
    """Equilibrated replicas and the stress target, made on the GPU by the engine."""
    from revsim import SwEngine, diamond as D, systems
    xs, vs, boxes = [], [], []
    for r in range(a.replicas):
        x, box = D.diamond_coords(a.cells, noise=SW_NOISE, seed=4 + r)
        xs.append(x)
        vs.append(D.mb_velocities(len(x), temp=300.0, seed=1000 + r))
        boxes.append(box)
    n = len(xs[0])
    p = diamond_params(a)
    eq = SwEngine([n] * a.replicas, boxes, temp=300.0, precision="mixed", device=device,
                  mlp=not a.sw_plain)
    eq.set_params(p)
    eq.set_state(np.concatenate(xs), np.concatenate(vs))
    eq.set_loss()
    eq.forward(systems.noise_seeds(2000 * a.replicas, seed=30).reshape(2000, a.replicas),
               SW_GAMMA, 2000, 2000, SW_DT, calc_loss=False)
    x0, v0 = eq.get_state()
    pt = p.copy()
    pt[0] *= 1.05
    pt[3] *= 0.95
    eq.set_params(pt)
    eq.forward(systems.noise_seeds(200 * a.replicas, seed=31).reshape(200, a.replicas),
               SW_GAMMA, 200, 200, SW_DT, calc_loss=False)
    target = eq.stress().mean(axis=0)
    eq.close()
    return x0, v0, boxes, p, target


def diamond_cpu_sample(a, x0, v0, box, p, target, n_s=2):
    """The FP64 oracle on n_s forward + n_s reverse steps of one replica (all host threads)."""
    from oracle import orc
    from revsim import systems
    n = len(x0)
    s = orc.make_sw_system(n, box, 300.0, mlp=len(p) > 7)
    L = orc.make_sw_loss(5e-8, target)
    seeds = systems.noise_seeds(n_s, seed=98)
    t0 = time.perf_counter()
    xf, vf, _, sx, sv = orc.sw_forward_sim(s, p, x0, v0, seeds, SW_GAMMA, n_s, n_s, SW_DT, L, 0,
                                           False)
    orc.sw_reverse_sim(s, p, xf, vf, seeds, SW_GAMMA, n_s, n_s, n_s, SW_DT, sx, sv, L)
    t1 = time.perf_counter()
    return n * n_s / (t1 - t0), orc.num_threads(), (
        f"{n_s} forward + {n_s} reverse steps of one {n}-atom replica, FP64 oracle "
        f"(its loss evaluations included)")


def run_reference_diamond(a):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import orc
    from revsim import diamond as D
    orc.build()
    x, box = D.diamond_coords(a.cells, noise=SW_NOISE, seed=4)
    v = D.mb_velocities(len(x), temp=300.0, seed=1000)
    p = diamond_params(a)
    vals = []
    for i in range(a.warmup + a.steps):
        val, cores, desc = diamond_cpu_sample(a, x, v, box, p, np.zeros(9))
        if i >= a.warmup:
            vals.append(val)
    value = statistics.mean(vals)
    n_tot = a.replicas * len(x)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": 1e3 * n_tot * a.sw_steps / value,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "impl": "reference", "config": diamond_config(a, {"precision": "fp64"}),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "note": "the reference is Julia (Molly/Enzyme/JAX); no Julia toolchain exists on these "
                   "machines, so this arm times the FP64 C restatement of its algorithm"}
    print(json.dumps(out), flush=True)


def run_ours_diamond(a):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import build as _build
    _build.build()
    import ctypes
    from revsim import SwEngine, _lib, systems

    x0, v0, boxes, p, target = diamond_prepare(a, local)
    R, n = a.replicas, len(x0) // a.replicas
    N = R * n
    K, NL = a.sw_steps, a.sw_steps_loss

    def make(prec):
        e = SwEngine([n] * R, boxes, temp=300.0, precision=prec, device=local, mlp=not a.sw_plain)
        e.set_params(p)
        e.set_loss(5e-8, target)
        e.set_state(x0, v0)
        return e

    eng = make(a.precision)
    seeds = systems.noise_seeds(K * R, seed=200 + rank).reshape(K, R)
    if a.profile:
        # one gradient between cudaProfilerStart/Stop (ncu --profile-from-start off)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        eng.forward(seeds, SW_GAMMA, K, NL, SW_DT)
        eng.reverse(seeds, SW_GAMMA, K, NL, NL, SW_DT)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        eng.close()
        return
    stream = torch.cuda.ExternalStream(eng.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def gradient(e=eng):
        lf, _ = e.forward(seeds, SW_GAMMA, K, NL, SW_DT)
        lr, g = e.reverse(seeds, SW_GAMMA, K, NL, NL, SW_DT)
        return lf, lr, g

    for _ in range(a.warmup):
        eng.set_state(x0, v0)
        gradient()
    n0 = eng.launch_count()
    times = []
    with Clocks(local) as clk:
        for _ in range(a.steps):
            eng.set_state(x0, v0)
            flush.zero_()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            lf, lr, g = gradient()
            e1.record(stream)
            barrier()
            times.append(e0.elapsed_time(e1))
    launches = (eng.launch_count() - n0) // a.steps
    clocks = clk.summary()
    total_ms = sum(times)
    if dist is not None:
        t = torch.tensor([total_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_step = total_ms / a.steps
    value = world * N * K / (ms_step * 1e-3)

    # end to end through the public API from pinned host buffers
    xh = torch.from_numpy(x0.copy()).pin_memory()
    vh = torch.from_numpy(v0.copy()).pin_memory()
    e2e_ms = []
    for _ in range(a.steps):
        flush.zero_()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.set_state(xh.numpy(), vh.numpy())
        gradient()
        e1.record(stream)
        barrier()
        e2e_ms.append(e0.elapsed_time(e1))
    e2e_total = sum(e2e_ms)
    if dist is not None:
        t = torch.tensor([e2e_total], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * N * K / (e2e_total / a.steps * 1e-3)
    h2d = 2 * 3 * N * 8 + 2 * K * R * 8
    d2h = 2 * R * 8 + R * len(p) * 8 + 2 * 3 * N * 8

    # roofline of the dominant kernel (the reverse terms kernel), timed per launch
    eng.set_state(x0, v0)
    eng.set_kernel_timing(True)
    gradient()
    # the reverse pass ends at the start state, rebuilt over the first loss block
    recon = {a.precision: recon_error(eng.get_state()[0], x0, np.repeat(np.asarray(boxes), n)),
             "steps_reconstructed": NL, "gamma_per_ps": SW_GAMMA,
             "integrator": "the reference's step arithmetic"}
    rt_ms, rt_n = eng.kernel_time(0)
    ft_ms, ft_n = eng.kernel_time(1)
    rg_ms, rg_n = eng.kernel_time(2)
    fg_ms, fg_n = eng.kernel_time(3)
    eng.set_kernel_timing(False)
    launch_ms = rt_ms / max(rt_n, 1)
    pairs = eng.active_pairs()
    deg = np.bincount(pairs.ravel(), minlength=N).astype(np.int64)
    flops_launch = int(SW_FLOPS_REV_PAIR * (deg * (deg - 1)).sum() + SW_FLOPS_REV_SLOT * deg.sum())
    n_mlp_slots = 0
    if not a.sw_plain:
        # both slots of every active pair within the learned term's 0.25 nm cutoff
        xs_now = eng.get_state()[0]
        L_pair = np.asarray(boxes)[pairs[:, 0] // n][:, None]
        d = xs_now[pairs[:, 1]] - xs_now[pairs[:, 0]]
        d -= L_pair * np.round(d / L_pair)
        n_mlp_slots = 2 * int((np.linalg.norm(d, axis=1) < 0.25).sum())
        flops_launch += SW_FLOPS_REV_MLP * n_mlp_slots
    achieved = flops_launch / (launch_ms * 1e-3) / 1e12
    peak = ctypes.c_double()
    _lib.load().revsim_probe_fp32_tflops(local, ctypes.byref(peak))
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": achieved / peak.value if peak.value else None, "traffic": None,
                "kernel": "k_terms<float, 16, TM_REV> (Stillinger-Weber reverse terms)",
                "launch_ms": launch_ms, "launches_timed": rt_n, "flops_per_launch": flops_launch,
                "mean_active_neighbours": float(deg.mean()),
                "learned_term_slots_per_launch": n_mlp_slots,
                "peak_source": "measured FP32 FFMA throughput of this GPU (revsim_probe_fp32_tflops)",
                "kernel_ms_per_launch": {"rev_terms": launch_ms, "fwd_terms": ft_ms / max(ft_n, 1),
                                         "rev_gather": rg_ms / max(rg_n, 1),
                                         "fwd_gather": fg_ms / max(fg_n, 1)},
                "step_kernels_share_of_gradient": (rt_ms + ft_ms + rg_ms + fg_ms) / ms_step}

    extra = {}
    if not a.no_compare and rank == 0:
        e64 = make("fp64")
        gradient(e64)
        s64 = torch.cuda.ExternalStream(e64.stream())
        e64.set_state(x0, v0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s64)
        _, _, g64 = gradient(e64)
        e1.record(s64)
        torch.cuda.synchronize()
        ms64 = e0.elapsed_time(e1)
        recon["fp64"] = recon_error(e64.get_state()[0], x0, a.box)
        eng.set_state(x0, v0)
        _, _, gm = gradient()
        short = {}
        for eng_, key in ((eng, "mixed"), (e64, "fp64")):
            eng_.set_state(x0, v0)
            eng_.forward(seeds[:100], SW_GAMMA, 100, 100, SW_DT)
            short[key] = eng_.reverse(seeds[:100], SW_GAMMA, 100, 100, 100, SW_DT)[1].mean(axis=0)

        def rel(gx, gref):
            # SW parameters in units of dL/dlog(theta); the MLP's (when present) relative to
            # the largest MLP entry
            q = p[:7]
            sc = np.abs(gref[:7] * q)
            e = float(np.max(np.abs((gx[:7] - gref[:7]) * q) / np.maximum(sc, 0.01 * sc.max())))
            if len(p) > 7:
                e = max(e, float(np.abs(gx[7:] - gref[7:]).max() / np.abs(gref[7:]).max()))
            return e
        extra = {"fp64_gpu": {"value": N * K / (ms64 * 1e-3), "ms_per_step": ms64,
                              "speedup_mixed_over_fp64": ms64 / ms_step},
                 "grad_rel_err_vs_fp64": {
                     "full_workload": rel(gm.mean(axis=0), g64.mean(axis=0)),
                     "first_100_steps": rel(short["mixed"], short["fp64"]),
                     "definition": "replica-mean gradient; max over the SW parameters of "
                                   "|g - g_fp64| |theta| / max(|g_fp64 theta|, 0.01 max_k "
                                   "|g_fp64,k theta_k|), and over the MLP parameters of "
                                   "|g - g_fp64| / max |g_fp64,mlp|"}}
        e64.close()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        val, cores, desc = diamond_cpu_sample(a, x0[:n], v0[:n], boxes[0], p, target)
        cpu = {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None,
               "dtype": "f32+f64" if a.precision == "mixed" else "f64", "data": "synthetic",
               "config": diamond_config(a, {"parallelism": f"replicas{world}" if world > 1 else "single"}),
               "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": d2h},
               "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
               "clocks": clocks, "recon": recon,
               "loss": {"forward": float(lf.mean()), "reverse": float(lr.mean())}}
        out.update(extra)
        print(json.dumps(out), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------------------- MLP workload
# Extra work of the learned pair correction per interacting pair (interval index and
# coordinate, cubic derivative; reverse also the second derivative and the coefficient
# adjoints): forward 12, reverse 24 flops.
MLP_FLOPS_FWD_EXTRA, MLP_FLOPS_REV_EXTRA = 12, 24


def mlp_config(a, extra=None):
    c = {"workload": f"water_895mol_3nm_lj+mlp_{a.precision}_1000fwd+1000rev",
         "n_atoms": 2685, "box_nm": 3.0, "n_steps": 1000, "n_steps_loss": 1000,
         "n_steps_trunc": 1000, "dt_ps": 0.001, "gamma_per_ps": 0.0,
         "learned_term": "per element pair (O-O, O-H, H-H) MLP 16 RBF (0-1 nm, width 0.05 nm) "
                         "-> 64 -> 64 SiLU -> 1, cosine cutoff, 15,939 parameters, seeded "
                         "Xavier init; tabulated on 1,024 intervals, cubic Hermite per pair",
         "loss": "O-O smoothed RDF, 200 bins 0-1 nm, squared error vs sigma x1.02 / eps x0.95 target",
         "training": "see the line's training object (4 x 400 waters, three seeds, equal "
                     "wall-clock, a teacher target outside the classical family)",
         "mlp_precision": a.mlp_precision, "integrator": a.integrator,
         "precision": a.precision, "l2": "flushed (256 MiB write) between timed steps"}
    if extra:
        c.update(extra)
    return c


def mlp_training_comparison(a, local, n_mol=400, box=2.48, R=4, n_steps=400, n_loss=100,
                            seeds=(1, 2, 3)):
    """The learned term's gain at equal wall-clock, against a target the classical model
    cannot represent: the O-O RDF of a teacher (default LJ plus a fixed MLP correction, the
    seeded initialisation + N(0, 0.05)).  Per seed, the classical model runs a.updates Adam
    updates (train()'s truncated schedule: gamma = 1/ps, loss every n_loss steps, reverse
    windows of n_loss steps, R replicas per update, the dynamics continuing across updates)
    and the classical + MLP model (network on the tensor cores) runs for the same wall-clock
    time; the score is the mean loss over the last quarter of each arm's updates.  Start
    state: a seeded lattice with 1 ps of Langevin dynamics on the GPU."""
    import torch
    from revsim import Engine, constants as C, mlp, oo_l2_term, systems
    p = np.array(C.default_params("lj"))
    eq = Engine(n_mol, box, precision="mixed", device=local)
    eq.set_params(p)
    eq.set_state(systems.water_coords(n_mol, box, seed=21), systems.mb_velocities(n_mol, seed=22))
    eq.forward(systems.noise_seeds(1000, seed=23), 5.0, 1000, 1000, 0.001, calc_loss=False)
    x, v = eq.get_state()
    eq.close()
    teach = Engine([n_mol] * R, [box] * R, precision="mixed", device=local, mlp=True)
    teach.set_mlp_precision(a.mlp_precision)
    teach.set_params(np.concatenate([p, mlp.init_params(11) + np.random.default_rng(12).normal(
        scale=0.05, size=mlp.N_PARAMS)]))
    teach.set_state(np.concatenate([x] * R), np.concatenate([v] * R))
    teach.forward(systems.noise_seeds(1000 * R, seed=13).reshape(1000, R), 5.0, 1000, 1000, 0.001,
                  calc_loss=False)
    teach.set_loss([oo_l2_term(np.zeros(200))])
    rdfs = []
    for k in range(4):
        teach.forward(systems.noise_seeds(250 * R, seed=14 + k).reshape(250, R), 1.0, 250, 250, 0.001,
                      calc_loss=False)
        rdfs += [teach.rdf(0, r) for r in range(R)]
    teach.close()
    target = np.mean(rdfs, axis=0)

    def arm(use_mlp, seed, n_updates=None, wall=None):
        th = np.concatenate([p, mlp.init_params(3)]) if use_mlp else p.copy()
        e = Engine([n_mol] * R, [box] * R, precision="mixed", device=local, mlp=use_mlp)
        if use_mlp:
            e.set_mlp_precision(a.mlp_precision)
        e.set_params(th)
        e.set_loss([oo_l2_term(target)])
        xs, vs = np.concatenate([x] * R), np.concatenate([v] * R)
        scale = np.full(len(th), 1e-3)
        scale[:len(p)] = 2e-3 * np.abs(p)
        opt = mlp.Adam(len(th), lr=scale)
        losses = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u = 0
        while (n_updates is not None and u < n_updates) or (wall is not None and time.perf_counter() - t0 < wall):
            e.set_params(th)
            e.set_state(xs, vs)
            sd = systems.noise_seeds(n_steps * R, seed=100000 * seed + u).reshape(n_steps, R)
            e.forward(sd, 1.0, n_steps, n_loss, 0.001, calc_loss=False)
            xs, vs = e.get_state()
            lr_, g = e.reverse(sd, 1.0, n_steps, n_loss, n_loss, 0.001)
            losses.append(float(np.mean(lr_)))
            th = opt.step(th, g.mean(axis=0))
            u += 1
        torch.cuda.synchronize()
        wall_s = time.perf_counter() - t0
        e.close()
        k = max(1, len(losses) // 4)
        return {"wall_s": wall_s, "updates": u, "loss_first": losses[0],
                "loss_last_quarter": float(np.mean(losses[-k:]))}

    per_seed = []
    for seed in seeds:
        cl = arm(False, seed, n_updates=a.updates)
        ml = arm(True, seed, wall=cl["wall_s"])
        per_seed.append({"seed": seed, "classical": cl, "classical+mlp": ml})
    mean_cl = float(np.mean([r["classical"]["loss_last_quarter"] for r in per_seed]))
    mean_ml = float(np.mean([r["classical+mlp"]["loss_last_quarter"] for r in per_seed]))
    return {"system": f"{R} x {n_mol} waters, {box} nm (the GPU training test's system)",
            "target": "O-O RDF of default LJ + a fixed MLP correction (seeded init + N(0, 0.05))",
            "schedule": f"per update {n_steps} steps, gamma 1/ps, loss every {n_loss}, reverse "
                        f"windows of {n_loss}; classical {a.updates} updates, classical + MLP the "
                        "same wall-clock; Adam, classical lr 2e-3 x |theta_0|, MLP lr 1e-3",
            "per_seed": per_seed, "mean_last_quarter": {"classical": mean_cl, "classical+mlp": mean_ml}}


def run_ours_mlp(a):
    """The 895-water system with the learned pair correction.  Timed: the full
    gradient (1,000 forward + 1,000 reverse steps) with the MLP on.  Then a training
    comparison, wall-clock timed: the classical + MLP model and the classical model alone,
    each trained for the same number of Adam updates from the same start."""
    import ctypes
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    import build as _build
    _build.build()
    from revsim import Engine, _lib, mlp, oo_l2_term, systems
    a.n_mol, a.box, a.form = 895, 3.0, "lj"
    x0, v0, p, target = prepare(a, local, a.equil_ps)
    theta0 = np.concatenate([p, mlp.init_params(3)])
    eng = integ(Engine(895, 3.0, inter_type="lj", precision=a.precision, device=local, mlp=True), a)
    eng.set_mlp_precision(a.mlp_precision)
    eng.set_params(theta0)
    eng.set_loss([oo_l2_term(target)])
    eng.set_state(x0, v0)
    shape = eng.autotune()
    seeds = systems.noise_seeds(1000, seed=300 + rank)
    stream = torch.cuda.ExternalStream(eng.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def gradient(e=eng):
        e.set_state(x0, v0)
        lf = e.forward(seeds, 0.0, 1000, 1000, 0.001)
        lr, g = e.reverse(seeds, 0.0, 1000, 1000, 1000, 0.001)
        return lf, lr, g

    if a.profile:
        # one gradient between cudaProfilerStart/Stop (ncu --profile-from-start off)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        gradient()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        eng.close()
        return

    for _ in range(a.warmup):
        gradient()
    n0 = eng.launch_count()
    times = []
    with Clocks(local) as clk:
        for _ in range(a.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            lf, lr, g = gradient()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    launches = (eng.launch_count() - n0) // a.steps
    clocks = clk.summary()
    ms_step = sum(times) / a.steps
    value = world * 2685 * 1000 / (ms_step * 1e-3)
    h2d = 2 * 3 * 2685 * 8 + 2 * 1000 * 8
    d2h = 8 * 2 + 8 * len(theta0)

    # roofline: the reverse step kernel with the learned term
    eng.set_kernel_timing(True)
    gradient()
    kt_ms, kt_n = eng.kernel_time(0)
    eng.set_kernel_timing(False)
    launch_ms = kt_ms / max(kt_n, 1)
    xs, _ = eng.get_state()
    recon = {a.precision: recon_error(xs, x0, 3.0), "steps_reconstructed": 1000,
             "integrator": a.integrator}
    pairs = eng.neighbor_pairs(0)
    ipairs, _ = count_ipairs(xs, 3.0, pairs)
    flops_launch = (FLOPS_REV_IPAIR + MLP_FLOPS_REV_EXTRA) * ipairs
    peak = ctypes.c_double()
    _lib.load().revsim_probe_fp32_tflops(local, ctypes.byref(peak))
    achieved = flops_launch / (launch_ms * 1e-3) / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": achieved / peak.value if peak.value else None, "traffic": None,
                "kernel": "k_water_step<float, LJ_MLP, reverse>", "launch_ms": launch_ms,
                "shape": {"reverse": dict(zip(("lanes_per_mol", "mols_per_cta", "unroll"), shape[0])),
                          "forward": dict(zip(("lanes_per_mol", "mols_per_cta", "unroll"), shape[1]))},
                "ipairs": ipairs, "flops_per_launch": flops_launch,
                "peak_source": "measured FP32 FFMA throughput of this GPU (revsim_probe_fp32_tflops)"}

    # the network per pair against the table: one evaluation at every atom pair within the
    # cutoff (what a per-pair network would run in each forward step), and at the table nodes
    d = xs[pairs[:, 1]] - xs[pairs[:, 0]]
    d -= 3.0 * np.round(d / 3.0)
    rr = np.sqrt((d * d).sum(1))
    rr = rr[rr <= 1.0]
    n_row = (len(rr) + 2) // 3
    r_rows = np.resize(rr, 3 * n_row).reshape(3, n_row)
    eng.mlp_eval_time(r_rows)
    per_pair_ms = min(eng.mlp_eval_time(r_rows) for _ in range(5))
    nodes_ms = min(eng.mlp_eval_time() for _ in range(5))
    eng.set_kernel_timing(True)
    eng.set_state(x0, v0)
    eng.forward(seeds[:100], 0.0, 100, 100, 0.001)
    fk_ms, fk_n = eng.kernel_time(1)
    eng.set_kernel_timing(False)
    fwd_launch_ms = fk_ms / max(fk_n, 1)
    network = {"pairs_within_cutoff": int(len(rr)), "per_pair_eval_ms": per_pair_ms,
               "table_nodes_eval_ms": nodes_ms, "forward_step_kernel_ms": fwd_launch_ms,
               "note": "per_pair_eval_ms: the tensor-core network evaluated once at every atom "
                       "pair within the cutoff (value and derivative), the cost a per-pair "
                       "network would add to each forward step; the engine instead evaluates "
                       "3 x 1,025 table nodes once per parameter update (table_nodes_eval_ms) "
                       "and reads cubic Hermite intervals inside the step kernel"}

    # accuracy: mixed vs FP64 GPU gradient over the first 100 steps
    e64 = Engine(895, 3.0, inter_type="lj", precision="fp64", device=local, mlp=True)
    e64.set_params(theta0)
    e64.set_loss([oo_l2_term(target)])
    short = {}
    for e_, key in ((eng, "mixed"), (e64, "fp64")):
        e_.set_state(x0, v0)
        e_.forward(seeds[:100], 0.0, 100, 100, 0.001)
        short[key] = e_.reverse(seeds[:100], 0.0, 100, 100, 100, 0.001)[1][0]
    gm, g64 = short["mixed"], short["fp64"]
    nc = len(p)
    scl = np.abs(g64[:nc] * p)
    err_cl = float(np.max(np.abs((gm[:nc] - g64[:nc]) * p) / np.maximum(scl, 0.01 * scl.max())))
    err_mlp = float(np.abs(gm[nc:] - g64[nc:]).max() / np.abs(g64[nc:]).max())
    e64.close()

    train = mlp_training_comparison(a, local) if rank == 0 else None
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32+f64" if a.precision == "mixed" else "f64",
           "data": "synthetic", "config": mlp_config(a),
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
           "gpu_launches": launches, "roofline": roofline, "cpu_baseline": None,
           "clocks": clocks, "loss": {"forward": float(lf[0]), "reverse": float(lr[0])},
           "grad_rel_err_vs_fp64_first_100_steps": {"classical": err_cl, "mlp": err_mlp},
           "training": train, "network_per_pair_vs_table": network, "recon": recon,
           "e2e_note": "every timed gradient starts from host arrays (set_state), so value is "
                       "end to end"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    eng.close()


# ------------------------------------------------------------ replicas workload
def replica_systems(n_rep, seed=2):
    """64 water boxes: molecule counts log-uniform in [300, 3000] and temperatures uniform in
    [280, 320] K from a seed; boxes at liquid density, at least 2.45 nm (the minimum image
    of the 1.2 nm neighbour cutoff needs a side above 2.4 nm, so replicas under ~480
    molecules are less dense)."""
    from revsim import systems
    rng = np.random.default_rng(seed)
    n_mol = np.round(np.exp(rng.uniform(np.log(300), np.log(3000), n_rep))).astype(int)
    temps = rng.uniform(280.0, 320.0, n_rep)
    boxes = np.array([max(systems.box_for_density(n), 2.45) for n in n_mol])
    return n_mol, boxes, temps


def replicas_config(a, n_mol, extra=None):
    c = {"workload": f"water_{a.n_replicas}replicas_{int(n_mol.sum())}mol_lj_{a.precision}_"
                     f"{a.rep_steps}fwd+{a.rep_steps}rev",
         "replicas": a.n_replicas, "n_mol_range": [int(n_mol.min()), int(n_mol.max())],
         "n_atoms": int(3 * n_mol.sum()), "temp_K_range": [280, 320], "n_steps": a.rep_steps,
         "n_steps_loss": 1000, "n_steps_trunc": 1000, "dt_ps": 0.001, "gamma_per_ps": 1.0,
         "loss": "O-O smoothed RDF, 200 bins 0-1 nm, squared error vs the replica-mean RDF of a "
                 "sigma x1.02 / eps x0.95 run; per-replica gradients averaged",
         "launch": "all replicas in one launch per step (per-CTA replica table), step launches "
                   "chained (programmatic dependent launch); the CUDA-graph mode "
                   "(revsim_set_graph_mode) is not used here: each step kernel runs ~0.6 ms, so "
                   "the launch queue never drains",
         "integrator": a.integrator,
         "precision": a.precision, "l2": "inputs larger than L2 are not guaranteed; flushed "
                                         "(256 MiB write) between timed steps"}
    if extra:
        c.update(extra)
    return c


def run_ours_replicas(a):
    """64 water boxes of uneven size and temperature in one handle; one bench step
    = one batched gradient (forward + reverse) whose per-replica gradients are averaged."""
    import ctypes
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import build as _build
    _build.build()
    from revsim import Engine, _lib, constants as C, oo_l2_term, systems
    from revsim.distributed import allreduce_mean, allreduce_sum, rank_share
    n_all, boxes_all, temps_all = replica_systems(a.n_replicas)
    R_all, K = a.n_replicas, a.rep_steps
    # this rank's share of the replicas (greedy atom-count balance); every per-replica input
    # is selected by replica index, so the job is the same at every rank count
    mine = rank_share(3 * n_all, world, rank)
    n_mol, boxes, temps = n_all[mine], boxes_all[mine], temps_all[mine]
    R = len(mine)
    p = np.array(C.default_params("lj"))
    x = np.concatenate([systems.water_coords(n_all[r], boxes_all[r], seed=10 + r) for r in mine])
    v = np.concatenate([systems.mb_velocities(n_all[r], temps_all[r], seed=100 + r) for r in mine])
    eq = Engine(n_mol, boxes, temp=temps, precision="mixed", device=local)
    eq.set_params(p)
    eq.set_state(x, v)
    for blk in range(2):
        eq.forward(systems.noise_seeds(1000 * R_all, seed=20 + blk).reshape(1000, R_all)[:, mine], 5.0,
                   1000, 1000, 0.001, calc_loss=False)
    x0, v0 = eq.get_state()
    pt = p.copy()
    pt[0] *= 1.02
    pt[1] *= 0.95
    eq.set_params(pt)
    eq.forward(systems.noise_seeds(1000 * R_all, seed=30).reshape(1000, R_all)[:, mine], 5.0, 1000, 1000,
               0.001, calc_loss=False)
    eq.set_loss([oo_l2_term(np.zeros(200))])
    # the target: the mean RDF over all replicas of all ranks (set-up, untimed)
    target = allreduce_sum(np.sum([eq.rdf(0, r) for r in range(R)], axis=0)) / R_all
    eq.close()
    eng = integ(Engine(n_mol, boxes, temp=temps, precision=a.precision, device=local), a)
    eng.set_params(p)
    eng.set_loss([oo_l2_term(target)])
    eng.set_state(x0, v0)
    shape = eng.autotune()
    seeds = systems.noise_seeds(K * R_all, seed=400).reshape(K, R_all)[:, mine]
    stream = torch.cuda.ExternalStream(eng.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def gradient():
        # one parameter update's gradient: every rank's replicas, averaged over all ranks
        # (the one collective of the path, P + 1 doubles)
        eng.set_state(x0, v0)
        lf = eng.forward(seeds, 1.0, K, 1000, 0.001)
        lr, g = eng.reverse(seeds, 1.0, K, 1000, 1000, 0.001)
        return lf, lr, allreduce_mean(g)

    if a.profile:
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        gradient()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        eng.close()
        return
    for _ in range(a.warmup):
        gradient()
    n0 = eng.launch_count()
    times = []
    with Clocks(local) as clk:
        for _ in range(a.steps):
            flush.zero_()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            lf, lr, g = gradient()
            e1.record(stream)
            barrier()
            times.append(e0.elapsed_time(e1))
    launches = (eng.launch_count() - n0) // a.steps
    clocks = clk.summary()
    total_ms = sum(times)
    if dist is not None:
        t = torch.tensor([total_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_step = total_ms / a.steps
    n_atoms = int(3 * n_all.sum())            # the whole job: every rank's replicas
    value = n_atoms * K / (ms_step * 1e-3)
    eng.set_kernel_timing(True)
    gradient()
    kt_ms, kt_n = eng.kernel_time(0)
    ft_ms, ft_n = eng.kernel_time(1)
    eng.set_kernel_timing(False)
    launch_ms = kt_ms / max(kt_n, 1)
    xs, _ = eng.get_state()
    # the reverse pass ends at the start state, rebuilt over the first 1,000-step block
    recon = {a.precision: recon_error(xs, x0, np.repeat(np.asarray(boxes, dtype=np.float64), 3 * np.asarray(n_mol))),
             "steps_reconstructed": 1000, "gamma_per_ps": 1.0, "integrator": a.integrator}
    ipairs = 0
    for r in range(R):
        sl = slice(int(3 * n_mol[:r].sum()), int(3 * n_mol[:r + 1].sum()))
        ipairs += count_ipairs(xs[sl], boxes[r], eng.neighbor_pairs(r))[0]
    flops_launch = FLOPS_REV_IPAIR * ipairs
    peak = ctypes.c_double()
    _lib.load().revsim_probe_fp32_tflops(local, ctypes.byref(peak))
    achieved = flops_launch / (launch_ms * 1e-3) / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": achieved / peak.value if peak.value else None, "traffic": None,
                "kernel": "k_water_step<float, LJ, reverse> over this rank's replicas",
                "launch_ms": launch_ms, "ipairs": ipairs, "flops_per_launch": flops_launch,
                "forward_step_launch_ms": ft_ms / max(ft_n, 1),
                "shape": {"reverse": dict(zip(("lanes_per_mol", "mols_per_cta", "unroll"), shape[0])),
                          "forward": dict(zip(("lanes_per_mol", "mols_per_cta", "unroll"), shape[1]))},
                "peak_source": "measured FP32 FFMA throughput of this GPU (revsim_probe_fp32_tflops)"}
    h2d = 2 * 3 * n_atoms * 8 + 2 * K * R_all * 8
    d2h = 2 * R_all * 8 + R_all * len(p) * 8
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "f32+f64" if a.precision == "mixed" else "f64",
           "data": "synthetic",
           "config": replicas_config(a, n_all, {
               "parallelism": f"replicas{world}" if world > 1 else "single",
               "gradient_exchange": "per-replica gradients averaged over all ranks by one "
                                    "all-reduce of P + 1 doubles per update (timed)",
               "sharding": "rank k runs partition_replicas(atoms, N)[k] of the 64 replicas "
                           "(greedy atom-count balance); the job is the same at every N"}),
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
           "gpu_launches": launches, "roofline": roofline, "cpu_baseline": None, "clocks": clocks,
           "loss": {"forward_mean": float(lf.mean()), "reverse_mean": float(lr.mean())},
           "recon": recon, "mean_gradient": [float(t) for t in g],
           "e2e_note": "every timed gradient starts from host arrays (set_state), so value is end to end"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    args = parse()
    if args.workload == "replicas":
        run_ours_replicas(args)
    elif args.workload == "cfg1":
        run_ours_cfg1(args)
    elif args.workload == "mlp":
        run_ours_mlp(args)
    elif args.workload == "diamond":
        run_reference_diamond(args) if args.impl == "reference" else run_ours_diamond(args)
    elif args.workload == "diffusion":
        run_reference_diffusion(args) if args.impl == "reference" else run_ours_diffusion(args)
    elif args.workload == "reweight":
        run_reference_reweight(args) if args.impl == "reference" else run_ours_reweight(args)
    elif args.workload == "equil":
        run_reference_equil(args) if args.impl == "reference" else run_ours_equil(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
