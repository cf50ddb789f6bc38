"""Benchmark of the FMM evaluation passes on B200 (one JSON line on rank 0).

Workload (the headline configuration): Laplace 3D, N = 4,000,000 points uniform on the
unit sphere surface (normalised Gaussian 3-vectors), sources = targets, charges N(0, 1),
p = 8, 128 points per leaf (adaptive octree), potential + gradient; mixed precision
(f32 points, expansions and P2P, f64 per-target accumulation).  Seeded synthetic input
(SplitMix64 + Box-Muller, restated here with numpy).  A step is one evaluation: charges
in, potentials and gradients out.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n N]

value     : N / (device time of one evaluation) in Mpoints/s, inputs resident in HBM,
            L2 flushed (a 512 MiB write) before every timed step, CUDA events on the
            evaluator's stream; the evaluation replayed from one captured CUDA graph of the
            whole sweep (fmmgpu_fmm_set_graph; direct launches reported beside it).
e2e       : the same through the public host API with pinned host buffers, host->device
            charges and device->host outputs inside the timed call: the f32 call
            (fmmgpu_fmm_evaluate_f32, the reference's Fmm<f32> value type, as its f32 runs
            use it) with its error at the sampled targets, the f64 call beside it.
plain_f64 : the plain f64 evaluator (the drop-in) on the same input, for the mixed/plain
            ratio of the metric.
error     : relative L2 of phi and grad at 2,000 sampled targets against an f64 direct sum
            (Neumaier-compensated, on the GPU) of all sources.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

import faulthandler

faulthandler.enable()

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

P = 8
LEAF = 128
N_DEFAULT = 4_000_000
SEED = 0x5EED_0002
SAMPLE = 2000
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# reference op model of P2P: 10 FP32 lane-ops per pair for phi, 15 with the gradient
# (fmm-validate/src/peaks.rs:12-17)
P2P_OPS = {False: 10, True: 15}


# ------------------------------------------------------------------------------------
# seeded synthetic input (SplitMix64 of fmm-validate/src/rng.rs, vectorised)
# ------------------------------------------------------------------------------------
def splitmix(seed, count):
    with np.errstate(over="ignore"):
        k = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform01(u):
    return (u >> np.uint64(11)).astype(np.float64) * (1.0 / float(1 << 53))


def normals(seed, count):
    """Box-Muller (cosine branch) on pairs of SplitMix64 uniforms, 1 - U in (0, 1]."""
    u = uniform01(splitmix(seed, 2 * count)).reshape(count, 2)
    return np.sqrt(-2.0 * np.log(1.0 - u[:, 0])) * np.cos(2.0 * np.pi * u[:, 1])


def sphere_problem(n, seed=SEED):
    g = normals(seed, 3 * n).reshape(n, 3)
    x = g / np.linalg.norm(g, axis=1, keepdims=True)
    q = normals(seed + 1, n)
    return np.ascontiguousarray(x), np.ascontiguousarray(q)


def sample_indices(n, count, seed=SEED + 2):
    r = splitmix(seed, count)
    order = np.arange(n)
    for i in range(count):
        j = i + int((int(r[i]) >> 32) * (n - i) >> 32)
        order[i], order[j] = order[j], order[i]
    return order[:count].copy()


# the batched workload: 256 clouds, N_i log-uniform in [1e4, 5e5], geometry uniform from
# {unit cube, unit sphere surface, Plummer sphere a = 0.1 clipped at r = 5 (resampled beyond)},
# 16 charge vectors U[-1, 1) per cloud, p = 6, 64 points per leaf, potentials
BATCH_CLOUDS = 256
BATCH_VECTORS = 16
BATCH_P = 6
BATCH_LEAF = 64


def batched_problem(seed=SEED + 7, clouds=BATCH_CLOUDS):
    """The batched workload's clouds and charges (numpy PCG64, seeded): a list of (N_i, 3)
    point arrays and the (sum N_i, 16) charges in cloud order."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(1e4), np.log(5e5), clouds)).astype(np.int64)
    kinds = rng.integers(0, 3, clouds)
    out = []
    for c in range(clouds):
        n = int(sizes[c])
        if kinds[c] == 0:
            x = rng.uniform(0.0, 1.0, (n, 3))
        elif kinds[c] == 1:
            g = rng.normal(size=(n, 3))
            x = g / np.linalg.norm(g, axis=1, keepdims=True)
        else:  # Plummer: r = a / sqrt(U^(-2/3) - 1), isotropic, resampled beyond r = 5
            r = np.empty(0)
            while len(r) < n:
                u = 1.0 - rng.uniform(size=2 * n)
                rr = 0.1 / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
                r = np.concatenate([r, rr[rr <= 5.0]])
            g = rng.normal(size=(n, 3))
            x = g / np.linalg.norm(g, axis=1, keepdims=True) * r[:n, None]
        out.append(np.ascontiguousarray(x))
    q = rng.uniform(-1.0, 1.0, (int(sizes.sum()), BATCH_VECTORS))
    return out, np.ascontiguousarray(q), kinds


# ------------------------------------------------------------------------------------
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"fmm_b200_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
            sm = [float(r[1]) for r in rows]
            smax = max(float(r[2]) for r in rows)
            reasons = set()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for r in rows:
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(name)
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                    "samples": len(rows)}
        except Exception as e:  # no nvidia-smi or no samples
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "error": str(e)[:80]}


def ncu_traffic(kernel):
    """DRAM bytes per work unit of `kernel` from a committed ncu summary (profiles/), or None."""
    try:
        t = json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic.json")))[kernel]
        return t
    except Exception:
        return None


def peaks():
    try:
        return json.load(open(PEAKS))
    except Exception:
        return {}


def passes_hbm(info, kinds, pk):
    """P2M, M2M, L2L and L2P+M2P as HBM passes: algorithmic bytes of one evaluation
    (f32 points, charges and expansions of n = (p+1)^2 coefficients, f64 target partials)
    over the kind's CUDA-event time, against the measured copy bandwidth."""
    s, nc, m, o = 4, (P + 1) ** 2, 1, 4  # bytes a float, coefficients, vectors, outputs a target
    nb, nl, ns, nt = info["nboxes"], info["nleaves"], info["nsources"], info["ntargets"]
    bytes_ = {
        "p2m": ns * (3 + m) * s + nl * m * nc * s,                 # points and charges in, leaf multipoles out
        "m2m": 2 * nb * m * nc * s,                                # a box's multipole in (child) and out (parent)
        "l2l": 2 * nb * m * nc * s,                                # a box's local in (parent) and out (child)
        "l2p_m2p": nt * 3 * s + nt * o * m * 8 + (nl + info["w_pairs"]) * m * nc * s,  # targets, partials, L and W
    }
    peak = float(pk.get("hbm_gbs", 6650.0))
    out = {"peak_gbs": peak, "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in pk else "fallback",
           "note": "algorithmic bytes per evaluation / the kind's CUDA-event ms; at p = 8 these passes are "
                   "FP32-bound (harmonic recurrences), not HBM-bound"}
    for k, b in bytes_.items():
        gbs = b / (kinds[k] * 1e-3) / 1e9 if kinds.get(k) else None
        out[k] = {"bytes": int(b), "gbs": round(gbs, 1) if gbs else None,
                  "frac": round(gbs / peak, 4) if gbs else None}
    return out


def log(msg):
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


def run_ours(args):
    import torch

    import fmm_b200 as F

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    n = args.n
    # weak scaling: every rank evaluates its own independent cloud (replicas of the
    # workload with different seeds); no data-path collective
    x, q = sphere_problem(n, SEED + 1000 * rank)
    sample = sample_indices(n, SAMPLE)

    def build(precision):
        # launch shapes timed at build (the results are the same bits for every shape),
        # or the ones given by --shapes
        b = F.FmmBuilder(P).gradients().max_points_per_leaf(LEAF).precision(precision).device(local)
        if args.shapes is None:
            return b.autotune().build(x)
        f = b.build(x)
        w, blk = (int(t) for t in args.shapes.split(","))
        f.set_launch_shapes(w, blk)
        return f

    log(f"problem n={n} generated")
    t0 = time.perf_counter()
    fmm = build("mixed")
    build_s = time.perf_counter() - t0
    info = fmm.info()
    log(f"built in {time.perf_counter() - t0:.2f} s: {info}")
    dev = torch.device("cuda", local)
    dq = torch.from_numpy(q).to(dev)
    dphi = torch.empty(n, dtype=torch.float64, device=dev)
    dg = torch.empty(n * 3, dtype=torch.float64, device=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    def device_steps(f, steps, warmup):
        stream = torch.cuda.ExternalStream(f.stream)  # the evaluator's own stream
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                f.evaluate_device(dq.data_ptr(), dphi.data_ptr(), dg.data_ptr())
            f.synchronize()
            total = 0.0
            for _ in range(steps):
                flush.zero_()
                s = torch.cuda.Event(enable_timing=True)
                e = torch.cuda.Event(enable_timing=True)
                s.record(stream)
                f.evaluate_device(dq.data_ptr(), dphi.data_ptr(), dg.data_ptr())
                e.record(stream)
                e.synchronize()
                total += s.elapsed_time(e)
            f.synchronize()
        return total / steps

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    # the product's repeated-evaluation mode: the whole sweep replayed from one captured
    # CUDA graph (the same kernels and floats as direct launches, one launch from the host)
    fmm.set_graph(True)
    with Clocks(local) as clk:
        ms = device_steps(fmm, args.steps, args.warmup)
    clocks = clk.summary()
    fmm.set_graph(False)
    launches_per_step = fmm.info()["launches"]  # counted by the evaluator on its last evaluation
    log(f"timed: {ms:.3f} ms/step, {launches_per_step} launches per step")
    if world > 1:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    # the same steps with every kernel launched directly from the host
    direct_ms = device_steps(fmm, args.steps, args.warmup)
    log(f"direct launches: {direct_ms:.3f} ms/step")
    if world > 1:
        t = torch.tensor([direct_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        direct_ms = float(t.item())
    # per-kind split and the dominant kernel: separate evaluations with every launch
    # bracketed by CUDA events on the evaluator's stream, L2 flushed before each; one
    # warm-up, then each kind's mean over three
    fmm.set_kind_timing(True)
    stream = torch.cuda.ExternalStream(fmm.stream)
    runs = []
    for _ in range(4):
        with torch.cuda.stream(stream):
            flush.zero_()
            fmm.evaluate_device(dq.data_ptr(), dphi.data_ptr(), dg.data_ptr())
        runs.append(fmm.kind_times())
    kinds = {n: sum(r[n] for r in runs[1:]) / 3 for n in runs[0]}
    log(f"kinds: {kinds}")
    fmm.set_kind_timing(False)
    # accuracy at sampled targets against the f64 direct sum on the GPU
    with torch.cuda.stream(stream):
        fmm.evaluate_device(dq.data_ptr(), dphi.data_ptr(), dg.data_ptr())
    fmm.synchronize()
    phi = dphi.cpu().numpy()
    grad = dg.cpu().numpy().reshape(n, 3)
    log("direct sum")
    ex_phi, ex_g = F.direct_sum(x, q, x[sample], device=local)
    log("e2e")
    err_phi = float(np.linalg.norm(phi[sample] - ex_phi) / np.linalg.norm(ex_phi))
    err_g = float(np.linalg.norm(grad[sample] - ex_g) / np.linalg.norm(ex_g))
    # e2e through the host API with pinned buffers
    hq = torch.from_numpy(q).pin_memory()
    hphi = torch.empty(n, dtype=torch.float64).pin_memory()
    hg = torch.empty(n * 3, dtype=torch.float64).pin_memory()
    fmm.set_graph(True)  # the host API in the same repeated-evaluation mode
    for _ in range(max(1, args.warmup)):
        F._check(F.lib().fmmgpu_fmm_evaluate(fmm._h, hq.data_ptr(), hphi.data_ptr(), hg.data_ptr()))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        F._check(F.lib().fmmgpu_fmm_evaluate(fmm._h, hq.data_ptr(), hphi.data_ptr(), hg.data_ptr()))
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    log(f"e2e (f64 host buffers) {e2e_ms:.3f} ms")
    # the same through the f32 host call, the reference's Fmm<f32> value type (its f32
    # runs take f32 charges and return f32 potentials and gradients): half the copies
    q32 = q.astype(np.float32)
    hq32 = torch.from_numpy(q32).pin_memory()
    hphi32 = torch.empty(n, dtype=torch.float32).pin_memory()
    hg32 = torch.empty(n * 3, dtype=torch.float32).pin_memory()
    for _ in range(max(1, args.warmup)):
        F._check(F.lib().fmmgpu_fmm_evaluate_f32(fmm._h, hq32.data_ptr(), hphi32.data_ptr(), hg32.data_ptr()))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        F._check(F.lib().fmmgpu_fmm_evaluate_f32(fmm._h, hq32.data_ptr(), hphi32.data_ptr(), hg32.data_ptr()))
    e2e32_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    fmm.close()
    log(f"e2e (f32 host buffers) {e2e32_ms:.3f} ms")
    # its error against the f64 direct sum of the charges it was given (rounded to f32)
    ex32_phi, ex32_g = F.direct_sum(x, q32.astype(np.float64), x[sample], device=local)
    phi32 = hphi32.numpy().astype(np.float64)
    g32 = hg32.numpy().astype(np.float64).reshape(n, 3)
    err32_phi = float(np.linalg.norm(phi32[sample] - ex32_phi) / np.linalg.norm(ex32_phi))
    err32_g = float(np.linalg.norm(g32[sample] - ex32_g) / np.linalg.norm(ex32_g))
    # the plain f64 evaluator on the same input, in the same graph mode
    plain = build("f64")
    plain_info = plain.info()
    plain.set_graph(True)
    plain_ms = device_steps(plain, max(2, args.steps // 2), max(1, args.warmup // 2))
    plain.set_graph(False)
    with torch.cuda.stream(torch.cuda.ExternalStream(plain.stream)):
        plain.evaluate_device(dq.data_ptr(), dphi.data_ptr(), dg.data_ptr())
    plain.synchronize()
    pphi = dphi.cpu().numpy()
    perr = float(np.linalg.norm(pphi[sample] - ex_phi) / np.linalg.norm(ex_phi))
    plain.close()

    # the metric's accuracy condition (rel-L2 <= 1e-6): each form at its smallest order
    iso = None
    if not args.no_iso and world == 1:
        try:
            iso = run_iso_accuracy(F, torch, flush, x, dq, dphi, dg, sample, ex_phi, ex_g, local)
        except Exception as e:  # reported, never fatal to the headline line
            iso = {"error": f"{type(e).__name__}: {str(e)[:200]}"}
    # the batched workload: every rank its share of the clouds (all ranks take part)
    batched = None
    if not args.no_batched:
        try:
            batched = run_batched(F, torch, dev, flush, rank, world)
        except Exception as e:  # reported, never fatal to the headline line
            batched = {"error": f"{type(e).__name__}: {str(e)[:200]}"}
    if rank != 0:
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    pk = peaks()
    sm_max = float(pk.get("sm_max_mhz", 1965.0))
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    dominant = max(kinds, key=kinds.get)
    roof = {"kind": dominant, "kernel": dominant}
    if dominant == "p2p":
        # the mixed P2P kernel: its sources from the near rows' streams when they were built
        roof["kernel"] = "p2p_st_kernel" if info.get("p2p_stream_bytes") else "p2p_x2_kernel"
        ops = info["near_pairs"] * P2P_OPS[True]
        peak = nsm * 128 * sm_max * 1e6 / 1e12
        achieved = ops / (kinds["p2p"] * 1e-3) / 1e12
        roof.update({"bound": "fp32", "achieved": round(achieved, 2), "peak": round(peak, 2),
                     "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                     "peak_source": f"derived: {nsm} SMs x 128 FP32 lanes x {sm_max:.0f} MHz "
                                    "(no FP32 peak in MEASURED_PEAKS.json)",
                     "op_model": "15 FP32 lane-ops per pair (fmm-validate/src/peaks.rs:12-17)",
                     "traffic": None})
        t = ncu_traffic(roof["kernel"])
        if t:
            roof["traffic"] = round(t["dram_bytes_per_unit"] * info["near_pairs"])
            roof["traffic_source"] = t["source"]
    elif dominant == "m2l" and "bf16_tflops" in pk:
        # the tensor-core M2L: 2 (p+1)^4 FLOP per V pair (the reference's count), against the
        # dense TF32 rate, half the measured BF16 one
        roof["kernel"] = "m2l_tc_kernel"
        flop = info["v_pairs"] * 2.0 * float((P + 1) ** 4)
        achieved = flop / (kinds["m2l"] * 1e-3) / 1e12
        peak = 0.5 * float(pk["bf16_tflops"])
        roof.update({"bound": "tensor", "achieved": round(achieved, 2), "peak": round(peak, 2), "unit": "TFLOP/s",
                     "frac": round(achieved / peak, 4), "traffic": None,
                     "peak_source": "derived: dense TF32 = half the measured BF16 burst (MEASURED_PEAKS.json)",
                     "op_model": "2 (p+1)^4 FLOP per V pair; the 3xTF32 split runs three such products"})
    else:
        roof.update({"bound": "unknown", "achieved": None, "peak": None, "unit": None, "frac": None,
                     "traffic": None})
    value = world * n / (ms * 1e-3) / 1e6
    line = {
        "metric": "Mpoints/s at rel-L2 <=1e-6 vs FP64 direct: mixed/batched vs plain FP64 GPU FMM",
        "value": round(value, 3),
        "unit": "Mpoints/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (f64 per-target accumulation)",
        "data": "synthetic (seeded SplitMix64: unit-sphere surface from normalised Gaussians, q ~ N(0,1))",
        "config": headline_config(n, world),
        "error": {"phi_rel_l2": err_phi, "grad_rel_l2": err_g, "sampled_targets": SAMPLE,
                  "against": "f64 direct sum (GPU, Neumaier)", "plain_f64_phi_rel_l2": perr},
        "plain_f64": {"ms_per_step": round(plain_ms, 4), "value": round(n / (plain_ms * 1e-3) / 1e6, 3),
                      "mixed_over_plain": round(plain_ms / ms, 3)},
        "direct_launches": {"ms_per_step": round(direct_ms, 4),
                            "value": round(world * n / (direct_ms * 1e-3) / 1e6, 3),
                            "note": "the same evaluation with every kernel launched from the host (no graph)"},
        "kinds_ms": {k: round(v, 4) for k, v in kinds.items()},
        "passes_hbm": passes_hbm(info, kinds, pk),
        "plan": {k: info[k] for k in ("nlevels", "nboxes", "nleaves", "near_pairs", "v_pairs", "w_pairs",
                                      "x_pairs", "device_bytes", "close_pairs")},
        "build_s": round(build_s, 3),
        "launch_shapes": {"p2p_warps": info["p2p_warps"], "leaf_block": info["leaf_block"],
                          "plain_f64_leaf_block": plain_info["leaf_block"],
                          "note": "timed at build (autotune); build_s includes it"},
        "e2e": {"value": round(n / (e2e32_ms * 1e-3) / 1e6, 3), "unit": "Mpoints/s",
                "ms_per_step": round(e2e32_ms, 4),
                "h2d_bytes_per_step": n * 4, "d2h_bytes_per_step": n * 4 * 4,
                "call": "fmmgpu_fmm_evaluate_f32 (the reference's Fmm<f32>: f32 charges in, f32 phi and "
                        "grad phi out, pinned host buffers, graph replay)",
                "phi_rel_l2": err32_phi, "grad_rel_l2": err32_g,
                "f64_host": {"value": round(n / (e2e_ms * 1e-3) / 1e6, 3), "ms_per_step": round(e2e_ms, 4),
                             "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8 * 4,
                             "call": "fmmgpu_fmm_evaluate (f64 charges in, f64 phi and grad phi out)"}},
        "gpu_launches": None,
        "roofline": roof,
        "clocks": clocks,
    }
    line["gpu_launches"] = launches_per_step * args.steps
    line["gpu_launches_per_step"] = launches_per_step
    if iso is not None:
        line["at_1e-6"] = iso
    if batched is not None:
        line["batched"] = batched
    if not args.no_batched and world == 1:
        for key, fn in (("helmholtz", lambda: run_helmholtz(F, torch, dev, flush)),
                        ("published_configs", lambda: run_published_configs(F, torch, dev, flush)),
                        ("adjoint", lambda: run_adjoint(F))):
            try:
                line[key] = fn()
            except Exception as e:  # reported, never fatal to the headline line
                line[key] = {"error": f"{type(e).__name__}: {str(e)[:200]}"}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
        if isinstance(line.get("helmholtz"), dict) and "mixed" in line["helmholtz"]:
            line["helmholtz"]["cpu_oracle"] = helmholtz_cpu_oracle()
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


ISO_TOL = 1e-6
ISO_ORDERS = (10, 11, 12)


def run_iso_accuracy(F, torch, flush, x, dq, dphi, dg, sample, ex_phi, ex_g, local=0):
    """The metric's accuracy condition on the headline's points (sphere, 128 per leaf,
    phi + grad): for each form, plain f64 and mixed, the smallest expansion order whose phi
    error at the sampled targets against the f64 direct sum is at most 1e-6, timed there
    like the headline (graph replays, L2 flushed); mixed_over_plain compares the two at
    their own orders.  Orders below 10 are not tried (p = 9 gives about 5e-6 here)."""
    n = len(x)
    out = {"target_phi_rel_l2": ISO_TOL, "orders_tried": list(ISO_ORDERS), "scan": []}
    for prec in ("f64", "mixed"):
        for p in ISO_ORDERS:
            t0 = time.perf_counter()
            f = F.FmmBuilder(p).gradients().max_points_per_leaf(LEAF).precision(prec).device(local).autotune().build(x)
            build_s = time.perf_counter() - t0
            stream = torch.cuda.ExternalStream(f.stream)
            with torch.cuda.stream(stream):
                f.evaluate_device(dq.data_ptr(), dphi.data_ptr(), dg.data_ptr())
            f.synchronize()
            phi = dphi.cpu().numpy()
            grad = dg.cpu().numpy().reshape(n, 3)
            ep = float(np.linalg.norm(phi[sample] - ex_phi) / np.linalg.norm(ex_phi))
            eg = float(np.linalg.norm(grad[sample] - ex_g) / np.linalg.norm(ex_g))
            row = {"precision": prec, "p": p, "phi_rel_l2": ep, "grad_rel_l2": eg, "build_s": round(build_s, 2)}
            out["scan"].append(row)
            log(f"iso-accuracy {prec} p={p}: phi {ep:.3e} grad {eg:.3e}")
            if ep <= ISO_TOL:
                ms = device_timed(f, torch, flush, dq, dphi, dg)
                row["ms_per_step"] = round(ms, 4)
                out[prec] = {"p": p, "phi_rel_l2": ep, "grad_rel_l2": eg, "ms_per_step": round(ms, 4),
                             "value": round(n / (ms * 1e-3) / 1e6, 3), "unit": "Mpoints/s",
                             "launches_per_step": f.info()["launches"]}
                f.close()
                break
            f.close()
        else:
            out[prec] = {"reached": False, "note": f"no order in {list(ISO_ORDERS)} reached {ISO_TOL}"}
    if "ms_per_step" in out["f64"] and "ms_per_step" in out["mixed"]:
        out["mixed_over_plain"] = round(out["f64"]["ms_per_step"] / out["mixed"]["ms_per_step"], 3)
    return out


def run_batched(F, torch, dev, flush, rank=0, world=1, steps=3, warmup=1):
    """The batched workload (256 clouds, 16 vectors, p = 6, 64 per leaf, potentials) as one
    forest: mixed and plain f64, device-timed like the headline, with the error of the
    first vector at sampled targets of the first clouds against the GPU f64 direct sum.
    On several ranks each rank takes its share of the clouds (fmm_b200.multigpu), the
    times are the slowest rank's and the value counts every rank's points.  Every rank
    takes the same collective steps, failures included."""
    from fmm_b200.multigpu import max_over_ranks, shard_clouds

    all_clouds, all_q, kinds = batched_problem()
    n_all = int(sum(len(c) for c in all_clouds))
    offs = np.concatenate([[0], np.cumsum([len(c) for c in all_clouds])])
    mine = shard_clouds([len(c) for c in all_clouds], world)[rank]
    clouds = [all_clouds[i] for i in mine]
    q = np.ascontiguousarray(np.concatenate([all_q[offs[i]:offs[i + 1]] for i in mine]))
    n = int(sum(len(c) for c in clouds))
    m = BATCH_VECTORS
    log(f"batched: {len(clouds)} of {len(all_clouds)} clouds, {n} of {n_all} points, {m} vectors")
    dq = torch.from_numpy(q).to(dev)
    dphi = torch.empty(m * n, dtype=torch.float64, device=dev)
    res = {"workload": f"{len(all_clouds)} clouds, N_i log-uniform in [1e4, 5e5] (cube / sphere / Plummer a=0.1 "
                       f"clipped at r=5), {m} vectors U[-1,1), p={BATCH_P}, {BATCH_LEAF} per leaf, potentials",
           "n_points": n_all, "vectors": m, "clouds_by_geometry": [int((kinds == i).sum()) for i in range(3)],
           "data": "synthetic (numpy PCG64, seeded)",
           "timing": "device: the whole evaluation replayed from one captured CUDA graph, L2 flushed before each step"}
    if world > 1:
        res["sharding"] = f"clouds dealt to {world} ranks by points (largest first), no data-path collective; " \
                          "times are the slowest rank's"

    def timed(f):
        # the whole sweep (every pass of every vector pass) replayed from one CUDA graph
        f.set_graph(True)
        stream = torch.cuda.ExternalStream(f.stream)
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                f.evaluate_device(dq.data_ptr(), dphi.data_ptr(), None)
            f.synchronize()
            total = 0.0
            for _ in range(steps):
                flush.zero_()
                s = torch.cuda.Event(enable_timing=True)
                e = torch.cuda.Event(enable_timing=True)
                s.record(stream)
                f.evaluate_device(dq.data_ptr(), dphi.data_ptr(), None)
                e.record(stream)
                e.synchronize()
                total += s.elapsed_time(e)
            f.synchronize()
        f.set_graph(False)
        return total / steps

    for precision in ("mixed", "f64"):
        t0 = time.perf_counter()
        try:
            f = (F.FmmBuilder(BATCH_P).vectors(m).max_points_per_leaf(BATCH_LEAF).precision(precision)
                 .autotune().build_batch(clouds))
            build_s = time.perf_counter() - t0
            info = f.info()
            ms = timed(f)
        except Exception as e:  # this rank failed: the others still take the collective below
            log(f"batched {precision} failed: {e}")
            f, ms = None, float("inf")
        ms = max_over_ranks(ms, dev)
        if f is None or not np.isfinite(ms):
            if f is not None:
                f.close()
            raise RuntimeError(f"batched {precision}: a rank failed")
        log(f"batched {precision}: build {build_s:.1f} s, {ms:.2f} ms/step (slowest rank)")
        if precision == "mixed":
            res.update({"ms_per_step": round(ms, 3), "value": round(n_all / (ms * 1e-3) / 1e6, 3), "unit": "Mpoints/s",
                        "point_vectors_per_s": round(n_all * m / (ms * 1e-3) / 1e6, 1), "build_s": round(build_s, 2),
                        "launches_per_step": f.info()["launches"],
                        "launch_shapes": {"p2p_warps": info["p2p_warps"], "leaf_block": info["leaf_block"]},
                        "plan": {k: info[k] for k in ("nlevels", "nboxes", "nleaves", "near_pairs", "v_pairs")}})
            # error of vector 0 at 250 sampled targets in each of this rank's first 4 clouds
            # (local work between collectives: a failure here is recorded, not raised)
            try:
                phi = dphi.view(m, n)[0].cpu().numpy()
                errs, off = [], 0
                for c in range(min(4, len(clouds))):
                    x = clouds[c]
                    pick = np.linspace(0, len(x) - 1, 250).astype(np.int64)
                    ex, _ = F.direct_sum(x, q[off:off + len(x), 0], x[pick], gradients=False)
                    errs.append(float(np.linalg.norm(phi[off + pick] - ex) / np.linalg.norm(ex)))
                    off += len(x)
                res["phi_rel_l2_first_clouds"] = errs
            except Exception as e:
                res["phi_rel_l2_first_clouds"] = f"failed: {type(e).__name__}: {str(e)[:120]}"
        else:
            res["plain_f64"] = {"ms_per_step": round(ms, 3), "value": round(n_all / (ms * 1e-3) / 1e6, 3)}
        f.close()
    res["mixed_over_plain"] = round(res["plain_f64"]["ms_per_step"] / res["ms_per_step"], 3)
    del dq, dphi
    torch.cuda.empty_cache()
    return res


def device_timed(f, torch, flush, charges, out_phi, out_grad, steps=10, warmup=3):
    """Device ms per evaluation replayed from the captured graph (L2 flushed before every
    step), the headline's timing on another problem."""
    f.set_graph(True)
    stream = torch.cuda.ExternalStream(f.stream)
    gp = out_grad.data_ptr() if out_grad is not None else None
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            f.evaluate_device(charges.data_ptr(), out_phi.data_ptr(), gp)
        f.synchronize()
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            f.evaluate_device(charges.data_ptr(), out_phi.data_ptr(), gp)
            s1.record(stream)
            s1.synchronize()
            total += s0.elapsed_time(s1)
    f.set_graph(False)
    return total / steps


def run_published_configs(F, torch, dev, flush):
    """The configurations with published device figures (an H100, the reference's CubeCL
    path; the cube workload of its own benchmark, fmm-bench/results/phase4s-gh200.md:62-64:
    N uniform in [0,1]^3, sources = targets, one charge vector, gradients on, 64 points per
    leaf; its times are the mean host call with one upload, one download and one sync):
    the same problems here (seeded numpy PCG64 in place of the reference's generator,
    charges U[-1,1)), timed both ways -- device-timed graph replays like the headline, and
    the mean wall clock of the host call (fmmgpu_fmm_evaluate_f32 for the f32 row, as the
    published run's Fmm<f32>; fmmgpu_fmm_evaluate for the f64 rows), the published figures' form --
    with the relative L2 error of phi at 1,000 sampled targets against the GPU f64 direct
    sum."""
    cases = [  # (name, N, p, points per leaf, precision, gradients, published ms, source)
        ("laplace_f64_p6_cube_1e5", 100_000, 6, 64, "f64", True, 2.544, "phase4s-gh200.md:101 (f64 p=6, 1e5)"),
        ("laplace_mixed_p8_cube_1e6", 1_000_000, 8, 64, "mixed", True, 21.67, "phase4s-gh200.md:96 (f32 p=8, 1e6)"),
        ("laplace_f64_p8_cube_1e6", 1_000_000, 8, 64, "f64", True, 35.06, "phase4s-gh200.md:107 (f64 p=8, 1e6)"),
    ]
    out = {"note": "published figures: the reference's device FMM on an H100 "
                   "(fmm-bench/results/phase4s-gh200.md); ours on one B200"}
    for name, n, p, leaf, prec, grad, pub_ms, src in cases:
        rng = np.random.default_rng(SEED + n + p)
        x = rng.uniform(0.0, 1.0, (n, 3))
        q = rng.uniform(-1.0, 1.0, n)
        b = F.FmmBuilder(p).max_points_per_leaf(leaf).precision(prec).autotune()
        if grad:
            b = b.gradients()
        f = b.build(x)
        dq = torch.from_numpy(q).to(dev)
        dphi = torch.empty(n, dtype=torch.float64, device=dev)
        dg = torch.empty(3 * n, dtype=torch.float64, device=dev) if grad else None
        ms = device_timed(f, torch, flush, dq, dphi, dg)
        phi = dphi.cpu().numpy()
        f.set_graph(True)
        # the host call in the published run's value type: f32 for its f32 rows (the mixed
        # form here, fmmgpu_fmm_evaluate_f32), f64 otherwise
        qh = q.astype(np.float32) if prec == "mixed" else q
        for _ in range(3):
            f.evaluate(qh)
        t0 = time.perf_counter()
        for _ in range(10):
            f.evaluate(qh)
        host_ms = (time.perf_counter() - t0) * 100.0
        pick = np.random.default_rng(SEED).choice(n, 1000, replace=False)
        ex, _ = F.direct_sum(x, q, x[pick], gradients=False)
        err = float(np.linalg.norm(phi[pick] - ex) / np.linalg.norm(ex))
        out[name] = {"n": n, "p": p, "leaf": leaf, "precision": prec, "gradients": grad,
                     "device_ms": round(ms, 4), "host_call_ms": round(host_ms, 4),
                     "host_call_value_type": str(qh.dtype),
                     "mpoints_per_s": round(n / (host_ms * 1e-3) / 1e6, 2), "phi_rel_l2": err,
                     "published_ms": pub_ms, "published_source": src,
                     "host_call_speedup_vs_published": round(pub_ms / host_ms, 2)}
        f.close()
        del dq, dphi, dg
    torch.cuda.empty_cache()
    return out


def run_adjoint(F, n=1_000_000, reps=2):
    """The differentiated form: N points from 32 isotropic Gaussians (centres uniform in the
    unit cube, sigma log-uniform in [0.005, 0.05]), charges N(0,1), p = 8, loss
    L = 1/2 sum q_i phi_i.  The VJP of the potentials with cotangent q / 2 gives
    dL/dq = phi / 2 + dq and dL/dx = dsources + dtargets (sources = targets); timed through
    the host call fmmgpu_fmm_vjp (copies included), checked at 1,000 sampled points against
    the GPU f64 direct sum's potentials and forces q_i grad phi(x_i)."""
    rng = np.random.default_rng(SEED + 5)
    cen = rng.uniform(0.0, 1.0, (32, 3))
    sig = np.exp(rng.uniform(np.log(0.005), np.log(0.05), 32))
    lab = rng.integers(0, 32, n)
    x = cen[lab] + rng.standard_normal((n, 3)) * sig[lab, None]
    q = rng.standard_normal(n)
    pick = np.random.default_rng(SEED + 6).choice(n, 1000, replace=False)
    ex_phi, ex_g = F.direct_sum(x, q, x[pick], gradients=True)
    # f64 central differences of the exact energy on 64 random coordinates (point i, axis k):
    # moving point i changes L by q_i (phi_i(x_i + eps e_k) - phi_i(x_i - eps e_k)), phi_i
    # the potential of the other charges; the point's own term q_i / (4 pi eps) is the same
    # at both ends and cancels in the difference, so the direct sum over every source serves
    fd_rng = np.random.default_rng(SEED + 8)
    fd_i = fd_rng.choice(n, 64, replace=False)
    fd_k = fd_rng.integers(0, 3, 64)
    def central_difference(eps):
        shift = np.zeros((64, 3))
        shift[np.arange(64), fd_k] = eps
        ph_p, _ = F.direct_sum(x, q, x[fd_i] + shift, gradients=False)
        ph_m, _ = F.direct_sum(x, q, x[fd_i] - shift, gradients=False)
        return q[fd_i] * (ph_p - ph_m) / (2 * eps)

    fd = central_difference(1e-4)  # the configuration's step
    fd_fine = central_difference(1e-6)  # a step well below the clusters' point spacing
    _, g_at = F.direct_sum(x, q, x[fd_i], gradients=True)
    exact = q[fd_i] * g_at[np.arange(64), fd_k]  # dL/dx from the direct sum's gradient

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out = {"workload": f"N={n} from 32 Gaussians, p=8, 64 per leaf, L = 1/2 sum q phi; dL/dq and dL/dx",
           "fd_check": "dL/dx at 64 random coordinates against f64 central differences of the exact energy "
                       "(eps = 1e-4, the configuration's, whose own truncation error the clusters' point spacing "
                       "makes visible, and eps = 1e-6) and against the direct sum's gradient; dL/dq and dL/dx "
                       "against the f64 direct sum at 1,000 points",
           "data": "synthetic (numpy PCG64, seeded)", "timing": "wall clock of the host call fmmgpu_fmm_vjp, "
                                                             "copies included; best of the timed calls"}
    for prec in ("mixed", "f64"):
        f = F.FmmBuilder(8).gradients().max_points_per_leaf(64).precision(prec).build(x)
        phi = f.evaluate(q).potential[0]
        f.vjp(q, 0.5 * q)  # warm
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            dq, dxs, dxt = f.vjp(q, 0.5 * q)
            best = min(best, time.perf_counter() - t0)
        dldq = 0.5 * phi + dq[:, 0]
        dldx = dxs + dxt
        forces = q[pick, None] * ex_g
        fd_got = dldx[fd_i, fd_k]
        out[prec] = {"ms": round(best * 1e3, 3), "mpoints_per_s": round(n / best / 1e6, 3),
                     "dldq_rel_l2": float(np.linalg.norm(dldq[pick] - ex_phi) / np.linalg.norm(ex_phi)),
                     "dldx_rel_l2": float(np.linalg.norm(dldx[pick] - forces) / np.linalg.norm(forces)),
                     "fd_64_coordinates": {"vjp_vs_fd_eps1e-4": rel(fd_got, fd), "vjp_vs_fd_eps1e-6": rel(fd_got, fd_fine),
                                           "vjp_vs_direct_gradient": rel(fd_got, exact),
                                           "fd_eps1e-4_vs_direct_gradient": rel(fd, exact),
                                           "fd_eps1e-6_vs_direct_gradient": rel(fd_fine, exact)}}
        f.close()
    return out


def run_helmholtz(F, torch, dev, flush, n=1_000_000, k=20.0, p=10, leaf=96, steps=5, warmup=2):
    """The Helmholtz configuration: N points uniform in the unit cube, k = 20 (about 3.2
    wavelengths across), complex charges N(0,1) + i N(0,1), p = 10 on every level, 96 points
    per leaf, potential and gradient of e^{ikr}/(4 pi r).  The whole FMM (near and far
    field) in f64 and in the mixed form: device time per evaluation (graph-free launches on
    the evaluator's stream, L2 flushed before every step, CUDA events), the host call with
    pinned buffers and the copies (best of four; complex64 for the mixed form, complex128
    for f64), the tables' host build time for the new k, and the relative
    L2 error of phi and grad at 1,000 sampled targets against the f64 direct sum (GPU,
    Neumaier, complex128); the near field alone (P2P) is timed beside it."""
    rng = np.random.default_rng(SEED + 11)
    x = rng.uniform(0.0, 1.0, (n, 3))
    q = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    pick = rng.choice(n, 1000, replace=False)
    ex, eg = F.helmholtz_direct_sum(k, x, q, x[pick])
    dq = torch.from_numpy(np.ascontiguousarray(q.view(np.float64))).to(dev)
    dphi = torch.empty(2 * n, dtype=torch.float64, device=dev)
    dg = torch.empty(6 * n, dtype=torch.float64, device=dev)
    res = {"workload": f"Helmholtz FMM, N={n} uniform in the unit cube, k={k}, p={p} on every level, {leaf} per leaf, "
                       "phi+grad, complex charges N(0,1)+iN(0,1)",
           "data": "synthetic (numpy PCG64, seeded)", "unit": "Mpoints/s",
           "timing": "device: CUDA events on the evaluator's stream, L2 flushed before each step; "
                     "host_call: the host call with pinned buffers and the copies, best of 4 (mixed: "
                     "fmmgpu_helmholtz_evaluate_f32, complex64 in and out; f64: fmmgpu_helmholtz_evaluate, "
                     "complex128)"}
    for prec in ("f64", "mixed"):
        t0 = time.perf_counter()
        f = F.FmmBuilder(p).gradients().max_points_per_leaf(leaf).precision(prec).build(x)
        build_s = time.perf_counter() - t0
        info = f.info()
        out = f.helmholtz_evaluate(k, q)  # builds the tables of this k
        table_s = f.helmholtz_table_seconds()
        stream = torch.cuda.ExternalStream(f.stream)
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                f.helmholtz_evaluate_device(k, dq.data_ptr(), dphi.data_ptr(), dg.data_ptr())
            total = 0.0
            for _ in range(steps):
                flush.zero_()
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s0.record(stream)
                f.helmholtz_evaluate_device(k, dq.data_ptr(), dphi.data_ptr(), dg.data_ptr())
                s1.record(stream)
                s1.synchronize()
                total += s0.elapsed_time(s1)
        ms = total / steps
        # the host call with pinned buffers, in the value type of the form: complex64 for
        # the mixed one (fmmgpu_helmholtz_evaluate_f32), complex128 for f64
        ct = torch.complex64 if prec == "mixed" else torch.complex128
        hq = torch.from_numpy(q.astype(np.complex64 if prec == "mixed" else np.complex128)).pin_memory()
        hphi = torch.empty(n, dtype=ct).pin_memory()
        hg = torch.empty(3 * n, dtype=ct).pin_memory()
        call = F.lib().fmmgpu_helmholtz_evaluate_f32 if prec == "mixed" else F.lib().fmmgpu_helmholtz_evaluate
        best = float("inf")
        for _ in range(4):
            t0 = time.perf_counter()
            F._check(call(f._h, float(k), 0.0, hq.data_ptr(), hphi.data_ptr(), hg.data_ptr()))
            best = min(best, time.perf_counter() - t0)
        hbytes = (hq.numel() + hphi.numel() + hg.numel()) * hq.element_size()
        ephi_h = float(np.linalg.norm(hphi.numpy().astype(np.complex128)[pick] - ex) / np.linalg.norm(ex))
        del hq, hphi, hg
        near = float("inf")
        for _ in range(2):
            t0 = time.perf_counter()
            f.helmholtz_near(k, q)
            near = min(near, time.perf_counter() - t0)
        ep = float(np.linalg.norm(out.potential[0][pick] - ex) / np.linalg.norm(ex))
        egr = float(np.linalg.norm(out.gradient[0][pick] - eg) / np.linalg.norm(eg))
        res[prec] = {"ms_per_step": round(ms, 3), "value": round(n / (ms * 1e-3) / 1e6, 3),
                     "host_call_ms": round(best * 1e3, 3), "e2e_value": round(n / best / 1e6, 3),
                     "host_call": {"value_type": str(ct).replace("torch.", ""), "copied_bytes": hbytes,
                                   "phi_rel_l2": ephi_h},
                     "phi_rel_l2": ep, "grad_rel_l2": egr, "build_s": round(build_s, 2),
                     "tables_s": round(table_s, 2), "nlevels": info["nlevels"], "v_pairs": info["v_pairs"],
                     "near_field_host_call_ms": round(near * 1e3, 3), "near_pairs": info["near_pairs"]}
        log(f"helmholtz {prec}: {ms:.2f} ms device, {best * 1e3:.1f} ms host call, phi {ep:.2e} grad {egr:.2e}")
        f.close()
    res["mixed_over_plain"] = round(res["f64"]["ms_per_step"] / res["mixed"]["ms_per_step"], 3)
    del dq, dphi, dg
    torch.cuda.empty_cache()
    return res


def helmholtz_cpu_oracle(n=5000, k=20.0, p=10, leaf=96):
    """The oracle's Helmholtz FMM (oracle/oracle.py helmholtz_fmm: per-box Python loops over the
    C operators of oracle/helmholtz_ops.c) timed on a bounded sample of the Helmholtz
    configuration: the test restatement of the reference's host-only Helmholtz path, reported
    beside the device numbers as the reference arm of this leg; it is not the reference's own
    host speed (its Rust operator cannot be built here)."""
    from oracle import oracle as O

    rng = np.random.default_rng(SEED + 13)
    x = rng.uniform(0.0, 1.0, (n, 3))
    q = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    t0 = time.perf_counter()
    O.helmholtz_fmm(x, q, x, k, p, leaf)
    s = time.perf_counter() - t0
    return {"value": round(n / s / 1e6, 6), "unit": "Mpoints/s", "seconds": round(s, 2), "cores": 1,
            "kind": "oracle", "sample": f"N={n} uniform in the unit cube, k={k}, p={p}, {leaf} per leaf, phi+grad, "
                                        "one evaluation (tables built inside it)",
            "note": "the oracle's Python-driven Helmholtz FMM: a checker, far slower than the reference's "
                    "host operator; the ratio to it says nothing about the kernels"}


CPU_REPEATS = 5
HOST_PATH = ("restated reference host path (LaplaceOperator with nd-fmm-simd on AVX-512F: P2P with vrsqrt14pd + "
             "two Newton steps, targets in lanes, 16 a block; batched M2L in blocks of 64 targets, 4 columns a "
             "pass; lists made at build), OpenMP over the host cores")
HOST_PATH_SCALAR = "restated reference host path without AVX-512F on this CPU: its scalar P2P, batched M2L"


def cpu_baseline(args, n_sample=None, repeats=CPU_REPEATS, warmup=1):
    """The restated reference host path (oracle/hostpath.c: its AVX-512 P2P and batched M2L,
    OpenMP over all host cores) on the headline workload (the same sphere problem,
    n_sample points), built once (plan and f64 tables, reported beside), then `warmup`
    untimed and `repeats` timed evaluations; the value is N over the median evaluation
    time, as the metric defines it (fmm-bench/src/measure.rs: build and tables excluded)."""
    from oracle import oracle as O

    n = n_sample or args.cpu_n
    x, q = sphere_problem(n, SEED)
    cores = os.cpu_count()
    t0 = time.perf_counter()
    f = O.Fmm(x, x, P, LEAF, gradients=True, host_path=True)
    build_s = time.perf_counter() - t0
    for _ in range(warmup):
        f.evaluate(q, threads=cores)
    times = []
    for _ in range(repeats):
        f.evaluate(q, threads=cores)
        times.append(O.fmm_last_eval_seconds())
    med = float(np.median(times))
    return {"value": round(n / med / 1e6, 4), "unit": "Mpoints/s", "cores": cores, "kind": "port",
            "path": HOST_PATH if O.lib().orc_hp_has_avx512() else HOST_PATH_SCALAR,
            "sample": f"sphere N={n} p={P} leaf={LEAF} phi+grad f64: median of {repeats} evaluations after "
                      f"{warmup} warm-up ({med:.2f} s each; plan, lists and tables built once in {build_s:.1f} s)",
            "evaluations_s": [round(v, 3) for v in times], "n_points": n}


def headline_config(n, world):
    """The workload both arms report (the reference arm times bounded samples of it)."""
    return {"workload": f"laplace3d sphere N={n} p={P} leaf={LEAF} phi+grad mixed",
            "n_points": n, "p": P, "max_points_per_leaf": LEAF, "gradients": True,
            "precision": "mixed", "l2": "flushed (512 MiB write) before every timed step",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"}


def run_reference(args):
    """The reference arm: the restated reference host path (oracle/hostpath.c) on the host cores, at
    the headline's own N (--ref-n, default the headline's): built once, --warmup untimed
    evaluations, then --steps timed evaluations; the value is N over the median step.
    Under torchrun only rank 0 runs it."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O

    n = args.ref_n or args.n
    x, q = sphere_problem(n, SEED)
    cores = os.cpu_count()
    t0 = time.perf_counter()
    f = O.Fmm(x, x, P, LEAF, gradients=True, host_path=True)
    build_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        f.evaluate(q, threads=cores)
    times = []
    for _ in range(args.steps):
        f.evaluate(q, threads=cores)
        times.append(O.fmm_last_eval_seconds())
    med = float(np.median(times))
    v = round(n / med / 1e6, 4)
    cfg = headline_config(n, 1)  # the workload ours runs (at the N timed here); computed in f64 (dtype)
    print(json.dumps({
        "impl": "reference",
        "metric": "Mpoints/s at rel-L2 <=1e-6 vs FP64 direct: mixed/batched vs plain FP64 GPU FMM",
        "value": v, "unit": "Mpoints/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(med * 1e3, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded SplitMix64 sphere)",
        "config": cfg,
        "cpu_baseline": {"value": v, "unit": "Mpoints/s", "cores": cores, "kind": "port",
                         "path": HOST_PATH if O.lib().orc_hp_has_avx512() else HOST_PATH_SCALAR,
                         "sample": f"the whole workload (N={n}) every step: one host evaluation; median of "
                                   f"{args.steps} after {args.warmup} warm-up; plan and tables built once "
                                   f"({build_s:.1f} s, not timed)"},
        "e2e": {"value": v, "unit": "Mpoints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    global P
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--cpu-n", type=int, default=N_DEFAULT, help="points of the CPU baseline's sample")
    ap.add_argument("--ref-n", type=int, default=0, help="points of the reference arm (default: --n)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched (256 clouds) measurement")
    ap.add_argument("--no-iso", action="store_true", help="skip the iso-accuracy (rel-L2 <= 1e-6) measurement")
    ap.add_argument("--p", type=int, default=P, help="expansion order of the headline workload (profiling runs)")
    ap.add_argument("--helmholtz-only", action="store_true",
                    help="run the Helmholtz configuration alone (--hn points) and print its JSON")
    ap.add_argument("--hn", type=int, default=1_000_000, help="points of the Helmholtz configuration")
    ap.add_argument("--shapes", default=None,
                    help="P2P warps,L2P/M2P threads (e.g. 1,128): set instead of timed at build "
                         "(profiler runs, whose serialised launches would mislead the timing)")
    args = ap.parse_args()
    P = args.p
    if args.helmholtz_only:
        import torch

        import fmm_b200 as F

        dev = torch.device("cuda", 0)
        flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        print(json.dumps(run_helmholtz(F, torch, dev, flush, n=args.hn, steps=args.steps, warmup=args.warmup)),
              flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
