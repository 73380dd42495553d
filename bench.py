"""Benchmark: closed-shell CCSD iterations per second on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload h2o6_vtz] [--method ccsd|dcsd]

A step is one FP64 CCSD iteration (T1-dressing, residual, Hylleraas energy,
amplitude update, DIIS, energy) of (H2O)_6/cc-pVTZ (o=24, v=318, nQ=846; the
largest single-GPU configuration): the water hexamer from the seeded cluster
generator, DF-HF (cc-pVTZ-JKFIT) and the frozen-core cc-pVTZ-RI integrals from
the library's GPU integral engine, prepared before any timing
(``--synthetic`` uses seeded synthetic factors of the same shape instead).
Inputs stay in HBM (T2 466 MB, B 792 MB: larger than the 126 MB L2, which is
also flushed between steps); steps are timed with CUDA events on the
library's stream.  The line also carries:

* ``e2e``: the same iterations through the C ABI with pinned host amplitudes
  (host-to-device and device-to-host copies inside the timed region);
* ``mixed``: CCSD(T) time-to-solution from the MP2 guess, all-FP64 against
  split-BF16 tensor-core products with FP64 refinement, and the energy
  difference in microhartree;
* ``rooflines``: the FP64 DMMA GEMM (against cuBLAS DGEMM measured in the same
  run), the tcgen05 GEMM (against the measured sustained BF16 peak) and the
  (T) energy kernel (against the measured HBM bandwidth), each from CUDA
  events around its launches;
* ``cpu_baseline``: the density-fitted numpy restatement of the reference
  algorithm (oracle/dfcc.py) on the host cores, sampled.

With N > 1 each rank runs an independent replica (the path runs on one GPU;
no data-path collective) and the slowest rank's time is reported.

``--impl reference`` times that CPU restatement (ElemCo.jl itself needs Julia,
absent here) on the host cores: its K timed steps execute exactly one CCSD
iteration of the same workload, split into K consecutive parts.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "elemco.jl_b200"))

import numpy as np  # noqa: E402


def algorithmic_flops(no, nv, nq, dc=False):
    """Per CCSD iteration: ladder 2o^2v^4 + DF rebuild 2nQv^4 + ring 16o^3v^3
    (8 for DCSD) + 4o^4v^2."""
    o, v = float(no), float(nv)
    ring = 8.0 if dc else 16.0
    return 2 * o**2 * v**4 + 2 * nq * v**4 + ring * o**3 * v**3 + 4 * o**4 * v**2


def max_over_ranks(x, dist=None, device="cuda"):
    """The largest of the ranks' values of x (every rank gets it); x itself
    when there is one process.  Replicas time their own steps and the job's
    time is the slowest rank's."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="h2o6_vtz")
    p.add_argument("--synthetic", action="store_true",
                   help="seeded synthetic DF factors of the workload's shape instead of the "
                        "molecule's integrals")
    p.add_argument("--method", default="ccsd", choices=["ccsd", "dcsd"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--cpu-sample", type=int, default=1,
                   help="ladder a-blocks timed in the CPU baseline (0: no CPU baseline)")
    p.add_argument("--tts", action="store_true",
                   help="CCSD(T) time-to-solution, FP64 vs mixed, on --workload (one line)")
    p.add_argument("--gradient", action="store_true",
                   help="analytic dE/dlambda (Lambda rrule) vs finite differences, FP64 and "
                        "mixed, on --workload (one line)")
    p.add_argument("--sweep", action="store_true",
                   help="DCSD time per iteration and device memory, FP64 vs mixed, over the "
                        "C6..C10 alkane sizes (one line)")
    p.add_argument("--tune", default="",
                   help="tune every GEMM shape during the warm-up and write the table here")
    p.add_argument("--occ", type=int, default=0,
                   help="--tts only: override the occupied count (smaller profiling cases)")
    return p.parse_args()


# ---------------------------------------------------------------- clocks


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------- CPU side


def load_workload(name, synthetic, ctx=None):
    """(B, h1, e0, no, description) of the workload: the molecule's integrals
    from the GPU integral engine (DF-HF + dfdump), or synthetic factors."""
    from ecgpu.synthetic import make_workload
    if synthetic:
        B, h1, e0, no = make_workload(name)
        return B, h1, e0, no, "seeded synthetic DF factors, canonical HF reference"
    import ecgpu
    from ecgpu.molecular import molecular_workload
    own = ctx is None
    c = ecgpu.Context(0) if own else ctx
    try:
        B, h1, e0, no, info = molecular_workload(c, name)
    finally:
        if own:
            c.close()
    desc = (f"{info['molecule']} from the seeded geometry generator: DF-HF {info['ao']}/"
            f"{info['jkfit']} (E_HF {info['E_HF']:.8f}, {info['scf_iterations']} iterations), "
            f"frozen-core {info['mpfit']} integrals, on the library's GPU integral engine")
    return B, h1, e0, no, desc


def _df_state(wl, dc, nsteps=20):
    """The DF CPU restatement (oracle/dfcc.py) of the workload (B, h1, e0, no),
    started from MP2 amplitudes; the ladder is cut into about 2*nsteps a-blocks."""
    from oracle.dfcc import DFCC
    B, h1, e0, no = wl[:4]
    nv = B.shape[0] - no
    d = DFCC(B, h1, e0, no, dc=dc, ablock=max(1, nv // (2 * max(nsteps, 1))))
    d.start()
    return d


def cpu_baseline_sample(wl, dc, nblocks=1, ntrip=4):
    """CPU iterations/s of the DF restatement: every task of one CCSD iteration
    except the ladder runs once, the ladder on `nblocks` of its a-blocks; the
    iteration time is the non-ladder time plus the ladder blocks' mean time
    times their number (the blocks are alike).  Also (T) TFLOP/s on `ntrip`
    triplets."""
    import oracle as O
    d = _df_state(wl, dc)
    t_other, t_lad, nlad, nrun = 0.0, 0.0, 0, 0
    for name, _, fn in d.iteration_tasks():
        if name.startswith("ladder"):
            nlad += 1
            if nrun >= nblocks:
                continue
            t0 = time.perf_counter()
            fn()
            t_lad += time.perf_counter() - t0
            nrun += 1
        else:
            t0 = time.perf_counter()
            fn()
            t_other += time.perf_counter() - t0
    t_iter = t_other + t_lad / nrun * nlad
    trip = list(O.ccref._triplets(d.no))
    pick = [trip[(i * len(trip)) // ntrip] for i in range(ntrip)]
    for x in {q for t in pick for q in t[:3]}:
        d.vvvo_k(x)  # the same work pert_t does per distinct occupied index
    t0 = time.perf_counter()
    d.pert_t(d.T1, d.T2, pick)
    t_t = time.perf_counter() - t0
    ft = ntrip * (12.0 * d.nv**4 + 12.0 * d.no * d.nv**3)
    return {"iter_s": t_iter, "sampled_s": t_other + t_lad, "ladder_blocks": nlad,
            "ladder_blocks_run": nrun, "pert_t_tflops": ft / t_t / 1e12, "pert_t_s": t_t,
            "triplets": ntrip}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _chunks(tasks, k):
    """Split the task list into k consecutive parts of about equal flops."""
    total = sum(w for _, w, _ in tasks)
    out, cur, acc, c = [], [], 0.0, 0
    for i, t in enumerate(tasks):
        cur.append(t)
        acc += t[1]
        left_tasks, left_chunks = len(tasks) - i - 1, k - len(out) - 1
        if left_chunks > 0 and (acc >= total * (len(out) + 1) / k or left_tasks == left_chunks):
            out.append(cur)
            cur = []
    out.append(cur)
    while len(out) < k:
        out.append([])
    return out


# ---------------------------------------------------------------- main


def run_reference(a, wl):
    """The reference arm: the DF numpy restatement of the reference algorithm
    on the host cores.  The K timed steps run exactly one CCSD iteration (its
    tasks in order, split into K parts of about equal flops), so the value is
    1 / (time of the K steps) iterations per second; the W warm-up steps run
    the first W parts of a preceding iteration."""
    no, nv, nq = wl
    W = load_workload(a.workload, a.synthetic)
    d = _df_state(W, a.method == "dcsd", a.steps)
    tasks = d.iteration_tasks()
    K = max(1, a.steps)
    parts = _chunks(tasks, K)
    for p_ in parts[:a.warmup]:
        for _, _, fn in p_:
            fn()
    d.start(d.T1, d.T2)  # the timed iteration starts from the current amplitudes
    parts = _chunks(d._tasks, K)
    ms = []
    for p_ in parts:
        t0 = time.perf_counter()
        for _, _, fn in p_:
            fn()
        ms.append((time.perf_counter() - t0) * 1000.0)
    total = sum(ms) / 1000.0
    rate = 1.0 / total
    cores = host_cores()
    sample = (f"one CCSD iteration ({total:.1f} s) of the workload in {K} steps of about "
              "equal flops, density-fitted numpy restatement of the reference algorithm "
              "(oracle/dfcc.py), BLAS threads = all host cores")
    line = {
        "impl": "reference", "metric": "CCSD iter/s", "value": rate, "unit": "iter/s",
        "n_gpus": a.gpus, "steps": K, "warmup": a.warmup, "ms_per_step": sum(ms) / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic" if a.synthetic else "real molecule (seeded geometry)",
        "config": {"workload": f"{a.workload} {a.method.upper()} (o={no}, v={nv}, nQ={nq}): "
                               f"{W[4]}"},
        "cpu_baseline": {"value": rate, "unit": "iter/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": "iter/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


COOLDOWN_S = 20.0


def run_tts(a):
    """CCSD(T) from the MP2 guess to the (T) energy, FP64 and mixed precision,
    timed with CUDA events on the library's stream (one JSON line)."""
    import torch
    import ecgpu
    from ecgpu.synthetic import WORKLOADS, make_workload
    no, nv, nq = WORKLOADS[a.workload]
    B, h1, e0, no = make_workload(a.workload, no=a.occ or None)
    ntrip = sum(1 for k in range(no) for j in range(k + 1) for i in range(j + 1)
                if not (i == j == k))
    ft = ntrip * (12.0 * nv**4 + 12.0 * no * nv**3)
    fcc = algorithmic_flops(no, nv, nq)
    out = {}
    with ecgpu.Context(0) as ctx:
        ctx.set_system(B, h1, e0, no)
        stream = torch.cuda.ExternalStream(ctx.stream())
        _, T1, T2 = ctx.mp2()
        for prec, name in ((ecgpu.ECG_PREC_FP64, "fp64"), (ecgpu.ECG_PREC_MIXED, "mixed")):
            if name == "mixed":
                # idle before the second leg, so that it does not start on a GPU
                # that the first one left power-capped (outside the timed region)
                time.sleep(COOLDOWN_S)
            ctx.set_precision(prec)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            torch.cuda.synchronize()
            clocks = Clocks(0)
            clocks.start()
            ev[0].record(stream)
            r = ctx.cc_solve(T1, T2)
            ev[1].record(stream)
            et, etb = ctx.pert_t()  # the converged amplitudes the context holds
            ev[2].record(stream)
            torch.cuda.synchronize()
            clk = clocks.stop()
            tcc = ev[0].elapsed_time(ev[1]) / 1000.0
            tt = ev[1].elapsed_time(ev[2]) / 1000.0
            out[name] = {"ccsd_s": tcc, "pert_t_s": tt, "total_s": tcc + tt, "clocks": clk,
                         "iterations": r["iterations"], "E_ccsd": r["E"], "E_T": et,
                         "ccsd_tflops_per_iter": fcc * r["iterations"] / tcc / 1e12,
                         "pert_t_tflops": ft / tt / 1e12}
    f64, mx = out["fp64"], out["mixed"]
    line = {"metric": "CCSD(T) time-to-solution",
            "workload": a.workload + (f" with o={no}" if a.occ else ""),
            "shape": {"o": no, "v": nv, "nQ": nq}, "unit": "s", "fp64": f64, "mixed": mx,
            "speedup": f64["total_s"] / mx["total_s"],
            "dE_uEh": abs((mx["E_ccsd"] + mx["E_T"]) - (f64["E_ccsd"] + f64["E_T"])) * 1e6,
            "dE_T_uEh": abs(mx["E_T"] - f64["E_T"]) * 1e6,
            "order": f"fp64, {COOLDOWN_S:.0f} s idle, mixed",
            "data": "synthetic DF factors (see ecgpu/synthetic.py)"}
    print(json.dumps(line), flush=True)


def run_gradient(a):
    """dE/dlambda for h + lambda P through the Lambda-equation rrule, against
    the fourth-order central difference (step 1e-3) of converged energies,
    in FP64 and mixed precision (one JSON line).  P: seeded random symmetric
    MO-basis one-electron operator standing in for a dipole component."""
    import torch
    import ecgpu
    from ecgpu.driver import ECInfo, FDump, rrule_cc_energy
    from ecgpu.synthetic import make_workload
    B, h, e0, no = make_workload(a.workload, no=a.occ or None)
    rng = np.random.default_rng(11)
    P = rng.standard_normal(h.shape)
    P = 0.5 * (P + P.T)
    P /= np.linalg.norm(P, 2)  # unit spectral norm, a field-like strength
    tight = dict(thr=1e-14, conven=1.0, maxit=200)
    dc = a.method == "dcsd"
    out = {}
    for prec in ("fp64", "mixed"):
        EC = ECInfo()
        EC.fd = FDump(h, e0, 2 * no, B=B)
        EC.set("cc", **tight)
        EC.set("gpu", precision=prec)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E, pullback = rrule_cc_energy(EC, a.method)
        torch.cuda.synchronize()
        t_an = time.perf_counter() - t0
        analytic = float(np.sum(pullback(1.0) * P))
        ctx = EC.context()
        ctx.set_precision(ecgpu.ECG_PREC_MIXED if prec == "mixed" else ecgpu.ECG_PREC_FP64)
        d = 1e-3
        Es = {}
        for k in (-2, -1, 1, 2):
            ctx.set_system(B, h + k * d * P, e0, no)
            _, _, ehf = ctx.fock()
            _, T1, T2 = ctx.mp2()
            r = ctx.cc_solve(T1, T2, dc=dc, opts=ctx.opts(**tight))
            Es[k] = ehf + r["E"]
        fd = (Es[-2] - 8 * Es[-1] + 8 * Es[1] - Es[2]) / (12 * d)
        out[prec] = {"E": E, "dE_dlambda": analytic, "fd4": fd, "abs_err": abs(analytic - fd),
                     "rrule_s": t_an}
        EC.context().close()
    line = {"metric": "CC energy gradient via Lambda rrule", "workload": a.workload,
            "method": a.method, "shape": {"o": no, "v": B.shape[0] - no, "nQ": B.shape[2]},
            "fp64": out["fp64"], "mixed": out["mixed"],
            "mixed_vs_fp64_dE_dlambda": abs(out["mixed"]["dE_dlambda"] - out["fp64"]["dE_dlambda"]),
            "mixed_vs_fp64_E_uEh": abs(out["mixed"]["E"] - out["fp64"]["E"]) * 1e6,
            "perturbation": "seeded random symmetric MO one-electron operator of unit spectral "
                            "norm, FD step 1e-3",
            "data": "synthetic DF factors (see ecgpu/synthetic.py)"}
    print(json.dumps(line), flush=True)


def run_sweep(a):
    """DCSD time per iteration (CUDA events on the library stream, mean of
    a.steps after a.warmup) and device memory in use, FP64 vs mixed, for the
    C6H14..C10H22/cc-pVDZ sizes (one JSON line)."""
    import torch
    import ecgpu
    from ecgpu.synthetic import WORKLOADS, make_workload
    rows = []
    for name in ("c6h14_vdz", "c7h16_vdz", "c8h18_vdz", "c9h20_vdz", "c10h22_vdz"):
        no, nv, nq = WORKLOADS[name]
        B, h1, e0, no = make_workload(name)
        row = {"workload": name, "o": no, "v": nv, "nQ": nq}
        for prec, pname in ((ecgpu.ECG_PREC_FP64, "fp64"), (ecgpu.ECG_PREC_MIXED, "mixed")):
            torch.cuda.synchronize()
            free0, _ = torch.cuda.mem_get_info()
            with ecgpu.Context(0) as ctx:
                ctx.set_precision(prec)
                ctx.set_system(B, h1, e0, no)
                _, T1, T2 = ctx.mp2()
                stream = torch.cuda.ExternalStream(ctx.stream())
                ctx.cc_load(T1, T2)
                for _ in range(a.warmup):
                    ctx.cc_step(dc=True)
                ctx.cc_load(T1, T2)
                torch.cuda.synchronize()
                e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                e[0].record(stream)
                for _ in range(a.steps):
                    ctx.cc_step(dc=True)
                e[1].record(stream)
                torch.cuda.synchronize()
                free1, _ = torch.cuda.mem_get_info()
                row[pname] = {"ms_per_iter": e[0].elapsed_time(e[1]) / a.steps,
                              "device_mem_gb": (free0 - free1) / 1e9,
                              "algorithmic_tflops": algorithmic_flops(no, nv, nq, dc=True)
                              * a.steps
                              / (e[0].elapsed_time(e[1]) / 1000.0) / 1e12}
        row["speedup"] = row["fp64"]["ms_per_iter"] / row["mixed"]["ms_per_iter"]
        rows.append(row)
    line = {"metric": "DCSD time per iteration, FP64 vs mixed, alkane size sweep",
            "unit": "ms/iter", "steps": a.steps, "warmup": a.warmup, "rows": rows,
            "note": "v^3 o intermediates are never formed: the ladder is built per a-block "
                    "from B^Q_ab",
            "data": "synthetic DF factors (see ecgpu/synthetic.py)"}
    print(json.dumps(line), flush=True)


# GEMM tuning table for B200 written by `bench.py --tune` (ecg_tune_save)
TUNE_TABLE = os.path.join(ROOT, "elemco.jl_b200", "ecgpu", "tuning", "b200.txt")


def measured_peaks():
    """HBM GB/s, burst and sustained dense BF16 TFLOP/s: MEASURED_PEAKS.json
    (written per pod by the benchmark driver), else the pool's earlier
    measurement (6650 GB/s, 1590 / 1400 TFLOP/s)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            m = json.load(f)
        return {"hbm_gbs": float(m["hbm_gbs"]), "bf16": float(m["bf16_tflops"]),
                "bf16_sustained": float(m.get("bf16_tflops_sustained", m["bf16_tflops"])),
                "source": "measured (MEASURED_PEAKS.json)"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16": 1590.0, "bf16_sustained": 1400.0,
                "source": "fallback (earlier measurement on this pool)"}


def cublas_dgemm_peak(torch):
    """cuBLAS DGEMM 8192^3, best of 3 (FP64 is not in MEASURED_PEAKS.json)."""
    x = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    y = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    torch.matmul(x, y)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        e0_ = torch.cuda.Event(enable_timing=True)
        e1_ = torch.cuda.Event(enable_timing=True)
        e0_.record()
        torch.matmul(x, y)
        e1_.record()
        torch.cuda.synchronize()
        best = min(best, e0_.elapsed_time(e1_) / 1000.0)
    del x, y
    torch.cuda.empty_cache()
    return 2 * 8192.0**3 / best / 1e12


def traffic_of(key):
    """DRAM bytes per launch from an ncu capture (profiles/roofline_traffic.json)."""
    tp = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if not os.path.exists(tp):
        return None
    with open(tp) as f:
        return json.load(f).get(key)


def main():
    a = parse_args()
    if a.tts:
        run_tts(a)
        return
    if a.gradient:
        run_gradient(a)
        return
    if a.sweep:
        run_sweep(a)
        return
    from ecgpu.synthetic import WORKLOADS, make_workload
    wl = WORKLOADS[a.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        if rank == 0:
            run_reference(a, wl)
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    import ecgpu
    from ecgpu._lib import ECG_KT_DGEMM, ECG_KT_TCGEMM, ECG_KT_TRIPLES
    dc = a.method == "dcsd"
    no, nv, nq = wl
    ctx = ecgpu.Context(local)
    W = load_workload(a.workload, a.synthetic, ctx)
    B, h1, e0, no, wdesc = W
    peaks = measured_peaks()
    fp64_peak = cublas_dgemm_peak(torch)
    from ecgpu._lib import ECG_OPT_AUTOTUNE
    tune_entries = ctx.tune_load(TUNE_TABLE) if os.path.exists(TUNE_TABLE) else 0
    ctx.set_system(B, h1, e0, no)
    _, T1, T2 = ctx.mp2()
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def restart():
        ctx.cc_load(T1, T2)

    def timed_steps(k, step):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(k)]
        for i in range(k):
            if i and i % RESTART == 0:
                restart()
            flush.zero_()
            torch.cuda.synchronize()
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        return sum(s_.elapsed_time(e_) for s_, e_ in ev)

    # ---- timed FP64 CCSD iterations (the value) ----
    RESTART = 8  # re-seed from MP2 amplitudes every 8 steps (outside timing)
    if a.tune:
        # tune every GEMM shape of an FP64 and a mixed iteration and of the
        # (T) sweep's first batch (outside any timing), then keep the table
        ctx.set_option(ECG_OPT_AUTOTUNE, 1)
        for prec in (ecgpu.ECG_PREC_FP64, ecgpu.ECG_PREC_MIXED):
            ctx.set_precision(prec)
            restart()
            ctx.cc_step(dc=dc)
            ctx.pert_t()
        ctx.set_option(ECG_OPT_AUTOTUNE, 0)
        ctx.set_precision(ecgpu.ECG_PREC_FP64)
        tune_entries = ctx.tune_save(a.tune)
    restart()
    for _ in range(a.warmup):
        ctx.cc_step(dc=dc)
    restart()
    torch.cuda.synchronize()
    clocks = Clocks(local) if rank == 0 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    launches0 = ctx.kernel_launches()
    total = timed_steps(a.steps, lambda: ctx.cc_step(dc=dc))
    launches = ctx.kernel_launches() - launches0
    if dist:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    total = max_over_ranks(total, dist)

    # ---- e2e: the same iterations through the C ABI with pinned host amplitudes ----
    n1, n2 = nv * no, nv * nv * no * no
    T1p = torch.empty((no, nv), dtype=torch.float64, pin_memory=True).numpy().T
    T2p = torch.empty((no, no, nv, nv), dtype=torch.float64, pin_memory=True).numpy().T
    T1p[...] = T1
    T2p[...] = T2
    restart()

    def host_step():
        ctx.cc_step_host(T1p, T2p, dc=dc)
    total_e2e = timed_steps(a.steps, host_step)
    total_e2e = max_over_ranks(total_e2e, dist)

    # ---- roofline of the FP64 DMMA GEMM: every GEMM launch of R FP64 steps ----
    R = 2
    restart()
    ctx.set_gemm_timing(True)
    ctx.kernel_time(ECG_KT_DGEMM)
    for _ in range(R):
        flush.zero_()
        torch.cuda.synchronize()
        ctx.cc_step(dc=dc)
    gms, glaunch, gflops = ctx.kernel_time(ECG_KT_DGEMM)
    F = algorithmic_flops(no, nv, nq, dc)
    gemm_s = gms / 1000.0 / R
    rl_dgemm = {"bound": "tensor", "achieved": F / gemm_s / 1e12, "peak": fp64_peak,
                "unit": "TFLOP/s", "frac": F / gemm_s / 1e12 / fp64_peak,
                "traffic": traffic_of(f"dgemm_{a.workload}_{a.method}"),
                "kernel": "dgemm_tma_kernel and dgemm_kernel (FP64 mma.sync m8n8k4 on the DMMA pipe; "
                          "TMA-staged or cp.async operands, per-shape tuned), all GEMMs of a step",
                "algorithmic_flops_per_step": F, "gemm_ms_per_step": gms / R,
                "gemm_launches_per_step": glaunch / R,
                "executed_gemm_tflops": gflops / R / gemm_s / 1e12,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 is not in "
                               "MEASURED_PEAKS.json)",
                "step_frac": F / (total / a.steps / 1000.0) / 1e12 / fp64_peak}

    # ---- mixed precision: iteration rate and the tcgen05 GEMM roofline ----
    ctx.set_precision(ecgpu.ECG_PREC_MIXED)
    restart()
    ctx.cc_step(dc=dc)  # first-use set-up of the tensor-core path
    restart()
    total_mx = timed_steps(a.steps, lambda: ctx.cc_step(dc=dc))
    restart()
    ctx.kernel_time(ECG_KT_TCGEMM)
    for _ in range(R):
        flush.zero_()
        torch.cuda.synchronize()
        ctx.cc_step(dc=dc)
    tms, tlaunch, twork = ctx.kernel_time(ECG_KT_TCGEMM)
    ctx.set_gemm_timing(False)
    tc_ach = twork / (tms / 1000.0) / 1e12
    rl_tc_ccsd = {"bound": "tensor", "achieved": tc_ach, "peak": peaks["bf16_sustained"],
                  "unit": "TFLOP/s", "frac": tc_ach / peaks["bf16_sustained"],
                  "traffic": traffic_of(f"mgemm_ccsd_{a.workload}"),
                  "kernel": "mgemm_bf16_kernel (tcgen05.mma kind::f16, TMA), all tensor-core "
                            "GEMMs of a mixed CCSD step",
                  "work": "BF16 products executed: 2 m n k per slice pair (6 pairs)",
                  "ms_per_step": tms / R, "launches_per_step": tlaunch / R,
                  "peak_source": "bf16_tflops_sustained, " + peaks["source"]}
    ctx.set_precision(ecgpu.ECG_PREC_FP64)

    # ---- CCSD(T) time-to-solution, FP64 then mixed, from the MP2 guess ----
    ntrip = sum(1 for k_ in range(no) for j_ in range(k_ + 1) for i_ in range(j_ + 1)
                if not (i_ == j_ == k_))
    ft = ntrip * (12.0 * nv**4 + 12.0 * no * nv**3)
    fcc = algorithmic_flops(no, nv, nq, dc)
    tts = {}
    for prec, name in ((ecgpu.ECG_PREC_FP64, "fp64"), (ecgpu.ECG_PREC_MIXED, "mixed")):
        if name == "mixed":
            # idle before the second leg, so that it does not start on a GPU
            # that the first one left power-capped (outside the timed region)
            time.sleep(COOLDOWN_S)
        ctx.set_precision(prec)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ck = Clocks(local) if rank == 0 else None
        if ck:
            ck.start()
        ev[0].record(stream)
        r = ctx.cc_solve(T1, T2, dc=dc)
        ev[1].record(stream)
        et, _ = ctx.pert_t()  # on the converged amplitudes the context holds
        ev[2].record(stream)
        torch.cuda.synchronize()
        ck = ck.stop() if ck else None
        tcc = ev[0].elapsed_time(ev[1]) / 1000.0
        tt = ev[1].elapsed_time(ev[2]) / 1000.0
        tts[name] = {"ccsd_s": tcc, "pert_t_s": tt, "total_s": tcc + tt,
                     "iterations": r["iterations"], "E_ccsd": r["E"], "E_T": et,
                     "ccsd_tflops_per_iter": fcc * r["iterations"] / tcc / 1e12,
                     "pert_t_tflops": ft / tt / 1e12, "clocks": ck}
    f64, mx = tts["fp64"], tts["mixed"]

    # ---- (T) kernels, mixed: first batch of the sweep (the rest replays from
    # a CUDA graph and is not event-timed) ----
    ctx.set_precision(ecgpu.ECG_PREC_MIXED)
    ctx.set_gemm_timing(True)
    for fam in (ECG_KT_TCGEMM, ECG_KT_TRIPLES):
        ctx.kernel_time(fam)
    ctx.pert_t()
    wms, wlaunch, wwork = ctx.kernel_time(ECG_KT_TCGEMM)
    ems, elaunch, ebytes = ctx.kernel_time(ECG_KT_TRIPLES)
    ctx.set_gemm_timing(False)
    ctx.set_precision(ecgpu.ECG_PREC_FP64)
    w_ach = wwork / (wms / 1000.0) / 1e12 if wms > 0 else None
    e_ach = ebytes / (ems / 1000.0) / 1e9 if ems > 0 else None
    rl_tc_t = {"bound": "tensor", "achieved": w_ach, "peak": peaks["bf16_sustained"],
               "unit": "TFLOP/s", "frac": w_ach / peaks["bf16_sustained"] if w_ach else None,
               "traffic": traffic_of(f"mgemm_pert_t_{a.workload}"),
               "kernel": "mgemm_bf16_kernel, batched four-segment (T) W GEMMs (2 BF16 slices, "
                         "3 pairs), first batch of the sweep",
               "launches": wlaunch, "ms": wms,
               "peak_source": "bf16_tflops_sustained, " + peaks["source"]}
    rl_energy = {"bound": "hbm", "achieved": e_ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                 "frac": e_ach / peaks["hbm_gbs"] if e_ach else None,
                 "traffic": traffic_of(f"triples_energy_{a.workload}"),
                 "kernel": "triples_energy_f32_kernel (FP32 K of mixed (T), one warp per orbit, TMA-staged "
                           "cubes), first batch",
                 "bytes_per_launch": ebytes / max(elaunch, 1), "ms_per_launch":
                 ems / max(elaunch, 1), "work": "bytes of K read once per element",
                 "peak_source": "hbm_gbs, " + peaks["source"]}

    value = world * a.steps / (total / 1000.0)
    line = {
        "metric": "CCSD iter/s", "value": value, "unit": "iter/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": total / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic" if a.synthetic else "real molecule (seeded geometry)",
        "config": {"workload": f"{a.workload} {a.method.upper()} (o={no}, v={nv}, nQ={nq}): "
                               f"{wdesc}",
                   "precision": "fp64",
                   "l2": (f"L2 flushed (256 MiB write) between steps; T2 "
                          f"{8 * n2 / 1e6:.0f} MB, B {8 * (no + nv) ** 2 * nq / 1e6:.0f} MB "
                          + ("(larger than the 126 MB L2)" if 8 * n2 > 126e6
                             else "(smaller than the 126 MB L2)")),
                   "parallelism": f"replicas x{world}",
                   "gemm_tuning": f"{tune_entries} tuned GEMM shapes "
                                  f"({os.path.relpath(TUNE_TABLE, ROOT)})" if tune_entries
                                  else "fixed tile rules"},
        "e2e": {"value": world * a.steps / (total_e2e / 1000.0), "unit": "iter/s",
                "h2d_bytes_per_step": 8 * (n1 + n2), "d2h_bytes_per_step": 8 * (n1 + n2)},
        "gpu_launches": launches,
        "roofline": rl_dgemm,
        "rooflines": {"dgemm_fp64_ccsd": rl_dgemm, "mgemm_bf16_ccsd": rl_tc_ccsd,
                      "mgemm_bf16_pert_t": rl_tc_t, "triples_energy": rl_energy},
        "clocks": clk,
        "mixed": {"metric": "CCSD(T) time-to-solution from the MP2 guess, FP64 vs mixed",
                  "precision": "split-BF16 tcgen05 GEMMs (CCSD: 3 slices, 6 products; (T): "
                               "2 slices, 3 products), FP32 accumulate, FP64 refinement",
                  "fp64": f64, "mixed": mx, "tts_speedup": f64["total_s"] / mx["total_s"],
                  "dE_uEh": abs((mx["E_ccsd"] + mx["E_T"]) - (f64["E_ccsd"] + f64["E_T"])) * 1e6,
                  "dE_T_uEh": abs(mx["E_T"] - f64["E_T"]) * 1e6,
                  "ccsd_iter_per_s": world * a.steps / (total_mx / 1000.0),
                  "triplets": ntrip, "pert_t_algorithmic_flops": ft,
                  "order": f"fp64, {COOLDOWN_S:.0f} s idle, mixed"},
    }
    if rank == 0 and world == 1 and a.cpu_sample > 0:
        cb = cpu_baseline_sample(W, dc, nblocks=a.cpu_sample)
        line["cpu_baseline"] = {
            "value": 1.0 / cb["iter_s"], "unit": "iter/s", "cores": host_cores(),
            "kind": "port",
            "sample": (f"one CCSD iteration of the same workload with the ladder on "
                       f"{cb['ladder_blocks_run']} of its {cb['ladder_blocks']} a-blocks "
                       f"({cb['sampled_s']:.1f} s; the other blocks at the sampled block's "
                       f"time: {cb['iter_s']:.1f} s per iteration), density-fitted numpy "
                       "restatement (oracle/dfcc.py), BLAS threads = all host cores; (T) on "
                       f"{cb['triplets']} triplets"),
            "pert_t_tflops": cb["pert_t_tflops"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
