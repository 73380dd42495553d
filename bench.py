"""Benchmark: closed-shell CCSD iterations per second on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload h2o4_vdz] [--method ccsd|dcsd] [--precision fp64]

A step is one CCSD iteration (T1-dressing, residual, Hylleraas energy,
amplitude update, DIIS, energy) of the (H2O)_4/cc-pVDZ-sized closed-shell
problem (o=16, v=76, nQ=336) built from seeded synthetic density-fitting
factors (no integral engine: see the workload generator).  Inputs stay in
HBM; the L2 cache is flushed (256 MiB write) between timed steps, which are
timed with CUDA events on the library's stream.  With N > 1 each rank runs an
independent replica (the path runs on one GPU; no data-path collective) and
the slowest rank's time is reported.

``--impl reference`` times the oracle (the numpy restatement of the
reference's algorithm — ElemCo.jl itself needs Julia, absent here) on the
host cores, same workload and metric.
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


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="h2o4_vdz")
    p.add_argument("--method", default="ccsd", choices=["ccsd", "dcsd"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--cpu-sample", type=int, default=2, help="CPU-baseline iterations")
    p.add_argument("--tts", action="store_true",
                   help="CCSD(T) time-to-solution, FP64 vs mixed, on --workload (one line)")
    p.add_argument("--gradient", action="store_true",
                   help="analytic dE/dlambda (Lambda rrule) vs finite differences, FP64 and "
                        "mixed, on --workload (one line)")
    p.add_argument("--sweep", action="store_true",
                   help="DCSD time per iteration and device memory, FP64 vs mixed, over the "
                        "C6..C10 alkane sizes (one line)")
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


def cpu_ccsd_rate(no, nv, nq, dc, iters):
    """Oracle CCSD iterations/s on the host (all cores via the BLAS)."""
    import oracle as O
    from ecgpu.synthetic import make_system
    B, h1, e0, _ = make_system(no, nv, nq)
    S = O.System.from_df(np.transpose(B, (2, 0, 1)), h1, e0, no)
    f = O.gen_fock(S)
    _, T1, T2 = O.mp2(S, f)
    eps = np.diag(f)
    eo, ev = eps[:no], eps[no:]
    diis = O.Diis(6, 10.0, dots=(O.cs_singles_dot, O.cs_doubles_dot))
    t0 = time.perf_counter()
    for _ in range(iters):
        R1, R2 = O.cc_resid(S, T1, T2, dc=dc)
        O.hylleraas(S, T1, T2, R1, R2, f)
        T2 = T2 + O.update_doubles(R2, eo, ev, 0.2)
        T1 = T1 + O.update_singles(R1, eo, ev, 0.15)
        diis.perform([T1, T2], [R1, R2])
        O.doubles_energy(S, T2) + O.singles_energy(S, T1, f)
    dt = time.perf_counter() - t0
    return iters / dt, dt


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- main


def run_reference(a, wl):
    no, nv, nq = wl
    K = max(1, min(a.steps, a.cpu_sample))
    for _ in range(min(a.warmup, 1)):
        pass  # the oracle has no compile/cache warm-up beyond the first BLAS call
    rate, dt = cpu_ccsd_rate(no, nv, nq, a.method == "dcsd", K)
    cores = host_cores()
    line = {
        "impl": "reference", "metric": "CCSD iter/s", "value": rate, "unit": "iter/s",
        "n_gpus": a.gpus, "steps": K, "warmup": a.warmup, "ms_per_step": 1000.0 / rate,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": f"{a.workload} {a.method.upper()} (o={no}, "
                                                    f"v={nv}, nQ={nq}), synthetic DF factors"},
        "cpu_baseline": {"value": rate, "unit": "iter/s", "cores": cores, "kind": "port",
                         "sample": f"{K} full CCSD iterations of the workload ({dt:.1f} s), "
                                   "numpy restatement of the reference algorithm, BLAS threads = "
                                   "all host cores"},
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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    import ecgpu
    dc = a.method == "dcsd"
    no, nv, nq = wl
    B, h1, e0, no = make_workload(a.workload)

    # measured FP64 GEMM peak (cuBLAS DGEMM 8192^3, best of 3) for the roofline
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
    fp64_peak = 2 * 8192.0**3 / best / 1e12
    del x, y

    ctx = ecgpu.Context(local)
    if a.precision == "mixed":
        ctx.set_precision(ecgpu.ECG_PREC_MIXED)
    ctx.set_system(B, h1, e0, no)
    _, T1, T2 = ctx.mp2()
    stream = torch.cuda.ExternalStream(ctx.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def restart():
        ctx.cc_load(T1, T2)

    RESTART = 8  # re-seed from MP2 amplitudes every 8 steps (outside timing)
    restart()
    for w in range(a.warmup):
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
    ms = []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(a.steps)]
    for k in range(a.steps):
        if k and k % RESTART == 0:
            restart()
        flush.zero_()
        torch.cuda.synchronize()
        ev[k][0].record(stream)
        ctx.cc_step(dc=dc)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    launches = ctx.kernel_launches() - launches0
    if dist:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    ms = [s.elapsed_time(e) for s, e in ev]
    total = sum(ms)
    if dist:
        t = torch.tensor([total], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    steps_launches = launches - (a.steps // RESTART) * 0

    # e2e: the same iterations through the C ABI with pinned host amplitudes
    n1, n2 = nv * no, nv * nv * no * no
    T1p = torch.empty((no, nv), dtype=torch.float64, pin_memory=True).numpy().T
    T2p = torch.empty((no, no, nv, nv), dtype=torch.float64, pin_memory=True).numpy().T
    T1p[...] = T1
    T2p[...] = T2
    restart()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(a.steps)]
    for k in range(a.steps):
        if k and k % RESTART == 0:
            restart()
            T1p[...] = T1
            T2p[...] = T2
        flush.zero_()
        torch.cuda.synchronize()
        ev2[k][0].record(stream)
        ctx.cc_step_host(T1p, T2p, dc=dc)
        ev2[k][1].record(stream)
    torch.cuda.synchronize()
    total_e2e = sum(s.elapsed_time(e) for s, e in ev2)
    if dist:
        t = torch.tensor([total_e2e], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_e2e = float(t.item())

    # roofline of the dominant kernel (FP64 GEMM), live GEMM event timing
    restart()
    R = 4
    ctx.set_gemm_timing(True)
    ctx.gemm_time()
    for _ in range(R):
        flush.zero_()
        torch.cuda.synchronize()
        ctx.cc_step(dc=dc)
    gms, glaunch, gflops = ctx.gemm_time()
    ctx.set_gemm_timing(False)
    F = algorithmic_flops(no, nv, nq, dc)
    gemm_s = gms / 1000.0 / R
    achieved = F / gemm_s / 1e12
    traffic = None
    tp = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(f"{a.workload}_{a.method}_{a.precision}")

    # time-to-solution, FP64 vs mixed (split-BF16 tensor-core products + FP64
    # refinement), full solves from the MP2 guess; energy difference in uEh
    def solve_timed(prec):
        ctx.set_precision(prec)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        torch.cuda.synchronize()
        ev0.record(stream)
        r = ctx.cc_solve(T1, T2, dc=dc)
        ev1.record(stream)
        torch.cuda.synchronize()
        return r, ev0.elapsed_time(ev1) / 1000.0
    solve_timed(ecgpu.ECG_PREC_MIXED)  # warm the tensor-core path (split buffers)
    r64, t64 = solve_timed(ecgpu.ECG_PREC_FP64)
    rmx, tmx = solve_timed(ecgpu.ECG_PREC_MIXED)
    # mixed-precision iteration rate (same step as above, tensor-core products)
    ctx.set_precision(ecgpu.ECG_PREC_MIXED)
    restart()
    ctx.cc_step(dc=dc)
    restart()
    evm = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(a.steps)]
    for k in range(a.steps):
        if k and k % RESTART == 0:
            restart()
        flush.zero_()
        torch.cuda.synchronize()
        evm[k][0].record(stream)
        ctx.cc_step(dc=dc)
        evm[k][1].record(stream)
    torch.cuda.synchronize()
    total_mx = sum(s_.elapsed_time(e_) for s_, e_ in evm)
    ctx.set_precision(ecgpu.ECG_PREC_FP64)
    # (T) on the converged FP64 amplitudes
    ntrip = sum(1 for k_ in range(no) for j_ in range(k_ + 1) for i_ in range(j_ + 1)
                if not (i_ == j_ == k_))
    ft = ntrip * (12.0 * nv**4 + 12.0 * no * nv**3)
    evt0, evt1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    evt0.record(stream)
    et, _ = ctx.pert_t(r64["T1"], r64["T2"])
    evt1.record(stream)
    torch.cuda.synchronize()
    t_t = evt0.elapsed_time(evt1) / 1000.0

    value = world * a.steps / (total / 1000.0)
    line = {
        "metric": "CCSD iter/s", "value": value, "unit": "iter/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": total / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"{a.workload} {a.method.upper()} (o={no}, v={nv}, nQ={nq}), "
                               "seeded synthetic DF factors, canonical HF reference",
                   "precision": a.precision, "l2": "flushed (256 MiB write) between steps",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": world * a.steps / (total_e2e / 1000.0), "unit": "iter/s",
                "h2d_bytes_per_step": 8 * (n1 + n2), "d2h_bytes_per_step": 8 * (n1 + n2)},
        "gpu_launches": steps_launches,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": fp64_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp64_peak, "traffic": traffic,
                     "kernel": "dgemm_kernel (FP64 mma.sync m8n8k4), all GEMMs of a step",
                     "algorithmic_flops_per_step": F, "gemm_ms_per_step": gms / R,
                     "gemm_launches_per_step": glaunch / R,
                     "executed_gemm_tflops": gflops / R / gemm_s / 1e12,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 is not in "
                                    "MEASURED_PEAKS.json)",
                     "step_frac": F / (total / a.steps / 1000.0) / 1e12 / fp64_peak},
        "clocks": clk,
        "mixed": {"iter_per_s": world * a.steps / (total_mx / 1000.0),
                  "precision": "split-BF16 (3 slices, 6 products) tcgen05 GEMMs, FP32 accumulate",
                  "tts_fp64_s": t64, "tts_mixed_s": tmx, "tts_speedup": t64 / tmx,
                  "iterations_fp64": r64["iterations"], "iterations_mixed": rmx["iterations"],
                  "dE_uEh": abs(rmx["E"] - r64["E"]) * 1e6, "E_corr_fp64": r64["E"]},
        "pert_t": {"seconds": t_t, "tflops": ft / t_t / 1e12, "E_T": et, "triplets": ntrip,
                   "algorithmic_flops": ft, "precision": "fp64"},
    }
    if rank == 0 and world == 1 and a.cpu_sample > 0:
        rate, dt = cpu_ccsd_rate(no, nv, nq, dc, a.cpu_sample)
        line["cpu_baseline"] = {"value": rate, "unit": "iter/s", "cores": host_cores(),
                                "kind": "port",
                                "sample": f"{a.cpu_sample} CCSD iterations of the same workload "
                                          f"({dt:.1f} s), numpy restatement, all host cores"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
