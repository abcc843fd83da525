"""Benchmark of the density-fitting contraction path on B200.

One step = one RI-MP2 energy + adjoint (Gamma = dE/dB, dE/deps) on the
synthetic RI-MP2 workload (naux 4800, nocc 120, nvir 1100) plus one DF-JK
build (J and K) on the synthetic DF-JK workload (n 600, naux 2400, nocc 60).
The metric is algorithmic TFLOP/s of the step:
    F = 2 naux nvir^2 P + 2 naux nov^2   (energy + adjoint, P = nocc(nocc+1)/2)
      + 4 naux n(n+1)/2 + 4 naux n^2 nocc   (J two passes, K occupied path)

``value``  : device-resident inputs, CUDA events on the launching stream.
``e2e``    : the same step through the host-array C ABI (fc_rimp2_energy_grad,
             fc_dfj_build, fc_dfk_build_occ) from pinned host buffers, copies
             inside the timed region.
``--impl reference`` times the CPU restatement of the reference algorithms
(the oracle port, NumPy/OpenBLAS on every host core) on a bounded sample of
the same step.

Under torchrun each rank runs its own replica of the step (independent
systems, no data-path collective): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

RIMP2 = dict(naux=4800, nocc=120, nvir=1100)
DFJK = dict(n=600, naux=2400, nocc=60)
PREC_NAMES = {"f64": 0, "mixed": 1, "mixed_fast": 2}
# tensor-core products per algorithmic product of the pair kernel: four int8
# slices, the ten products of level <= 3 (mixed); hi+lo bf16 (mixed_fast)
EXECUTED_PRODUCTS = {"f64": 1, "mixed": 10, "mixed_fast": 3}


def step_flops():
    naux, nocc, nvir = RIMP2["naux"], RIMP2["nocc"], RIMP2["nvir"]
    nov = nocc * nvir
    P = nocc * (nocc + 1) / 2
    f_e = 2.0 * naux * nvir * nvir * P
    f_g = 2.0 * naux * nov * nov
    n, na, no = DFJK["n"], DFJK["naux"], DFJK["nocc"]
    f_j = 4.0 * na * n * (n + 1) / 2
    f_k = 4.0 * na * n * n * no
    return dict(rimp2_e=f_e, rimp2_grad=f_g, dfj=f_j, dfk=f_k, total=f_e + f_g + f_j + f_k)


# ---------------------------------------------------------------- clocks --

class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, reasons)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ workloads --

def make_inputs(torch, dev):
    """Seeded synthetic tensors of both workloads, generated on the device."""
    import numpy as np
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    naux, nocc, nvir = RIMP2["naux"], RIMP2["nocc"], RIMP2["nvir"]
    b_ov = torch.randn((naux, nocc * nvir), generator=g, device=dev, dtype=torch.float64)
    decay = 3000.0 * naux / 4800.0
    b_ov *= 0.02 * torch.exp(-torch.arange(naux, device=dev, dtype=torch.float64) / decay)[:, None]
    r2 = np.random.default_rng(30)
    eo = torch.from_numpy(np.sort(r2.uniform(-20.0, -0.3, nocc))).to(dev)
    ev = torch.from_numpy(np.sort(r2.uniform(0.05, 6.0, nvir))).to(dev)

    n, na, no = DFJK["n"], DFJK["naux"], DFJK["nocc"]
    g.manual_seed(2)
    idx = torch.arange(n, device=dev, dtype=torch.float64)
    env = 0.05 * torch.exp(-(idx[:, None] - idx[None, :]).abs() / 50.0)
    bjk = torch.empty((na, n, n), device=dev, dtype=torch.float64)
    for q0 in range(0, na, 256):
        x = torch.randn((min(256, na - q0), n, n), generator=g, device=dev, dtype=torch.float64) * env
        bjk[q0:q0 + x.shape[0]] = (x + x.transpose(1, 2)) / (2.0 ** 0.5)
    rc = np.random.default_rng(20)
    c_occ, _ = np.linalg.qr(rc.standard_normal((n, no)))
    c = torch.from_numpy(np.ascontiguousarray(c_occ)).to(dev)
    d = c @ c.T
    return dict(b_ov=b_ov, eo=eo, ev=ev, bjk=bjk, c=c, d=d)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def measure_i8_tops(torch, dev, seconds=2.0):
    """Int8 tensor peak for the integer-slice kernels: cuBLAS int8 GEMM
    (torch._int_mm, 8192^3, int32 accumulation) back to back for `seconds`
    (sustained under the power cap, like the kernels it is compared with)."""
    g = torch.Generator(device=dev).manual_seed(5)
    a = torch.randint(-127, 128, (8192, 8192), generator=g, device=dev, dtype=torch.int8)
    b = torch.randint(-127, 128, (8192, 8192), generator=g, device=dev, dtype=torch.int8).t()
    for _ in range(3):
        torch._int_mm(a, b)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    torch._int_mm(a, b)
    e1.record()
    torch.cuda.synchronize(dev)
    reps = max(3, int(seconds * 1e3 / max(e0.elapsed_time(e1), 1e-3)))
    e0.record()
    for _ in range(reps):
        torch._int_mm(a, b)
    e1.record()
    torch.cuda.synchronize(dev)
    return 2.0 * 8192 ** 3 * reps / (e0.elapsed_time(e1) * 1e-3) / 1e12


def measure_dgemm_tflops(torch, dev):
    """FP64 peak for the plain set: cuBLAS DGEMM 8192^3, best of 5 (CUDA events)."""
    a = torch.randn((8192, 8192), device=dev, dtype=torch.float64)
    b = torch.randn((8192, 8192), device=dev, dtype=torch.float64)
    for _ in range(2):
        a @ b
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * 8192 ** 3 / (best * 1e-3) / 1e12


def read_traffic(kernel):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 2 and parts[0] == kernel:
                return float(parts[1])
    except OSError:
        pass
    return None


# --------------------------------------------------------------- CPU arm --

def cpu_sample(inputs_host, occ_sample=(0, 1), k_rows=240):
    """Oracle port on the host cores: a bounded sample of one step.

    RI-MP2: the recompute-per-i energy + adjoint for occupied rows
    ``occ_sample``; DF-J: both passes in full; DF-K: the occupied path over
    the first ``k_rows`` aux rows.  Returns (tflops, seconds, description).
    """
    import numpy as np
    from oracle import dfjk as odfjk
    from oracle import rimp2 as ormp2
    b, eo, ev, bp, bsq_rows, c, d = (inputs_host[k] for k in ("b_ov", "eo", "ev", "bp", "bsq_rows", "c", "d"))
    naux, nocc, nvir = RIMP2["naux"], RIMP2["nocc"], RIMP2["nvir"]
    nov = nocc * nvir
    n = DFJK["n"]
    t0 = time.perf_counter()
    ormp2.energy_gamma_deps(b, eo, ev, occ=occ_sample)
    t1 = time.perf_counter()
    w = odfjk.packed_density_weights(d)
    dp = bp @ w
    _ = bp.T @ dp
    t2 = time.perf_counter()
    odfjk.df_k_occ(bsq_rows, c)
    t3 = time.perf_counter()
    f_rimp2 = len(occ_sample) * (2.0 * naux * nvir * nov * 2)   # G_i and x_i per sampled i
    f_j = 4.0 * bp.shape[0] * bp.shape[1]
    f_k = 4.0 * bsq_rows.shape[0] * n * n * c.shape[1]
    secs = t3 - t0
    desc = (f"RI-MP2 E+grad for {len(occ_sample)} of {nocc} occupied rows ({t1 - t0:.2f} s), "
            f"DF-J full ({t2 - t1:.2f} s), DF-K over {bsq_rows.shape[0]} of {DFJK['naux']} aux rows "
            f"({t3 - t2:.2f} s)")
    return (f_rimp2 + f_j + f_k) / secs / 1e12, secs, desc


def host_threads():
    try:
        from threadpoolctl import threadpool_info
        n = [i.get("num_threads", 0) for i in threadpool_info() if i.get("internal_api") == "openblas"]
        if n:
            return max(n)
    except Exception:  # noqa: BLE001
        pass
    return os.cpu_count()


def host_inputs_from(torch, inp):
    import numpy as np
    from oracle import dfjk as odfjk
    k_rows = 240
    bsq_rows = inp["bjk"][:k_rows].cpu().numpy()
    n = DFJK["n"]
    il, jl = np.tril_indices(n)
    il_t = torch.from_numpy(il).to(inp["bjk"].device)
    jl_t = torch.from_numpy(jl).to(inp["bjk"].device)
    bp = inp["bjk"][:, il_t, jl_t].cpu().numpy()
    return dict(b_ov=inp["b_ov"].cpu().numpy(), eo=inp["eo"].cpu().numpy(), ev=inp["ev"].cpu().numpy(),
                bp=bp, bsq_rows=bsq_rows, c=inp["c"].cpu().numpy(), d=inp["d"].cpu().numpy()), odfjk


# ------------------------------------------------------------------ main --

def alkane_shape(n):
    """(naux, nocc, nvir) of all-trans C_nH_2n+2 in cc-pVDZ / cc-pVDZ-RI."""
    return 84 * n + 28, 4 * n + 1, 20 * n + 9


def batch_leg(torch, dev, nmol):
    """Config 4: nmol alkanes C1..C8 (n ~ U{1..8}, seed 4), synthetic B of their
    exact shapes (the config-3 distributions), one batched E+grad replay
    timed; the diagonal-tile schedule of each size bucket autotuned; errors
    against FP64 on one molecule of every size."""
    import numpy as np
    from ferric_b200 import rimp2
    from ferric_b200.batch import Rimp2Batch
    os.environ.setdefault("FERRIC_CUDA_AUTOTUNE", "1")
    ns = np.random.default_rng(4).integers(1, 9, nmol)
    g = torch.Generator(device=dev)
    g.manual_seed(4)
    mols = []
    for n in ns:
        naux, nocc, nvir = alkane_shape(int(n))
        b = torch.randn((naux, nocc * nvir), generator=g, device=dev, dtype=torch.float64)
        b *= 0.02 * torch.exp(-torch.arange(naux, device=dev, dtype=torch.float64) / (3000.0 * naux / 4800.0))[:, None]
        eo = torch.sort(torch.rand(nocc, generator=g, device=dev, dtype=torch.float64) * 19.7 - 20.0).values
        ev = torch.sort(torch.rand(nvir, generator=g, device=dev, dtype=torch.float64) * 5.95 + 0.05).values
        mols.append((b, eo, ev))
    t0 = time.time()
    bt = Rimp2Batch(mols, grad=True)
    create_s = time.time() - t0
    ms = []
    for r in range(4):
        bt.run()
        e_os, e_ss = bt.energies()
        if r:
            ms.append(bt.info()["last_ms"])
    info = bt.info()
    errs = []
    seen = set()
    for m, n in enumerate(ns):
        if int(n) in seen:
            continue
        seen.add(int(n))
        b, eo, ev = mols[m]
        sc, g64, _, _ = rimp2.rimp2_energy_grad(b, eo, ev, precision="f64")
        errs.append({"n": int(n), "e_abs": float(e_os[m] + e_ss[m] - sc.e_total),
                     "e_rel": float((e_os[m] + e_ss[m] - sc.e_total) / abs(sc.e_total)),
                     "gamma_max_rel": float((bt.gamma[m] - g64).abs().max() / g64.abs().max())})
    t_ms = statistics.median(ms)
    out = {"molecules": int(nmol), "sizes": {str(k): int((ns == k).sum()) for k in range(1, 9)},
           "data": "synthetic B of the alkane shapes (naux 84n+28, nocc 4n+1, nvir 20n+9), seeded",
           "ms_e_grad": t_ms, "tflops": info["flops"] / (t_ms * 1e-3) / 1e12, "flops": info["flops"],
           "graph_launches": info["launches"], "pair_launches": info["pair_launches"], "groups": info["groups"],
           "create_s": create_s, "plan": bt.plan(), "error_vs_f64": errs}
    bt.close()
    return out


def dress_leg(torch, dev, naux=2150, n=872, nocc=81):
    """MO transform + metric dressing at config 5's shapes (C20H42 in def2-TZVP
    / def2-TZVP-RIFIT): synthetic (Q|mu nu) symmetric in mu nu (the config-2
    distribution), M = L^-1 of a seeded SPD metric, orthonormal orbitals;
    FP64 and split-BF16 dressing timed once each (after a warm-up at small
    size), the mixed result's error against FP64 stated."""
    from ferric_b200.dress import mo_dress
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    idx = torch.arange(n, device=dev, dtype=torch.float64)
    env = 0.05 * torch.exp(-(idx[:, None] - idx[None, :]).abs() / 50.0)
    t3 = torch.empty((naux, n, n), device=dev, dtype=torch.float64)
    for q0 in range(0, naux, 128):
        x = torch.randn((min(128, naux - q0), n, n), generator=g, device=dev, dtype=torch.float64) * env
        t3[q0:q0 + x.shape[0]] = (x + x.transpose(1, 2)) / (2.0 ** 0.5)
    a = torch.randn((naux, naux), generator=g, device=dev, dtype=torch.float64)
    v = a @ a.T / naux + torch.eye(naux, device=dev, dtype=torch.float64)
    m = torch.linalg.inv(torch.linalg.cholesky(v))
    c, _ = torch.linalg.qr(torch.randn((n, n), generator=g, device=dev, dtype=torch.float64))
    cl, cr = c[:, :nocc].contiguous(), c[:, nocc:].contiguous()
    mo_dress(t3[:8, :64, :64].contiguous(), m[:8, :8].contiguous(), cl[:64].contiguous(), cr[:64].contiguous(),
             precision="mixed")
    out = {"naux": naux, "n": n, "nocc": nocc, "nvir": n - nocc,
           "data": "synthetic (Q|mu nu), seeded SPD metric, orthonormal orbitals"}
    res = {}
    for prec in ("f64", "mixed"):
        st = {}
        b = mo_dress(t3, m, cl, cr, precision=prec, stats=st)
        torch.cuda.synchronize()
        res[prec] = b
        out[prec] = {"ms": st["kernel_ms"], "tflops": st["flops"] / (st["kernel_ms"] * 1e-3) / 1e12,
                     "dressing_gemm_ms": st["main_ms"],
                     "dressing_gemm_tflops": st["main_flops"] / (st["main_ms"] * 1e-3) / 1e12}
    out["flops"] = st["flops"]
    out["mixed_b_max_rel_err"] = float((res["mixed"] - res["f64"]).abs().max() / res["f64"].abs().max())
    out["speedup_mixed_vs_f64"] = out["f64"]["ms"] / out["mixed"]["ms"]
    del t3, res
    torch.cuda.empty_cache()
    return out


def max_over_ranks(torch, ms, world, dev):
    """The slowest rank's device time: every rank takes part in one MAX all-reduce."""
    if world <= 1:
        return float(ms)
    t = torch.tensor([float(ms)], device=dev, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, flops_per_step, ms_step):
    """Whole-job TFLOP/s of `world` replicas that each ran one step's flops in ms_step."""
    return world * flops_per_step / (ms_step * 1e-3) / 1e12


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["auto", "f64", "mixed"], default="auto")
    ap.add_argument("--no-plain", action="store_true", help="skip the one FP64-plain reference step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched config-4 leg")
    ap.add_argument("--batch-mols", type=int, default=512)
    ap.add_argument("--no-dress", action="store_true", help="skip the MO-dressing leg")
    ap.add_argument("--size", choices=["full", "small", "c5"], default="full",
                    help="small: naux 2400, nocc 60, nvir 550 + n 300, naux 1200, nocc 30 "
                         "(the profiling case; inputs still larger than L2); c5: the shapes of "
                         "all-trans C20H42 in def2-TZVP (naux 2150 def2-TZVP-RIFIT, nocc 81, nvir 791 + "
                         "n 872, naux 2256 def2-universal-jkfit, nocc 81) with the synthetic distributions")
    args = ap.parse_args()
    if args.size == "small":
        RIMP2.update(naux=2400, nocc=60, nvir=550)
        DFJK.update(n=300, naux=1200, nocc=30)
    elif args.size == "c5":
        RIMP2.update(naux=2150, nocc=81, nvir=791)
        DFJK.update(n=872, naux=2256, nocc=81)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    flops = step_flops()
    config = {"workload": f"synthetic RI-MP2 E+grad (naux {RIMP2['naux']}, nocc {RIMP2['nocc']}, "
                          f"nvir {RIMP2['nvir']}) + DF-JK build (n {DFJK['n']}, naux {DFJK['naux']}, "
                          f"nocc {DFJK['nocc']}), one replica per GPU",
              "rimp2": RIMP2, "dfjk": DFJK,
              "l2": "inputs larger than L2 (B_ov %.2f GB, B_JK %.2f GB)" % (
                  8e-9 * RIMP2["naux"] * RIMP2["nocc"] * RIMP2["nvir"], 8e-9 * DFJK["naux"] * DFJK["n"] ** 2),
              "parallelism": f"replica x{world}"}

    if args.impl == "reference":
        if rank != 0:
            return
        import numpy as np
        dev = torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")
        inp = make_inputs(torch, dev)
        host, _ = host_inputs_from(torch, inp)
        del inp
        vals = []
        for s in range(args.warmup + args.steps):
            v, secs, desc = cpu_sample(host, occ_sample=(s % RIMP2["nocc"],))
            if s >= args.warmup:
                vals.append(v)
        value = statistics.median(vals)
        ms = flops["total"] / (value * 1e12) * 1e3
        out = {"impl": "reference", "metric": "RI-MP2 E+grad & DF-JK step throughput (algorithmic TFLOP/s)",
               "value": value, "unit": "TFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "config": config,
               "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": host_threads(), "kind": "port",
                                "sample": "per step: " + desc},
               "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return

    import numpy as np
    from ferric_b200 import _lib, rimp2
    from ferric_b200.dfjk import DfJK

    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    _lib.init(local)
    prec = args.precision
    if prec == "auto":
        prec = os.environ.get("FERRIC_BENCH_PRECISION", "mixed")
        try:  # the integer-slice kernels; FP64 plain when this build has none
            tb = torch.zeros((64, 2), dtype=torch.float64, device=dev)
            rimp2.rimp2_energy(tb, torch.zeros(1, dtype=torch.float64, device=dev) - 1,
                               torch.ones(2, dtype=torch.float64, device=dev), precision=prec)
        except _lib.FcError:
            prec = "f64"

    inp = make_inputs(torch, dev)
    naux, nocc, nvir = RIMP2["naux"], RIMP2["nocc"], RIMP2["nvir"]
    gamma = torch.empty_like(inp["b_ov"])
    d_o = torch.empty_like(inp["eo"])
    d_v = torch.empty_like(inp["ev"])
    dfj_prec = dfk_prec = prec
    try:
        jk = DfJK(inp["bjk"], layout="square", precision=prec)
    except _lib.FcError:
        dfj_prec = dfk_prec = "f64"
        jk = DfJK(inp["bjk"], layout="square", precision="f64")
    if dfk_prec != "f64":
        try:  # K on the handle's mixed path when this build has one, FP64 on the device otherwise
            jk.k_from_occ(inp["c"][:, :1])
        except _lib.FcError:
            dfk_prec = "f64"
    jbuf = torch.empty_like(inp["d"])
    kbuf = torch.empty_like(inp["d"])
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    last = {}

    def step():
        st_r, st_j, st_k = {}, {}, {}
        sc, *_ = rimp2.rimp2_energy_grad(inp["b_ov"], inp["eo"], inp["ev"], precision=prec, stats=st_r,
                                         out=(gamma, d_o, d_v))
        jk.set_precision(dfj_prec)
        jk.j(inp["d"], out=jbuf, stats=st_j)
        jk.set_precision(dfk_prec)
        jk.k_from_occ(inp["c"], out=kbuf, stats=st_k)
        last.update(rimp2=st_r, dfj=st_j, dfk=st_k, energy=sc)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    launches = 0
    main_ms = main_flops = 0.0
    main_launch = 0
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
            launches += sum(last[k]["launches"] for k in ("rimp2", "dfj", "dfk"))
            main_ms += last["rimp2"]["main_ms"]
            main_flops += last["rimp2"]["main_flops"]
            main_launch += last["rimp2"]["main_launches"]
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms_total = max_over_ranks(torch, e0.elapsed_time(e1), world, dev)
    ms_step = ms_total / args.steps
    value = replica_throughput(world, flops["total"], ms_step)
    sc = last["energy"]

    # ---- roofline of the dominant kernel (the fused RI-MP2 pair kernel)
    peaks, peak_src = measured_peaks()
    avg_launch_ms = main_ms / max(1, main_launch)
    flops_per_launch = main_flops / max(1, main_launch)
    executed = EXECUTED_PRODUCTS[prec]
    if prec == "f64":
        peak = measure_dgemm_tflops(torch, dev)
        peak_note = "measured in this run: cuBLAS DGEMM 8192^3 (FP64 tensor path)"
        achieved = flops_per_launch / (avg_launch_ms * 1e-3) / 1e12
    elif prec == "mixed":
        peak = measure_i8_tops(torch, dev)
        peak_note = ("measured in this run: cuBLAS int8 GEMM 8192^3 sustained (torch._int_mm); "
                     f"executed = {executed} x algorithmic int8 ops")
        achieved = executed * flops_per_launch / (avg_launch_ms * 1e-3) / 1e12
    else:
        peak = peaks.get("bf16_tflops_sustained", peaks["bf16_tflops"])
        peak_note = f"{peak_src} bf16 dense (sustained), executed = {executed} x algorithmic flops"
        achieved = executed * flops_per_launch / (avg_launch_ms * 1e-3) / 1e12
    roofline = {"bound": "tensor", "kernel": "rimp2 pair kernel (fused G_ij + denominator epilogue)",
                "achieved": achieved, "peak": peak, "unit": "TOP/s" if prec == "mixed" else "TFLOP/s",
                "frac": achieved / peak,
                "peak_source": peak_note, "flops_per_launch": flops_per_launch,
                "avg_launch_ms": avg_launch_ms,
                "traffic": read_traffic(f"rimp2_pair_{prec}")}
    dfj = last["dfj"]
    roof_dfj = {"bound": "hbm", "achieved": dfj["main_bytes"] / (dfj["main_ms"] * 1e-3) / 1e9,
                "peak": peaks["hbm_gbs"], "unit": "GB/s"}
    roof_dfj["frac"] = roof_dfj["achieved"] / roof_dfj["peak"]

    # ---- one FP64-plain step on the same inputs (the "mixed vs FP64 plain" ratio)
    plain = None
    if prec != "f64" and not args.no_plain:
        sp_r, sp_j, sp_k = {}, {}, {}
        jk64 = DfJK(inp["bjk"], layout="square", precision="f64")
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        sc64, g64, _, _ = rimp2.rimp2_energy_grad(inp["b_ov"], inp["eo"], inp["ev"], precision="f64", stats=sp_r)
        j64 = jk64.j(inp["d"], stats=sp_j)
        k64 = jk64.k_from_occ(inp["c"], stats=sp_k)
        p1.record(stream)
        torch.cuda.synchronize()
        pms = p0.elapsed_time(p1)
        plain = {"ms_per_step": pms, "value": flops["total"] / (pms * 1e-3) / 1e12, "unit": "TFLOP/s",
                 "speedup_mixed_vs_plain": pms / ms_step,
                 "components_ms": {"rimp2_e_grad": sp_r["kernel_ms"], "dfj": sp_j["kernel_ms"],
                                   "dfk": sp_k["kernel_ms"]},
                 "mixed_error": {"e_total_abs": (sc.e_os + sc.e_ss) - sc64.e_total,
                                 "e_total_rel": ((sc.e_os + sc.e_ss) - sc64.e_total) / abs(sc64.e_total),
                                 "gamma_max_rel": float((gamma - g64).abs().max() / g64.abs().max()),
                                 "j_max_abs": float((jbuf - j64).abs().max()),
                                 "k_max_abs": float((kbuf - k64).abs().max())}}
        del g64, j64, k64
        jk64.close()

    # ---- e2e through the host-array C ABI, pinned host buffers
    e2e = None
    if not args.no_e2e:
        hb = torch.empty(inp["b_ov"].shape, dtype=torch.float64, pin_memory=True)
        hb.copy_(inp["b_ov"])
        hg = torch.empty_like(hb, pin_memory=True)
        heo, hev = inp["eo"].cpu().numpy(), inp["ev"].cpu().numpy()
        hd = torch.empty(inp["d"].shape, dtype=torch.float64, pin_memory=True)
        hd.copy_(inp["d"])
        hc = torch.empty(inp["c"].shape, dtype=torch.float64, pin_memory=True)
        hc.copy_(inp["c"])
        hj = torch.empty_like(hd, pin_memory=True)
        hk = torch.empty_like(hd, pin_memory=True)
        import ctypes
        from ferric_b200._lib import FcStats, check, ptr
        eo_, es_ = ctypes.c_double(), ctypes.c_double()
        ddo, ddv = np.empty(nocc), np.empty(nvir)
        pr = PREC_NAMES[prec]

        def e2e_step():
            s = FcStats()
            check(_lib.lib.fc_rimp2_energy_grad(ptr(hb), naux, nocc, nvir, ptr(heo), ptr(hev), pr,
                                                ctypes.byref(eo_), ctypes.byref(es_), ptr(hg), ptr(ddo),
                                                ptr(ddv), ctypes.byref(s)))
            s2, s3 = FcStats(), FcStats()
            jk.set_precision(dfj_prec)
            check(_lib.lib.fc_dfj_build(jk._h, ptr(hd), ptr(hj), ctypes.byref(s2)))
            jk.set_precision(dfk_prec)
            check(_lib.lib.fc_dfk_build_occ(jk._h, ptr(hc), DFJK["nocc"], ptr(hk), ctypes.byref(s3)))
            return s.h2d_bytes + s2.h2d_bytes + s3.h2d_bytes, s.d2h_bytes + s2.d2h_bytes + s3.d2h_bytes

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            h2d, d2h = e2e_step()
        torch.cuda.synchronize()
        t_e2e = (time.perf_counter() - t0) / args.steps
        if world > 1:
            t = torch.tensor([t_e2e], device=dev, dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            t_e2e = float(t.item())
        e2e = {"value": world * flops["total"] / t_e2e / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "ms_per_step": t_e2e * 1e3}
        del hb, hg

    # ---- CPU baseline (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        host, _ = host_inputs_from(torch, inp)
        v, secs, desc = cpu_sample(host)
        cpu = {"value": v, "unit": "TFLOP/s", "cores": host_threads(), "kind": "port",
               "sample": desc, "seconds": secs}

    # ---- config 4: batched RI-MP2 E+grad over 512 molecules of uneven size
    batch = None
    if prec == "mixed" and not args.no_batch:
        del gamma, inp
        torch.cuda.empty_cache()
        batch = batch_leg(torch, dev, args.batch_mols)

    # ---- the step before the path: MO transform + metric dressing, config-5 shapes
    dress = None
    if prec == "mixed" and not args.no_dress:
        dress = dress_leg(torch, dev)

    if rank == 0:
        out = {
            "metric": "RI-MP2 E+grad & DF-JK step throughput (algorithmic TFLOP/s)",
            "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"f64": "f64",
                      "mixed": "int8 x3 integer slices, 6 products, exact int32 accumulation, f64 epilogue"}[prec],
            "precision": prec, "dfj_precision": dfj_prec, "dfk_precision": dfk_prec,
            "data": "synthetic (seeded, generated on device)", "config": config,
            "components_ms": {"rimp2_e_grad": last["rimp2"]["kernel_ms"], "dfj": last["dfj"]["kernel_ms"],
                              "dfk": last["dfk"]["kernel_ms"]},
            "flops": flops, "energy": {"e_os": sc.e_os, "e_ss": sc.e_ss},
            "roofline": roofline, "roofline_dfj": roof_dfj,
            "plain_f64": plain,
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
            "config4_batch": batch, "mo_dressing": dress,
        }
        print(json.dumps(out))
    jk.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
