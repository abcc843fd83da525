"""Benchmark of the density-fitting contraction path on B200.

One step = one RI-MP2 energy + adjoint (Gamma = dE/dB, dE/deps) on the
synthetic RI-MP2 workload (naux 4800, nocc 120, nvir 1100) plus one DF-JK
build (J and K of C_occ in one fc_dfjk_build_occ call: J's first pass read
off K's stage-1 product) on the synthetic DF-JK workload (n 600, naux 2400,
nocc 60); the FP64 plain step uses the same calls.
The metric is algorithmic TFLOP/s of the step:
    F = 2 naux nvir^2 P + 2 naux nov^2   (energy + adjoint, P = nocc(nocc+1)/2)
      + 4 naux n(n+1)/2 + 4 naux n^2 nocc   (J two passes, K occupied path)

``value``  : device-resident inputs, CUDA events on the launching stream.
``e2e``    : the same step through the host-array C ABI (fc_rimp2_energy_grad,
             fc_dfjk_build_occ) from pinned host buffers, copies inside the
             timed region.
``--impl reference`` and ``cpu_baseline`` time the C++ restatement of the
reference's host algorithms (oracle/cpu_ref.cpp: OpenMP over work units,
OpenBLAS at one thread per unit, on every physical host core) on a bounded
sample of the same step: RI-MP2 units (i, j-block) spread over the whole
occupied range, scaled to the full step, plus one whole DF-J and DF-K build.
``roofline`` is the dominant kernel of the step (by device time, CUDA events
in this run), ``roofline_kernels`` both RI-MP2 kernels: achieved = executed
tensor-core work per launch in BF16-equivalent flops (an int8 MMA of K = 32
takes the time of a bf16 one of K = 16) / mean launch time, against the
measured sustained BF16 peak (MEASURED_PEAKS.json); ``traffic`` is the DRAM
bytes per launch of an ncu capture committed in profiles/traffic.txt, with
the commit it was captured at.

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
# the adjoint contraction: three int8 slices, six products (mixed)
ADJOINT_PRODUCTS = {"f64": 1, "mixed": 6, "mixed_fast": 6}


def step_flops(rim=None, jkc=None):
    rim = rim or RIMP2
    jkc = jkc or DFJK
    naux, nocc, nvir = rim["naux"], rim["nocc"], rim["nvir"]
    nov = nocc * nvir
    P = nocc * (nocc + 1) / 2
    f_e = 2.0 * naux * nvir * nvir * P
    f_g = 2.0 * naux * nov * nov
    n, na, no = jkc["n"], jkc["naux"], jkc["nocc"]
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

def make_inputs(torch, dev, rim=None, jkc=None):
    """Seeded synthetic tensors of both workloads, generated on the device."""
    import numpy as np
    rim = rim or RIMP2
    jkc = jkc or DFJK
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    naux, nocc, nvir = rim["naux"], rim["nocc"], rim["nvir"]
    b_ov = torch.randn((naux, nocc * nvir), generator=g, device=dev, dtype=torch.float64)
    decay = 3000.0 * naux / 4800.0
    b_ov *= 0.02 * torch.exp(-torch.arange(naux, device=dev, dtype=torch.float64) / decay)[:, None]
    r2 = np.random.default_rng(30)
    eo = torch.from_numpy(np.sort(r2.uniform(-20.0, -0.3, nocc))).to(dev)
    ev = torch.from_numpy(np.sort(r2.uniform(0.05, 6.0, nvir))).to(dev)

    n, na, no = jkc["n"], jkc["naux"], jkc["nocc"]
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
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary
    (profiles/traffic.txt: `<key> <bytes> <commit> <capture>`), with the
    commit and capture it came from; (None, None) if there is none."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for line in open(path):
            parts = line.split(None, 3)
            if len(parts) >= 2 and parts[0] == kernel:
                src = (f"ncu dram__bytes_read.sum + dram__bytes_write.sum at commit {parts[2]}: {parts[3].strip()}"
                       if len(parts) == 4 else "ncu (profiles/traffic.txt)")
                return float(parts[1]), src
    except OSError:
        pass
    return None, None


# --------------------------------------------------------------- CPU arm --

def rimp2_cpu_units(nocc, cores, width=4, offset=0):
    """A bounded sample of RI-MP2 units (i, j0, j0 + width): one per core,
    i spread over the whole occupied range (the work of a unit does not
    depend on i) and the j-blocks over the whole range too."""
    nblk = -(-nocc // width)
    units = []
    for k in range(cores):
        i = (k * nocc // cores + offset) % nocc
        jb = (k * 7 + 3 * offset) % nblk
        units.append((i, jb * width, min(nocc, (jb + 1) * width)))
    return units, nocc * nblk


def cpu_sample(inputs_host, offset=0):
    """The C++ restatement of the reference's host algorithms on every
    physical core: a sample of RI-MP2 units (one per core, scaled to the full
    step), one whole DF-J and one whole DF-K build.  Returns (tflops of the
    whole step, extrapolated step seconds, cores, description)."""
    from oracle import cpu_ref
    cores = cpu_ref.physical_cores()
    b, eo, ev, bp, w, bsq, c = (inputs_host[k] for k in ("b_ov", "eo", "ev", "bp", "w", "bsq", "c"))
    nocc = len(eo)
    units, total_units = rimp2_cpu_units(nocc, cores, offset=offset)
    t_r, _, _ = cpu_ref.rimp2_units(b, eo, ev, units, cores)
    t_j, _ = cpu_ref.dfj(bp, w, cores)
    t_k, _ = cpu_ref.dfk(bsq, c, cores)
    t_rimp2 = t_r * total_units / len(units)
    secs = t_rimp2 + t_j + t_k
    desc = (f"C++ port (OpenMP over units, OpenBLAS 1 thread each) on {cores} physical cores: "
            f"RI-MP2 E+grad {len(units)} of {total_units} units (i, 4-orbital j-block) spread over the "
            f"occupied range in {t_r:.2f} s, scaled to {t_rimp2:.1f} s; DF-J full {t_j:.2f} s; "
            f"DF-K full {t_k:.2f} s")
    return step_flops()["total"] / secs / 1e12, secs, cores, desc


def host_inputs_from(torch, inp):
    """Host copies of the step's inputs for the CPU arm: B_ov, the DF-JK
    tensor square (DF-K) and as packed lower rows (DF-J), the packed density
    weights, C_occ."""
    import numpy as np
    from oracle import dfjk as odfjk
    n = DFJK["n"]
    il, jl = np.tril_indices(n)
    il_t = torch.from_numpy(il).to(inp["bjk"].device)
    jl_t = torch.from_numpy(jl).to(inp["bjk"].device)
    bp = inp["bjk"][:, il_t, jl_t].cpu().numpy()
    d = inp["d"].cpu().numpy()
    return dict(b_ov=inp["b_ov"].cpu().numpy(), eo=inp["eo"].cpu().numpy(), ev=inp["ev"].cpu().numpy(),
                bp=bp, w=odfjk.packed_density_weights(d), bsq=inp["bjk"].cpu().numpy(),
                c=inp["c"].cpu().numpy(), d=d)


# ------------------------------------------------------------------ main --

def alkane_shape(n):
    """(naux, nocc, nvir) of all-trans C_nH_2n+2 in cc-pVDZ / cc-pVDZ-RI."""
    return 84 * n + 28, 4 * n + 1, 20 * n + 9


ALKANES = os.path.join(ROOT, "tests", "golden", "_cache", "alkanes_c1_c8.npz")


def batch_leg(torch, dev, nmol):
    """Config 4: nmol alkanes C1..C8 (n ~ U{1..8}, seed 4), one batched E+grad
    replay timed; the diagonal-tile schedule of each size bucket autotuned;
    errors against FP64 on one molecule of every size.  Inputs: B_ov and
    orbital energies of the oracle's RHF for all-trans C_nH_2n+2 in cc-pVDZ /
    cc-pVDZ-RI (tests/golden/make_alkanes.py), one device copy per molecule,
    with the oracle's FP64 energies; synthetic B of the exact shapes (the
    config-3 distributions) when that file is absent."""
    import numpy as np
    from ferric_b200 import rimp2
    from ferric_b200.batch import Rimp2Batch
    os.environ.setdefault("FERRIC_CUDA_AUTOTUNE", "1")
    ns = np.random.default_rng(4).integers(1, 9, nmol)
    real = os.path.exists(ALKANES)
    src = np.load(ALKANES) if real else None
    g = torch.Generator(device=dev)
    g.manual_seed(4)
    mols = []
    for n in ns:
        naux, nocc, nvir = alkane_shape(int(n))
        if real:
            b = torch.from_numpy(src[f"c{n}_b_ov"]).to(dev)
            eo = torch.from_numpy(src[f"c{n}_eps_occ"]).to(dev)
            ev = torch.from_numpy(src[f"c{n}_eps_vir"]).to(dev)
            assert tuple(b.shape) == (naux, nocc * nvir)
        else:
            b = torch.randn((naux, nocc * nvir), generator=g, device=dev, dtype=torch.float64)
            b *= 0.02 * torch.exp(-torch.arange(naux, device=dev, dtype=torch.float64)
                                  / (3000.0 * naux / 4800.0))[:, None]
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
        e = {"n": int(n), "e_mp2": sc.e_total, "e_abs": float(e_os[m] + e_ss[m] - sc.e_total),
             "e_os_abs": float(e_os[m] - sc.e_os), "e_ss_abs": float(e_ss[m] - sc.e_ss),
             "e_rel": float((e_os[m] + e_ss[m] - sc.e_total) / abs(sc.e_total)),
             "gamma_max_rel": float((bt.gamma[m] - g64).abs().max() / g64.abs().max())}
        if real:  # the FP64 device energy against the oracle's
            e["f64_vs_oracle_abs"] = sc.e_total - float(src[f"c{n}_e_os"] + src[f"c{n}_e_ss"])
        errs.append(e)
    t_ms = statistics.median(ms)
    out = {"molecules": int(nmol), "sizes": {str(k): int((ns == k).sum()) for k in range(1, 9)},
           "data": ("oracle RHF tensors of all-trans C_nH_2n+2 (cc-pVDZ / cc-pVDZ-RI), one copy per molecule"
                    if real else "synthetic B of the alkane shapes (naux 84n+28, nocc 4n+1, nvir 20n+9), seeded; "
                                 "the oracle's alkane tensors were not found"),
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


C5_RIMP2 = dict(naux=2150, nocc=81, nvir=791)
C5_DFJK = dict(n=872, naux=2256, nocc=81)


def c5_leg(torch, dev, prec, steps=3):
    """Config 5 at the shapes of all-trans C20H42 in def2-TZVP (RI-MP2: naux
    2150 def2-TZVP-RIFIT, nocc 81, nvir 791; DF-JK: n 872, naux 2256
    def2-universal-jkfit, nocc 81), synthetic tensors with the config-3 /
    config-2 distributions: the mixed step (median of `steps` after a
    warm-up) and one FP64-plain step, the speed-up, the mixed errors against
    FP64, and the pair kernel's and the adjoint's device time."""
    from ferric_b200 import rimp2
    from ferric_b200.dfjk import DfJK
    inp = make_inputs(torch, dev, C5_RIMP2, C5_DFJK)
    fl = step_flops(C5_RIMP2, C5_DFJK)
    stream = torch.cuda.current_stream(dev)
    out = {"rimp2": C5_RIMP2, "dfjk": C5_DFJK, "flops": fl["total"],
           "data": "synthetic (seeded, generated on device) at the C20H42 def2-TZVP shapes"}
    res = {}
    for p in (prec, "f64"):
        jk = DfJK(inp["bjk"], layout="square", precision=p)
        gamma, d_o, d_v = torch.empty_like(inp["b_ov"]), torch.empty_like(inp["eo"]), torch.empty_like(inp["ev"])

        def one():
            st = ({}, {}, {})
            sc, *_ = rimp2.rimp2_energy_grad(inp["b_ov"], inp["eo"], inp["ev"], precision=p, stats=st[0],
                                             out=(gamma, d_o, d_v))
            j, k = jk.jk_from_occ(inp["c"], stats=st[1])
            return sc, st, j, k
        one()
        ms = []
        for _ in range(steps if p == prec else 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            sc, st, j, k = one()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        t = statistics.median(ms)
        r = st[0]
        res[p] = dict(sc=sc, gamma=gamma.clone(), j=j, k=k)
        out[p] = {"ms_per_step": t, "tflops": fl["total"] / (t * 1e-3) / 1e12,
                  "components_ms": {"rimp2_e_grad": r["kernel_ms"], "dfjk": st[1]["kernel_ms"],
                                    "dfk_stages": st[1]["main_ms"], "dfj_pass2": st[1]["aux_ms"]},
                  "pair_kernel_ms": r["main_ms"], "pair_launches": r["main_launches"],
                  "adjoint_ms": r["aux_ms"], "adjoint_launches": r["aux_launches"]}
        jk.close()
        del gamma
    m, f = res[prec], res["f64"]
    out["speedup_mixed_vs_plain"] = out["f64"]["ms_per_step"] / out[prec]["ms_per_step"]
    out["mixed_error"] = {"e_total_abs": m["sc"].e_total - f["sc"].e_total,
                          "e_os_abs": m["sc"].e_os - f["sc"].e_os, "e_ss_abs": m["sc"].e_ss - f["sc"].e_ss,
                          "e_corr_f64": f["sc"].e_total,
                          "e_total_rel": (m["sc"].e_total - f["sc"].e_total) / abs(f["sc"].e_total),
                          "gamma_max_rel": float((m["gamma"] - f["gamma"]).abs().max() / f["gamma"].abs().max()),
                          "j_max_abs": float((m["j"] - f["j"]).abs().max()),
                          "k_max_abs": float((m["k"] - f["k"]).abs().max())}
    del inp, res, m, f
    torch.cuda.empty_cache()
    return out


def dfjk_leg(torch, dev, prec, index, builds=20):
    """One DF-JK build at config 2 (n 600, naux 2400, nocc 60) as the SCF runs
    it, one build after another: the fused J + K call, mixed and FP64 plain,
    each the median of `builds` device-timed calls after three warm-up calls,
    with the SM clocks sampled during them.  The step's own DF-JK figure is
    taken right after the RI-MP2 gradient, at the clock that part's power draw
    sets; this leg gives the builds at the clock they run at on their own."""
    from ferric_b200.dfjk import DfJK
    inp = make_inputs(torch, dev, dict(naux=64, nocc=2, nvir=8), DFJK)
    out = {"dfjk": DFJK, "builds": builds}
    for p in (prec, "f64"):
        jk = DfJK(inp["bjk"], layout="square", precision=p)
        j, k = torch.empty_like(inp["d"]), torch.empty_like(inp["d"])
        for _ in range(3):
            jk.jk_from_occ(inp["c"], out=(j, k))
        ms = []
        with ClockSampler(index) as clk:
            for _ in range(builds):
                st = {}
                jk.jk_from_occ(inp["c"], out=(j, k), stats=st)
                ms.append(st["kernel_ms"])
        out[p] = {"ms": statistics.median(ms), "min_ms": min(ms), "max_ms": max(ms), "clocks": clk.summary()}
        jk.close()
    out["speedup_mixed_vs_plain"] = out["f64"]["ms"] / out[prec]["ms"]
    del inp
    torch.cuda.empty_cache()
    return out


def rimp2_leg(torch, dev, prec, calls=3):
    """The RI-MP2 energy + gradient alone at --size's shapes: `calls` calls
    (the first a warm-up), the library's stats of the last (profiling case)."""
    from ferric_b200 import rimp2
    inp = make_inputs(torch, dev, RIMP2, dict(n=16, naux=16, nocc=2))
    st = {}
    for _ in range(calls):
        st = {}
        sc, *_ = rimp2.rimp2_energy_grad(inp["b_ov"], inp["eo"], inp["ev"], precision=prec, stats=st)
    return {"rimp2": RIMP2, "precision": prec, "kernel_ms": st["kernel_ms"], "pair_kernel_ms": st["main_ms"],
            "pair_launches": st["main_launches"], "adjoint_ms": st["aux_ms"], "adjoint_launches": st["aux_launches"],
            "e_total": sc.e_total}


def dens_leg(torch, dev, prec):
    """The gradient call with the full unrelaxed densities P_oo / P_vv at the
    config-3 RI-MP2 shapes: device time against the gradient call alone (one
    warm-up, then one timed call of each), and the densities' own checks at
    full size (2 diag P against the pair kernel's dE/deps, symmetry)."""
    from ferric_b200 import rimp2
    inp = make_inputs(torch, dev, RIMP2, None)
    stream = torch.cuda.current_stream(dev)
    out = {"rimp2": RIMP2, "precision": prec}
    for name in ("grad", "grad_dens", "grad_dens_timed", "grad_timed"):
        dens = "dens" in name
        st = {}
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        if dens:
            sc, g, d_o, d_v, p_oo, p_vv = rimp2.rimp2_energy_grad_dens(inp["b_ov"], inp["eo"], inp["ev"],
                                                                       precision=prec, stats=st)
        else:
            sc, g, d_o, d_v = rimp2.rimp2_energy_grad(inp["b_ov"], inp["eo"], inp["ev"], precision=prec, stats=st)
        e1.record(stream)
        torch.cuda.synchronize()
        if name.endswith("timed"):
            key = "grad_dens" if dens else "grad"
            out[key] = {"ms": e0.elapsed_time(e1), "kernel_ms": st["kernel_ms"], "pair_launches": st["main_launches"],
                        "pair_kernel_ms": st["main_ms"], "adjoint_ms": st["aux_ms"]}
            if dens:
                out["checks"] = {
                    "diag_oo_vs_de_docc_rel": float((2.0 * torch.diagonal(p_oo) - d_o).abs().max() / d_o.abs().max()),
                    "diag_vv_vs_de_dvir_rel": float((2.0 * torch.diagonal(p_vv) - d_v).abs().max() / d_v.abs().max()),
                    "symmetric": bool(torch.equal(p_oo, p_oo.T) and torch.equal(p_vv, p_vv.T)),
                    "e_total": sc.e_total}
        del g
    out["overhead_vs_grad"] = out["grad_dens"]["ms"] / out["grad"]["ms"]
    del inp
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
    ap.add_argument("--no-c5", action="store_true", help="skip the config-5 leg")
    ap.add_argument("--no-dens", action="store_true", help="skip the densities leg")
    ap.add_argument("--leg", choices=["dfjk", "dens", "rimp2"], default=None,
                    help="run only this side leg at --size's shapes and print its JSON (profiling cases)")
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
    if args.leg:
        from ferric_b200 import _lib
        dev = torch.device("cuda", local)
        torch.cuda.set_device(dev)
        _lib.init(local)
        prec = "mixed" if args.precision == "auto" else args.precision
        if args.leg == "dfjk":
            leg = dfjk_leg(torch, dev, prec, local, builds=3)
        elif args.leg == "dens":
            leg = dens_leg(torch, dev, prec)
        else:
            leg = rimp2_leg(torch, dev, prec)
        print(json.dumps({"leg": args.leg, "size": args.size, **leg}))
        return
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
        host = host_inputs_from(torch, inp)
        del inp
        torch.cuda.empty_cache()
        vals = []
        for s in range(args.warmup + args.steps):
            v, secs, cores, desc = cpu_sample(host, offset=s)
            if s >= args.warmup:
                vals.append(v)
        value = max(vals)   # the fastest of the timed samples (min time)
        ms = flops["total"] / (value * 1e12) * 1e3
        out = {"impl": "reference", "metric": "RI-MP2 E+grad & DF-JK step throughput (algorithmic TFLOP/s)",
               "value": value, "unit": "TFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "config": config,
               "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": cores, "kind": "port",
                                "sample": f"per step (best of {args.steps}, after {args.warmup} warm-up): " + desc},
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
        jk.set_precision(dfk_prec)
        jk.jk_from_occ(inp["c"], out=(jbuf, kbuf), stats=st_j)
        last.update(rimp2=st_r, dfjk=st_j, energy=sc)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    launches = 0
    main_ms = main_flops = 0.0
    main_launch = 0
    aux_ms = aux_flops = 0.0
    aux_launch = 0
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
            launches += sum(last[k]["launches"] for k in ("rimp2", "dfjk"))
            main_ms += last["rimp2"]["main_ms"]
            main_flops += last["rimp2"]["main_flops"]
            main_launch += last["rimp2"]["main_launches"]
            aux_ms += last["rimp2"]["aux_ms"]
            aux_flops += last["rimp2"]["aux_flops"]
            aux_launch += last["rimp2"]["aux_launches"]
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms_total = max_over_ranks(torch, e0.elapsed_time(e1), world, dev)
    ms_step = ms_total / args.steps
    value = replica_throughput(world, flops["total"], ms_step)
    sc = last["energy"]

    # ---- rooflines of the two RI-MP2 kernels; `roofline` is the one with
    # more device time in the timed steps
    peaks, peak_src = measured_peaks()
    bf16_peak = peaks.get("bf16_tflops_sustained", peaks["bf16_tflops"])
    i8_peak = measure_i8_tops(torch, dev) if prec == "mixed" else None
    f64_peak = measure_dgemm_tflops(torch, dev) if prec == "f64" else None
    kern = {"pair": dict(ms=main_ms, flops=main_flops, launches=main_launch, products=EXECUTED_PRODUCTS[prec],
                         name="pair kernel: G_ij tiles + denominator / energy / amplitude epilogue",
                         traffic_key=f"rimp2_pair_{prec}"),
            "adjoint": dict(ms=aux_ms, flops=aux_flops, launches=aux_launch, products=ADJOINT_PRODUCTS[prec],
                            name="adjoint contraction Gamma += 4 B Tt^T",
                            traffic_key=f"rimp2_adjoint_{prec}")}
    rooflines = {}
    for key, k in kern.items():
        if k["launches"] == 0 or k["ms"] <= 0.0:
            continue
        avg_ms = k["ms"] / k["launches"]
        alg = k["flops"] / k["launches"]                        # algorithmic flops per launch
        alg_tf = alg / (avg_ms * 1e-3) / 1e12
        traffic, tsrc = read_traffic(k["traffic_key"])
        r = {"bound": "tensor", "kernel": k["name"], "launches_per_step": k["launches"] // args.steps,
             "avg_launch_ms": avg_ms, "algorithmic_flops_per_launch": alg, "algorithmic_tflops": alg_tf,
             "traffic": traffic, "traffic_source": tsrc}
        if prec == "f64":
            r.update(achieved=alg_tf, peak=f64_peak, unit="TFLOP/s", frac=alg_tf / f64_peak,
                     peak_source="cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor path)")
        else:
            # int8 (kind::i8): an MMA of K = 32 takes the time of a bf16 MMA of K = 16
            per_bf16 = 0.5 if prec == "mixed" else 1.0
            ex = k["products"] * per_bf16 * alg_tf
            r.update(achieved=ex, peak=bf16_peak, unit="TFLOP/s", frac=ex / bf16_peak,
                     peak_source=f"{peak_src} bf16_tflops_sustained (MEASURED_PEAKS.json)",
                     achieved_note=(f"BF16-equivalent executed: {k['products']} tensor-core products per "
                                    f"algorithmic product" + (" at int8 (half a bf16 MMA each)"
                                                              if prec == "mixed" else "")))
            if i8_peak:
                r["int8_tops"] = k["products"] * alg_tf
                r["int8_peak_measured"] = i8_peak
                r["int8_frac"] = r["int8_tops"] / i8_peak
        rooflines[key] = r
    dom = max(rooflines, key=lambda x: kern[x]["ms"])
    roofline = dict(rooflines[dom], which=dom)
    # DF-JK: J's second pass (GEMV over the packed rows) and K's stages
    # (stage 1 reads the B slices once), both HBM rooflines
    djk = last["dfjk"]
    roof_dfj = {"bound": "hbm", "kernel": "DF-J second pass", "ms": djk["aux_ms"],
                "achieved": djk["aux_bytes"] / (djk["aux_ms"] * 1e-3) / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s"}
    roof_dfj["frac"] = roof_dfj["achieved"] / roof_dfj["peak"]
    roof_dfk = {"bound": "hbm", "kernel": "DF-K stages (stage 1 reads B once)", "ms": djk["main_ms"],
                "achieved": djk["main_bytes"] / (djk["main_ms"] * 1e-3) / 1e9, "peak": peaks["hbm_gbs"],
                "unit": "GB/s"}
    roof_dfk["frac"] = roof_dfk["achieved"] / roof_dfk["peak"]

    # ---- one FP64-plain step on the same inputs (the "mixed vs FP64 plain" ratio)
    plain = None
    if prec != "f64" and not args.no_plain:
        sp_r, sp_j, sp_k = {}, {}, {}
        jk64 = DfJK(inp["bjk"], layout="square", precision="f64")
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        sc64, g64, _, _ = rimp2.rimp2_energy_grad(inp["b_ov"], inp["eo"], inp["ev"], precision="f64", stats=sp_r)
        j64, k64 = jk64.jk_from_occ(inp["c"], stats=sp_j)
        p1.record(stream)
        torch.cuda.synchronize()
        pms = p0.elapsed_time(p1)
        cm = {"rimp2_e_grad": last["rimp2"]["kernel_ms"], "dfjk": last["dfjk"]["kernel_ms"]}
        plain = {"ms_per_step": pms, "value": flops["total"] / (pms * 1e-3) / 1e12, "unit": "TFLOP/s",
                 "speedup_mixed_vs_plain": pms / ms_step,
                 "speedup_rimp2_e_grad": sp_r["kernel_ms"] / cm["rimp2_e_grad"],
                 "speedup_dfjk": sp_j["kernel_ms"] / cm["dfjk"],
                 "components_ms": {"rimp2_e_grad": sp_r["kernel_ms"], "dfjk": sp_j["kernel_ms"],
                                   "dfk_stages": sp_j["main_ms"], "dfj_pass2": sp_j["aux_ms"]},
                 "mixed_error": {"e_total_abs": (sc.e_os + sc.e_ss) - sc64.e_total,
                                 "e_os_abs": sc.e_os - sc64.e_os, "e_ss_abs": sc.e_ss - sc64.e_ss,
                                 "e_corr_f64": sc64.e_total,
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
            s2 = FcStats()
            jk.set_precision(dfk_prec)
            check(_lib.lib.fc_dfjk_build_occ(jk._h, ptr(hc), DFJK["nocc"], ptr(hj), ptr(hk), ctypes.byref(s2)))
            return s.h2d_bytes + s2.h2d_bytes, s.d2h_bytes + s2.d2h_bytes

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
        host = host_inputs_from(torch, inp)
        v, secs, cores, desc = cpu_sample(host)
        cpu = {"value": v, "unit": "TFLOP/s", "cores": cores, "kind": "port",
               "sample": desc, "seconds_per_step": secs}
        del host

    jk.close()
    del gamma, inp
    torch.cuda.empty_cache()
    # ---- config 5: C20H42 def2-TZVP shapes, mixed vs FP64 plain
    c5 = None
    if prec == "mixed" and args.size == "full" and not args.no_c5:
        c5 = c5_leg(torch, dev, prec)

    # ---- DF-JK builds one after another, as the SCF runs them (config 2)
    dfjk_alone = None
    if prec == "mixed" and args.size == "full":
        dfjk_alone = dfjk_leg(torch, dev, prec, local)

    # ---- the gradient with the full densities, config-3 RI-MP2 shapes
    dens = None
    if prec == "mixed" and args.size == "full" and not args.no_dens:
        dens = dens_leg(torch, dev, prec)

    # ---- config 4: batched RI-MP2 E+grad over 512 molecules of uneven size
    batch = None
    if prec == "mixed" and not args.no_batch:
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
                      "mixed": ("int8 integer slices, exact int32 accumulation, f64 epilogue (pair kernel: 4 slices, "
                                "10 products; adjoint: 3 slices, 6 products)")}[prec],
            "precision": prec, "dfj_precision": dfj_prec, "dfk_precision": dfk_prec,
            "data": "synthetic (seeded, generated on device)", "config": config,
            "components_ms": {"rimp2_e_grad": last["rimp2"]["kernel_ms"], "dfjk": last["dfjk"]["kernel_ms"],
                              "dfk_stages": last["dfjk"]["main_ms"], "dfj_pass2": last["dfjk"]["aux_ms"]},
            "flops": flops, "energy": {"e_os": sc.e_os, "e_ss": sc.e_ss},
            "roofline": roofline, "roofline_kernels": rooflines, "roofline_dfj": roof_dfj, "roofline_dfk": roof_dfk,
            "plain_f64": plain,
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
            "config4_batch": batch, "config5": c5, "mo_dressing": dress, "densities": dens,
            "dfjk_builds": dfjk_alone,
        }
        print(json.dumps(out))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
