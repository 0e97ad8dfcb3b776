"""Benchmark of the libOMM hot path on B200: omm() CG iterations per second and
time to a 1e-9 relative energy change, plus the SpMM's HBM bandwidth.

A step is one complete omm() solve of the workload from the reference's own
start (LCG C0 under NORAND, new_S, dealloc), to the reference's default
tolerance cg_tol = 1e-9; `value` = CG iterations of all ranks / max-over-ranks
device time.  Inputs (H, S as CSC, and every work matrix) live in HBM before
the timed region; every input matrix is larger than the 126 MB L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload lattice_8x8x8] [--label gpu|gmx]

Multi-GPU: one process per GPU, each solving its own spin/k-point problem
(the reference's independent `ip` units, omm.F90:34-35); no collective on the
data path.  The reference arm times the CPU restatement of libOMM (oracle/,
dense BLAS on the host OpenBLAS, all host threads) on a bounded sample of CG
steps of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "omm-bundle_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

METRIC = "omm_cg_iters_per_s"
# DRAM bytes (read + write) of one spmm_tc_kernel launch of the roofline below, from an ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of `python bench.py --roofline-only --workload W`;
# None when not captured
SPMM_TC_TRAFFIC: dict = {"lattice_8x8x8": 231130624 + 248416768}
# the same for the dominant kernel of the FP64 solve, keyed by (kernel, workload)
KERNEL_TRAFFIC: dict = {}
UNIT = "CG iterations/s"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=6)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def combine_ranks(ms: float, iters: float, world: int, device: str = "cuda"):
    """Whole-job numbers: (max device time over ranks in ms, sum of CG iterations over ranks).

    Every rank calls this once, in the same order (two all-reduces)."""
    if world <= 1:
        return float(ms), float(iters)
    import torch
    import torch.distributed as dist

    mx = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    sm = torch.tensor([float(iters)], dtype=torch.float64, device=device)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(sm[0])


def spmm_algorithmic_bytes(nnz: int, m: int, n: int, val_b: int, in_b: int, out_b: int) -> int:
    # nnz*(val + 4-byte row index) + (m+1)*4 column pointers + input n x m + output n x m
    return nnz * (val_b + 4) + (m + 1) * 4 + n * m * in_b + n * m * out_b


def spmm_tc_algorithmic_bytes(nnz: int, m: int, n: int) -> int:
    # the solver's fused product [HC, SC] = C [H, S]: two CSC operands (bf16 values + 4-byte row
    # indices + column pointers), the bf16 input read once, two FP64 outputs
    return 2 * (nnz * (2 + 4) + (m + 1) * 4) + n * m * 2 + 2 * n * m * 8


def spmm_rooflines(G, torch, stream, p, Hg, Sg, csc, lab, reps=20):
    """Roofline of the tensor-core SpMM the mixed solver runs every CG step (fused H and S,
    bf16 operands, FP32 accumulation, FP64 output), timed alone with CUDA events on the
    library's stream; the FP64 SpMM (psp_gemspm of C*H, FP64 tensor cores) beside it."""
    if not csc:
        return None, {}
    m, n = p.m, p.n
    hbm, bf16, peak_kind = peaks()
    Cd = G.Matrix.from_numpy(np.asfortranarray(np.random.default_rng(0).standard_normal((n, m)) * 1e-2))
    O1, O2 = G.Matrix.allocate(n, m, lab), G.Matrix.allocate(n, m, lab)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    roof = None
    if p.is_real:
        G.spmm_lowp_prepare(Cd, 1)
        for _ in range(3):
            G.spmm_lowp_apply(Hg, O1, 1, B2=Sg, C2=O2)
        if G.tc_errors():
            raise RuntimeError("tensor-core SpMM reported a timed-out pipeline wait")
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(reps):
            G.spmm_lowp_apply(Hg, O1, 1, B2=Sg, C2=O2)
        b.record(stream)
        torch.cuda.synchronize()
        if G.tc_errors():
            raise RuntimeError("tensor-core SpMM reported a timed-out pipeline wait")
        sec = a.elapsed_time(b) / 1e3 / reps
        byt = spmm_tc_algorithmic_bytes(p.H.nnz, m, n)
        gbs = byt / sec / 1e9
        roof = {"bound": "hbm", "achieved": round(gbs, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(gbs / hbm, 4), "traffic": SPMM_TC_TRAFFIC.get(p.name),
                "kernel": "spmm_tc_kernel<1,4,1> ([HC, SC] = C [H, S] in one N = 2G MMA per row block, bf16 in, FP32 accumulate, FP64 out)",
                "algorithmic_bytes_per_launch": byt, "peak_kind": peak_kind, "ms_per_launch": round(sec * 1e3, 4),
                "tensor_tflops": round(2.0 * 2 * p.H.nnz * n / sec / 1e12, 2)}
    extra = {}
    if p.is_real:
        extra["spmm_tc_f32"] = spmm_tc2_roofline(G, torch, stream, p, Hg, Sg, hbm, peak_kind, reps, groups=1)
        extra["spmm_tc_groups"] = spmm_tc2_roofline(G, torch, stream, p, Hg, Sg, hbm, peak_kind, reps, groups=4)
    # FP64 SpMM (psp_gemspm of C*H) on the FP64 tensor cores (DMMA): reported in TFLOP/s too
    for _ in range(3):
        G.psp_gemspm(n, m, m, Cd, "n", Hg, "n", O1, 1.0, 0.0)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps // 2):
        G.psp_gemspm(n, m, m, Cd, "n", Hg, "n", O1, 1.0, 0.0)
    b.record(stream)
    torch.cuda.synchronize()
    sec = a.elapsed_time(b) / 1e3 / (reps // 2)
    byt = spmm_algorithmic_bytes(p.H.nnz, m, n, 8, 8, 8)
    extra.update({"spmm_fp64": {"kernel": "cgu_dmma_kernel<G,1> (C*H, psp_gemspm, FP64 tensor cores)", "ms": round(sec * 1e3, 4),
                           "achieved_gbs": round(byt / sec / 1e9, 1), "hbm_frac": round(byt / sec / 1e9 / hbm, 4),
                           "fp64_tflops": round(2.0 * p.H.nnz * n / sec / 1e12, 3)}})
    if p.is_real:
        extra["spmm_fp64_int8"] = spmm_f64_timing(G, torch, stream, p, Hg, Sg, Cd, reps // 2)
    del Cd, O1, O2
    extra["gemm_bf16"] = gemm_roofline(G, torch, stream, 2 * n, n, m, bf16)
    if p.is_real:
        extra["gemm_fp64_int8"] = gemm_f64_timing(G, torch, stream, 2 * n, n, m)
    return roof, extra


def spmm_f64_timing(G, torch, stream, p, Hg, Sg, Cd, reps):
    """The FP64 CG step's [HG; SG] = D [H, S] on the int8 tensor cores (omm_gpu_spmm_f64: D's
    residues with their k-blocked copy, 16 int8 SpMMs, the CRT reconstruction of both halves),
    whole and per kernel (the library's CUDA events), against the FP64 DMMA SpMM of both."""
    import ctypes as ct

    L = G.lib()
    f = L.omm_gpu_spmm_f64
    f.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int]
    f.restype = ct.c_int
    n, m = p.n, p.m
    Y = torch.empty(m, 2 * n, device="cuda", dtype=torch.float64)
    ptr = Cd.device_ptr()

    def run():
        rc = f(ptr, n, n, Hg.h, Sg.h, Y.data_ptr(), 2 * n)
        if rc != 0:
            raise RuntimeError(L.omm_gpu_last_error().decode())

    def timed():
        for _ in range(2):
            run()
        torch.cuda.synchronize()
        kt = kernel_timing(G, True)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            run()
        b.record(stream)
        torch.cuda.synchronize()
        ks = kt.read(1.0)
        L.omm_gpu_kernel_timing(0)
        per = {nm: round(k["ms"] / k["launches"], 4) for nm, k in ks.items()}
        return a.elapsed_time(b) / 1e3 / reps, per

    # the kernel's other forms (one column group per CTA with one chunk pair per stage, two groups
    # per CTA) for comparison, then the default (one group, three chunk pairs per stage)
    forms = {}
    for form, name in ((0, "one_group_one_pair_per_stage"), (2, "two_groups_per_cta")):
        L.omm_gpu_set_oz_spmm_form(form)
        _, perf = timed()
        forms[name] = perf.get("oz_spmm_kernel")
    L.omm_gpu_set_oz_spmm_form(1)
    sec, per = timed()
    fl = 2.0 * (p.H.nnz + p.S.nnz) * n
    out = {"what": "[HG; SG] = D [H, S] in FP64: residues of D + oz_spmm_kernel + 2 reconstructions",
           "ms": round(sec * 1e3, 4), "fp64_equivalent_tflops": round(fl / sec / 1e12, 2),
           "ms_per_launch": per, "oz_spmm_kernel_ms_other_forms": forms}
    if "oz_spmm_kernel" in per:
        out["oz_spmm_kernel_ms"] = per["oz_spmm_kernel"]
    return out


def int8_peak(torch, stream, n=8192, reps=10):
    """Dense int8 tensor throughput of this GPU as the vendor library reaches it: torch._int_mm
    (cuBLASLt, int8 x int8 -> int32) at n^3, best of reps launches; the denominator of the int8
    GEMM's roofline (the driver's peak file measures bf16 and HBM only)."""
    try:
        g = torch.Generator(device="cuda").manual_seed(7)
        a = torch.randint(-128, 128, (n, n), generator=g, device="cuda", dtype=torch.int8)
        b = torch.randint(-128, 128, (n, n), generator=g, device="cuda", dtype=torch.int8).t()
        for _ in range(3):
            torch._int_mm(a, b)
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            torch._int_mm(a, b)
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            best = t if best is None else min(best, t)
        return round(2.0 * n ** 3 / best / 1e12, 1)
    except Exception as exc:  # no int8 GEMM in this torch build
        return "unavailable: %s" % str(exc)[:80]


def gemm_f64_timing(G, torch, stream, M, N, K, reps=10):
    """The FP64 product on the int8 tensor cores (residues of both operands, 16 int8 tcgen05
    GEMMs, CRT reconstruction) at the Gram shape [HWd; SWd] = X D^T, timed whole with CUDA
    events on the library stream, against torch's cuBLAS DGEMM at the same shape."""
    import ctypes as ct

    L = G.lib()
    f = L.omm_gpu_gemm_f64_async
    f.argtypes = [ct.c_char, ct.c_char, ct.c_int, ct.c_int, ct.c_int, ct.c_double, ct.c_void_p, ct.c_int,
                  ct.c_void_p, ct.c_int, ct.c_double, ct.c_void_p, ct.c_int]
    f.restype = ct.c_int
    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn(K, M, generator=g, device="cuda", dtype=torch.float64)  # column-major M x K
    D = torch.randn(K, N, generator=g, device="cuda", dtype=torch.float64)  # column-major N x K
    out = torch.empty(N, M, device="cuda", dtype=torch.float64)

    def run():
        rc = f(b"n", b"t", M, N, K, 1.0, X.data_ptr(), M, D.data_ptr(), N, 0.0, out.data_ptr(), M)
        if rc != 0:
            raise RuntimeError(L.omm_gpu_last_error().decode())

    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        run()
    b.record(stream)
    torch.cuda.synchronize()
    if G.tc_errors():
        raise RuntimeError("int8 tcgen05 GEMM reported a timed-out pipeline wait")
    sec = a.elapsed_time(b) / 1e3 / reps
    ref = X.t() @ D
    for _ in range(2):
        ref = X.t() @ D
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        ref = X.t() @ D
    b.record(stream)
    torch.cuda.synchronize()
    sec_ref = a.elapsed_time(b) / 1e3 / reps
    fl = 2.0 * M * N * K
    i8 = int8_peak(torch, stream)
    return {"kernels": "oz_exp/oz_res (residues) + oz_gemm_pair_kernel (16 int8 tcgen05 GEMMs on SM pairs) + "
                       "oz_reconstruct_kernel",
            "int8_reference_tops": i8,
            "shape": [M, N, K], "ms": round(sec * 1e3, 4), "fp64_equivalent_tflops": round(fl / sec / 1e12, 2),
            "int8_tops_incl_residues": round(16 * fl / sec / 1e12, 1),
            "cublas_dgemm_ms": round(sec_ref * 1e3, 4), "cublas_dgemm_tflops": round(fl / sec_ref / 1e12, 2)}


def spmm_tc2_algorithmic_bytes(nnz: int, m: int, n: int) -> int:
    # [HC, SC] = C [H, S] as the mixed CG step runs it: two CSC operands (bf16 values + 4-byte row
    # indices + column pointers), the bf16 input read once, two FP32 outputs
    return 2 * (nnz * (2 + 4) + (m + 1) * 4) + n * m * 2 + 2 * n * m * 4


def spmm_tc2_roofline(G, torch, stream, p, Hg, Sg, hbm, peak_kind, reps=20, groups=4):
    """The mixed solver's per-step SpMM (FP32 out, plus the Gram's bf16 shadows of the result) on
    the operand prepared by spmm_lowp_prepare, timed alone with CUDA events on the library
    stream: groups = 1, spmm_tc_kernel (one column group per CTA), or 4, spmm_tc2_kernel
    (blocks of four column groups)."""
    import ctypes as ct

    L = G.lib()
    L.omm_gpu_set_spmm_groups(groups)
    f = L.omm_gpu_spmm_lowp_apply_f32
    f.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_int]
    f.restype = ct.c_int
    m, n = p.m, p.n
    Y = torch.empty(m, 2 * n, device="cuda", dtype=torch.float32)
    ldt = (m + 7) // 8 * 8
    th = torch.empty(2 * n, ldt, device="cuda", dtype=torch.bfloat16)

    def run(shadow):
        rc = f(Hg.h, Sg.h, Y.data_ptr(), 2 * n, th.data_ptr() if shadow else None, None, ldt, 1)
        if rc != 0:
            raise RuntimeError(L.omm_gpu_last_error().decode())

    out = {}
    for shadow in (False, True):
        for _ in range(3):
            run(shadow)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            run(shadow)
        b.record(stream)
        torch.cuda.synchronize()
        if G.tc_errors():
            raise RuntimeError("tensor-core SpMM reported a timed-out pipeline wait")
        out[shadow] = a.elapsed_time(b) / 1e3 / reps
    L.omm_gpu_set_spmm_groups(1)
    byt = spmm_tc2_algorithmic_bytes(p.H.nnz, m, n)
    gbs = byt / out[False] / 1e9
    what = ("spmm_tc2_kernel<1,8> ([HC, SC] = C [H, S], CTAs of 4 column groups, bf16 in, FP32 out)" if groups == 4
            else "spmm_tc_kernel<1,4,1> ([HC, SC] = C [H, S], one column group per CTA, bf16 in, FP32 out)")
    return {"bound": "hbm", "achieved": round(gbs, 1), "peak": hbm, "unit": "GB/s", "frac": round(gbs / hbm, 4),
            "kernel": what,
            "algorithmic_bytes_per_launch": byt, "peak_kind": peak_kind, "ms_per_launch": round(out[False] * 1e3, 4),
            "ms_with_gram_shadows": round(out[True] * 1e3, 4), "shadow_bytes": 2 * n * m * 2,
            "tensor_tflops": round(2.0 * 2 * p.H.nnz * n / out[False] / 1e12, 2)}


def gemm_roofline(G, torch, stream, M, N, K, peak, reps=20):
    """The tcgen05 BF16 GEMM at the shape of the solver's Gram products ([HWd; SWd] = X D^T:
    M = 2n, N = n, K = m), bf16 operands, FP64 output, timed alone with CUDA events."""
    import ctypes as ct

    L = G.lib()
    f = L.omm_gpu_gemm_bf16_async
    f.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p,
                  ct.c_int, ct.c_int, ct.c_double, ct.c_double, ct.c_void_p, ct.c_int]
    f.restype = ct.c_int
    ld = (K + 7) // 8 * 8
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(M, ld, generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn(N, ld, generator=g, device="cuda").to(torch.bfloat16)
    out = torch.empty(N, M, device="cuda", dtype=torch.float64)

    def run():
        rc = f(M, N, K, A.data_ptr(), None, ld, B.data_ptr(), None, ld, 1, 1.0, 0.0, out.data_ptr(), M)
        if rc != 0:
            raise RuntimeError(L.omm_gpu_last_error().decode())

    def timed(pairs):
        L.omm_gpu_tc_set_pairs(pairs)
        try:
            for _ in range(3):
                run()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(reps):
                run()
            b.record(stream)
            torch.cuda.synchronize()
        finally:
            L.omm_gpu_tc_set_pairs(1)
        if G.tc_errors():
            raise RuntimeError("tcgen05 GEMM reported a timed-out pipeline wait")
        return a.elapsed_time(b) / 1e3 / reps

    sec1 = timed(0)
    sec = timed(1)
    tf = 2.0 * M * N * K / sec / 1e12
    return {"kernel": "gemm_bf16_pair_kernel (Gram product, M=2n N=n K=m, bf16 in, FP64 out; 256 x 256 tiles "
                      "on SM pairs)", "bound": "tensor", "one_sm_kernel_ms": round(sec1 * 1e3, 4),
            "ms": round(sec * 1e3, 4), "achieved_tflops": round(tf, 1), "peak_tflops": peak,
            "frac": round(tf / peak, 4)}


# --------------------------------------------------------------------------- target configs
def density_rel_diff(torch, D, Dref, m):
    """Relative Frobenius difference of two m x m device densities, in column slabs."""
    num = den = 0.0
    for j0 in range(0, m, 1024):
        num += float(torch.linalg.norm(D[j0:j0 + 1024] - Dref[j0:j0 + 1024])) ** 2
        den += float(torch.linalg.norm(Dref[j0:j0 + 1024])) ** 2
    return (num / den) ** 0.5 if den > 0 else None


def targets_block(G, torch, stream, names):
    """The metric's target comparison on further workloads, in the same invocation: for each,
    one untimed and one timed solve with the FP64 path ("gpu") and with the mixed solver
    ("gmx"), each from the reference's start to cg_tol = 1e-9, timed with CUDA events on the
    library stream; energies against the dense eigensolver's band energy and the mixed
    density against the FP64 one."""
    from ommgpu import synth

    out = {}
    for name in names:
        w0 = time.perf_counter()
        p = synth.workload(name)
        gen_s = time.perf_counter() - w0
        m, n = p.m, p.n
        csc = isinstance(p.H, synth.CSCMatrix)
        Hg = G.Matrix.from_csc(p.H) if csc else G.Matrix.from_numpy(p.H)
        Sg = G.Matrix.from_csc(p.S) if csc else G.Matrix.from_numpy(p.S)
        lab = "gdden" if p.is_real else "gzden"
        Dt = torch.empty(m, m, dtype=torch.float64 if p.is_real else torch.complex128, device="cuda")
        Dg = G.Matrix.register_gden(Dt.data_ptr(), m, m, not p.is_real, keep=Dt)
        Cg = G.Matrix.allocate(n, m, lab)
        res = {}
        for label in ("gpu", "gmx"):
            times = []
            for _ in range(2):  # the first solve is the warm-up
                torch.cuda.synchronize()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                e, rc = G.omm(m, n, Hg, Sg, True, Dg, False, 0.0, Cg, False, dealloc=True, m_operation=label,
                              m_storage=lab)
                b.record(stream)
                torch.cuda.synchronize()
                if rc != 0:
                    raise RuntimeError("omm did not converge (%s, %s)" % (name, label))
                times.append(a.elapsed_time(b) / 1e3)
            st = G.stats()
            res[label] = {"time_to_tol_s": round(times[-1], 4), "cg_steps": st["icg"],
                          "iters_per_s": round(st["icg"] / times[-1], 3), "energy": e,
                          "energy_rel_err_vs_eigensolver": abs(e - p.e_exact) / abs(p.e_exact),
                          "steps_bf16_or_split": st["icg_low"], "steps_refined": st["icg_fp64"]}
            if label == "gpu":
                D64 = Dt.clone()
        dd = density_rel_diff(torch, Dt, D64, m)
        del D64, Dg, Dt
        torch.cuda.empty_cache()
        g64, gmx = res["gpu"], res["gmx"]
        out[name] = {"m": m, "n": n, "nnz": p.H.nnz if csc else m * m,
                     "fp64": {k: g64[k] for k in ("time_to_tol_s", "cg_steps", "iters_per_s",
                                                  "energy_rel_err_vs_eigensolver")},
                     "mixed": {k: gmx[k] for k in ("time_to_tol_s", "cg_steps", "iters_per_s", "steps_bf16_or_split",
                                                   "steps_refined", "energy_rel_err_vs_eigensolver")},
                     "speedup_mixed_vs_fp64": round(g64["time_to_tol_s"] / gmx["time_to_tol_s"], 3),
                     "energy_rel_diff_mixed_vs_fp64": abs(gmx["energy"] - g64["energy"]) / abs(g64["energy"]),
                     "density_rel_frobenius_diff_mixed_vs_fp64": dd,
                     "generation_s": round(gen_s, 2)}
    return out


class kernel_timing:
    """omm_gpu_kernel_timing: CUDA events the library records on its stream around each launch of
    its dominant kernels, with each launch's algorithmic work."""

    NAMES = ("cgu_dmma_kernel", "oz_spmm_kernel", "oz_gemm_pair_kernel", "oz_gemm_kernel", "spmm_tc_kernel",
             "spmm_tc2_kernel", "gemm_bf16_pair_kernel", "gemm_bf16_kernel", "oz_exp_kernel", "oz_res_rows_kernel",
             "oz_res_kc_kernel", "oz_reconstruct_kernel", "oz_axpby_exps_kernel")

    def __init__(self, G, on):
        import ctypes as ct

        self.L = G.lib()
        self.L.omm_gpu_kernel_timing(int(on))

    def read(self, ms_per_solve):
        import ctypes as ct

        out = {}
        for nm in self.NAMES:
            n, ms, w = ct.c_longlong(), ct.c_double(), ct.c_double()
            self.L.omm_gpu_kernel_timing_get(nm.encode(), ct.byref(n), ct.byref(ms), ct.byref(w))
            if n.value:
                out[nm] = {"launches": n.value, "ms": ms.value, "work": w.value}
        return out


def fp64_peak(torch, stream, n=8192, reps=5):
    """FP64 tensor throughput as the vendor library reaches it: cuBLAS DGEMM (torch.matmul on
    float64) at n^3, best of reps; the denominator of the FP64 SpMM's roofline (the peak file
    measures bf16 and HBM only)."""
    g = torch.Generator(device="cuda").manual_seed(9)
    a = torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64)
    b = torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64)
    for _ in range(2):
        torch.matmul(a, b)
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        torch.matmul(a, b)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        best = t if best is None else min(best, t)
    return round(2.0 * n ** 3 / best / 1e12, 2)


HBM_PASSES = {
    "oz_exp_kernel": "oz_exp_rows_kernel / oz_exp_kc_kernel (binary exponents of the rows of an FP64 operand)",
    "oz_res_rows_kernel": "oz_res_rows_kernel (16 int8 residue planes of a row-contiguous FP64 operand)",
    "oz_res_kc_kernel": "oz_res_kc_kernel (16 int8 residue planes of a K-contiguous FP64 operand)",
    "oz_reconstruct_kernel": "oz_reconstruct_kernel (FP64 outputs from 16 residue planes by the CRT)",
    "oz_axpby_exps_kernel": "oz_axpby_exps_kernel (the step's D and X updates with the exponents of the result's "
                            "rows and columns)",
}


def solve_roofline(ktimes, torch, stream, p):
    """The roofline of the timed FP64 solve's dominant kernel (the largest summed event time of
    the instrumented kernels), from the library's events inside the timed region: achieved =
    summed algorithmic work / summed launch time, against the vendor library's measured rate of
    the same pipe in this run (cuBLAS DGEMM for the FP64 tensor pipe, cuBLASLt int8 for int8)."""
    if not ktimes:
        return None, {}
    rows = {}
    for nm, k in ktimes.items():
        sec = k["ms"] / 1e3
        if nm == "cgu_dmma_kernel":
            peak = fp64_peak(torch, stream)
            ach = k["work"] / sec / 1e12
            rows[nm] = {"bound": "tensor", "achieved": round(ach, 2), "peak": peak, "unit": "TFLOP/s",
                        "frac": round(ach / peak, 4), "peak_kind": "cuBLAS DGEMM 8192^3 in this run (FP64 tensor)",
                        "kernel": "cgu_dmma_kernel<G,2> (FP64 [HG, SG] = D [H, S] on DMMA, mma.sync m8n8k4 f64)"}
        elif nm == "oz_spmm_kernel":
            # work counted as the FP64 flops of the product it computes (2 nnz n), so that its rate
            # reads against the FP64 tensor pipe of the DMMA SpMM it replaces
            peak = fp64_peak(torch, stream)
            ach = k["work"] / sec / 1e12
            rows[nm] = {"bound": "tensor", "achieved": round(ach, 2), "peak": peak, "unit": "TFLOP/s (FP64 equivalent)",
                        "frac": round(ach / peak, 4),
                        "peak_kind": "cuBLAS DGEMM 8192^3 in this run (the FP64 rate of the SpMM it replaces)",
                        "kernel": "oz_spmm_kernel (FP64 [HG, SG] = D [H, S] as 16 int8 tcgen05 SpMMs, excluding the "
                                  "residue and reconstruction passes)"}
        elif nm in ("oz_gemm_kernel", "oz_gemm_pair_kernel"):
            peak = int8_peak(torch, stream)
            if not isinstance(peak, float):
                continue
            ach = k["work"] / sec / 1e12
            what = ("256 x 256 tiles on SM pairs, cta_group::2" if nm == "oz_gemm_pair_kernel"
                    else "128 x 256 tiles, one SM each")
            rows[nm] = {"bound": "tensor", "achieved": round(ach, 1), "peak": peak, "unit": "TOP/s (int8)",
                        "frac": round(ach / peak, 4), "peak_kind": "cuBLASLt int8 GEMM 8192^3 in this run",
                        "kernel": "%s (persistent tcgen05 kind::i8, %s; 16 moduli of the FP64 products)" % (nm, what)}
        elif nm in HBM_PASSES:
            # the passes around the int8 products: FP64 operands in, residue planes out (or back)
            peak = peaks()[0]
            ach = k["work"] / sec / 1e9
            rows[nm] = {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(ach / peak, 4), "peak_kind": "measured" if peaks()[2] == "measured" else "fallback",
                        "kernel": HBM_PASSES[nm]}
        else:
            continue
        rows[nm].update({"launches": k["launches"], "ms_per_launch": round(k["ms"] / k["launches"], 4),
                         "ms_total": round(k["ms"], 2), "algorithmic_work_per_launch": k["work"] / k["launches"],
                         "traffic": None})
    if not rows:
        return None, {}
    top = max(rows, key=lambda nm: ktimes[nm]["ms"])
    others = {nm: r for nm, r in rows.items() if nm != top}
    return rows[top], others


# --------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch

    import ommgpu as G
    from ommgpu import synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    G.lib().omm_gpu_set_device(local)
    # the library runs on an explicit torch stream so that the CUDA events below
    # bracket its kernels (torch's default stream is the legacy NULL stream)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    G.set_stream(stream.cuda_stream)
    G.set_log(None)

    p = synth.workload(args.workload)
    m, n = p.m, p.n
    csc = isinstance(p.H, synth.CSCMatrix)
    Hg = G.Matrix.from_csc(p.H) if csc else G.Matrix.from_numpy(p.H)
    Sg = G.Matrix.from_csc(p.S) if csc else G.Matrix.from_numpy(p.S)
    H0, S0 = Hg, Sg  # as generated (CSC for the lattices): the roofline and the adjoint use these
    lab = "gdden" if p.is_real else "gzden"
    if args.roofline_only:
        roof, extra = spmm_rooflines(G, torch, stream, p, Hg, Sg, csc, lab)
        if rank == 0:
            print(json.dumps({"workload": args.workload, "roofline": roof, **extra}))
        return
    if args.profile_solve:
        # for launch lists under a profiler: --warmup solves, then one more, of the given label
        Cg = G.Matrix.allocate(n, m, lab)
        Dg = G.Matrix.allocate(m, m, lab)
        for _ in range(args.warmup + 1):
            e, rc = G.omm(m, n, Hg, Sg, True, Dg, False, 0.0, Cg, False, dealloc=True,
                          m_operation=args.profile_solve, m_storage=lab)
        torch.cuda.synchronize()
        print(json.dumps({"workload": args.workload, "label": args.profile_solve, "energy": e, "rc": rc,
                          "cg_steps": G.stats()["icg"]}))
        return
    reset = None
    Dt = None
    if args.flavour in (1, 2) and csc:
        # the Cholesky flavours factor S and transform H in place (omm.F90:306-309) and need them
        # dense (the reference dies on CSC, omm_ops.F90:444-476): dense device copies, rebuilt from
        # the CSC before every solve, outside the timed region
        Hd = torch.empty(m, m, dtype=torch.float64, device="cuda")
        Sd = torch.empty(m, m, dtype=torch.float64, device="cuda")
        fills = [(t, synth.csc_device_index(A, "cuda")) for t, A in ((Hd, p.H), (Sd, p.S))]

        def reset():
            for t, (rows, cols, vals) in fills:
                t.zero_()
                t[cols, rows] = vals  # row-major (m, m) storage = the column-major matrix
            torch.cuda.synchronize()

        Hg = G.Matrix.register_gden(Hd.data_ptr(), m, m, False, keep=Hd)
        Sg = G.Matrix.register_gden(Sd.data_ptr(), m, m, False, keep=Sd)
    # D_min in a torch tensor handed to the library as device storage: the FP64 and mixed
    # densities are compared on the device after the timed solves
    Dt = torch.empty(m, m, dtype=torch.float64 if p.is_real else torch.complex128, device="cuda")
    Dg = G.Matrix.register_gden(Dt.data_ptr(), m, m, not p.is_real, keep=Dt)
    Cg = G.Matrix.allocate(n, m, lab)

    def solve(label):
        e, rc = G.omm(m, n, Hg, Sg, True, Dg, False, 0.0, Cg, False, dealloc=True, m_operation=label,
                      m_storage=lab, flavour=args.flavour)
        if rc != 0:
            raise RuntimeError("omm did not converge (%s)" % label)
        return e, G.stats()

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    def timed(label, steps, warmup):
        for _ in range(warmup):
            if reset:
                reset()
            solve(label)
        barrier()
        torch.cuda.synchronize()
        l0 = G.kernel_launches()
        kt = kernel_timing(G, True)  # CUDA events around the dominant kernels, inside the timed region
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        iters, energies, stats = 0, [], []
        ms = 0.0
        t0.record(stream)
        for _ in range(steps):
            if reset:  # inputs rebuilt between solves: each solve timed on its own
                t1.record(stream)
                torch.cuda.synchronize()
                ms += t0.elapsed_time(t1)
                reset()
                t0.record(stream)
            e, st = solve(label)
            iters += st["icg"]
            energies.append(e)
            stats.append(st)
        t1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms += t0.elapsed_time(t1)
        t_max, it_tot = combine_ranks(ms, iters, world, "cuda")
        ktimes = kt.read(ms / steps)
        kernel_timing(G, False)
        return {"ms_per_solve": t_max / steps, "iters_per_s": it_tot / (t_max / 1e3), "iters": iters / steps,
                "energy": energies[-1], "launches": G.kernel_launches() - l0, "stats": stats[-1],
                "kernels": ktimes}

    with ClockSampler(local) as clk:
        r64 = timed("gpu", args.steps, args.warmup)
        # the mixed solver takes real problems and complex ones with dense H and S
        do_mixed = p.is_real or not csc
        if do_mixed:  # the library's cached buffers back to the driver before the m x m copy
            G.finalize()
            torch.cuda.empty_cache()
        D64 = Dt.clone() if do_mixed else None
        rmx = timed("gmx", args.steps, args.warmup) if do_mixed else None
    dens_diff = None
    if rmx:  # relative Frobenius difference of the densities, in column slabs (no m x m temporary)
        G.finalize()  # the library's buffers back to the driver first: at large m both densities fill HBM
        torch.cuda.empty_cache()
        dens_diff = density_rel_diff(torch, Dt, D64, m)
        del D64
    main = rmx if (args.label == "gmx" and rmx) else r64
    value = main["iters_per_s"]
    ms_per_step = main["ms_per_solve"]
    launches = main["launches"]
    it_tot = main["iters"] * args.steps * world
    e_final = main["energy"]
    rel_err = abs(e_final - p.e_exact) / abs(p.e_exact) if p.e_exact else None
    mixed = None
    if rmx:
        st = rmx["stats"]
        mixed = {"time_to_tol_s": round(rmx["ms_per_solve"] / 1e3, 4),
                 "fp64_time_to_tol_s": round(r64["ms_per_solve"] / 1e3, 4),
                 "speedup_vs_fp64": round(r64["ms_per_solve"] / rmx["ms_per_solve"], 3),
                 "cg_steps": st["icg"], "steps_bf16_or_split": st["icg_low"], "steps_refined": st["icg_fp64"],
                 "fp64_cg_steps": r64["iters"],
                 "energy_rel_err_vs_eigensolver": abs(rmx["energy"] - p.e_exact) / abs(p.e_exact),
                 "energy_rel_diff_vs_fp64": abs(rmx["energy"] - r64["energy"]) / abs(r64["energy"]),
                 "density_rel_frobenius_diff_vs_fp64": dens_diff,
                 "phase_s": {"setup": round(st["t_setup"], 4), "cg": round(st["t_loop"], 4),
                             "density": round(st["t_final"], 4)},
                 "iters_per_s": round(rmx["iters_per_s"], 3)}

    spmm_roof, spmm_extra = spmm_rooflines(G, torch, stream, p, H0, S0, csc, lab)
    # the headline solve's dominant kernel, from the library's CUDA events inside the timed region
    roof, roof_others = solve_roofline(r64["kernels"], torch, stream, p)
    if roof is not None:
        roof["traffic"] = KERNEL_TRAFFIC.get((roof["kernel"].split(" ")[0].split("<")[0], p.name))
    if rmx:
        mixed["kernels_ms_per_solve"] = {nm: round(k["ms"] / args.steps, 3) for nm, k in rmx["kernels"].items()}

    # ---- dE/dtheta_k for the workload's perturbations V_k from the last solve's C (the adjoint
    # kernel, C recomputed into the density on the fly), against libOMM's gradient
    # Re sum conj(D_min) o V_k from the returned density
    adjoint = None
    if p.V and rank == 0:
        Vh = [G.Matrix.from_csc(v) for v in p.V]
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        grad = G.energy_adjoint(m, n, S0, Cg, Vh)
        torch.cuda.synchronize()
        t_adj = time.perf_counter() - w0
        worst = 0.0
        for k, V in enumerate(p.V):
            rows, cols, vals = synth.csc_device_index(V, "cuda")
            if Dt is not None:
                dv = Dt[cols, rows]  # row-major storage of the column-major D_min
            else:
                dv = torch.from_numpy(Dg.numpy()).cuda()[rows, cols]
            gd = float(torch.real(torch.sum(torch.conj(dv) * vals)).item())
            worst = max(worst, abs(grad[k] - gd) / max(1.0, abs(gd)))
        adjoint = {"perturbations": len(p.V), "seconds": round(t_adj, 4),
                   "max_rel_diff_vs_density_gradient": worst, "solver_of_C": "gmx" if rmx else "gpu"}

    # ---- end to end through the C ABI with host buffers (pinned): H/S registered from host CSC
    # arrays each step, C_min and D_min as host (sdden) matrices staged in and out.
    e2e = None
    if (rank == 0 or world > 1) and not args.no_e2e:
        hdt = torch.float64 if p.is_real else torch.complex128
        pin = lambda shape: torch.empty(shape[::-1], dtype=hdt, pin_memory=True).numpy().T  # noqa: E731
        Ch = pin((n, m))
        Dh = pin((m, m))
        Ch[:] = 0.0
        h2d = d2h = 0
        t_e2e = 0.0
        it_e2e = 0
        ksteps = max(1, min(args.steps, 3))
        pool0 = None
        for s_ in range(ksteps + 1):
            if s_ == 1:
                pool0 = G.pool_stats()
            torch.cuda.synchronize()
            w0 = time.perf_counter()
            if csc:
                Hh = G.Matrix.from_csc(p.H, "sdcsc")
                Sh = G.Matrix.from_csc(p.S, "sdcsc")
            else:
                Hh, Sh = G.Matrix.register_sden(p.H), G.Matrix.register_sden(p.S)
            e, rc = G.omm(m, n, Hh, Sh, True, G.Matrix.register_sden(Dh), False, 0.0, G.Matrix.register_sden(Ch),
                          False, dealloc=True, m_storage="sdden" if p.is_real else "szden", m_operation=args.label)
            w1 = time.perf_counter()
            if s_ > 0:  # the first call is a warm-up (plan build)
                t_e2e += w1 - w0
                it_e2e += G.stats()["icg"]
        es = 8 if p.is_real else 16
        if csc:
            h2d = 2 * (p.H.nnz * (es + 4) + (m + 1) * 4) + n * m * es
        else:
            h2d = 2 * m * m * es + n * m * es
        d2h = n * m * es + m * m * es
        e2e = {"value": round(it_e2e / t_e2e, 3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": round(1e3 * t_e2e / ksteps, 3), "steps": ksteps,
               "device_mallocs_per_step": round((G.pool_stats()["mallocs"] - pool0["mallocs"]) / ksteps, 1),
               "note": "one omm() call per step with host (pinned) buffers; wall clock"}

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.label != "gmx" else "bf16/f32 bulk + f64 refinement",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": args.workload, "m": m, "n": n, "nnz": p.H.nnz if csc else m * m,
                   "storage": "gdcsc" if csc else lab, "m_operation": args.label, "cg_tol": 1e-9,
                   "iters_per_solve": it_tot / (args.steps * world), "time_to_tol_s": round(ms_per_step / 1e3, 4),
                   "energy_rel_err_vs_eigensolver": rel_err, "parallelism": "one ip per GPU (replicas)",
                   "l2": "inputs larger than L2 (H, S CSC 233 MB, C 151 MB at m=12288)"},
        "roofline": roof, "rooflines_other_kernels": roof_others,
        "kernels_ms_per_solve": {nm: round(k["ms"] / args.steps, 3) for nm, k in r64["kernels"].items()},
        "spmm_tc_pergroup": spmm_roof, "e2e": e2e, "clocks": clk.summary(), "gpu_launches": launches,
        "mixed": mixed,
    }
    if adjoint:
        out["adjoint"] = adjoint
    if world == 1 and args.targets:
        del Dt, Dg
        torch.cuda.empty_cache()
        out["targets"] = targets_block(G, torch, stream, [t for t in args.targets.split(",") if t])
    if args.flavour:
        out["config"]["flavour"] = args.flavour
    out.update(spmm_extra)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(p, args, sample_steps=2)
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# --------------------------------------------------------------------------- CPU arms
def cpu_sample(p, steps: int, nthreads: int):
    """Time `steps` CG iterations of the oracle (CPU restatement of omm) on the workload.

    Two calls with a step cap (max_steps = 1 and 1 + steps) isolate the per-step time
    from the set-up (initial products, C0) that both calls share."""
    import oracle as O
    from ommgpu import synth

    def run(cap):
        orc = O.OmmOracle(nthreads=nthreads)
        C = np.zeros((p.n, p.m), dtype=np.float64 if p.is_real else np.complex128, order="F")
        D = np.zeros((p.m, p.m), dtype=C.dtype, order="F")
        if isinstance(p.H, synth.CSCMatrix):
            H = O.CSC(p.m, p.m, p.H.colptr, p.H.rowind, p.H.val.copy())
            S = O.CSC(p.m, p.m, p.S.colptr, p.S.rowind, p.S.val.copy())
        else:
            H, S = p.H.copy(order="F"), p.S.copy(order="F")
        t = time.perf_counter()
        orc.omm(p.m, p.n, H, S, True, D, False, 0.0, C, False, dealloc=True, max_steps=cap)
        return time.perf_counter() - t, orc.icg

    t1, i1 = run(1)
    t2, i2 = run(1 + steps)
    per = max(1e-9, (t2 - t1) / max(1, i2 - i1))
    return 1.0 / per, per, t1


def cpu_baseline(p, args, sample_steps=2):
    nth = os.cpu_count() or 1
    val, per, setup = cpu_sample(p, sample_steps, nth)
    return {"value": round(val, 5), "unit": UNIT, "cores": nth, "kind": "port",
            "sample": "%d CG steps of omm() on %s (m=%d, n=%d) after the initial products; "
                      "%.1f s per step, %.1f s set-up" % (sample_steps, args.workload, p.m, p.n, per, setup)}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    from ommgpu import synth

    p = synth.workload(args.workload)
    nth = os.cpu_count() or 1
    # a bounded sample: warmup and steps count CG iterations of the CPU restatement
    steps = max(1, min(args.steps, 4))
    val, per, setup = cpu_sample(p, steps, nth)
    out = {"impl": "reference", "metric": METRIC, "value": round(val, 5), "unit": UNIT, "n_gpus": world,
           "steps": steps, "warmup": args.warmup, "ms_per_step": round(per * 1e3, 1), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
           "config": {"workload": args.workload, "m": p.m, "n": p.n, "cg_tol": 1e-9,
                      "note": "CPU restatement of libOMM omm() (reference is Fortran; no Fortran compiler here)"},
           "cpu_baseline": {"value": round(val, 5), "unit": UNIT, "cores": nth, "kind": "port",
                            "sample": "%d CG steps after the initial products" % steps},
           "e2e": {"value": round(val, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def spawn_ranks(n: int) -> int:
    """--gpus N with no outer launcher: start N copies of this command, one per GPU, with
    RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR=127.0.0.1 / MASTER_PORT set the way torchrun
    sets them.  Rank 0's stdout is this process's; if a rank fails, the others are stopped
    (by their own PIDs) and its exit code is returned."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + sys.argv[1:], env=env,
                                      stdout=None if r == 0 else subprocess.DEVNULL))
    rc = 0
    live = list(procs)
    while live:
        for pr in list(live):
            code = pr.poll()
            if code is None:
                continue
            live.remove(pr)
            if code != 0 and rc == 0:
                rc = code
                for other in live:
                    other.kill()
        time.sleep(0.05)
    return rc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="lattice_8x8x8")
    ap.add_argument("--label", default="gpu", choices=["gpu", "gmx"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--flavour", type=int, default=0, help="omm flavour (1: Cholesky, on dense device copies)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end solves")
    ap.add_argument("--targets", default="lattice_16x8x8,zdense_4096",
                    help="further workloads whose FP64 and mixed solves are reported in the 'targets' block "
                         "(comma-separated; empty to skip)")
    ap.add_argument("--profile-solve", default="", choices=["", "gpu", "gmx"],
                    help="run --warmup + 1 solves with this label and exit (for profiler launch lists)")
    ap.add_argument("--roofline-only", action="store_true",
                    help="time only the SpMM kernels of the roofline (for profiling them)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
