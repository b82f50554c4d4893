#!/usr/bin/env python
"""Benchmark of the selected-CI hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): the CSR Hamiltonian of the CAS(12e,12o) full-CI space --
853,776 determinants as bitset<64>, seeded synthetic integrals (seed 0,
orbital energies -1.5 + 2.5 p/(n-1), symmetric N(0, 0.02^2) one-electron
off-diagonals, (pq|rs) = sum_{L<2n} B^L_pq B^L_rs with B^L entries
N(0, (0.3 exp(-L/n))^2)), FP64 values, int32 indices, |h| > DBL_EPSILON.
With N GPUs each rank builds the row block of the reference's row partition
(make_dist_csr_hamiltonian) of the same matrix (strong scaling).

`value` is H-build nnz/s with the determinants resident in HBM; `e2e` is the
same through the C ABI with pinned host buffers (determinants in, full CSR
out). After the timed steps (rank 0, N = 1) the same run reports the SpMV,
FP64 and mixed-precision Davidson on this matrix and an ASCI search on an
n = 48 bitset<128> instance, outside `value`.
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
sys.path.insert(0, ROOT)

METRIC = ("ASCI time & H-build nnz/s: learned+mixed vs plain FP64, one GPU, "
          "ΔE≤0.1mEh")
WORKLOAD = ("CAS(12e,12o) full-CI CSR Hamiltonian build: 853,776 dets "
            "(bitset<64>), synthetic integrals seed 0, FP64 values, int32 "
            "indices, |h| > DBL_EPSILON")
DATA = ("synthetic: seeded integrals (seed 0; orbital energies on a ramp, "
        "N(0, 0.02^2) off-diagonal one-body terms, two-body terms as sums of "
        "products of symmetric random factors), no dataset")
NORB, NA, NB, SEED = 12, 6, 6, 0
THRESH = float(np.finfo(np.float64).eps)


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def c2_inputs():
    import macis_b200 as mb
    T, V = mb.synthetic_integrals(NORB, SEED)
    dets = mb.generate_hilbert_space(NORB, NA, NB, 64)
    return T, V, dets


def c2_inputs_reference(R):
    """The same workload for the reference arm without importing the package
    (whose import loads the CUDA library): the integral recipe from
    macis_b200/integrals.py loaded by path (numpy only), the determinant list
    from the reference's own generate_hilbert_space<64>."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "macis_b200_integrals", os.path.join(ROOT, "macis_b200", "integrals.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    T, V = mod.synthetic_integrals(NORB, SEED)
    return T, V, R.hilbert_space(64, NORB, NA, NB)


def bench_config(ndets, world):
    """`config` of both arms (the workload, not how either arm samples it)."""
    return {"workload": WORKLOAD, "ndets": ndets,
            "l2": "256 MB flush between steps; output 18.6 GB > L2",
            "parallelism": f"row-block x{world}"}


def sample_blocks(N, rows, nblocks=32):
    """`nblocks` row blocks of about rows / nblocks rows each, spread evenly
    over the N rows (a sample of the whole matrix, not of its first rows)."""
    nblocks = max(1, min(nblocks, rows))
    b = max(1, rows // nblocks)
    starts = np.linspace(0, N - b, nblocks).astype(np.int64)
    return [(int(r), int(r) + b) for r in starts]


def _bra_of(dets, blocks):
    return np.ascontiguousarray(np.concatenate([dets[a:b] for a, b in blocks]))


def reference_sample(R, h, dets, target_s, nthreads):
    """Row blocks whose reference build takes about target_s seconds on
    nthreads threads (probed on a small sample)."""
    N = len(dets)
    probe = sample_blocks(N, max(512, 64 * nthreads), 16)
    bra = _bra_of(dets, probe)
    t = time.perf_counter()
    R.csr(h, bra, dets, THRESH, nthreads=nthreads)
    per_row = (time.perf_counter() - t) / len(bra)
    rows = int(min(N, max(len(bra), target_s / max(per_row, 1e-9))))
    return sample_blocks(N, rows)


def alg_bytes(nnz, nrows, nbra, nket, idx_b=4, val_b=8, det_b=8):
    """Algorithmic bytes of one build: CSR written once, dets read once."""
    return nnz * (idx_b + val_b) + (nrows + 1) * idx_b + (nbra + nket) * det_b


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class NvmlClocks:
    """SM clock and clock-event reasons of the CUDA device, read through NVML
    every few milliseconds in a thread (reading only: nothing is set), so
    that a timed region of tens of milliseconds still gets several samples.
    The device is matched by UUID, which holds under CUDA_VISIBLE_DEVICES."""

    def __init__(self, cuda_index, period_s=0.005):
        import threading

        import pynvml as nv
        import torch
        nv.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(cuda_index).uuid)
        self.nv = nv
        self.h = nv.nvmlDeviceGetHandleByUUID(
            uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        self.smax = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
        self.reason_fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons",
                                 None) or nv.nvmlDeviceGetCurrentClocksThrottleReasons
        self.bits = {
            "hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
            "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
            "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
            "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        self.sm, self.reasons = [], set()
        self.done = threading.Event()
        self.period = period_s
        self.sample()                     # fails here, not in the thread
        self.t = threading.Thread(target=self.run, daemon=True)
        self.t.start()

    def sample(self):
        nv = self.nv
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
        r = int(self.reason_fn(self.h))
        self.reasons.update(k for k, b in self.bits.items() if r & b)

    def run(self):
        while not self.done.wait(self.period):
            try:
                self.sample()
            except Exception:
                return

    def stop(self):
        self.done.set()
        self.t.join(timeout=5)
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.smax,
                "samples": len(self.sm), "reasons": sorted(self.reasons),
                "source": "nvml"}


def start_clocks(cuda_index):
    """NVML sampling when the bindings and the driver answer, else the
    nvidia-smi sampler."""
    try:
        return NvmlClocks(cuda_index)
    except Exception:
        return Clocks(cuda_index)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
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
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                smax = float(c[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown",
                                "sw_thermal_slowdown", "sw_power_cap"), c[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def cpu_reference_rate(T, V, dets, target_s=10.0, nthreads=None):
    """Reference MACIS (compiled oracle/_ref) H build over a bounded sample of
    rows spread over the matrix, all host threads: nnz/s. Also returns the
    sample's row blocks and its CSR arrays for the parity check of the
    device-built matrix."""
    import oracle
    R = oracle.ref()
    nthreads = nthreads or os.cpu_count() or 1
    R.set_threads(1)
    h = R.ham(64, NORB, T, V)
    blocks = reference_sample(R, h, dets, target_s, nthreads)
    bra = _bra_of(dets, blocks)
    t = time.perf_counter()
    A = R.csr(h, bra, dets, THRESH, nthreads=nthreads)
    dt = time.perf_counter() - t
    out = {"value": A.nnz / dt, "unit": "nnz/s", "cores": nthreads,
           "kind": "reference", "rows": len(bra), "seconds": dt, "nnz": A.nnz,
           "sample": f"reference DoubleLoop make_csr_hamiltonian_block on "
                     f"{len(bra)} rows ({len(blocks)} row blocks spread over "
                     f"the {len(dets)} rows) x all {len(dets)} kets of the "
                     f"same matrix, {nthreads} threads over row blocks (the "
                     f"reference build loop itself is single-threaded)"}
    return out, blocks, A.arrays()


def csr_parity(A, blocks, ref_arrays):
    """The device-built matrix's rows of the sampled blocks against the
    reference's CSR of the same rows: rowptr, colind and nzval bit for bit."""
    rr, rc, rz = ref_arrays
    off, exact, nnz = 0, True, 0
    for a, b in blocks:
        rp, ci, nz = A.rows(a, b)
        lo, hi = int(rr[off]), int(rr[off + b - a])
        exact &= bool(np.array_equal(rp.astype(np.int64),
                                     rr[off:off + b - a + 1].astype(np.int64) - lo))
        exact &= bool(np.array_equal(ci.astype(np.int64),
                                     rc[lo:hi].astype(np.int64)))
        exact &= bool(np.array_equal(nz, rz[lo:hi]))
        nnz += hi - lo
        off += b - a
    return {"rows": off, "blocks": len(blocks), "nnz": nnz,
            "bit_exact": exact,
            "against": "compiled reference make_csr_hamiltonian_block "
                       "(DoubleLoopHamiltonianGenerator), the cpu_baseline "
                       "sample's rows"}


# ---------------------------------------------------------------- reference
def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "compiled reference oracle/_ref/libmacis_ref.so "
                          "missing"}))
        return 0
    nthreads = os.cpu_count() or 1
    R = oracle.ref()
    R.set_threads(1)
    T, V, dets = c2_inputs_reference(R)
    h = R.ham(64, NORB, T, V)
    # each step about 5 s of host work: the whole --steps/--warmup run stays
    # within a few minutes
    blocks = reference_sample(R, h, dets, 5.0, nthreads)
    bra = _bra_of(dets, blocks)
    for _ in range(args.warmup):
        R.csr(h, bra, dets, THRESH, nthreads=nthreads)
    times, nnz = [], 0
    for _ in range(args.steps):
        t = time.perf_counter()
        A = R.csr(h, bra, dets, THRESH, nthreads=nthreads)
        times.append(time.perf_counter() - t)
        nnz = A.nnz
        del A
    tot = sum(times)
    value = nnz * len(times) / tot
    sample = (f"{len(bra)} rows per step ({len(blocks)} row blocks spread "
              f"over the {len(dets)}-row matrix) x all {len(dets)} kets "
              f"(DoubleLoopHamiltonianGenerator via make_csr_hamiltonian_block,"
              f" {nthreads} threads over row blocks; the reference build loop "
              f"itself is single-threaded)")
    out = {"impl": "reference", "metric": METRIC, "value": value,
           "unit": "nnz/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
           "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "f64",
           "data": DATA,
           "config": bench_config(len(dets), world),
           "sample_rows": len(bra),
           "cpu_baseline": {"value": value, "unit": "nnz/s",
                            "cores": nthreads, "kind": "reference",
                            "sample": sample},
           "e2e": {"value": value, "unit": "nnz/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


# --------------------------------------------------------------------- ours
def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    import macis_b200 as mb
    from macis_b200 import _lib
    from macis_b200._lib import LIB, check

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local_rank)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    from macis_b200.dist import reduce_max, reduce_sum

    T, V, dets = c2_inputs()
    N = len(dets)
    lo, hi = mb.row_bounds(N, world, rank)
    H = mb.HamiltonianGenerator(T, V, 64)
    d_dets = torch.from_numpy(dets.view(np.int64)).to(dev)  # resident input
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    import ctypes as C

    def build_device():
        c = C.c_void_p()
        base = d_dets.data_ptr()
        check(LIB.macis_b200_build_csr(H.handle, base + lo * 8, hi - lo, base,
                                       N, THRESH, 4, 8, _lib.DEVICE_PTRS,
                                       C.byref(c)))
        return mb.DeviceCSR(c, H)

    for _ in range(args.warmup):
        A = build_device()
        del A
    barrier()
    clocks = start_clocks(torch.cuda.current_device()) if rank == 0 else None
    launches0 = LIB.macis_b200_launch_count()
    step_ms, fill_ms, nnz = [], [], 0
    st = _lib.BuildStatsC()
    barrier()
    for _ in range(args.steps):
        flush.zero_()                                   # L2 flush (256 MB)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        A = build_device()
        e1.record()
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        check(LIB.macis_b200_csr_build_stats(A.handle, C.byref(st)))
        fill_ms.append(st.fill_ms)
        nnz = A.nnz
        direct = bool(st.direct_product)
        del A
    barrier()
    launches = LIB.macis_b200_launch_count() - launches0
    ck = clocks.stop() if clocks else None
    tot_ms = reduce_max(sum(step_ms), device=dev)
    nnz_all = reduce_sum(float(nnz), device=dev)
    value = nnz_all * args.steps / (tot_ms / 1e3)
    res = {}
    if rank == 0:
        peak, peak_kind = peaks()
        fill_avg = sum(fill_ms) / len(fill_ms)
        B = alg_bytes(nnz, hi - lo, hi - lo, N)
        achieved = B / (fill_avg / 1e3) / 1e9
        traffic = None
        tf = os.path.join(ROOT, "profiles", "hbuild_fill_c2_traffic.json")
        if os.path.exists(tf):
            with open(tf) as f:
                traffic = json.load(f).get("dram_bytes_per_launch")
        res.update({
            "metric": METRIC, "value": value, "unit": "nnz/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": DATA,
            "config": bench_config(N, world),
            "matrix": {"nnz": int(nnz_all), "rows_per_rank": hi - lo,
                       "direct_product_path": direct},
            "clocks": ck,
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "dp_fill_k",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "frac_of_8TBs": achieved / 8000.0,
                         "alg_bytes_per_launch": B, "fill_ms": fill_avg,
                         "traffic": traffic},
        })
    # ---------------- end-to-end through the C ABI with host buffers
    e2e = None
    if world == 1 and not args.no_e2e:
        e2e = bench_e2e(args, mb, LIB, check, _lib, H, dets, torch)
    barrier()
    if rank == 0:
        res["e2e"] = e2e
        if world == 1 and not args.no_extras:
            res["extras"] = extras(mb, H, dets, torch)
        if world == 1 and not args.no_asci:
            try:
                res["asci"] = asci_iteration(mb, peaks()[0])
            except Exception as e:  # noqa: BLE001
                res["asci"] = {"error": str(e)}
        if world == 1 and not args.no_cpu:
            try:
                res["cpu_baseline"], blocks, ref_arrays = cpu_reference_rate(
                    T, V, dets)
                A = build_device()
                res["parity"] = csr_parity(A, blocks, ref_arrays)
                del A, ref_arrays
            except Exception as e:  # noqa: BLE001
                res["cpu_baseline"] = {"unavailable": str(e)}
        print(json.dumps(res))
    if world > 1:
        dist.destroy_process_group()
    return 0


def bench_e2e(args, mb, LIB, check, _lib, H, dets, torch):
    import ctypes as C
    N = len(dets)
    h_dets = torch.from_numpy(dets.view(np.int64)).pin_memory()
    c = C.c_void_p()
    p = h_dets.data_ptr()
    check(LIB.macis_b200_build_csr(H.handle, p, N, p, N, THRESH, 4, 8, 0,
                                   C.byref(c)))
    A = mb.DeviceCSR(c, H)
    nnz = A.nnz
    try:
        rp = torch.empty(N + 1, dtype=torch.int32, pin_memory=True)
        ci = torch.empty(nnz, dtype=torch.int32, pin_memory=True)
        nz = torch.empty(nnz, dtype=torch.float64, pin_memory=True)
        pinned = True
    except RuntimeError:
        rp = torch.empty(N + 1, dtype=torch.int32)
        ci = torch.empty(nnz, dtype=torch.int32)
        nz = torch.empty(nnz, dtype=torch.float64)
        pinned = False
    del A
    steps = max(1, min(args.steps, 3))
    times = []
    for it in range(steps + 1):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        c = C.c_void_p()
        check(LIB.macis_b200_build_csr(H.handle, p, N, p, N, THRESH, 4, 8, 0,
                                       C.byref(c)))
        check(LIB.macis_b200_csr_download(c, rp.data_ptr(), ci.data_ptr(),
                                          nz.data_ptr(), 0))
        LIB.macis_b200_csr_destroy(c)
        e1.record()
        torch.cuda.synchronize()
        if it:                                    # first call is a warm-up
            times.append(e0.elapsed_time(e1))
    t = sum(times) / len(times) / 1e3
    return {"value": nnz / t, "unit": "nnz/s", "ms_per_step": t * 1e3,
            "h2d_bytes_per_step": int(h_dets.numel() * 8),
            "d2h_bytes_per_step": int((N + 1) * 4 + nnz * 12),
            "pinned": pinned, "steps": len(times)}


def extras(mb, H, dets, torch):
    """SpMV, Davidson (FP64 / mixed) and ASCI timings outside `value`."""
    import ctypes as C

    from macis_b200._lib import LIB, check
    out = {}
    N = len(dets)
    peak, _ = peaks()
    for prec, vt in (("fp64", np.float64), ("mixed", np.float32)):
        A = mb.make_csr_hamiltonian(dets, H, THRESH, value_t=vt)
        x = torch.randn(N, dtype=torch.float64, device="cuda")
        y = torch.empty(N, dtype=torch.float64, device="cuda")
        for _ in range(3):
            check(LIB.macis_b200_spmv(A.handle, 1, 1.0, x.data_ptr(), N, 0.0,
                                      y.data_ptr(), N, 1))
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 10
        e0.record()
        for _ in range(reps):
            check(LIB.macis_b200_spmv(A.handle, 1, 1.0, x.data_ptr(), N, 0.0,
                                      y.data_ptr(), N, 1))
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        vb = 8 if prec == "fp64" else 4
        B = A.nnz * (4 + vb) + (N + 1) * 4 + 2 * N * 8 + (N * 8 if vb == 4 else 0)
        out[f"spmv_{prec}"] = {"ms": ms, "GBps": B / ms / 1e6,
                               "frac_of_measured_hbm": B / ms / 1e6 / peak,
                               "nnz": A.nnz}
        if prec == "fp64":
            # warm-up solve: the timed solves below run warm
            try:
                mb.davidson(N, 40, mb.SparseMatrixOperator(A), None, 1e-8,
                            np.zeros(N), use_guess=False, restart_keep=8,
                            max_iter=3000)
            except RuntimeError:
                pass
        X = np.zeros(N)
        t = time.perf_counter()
        try:
            it, E = mb.davidson(N, 40, mb.SparseMatrixOperator(A), None, 1e-8,
                                X, use_guess=False, restart_keep=8,
                                max_iter=3000)
            secs = time.perf_counter() - t
            ds = mb.davidson_stats()
            vec_ms = ds["rayleigh_ms"] + ds["residual_ms"] + ds["ortho_ms"]
            out[f"davidson_{prec}"] = {
                "seconds": secs, "iterations": it, "E0": E, "max_m": 40,
                "restart_keep": 8, "tol": 1e-8,
                "device_ms": {k: ds[k] for k in ("apply_ms", "rayleigh_ms",
                                                 "residual_ms", "ortho_ms")},
                "host_ms": ds["wall_ms"] - ds["apply_ms"] - vec_ms,
                "vector_kernels": {
                    "GBps": ds["vector_bytes"] / max(vec_ms, 1e-9) / 1e6,
                    "frac_of_measured_hbm": ds["vector_bytes"] / max(
                        vec_ms, 1e-9) / 1e6 / peak,
                    "alg_bytes": ds["vector_bytes"],
                    "basis": "multi-dot, Ritz/residual and CGS2 kernels: "
                             "every V / AV column read once per pass"}}
        except RuntimeError as e:
            out[f"davidson_{prec}"] = {"error": str(e)}
        del A
    if "E0" in out.get("davidson_fp64", {}) and "E0" in out.get("davidson_mixed", {}):
        out["mixed_dE_Eh"] = out["davidson_mixed"]["E0"] - out["davidson_fp64"]["E0"]
    return out


def _n48_core(mb, ncore, seed=0, n=48, k=12, nbits=128):
    """n = 48 orbitals, 12 alpha / 12 beta, bitset<128>: HF plus products of
    its low single / double alpha and beta excitations, ordered by total
    excitation degree, as the core set, with decaying coefficients
    (C3-shaped). Other shapes through n, k (electrons per spin) and nbits
    (C5: 100, 20, 256)."""
    T, V = mb.synthetic_integrals(n, seed)
    H = mb.HamiltonianGenerator(T, V, nbits)
    rng = np.random.default_rng(seed)
    top = max(200, int(np.ceil(np.sqrt(ncore))) + 8)
    hf = (1 << k) - 1
    alphas = {hf}
    while len(alphas) < 2 * top:
        a = hf
        for _ in range(rng.integers(1, 3)):
            i = int(rng.integers(0, k))
            v = int(rng.integers(k, n))
            if a >> i & 1 and not a >> v & 1:
                a ^= (1 << i) ^ (1 << v)
        alphas.add(a)
    alphas = sorted(alphas, key=lambda x: bin(x ^ hf).count("1"))
    pairs = [(a, b) for a in alphas[:top] for b in alphas[:top]]
    pairs.sort(key=lambda ab: bin(ab[0] ^ hf).count("1") + bin(ab[1] ^ hf).count("1"))
    pairs = pairs[:ncore]
    core = mb.sd.make_dets([a for a, _ in pairs], [b for _, b in pairs], nbits)
    C = np.exp(-0.5 * np.arange(len(core)) / 100.0)
    C /= np.linalg.norm(C)
    hd = H.matrix_element(core[:1], core[:1])
    return n, H, core, C, hd - 0.5


def asci_rooflines(st, nbits, peak):
    """HBM rooflines of the exact search's two dominant phases from its
    statistics: contribution generation (units_k count and fill passes:
    every raw record written once) and the candidate sort (lower bound: one
    read and one write of every record; per pass: the digit passes run).
    A record is a determinant and its score, or a ranked key (alpha and beta
    string ranks, 8 B) and its score when the search sorted by ranked keys
    (key_bits > 0)."""
    rec = 16 if st.get("key_bits") else 8 * (nbits // 64) + 8
    gen_b = st["raw_pairs"] * rec
    gen = gen_b / (st["pairs_ms"] * 1e-3) / 1e9
    lb_b = 2 * st["raw_pairs"] * rec
    pass_b = 2 * st["sort_pass_items"] * rec
    sort_lb = lb_b / (st["sort_ms"] * 1e-3) / 1e9
    sort_pass = pass_b / (st["sort_ms"] * 1e-3) / 1e9
    return {
        "units_k": {"bound": "hbm", "achieved": gen, "peak": peak,
                    "unit": "GB/s", "frac": gen / peak,
                    "alg_bytes": gen_b, "ms": st["pairs_ms"],
                    "basis": f"raw contributions x {rec} B written, over the "
                             "count + generation passes",
                    "key_bits": st.get("key_bits", 0)},
        "sort": {"bound": "hbm", "achieved": sort_lb, "peak": peak,
                 "unit": "GB/s", "frac": sort_lb / peak, "alg_bytes": lb_b,
                 "ms": st["sort_ms"],
                 "per_pass_GBps": sort_pass, "per_pass_frac": sort_pass / peak,
                 "digit_passes": st["sort_pass_items"] / max(st["raw_pairs"], 1),
                 "basis": "lower bound 2 x raw contributions x record (one "
                          "read + one write); per pass: 2 x record x records "
                          "per digit pass, summed over passes"}}


def asci_iteration(mb, peak, ncore=100000, ndets=1000000, seed=0,
                   cpu_ncore=50, cpu_ndets=20000, problem=None, nbits=128,
                   net=None, warm=True, keep_frac=0.2):
    """One C3-shaped ASCI iteration (asci_iter, iteration.hpp:17-68) both
    ways on n = 48, 12 alpha / 12 beta, bitset<128>: `ncore` core
    determinants -> `ndets` determinants -> rediagonalisation.

    exact_fp64: the exact asci_search, then the FP64 CSR H and Davidson.
    learned_mixed: the network trained (timed) on the samples the previous
    iteration's search recorded (a recording search over the leading
    ncore / 4 core determinants, not timed), the screened search (top 20 %
    of the units by prediction plus 2 % random), then the FP32-H CSR and
    the mixed-precision Davidson (FP64 residual, CGS2, Rayleigh-Ritz).
    dE = E(learned_mixed) - E(exact_fp64) at equal determinant count; the
    learned run's wavefunction is also evaluated with the FP64 H.
    cpu_baseline: the compiled reference asci_search (serial,
    determinant_search.hpp:395-663) and the GPU search on a matched small
    core set.

    problem = (n, H, core, C, E0) runs the iteration on a given core set
    (of nbits-bit determinants) instead; net = a network already trained
    online (then the learned time holds no training); warm = False skips
    the warm-up search (the caller's run has grown the memory pool)."""
    from macis_b200.solvers import FP64, MIXED
    if problem is None:
        n, H, core, C, E0 = _n48_core(mb, ncore, seed)
    else:
        n, H, core, C, E0 = problem
    s = mb.ASCISettings()
    dav = dict(restart_keep=8, max_iter=4000)
    if warm:
        # warm-up: a search of the same size grows the memory pool, as the
        # previous iteration of a refine loop would; a small solve loads
        # the solver kernels
        w = mb.asci_search(s, ndets, core, E0, C, n, H)
        mb.selected_ci_diag(w[:20000], H, THRESH, 40, 1e-8, **dav)
        mb.selected_ci_diag(w[:20000], H, THRESH, 40, 1e-8, precision=MIXED,
                            **dav)
        del w
    # exact search + FP64
    t0 = time.perf_counter()
    dets_e = mb.asci_search(s, ndets, core, E0, C, n, H)
    t_se = time.perf_counter() - t0
    st_e = mb.last_search_stats(H)
    te = {}
    E_e, X_e = mb.selected_ci_diag(dets_e, H, THRESH, 40, 1e-8,
                                   precision=FP64, timings=te, **dav)
    t_exact = time.perf_counter() - t0
    del X_e
    rec = mb.ScreenSettings()
    if net is None:
        # learned: the previous iteration's recording search (untimed)
        nprev = max(1, len(core) // 4)
        net = mb.ScreeningNetwork(nbits=nbits, seed=seed)
        rec = mb.ScreenSettings(network=net, max_samples=1000000)
        mb.asci_search(s, ndets // 4, core[:nprev], E0, C[:nprev], n, H,
                       screen=rec)
    sc = mb.ScreenSettings(network=net, keep_frac=keep_frac,
                           explore_frac=0.02, train=False, seed=seed)
    mb.asci_search(s, 1000, core[:200], E0, C[:200], n, H, screen=sc,
                   use_net=True)                  # loads the network kernels
    t0 = time.perf_counter()
    loss = None
    if rec.network is not None:
        net.clamp_samples(rec.clamp_quantile)
        loss = net.train(None, None, rec.epochs, rec.batch, rec.lr, seed)
    t_train = time.perf_counter() - t0
    t1 = time.perf_counter()
    dets_l = mb.asci_search(s, ndets, core, E0, C, n, H, screen=sc,
                            use_net=True)
    t_sl = time.perf_counter() - t1
    st_l = mb.last_search_stats(H)
    tl = {}
    E_l, X_l = mb.selected_ci_diag(dets_l, H, THRESH, 40, 1e-8,
                                   precision=MIXED, timings=tl, **dav)
    t_learned = time.perf_counter() - t0
    try:  # the FP64 H: stored when it fits, else applied matrix-free
        A = mb.make_csr_hamiltonian(dets_l, H, THRESH, np.int64)
    except mb.MacisError:
        A = mb.MatrixFreeHamiltonian(dets_l, H, THRESH)
    E_l64 = float(X_l @ A.spmv(X_l)) / float(X_l @ X_l)
    del A
    recall = mb.topk_recall(dets_l, dets_e, len(core))
    out = {
        "workload": f"ASCI iteration: n = {n}, bitset<{nbits}>, "
                    f"{len(core)} core dets -> {len(dets_e)} dets, synthetic "
                    f"integrals seed {seed}; Davidson to 1e-8 (max_m 40, "
                    f"thick restart 8)",
        "exact_fp64": {"seconds": t_exact, "search_s": t_se,
                       "h_build_s": te["h_ms"] / 1e3,
                       "davidson_s": te["dav_ms"] / 1e3,
                       "davidson_iterations": te["niter"], "E": E_e,
                       "ndets": len(dets_e), "raw_pairs": st_e["raw_pairs"],
                       "unique_pairs": st_e["unique_pairs"],
                       "phase_ms": {k: st_e[k] for k in
                                    ("pairs_ms", "sort_ms", "keep_ms")}},
        "learned_mixed": {"seconds": t_learned, "train_s": t_train,
                          "train_loss": loss, "search_s": t_sl,
                          "keep_frac": keep_frac,
                          "h_build_s": tl["h_ms"] / 1e3,
                          "davidson_s": tl["dav_ms"] / 1e3,
                          "davidson_iterations": tl["niter"], "E": E_l,
                          "E_with_fp64_H": E_l64, "ndets": len(dets_l),
                          "raw_pairs": st_l["raw_pairs"],
                          "units_kept": [st_l["units_kept"],
                                         st_l["units_total"]],
                          "predict_ms": st_l["predict_ms"],
                          "topk_recall": recall},
        "speedup": t_exact / t_learned,
        "dE_Eh": E_l - E_e,
        "dE_target_Eh": 1e-4,
        "within_target": abs(E_l - E_e) <= 1e-4,
        "roofline": asci_rooflines(st_e, nbits, peak),
    }
    del dets_e, dets_l, X_l
    if nbits == 128 and problem is None:
        out["cpu_baseline"] = asci_cpu_baseline(
            mb, n, H, core[:cpu_ncore], C[:cpu_ncore], E0, cpu_ndets, seed)
    return out


def asci_cpu_baseline(mb, n, H, core, C, E0, ndets, seed):
    """The compiled reference asci_search (one thread: its contribution loop
    and sort are serial, determinant_search.hpp:54-141 / determinant_sort.hpp:
    40-83) and the GPU search on the same small core set."""
    try:
        import oracle
        if not oracle.ref_available():
            return {"unavailable": "compiled reference oracle/_ref missing"}
        R = oracle.ref()
        T, V = mb.synthetic_integrals(n, seed)
        hr = R.ham(128, n, T, V)
        so = oracle.AsciSettings.default()
        t = time.perf_counter()
        r = R.asci_search(hr, so, ndets, core, float(E0), C)
        t_ref = time.perf_counter() - t
        s = mb.ASCISettings()
        mb.asci_search(s, ndets, core, E0, C, n, H)
        t = time.perf_counter()
        g = mb.asci_search(s, ndets, core, E0, C, n, H)
        t_gpu = time.perf_counter() - t
        st = mb.last_search_stats(H)
        same = len(set(map(bytes, r)) ^ set(map(bytes, g)))
        return {"value": t_ref, "unit": "s", "cores": 1, "kind": "reference",
                "gpu_s": t_gpu, "raw_pairs": st["raw_pairs"],
                "ref_raw_pairs_per_s": st["raw_pairs"] / t_ref,
                "gpu_raw_pairs_per_s": st["raw_pairs"] / t_gpu,
                "selection_differences": same,
                "sample": f"asci_search, n = 48 12a/12b bitset<128>, "
                          f"{len(core)} core dets -> {ndets} dets, the same "
                          f"inputs on both sides"}
    except Exception as e:  # noqa: BLE001
        return {"unavailable": str(e)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-asci", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 0)
    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local_rank = env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
