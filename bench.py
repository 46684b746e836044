"""Assembly throughput benchmark (assembled CSR nonzeros per second), and the
solve+grad leg of the same metric (mixed-precision solve and adjoint
gradient against the plain FP64 assembly + solve, in the "solve" object).

One step = one pass of the system-assembly hot path over the workload:
element matrices (curl-curl, mass and k-parallel terms with the PML
stretch), dual face transform, DOF signs, essential elimination and the
atomic-free gather into the CSR values, all on device-resident inputs
(``lfasm_assemble``).

Default workload: the line grating (pitch 64 nm, CD 32 nm, 60 nm absorber
over a 40 nm underlayer, 64 x 16 nm cell, lambda 13.5 nm, theta 6 deg,
Nedelec p = 3, ~1.35M complex DOF), the configuration of the reference's
published GPU assembly timing.  Synthetic, seeded mesh (no external data).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: the path does not shard a single mesh; N ranks run independent
replicas (weak scaling), value = total nonzeros / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from lithofem_b200 import replicas  # noqa: E402  (host-only, no CUDA at import)

METRIC = "assembly nnz/s"
UNIT = "nnz/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=3,
                    help="1-4: one mesh; 5: the 16 polygon-hole meshes in one CUDA-graph launch")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solve", action="store_true",
                    help="skip the solve+grad leg (device LU, plain complex128 vs mixed)")
    ap.add_argument("--solve-only", action="store_true",
                    help="run only the solve+grad leg")
    ap.add_argument("--solve-reps", type=int, default=2)
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-meshes leg (the 16 polygon-hole meshes of --config 5 "
                         "in one graph launch) of the default line")
    ap.add_argument("--pml-variant", type=int, default=-1,
                    help="force the PML kernel (0 k_pml_mma, 1 k_pml_ws at p = 3, 2 k_pml_sym); "
                         "default: autotune")
    ap.add_argument("--bulk-variant", type=int, default=-1,
                    help="force the bulk-element kernel (0 SIMT, 1/2 DMMA with 4/2 tiles a warp, "
                         "3/4 the same without block barriers); default: autotune")
    return ap.parse_args()


def workload_config(case, a) -> dict:
    return {"workload": case.name + f" (~{case.ad.height / 1e6:.2f}M DOF)",
            "p": case.p, "theta_deg": case.theta, "elements": case.ad.ne,
            "ndof": case.ad.height, "nnz": int(case.nnz) if hasattr(case, "nnz") else None,
            "l2_policy": "inputs larger than L2 (element buffer and CSR >> 126 MB)",
            "replicas": a.gpus, "scale": a.scale}


class ClockSampler:
    """SM clock and clock-event (throttle) reasons during the timed region.

    Samples NVML every 2 ms from a thread (read-only queries of the device
    the CUDA context runs on, matched by UUID); where NVML is unavailable,
    falls back to an `nvidia-smi -lms 100` poller."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, dev: int):
        self.dev = dev
        self.proc = None
        self.nv = None
        self.lines: list[str] = []
        self.samples: list[tuple[float, float, int]] = []
        self._stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.dev)
        try:
            uuid = str(props.uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(
                uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def start(self):
        try:
            self.nv, self.h = self._nvml_handle()
            self.smax = float(self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM))
            self._t = threading.Thread(target=self._poll, daemon=True)
            self._t.start()
            return
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _poll(self):
        nv, h = self.nv, self.h
        while not self._stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.samples.append((sm, self.smax, rs))
            except Exception:
                pass
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.nv is not None:
            self._stop.set()
            self._t.join(timeout=2)
            nv = self.nv
            bits = {"hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
                    "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
                    "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
                    "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4)}
            reasons = sorted({nm for _, _, rs in self.samples for nm, b in bits.items() if rs & b})
            sm = [x[0] for x in self.samples]
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.smax,
                    "samples": len(sm), "reasons": reasons, "source": "NVML, every 2 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons), "source": "nvidia-smi -lms 100"}


PML_KERNELS = ["k_pml_mma", "k_pml_ws", "k_pml_sym"]
BULK_KERNELS = ["k_bulk (SIMT)", "k_bulk_mma<4 tiles/warp> (DMMA)", "k_bulk_mma<2 tiles/warp> (DMMA)",
                "k_bulk_mma_nb<4 tiles/warp> (DMMA, no block barriers)",
                "k_bulk_mma_nb<2 tiles/warp> (DMMA, no block barriers)",
                "k_bulk_tma<4 tiles/warp> (DMMA, records staged by cp.async.bulk)"]


def pml_flops(n_pml: int, nd: int, nq_cc: int, nq_mass: int, cross: bool, variant: int) -> float:
    """Algorithmic FP64 flops of the PML element kernel (real x complex
    multiply-adds, 4 flops per staged row and matrix entry).  k_pml_mma and
    k_pml_ws form every entry of X^T (W X): 3 rows per curl point, 3 (6 with
    the cross terms) per mass point.  k_pml_sym forms the symmetric part on
    and above the diagonal (3 rows per point of both rules) and every entry
    of the cross part (3 rows per mass point)."""
    if variant == 2:
        f = 4.0 * 3 * (nq_cc + nq_mass) * nd * (nd + 1) / 2
        if cross:
            f += 4.0 * 3 * nq_mass * nd * nd
    else:
        f = 4.0 * (3 * nq_cc + (6 if cross else 3) * nq_mass) * nd * nd
    return n_pml * f


def fp64_peak_tflops(torch) -> float:
    """Measured FP64 reference peak: cuBLAS DGEMM 8192^3, best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def measured_peaks() -> dict:
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


def _reference_csr(case):
    """The reference's symbolic CSR of the mesh (build_csr_symbolic) and its
    context, or the oracle's CSR and None without the reference build."""
    from oracle import oracle
    if oracle.ref_available():
        rc = oracle.RefContext(case.ad, case.prob)
        I, J = rc.build_csr()
        return rc, I, J
    I, J = oracle.csr(case.ad)
    return None, I, J


def cpu_baseline_reference(case, budget_s: float, threads: int, csr=None) -> dict:
    """The reference's serial CPU reassembler (reassemble_all,
    solver/asm_data.inc:374-402, compiled from its sources) on a bounded
    share of the mesh: every k-th element (a mix of bulk and PML elements
    like the whole mesh) reassembled once into the full rows of the mesh's
    CSR, the share sized from a probe to take about ``budget_s``; nnz/s =
    full nnz x (share elements / all elements) / wall.  With threads > 1,
    that many disjoint strided shares run concurrently."""
    from oracle import oracle
    ne = case.ad.ne
    if not oracle.ref_available():
        return cpu_baseline_port(case, budget_s, threads)
    _, I, J = csr if csr is not None else _reference_csr(case)
    probe = oracle.RefShares(case.ad, case.prob, I, J, [np.arange(0, ne, max(1, ne // 200))])
    t_probe = probe.time_parallel(1)
    per_el = max(t_probe / probe.sizes[0], 1e-7)
    del probe
    m = int(min(ne // max(threads, 1), max(50, budget_s / per_el)))
    stride = max(1, ne // (m * threads))
    shares = [np.arange(k, ne, stride)[:m] for k in range(threads)]
    sh = oracle.RefShares(case.ad, case.prob, I, J, shares)
    wall = sh.time_parallel(threads)
    elems = sum(sh.sizes)
    value = len(J) * (elems / ne) / wall
    return {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{elems} of {ne} elements (every {stride}th, {threads} thread(s) x {m}), "
                      f"reassemble_all into the full rows of the mesh's CSR; nnz/s = full nnz x "
                      f"sampled fraction / wall",
            "seconds": wall}


def cpu_baseline_port(case, budget_s: float, threads: int) -> dict:
    """Without the reference build: the oracle (this repository's C++
    restatement of reassemble_all) on bounded element samples, each on its
    sample's own CSR."""
    rng = np.random.default_rng(7)
    ne = case.ad.ne
    probe = np.sort(rng.choice(ne, size=min(ne, 200), replace=False))
    t_probe = _run_sample(_prepare_sample(case, probe, "port"))
    per_el = max(t_probe / len(probe), 1e-7)
    m = int(min(ne, max(50, budget_s / per_el / max(threads, 1))))
    samples = [np.sort(rng.choice(ne, size=m, replace=False)) for _ in range(threads)]
    prepared = [_prepare_sample(case, smp, "port") for smp in samples]
    import concurrent.futures as cf
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(_run_sample, prepared))
    wall = time.perf_counter() - t0
    elems = m * threads
    return {"value": case.nnz * (elems / ne) / wall, "unit": UNIT, "cores": threads,
            "kind": "port",
            "sample": f"{elems} of {ne} elements ({threads} thread(s) x {m}), the oracle's "
                      f"reassembly on the sample's own CSR; nnz/s = full nnz x sampled "
                      f"fraction / wall",
            "seconds": wall}


def _prepare_sample(case, elements, kind):
    """The untimed part of one sample: the reference context and its CSR
    (or, for the port, the sub-mesh and its CSR)."""
    from oracle import oracle
    if kind == "reference":
        rc = oracle.RefContext(case.ad, case.prob, elements=elements)
        rc.build_csr()
        return ("reference", rc)
    sub = _subset_ad(case.ad, elements)
    I, J = oracle.csr(sub)
    return ("port", (sub, case.prob, I, J))


def _run_sample(prepared) -> float:
    """Seconds of one reassembly of a prepared sample."""
    from oracle import oracle
    kind, obj = prepared
    if kind == "reference":
        return obj.time_reassemble()
    sub, prob, I, J = obj
    t0 = time.perf_counter()
    oracle.assemble(sub, prob, I, J, sub.ess, eliminate=False)
    return time.perf_counter() - t0


def _subset_ad(ad, elements):
    import copy
    sub = copy.copy(ad)
    nd = ad.nd
    sub.ne = len(elements)
    sub.dof = np.ascontiguousarray(ad.dof.reshape(ad.ne, nd)[elements].reshape(-1))
    sub.sign = np.ascontiguousarray(ad.sign.reshape(ad.ne, nd)[elements].reshape(-1))
    sub.fo = np.ascontiguousarray(ad.fo.reshape(ad.ne, 4)[elements].reshape(-1)) if ad.p > 1 else ad.fo
    sub.attr = np.ascontiguousarray(ad.attr[elements])
    for k, w in (("J", 9), ("Jinv", 9), ("detJ", 1), ("v0", 3)):
        setattr(sub, k, np.ascontiguousarray(getattr(ad, k).reshape(ad.ne, w)[elements].reshape(-1)))
    sub.ess = np.zeros(0, dtype=np.int32)
    return sub


def dist_setup(a):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def main():
    a = parse()
    rank, world, local = dist_setup(a)
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if a.config == 5:
        if a.impl == "reference":
            return run_reference_batch(a, rank, world, dist)
        return run_batch(a, rank, world, local, dist, torch)
    if a.impl == "reference":
        return run_reference(a, rank, world, dist)
    return run_ours(a, rank, world, local, dist, torch)


def run_reference(a, rank, world, dist):
    """The reference's CPU assembly of the whole mesh per step: its
    reassemble_all over disjoint contiguous element shares (four per host
    thread, handed out as threads free up) into the full rows of the mesh's
    CSR, on every host thread; each timed step is one full pass over all
    elements, wall clock."""
    from lithofem_b200 import configs
    from oracle import oracle
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    case = configs.config(a.config, scale=a.scale)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    rc, I, J = _reference_csr(case)
    t_csr = time.perf_counter() - t0
    case.nnz = len(J)
    if rc is not None:
        shares = oracle.contiguous_shares(case.ad.ne, 4 * threads)
        sh = oracle.RefShares(case.ad, case.prob, I, J, shares)
        walls = [sh.time_parallel(threads) for _ in range(a.warmup + a.steps)][a.warmup:]
        del sh
        kind = "reference"
        sample = (f"all {case.ad.ne} elements every step: reassemble_all over {len(shares)} "
                  f"contiguous element shares on {threads} threads, into the full rows of "
                  f"the mesh's CSR (build_csr_symbolic)")
    else:
        walls = []
        for _ in range(a.warmup + a.steps):
            info = cpu_baseline_port(case, 4.0, threads)
            walls.append(case.nnz / info["value"])
        walls = walls[a.warmup:]
        kind, sample = "port", info["sample"]
    ms = 1e3 * float(np.mean(walls))
    v = case.nnz / (ms * 1e-3)
    gpu_ref = reference_cuda_kernels(case, a, rc)
    if gpu_ref is not None and rc is not None:
        gpu_ref["host_csr_build_s"] = t_csr
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(case, a),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "step_wall_s": [round(w, 4) for w in walls],
            "reference_cuda_kernels": gpu_ref}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def reference_cuda_kernels(case, a, rc=None) -> dict | None:
    """Informational: the reference's own CUDA assembly (asm_gpu.inc:
    ComputeLocal + ScatterEliminate) compiled for sm_100a from its sources,
    on the same inputs, timed with CUDA events (per-iteration average)."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
        if rc is None:
            return None
        _, ml, msc = rc.gpu_global(case.ad.ess, eliminate=True, iters=max(1, min(a.steps, 5)),
                                   download=False)
        ms = ml + msc
        return {"ms_per_step": ms, "value": case.nnz / (ms * 1e-3), "unit": UNIT,
                "local_ms": ml, "scatter_eliminate_ms": msc,
                "what": "reference solver/asm_gpu.inc kernels compiled for sm_100a, same inputs"}
    except Exception as exc:  # report, never fake
        return {"error": str(exc)[:200]}


def run_ours(a, rank, world, local, dist, torch):
    from lithofem_b200 import _lib, configs
    from lithofem_b200.asm import AsmGpuGlobal
    dev = local
    torch.cuda.set_device(dev)
    case = configs.config(a.config, scale=a.scale)
    ad, prob = case.ad, case.prob
    if a.solve_only:
        out = run_solve(a, case, dev, torch)
        if rank == 0:
            print(json.dumps({"solve": out}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    stream = torch.cuda.current_stream()
    g = AsmGpuGlobal(prob)
    assert g.Init(ad, dev), "lfasm_init failed"
    assert g.SetStream(stream.cuda_stream)
    assert g.BuildGlobal(ad.ess)
    case.nnz = g.nnz()
    nb, npml = g.PathCounts()
    assert g.Autotune()
    if a.bulk_variant >= 0:
        assert g.SetBulkVariant(a.bulk_variant)
    if a.pml_variant >= 0:
        assert g.SetPmlVariant(a.pml_variant)
    tuning = g.Tuning()
    pml_tuning = g.PmlTuning()
    # warm-up
    for _ in range(a.warmup):
        assert g.Assemble(True)
    # per-stage profile (separate, untimed pass)
    assert g.SetProfile(True)
    stages = np.zeros(3)
    nprof = 3
    for _ in range(nprof):
        assert g.Assemble(True)
        stages += np.array(g.StageTimes())
    stages /= nprof
    assert g.SetProfile(False)
    torch.cuda.synchronize()

    # timed region: K steps on resident inputs, device events on the stream
    assert g.SetAsync(True)
    clk = ClockSampler(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clk.start()
    launches0 = _lib.lib().lfasm_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(a.steps):
        if not g.Assemble(True):
            raise RuntimeError("assembly failed")
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    launches = _lib.lib().lfasm_launch_count() - launches0
    clocks = clk.stop()
    assert g.SetAsync(False)
    ms = ev0.elapsed_time(ev1) / a.steps
    ms = replicas.max_over_ranks(ms, dist, "cuda")
    if dist is not None:
        dist.barrier()
    value = case.nnz * world / (ms * 1e-3)

    # e2e through the C ABI with host buffers: init (uploads from pinned host
    # memory) + build_global + assemble + download of the CSR values
    e2e = run_e2e(a, case, dev, torch, stream)

    # the metric's second half on one GPU: solve+grad, mixed vs plain FP64
    solve = None
    if not a.no_solve and world == 1:
        assert g.SetAsync(False)
        solve = run_solve(a, case, dev, torch, g)

    # the batched uneven meshes (the --config 5 workload) on the same GPU
    batch = None
    if not a.no_batch and world == 1:
        batch = run_batch_leg(a, dev, torch, stream)

    if rank != 0:
        g.Release()
        if dist is not None:
            dist.destroy_process_group()
        return

    # roofline for the dominant stage
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    hbm_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    nd = ad.nd
    alg = {
        "bulk": nb * (nd * nd * 16 + 320 + 8 * 3),
        "gather": ad.ne * nd * nd * (16 + 2) + ad.ne * nd * 4 + (ad.height + 1) * 8
                  + case.nnz * 16,
    }
    rm, rc = ad.rule_mass, ad.rule_cc
    flops_pml = pml_flops(npml, nd, rc.nq, rm.nq, prob.has_kpar, pml_tuning[0])
    fp64 = fp64_peak_tflops(torch)
    stage_names = ["prep+bulk", "pml", "gather"]
    kern = {}
    for nm, t in zip(stage_names, stages):
        kern[nm] = {"ms": float(t), "share": float(t / stages.sum())}
    kern["prep+bulk"]["GB/s"] = alg["bulk"] / (stages[0] * 1e-3) / 1e9
    kern["gather"]["GB/s"] = alg["gather"] / (stages[2] * 1e-3) / 1e9
    kern["pml"]["TFLOP/s"] = flops_pml / (stages[1] * 1e-3) / 1e12 if stages[1] > 0 else 0.0
    top = int(np.argmax(stages))
    if top == 1:
        ach = kern["pml"]["TFLOP/s"]
        roof = {"kernel": PML_KERNELS[pml_tuning[0]],
                "what": "PML elements, FP64 quadrature contraction on DMMA",
                "bound": "tensor",
                "achieved": ach, "peak": fp64, "unit": "TFLOP/s", "frac": ach / fp64,
                "peak_source": "measured in-run: cuBLAS DGEMM 8192^3", "traffic": None}
    else:
        nm = stage_names[top]
        ach = kern[nm]["GB/s"]
        roof = {"kernel": {"prep+bulk": BULK_KERNELS[tuning[0]].split("<")[0].split(" ")[0],
                           "gather": "k_gather"}[nm], "bound": "hbm",
                "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "peak_source": f"{hbm_src} (MEASURED_PEAKS.json hbm_gbs)", "traffic": None}
    prof_path = ROOT / "profiles" / "traffic_c3_line_grating_p3.json"
    if prof_path.exists() and a.config == 3 and a.scale == 1.0:
        try:
            tr = json.loads(prof_path.read_text())
            roof["traffic"] = tr.get(roof["kernel"])
            roof["traffic_source"] = "profiles/traffic_c3_line_grating_p3.json (ncu, scaled)"
        except Exception:
            pass

    cpu = None
    if not a.no_cpu_baseline and world == 1:
        try:
            cpu = cpu_baseline_reference(case, a.cpu_seconds, 1)
            cpu.pop("seconds", None)
        except Exception as exc:  # report, never fake
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"failed: {exc}"}

    # the same extraction on the device (lfasm_extract, host copies included)
    from lithofem_b200 import space
    t0 = time.perf_counter()
    space.build_asm_data_device(case.mesh, case.p, prob, gpu_id=dev)
    extract_s = {"extract": time.perf_counter() - t0,
                 "what": "lfasm_extract of the same mesh: mesh upload, device numbering and "
                         "per-mesh data, download of the arrays (wall clock)"}
    cfg = workload_config(case, a)
    cfg["nnz"] = int(case.nnz)
    cfg["bulk_elements"], cfg["pml_elements"] = nb, npml
    cfg["parallelism"] = f"replicas x{world}"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (complex128)", "data": "synthetic",
            "config": cfg, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
            "roofline": roof, "cpu_baseline": cpu, "solve": solve, "batch": batch,
            "kernels": kern,
            "fp64_peak_tflops": fp64,
            "host_build_s": dict(case.host_s, what="host mesh generation and space / per-mesh "
                                 "data extraction (build_asm_data) of this mesh, once per "
                                 "mesh, outside the timed regions"),
            "device_extract_s": extract_s,
            "tuning": {"bulk_variant": BULK_KERNELS[tuning[0]],
                       "bulk_ms": tuning[1],
                       "pml_variant": PML_KERNELS[pml_tuning[0]],
                       "pml_ms": pml_tuning[1]}}
    print(json.dumps(line), flush=True)
    g.Release()
    if dist is not None:
        dist.destroy_process_group()


def _timed(torch, fn):
    """Host wall seconds of fn() with the device synchronized on both sides."""
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = fn()
    torch.cuda.synchronize()
    return time.perf_counter() - t0, out


def run_solve(a, case, dev, torch, g=None) -> dict:
    """The solve+grad leg on the same mesh: the plain path (assembly, complex128
    factorization, one solve) against the mixed-precision path (assembly,
    complex64 factorization, FP64-refined solve to 1e-10, the adjoint seed
    of the zeroth order on a plane above the structure, FP64-refined
    transposed solve, the per-element eps gradient), both on the device
    through liblfasm + liblfsolve, wall clock with device syncs; the field
    error of the mixed solution against the plain one.  The ordering (host
    analysis, once per mesh) is reported apart."""
    from lithofem_b200 import incident, ndbasis
    from lithofem_b200.asm import AsmGpuGlobal
    from lithofem_b200.solver import C64, C128, DirectSolver
    ad, prob = case.ad, case.prob
    own = g is None
    if own:
        g = AsmGpuGlobal(prob)
        assert g.Init(ad, dev) and g.BuildGlobal(ad.ess)
    assert g.Assemble(True)
    n = ad.height
    nnz = int(g.nnz())
    parts = [incident.planewave_parts(case.stack, case.theta, 0.0, "s", 1.0, True)]
    b = torch.zeros(n, dtype=torch.complex128, device="cuda")
    assert g.AssembleRHS(parts, [0], 1, True, b.data_ptr())
    assert g.SetBasis(ndbasis.nd_element(ad.p))
    st = case.stack
    z_plane = st.z_max - 0.25 * (st.z_max - st.slabs[-2]) if len(st.slabs) > 2 else st.z_max * 0.9
    s = DirectSolver(dev)
    t_an, ok = _timed(torch, lambda: s.AnalyzeAssembly(g, ad))
    assert ok, s.last_error
    stats = s.Stats()
    V = g._csr()[2]
    x128 = torch.empty_like(b)
    x64 = torch.empty_like(b)
    lam = torch.empty_like(b)
    cvec = torch.empty_like(b)
    grad = torch.zeros(ad.ne, dtype=torch.complex128, device="cuda")

    def plain():
        assert g.Assemble(True)
        assert s.FactorDevice(V, C128), s.last_error
        f_ms = s.Stats()["factor_ms"]
        assert s.Backsolve(1, b.data_ptr(), x128.data_ptr()), s.last_error
        return f_ms

    def mixed():
        assert g.Assemble(True)
        assert s.FactorDevice(V, C64), s.last_error
        f_ms = s.Stats()["factor_ms"]
        ok1, rel1, it1 = s.SolveRefined(g, 1, b.data_ptr(), x64.data_ptr(), False, 1e-10)
        assert ok1, s.last_error
        assert g.PlaneSeed(st.lx, st.ly, z_plane, 16, 16, 0, 0, 0, cvec.data_ptr())
        ok2, rel2, it2 = s.SolveRefined(g, 1, cvec.data_ptr(), lam.data_ptr(), True, 1e-10)
        assert ok2, s.last_error
        assert g.EpsGradient(parts, x64.data_ptr(), lam.data_ptr(), grad.data_ptr())
        return f_ms, rel1[0], it1, rel2[0], it2

    reps = max(1, a.solve_reps)
    tp, tm, fp, fm, info = [], [], [], [], None
    for _ in range(reps):
        t, f = _timed(torch, plain)
        tp.append(t)
        fp.append(f)
    res128 = g.ResidualDevice(x128.data_ptr(), b.data_ptr())[1]
    s.Release()            # the complex128 factors out of memory
    s = DirectSolver(dev)
    assert s.AnalyzeAssembly(g, ad)
    for _ in range(reps):
        t, info = _timed(torch, mixed)
        tm.append(t)
        fm.append(info[0])
    res64 = g.ResidualDevice(x64.data_ptr(), b.data_ptr())[1]
    err = float(torch.linalg.vector_norm(x64 - x128) / torch.linalg.vector_norm(x128))
    s.Release()
    if own:
        g.Release()
    fl = stats["factor_flops"]
    return {
        "workload": case.name, "ndof": n, "nnz": nnz,
        "what": "plain: assembly + complex128 LU + solve; mixed: assembly + complex64 LU + "
                "FP64-refined solve (1e-10) + zeroth-order adjoint seed + FP64-refined "
                "transposed solve + per-element eps gradient",
        "timer": "host wall clock with device synchronize on both sides, best of reps",
        "plain_s": min(tp), "mixed_s": min(tm), "mixed_over_plain": min(tm) / min(tp),
        "factor_c128_ms": min(fp), "factor_c64_ms": min(fm),
        "factor_tflops_c128": fl / (min(fp) * 1e-3) / 1e12,
        "factor_tflops_c64": fl / (min(fm) * 1e-3) / 1e12,
        "field_rel_err_mixed_vs_plain": err, "residual_plain": res128, "residual_mixed": res64,
        "refine": {"forward_rel": info[1], "forward_corrections": info[2],
                   "transposed_rel": info[3], "transposed_corrections": info[4]},
        "analysis_s": t_an,
        "fronts": stats["n_fronts"], "max_front": stats["max_front"],
        "factor_entries": stats["factor_entries"], "factor_flops": fl,
        "reps": reps}


def run_e2e(a, case, dev, torch, stream) -> dict | None:
    from lithofem_b200.asm import AsmGpuGlobal
    import copy
    if a.e2e_steps <= 0:
        return None
    ad = copy.copy(case.ad)
    h2d = 0
    # inputs in pinned host memory
    for name in ("dof", "sign", "fo", "attr", "J", "Jinv", "detJ", "v0"):
        arr = getattr(ad, name)
        t = torch.empty(arr.shape, dtype=getattr(torch, str(arr.dtype)), pin_memory=True)
        t.numpy()[...] = arr
        setattr(ad, name, t.numpy())
        h2d += arr.nbytes
    for r in (ad.rule_cc, ad.rule_mass):
        h2d += r.ip.nbytes + r.w.nbytes + r.vshape.nbytes + r.curl.nbytes
    h2d += ad.ess.nbytes
    nnz = case.nnz
    out = torch.empty(2 * nnz, dtype=torch.float64, pin_memory=True)
    from lithofem_b200.asm import DeviceVector
    times = []
    parts = []
    for it in range(1 + a.e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g = AsmGpuGlobal(case.prob)
        assert g.Init(ad, dev)
        t1 = time.perf_counter()
        assert g.BuildGlobal(ad.ess)
        t2 = time.perf_counter()
        assert g.Assemble(True)
        t3 = time.perf_counter()
        # D2H of the result (the CSR values) through a borrowed device view
        _, _, V, _, nz = g._csr()
        dv = torch.as_tensor(DeviceVector(V, (2 * nz,), "<f8"), device="cuda")
        out.copy_(dv)
        torch.cuda.synchronize()
        del dv
        t4 = time.perf_counter()
        g.Release()
        t5 = time.perf_counter()
        if it >= 1:
            times.append(t5 - t0)
            parts.append([t1 - t0, t2 - t1, t3 - t2, t4 - t3, t5 - t4])
    t = float(np.median(times))
    br = np.median(np.array(parts), axis=0) * 1e3
    return {"value": nnz / t, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(16 * nnz), "ms_per_step": 1e3 * t,
            "what": "lfasm_init (uploads from pinned host arrays) + lfasm_build_global "
                    "(device symbolic CSR + maps) + lfasm_assemble + D2H of the CSR values",
            "timer": "host wall clock with device synchronize on both sides",
            "breakdown_ms": {"init": br[0], "build_global": br[1], "assemble": br[2],
                             "d2h": br[3], "release": br[4]}}


def run_batch_leg(a, dev, torch, stream) -> dict:
    """The 16 polygon-hole meshes of --config 5 assembled by one graph launch
    (lfasm_batch_assemble) on this GPU, device-timed like the main line:
    value = total nnz / time per launch; the meshes' host build apart."""
    from lithofem_b200 import _lib, configs
    from lithofem_b200.asm import AsmBatch, AsmGpuGlobal
    t0 = time.perf_counter()
    cases = configs.batch_config(scale=a.scale)
    t_build = time.perf_counter() - t0
    hs = []
    for c in cases:
        h = AsmGpuGlobal(c.prob)
        assert h.Init(c.ad, dev) and h.BuildGlobal(c.ad.ess)
        c.nnz = h.nnz()
        assert h.Assemble(True)          # tunes the handle
        hs.append(h)
    b = AsmBatch(hs)
    assert b.SetStream(stream.cuda_stream)
    for _ in range(max(3, a.warmup)):
        assert b.Assemble(True)
    torch.cuda.synchronize()
    launches0 = _lib.lib().lfasm_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(a.steps):
        assert b.Assemble(True)
    ev1.record(stream)
    ev1.synchronize()
    launches = _lib.lib().lfasm_launch_count() - launches0
    ms = ev0.elapsed_time(ev1) / a.steps
    b.Release()
    for h in hs:
        h.Release()
    total = sum(c.nnz for c in cases)
    cfg = batch_workload_config(cases, a)
    cfg.pop("meshes")
    return {"metric": METRIC, "value": total / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "steps": a.steps, "config": cfg, "gpu_launches_per_step": launches / a.steps,
            "host_build_s": t_build,
            "timer": "CUDA events on the launching stream around the graph launches"}


def batch_workload_config(cases, a) -> dict:
    return {"workload": f"C5 batched uneven meshes: {len(cases)} polygon holes, p = 1, 2, 3 "
                        f"cycled, {min(c.ad.height for c in cases) / 1e3:.0f}k-"
                        f"{max(c.ad.height for c in cases) / 1e3:.0f}k DOF, one CUDA-graph launch",
            "meshes": [{"name": c.name, "p": c.p, "elements": c.ad.ne, "ndof": c.ad.height,
                        "nnz": int(getattr(c, "nnz", 0))} for c in cases],
            "ndof": int(sum(c.ad.height for c in cases)),
            "nnz": int(sum(getattr(c, "nnz", 0) for c in cases)),
            "l2_policy": "inputs larger than L2 (element buffers and CSR >> 126 MB)",
            "replicas": a.gpus, "scale": a.scale}


def run_batch(a, rank, world, local, dist, torch):
    """The batched workload: 16 polygon-hole meshes assembled by one graph
    launch (lfasm_batch_assemble); value = total nnz / time per launch."""
    from lithofem_b200 import _lib, configs
    from lithofem_b200.asm import AsmBatch, AsmGpuGlobal
    dev = local
    torch.cuda.set_device(dev)
    # one share of the 16 meshes per rank (all of them at one GPU)
    mine = replicas.shard(16, rank, world)
    cases = configs.batch_config(scale=a.scale, only=mine)
    stream = torch.cuda.current_stream()
    hs = []
    for c in cases:
        g = AsmGpuGlobal(c.prob)
        assert g.Init(c.ad, dev) and g.BuildGlobal(c.ad.ess)
        c.nnz = g.nnz()
        hs.append(g)
    total = sum(c.nnz for c in cases)
    # per-mesh stage profile (serial, untimed) and the serial per-handle time
    stages = np.zeros(3)
    serial_ms = 0.0
    per_mesh = []
    pml_var, bulk_var = [], []
    for g in hs:
        assert g.Assemble(True)          # tunes the handle
        pml_var.append(g.PmlTuning()[0])
        bulk_var.append(g.Tuning()[0])
        assert g.SetProfile(True)
        assert g.Assemble(True)
        st = np.array(g.StageTimes())
        stages += st
        serial_ms += float(st.sum())
        per_mesh.append([round(float(x), 4) for x in st])
        assert g.SetProfile(False)
    b = AsmBatch(hs)
    assert b.SetStream(stream.cuda_stream)
    for _ in range(a.warmup):
        assert b.Assemble(True)
    torch.cuda.synchronize()
    clk = ClockSampler(dev)
    if dist is not None:
        dist.barrier()
    clk.start()
    launches0 = _lib.lib().lfasm_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(a.steps):
        assert b.Assemble(True)
    ev1.record(stream)
    ev1.synchronize()
    launches = _lib.lib().lfasm_launch_count() - launches0
    clocks = clk.stop()
    ms = ev0.elapsed_time(ev1) / a.steps
    ms = replicas.max_over_ranks(ms, dist, "cuda")
    total_all = replicas.sum_over_ranks(total, dist, "cuda")
    if dist is not None:
        dist.barrier()
    value = total_all / (ms * 1e-3)
    b.Release()
    for g in hs:
        g.Release()
    e2e = run_batch_e2e(a, cases, dev, torch)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs") or 6650.0
    fp64 = fp64_peak_tflops(torch)
    kern = {nm: {"ms": float(t)} for nm, t in zip(["prep+bulk", "pml", "gather"], stages)}
    gb = sum(c.ad.ne * c.ad.nd * c.ad.nd * 18 + c.ad.ne * c.ad.nd * 4 + (c.ad.height + 1) * 8
             + c.nnz * 16 for c in cases)
    kern["gather"]["GB/s"] = gb / (stages[2] * 1e-3) / 1e9
    flops = 0.0
    for c, v in zip(cases, pml_var):
        flops += pml_flops(int(np.sum(_pml_mask(c))), c.ad.nd, c.ad.rule_cc.nq,
                           c.ad.rule_mass.nq, c.prob.has_kpar, v)
    kern["pml"]["TFLOP/s"] = flops / (stages[1] * 1e-3) / 1e12 if stages[1] > 0 else 0.0
    kern["pml"]["variants"] = [PML_KERNELS[v] for v in pml_var]
    top = int(np.argmax(stages))
    if top == 1:
        roof = {"kernel": "/".join(sorted({PML_KERNELS[v] for v in pml_var})), "bound": "tensor",
                "achieved": kern["pml"]["TFLOP/s"],
                "peak": fp64, "unit": "TFLOP/s", "frac": kern["pml"]["TFLOP/s"] / fp64,
                "peak_source": "measured in-run: cuBLAS DGEMM 8192^3", "traffic": None}
    else:
        nm = "gather" if top == 2 else "prep+bulk"
        if nm == "prep+bulk":
            bb = sum(float(np.sum(~_pml_mask(c))) * (c.ad.nd ** 2 * 16 + 256) for c in cases)
            kern[nm]["GB/s"] = bb / (stages[0] * 1e-3) / 1e9
        bulk_names = "/".join(sorted({BULK_KERNELS[v].split("<")[0].split(" ")[0] for v in bulk_var}))
        roof = {"kernel": {"gather": "k_gather", "prep+bulk": bulk_names}[nm], "bound": "hbm",
                "achieved": kern[nm]["GB/s"], "peak": hbm, "unit": "GB/s",
                "frac": kern[nm]["GB/s"] / hbm,
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)", "traffic": None}
    roof["what"] = "stage times summed over the 16 meshes (serial profile pass)"
    cpu = None
    if not a.no_cpu_baseline and world == 1:
        cpu = cpu_baseline_batch(cases, a.cpu_seconds, 1)
    cfg = batch_workload_config(cases, a)
    cfg["parallelism"] = (f"16 meshes sharded round-robin over {world} GPUs"
                          if world > 1 else "one GPU")
    cfg["nnz_all_ranks"] = int(total_all)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": "f64 (complex128)", "data": "synthetic",
            "config": cfg, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clocks, "roofline": roof,
            "cpu_baseline": cpu, "kernels": kern, "fp64_peak_tflops": fp64,
            "serial_per_handle_ms": serial_ms,
            "per_mesh_stage_ms": per_mesh}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def _pml_mask(c) -> np.ndarray:
    """Elements with a quadrature point in the PML (the classification of the
    library: z outside [z_min, z_max] at any point of either rule)."""
    ad, prob = c.ad, c.prob
    J = ad.J.reshape(ad.ne, 3, 3)
    z0 = ad.v0.reshape(ad.ne, 3)[:, 2]
    out = np.zeros(ad.ne, dtype=bool)
    for r in (ad.rule_cc, ad.rule_mass):
        z = z0[:, None] + J[:, 2, :] @ np.asarray(r.ip).reshape(-1, 3).T
        out |= ((z < prob.z_min) | (z > prob.z_max)).any(axis=1)
    return out


def run_batch_e2e(a, cases, dev, torch) -> dict | None:
    """e2e of the batch: every mesh's lfasm_init from pinned host arrays +
    lfasm_build_global, one batched assembly, D2H of all CSR values."""
    from lithofem_b200.asm import AsmBatch, AsmGpuGlobal, DeviceVector
    import copy
    if a.e2e_steps <= 0:
        return None
    ads, h2d = [], 0
    for c in cases:
        ad = copy.copy(c.ad)
        for name in ("dof", "sign", "fo", "attr", "J", "Jinv", "detJ", "v0"):
            arr = getattr(ad, name)
            t = torch.empty(arr.shape, dtype=getattr(torch, str(arr.dtype)), pin_memory=True)
            t.numpy()[...] = arr
            setattr(ad, name, t.numpy())
            h2d += arr.nbytes
        for r in (ad.rule_cc, ad.rule_mass):
            h2d += r.ip.nbytes + r.w.nbytes + r.vshape.nbytes + r.curl.nbytes
        h2d += ad.ess.nbytes
        ads.append(ad)
    total = sum(c.nnz for c in cases)
    outs = [torch.empty(2 * c.nnz, dtype=torch.float64, pin_memory=True) for c in cases]
    times = []
    parts = []
    for it in range(1 + a.e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hs = []
        for c, ad in zip(cases, ads):
            g = AsmGpuGlobal(c.prob)
            assert g.Init(ad, dev) and g.BuildGlobal(ad.ess)
            hs.append(g)
        ta = time.perf_counter()
        b = AsmBatch(hs)
        assert b.Assemble(True)
        tb = time.perf_counter()
        for g, o in zip(hs, outs):
            _, _, V, _, nz = g._csr()
            o.copy_(torch.as_tensor(DeviceVector(V, (2 * nz,), "<f8"), device="cuda"),
                    non_blocking=True)
        torch.cuda.synchronize()
        tc = time.perf_counter()
        b.Release()
        for g in hs:
            g.Release()
        t1 = time.perf_counter()
        if it >= 1:
            times.append(t1 - t0)
            parts.append([ta - t0, tb - ta, tc - tb, t1 - tc])
    t = float(np.median(times))
    return {"value": total / t, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(16 * total), "ms_per_step": 1e3 * t,
            "what": "per mesh lfasm_init (pinned host arrays) + lfasm_build_global, one "
                    "lfasm_batch_assemble (graph capture included), D2H of all CSR values",
            "breakdown_ms": dict(zip(["init+build_global (16 handles)",
                                      "batch create+capture+assemble", "d2h", "release"],
                                     (np.median(np.array(parts), axis=0) * 1e3).tolist())),
            "timer": "host wall clock with device synchronize on both sides"}


def cpu_baseline_batch(cases, budget_s: float, threads: int) -> dict:
    """The reference's CPU reassembler on a bounded sample of every mesh;
    nnz/s = total nnz / sum of the per-mesh extrapolated times."""
    t_sum, kinds, elems = 0.0, set(), 0
    for c in cases:
        info = cpu_baseline_reference(c, budget_s / len(cases), threads)
        t_sum += c.nnz / info["value"]
        kinds.add(info["kind"])
        elems += int(info["sample"].split(" of ")[0])
    return {"value": sum(c.nnz for c in cases) / t_sum, "unit": UNIT, "cores": threads,
            "kind": "reference" if kinds == {"reference"} else "port",
            "sample": f"{elems} elements over {len(cases)} meshes, reassemble_all per mesh on "
                      f"its sample's own CSR, extrapolated per mesh"}


def run_reference_batch(a, rank, world, dist):
    """The reference's CPU assembly of all 16 meshes per step, each mesh as
    in run_reference (reassemble_all over contiguous element shares into the
    mesh's full CSR rows, on every host thread); a step's wall time is the
    sum over the meshes."""
    from lithofem_b200 import configs
    from oracle import oracle
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    cases = configs.batch_config(scale=a.scale)
    threads = os.cpu_count() or 1
    shs = []
    for c in cases:
        rc, I, J = _reference_csr(c)
        c.nnz = len(J)
        if rc is not None:
            shs.append(oracle.RefShares(c.ad, c.prob, I, J,
                                        oracle.contiguous_shares(c.ad.ne, 4 * threads)))
    total = sum(c.nnz for c in cases)
    if len(shs) == len(cases):
        walls = [sum(sh.time_parallel(threads) for sh in shs)
                 for _ in range(a.warmup + a.steps)][a.warmup:]
        kind = "reference"
        sample = (f"all elements of all {len(cases)} meshes every step: reassemble_all over "
                  f"{4 * threads} contiguous element shares per mesh on {threads} threads, "
                  f"into each mesh's full CSR rows")
    else:
        walls = []
        for _ in range(a.warmup + a.steps):
            info = cpu_baseline_batch(cases, 4.0, threads)
            walls.append(total / info["value"])
        walls = walls[a.warmup:]
        kind, sample = "port", info["sample"]
    del shs
    ms = 1e3 * float(np.mean(walls))
    v = total / (ms * 1e-3)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": batch_workload_config(cases, a),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "step_wall_s": [round(w, 4) for w in walls]}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
