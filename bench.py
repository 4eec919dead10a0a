"""Benchmark: eigensolves/s at relative residual <= 1e-10 on one B200.

Workload (the single complex non-Hermitian solve): n = 16384 dense complex A
in split re/im FP64 planes (reference layout), entries N(0, 1/n) (each plane
N(0, 1/(2n))) plus 4 added on 16 seeded diagonal positions; the 16
largest-magnitude eigenpairs, Krylov dimension m = 64; an eigensolve counts
only when every wanted pair has ||A x - l x|| / (|l_1| ||x||) <= 1e-10 in
FP64 against the FP64 operator.  Synthetic seeded data; A (4 GiB) is far
larger than L2, so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One JSON line on rank 0.  `value` is the chosen form (split-BF16 tcgen05
block subspace iteration, then FP64-anchored refinement: FP64-class residual
passes on int8 operator slices (integer tcgen05) and FP32-class Sylvester
corrections) with A resident in HBM;
`plain_fp64` is the plain FP64 GPU
Arnoldi on the same problem; `e2e` runs the C-ABI entry that takes HOST
buffers (pinned), with the 4 GiB host-to-device copy of A inside every step.
With N > 1 GPUs every rank solves its own replica (the solve does not shard).
`--impl reference` times the CPU implementation of the path (the oracle's
FP64 IRAM) on this host's cores, on a bounded sample of the same workload.
"""

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N, K_WANTED, M_KRYLOV, NPLANT, SHIFT, TOL = 16384, 16, 64, 16, 4.0, 1e-10
DMMA_PEAK_TFLOPS = 37.1  # mma.sync.m16n8k4.f64 throughput measured on B200 (register operands)
FMA64_PEAK_TFLOPS = 34.0  # FP64 FMA throughput measured on B200 (register operands)
METRIC = "eigensolves/s at residual≤1e-10: chosen form vs plain FP64 GPU Arnoldi"
WORKLOAD = "complex non-Hermitian dense A, n=16384, split re/im FP64, N(0,1/n) + 4 on 16 planted diagonal entries; top-16 LM, m=64"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--e2e-steps", type=int, default=None)
    p.add_argument("--plain-steps", type=int, default=None)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--n", type=int, default=N)
    p.add_argument("--quick", action="store_true",
                   help="profiling run: time one form only, no plain / e2e / CPU legs")
    p.add_argument("--form", default="mixed", choices=["mixed", "plain"],
                   help="form timed by --quick")
    p.add_argument("--no-tc", action="store_true",
                   help="FP32 block passes on CUDA cores instead of the split-BF16 tensor-core pass")
    p.add_argument("--train", type=int, default=20000, help="warm-start training solves")
    p.add_argument("--held-out", type=int, default=48, help="warm-start evaluation solves")
    p.add_argument("--gram-side", type=int, default=128,
                   help="image side of the --config gram --quick build (4096 images)")
    p.add_argument("--train-smooth", type=int, default=4096,
                   help="warm-start training solves of the family with its parameter operators scaled by 0.01")
    p.add_argument("--config", default="single", choices=["single", "batched", "gram", "warmstart"],
                   help="single: the n=16384 complex solve (default line); batched: 2048 uneven "
                        "complex problems n in [32, 512], top-4, hdim=min(n, 24)")
    p.add_argument("--batch", type=int, default=2048)
    p.add_argument("--no-others", action="store_true",
                   help="default line without the bounded n=256, Gram-build and batched sub-results")
    return p.parse_args()


def make_operator(n, seed, device):
    """Seeded complex A on `device` as two FP64 planes (rows, columns)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    s = (1.0 / (2.0 * n)) ** 0.5
    are = torch.randn(n, n, dtype=torch.float64, device=device, generator=g).mul_(s)
    aim = torch.randn(n, n, dtype=torch.float64, device=device, generator=g).mul_(s)
    pos = torch.randperm(n, generator=g, device=device)[:NPLANT]
    are[pos, pos] += SHIFT
    return are, aim


def fp64_residuals(are, aim, ev, xre, xim):
    """||A x_q - l_q x_q|| / (|l_1| ||x_q||) for every pair, recomputed from
    the FP64 operator planes with torch (cuBLAS DGEMM, outside the library):
    are / aim (n, n) device FP64, xre / xim (n, k) device FP64 (column q =
    eigenvector q), ev the k eigenvalues (l_1 = the largest |l|)."""
    import torch
    lr = torch.tensor([e.real for e in ev], dtype=torch.float64, device=are.device)
    li = torch.tensor([e.imag for e in ev], dtype=torch.float64, device=are.device)
    if aim is None:
        wr, wi = are @ xre, are @ xim if xim is not None else None
    else:
        wr = are @ xre - aim @ xim
        wi = are @ xim + aim @ xre
    xi = xim if xim is not None else torch.zeros_like(xre)
    wi = wi if wi is not None else torch.zeros_like(xre)
    rr = wr - (xre * lr - xi * li)
    ri = wi - (xre * li + xi * lr)
    num = torch.sqrt((rr * rr + ri * ri).sum(0))
    den = torch.sqrt((xre * xre + xi * xi).sum(0)) * max(abs(e) for e in ev)
    return (num / den).tolist()


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.f.flush()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            rows = open(self.f.name).read().strip().splitlines()
        except OSError:
            rows = []
        for row in rows:
            parts = [x.strip() for x in row.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic():
    """dram bytes per launch of the FP32 matvec from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


class gpu_local_cpus:
    """Within the block, run on the CPUs NVML reports as local to GPU
    `index` (so host memory allocated there lands on its NUMA node); the
    previous affinity is restored on exit.  No-op where NVML or affinity
    control is unavailable."""

    def __init__(self, index):
        self.index = index
        self.old = None

    def __enter__(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            # NVML numbers GPUs without CUDA_VISIBLE_DEVICES: find ours by PCI address
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            words = pynvml.nvmlDeviceGetCpuAffinity(h, 16)
            cpus = {i * 64 + b for i, w in enumerate(words) for b in range(64) if (int(w) >> b) & 1}
            cpus &= set(range(os.cpu_count() or 1))
            if cpus:
                self.old = os.sched_getaffinity(0)
                os.sched_setaffinity(0, cpus)
        except Exception:
            self.old = None
        return self

    def __exit__(self, *exc):
        if self.old:
            try:
                os.sched_setaffinity(0, self.old)
            except OSError:
                pass
        return False


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(world, x):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allsum(world, x):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# --------------------------------------------------------------- CPU arm --
def config_dict(world, n):
    """The workload description both arms print (the same dict)."""
    return {"workload": WORKLOAD, "n": n, "wanted": K_WANTED, "hdim": M_KRYLOV, "tolerance": TOL,
            "chosen_form": ("split-BF16 tcgen05 (FP32-class) block subspace iteration, its leading powers "
                            "on the BF16 hi planes, then FP64-anchored refinement: FP64-class residual on "
                            "int8 operator slices (integer tcgen05) + "
                            "Sylvester corrections (leading sweeps BF16, the rest FP32-class)"),
            "parallelism": "replicas" if world > 1 else "single GPU",
            "l2": "inputs (4 GiB FP64 + 2 GiB BF16 hi/lo + 3 GiB int8-slice operator) exceed L2; no flush"}


def oracle_solve(are_h, aim_h):
    """One whole FP64 eigensolve of the workload by the CPU oracle (textbook
    IRAM, OpenMP matvec on all host cores): (seconds, converged, result)."""
    import oracle as O
    t0 = time.perf_counter()
    r = O.iram_planes(are_h, aim_h, K_WANTED, M_KRYLOV, which="LM", tol=TOL, seed=1)
    dt = time.perf_counter() - t0
    ok = r["rc"] == 0 and r["converged"] and float(r["residuals"].max()) <= TOL
    return dt, ok, r


def cpu_sample(are_h, aim_h, budget_s, n):
    """The CPU implementation of the path timed on this host: whole oracle
    FP64 IRAM solves of the full workload until `budget_s` is spent (at
    least one); eigensolves/s = converged solves / their time."""
    import oracle as O
    times, conv, r = [], 0, None
    t_start = time.perf_counter()
    while not times or time.perf_counter() - t_start < budget_s:
        dt, ok, r = oracle_solve(are_h, aim_h)
        times.append(dt)
        conv += int(ok)
    total = sum(times)
    return {"value": conv / total, "unit": "eigensolves/s", "cores": O.num_threads(), "kind": "port",
            "sample": ("%d whole oracle FP64 IRAM solves of the n=%d workload (%d converged, %.2f s each, "
                       "%d restarts, %d operator applications + %d residual checks each)")
            % (len(times), n, conv, total / len(times), r["restarts"], r["matvecs"], K_WANTED),
            "solve_seconds": total / len(times), "eigenvalues": r["eigenvalues"]}


def run_reference(args, world, rank):
    if rank != 0:
        return
    import torch
    n = args.n
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    are, aim = make_operator(n, 1, dev)
    are_h = are.cpu().numpy()
    aim_h = aim.cpu().numpy()
    del are, aim
    import oracle as O
    # every step is one whole solve of the workload by the oracle's FP64 IRAM
    # on all host cores; the timed region is the K timed steps
    for _ in range(args.warmup):
        oracle_solve(are_h, aim_h)
    t0 = time.perf_counter()
    conv, per = 0, []
    r = None
    for _ in range(args.steps):
        dt, ok, r = oracle_solve(are_h, aim_h)
        per.append(dt)
        conv += int(ok)
    secs = time.perf_counter() - t0
    v = conv / secs
    sample = ("one whole oracle FP64 IRAM solve of the n=%d workload per step (%.2f s median, %d restarts, "
              "%d operator applications + %d residual checks), %d of %d converged to 1e-10") % (
        n, statistics.median(per), r["restarts"], r["matvecs"], K_WANTED, conv, args.steps)
    out = {"metric": METRIC, "value": v, "unit": "eigensolves/s", "impl": "reference",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
           "data": "synthetic (seeded)",
           "config": config_dict(world, n),
           "cpu_baseline": {"value": v, "unit": "eigensolves/s", "cores": O.num_threads(), "kind": "port",
                            "sample": sample},
           "e2e": {"value": v, "unit": "eigensolves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# --------------------------------------------------------------- GPU arm --
def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    import oap_b200 as B

    torch.cuda.set_device(local)
    n = args.n
    are, aim = make_operator(n, 1 + rank, "cuda")
    torch.cuda.synchronize()

    def solver(prec):
        s = B.Arnoldi(n, M_KRYLOV, K_WANTED, is_complex=True, precision=prec, tolerance=TOL,
                      profile=True, seed=3 + rank, tensor_cores=not args.no_tc)
        s.set_operator(are, aim)
        return s

    def timed(s, steps, warm):
        for _ in range(warm):
            ev, res, st = s.solve()
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = s.stats()["kernel_launches"]
        prof = {"matvec_seconds": 0.0, "matvec_timed": 0, "block_seconds": 0.0, "block_timed": 0,
                "block_fp32_seconds": 0.0, "block_fp32_timed": 0, "block_fp32_width": 0,
                "block_bf16_seconds": 0.0, "block_bf16_timed": 0,
                "pass_kernel_seconds": [0.0, 0.0, 0.0], "pass_kernel_timed": [0, 0, 0]}
        conv = 0
        # per-launch CUDA events (the roofline's kernel times) on the last
        # third of the timed solves: an event pair around a pass also breaks
        # the dependent-launch overlap of its kernels, so the rest run bare
        nprof = max(1, steps // 3)
        s.set_profile(False)
        e0.record()
        for i in range(steps):
            if i == steps - nprof:
                s.set_profile(True)
            ev, res, st = s.solve(allow_not_converged=True)
            stt = s.stats()
            for key in prof:
                if key == "block_fp32_width":
                    prof[key] = stt[key]
                elif isinstance(prof[key], list):
                    prof[key] = [x + y for x, y in zip(prof[key], stt[key])]
                else:
                    prof[key] += stt[key]
            conv += int(st == B.OK and max(res) <= TOL)
        e1.record()
        torch.cuda.synchronize()
        barrier(world)
        ms = e0.elapsed_time(e1)
        prof["profiled_solves"] = nprof
        return ms / 1e3, conv, prof, s.stats()["kernel_launches"] - launches0, stt, ev

    if args.quick:
        s_q = solver(B.PREC_MIXED if args.form == "mixed" else B.PREC_FP64)
        secs, conv, prof, launches, stt, _ = timed(s_q, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"quick": True, "form": args.form, "n": n, "steps": args.steps,
                              "seconds": secs, "converged": conv, "launches": launches, "profile": prof,
                              "stats": stt}), flush=True)
        s_q.close()
        return
    # chosen form
    mixed = solver(B.PREC_MIXED)
    with Clocks(local) as clk:
        secs, conv, prof, launches, stt, ev_mixed = timed(mixed, args.steps, args.warmup)
    clocks = clk.summary()
    secs_max = allmax(world, secs)
    conv_all = allsum(world, conv)
    value = conv_all / secs_max
    # plain FP64 GPU Arnoldi
    plain = solver(B.PREC_FP64)
    psteps = args.plain_steps or max(2, args.steps // 2)
    psecs, pconv, pprof, _, pstt, ev_plain = timed(plain, psteps, 1)
    pvalue = allsum(world, pconv) / allmax(world, psecs)
    plain.close()
    # parity of the timed solves: one chosen-form solve's eigenpairs rechecked
    # outside the library (FP64 planes x eigenvectors by torch's FP64 GEMM),
    # and its eigenvalues against the plain FP64 GPU Arnoldi's, matched in the
    # SortLargestValues order
    import oracle as O
    xr = torch.zeros(n, K_WANTED, dtype=torch.float64, device="cuda")
    xi = torch.zeros(n, K_WANTED, dtype=torch.float64, device="cuda")
    ev_chk, res_chk, st_chk = mixed.solve(vectors=(xr, xi), allow_not_converged=True)
    fp64_res = fp64_residuals(are, aim, ev_chk, xr, xi)
    del xr, xi
    lm = lambda ev: sorted(ev, key=lambda e: -abs(e))
    fp64_check = {"max_residual": max(fp64_res), "library_max_residual": max(res_chk), "status": st_chk,
                  "method": "torch FP64 GEMM of the FP64 operator planes with the returned eigenvectors",
                  "eig_err_vs_fp64": O.match_eigenvalues(lm(ev_mixed), lm(ev_plain)),
                  "eig_err_note": "max |l_chosen - l_plain| / max|l| over the 16 wanted values, "
                                  "plain FP64 GPU Arnoldi of the same run, SortLargestValues order"}
    # per-operator preparation of the chosen form (BF16 hi / lo planes and
    # int8 slices), outside `value`'s timed loop: set_operator on a handle
    # whose buffers exist (a new operator for a reused handle), and the first
    # set_operator of a fresh handle (which also allocates about 5 GiB)
    prep = B.Arnoldi(n, M_KRYLOV, K_WANTED, is_complex=True, precision=B.PREC_MIXED, tolerance=TOL,
                     seed=3 + rank)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prep.set_operator(are, aim)
    torch.cuda.synchronize()
    prep_first_ms = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    prep.set_operator(are, aim)
    torch.cuda.synchronize()
    prep_ms = (time.perf_counter() - t0) * 1e3
    prep.close()
    # end to end through the host-buffer entry point (pinned host planes)
    # the pinned host planes on the GPU's own NUMA node (as a serving process
    # bound to its GPU's socket would have them)
    with gpu_local_cpus(local):
        are_h = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        aim_h = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        are_h.copy_(are)
        aim_h.copy_(aim)
    e2e_solver = B.Arnoldi(n, M_KRYLOV, K_WANTED, is_complex=True, precision=B.PREC_MIXED,
                           tolerance=TOL, seed=3 + rank)
    ar_np, ai_np = are_h.numpy(), aim_h.numpy()
    esteps = args.e2e_steps or max(2, args.steps // 2)
    e2e_solver.solve_host(ar_np, ai_np, vectors=True)  # warm-up (allocations)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    econv = 0
    for _ in range(esteps):
        ev, res, st, X = e2e_solver.solve_host(ar_np, ai_np, vectors=True)
        econv += int(st == B.OK and max(res) <= TOL)
    e1.record()
    torch.cuda.synchronize()
    esecs = allmax(world, e0.elapsed_time(e1) / 1e3)
    e2e_value = allsum(world, econv) / esecs
    e2e_solver.close()

    # roofline of the dominant kernel of the chosen form (largest total device
    # time among the timed operator kernels), HBM-bound by design
    hbm, peak_kind = peaks()
    bw = prof["block_fp32_width"] or K_WANTED
    # algorithmic bytes per pass: the operator once (FP32-class pass: BF16
    # hi + lo of both planes, 8 n^2; BF16 pass: the hi planes, 4 n^2; FP64
    # pass: 16 n^2) plus X in and W out (FP64 planes, 32 b n); flops 8 b n^2
    # (complex)
    fp32_name = ("k_block_matvec_tc<complex> (split-BF16 tcgen05 block pass, %d vectors)" % bw if not args.no_tc
                 else "k_block_matvec<float,complex> (FP32 CUDA-core block pass, %d vectors)" % bw)
    # the FP64-class pass of the chosen form: int8 operator slices on the
    # integer tensor cores (6 slices of both planes, 12 n kp bytes a pass;
    # 27 slice products of M 128, N 2 QB, K kp) or, where it does not apply,
    # the FP64 DMMA pass (16 n^2 bytes)
    i8 = (not args.no_tc) and stt.get("block_i8", 0) > 0
    kp = (n + 127) // 128 * 128
    qb = (bw + 7) // 8 * 8
    fp64_name = ("k_block_matvec_i8<complex> (FP64-class int8-slice tcgen05 block pass)" if i8
                 else "k_block_matvec_dmma<complex> (FP64 DMMA block pass)" if not args.no_tc
                 else "k_block_matvec<double,complex> (FP64 CUDA-core block pass)")
    fp64_bytes = (12.0 * n * kp if i8 else 16.0 * n * n) + 32.0 * bw * n
    # the tensor-core passes are timed by events right around their kernel
    # (pass_kernel_*: [0] FP64-class, [1] split, [2] BF16); the unit times
    # (block_*_seconds) also hold the vector split and the stream-K reduction
    pk_s, pk_n = prof["pass_kernel_seconds"], prof["pass_kernel_timed"]
    tc_fp32 = (not args.no_tc) and pk_n[1] > 0
    tc_fp64 = (not args.no_tc) and pk_n[0] > 0
    kernels = {
        "k_matvec<float,complex> (FP32 complex matvec)":
            (prof["matvec_seconds"], prof["matvec_timed"], 8.0 * n * n + 16.0 * n, 8.0 * n * n),
        fp32_name:
            ((pk_s[1], pk_n[1]) if tc_fp32 else (prof["block_fp32_seconds"], prof["block_fp32_timed"])) +
            (8.0 * n * n + 32.0 * bw * n, 8.0 * bw * n * n),
        fp64_name:
            ((pk_s[0], pk_n[0]) if tc_fp64 else (prof["block_seconds"], prof["block_timed"])) +
            (fp64_bytes, 8.0 * bw * n * n),
    }
    if not args.no_tc:
        kernels["k_block_matvec_tc<complex, BF16> (BF16 hi-plane tcgen05 block pass)"] = (
            pk_s[2], pk_n[2], 4.0 * n * n + 32.0 * bw * n, 8.0 * bw * n * n)
    # the same passes with their vector split and stream-K reduction (what a
    # pass costs the solve)
    units = {fp32_name: (prof["block_fp32_seconds"], prof["block_fp32_timed"]),
             fp64_name: (prof["block_seconds"], prof["block_timed"])}
    if not args.no_tc:
        units["k_block_matvec_tc<complex, BF16> (BF16 hi-plane tcgen05 block pass)"] = (
            prof["block_bf16_seconds"], prof["block_bf16_timed"])
    name, (tot, cnt, alg_bytes, flops) = max(kernels.items(), key=lambda kv: kv[1][0])
    per_launch = tot / max(1, cnt)
    achieved = alg_bytes / per_launch / 1e9 if per_launch > 0 else 0.0
    traffic = ncu_traffic()
    roof = {"bound": "hbm", "kernel": name,
            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind),
            "traffic": (traffic or {}).get(name.split(" (")[0], {}).get("bytes_per_launch") if traffic else None,
            "launch_ms": per_launch * 1e3, "launches_timed": cnt, "algorithmic_bytes_per_launch": alg_bytes,
            "tflops": flops / per_launch / 1e12 if per_launch > 0 else 0.0,
            "timing": "CUDA events recorded right before and after the pass kernel's launch on its stream",
            # the kernel's device time per profiled solve over the time per solve
            "share_of_step": (tot / prof["profiled_solves"]) / (secs / args.steps) if secs > 0 else None,
            "with_split_and_reduce": {k: {"launches": v[1], "ms_per_launch": v[0] / v[1] * 1e3 if v[1] else None,
                                          "frac": (kernels[k][2] / (v[0] / v[1]) / 1e9 / hbm) if v[1] else None}
                                      for k, v in units.items()},
            "all_kernels": {k: {"launches": v[1], "total_ms": v[0] * 1e3,
                                "GBs": (v[2] / (v[0] / v[1]) / 1e9) if v[1] else None,
                                "frac": (v[2] / (v[0] / v[1]) / 1e9 / hbm) if v[1] else None,
                                "algorithmic_bytes_per_launch": v[2],
                                "tflops": (v[3] / (v[0] / v[1]) / 1e12) if v[1] else None,
                                "traffic": (traffic or {}).get(k.split(" (")[0], {}).get("bytes_per_launch")}
                            for k, v in kernels.items()},
            # the int8-slice pass is HBM-bound (its fraction of the measured
            # copy bandwidth, and its integer tensor throughput: 2 x 2 planes x
            # 27 products x 2 QB x n x kp ops); the FP64 DMMA pass is bound by
            # the FP64 tensor pipe (its fraction of the DMMA throughput measured
            # on this pool with a register-only mma.sync f64 loop)
            "fp64_pass": ({"bound": "hbm", "kernel": fp64_name,
                           "GBs": fp64_bytes / (kernels[fp64_name][0] / kernels[fp64_name][1]) / 1e9,
                           "peak": hbm, "frac": fp64_bytes / (kernels[fp64_name][0] / kernels[fp64_name][1]) / 1e9 / hbm,
                           "int8_tops": 2.0 * 2 * 27 * 2 * qb * n * kp /
                           (kernels[fp64_name][0] / kernels[fp64_name][1]) / 1e12,
                           "launch_ms": kernels[fp64_name][0] / kernels[fp64_name][1] * 1e3,
                           "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)"}
                          if i8 and kernels[fp64_name][1] else
                          {"bound": "fp64 fma" if args.no_tc else "fp64 tensor",
                           "tflops": kernels[fp64_name][3] / (kernels[fp64_name][0] / kernels[fp64_name][1]) / 1e12,
                           "peak_tflops": FMA64_PEAK_TFLOPS if args.no_tc else DMMA_PEAK_TFLOPS,
                           "frac": kernels[fp64_name][3] / (kernels[fp64_name][0] / kernels[fp64_name][1]) / 1e12 /
                           (FMA64_PEAK_TFLOPS if args.no_tc else DMMA_PEAK_TFLOPS),
                           "peak_source": "own throughput probe (register operands)"}
                          if kernels[fp64_name][1] else None),
            "plain_fp64_matvec_GBs": ((16.0 * n * n + 32.0 * n) / (pprof["matvec_seconds"] / pprof["matvec_timed"]) / 1e9
                                      if pprof["matvec_timed"] else None)}

    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_sample(ar_np, ai_np, args.cpu_seconds, n)
        fp64_check["eig_err_vs_oracle"] = O.match_eigenvalues(lm(ev_chk), lm(cpu["eigenvalues"]))
    # the other configurations, bounded, at one GPU (their own workloads)
    others = None
    if world == 1 and not args.no_others:
        del ar_np, ai_np, are_h, aim_h
        others = {"c1_n256_real_symmetric": c1_result(), "c3_gram_build": c3_result(),
                  "c4_batched": c4_result(), "c5_warmstart_smooth": c5_result()}
    out = {"metric": METRIC, "value": value, "unit": "eigensolves/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs_max * 1e3 / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3(fp32-class)+int8-slice(fp64-class)+f64",
           "data": "synthetic (seeded)",
           "config": config_dict(world, n),
           "converged_steps": conv_all,
           "plain_fp64": {"value": pvalue, "ms_per_step": allmax(world, psecs) * 1e3 / psteps,
                          "steps": psteps, "restarts": pstt["restarts"], "matvecs": pstt["matvecs"]},
           "speedup_vs_plain_fp64": value / pvalue if pvalue else None,
           "solve": {"restarts": stt["restarts"], "matvecs": stt["matvecs"],
                     "block_matvecs": stt["block_matvecs"], "bf16_passes": stt["block_bf16"],
                     "refine_iterations": stt["refine_iterations"],
                     "max_residual": stt["max_residual"]},
           "e2e": {"value": e2e_value, "unit": "eigensolves/s",
                   "h2d_bytes_per_step": 2 * 8 * n * n,
                   "d2h_bytes_per_step": 3 * 8 * K_WANTED + 2 * 8 * n * K_WANTED,
                   "steps": esteps},
           "fp64_check": fp64_check,
           "prep_ms": prep_ms,
           "prep_first_ms": prep_first_ms,
           "value_incl_prep": conv_all / (secs_max + prep_ms / 1e3 * args.steps),
           "other_configs": others,
           "roofline": roof, "clocks": clocks,
           "gpu_launches": int(launches),
           "cpu_baseline": None if cpu is None else {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}}
    mixed.close()
    if rank == 0:
        print(json.dumps(out), flush=True)


def make_batch(count, seed):
    """`count` complex problems, n ~ U{32..512} (numpy seed), entries N(0, 1/n)
    split re / im FP64 plus 4 on 4 seeded diagonal positions, on the device."""
    import numpy as np
    import torch
    rng = np.random.default_rng(seed)
    sizes = rng.integers(32, 513, size=count)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    mats = []
    for n in sizes:
        n = int(n)
        s = (1.0 / (2.0 * n)) ** 0.5
        re = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g).mul_(s)
        im = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g).mul_(s)
        pos = torch.randperm(n, generator=g, device="cuda")[:4]
        re[pos, pos] += SHIFT
        mats.append((re, im))
    return rng, sizes, mats


def c1_result():
    """The reference's CPU-sized case (n = 256 real symmetric, Q diag(l) Q^T
    with Q from the QR of a seeded N(0,1) matrix, l geometric 1 .. 1e-3,
    top-5 LM, m = 32, residual goal 1e-10): GPU solves/s (the chosen form's
    handle; below n = 8192 it runs the plain FP64 restart loop) beside the
    CPU oracle's whole solves, and the eigenvalue errors against the exact
    values and the oracle."""
    import numpy as np
    import torch
    import oap_b200 as B
    import oracle as O
    n, k, m = 256, 5, 32
    rng = np.random.default_rng(0)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    lam = 10.0 ** (-3.0 * np.arange(n) / (n - 1))
    A = (Q * lam) @ Q.T
    s = B.Arnoldi(n, m, k, precision=B.PREC_MIXED, tolerance=TOL, seed=1)
    s.set_operator(torch.from_numpy(A).cuda())
    for _ in range(3):
        s.solve()
    steps, conv = 50, 0
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        ev, res, st = s.solve(allow_not_converged=True)
        conv += int(st == B.OK and max(res) <= TOL)
    e1.record()
    torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    stt = s.stats()
    s.close()
    ev = np.array(sorted(ev, key=lambda e: -abs(e)))
    t0, cnt, o = time.perf_counter(), 0, None
    while cnt < 3 or time.perf_counter() - t0 < 1.0:
        o = O.iram(A, k, m, which="LM", tol=TOL, seed=1)
        cnt += 1
    cpu_s = (time.perf_counter() - t0) / cnt
    oev = np.array(sorted(o["eigenvalues"], key=lambda e: -abs(e)))
    # the reference's own algorithm as written (oracle reference-faithful
    # mode: V^T projections over all columns, 1e-3 triangular gate,
    # CHECK_INTERNAL stop) on the same matrix and start-vector seed
    rf = O.iram_reference(A, k, m, which="LM", seed=1)
    rev = np.array(sorted(rf["eigenvalues"], key=lambda e: -abs(e)))
    ref_faithful = {"eig_err_vs_exact": float(np.abs(rev.real - lam[:k]).max() / lam[0]),
                    "eig_err_vs_textbook_oracle": O.match_eigenvalues(rev, oev),
                    "restarts": rf["restarts"], "matvecs": rf["matvecs"],
                    "note": "CuHArnoldi::execute restated as written; stops by CHECK_INTERNAL"}
    return {"workload": "n=256 real symmetric, l geometric 1..1e-3, top-5 LM, m=32, residual<=1e-10",
            "gpu_solves_per_s": conv / secs, "gpu_ms_per_solve": secs * 1e3 / steps, "converged": conv,
            "steps": steps, "restarts": stt["restarts"], "matvecs": stt["matvecs"],
            "cpu_oracle_solves_per_s": 1.0 / cpu_s, "cpu_oracle_cores": O.num_threads(),
            "eig_err_vs_exact": float(np.abs(ev.real - lam[:k]).max() / lam[0]),
            "eig_err_vs_oracle": O.match_eigenvalues(ev, oev),
            "max_residual": float(max(res)), "reference_faithful": ref_faithful}


def c3_result():
    """Gram build of 4096 synthetic 256 x 256 images (A = X X^T, split-BF16
    tcgen05, FP32 accumulation): milliseconds and algorithmic TFLOP/s
    (2 N^2 P counted once) against the measured bf16 peak."""
    import torch
    import oap_b200 as B
    count, side = 4096, 256
    X = synthetic_images(count, side, 21, "cuda")
    A, _ = B.gram_build(X)
    torch.cuda.synchronize()
    reps = 5
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        B.gram_build(X)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    flops = 2.0 * count * count * side * side
    peak, kind = bf16_peak()
    idx = torch.arange(0, count, 128, device="cuda")
    Xd = X.double()
    ref = Xd[idx] @ Xd.T
    rel = ((A[idx].double() - ref).abs() / ref.abs().clamp_min(1e-300)).max().item()
    del X, Xd, A
    return {"workload": "A = X X^T, X 4096 x 65536 FP32 synthetic images (8 Gaussian blobs + U[0,16) noise)",
            "build_ms": ms, "tflops_algorithmic": flops / ms / 1e9, "peak_bf16_tflops": peak,
            "peak_source": kind, "frac": flops / ms / 1e9 / peak, "rel_error_vs_fp64_max": rel,
            "note": "2 N^2 P flops counted once (the split runs three BF16 products)"}


def c5_result():
    """The learned warm start, bounded: the n = 2048 real symmetric family
    with the parameter operators scaled by 0.01 (where the wanted subspace is
    a smooth function of theta), 1024 training solves, 16 held-out solves
    from the prediction and from the random start on reused handles; the
    specified family (20k training solves) runs under --config warmstart."""
    from oap_b200 import warmstart as W
    n, k, hdim = 2048, 8, 24
    fam = W.ParamFamily(n=n, nparams=16, seed=31, scale=0.01)
    r = warmstart_family(fam, n, k, hdim, 1024, 16, 78, epochs=160)
    ho = r["held_out"]
    return {"workload": "A(theta) = A0 + 0.01 sum theta_i B_i, n=2048 real symmetric, 16 params, top-8 LR, "
                        "hdim 24; 1024 training solves, 16 held-out",
            "matvecs_per_solve_warm": ho["warm"]["matvecs_per_solve"],
            "matvecs_per_solve_random": ho["random"]["matvecs_per_solve"],
            "ms_per_solve_warm": ho["warm"]["seconds_per_solve"] * 1e3,
            "ms_per_solve_random": ho["random"]["seconds_per_solve"] * 1e3,
            "matvec_ratio": r["matvec_ratio"], "speedup_time": r["speedup_time"],
            "converged_warm": ho["warm"]["converged"], "converged_random": ho["random"]["converged"],
            "fallbacks": ho["warm"]["fallbacks"], "prediction_eps_median": r["prediction_eps_median"],
            "training_loss": [r["training"]["loss_first"], r["training"]["loss_last"]],
            "training_seconds": r["training"]["data_seconds"] + r["training"]["train_seconds"]}


def c4_result():
    """2048 uneven complex problems (n ~ U{32..512}, top-4 LM, hdim =
    min(n, 24)) in one persistent launch: solves/s, converged count, and the
    eigenvalue error against the plain FP64 Arnoldi on a sample of them."""
    import numpy as np
    import torch
    import oap_b200 as B
    import oracle as O
    rng, sizes, mats = make_batch(2048, 11)
    B.solve_batched(mats, 4, hdim=24, tolerance=TOL)
    torch.cuda.synchronize()
    reps, conv = 3, 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        ev, res, st, stats, rc = B.solve_batched(mats, 4, hdim=24, tolerance=TOL)
        conv += int((st == B.OK).sum())
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    err = 0.0
    for i in rng.choice(len(mats), 8, replace=False):
        re, im = mats[i]
        n = re.shape[0]
        p = B.Arnoldi(n, min(n, 24), 4, is_complex=True, tolerance=TOL, seed=3)
        p.set_operator(re, im)
        pev, _, _ = p.solve(allow_not_converged=True)
        p.close()
        err = max(err, O.match_eigenvalues(ev[i], pev))
    del mats
    hbm, kind = peaks()
    gbs = stats["operator_bytes"] / (ms / 1e3) / 1e9
    return {"workload": "2048 complex problems n~U[32,512], top-4 LM, hdim=min(n,24), one persistent launch",
            "solves_per_s": conv / reps / (ms / 1e3), "launch_ms": ms, "converged_per_launch": conv / reps,
            "variant": stats["variant"], "threads": stats["threads"], "ctas": stats["ctas"],
            "matvecs": stats["matvecs"], "restarts": stats["restarts"],
            "roofline": {"bound": "hbm", "algorithmic_bytes": stats["operator_bytes"], "achieved_GBs": gbs,
                         "peak": hbm, "frac": gbs / hbm,
                         "note": "operator bytes of every matvec (16 n^2 each, complex) over the launch time; the "
                                 "problems in flight exceed L2, so each matvec streams its operator from HBM"},
            "problems": len(sizes), "max_residual": float(res.max()),
            "eig_err_vs_plain_fp64_sample8": err}


def bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured (MEASURED_PEAKS.json bf16_tflops)"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def run_batched(args, world, rank, local):
    """2048 independent complex problems, sizes uniform in [32, 512], entries
    N(0, 1/n) split re/im FP64 plus 4 on 4 planted diagonal entries, top-4 LM,
    hdim = min(n, 24): one persistent launch vs the plain FP64 Arnoldi one
    problem at a time (timed on a sample of the same problems)."""
    import numpy as np
    import torch
    import oap_b200 as B
    torch.cuda.set_device(local)
    rng, sizes, mats = make_batch(args.batch, 11 + rank)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        B.solve_batched(mats, 4, hdim=24, tolerance=TOL)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    conv = 0
    for _ in range(args.steps):
        ev, res, st, stats, rc = B.solve_batched(mats, 4, hdim=24, tolerance=TOL)
        conv += int((st == B.OK).sum())
    e1.record()
    torch.cuda.synchronize()
    secs = allmax(world, e0.elapsed_time(e1) / 1e3)
    value = allsum(world, conv) / secs
    # plain FP64 Arnoldi, one problem at a time, on a sample of 64 problems
    idx = rng.choice(len(mats), 64, replace=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pconv = 0
    for i in idx:
        re, im = mats[i]
        n = re.shape[0]
        s1 = B.Arnoldi(n, min(n, 24), 4, is_complex=True, tolerance=TOL, seed=3)
        s1.set_operator(re, im)
        e, r, stt = s1.solve(allow_not_converged=True)
        pconv += int(stt == B.OK)
        s1.close()
    torch.cuda.synchronize()
    pt = time.perf_counter() - t0
    pvalue = pconv / pt
    algo_bytes = float(sum(16 * int(n) * int(n) for n in sizes))
    out = {"metric": METRIC, "value": value, "unit": "eigensolves/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
           "data": "synthetic (seeded)",
           "config": {"workload": "batched: %d complex problems n~U[32,512], top-4 LM, hdim=min(n,24)" % len(mats),
                      "parallelism": "replicas" if world > 1 else "single GPU"},
           "batched": {"converged_per_step": conv / args.steps, "matvecs_per_step": stats["matvecs"],
                       "restarts_per_step": stats["restarts"], "ctas": stats["ctas"],
                       "operator_bytes_all_problems": algo_bytes},
           "plain_fp64_one_at_a_time": {"value": pvalue, "sample": 64},
           "speedup_vs_plain_fp64": value / pvalue if pvalue else None}
    if rank == 0:
        print(json.dumps(out), flush=True)


def synthetic_images(count, side, seed, device):
    """uint8 images: each the sum of 8 Gaussian blobs (seeded centres,
    sigma in [4, 32] px, amplitudes in [40, 120]) plus U[0, 16) noise, clamped;
    returned as FP32 rows (count x side^2) scaled by 1/255."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    yy, xx = torch.meshgrid(torch.arange(side, device=device, dtype=torch.float32),
                            torch.arange(side, device=device, dtype=torch.float32), indexing="ij")
    X = torch.empty(count, side * side, dtype=torch.float32, device=device)
    chunk = 256
    for c0 in range(0, count, chunk):
        c1 = min(count, c0 + chunk)
        nimg = c1 - c0
        img = torch.rand(nimg, side, side, generator=g, device=device) * 16.0
        cx = torch.rand(nimg, 8, 1, 1, generator=g, device=device) * side
        cy = torch.rand(nimg, 8, 1, 1, generator=g, device=device) * side
        sg = 4.0 + torch.rand(nimg, 8, 1, 1, generator=g, device=device) * 28.0
        amp = 40.0 + torch.rand(nimg, 8, 1, 1, generator=g, device=device) * 80.0
        for b in range(8):
            d2 = (xx - cx[:, b]) ** 2 + (yy - cy[:, b]) ** 2
            img += amp[:, b] * torch.exp(-d2 / (2.0 * sg[:, b] ** 2))
        X[c0:c1] = img.clamp_(0, 255).floor_().reshape(nimg, -1) / 255.0
    return X


def run_gram(args, world, rank, local):
    """Gram operator from synthetic images (4096 x 65536 px): A = X X^T by the
    split-BF16 tensor-core kernel, then the top-32 eigenpairs with hdim 96."""
    import torch
    import oap_b200 as B
    torch.cuda.set_device(local)
    count, side = 4096, 256
    if args.quick:
        # profiling run: the build alone on 4096 images of side x side pixels
        side = args.gram_side
        X = synthetic_images(count, side, 21 + rank, "cuda")
        for _ in range(args.warmup):
            B.gram_build(X)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            B.gram_build(X)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        flops = 2.0 * count * count * side * side
        if rank == 0:
            print(json.dumps({"quick": True, "config": "gram build", "images": count, "pixels": side * side,
                              "build_ms": ms, "tflops_algorithmic": flops / ms / 1e9}), flush=True)
        return
    X = synthetic_images(count, side, 21 + rank, "cuda")
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        A, A64 = B.gram_build(X, fp64=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        A, A64 = B.gram_build(X, fp64=True)
    e1.record()
    torch.cuda.synchronize()
    gram_s = e0.elapsed_time(e1) / 1e3 / args.steps
    flops = 2.0 * count * count * side * side
    # build error vs FP64 on a sample of rows
    idx = torch.arange(0, count, 64, device="cuda")
    Xd = X.double()
    ref = Xd[idx] @ Xd.T
    rel = ((A64[idx] - ref).abs() / ref.abs().clamp_min(1e-300)).max().item()
    res, evs = {}, {}
    for name, prec in (("mixed", B.PREC_MIXED), ("plain_fp64", B.PREC_FP64)):
        s = B.Arnoldi(count, 96, 32, precision=prec, tolerance=TOL, seed=5, profile=True)
        s.set_operator(A64)
        s.solve(allow_not_converged=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev, r, st = s.solve(allow_not_converged=True)
        torch.cuda.synchronize()
        res[name] = {"seconds": time.perf_counter() - t0, "status": st, "max_residual": max(r),
                     "stats": {k: v for k, v in s.stats().items() if k in ("restarts", "matvecs", "block_matvecs",
                                                                           "refine_iterations")},
                     "top3": [e.real for e in ev[:3]]}
        evs[name] = ev
        s.close()
    # the implicit operator: A v = X (X^T v), A never formed (two passes over X)
    s = B.Arnoldi(count, 96, 32, tolerance=TOL, seed=5)
    s.set_gram_operator(X)
    s.solve(allow_not_converged=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ev, r, st = s.solve(allow_not_converged=True)
    torch.cuda.synchronize()
    res["implicit_fp64"] = {"seconds": time.perf_counter() - t0, "status": st, "max_residual": max(r),
                            "stats": {k: v for k, v in s.stats().items() if k in ("restarts", "matvecs")},
                            "top3": [e.real for e in ev[:3]],
                            "x_bytes_per_matvec": 2 * 4 * count * side * side}
    s.close()
    # eigenvalue errors: the split-BF16 built operator's 32 values against the
    # exact Gram of the FP32 images (implicit operator), and the chosen form
    # against the plain FP64 solve of the same built operator
    import oracle as O
    lm = lambda e: sorted(e, key=lambda z: -abs(z))
    res["eig_err_built_vs_exact_gram"] = O.match_eigenvalues(lm(evs["plain_fp64"]), lm(ev))
    res["eig_err_mixed_vs_plain_fp64"] = O.match_eigenvalues(lm(evs["mixed"]), lm(evs["plain_fp64"]))
    peak = 1642.4
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"]
    except (OSError, KeyError, ValueError):
        pass
    out = {"config": {"workload": "Gram of 4096 synthetic 256x256 images (8 Gaussian blobs + U[0,16) noise), "
                                  "top-32, hdim 96"},
           "gram": {"ms": gram_s * 1e3, "tflops_algorithmic": flops / gram_s / 1e12, "peak_bf16_tflops": peak,
                    "frac": flops / gram_s / 1e12 / peak, "rel_error_vs_fp64_max": rel,
                    "note": "2 N^2 P flops counted once (the split runs three BF16 products)"},
           "solve": res}
    if rank == 0:
        print(json.dumps(out), flush=True)


def warmstart_family(fam, n, k, hdim, n_train, n_test, seed, epochs=40):
    """Train the network on plain-method solves of A(theta) and compare
    held-out solves from its prediction with the random start."""
    import numpy as np
    import torch
    import oap_b200 as B
    from oap_b200 import warmstart as W
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    th_train = torch.rand(n_train, 16, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    th_test = torch.rand(n_test, 16, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    t0 = time.perf_counter()
    T, evs, st = W.make_targets(fam, th_train, wanted=k, nshift=8, chunk=256)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    net = W.Net([16, 256, 256, n + 8], seed=1)
    ok = st == B.OK  # targets from the plain method's converged solves only
    keep = torch.from_numpy(np.nonzero(ok)[0]).cuda()
    t0 = time.perf_counter()
    losses = net.train(th_train[keep].float().contiguous(), torch.from_numpy(T[ok]).cuda(), epochs=epochs, batch=256,
                       lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    ops = fam.operators(th_test)
    res = {"warm": {"matvecs": 0, "restarts": 0, "seconds": 0.0, "fallbacks": 0, "converged": 0},
           "random": {"matvecs": 0, "restarts": 0, "seconds": 0.0, "converged": 0}}
    eps = []
    # one handle per method, created before the timing (the settings of
    # warmstart.solve_from_prediction / solve_random): a held-out solve is timed
    # from the network's forward pass (warm) or from the solve call (random) to
    # its result, without a handle's creation
    warm_h = B.Arnoldi(n, hdim, k, sort="LR", tolerance=TOL, max_restarts=300, seed=7, init=B.INIT_USER,
                       fallback_random=True)
    rand_h = B.Arnoldi(n, hdim, k, sort="LR", tolerance=TOL, max_restarts=300, seed=7)
    for i in range(th_test.shape[0]):
        A = ops[i].contiguous()
        warm_h.set_operator(A)
        rand_h.set_operator(A)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        pred = net.forward(th_test[i:i + 1].float().contiguous())[0]
        warm_h.set_start_vector(pred[:n].double().contiguous())
        ev, r, stw = warm_h.solve(allow_not_converged=True)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        ev, r2, str_ = rand_h.solve(allow_not_converged=True)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        s_w, s_r = warm_h.stats(), rand_h.stats()
        _, _, _, _, X = W.solve_random(A, n, wanted=k, hdim=hdim, vectors=True)
        eps.append(W.start_error(pred[:n], X))
        for key, s_, st_, rr, dt in (("warm", s_w, stw, r, t2 - t1), ("random", s_r, str_, r2, t3 - t2)):
            res[key]["matvecs"] += s_["matvecs"]
            res[key]["restarts"] += s_["restarts"]
            res[key]["seconds"] += dt
            res[key]["converged"] += int(st_ == B.OK and max(rr) <= TOL)
        res["warm"]["fallbacks"] += s_w["fallbacks"]
    warm_h.close()
    rand_h.close()
    m = th_test.shape[0]
    for key in res:
        for f in ("matvecs", "restarts", "seconds"):
            res[key][f + "_per_solve"] = res[key][f] / m
    return {"training": {"solves": n_train, "data_seconds": t_data, "train_seconds": t_train,
                         "loss_first": losses[0], "loss_last": losses[-1],
                         "plain_solves_converged": int((st == B.OK).sum())},
            "held_out": res, "prediction_eps_median": float(np.median(eps)),
            "speedup_time": res["random"]["seconds"] / res["warm"]["seconds"] if res["warm"]["seconds"] else None,
            "matvec_ratio": res["random"]["matvecs"] / max(1, res["warm"]["matvecs"])}


def run_warmstart(args, world, rank, local):
    """Learned warm start on A(theta) = A0 + sum_i theta_i B_i (n = 2048 real
    symmetric, 16 parameters, top-8): training targets from plain FP64 IRAM
    solves (batched), network 16 -> 256 -> 256 -> 2048 + 8 trained on the
    GPU, then held-out solves from the prediction vs from a random start;
    then the same with the B_i scaled by 0.01, where the wanted subspace is a
    smooth function of theta."""
    import torch
    from oap_b200 import warmstart as W
    torch.cuda.set_device(local)
    n, k, hdim = 2048, 8, 24
    fam = W.ParamFamily(n=n, nparams=16, seed=31 + rank)
    spec = warmstart_family(fam, n, k, hdim, args.train, args.held_out, 77 + rank)
    del fam
    fam = W.ParamFamily(n=n, nparams=16, seed=31 + rank, scale=0.01)
    smooth = warmstart_family(fam, n, k, hdim, args.train_smooth, args.held_out, 78 + rank)
    out = {"config": {"workload": "A(theta) = A0 + sum theta_i B_i, n=2048 real symmetric, 16 params, top-8 LR, "
                                  "hdim 24; network 16-256-256-2056 BF16",
                      "training_solves": args.train, "held_out": args.held_out},
           "specified_family": spec,
           "smooth_family_scale_0.01": smooth}
    if rank == 0:
        print(json.dumps(out), flush=True)


def main():
    args = parse()
    world, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.config == "batched":
            run_batched(args, world, rank, local)
        elif args.config == "gram":
            run_gram(args, world, rank, local)
        elif args.config == "warmstart":
            run_warmstart(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
