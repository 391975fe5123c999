#!/usr/bin/env python
"""Benchmark: SF-CIS + SF-CPS(D-3) roots per second on B200.

One step = the whole pipeline of the workload: SF-CIS Davidson (residual
1e-8) for every requested root, ground CPS(D) T^(1)/T^(2), the J^(2)/J^(3)
intermediates and EE-CPS(D-3) orders 1-3 for every root, with the integrals
resident in HBM.  Default workload: the large run, D2h, nmo 400, nocc
20/18, 10 spin-flip roots (93.5 GB of synthetic seeded integrals built on
the device, see synth.py); --config d2h_nmo200 gives the precision-form
workload (D2h, nmo 200, nocc 10/8, 5 roots).  The headline value is the
mixed mode (contractions of at least 1 GFLOP on the int8 tensor cores with
--digits 7-bit digits per FP64 value, exact integer sums, FP64 everywhere
else; 6 digits on d2h_nmo400, 5 elsewhere unless given); the plain FP64
path is timed beside it (fp64_path), every root's deviation from it is
reported, and the line fails its gate (gate.pass = false, exit status 3)
when any excitation energy, w^(2) or w^(3) is more than 1 micro-Eh away.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--digits D]
  python bench.py --impl reference ...   (CPU restatement on the host cores)

Multi-GPU: one process per GPU (torchrun); every rank runs an independent
replica of the workload (replicas only: the path has no exchange step);
value = roots of all ranks / max-over-ranks device time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
METRIC = "SF-CPS(D) roots/sec: mixed+batched vs FP64 GPU at ≤1 µEh; contraction TFLOP/s"
# digits per workload that keep every energy within the 1 micro-Eh gate:
# the synthetic nmo-400 system has |w^(3)| up to 1.5e3 Eh, where 5 digits
# leave 1.6e-5 Eh and 6 digits 1.6e-7 Eh
DEFAULT_DIGITS = {"d2h_nmo400": 6}
GATE_EH = 1e-6
# integrals above this size are built on the device (the host build is too
# slow) and the CPU baseline gets them by a copy from there
DEVICE_BUILD_BYTES = 16e9


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="d2h_nmo400")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-threads", type=int, default=0)
    ap.add_argument("--digits", type=int, default=-1,
                    help="7-bit digits per FP64 value on the int8 tensor cores (0 = FP64 path only; "
                         "default 6 on d2h_nmo400, 5 elsewhere)")
    ap.add_argument("--cpu-samples", type=int, default=1,
                    help="samples of the CPU baseline (one root's chain each) after one warm-up pass")
    ap.add_argument("--cpu-worker", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-fp64-path", action="store_true", help="skip timing the plain FP64 path beside the headline")
    ap.add_argument("--no-phase-overlap", action="store_true",
                    help="run the pipeline's phases one after the other (SF-CIS is otherwise beside the ground state)")
    ap.add_argument("--case-nmo", type=int, default=100)
    ap.add_argument("--directions", type=int, default=200, help="finite-difference directions of --case grad")
    ap.add_argument("--workers", type=int, default=8, help="concurrent molecules of --case batch")
    ap.add_argument("--wave-gb", type=float, default=140.0, help="device-memory budget of one --case batch wave")
    ap.add_argument("--kernel", default="c1_r2abci", choices=sorted(KERNEL_CASES),
                    help="lib_cc kernel of --case kernel")
    ap.add_argument("--case", default="", choices=["", "ladder", "grad", "grad3", "batch", "kernel"],
                    help="time one contraction on its own (kernel profiling) instead of the pipeline")
    a = ap.parse_args()
    if a.digits < 0:
        a.digits = DEFAULT_DIGITS.get(a.config, 5)
    return a


def workload_desc(s, name):
    return (f"{name}: SF-CIS (spin-flip a->b, Davidson residual 1e-8) + ground CPS(D) + J2/J3 + "
            f"EE-CPS(D-3) orders 1-3; {['C1','Cs','','C2v','','','','D2h'][s.nirrep-1] or s.nirrep} "
            f"nirrep={s.nirrep}, nmo={s.nmo}, nocc {s.nocc_a}/{s.nocc_b}, o={int(s.popo.sum())}, "
            f"v={int(s.popv.sum())}, roots={s.nroots}, FP64")


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        busy = [x for x in sm if smax and x > 0.5 * smax] or sm
        return {"sm_mhz": float(np.median(busy)) if busy else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def hbm_peak_gbs():
    """measured HBM copy bandwidth of this pool (MEASURED_PEAKS.json), else
    the pool's earlier measurement of 6650 GB/s"""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def measured_fp64_peak(torch):
    """cuBLAS DGEMM throughput on this GPU (TFLOP/s), the FP64 roofline."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def is_big(name):
    """integrals too large for the host build: built on the device"""
    from cpsd_b200 import synth
    return synth.config_integral_bytes(name) > DEVICE_BUILD_BYTES


def big_workload(name):
    """(built on the device?, synth.System; host integrals only when not)"""
    from cpsd_b200 import synth
    big = is_big(name)
    return big, synth.make(name, host_ints=not big)


def cpu_worker(args):
    """The CPU restatement (oracle) on a bounded sample of the workload, in
    a process of its own (both arms run this same function the same way):
    one warm-up pass (the c2v_nmo48 pipeline: thread pool, BLAS, first
    touch), then --cpu-samples samples of one root's whole chain (CIS
    Davidson for that root, ground CPS(D), J2/J3, EE orders 1-3), each
    stage timed; the workload's roots/s is extrapolated from the mean stage
    times as nroot / (T_cis nroot + T_ground + T_J + T_root nroot).  Large
    workloads' integrals are built on the GPU and copied to host memory
    before anything is timed (input generation only: the timed work is the
    oracle on the host cores).  Prints one JSON line."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import conftest  # noqa: F401  (registers the package)
    import oracle_ffi as of
    from cpsd_b200 import synth
    threads = args.cpu_threads or os.cpu_count() or 1
    t_start = time.time()
    of.Oracle(synth.make("c2v_nmo48"), nthreads=threads).pipeline()
    big, s = big_workload(args.config)
    if big:
        import torch
        d = synth.device_integrals(s)
        for k in api_keys():
            s.ints[k] = d[k].cpu().numpy()
            d[k] = None
        del d
        torch.cuda.empty_cache()
    nroot = s.nroots
    s.estate_sym[:] = 0
    s.estate_sym[0] = 1
    orc = of.Oracle(s, nthreads=threads)
    samples = []
    for _ in range(max(args.cpu_samples, 1)):
        t0 = time.perf_counter()
        om, R, _ = orc.cis()
        t1 = time.perf_counter()
        g = orc.ground()
        t2 = time.perf_counter()
        J = orc.jints(g)
        t3 = time.perf_counter()
        orc.root(g, J, 1, om[0], R[:s.r1_len(1)])
        t4 = time.perf_counter()
        samples.append((t1 - t0, t2 - t1, t3 - t2, t4 - t3))
    tc, tg, tj, tr = np.mean(np.array(samples), axis=0)
    v = nroot / (tc * nroot + tg + tj + tr * nroot)
    print(json.dumps({"value": v, "threads": threads, "samples": len(samples), "nroot": nroot,
                      "stage_seconds": dict(t_cis_per_root=tc, t_ground=tg, t_J=tj, t_root=tr),
                      "sample_wall_s": float(np.mean([sum(x) for x in samples])),
                      "worker_wall_s": time.time() - t_start}), flush=True)


def api_keys():
    return ("ijkl", "ijka", "abij", "iabj", "abci", "abcd")


def cpu_baseline(config, threads, samples):
    """CPU baseline by cpu_worker in a fresh process: the same protocol,
    process state and sample count for the GPU arm's cpu_baseline leg and
    the reference arm.  Returns the cpu_baseline object (or None with the
    reason on failure)."""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--cpu-worker", "--config", config,
           "--cpu-threads", str(threads), "--cpu-samples", str(samples)]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=3600, env=env, cwd=ROOT)
    lines = [ln for ln in r.stdout.strip().splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        return None, f"cpu worker failed (rc {r.returncode}): {r.stderr.strip()[-300:]}"
    w = json.loads(lines[-1])
    big = is_big(config)
    return {"value": w["value"], "unit": "roots/s", "cores": w["threads"], "cpu_model": cpu_model(),
            "kind": "port",
            "sample": (f"one root's chain (CIS Davidson for it, ground CPS(D), J2/J3, EE orders 1-3) of "
                       f"{config}, {w['samples']} sample(s) after one warm-up pass (c2v_nmo48 pipeline) in a "
                       f"fresh process; stage times extrapolated to the workload's {w['nroot']} roots" +
                       ("; integrals built on the GPU and copied to host memory before timing" if big else "")),
            "stage_seconds": {k: round(x, 4) for k, x in w["stage_seconds"].items()},
            "sample_wall_s": round(w["sample_wall_s"], 2)}, None


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = args.cpu_threads or os.cpu_count() or 1
    t0 = time.time()
    cpu, why = cpu_baseline(args.config, threads, args.cpu_samples)
    if cpu is None:
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return
    v = cpu["value"]
    line = {
        "metric": METRIC, "value": v, "unit": "roots/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * cpu["sample_wall_s"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": args.config, "note": "CPU restatement of the reference's FP64 path "
                   "(the Fortran reference cannot be built: no Fortran compiler here or on the GPU box)"},
        "cpu_baseline": cpu,
        "e2e": {"value": v, "unit": "roots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(time.time() - t0, 1),
    }
    print(json.dumps(line), flush=True)


def measured_int8_peak(torch):
    """cuBLASLt int8 GEMM (torch._int_mm, 8192^3) on this GPU in TOPS, the
    roofline of the int8-digit contraction kernel; None if unavailable."""
    try:
        n = 8192
        a = torch.randint(-127, 128, (n, n), dtype=torch.int8, device="cuda")
        b = torch.randint(-127, 128, (n, n), dtype=torch.int8, device="cuda")
        for _ in range(2):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * n ** 3 / best / 1e12
    except Exception:
        return None


def contraction_records(api):
    """per-launch (ms, flops, kind) of the contraction timing buffer"""
    import ctypes
    lib = api.lib()
    n = 16384
    ms = np.zeros(n)
    fl = np.zeros(n)
    sh = np.zeros(4 * n, np.int64)
    nr = ctypes.c_int64()
    lib.cpsd_contract_records(ms.ctypes.data_as(ctypes.c_void_p), fl.ctypes.data_as(ctypes.c_void_p),
                              sh.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(n), ctypes.byref(nr))
    k = nr.value
    return ms[:k], fl[:k], sh[:4 * k].reshape(k, 4)[:, 3], sh[:4 * k].reshape(k, 4)[:, :3]


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import __graft_entry__ as ge
    ge.load_package()
    from cpsd_b200 import api, synth

    torch.cuda.set_device(local_rank)
    big, s = big_workload(args.config)
    api.init(s.nirrep, s.dirprd)
    api.use_torch_stream()
    api.set_phase_overlap(not args.no_phase_overlap)
    if big:  # built on the device (same values as the host build up to summation order)
        ints = api.DeviceIntegrals.from_tensors(synth.device_integrals(s))
    else:
        ints = api.DeviceIntegrals(s)
    sysc = api.make_system(s)
    par = api.make_params(s, batch_roots=1)
    stream = torch.cuda.current_stream()
    digits = args.digits

    def step():
        return api.pipeline(s, sysc, ints, par)

    step_each = {}  # per-step times of each mode (events between the steps; diagnostics)

    def timed(mode_digits):
        api.set_mixed(mode_digits, 1.0)
        for _ in range(args.warmup):
            out = step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        api.launch_count(True)
        api.flop_count(True)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        ev[0].record(stream)
        for i in range(args.steps):
            out = step()
            ev[i + 1].record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = ev[0].elapsed_time(ev[-1])
        each = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
        launches = api.launch_count(True)
        flops = api.flop_count(True)
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_each[mode_digits] = each
        return float(t.item()), out, launches, flops

    clocks = ClockSampler(local_rank)
    if digits:
        ms_max, out, launches, flops = timed(digits)
        ms64, out64, launches64, flops64 = (ms_max, out, launches, flops) if args.no_fp64_path else timed(0)
    else:
        ms64, out64, launches64, flops64 = timed(0)
        ms_max, out, launches, flops = ms64, out64, launches64, flops64
    ck = clocks.stop()
    err = api.mixed_error() if digits else 0
    value = world * s.nroots * args.steps / (ms_max / 1e3)
    value64 = world * s.nroots * args.steps / (ms64 / 1e3)
    dev_fp64 = max(float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) for a, b in zip(out, out64))
    per_root_dev = np.max(np.abs(np.asarray(out) - np.asarray(out64)), axis=0)  # over (w0, w2, w3)
    gate = {"bound_eh": GATE_EH, "max_abs_dev_eh": dev_fp64, "pass": bool(dev_fp64 <= GATE_EH),
            "against": "the plain FP64 GPU path on the same inputs (itself tested against the oracle: "
                       "1e-9 Eh per root at d2h_nmo200)"}
    om, w2, w3 = out
    step_ms = ms_max / args.steps
    int_gb = ints.nbytes / 1e9

    # per-launch CUDA-event timing of every contraction launch in one extra
    # step of the headline mode: roofline of the digit GEMM (int8 tensor
    # cores) and of the FP64 tensor-pipe kernel
    lib = api.lib()
    api.set_mixed(digits, 1.0)
    lib.cpsd_contract_timing(1)
    lib.cpsd_contract_time(None, None, None, 1)
    step()
    torch.cuda.synchronize()
    rms, rfl, rkind, rshape = contraction_records(api)
    lib.cpsd_contract_time(None, None, None, 1)
    lib.cpsd_contract_timing(0)
    api.set_mixed(0)
    fp64_peak = measured_fp64_peak(torch)
    pairs = digits * (digits + 1) // 2 if digits else 0
    roof = None
    if digits:
        int8_peak = measured_int8_peak(torch)
        sel = rkind == 12
        g_ms, g_fl = float(rms[sel].sum()), float(rfl[sel].sum())
        ach = g_fl * pairs / (g_ms / 1e3) / 1e12 if g_ms > 0 else 0.0
        # per launch the slower of its int8 ops at the measured int8 peak and
        # its digit-tile bytes at the measured HBM bandwidth: launches with
        # few output columns stream their digit tiles once and are HBM-bound
        hbm = hbm_peak_gbs()
        att_ms = 0.0
        for f_, b_ in zip(rfl[sel], rshape[sel][:, 1]):
            t_tensor = f_ * pairs / (int8_peak * 1e12) if int8_peak else 0.0
            t_hbm = float(b_) / (hbm * 1e9) if hbm else 0.0
            att_ms += 1e3 * max(t_tensor, t_hbm)
        # DRAM traffic per launch: the algorithmic bytes (digit tiles once,
        # C read and written per K chunk) times the traffic / algorithmic
        # ratio ncu measured on this kernel (1.05 on the nmo-80 ladder at 6
        # digits, profiles/k_oz_gemm_ladder_nmo80.md); traffic grows with the tiles
        alg = rshape[sel][:, 1].astype(float) + rshape[sel][:, 2].astype(float)
        nsel = max(int(sel.sum()), 1)
        roof = {"bound": "tensor", "kernel": f"k_oz_gemm (tcgen05 kind::i8, {digits} digits, {pairs} digit products)",
                "achieved": ach, "peak": int8_peak, "unit": "TOPS (int8)",
                "frac": ach / int8_peak if int8_peak else None,
                "traffic": 1.05 * float(alg.sum()) / nsel,
                "traffic_note": "bytes per launch: algorithmic bytes (digit tiles + C read/write) x 1.05, the "
                                "dram__bytes_read+write / algorithmic ratio of the ncu capture of this kernel "
                                "(nmo-80 ladder at 6 digits, profiles/k_oz_gemm_ladder_nmo80.md)",
                "algorithmic_bytes_per_launch": float(alg.sum()) / nsel,
                "peak_source": "measured cuBLASLt int8 GEMM 8192^3 (torch._int_mm) on this GPU",
                "fp64_equivalent_tflops": g_fl / (g_ms / 1e3) / 1e12 if g_ms > 0 else 0.0,
                "share_of_step": g_ms / step_ms, "launches_per_step": int(sel.sum()),
                "digit_tile_bytes_per_step": int(rshape[sel][:, 1].sum()),
                "attainable_ms": att_ms, "frac_of_attainable": att_ms / g_ms if g_ms > 0 else None,
                "attainable_note": "per launch max(int8 ops / measured int8 peak, digit-tile bytes / measured "
                                   "HBM copy bandwidth of MEASURED_PEAKS.json)"}
    sel = rkind < 10
    d_ms, d_fl = float(rms[sel].sum()), float(rfl[sel].sum())
    roof64 = {"bound": "tensor", "kernel": "k_contract (FP64 mma.sync m8n8k4 grouped contraction)",
              "achieved": d_fl / (d_ms / 1e3) / 1e12 if d_ms > 0 else 0.0, "peak": fp64_peak, "unit": "TFLOP/s",
              "frac": (d_fl / (d_ms / 1e3) / 1e12) / fp64_peak if d_ms > 0 and fp64_peak else None,
              "traffic": None, "peak_source": "measured cuBLAS DGEMM 8192^3 on this GPU",
              "share_of_step": d_ms / step_ms, "launches_per_step": int(sel.sum())}
    sel = rkind == 22
    s_ms, s_bytes = float(rms[sel].sum()), 16.0 * float(rshape[sel][:, 2].sum())
    hbm = hbm_peak_gbs()
    roof_sk = {"bound": "hbm", "kernel": "k_shortk (short contracted range, output read-modify-write)",
               "achieved": s_bytes / (s_ms / 1e3) / 1e9 if s_ms > 0 else 0.0, "peak": hbm, "unit": "GB/s",
               "frac": (s_bytes / (s_ms / 1e3) / 1e9) / hbm if s_ms > 0 else None,
               "algorithmic_bytes_per_step": s_bytes,
               "bytes_note": "16 B per output element (read + write of C); the operand tiles are not counted",
               "peak_source": "MEASURED_PEAKS.json hbm_gbs (copy bandwidth)",
               "share_of_step": s_ms / step_ms, "launches_per_step": int(sel.sum())}
    shares = {lab: round(float(rms[m].sum()) / step_ms, 4) for lab, m in
              (("digit_gemm", rkind == 12), ("digit_slicing", (rkind == 10) | (rkind == 11)),
               ("fp64_tiles", rkind < 10), ("narrow", (rkind == 20) | (rkind == 21)), ("shortk", rkind == 22),
               ("davidson", (rkind == 30) | (rkind == 31)), ("diis_solver", rkind == 32),
               ("pair_transforms", rkind == 40))}

    # end to end through the public API with host buffers: H2D of every
    # integral tensor from pinned memory, the pipeline, results back on the
    # host (the pipeline returns its energies on the host)
    e2e = None
    if not args.no_e2e:
        import psutil
        nloc = int(os.environ.get("LOCAL_WORLD_SIZE", "1"))
        need = float(ints.nbytes)
        avail = float(psutil.virtual_memory().available)
        if need * nloc > 0.8 * avail:
            e2e = {"value": None, "unit": "roots/s", "skipped": f"pinned host copies of {need / 1e9:.1f} GB per rank "
                   f"x {nloc} ranks exceed the host memory available ({avail / 1e9:.0f} GB)"}
        else:
            api.set_mixed(digits, 1.0)
            host = {}
            for k, t in ints.t.items():
                if t is not None:
                    h = torch.empty(t.numel(), dtype=torch.float64, pin_memory=True)
                    h.copy_(t)
                    host[k] = h
            h2d = sum(v.numel() * 8 for v in host.values())
            d2h = 3 * s.nroots * 8
            e2e_steps = min(args.steps, 5) if big else args.steps
            torch.cuda.synchronize()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            for _ in range(e2e_steps):
                for k, v in host.items():
                    ints.t[k].copy_(v, non_blocking=True)
                step()
            f1.record(stream)
            torch.cuda.synchronize()
            t2 = torch.tensor([f0.elapsed_time(f1)], dtype=torch.float64, device="cuda")
            if world > 1:
                dist.all_reduce(t2, op=dist.ReduceOp.MAX)
            e2e = {"value": world * s.nroots * e2e_steps / (float(t2.item()) / 1e3), "unit": "roots/s",
                   "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                   "note": "every step copies all integral tensors from pinned host memory, runs cpsd_pipeline "
                           "and reads the energies back"}
            api.set_mixed(0)
            del host
            import gc
            gc.collect()
            torch._C._host_emptyCache()  # give the pinned pages back (torch caches them otherwise)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = args.cpu_threads or os.cpu_count() or 1
        if big:  # the worker builds the integrals on the GPU: give the memory back first
            import gc
            del ints
            gc.collect()
            api.release_device_cache()
            torch.cuda.empty_cache()
        cpu, why = cpu_baseline(args.config, threads, args.cpu_samples)
        if cpu is None:
            cpu = {"value": None, "unit": "roots/s", "unavailable": why}
    if rank == 0:
        mode = (f"mixed: contractions >= 1 GFLOP on the int8 tensor cores with {digits} 7-bit digits per FP64 "
                f"value (exact int32 sums, FP64 epilogue); everything else FP64" if digits else "FP64")
        line = {
            "metric": METRIC, "value": value, "unit": "roots/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (int8 digits)" if digits else "f64",
            "data": "synthetic (seeded generator, synth.py)",
            "config": {"workload": workload_desc(s, args.config), "inputs": "resident in HBM, "
                       f"{int_gb:.2f} GB of integrals (larger than L2)" + (", built on the device" if big else ""),
                       "parallelism": f"replicas x{world}", "roots_batched": True, "mode": mode,
                       "phases": "SF-CIS in order with the ground state" if args.no_phase_overlap else
                       "SF-CIS beside the ground state + J2/J3 (two worker streams), then the excited orders"},
            "max_abs_dev_vs_fp64_eh": dev_fp64,
            "per_root_dev_vs_fp64_eh": [float(x) for x in per_root_dev],
            "gate": gate,
            "fp64_path": {"value": value64, "unit": "roots/s", "ms_per_step": ms64 / args.steps,
                          "gpu_launches": launches64, "contraction_tflops": flops64 / (ms64 / 1e3) / 1e12,
                          "ms_each_step": step_each.get(0)},
            "ms_each_step": step_each.get(digits),
            "roofline": roof or roof64,
            "roofline_fp64_tiles": roof64,
            "roofline_shortk": roof_sk,
            "contraction_shares_of_step": shares,
            "contraction_tflops": flops / (ms_max / 1e3) / 1e12,
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": ck,
            "digit_path_timeouts": err,
            "results": {"omega_cis": [float(x) for x in om], "w2": [float(x) for x in w2],
                        "w3": [float(x) for x in w3]},
        }
        print(json.dumps(line), flush=True)
    if not gate["pass"]:
        sys.exit(3)


def run_case(args):
    """One contraction of the pipeline on its own, for kernel profiling:
    'ladder' = the particle-particle ladder V(ab,ef) T(ef,ij) -> C(ab,ij)
    (c2_r2abcd's engine call) on one irrep, nmo 100, nocc 10/8 (v = 182,
    16471 packed pairs: 2.2 GB of integrals), random data; --digits 0 runs
    the FP64 tensor-pipe kernel, otherwise the int8-digit kernels."""
    import torch
    import __graft_entry__ as ge
    ge.load_package()
    from cpsd_b200 import api
    from cpsd_b200.dpd import Symmetry, xor_dirprd
    nmo, na, nb_ = args.case_nmo, 10, 8
    o = np.array([na + nb_, 0, 0, 0, 0, 0, 0, 0])
    v = np.array([2 * nmo - na - nb_, 0, 0, 0, 0, 0, 0, 0])
    sym = Symmetry(1, xor_dirprd(1))
    api.init(1, xor_dirprd(1))
    api.use_torch_stream()
    api.set_mixed(args.digits, 0.0)
    la = sym.idsymsoc(1, v, v, 0, v, v, 0)
    lt = sym.idsymsoc(1, v, v, 0, o, o, 0)
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(la, dtype=torch.float64, device="cuda", generator=g) * 0.05
    T = torch.randn(lt, dtype=torch.float64, device="cuda", generator=g) * 0.01
    C = torch.zeros(lt, dtype=torch.float64, device="cuda")
    d4 = ([v, v, v, v], (0, 0), 1)
    dt = ([v, v, o, o], (0, 0), 1)

    def step():
        api.vv2v_dpd_444(A, d4, "abef", T, dt, "efij", C, dt, "abij", 1.0, 0.0)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    fl = 2.0 * float(np.sqrt(la)) ** 2 * (lt / np.sqrt(la))  # 2 M N K with M = K = pairs
    print(json.dumps({"case": args.case, "digits": args.digits, "ms_per_call": ms, "fp64_equivalent_tflops":
                      fl / (ms / 1e3) / 1e12, "M": int(round(np.sqrt(la))), "N": int(round(lt / np.sqrt(la)))}),
          flush=True)


# --case kernel: lib_cc kernels on the workload's integrals, operand layouts
# as (pop letters, iops): out, amplitude, integral list
KERNEL_CASES = {
    "c1_r2abci": (("vozz", (1, 1)), ("vvoo", (0, 0)), "abci"),   # long-K narrow kernel
    "c2_r1abci": (("vvoo", (0, 0)), ("vozz", (1, 1)), "abci"),   # short-K narrow kernel
    "Wmbej_r1abci": (("vovo", (1, 1)), ("vozz", (1, 1)), "abci"),  # row-dot kernel
    "c1_r1iabj": (("vozz", (1, 1)), ("vozz", (1, 1)), "iabj"),   # CIS sigma
}


def run_kernel_case(args):
    """One lib_cc kernel (--kernel) of the pipeline on its own, on the
    integrals of --config (resident in HBM) and a random amplitude of irrep
    1: --warmup untimed calls, then --steps timed ones (CUDA events).  For
    kernel profiling: the launches are the kernel's own (and, for an integral
    the engine expands, the pair transform of the first call)."""
    import torch
    import __graft_entry__ as ge
    ge.load_package()
    from cpsd_b200 import api, synth
    big, s = big_workload(args.config)
    api.init(s.nirrep, s.dirprd)
    api.use_torch_stream()
    ints = api.DeviceIntegrals.from_tensors(synth.device_integrals(s)) if big else api.DeviceIntegrals(s)
    zorb = np.array([1, 0, 0, 0, 0, 0, 0, 0], np.int64)
    space = {"o": s.popo, "v": s.popv, "z": zorb}
    (lo, io), (la, ia), vname = KERNEL_CASES[args.kernel]
    po, pa = [space[c] for c in lo], [space[c] for c in la]
    g = torch.Generator(device="cuda").manual_seed(0)
    na = s.sym.idsymsoc(1, pa[0], pa[1], ia[0], pa[2], pa[3], ia[1])
    no = s.sym.idsymsoc(1, po[0], po[1], io[0], po[2], po[3], io[1])
    a = torch.randn(na, dtype=torch.float64, device="cuda", generator=g)
    out = torch.zeros(no, dtype=torch.float64, device="cuda")
    V = ints.t[vname]
    vpops = {"abci": ("vvvo", (0, 1)), "iabj": ("vovo", (1, 1))}[vname]
    pv = [space[c] for c in vpops[0]]
    O, A, B = api.opt(po, io, 1, out), api.opt(pa, ia, 1, a), api.opt(pv, vpops[1], 1, V)
    for _ in range(args.warmup):
        api.kernel(args.kernel, O, A, B, 1.0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        api.kernel(args.kernel, O, A, B, 1.0)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    vb = V.numel() * 8
    print(json.dumps({"case": "kernel", "kernel": args.kernel, "config": args.config, "ms_per_call": ms,
                      "integral_bytes": vb, "integral_GBps": vb / (ms / 1e3) / 1e9}), flush=True)


def run_grad(args):
    """Differentiation form: C2v, nmo 120, nocc 8/6, 4 roots of irrep 1.
    Times the SF-CIS(D) energies (cpsd_cisd_energies: Davidson to 1e-12 and
    w^(2)) and one adjoint gradient per root (cpsd_cisd_gradient, FP64),
    then checks every root's gradient against central finite differences of
    the device energies (step 1e-5) along --directions seeded integral-
    perturbation directions (DPD images of moves of the generator's (pq|rs)
    factor and orbital energies)."""
    import torch
    import __graft_entry__ as ge
    ge.load_package()
    from cpsd_b200 import api, synth
    keys = ("ijka", "abij", "iabj", "abci", "eorb")
    s = synth.make("c2v_nmo120", skip_abcd=True)
    symR, nroot = 1, int(s.estate_sym[0])
    api.use_torch_stream()
    t = {k: torch.from_numpy(s.ints[k] if k != "eorb" else s.eorb).cuda() for k in keys}
    par = api.make_params(s, davidson_conv=12, davidson_cyc=100, diis_max_err=1e-12, diis_cyc=200)
    sysc = api.make_system(s)
    st = api.integrals_struct(t)

    def forward(tt=None):
        return api.cisd_energies(s, sysc, api.integrals_struct(tt) if tt else st, par, symR, nroot)

    def backward(w0, L):
        out = []
        for r in range(nroot):
            g = np.zeros(nroot)
            g[r] = 1.0
            G = {k: torch.zeros_like(v) for k, v in t.items()}
            api.cisd_gradient(sysc, st, par, symR, w0, L, g, g, G)
            out.append(G)
        return out

    def timed(fn, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            res = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n, res

    for _ in range(args.warmup):
        w0, w2, L = forward()
        backward(w0, L)
    f_ms, (w0, w2, L) = timed(forward, args.steps)
    b_ms, Gs = timed(lambda: backward(w0, L), args.steps)
    rng = np.random.default_rng(0)
    h = 1e-5
    rel, absn, fds = [], [], []
    t0 = time.time()
    for _ in range(args.directions):
        d = s.integral_direction(*s.input_direction(rng))
        dt = {k: torch.from_numpy(d[k]).cuda() for k in keys}
        E = []
        for sg in (1.0, -1.0):
            a, b, _ = forward({k: t[k] + sg * h * dt[k] for k in keys})
            E.append(a + b)
        fd = (E[0] - E[1]) / (2 * h)
        for r in range(nroot):
            pred = sum(float(torch.dot(Gs[r][k], dt[k])) for k in keys)
            rel.append(abs(pred - fd[r]) / abs(fd[r]))
            absn.append(abs(pred - fd[r]))
            fds.append(abs(fd[r]))
    rel, absn = np.array(rel), np.array(absn)
    print(json.dumps({
        "case": "grad", "workload": "c2v_nmo120", "config": (f"c2v_nmo120: SF-CIS (Davidson residual 1e-12) + w^(2) and d(w0 + w2)/d(ijka, abij, iabj, "
                   f"abci, Eorb) per root; C2v nirrep={s.nirrep}, nmo={s.nmo}, nocc {s.nocc_a}/{s.nocc_b}, "
                   f"o={int(s.popo.sum())}, v={int(s.popv.sum())}"), "roots": nroot,
        "dtype": "f64", "data": "synthetic (seeded generator)",
        "forward_ms": f_ms, "backward_ms_all_roots": b_ms, "backward_ms_per_root": b_ms / nroot,
        "w0": [float(x) for x in w0], "w2": [float(x) for x in w2],
        "fd": {"directions": args.directions, "step": h, "checks": int(rel.size),
               "max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)),
               "max_abs_err": float(absn.max()), "median_abs_derivative": float(np.median(fds)),
               "within_1e-6": int((rel < 1e-6).sum()), "seconds": time.time() - t0},
    }), flush=True)


def run_grad3(args):
    """Differentiation form with the third-order correction: C2v, nmo 120,
    nocc 8/6, 4 roots of irrep 1, the six DPD lists built on the device from
    a dense (pq|rs) (cpsd_eri_lists).  Times cpsd_cpsd3_energies (Davidson to
    1e-12, w^(2), w^(3) with its ground state) and one adjoint gradient per
    root (cpsd_cpsd3_gradient chained to (pq|rs) by cpsd_eri_adjoint), then
    checks every root's d(w0 + w2 + w3)/d(pq|rs) against central finite
    differences of the device energies (step 1e-5) along --directions seeded
    random (pq|rs) directions with the integrals' 8-fold symmetry."""
    import torch
    import __graft_entry__ as ge
    ge.load_package()
    from cpsd_b200 import api, synth
    lists = ("ijkl", "ijka", "abij", "iabj", "abci", "abcd")
    s = synth.make("c2v_nmo120", skip_abcd=True, host_ints=False)
    api.init(s.nirrep, s.dirprd)
    symR, nroot, n = 1, int(s.estate_sym[0]), s.nmo
    api.use_torch_stream()
    Lf = torch.from_numpy(s.L).cuda()
    eri0 = torch.einsum("Ppr,Pqs->prqs", Lf, Lf).contiguous().reshape(-1)
    del Lf
    eorb = torch.from_numpy(s.eorb).cuda()
    mo, sp = api.orbital_map(s)
    lens = s.lengths()
    sysc = api.make_system(s)
    par = api.make_params(s, davidson_conv=12, davidson_cyc=100, diis_max_err=1e-12, diis_cyc=200)

    def lists_of(e):
        out = {k: torch.zeros(lens[k], dtype=torch.float64, device="cuda") for k in lists}
        api.eri_lists(sysc, mo, sp, n, e, out)
        out["eorb"] = eorb
        return out

    t = lists_of(eri0)
    st = api.integrals_struct(t)

    def forward(tt=None):
        return api.cpsd3_energies(s, sysc, api.integrals_struct(tt) if tt else st, par, symR, nroot)

    def backward(w0, L):
        out = []
        for r in range(nroot):
            g = np.zeros(nroot)
            g[r] = 1.0
            G = {k: torch.zeros_like(v) for k, v in t.items()}
            api.cpsd3_gradient(sysc, st, par, symR, w0, L, g, g, g, G)
            out.append(G)
        return out

    def timed(fn, k):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(k):
            res = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k, res

    for _ in range(args.warmup):
        w0, w2, w3, L = forward()
        backward(w0, L)
    f_ms, (w0, w2, w3, L) = timed(forward, args.steps)
    b_ms, Gs = timed(lambda: backward(w0, L), args.steps)
    geri = []
    for r in range(nroot):
        G = torch.zeros(n ** 4, dtype=torch.float64, device="cuda")
        api.eri_adjoint(sysc, mo, sp, n, {k: Gs[r][k] for k in lists}, G)
        geri.append(G)
    del Gs
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0)
    h = 1e-5
    rel, absn, fds = [], [], []
    t0 = time.time()
    for _ in range(args.directions):
        D = torch.randn((n, n, n, n), generator=gen, dtype=torch.float64, device="cuda")
        D = D + D.permute(1, 0, 2, 3)
        D = D + D.permute(0, 1, 3, 2)
        D = D + D.permute(2, 3, 0, 1)
        D = (D / D.abs().max()).reshape(-1)
        E = []
        for sg in (1.0, -1.0):
            a, b, c, _ = forward(lists_of(eri0 + sg * h * D))
            E.append(a + b + c)
        fd = (E[0] - E[1]) / (2 * h)
        for r in range(nroot):
            pred = float(torch.dot(geri[r], D))
            rel.append(abs(pred - fd[r]) / abs(fd[r]))
            absn.append(abs(pred - fd[r]))
            fds.append(abs(fd[r]))
        del D
    rel, absn = np.array(rel), np.array(absn)
    print(json.dumps({
        "case": "grad3", "workload": "c2v_nmo120", "config": (
            f"c2v_nmo120: SF-CIS (Davidson residual 1e-12) + w^(2) + w^(3) and d(w0 + w2 + w3)/d(pq|rs) per root "
            f"(six DPD lists and Eorb, chained to the dense (pq|rs)); C2v nirrep={s.nirrep}, nmo={s.nmo}, nocc "
            f"{s.nocc_a}/{s.nocc_b}, o={int(s.popo.sum())}, v={int(s.popv.sum())}"), "roots": nroot,
        "dtype": "f64", "data": "synthetic (seeded generator; lists from its dense (pq|rs) on the device)",
        "forward_ms": f_ms, "backward_ms_all_roots": b_ms, "backward_ms_per_root": b_ms / nroot,
        "w0": [float(x) for x in w0], "w2": [float(x) for x in w2], "w3": [float(x) for x in w3],
        "fd": {"directions": args.directions, "direction": "random (pq|rs), 8-fold symmetric, max |D| = 1",
               "step": h, "checks": int(rel.size), "max_rel_err": float(rel.max()),
               "median_rel_err": float(np.median(rel)), "max_abs_err": float(absn.max()),
               "median_abs_derivative": float(np.median(fds)), "within_1e-6": int((rel < 1e-6).sum()),
               "seconds": time.time() - t0},
    }), flush=True)


def run_batch(args):
    """Batching workload: synth.batch_draw() - 64 independent molecules,
    nmo ~ U{60..240}, nocc_alpha ~ U{4..12}, nocc_beta = nocc_alpha - 2,
    nirrep from {1, 2, 4, 8}, 4-8 roots each (392 roots), lowest-root
    Davidson.  Their abcd + abci integrals alone take 846 GB in FP64, more
    than four B200s hold, so the molecules run in waves whose estimated
    footprint (integrals, cached digit tiles, scratch) fits in --wave-gb:
    each wave's integrals are built on the device (synth.device_integrals),
    then the wave runs as one cpsd_pipeline_batch on --workers streams in
    the mixed mode and in plain FP64, each timed with CUDA events with the
    wave's inputs resident.  value = all roots / summed mixed wave times;
    the FP64 figure and the largest energy deviation between the two modes
    are reported beside it."""
    import gc
    import torch
    import __graft_entry__ as ge
    ge.load_package()
    from cpsd_b200 import api, synth
    t_start = time.time()
    draws = synth.batch_draw()
    mols = [synth.System(**d, host_ints=False, run_opts={"lowest": 1}) for d in draws]
    api.use_torch_stream()
    stream = torch.cuda.current_stream()

    def need(s):
        L = s.lengths()
        ints = 8.0 * sum(L.values())
        digits = 0.7 * 8.0 * (L["abcd"] + L["abci"])  # digit tiles of the cached integrals
        scratch = 8.0 * s.nroots * 14 * s.r2_len(1)
        return ints + digits + scratch + 1.5e9

    order = sorted(range(len(mols)), key=lambda i: -need(mols[i]))
    budget = args.wave_gb * 1e9
    waves, cur, tot = [], [], 0.0
    for i in order:
        if cur and tot + need(mols[i]) > budget:
            waves.append(cur)
            cur, tot = [], 0.0
        cur.append(i)
        tot += need(mols[i])
    waves.append(cur)
    res = {0: [None] * len(mols), args.digits: [None] * len(mols)}
    wave_ms = []
    times = {0: 0.0, args.digits: 0.0}
    gen_s, launches = 0.0, {0: 0, args.digits: 0}
    for w in waves:
        g0 = time.time()
        tens = [synth.device_integrals(mols[i]) for i in w]
        torch.cuda.synchronize()
        gen_s += time.time() - g0
        ints = [api.DeviceIntegrals.from_tensors(t) for t in tens]
        pars = [api.make_params(mols[i]) for i in w]
        for mode in (args.digits, 0):
            api.set_mixed(mode, 1.0)
            for _ in range(args.warmup):
                api.pipeline_batch([mols[i] for i in w], ints, pars, nworkers=args.workers)
            torch.cuda.synchronize()
            api.launch_count(True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                out = api.pipeline_batch([mols[i] for i in w], ints, pars, nworkers=args.workers)
            e1.record(stream)
            torch.cuda.synchronize()
            times[mode] += e0.elapsed_time(e1) / args.steps / 1e3
            wave_ms.append(round(e0.elapsed_time(e1) / args.steps, 1))
            launches[mode] += api.launch_count(True) // max(args.steps, 1)
            for i, o in zip(w, out):
                res[mode][i] = o
        api.set_mixed(0)
        del ints, tens, out
        gc.collect()
        torch.cuda.empty_cache()
        api.release_device_cache()
    nroots = sum(s.nroots for s in mols)
    per = []
    for i, s in enumerate(mols):
        d = [float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) for a, b in zip(res[args.digits][i], res[0][i])]
        mag = [float(np.max(np.abs(np.asarray(b)))) for b in res[0][i]]
        per.append({"molecule": i, "nmo": s.nmo, "nirrep": s.nirrep, "nocc_a": s.nocc_a, "roots": s.nroots,
                    "dev_omega_w2_w3": d, "max_abs_omega_w2_w3": mag})
    dev = max(max(p["dev_omega_w2_w3"]) for p in per)
    rel = max(max(x / max(m, 1e-30) for x, m in zip(p["dev_omega_w2_w3"], p["max_abs_omega_w2_w3"])) for p in per)
    worst = sorted(per, key=lambda p: -max(p["dev_omega_w2_w3"]))[:5]
    print(json.dumps({
        "case": "batch", "metric": METRIC, "unit": "roots/s", "dtype": "f64 (int8 digits)",
        "data": "synthetic (seeded generator, synth.batch_draw)",
        "config": {"workload": "batching form: 64 independent molecules, nmo ~U{60..240}, nocc_a ~U{4..12}, "
                               "nocc_b = nocc_a - 2, nirrep from {1,2,4,8}, 4-8 roots each (lowest roots)",
                   "molecules": len(mols), "roots": nroots, "waves": [len(w) for w in waves],
                   "wave_budget_gb": args.wave_gb, "workers": args.workers,
                   "abcd_abci_fp64_gb": round(sum(8.0 * (s.lengths()["abcd"] + s.lengths()["abci"])
                                                  for s in mols) / 1e9, 1),
                   "mode": f"mixed: contractions >= 1 GFLOP on the int8 tensor cores with {args.digits} digits"},
        "value": nroots / times[args.digits], "ms_total": 1e3 * times[args.digits],
        "fp64_path": {"value": nroots / times[0], "ms_total": 1e3 * times[0], "gpu_launches": launches[0]},
        "mixed_over_fp64": times[0] / times[args.digits],
        "max_abs_dev_vs_fp64_eh": dev, "max_rel_dev_vs_fp64": rel, "worst_molecules": worst,
        "gpu_launches": launches[args.digits],
        "wave_ms_mixed_fp64": [wave_ms[k:k + 2] for k in range(0, len(wave_ms), 2)],
        "steps": args.steps, "warmup": args.warmup, "device_generation_s": gen_s,
        "wall_s": time.time() - t_start,
        "roots_per_molecule": [[float(x) for x in res[args.digits][i][0]] for i in range(len(mols))][:3],
    }), flush=True)


def main():
    args = parse()
    if args.cpu_worker:
        import __graft_entry__ as ge
        ge.load_package()
        cpu_worker(args)
        return
    if args.case == "grad":
        run_grad(args)
    elif args.case == "grad3":
        run_grad3(args)
        return
    if args.case == "batch":
        run_batch(args)
        return
    if args.case == "kernel":
        run_kernel_case(args)
        return
    if args.case:
        run_case(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if world > 1 and rank != 0:
            return
        import __graft_entry__ as ge
        ge.load_package()
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
