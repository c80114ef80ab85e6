"""Benchmark: the CV-to-DV state-transfer circuit at 2^28 amplitudes.

Workload (one step): the 42 gates of the 14-round state-transfer circuit
(H, conditional displacement, Rz per round) on a resident 2^28-amplitude state
([1]*14 + [14] registers), complex128 (the reference's arithmetic).  The state
(4 GiB) is 32x the 126 MB L2, so no L2 flush is needed between steps.

  value      gates/s on the device-resident state (CUDA events on the library's
             stream, max over ranks), whole job
  e2e        gates/s through the public API with host buffers: separable
             register arrays from pinned host memory -> initStateVector ->
             state preparation -> 42 gates -> the 14 qubit marginals to the host
  roofline   the dominant kernel (the FFT pass) from per-launch CUDA events
             taken inside the timed region, against the measured HBM peak
  cpu_baseline  the CPU oracle (numpy/scipy restatement of the reference's
             decompositions) on a bounded sample, rank 0 at N=1 only

--impl reference times the CPU oracle (the reference's own implementation is
Python that cannot be shipped here; its CUDA library needs cuTENSOR) on the
same workload, one gate per step.

Multi-GPU: replicas only (the path does not shard); every rank runs its own
copy of the circuit and value sums the ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cuda-cvdv_b200"))
sys.path.insert(0, ROOT)

METRIC = "gates/s (CV-to-DV state transfer, 2^28 amplitudes)"
UNIT = "gates/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """SM clock and clock-event reasons sampled DURING the timed region: NVML read
    every 5 ms from a background thread and every 2 ms from the timing loop while it
    waits for the timed steps (the region lasts tens of milliseconds, too short for
    nvidia-smi's sampling); nvidia-smi at 200 ms if NVML is missing.  Read-only
    queries: no clock or power setting is touched."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.p = None
        self.thread = None
        self.samples = []
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(gpu)
        except Exception:
            self.nvml = None

    def sample(self):
        """One NVML reading (also called from the timing loop while the GPU works)."""
        nv = self.nvml
        if nv is None:
            return
        try:
            sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
            smax = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            get = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self.samples.append((sm, smax, int(get(self.h))))
        except Exception:
            pass

    def _poll(self):
        while not self.done:
            self.sample()
            time.sleep(0.005)

    def start(self):
        if self.nvml is not None:
            import threading
            self.done = False
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.thread is not None:
            self.done = True
            self.thread.join(timeout=5)
            sm = [x[0] for x in self.samples]
            reasons = sorted(k for k, bit in self.REASONS.items() if any(x[2] & bit for x in self.samples))
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": max(x[1] for x in self.samples) if sm else None,
                    "reasons": reasons, "samples": len(sm), "source": "nvml, 2-5 ms"}
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


_BACKEND = "nccl"


def dist_init():
    """One process per GPU under torchrun (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_*).
    NCCL on GPU boxes; gloo where CUDA is absent (the CPU tests of the multi-rank path)."""
    global _BACKEND
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        _BACKEND = os.environ.get("CVDV_DIST_BACKEND", "nccl" if torch.cuda.is_available() else "gloo")
        dist.init_process_group(_BACKEND, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if _BACKEND == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- CPU oracle
def oracle_mode_state(circ):
    """Mode register after the preparation gates, computed on the mode alone
    (the initial state is a product, so the prepared state is too)."""
    from oracle.cvdv_oracle import OracleSim
    from cvdv_b200 import workloads as W
    q = circ["qubits"][-1]
    m = OracleSim([q])
    sep = W.separable_arrays(circ)
    m.init_from_separable([sep.register_arrays[-1].numpy()])
    mode = len(circ["qubits"]) - 1
    for meth, args in circ["prep"]:
        if args[0] == mode:
            getattr(m, meth)(0, *args[1:])
    return sep, m.get_state()


def cpu_oracle_gates(circ, gate_indices, threads):
    """Time the oracle on the full-size state for the listed gates; returns
    (seconds per gate list, gates timed)."""
    import numpy as np
    from oracle.cvdv_oracle import OracleSim
    sep, mode = oracle_mode_state(circ)
    o = OracleSim(circ["qubits"], workers=threads)
    arrays = [a.numpy() for a in sep.register_arrays[:-1]] + [mode]
    o.init_from_separable(arrays)
    times = []
    for gi in gate_indices:
        meth, args = circ["gates"][gi % len(circ["gates"])]
        t0 = time.perf_counter()
        getattr(o, meth)(*args)
        times.append(time.perf_counter() - t0)
    del o
    np.zeros(1)
    return times


def run_reference(args, world, rank):
    if rank != 0:
        return
    from cvdv_b200 import workloads as W
    threads = os.cpu_count() or 1
    circ = W.state_transfer() if args.workload == "full" else W.state_transfer(n_qubits=10)
    # one gate per step, cycling through the circuit; warm-up gates are untimed
    nq = len(circ["qubits"]) - 1
    n_tot = sum(circ["qubits"])
    n = args.warmup + args.steps
    times = cpu_oracle_gates(circ, list(range(n)), threads)
    timed = times[args.warmup:]
    sec = sum(timed)
    value = len(timed) / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sec / len(timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded circuit, seed 2)",
        "config": {"workload": f"state_transfer [1]*{nq}+[14], 2^{n_tot} amplitudes, complex128",
                   "step": "one gate of the circuit (cycling), CPU oracle"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{len(timed)} gates of the {len(circ['gates'])}-gate circuit at 2^{n_tot} "
                                   f"(numpy elementwise slabs and scipy FFT on {threads} threads)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
def run_gpu(args, world, rank, local):
    import numpy as np
    import torch
    from cvdv_b200 import CudaCvdv, _lib
    from cvdv_b200 import workloads as W

    torch.cuda.set_device(local)
    L = _lib.load()
    # "small" (10 qubit registers, 2^24 amplitudes) exists for profiler captures
    circ = W.state_transfer() if args.workload == "full" else W.state_transfer(n_qubits=10)
    G = len(circ["gates"])
    hbm, peak_kind = peaks()
    out = {}

    def timed_run(precision, fusion=True, keep=False):
        sim = CudaCvdv(circ["qubits"], precision=precision, check_errors=True, fusion=fusion)
        sim.initStateVector(W.separable_arrays(circ, device="cuda"))
        W.apply(sim, circ["prep"])
        sim.synchronize()
        stream = torch.cuda.ExternalStream(L.cvdvGetStream(sim.ctx))
        for _ in range(args.warmup):
            W.apply(sim, circ["gates"])
            L.cvdvFlush(sim.ctx)
        sim.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        L.cvdvSetTiming(sim.ctx, 1)
        _lib.kernel_stats(sim.ctx)  # reset
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        n0 = L.cvdvLaunchCount()
        clk = Clocks(local)
        clk.start()
        e0.record(stream)
        for _ in range(args.steps):
            W.apply(sim, circ["gates"])
            L.cvdvFlush(sim.ctx)
        e1.record(stream)
        while not e1.query():  # read the clocks while the timed steps run on the GPU
            clk.sample()
            time.sleep(0.002)
        e1.synchronize()
        clocks = clk.stop()
        launches = L.cvdvLaunchCount() - n0
        ms = e0.elapsed_time(e1) / args.steps
        stats = _lib.kernel_stats(sim.ctx)
        L.cvdvSetTiming(sim.ctx, 0)
        torch.cuda.synchronize()
        barrier(world)
        ms = max_over_ranks(ms, world)
        norm = sim.m()
        if keep:
            return ms, stats, launches, clocks, norm, sim
        del sim
        torch.cuda.empty_cache()
        return ms, stats, launches, clocks, norm

    ms, stats, launches, clocks, norm, sim128 = timed_run("complex128", keep=True)
    n_amp = 1 << sum(circ["qubits"])
    total_kernel_ms = sum(v[0] for v in stats.values())
    # Every kernel of this workload is one read + write of the state: the
    # algorithmic bytes of a launch are 2 * 2^n * 16 B (complex128).
    alg_bytes = 2 * n_amp * 16
    KNAME = {"seq": "k_seq (qubit-gate sequence: H, conditional phase in p and Rz on up to five qubits per pass)",
             "pair": "k_pair (one qubit gate with the neighbouring diagonal runs)",
             "fft_pass": "k_rowq (row program: mode DFT + diagonal runs; 2^14-point rows on an 8-CTA cluster of "
                         "128-thread CTAs)"}

    def kern_roof(st, nbytes):
        out = {}
        for k in ("seq", "pair", "fft_pass"):
            t, n = st[k]
            if n:
                per = t / n
                out[k] = {"kernel": KNAME[k], "launches": n, "avg_launch_ms": per,
                          "achieved_gbs": nbytes / (per * 1e-3) / 1e9,
                          "share_of_kernel_time": t / max(sum(v[0] for v in st.values()), 1e-12)}
        return out

    kr = kern_roof(stats, alg_bytes)
    dom = max(kr, key=lambda k: kr[k]["share_of_kernel_time"])
    # DRAM bytes (read + write) per launch from ncu captures of the same kernels on the
    # 2^24-amplitude version of this workload (profiles/*_state_transfer_2p24.md),
    # scaled by the 16x larger state: the kernels stream the state once per launch,
    # so their traffic grows with the rows / sites processed.
    ncu_traffic_2p24 = {"fft_pass": ((268.6 + 218.8) + (268.6 + 218.6)) / 2 * 1e6,  # k_rowq, two launches
                        "seq": (270.4 + 212.4) * 1e6}                                  # k_seq<double2, 5, 1, u32, 0>
    scale = n_amp / float(1 << 24)
    traffic = ncu_traffic_2p24[dom] * scale if (dom in ncu_traffic_2p24 and args.workload == "full") else None
    achieved = kr[dom]["achieved_gbs"]
    value = G * world / (ms * 1e-3)

    # ---- e2e through the public API with host buffers
    sep_host = W.separable_arrays(circ, device="cpu")
    for r in range(len(sep_host.register_arrays)):
        sep_host.register_arrays[r] = sep_host.register_arrays[r].pin_memory()
    h2d = sum(a.numel() * 16 for a in sep_host.register_arrays)
    nq = len(circ["qubits"]) - 1
    d2h = nq * 2 * 8

    def e2e_run(fusion):
        sim = CudaCvdv(circ["qubits"], check_errors=True, fusion=fusion)
        times = []
        for it in range(args.warmup + max(2, min(args.steps, 5))):
            torch.cuda.synchronize()
            barrier(world)
            t0 = time.perf_counter()
            sim.initStateVector(sep_host)
            W.apply(sim, circ["prep"])
            W.apply(sim, circ["gates"])
            sim.mEach(list(range(nq)))
            t1 = time.perf_counter()
            if it >= args.warmup:
                times.append(t1 - t0)
        del sim
        torch.cuda.empty_cache()
        return max_over_ranks(statistics.median(times), world)

    e2e_s = e2e_run(True)
    # the same with the preparation gates run on the full state (product deferral off)
    e2e_nodefer_s = e2e_run(15)

    # ---- every transform executed (queue cancellation off), complex128
    msnf, statsnf, launchesnf, _, normnf = timed_run("complex128", fusion=False)
    krnf = kern_roof(statsnf, alg_bytes)
    # ---- mixed precision (complex64 state) on the same circuit
    ms64, stats64, launches64, clocks64, norm64, sim64 = timed_run("complex64", keep=True)
    kr64 = kern_roof(stats64, alg_bytes // 2)
    # both timed runs applied the circuit W + K times to the same prepared state
    acc_repeated = compare_states(sim128.stateTensor(), sim64.stateTensor())
    acc_repeated["circuits_applied"] = args.warmup + args.steps
    del sim128, sim64
    torch.cuda.empty_cache()
    acc_once = None if args.no_accuracy else state_transfer_accuracy(circ)

    extras = {} if args.no_extras else {"gaussian_network_c3": gaussian_c3(args), "batched_c4": batched_c4(args),
                                         "variational_c5": variational_c5(args), "husimi": husimi_readout(args)}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded circuit, seed 2)",
        "config": {"workload": "state_transfer: registers [1]*14+[14], 2^28 amplitudes, 42 gates "
                               "(14 x H, cd, Rz), complex128 state",
                   "l2": "state 4 GiB > L2 126 MB, no flush needed", "parallelism": f"replicas x{world}"},
        "amplitudes_per_s": value * n_amp,
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": KNAME[dom],
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": peak_kind, "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the 2^24 capture "
                                       "in profiles/, x16 (writes still in L2 at kernel end are not counted)",
                     "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": kr[dom]["avg_launch_ms"],
                     "launches": kr[dom]["launches"], "share_of_kernel_time": kr[dom]["share_of_kernel_time"],
                     "kernels": kr},
        "kernel_ms_per_step": {k: v[0] / args.steps for k, v in stats.items() if v[1]},
        "clocks": clocks,
        "e2e": {"value": G * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "includes": "init from host arrays + 2 prep gates + 42 gates + 14 marginals",
                "not_value_plus_copies": "each e2e step starts from the product state, so product deferral runs the "
                                         "preparation and the first forward transform on the mode's 2^14 array; "
                                         "the timed value loop repeats the circuit on an entangled state (two "
                                         "full-state row programs per step). value_product_deferral_off is the "
                                         "like-for-like end-to-end figure",
                "product_deferral": "gates queued after the separable init that act on the mode alone (the "
                                    "preparation and the first transform) run on the mode's 2^14 array before "
                                    "the product state is formed; the first qubit-gate sequence pass then forms "
                                    "each amplitude from the product tables instead of reading a written product",
                "value_product_deferral_off": G * world / e2e_nodefer_s},
        "norm_after": norm,
        "queue_fusion": "FtP2Q/FtQ2P pairs separated only by gates on other registers are cancelled "
                        "(exact identity) and chains of qubit gates on up to five qubits run as one pass; "
                        "every_transform_executed is the run with both off (one pass per gate)",
        "every_transform_executed": {"value": G * world / (msnf * 1e-3), "ms_per_step": msnf,
                                     "gpu_launches": int(launchesnf), "kernels": krnf, "norm_after": normnf},
        "mixed_c64": {"value": G * world / (ms64 * 1e-3), "ms_per_step": ms64, "gpu_launches": int(launches64),
                      "kernels": kr64, "norm_after": norm64, "speedup_vs_plain": ms / ms64,
                      "accuracy": {"against": "the complex128 path on the GPU (equal to the FP64 oracle within 1e-10 "
                                              "relative in the parity tests), same circuit and input",
                                   "one_circuit": acc_once, "after_timed_runs": acc_repeated,
                                   "target_infidelity": 1e-6}},
    }
    line.update(extras)
    if world == 1 and rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        n_cpu = 30 if args.workload == "full" else 42
        times = cpu_oracle_gates(circ, list(range(n_cpu)), threads)
        line["cpu_baseline"] = {"value": n_cpu / sum(times), "unit": UNIT, "cores": threads, "kind": "port",
                                "seconds": sum(times),
                                "sample": f"the first {n_cpu} gates ({n_cpu // 3} (H, cd, Rz) rounds) of the circuit at "
                                          "full size on the CPU oracle (numpy elementwise slabs and scipy FFT on all "
                                          "host threads)"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def compare_states(a, b):
    from cvdv_b200.accuracy import compare_states as cs
    return cs(a, b)


def state_transfer_accuracy(circ):
    """The circuit applied once to the prepared state in complex64 and in complex128."""
    import torch
    from cvdv_b200 import CudaCvdv
    from cvdv_b200 import workloads as W
    sims = {}
    for prec in ("complex128", "complex64"):
        sim = CudaCvdv(circ["qubits"], precision=prec, check_errors=True)
        sim.initStateVector(W.separable_arrays(circ, device="cuda"))
        W.apply(sim, circ["prep"])
        W.apply(sim, circ["gates"])
        sim.synchronize()
        sims[prec] = sim
    out = compare_states(sims["complex128"].stateTensor(), sims["complex64"].stateTensor())
    out["qubit_marginal_max_abs_err"] = max(
        float(abs(a - b).max()) for a, b in zip(sims["complex128"].mEach(list(range(len(circ["qubits"]) - 1))),
                                                 sims["complex64"].mEach(list(range(len(circ["qubits"]) - 1)))))
    del sims
    torch.cuda.empty_cache()
    return out


def batched_c4(args):
    """512 independent uneven circuits (1-3 qubits + a 2^8..2^14 mode, 50 gates each,
    complex64): one persistent launch per gate stage, replayed as a CUDA graph, against a
    per-instance loop through CudaCvdv on the first 32 instances."""
    import torch
    from cvdv_b200 import CudaCvdv
    from cvdv_b200 import workloads as W
    from cvdv_b200.batch import BatchedCircuits, random_instances
    insts = random_instances(seed=4, count=512, gates=50)
    B = BatchedCircuits(insts, precision="complex64")
    # the default shapes, then the autotuned ones (grid, pair chunk, row-task shape per mode length)
    psi_tmp = [W.product_state(i["qubits"], i["init"]) for i in insts]
    B.set_initial(psi_tmp)
    ms_default = B._time(3)
    grid, chunk = B.autotune(reps=2)
    psi0 = [W.product_state(i["qubits"], i["init"]) for i in insts]
    B.set_initial(psi0)
    B.run(graph=True)  # one run + capture
    reps = max(args.steps, 3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        B.run(graph=True)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    loop_n = 32
    sims = []
    for inst, p0 in zip(insts[:loop_n], psi0[:loop_n]):
        sim = CudaCvdv(inst["qubits"], precision="complex64")
        sim.initFromArray(p0)
        sims.append(sim)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for inst, sim in zip(insts[:loop_n], sims):
        W.apply(sim, inst["gates"])
        sim.synchronize()
    loop_s = time.perf_counter() - t0
    amps = sum(1 << sum(i["qubits"]) for i in insts)
    return {"value": len(insts) / (ms * 1e-3), "unit": "instances/s", "ms_per_run": ms,
            "instances": len(insts), "gates_per_instance": 50, "amplitudes": amps,
            "state_bytes": amps * 8, "gpu_launches_per_run": B.n_stages, "grid": grid, "pair_chunk": chunk,
            "row_loge": {str(k): v for k, v in sorted(B.row_loge.items())},
            "ms_per_run_default_shapes": ms_default,
            "autotune_trials": {"grid_chunk": B.tuning["grid_chunk"], "row_loge": B.tuning["row_loge"]},
            "per_instance_loop": {"value": loop_n / loop_s, "unit": "instances/s", "instances": loop_n,
                                  "how": "CudaCvdv complex64, one instance after another, wall clock"},
            "speedup_vs_loop": (len(insts) / (ms * 1e-3)) / (loop_n / loop_s),
            "note": "whole batch is L2-resident (state_bytes < 126 MB)"}


def gaussian_c3(args):
    """Two modes [13, 13] (2^26 amplitudes; [12, 12] for --workload small), complex128 and
    complex64: layers of (beam splitter, rotation of each mode, displacement of each mode);
    20 layers per step, then the Wigner function of mode 0 (read back)."""
    import torch
    from cvdv_b200 import CudaCvdv, _lib
    from cvdv_b200 import workloads as W
    L = _lib.load()
    layers = 20
    mq = 13 if args.workload == "full" else 12
    circ = W.gaussian_network(layers=layers, mode_qubits=mq)
    out = {"unit": "layers/s", "layers_per_step": layers, "gates_per_layer": len(circ["gates"]) // layers}
    # complex64_tensor_core: the same complex64 run with mode 0's transforms as
    # chained four-step passes of DFT-matrix products on the tensor cores (fusion
    # bit 5, opt-in) instead of the one-pass column programs
    for prec, label, flags in (("complex128", "complex128", 31), ("complex64", "complex64", 31),
                               ("complex64", "complex64_tensor_core", 63)):
        sim = CudaCvdv(circ["qubits"], precision=prec, check_errors=True, fusion=flags)
        sim.initStateVector(W.separable_arrays(circ, device="cuda"))
        W.apply(sim, circ["prep"])
        W.apply(sim, circ["gates"])  # warm-up
        sim.synchronize()
        stream = torch.cuda.ExternalStream(L.cvdvGetStream(sim.ctx))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(1, min(args.steps, 3))
        e0.record(stream)
        for _ in range(reps):
            W.apply(sim, circ["gates"])
            L.cvdvFlush(sim.ctx)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / (reps * layers)
        # per-kind kernel times of one more step, with per-launch events on
        L.cvdvSetTiming(sim.ctx, 1)
        _lib.kernel_stats(sim.ctx)
        W.apply(sim, circ["gates"])
        L.cvdvFlush(sim.ctx)
        st = _lib.kernel_stats(sim.ctx)
        L.cvdvSetTiming(sim.ctx, 0)
        kern = {k: {"ms_per_layer": v[0] / layers, "launches_per_layer": v[1] / layers}
                for k, v in st.items() if v[1]}
        state_bytes = (16 if prec == "complex128" else 8) << sum(circ["qubits"])
        for k in ("col", "col_tc"):  # one column pass reads and writes the state once
            if k in kern:
                avg = kern[k]["ms_per_layer"] / kern[k]["launches_per_layer"]
                kern[k]["achieved_gbs"] = 2 * state_bytes / (avg * 1e-3) / 1e9
        t0 = time.perf_counter()
        w = sim.getWigner(0)
        wig_s = time.perf_counter() - t0
        out[label] = {"value": 1e3 / ms, "ms_per_layer": ms, "wigner_s": wig_s, "wigner_shape": list(w.shape),
                      "kernels": kern}
        del sim
        torch.cuda.empty_cache()
    out["value"] = out["complex128"]["value"]
    if not getattr(args, "no_accuracy", False):
        out["accuracy_complex64"] = gaussian_c3_accuracy(mq)
    return out


def gaussian_c3_accuracy(mq, layers=200, n=256, bound=6.0):
    """The whole configured network (200 layers) in complex64 and complex128 from the same
    input: state errors, both position marginals, and mode 0's Wigner function on the
    256 x 256 grid over [-6, 6]^2 (FP64 bilinear resampling of the native grid)."""
    import numpy as np
    import torch
    from cvdv_b200 import CudaCvdv
    from cvdv_b200 import workloads as W
    from cvdv_b200.accuracy import wigner_grid, wigner_mean
    circ = W.gaussian_network(layers=layers, mode_qubits=mq)
    sims, wig, marg = {}, {}, {}
    for prec, label, flags in (("complex128", "complex128", 31), ("complex64", "complex64", 31),
                               ("complex64", "tc", 63)):
        sim = CudaCvdv(circ["qubits"], precision=prec, check_errors=True, fusion=flags)
        sim.initStateVector(W.separable_arrays(circ, device="cuda"))
        W.apply(sim, circ["prep"])
        W.apply(sim, circ["gates"])
        sim.synchronize()
        sims[label] = sim
        marg[label] = sim.mEach([0, 1])
        wig[label] = sim.getWigner(0) if label != "tc" else None
    acc = compare_states(sims["complex128"].stateTensor(), sims["complex64"].stateTensor())
    acc["tensor_core_columns"] = compare_states(sims["complex128"].stateTensor(), sims["tc"].stateTensor())
    del sims
    torch.cuda.empty_cache()
    g128, g64 = wigner_grid(wig["complex128"], n, bound), wigner_grid(wig["complex64"], n, bound)
    c = wigner_mean(wig["complex128"])
    h128, h64 = wigner_grid(wig["complex128"], n, bound, c), wigner_grid(wig["complex64"], n, bound, c)
    acc.update({"layers": layers, "against": "the complex128 path on the GPU",
                "marginal_max_abs_err": max(float(np.abs(a - b).max()) for a, b in zip(marg["complex128"],
                                                                                      marg["complex64"])),
                "marginal_max": max(float(a.max()) for a in marg["complex128"]),
                "wigner_native_max_abs_err": float(np.abs(wig["complex64"] - wig["complex128"]).max()),
                "wigner_native_max_abs": float(np.abs(wig["complex128"]).max()),
                "wigner_grid": f"{n}x{n} over [-{bound}, {bound}]^2, bilinear FP64 resampling of the native grid",
                "wigner_grid_max_abs_err": float(np.abs(g64 - g128).max()),
                "wigner_grid_max_abs": float(np.abs(g128).max()),
                "wigner_grid_note": "200 random displacements walk mode 0 to |alpha| ~ 14, outside the origin square; "
                                    "the centred grid is the same size around the state's mean (x, p)",
                "wigner_centred_grid_center": list(c),
                "wigner_centred_grid_max_abs_err": float(np.abs(h64 - h128).max()),
                "wigner_centred_grid_max_abs": float(np.abs(h128).max())})
    return acc


def variational_c5(args):
    """64 parameter sets of [1, 12] x 40 layers (Rx, cd), complex64: loss and adjoint gradient."""
    import torch
    from cvdv_b200 import workloads as W
    from cvdv_b200.variational import VariationalCircuit, layered_gates
    w = W.variational()
    psi0 = W.product_state(w["qubits"], w["init"]).cuda()
    tgt = W.product_state(w["qubits"], w["target"]).cuda()
    params = torch.tensor(w["params"], device="cuda")

    def time_steps(graphs):
        circ = VariationalCircuit(w["qubits"], layered_gates(40), precision="complex64", checkpoint_every=16,
                                  graphs=graphs)

        def step():
            p = params.clone().requires_grad_(True)
            circ.fidelity_loss(p, psi0, tgt).sum().backward()
            return p.grad

        for _ in range(2):
            step()
        reps = max(args.steps, 3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            step()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    ms = time_steps(True)
    ms_eager = time_steps(False)

    # adjoint gradients against central differences (h = 1e-4) of the complex128
    # forward, all 2 x 64 x 80 perturbed sets in one batched forward
    def grad_of(precision):
        c = VariationalCircuit(w["qubits"], layered_gates(40), precision=precision, checkpoint_every=16)
        p = params.clone().requires_grad_(True)
        c.fidelity_loss(p, psi0, tgt).sum().backward()
        return p.grad.detach()

    B, P = params.shape
    fdc = VariationalCircuit(w["qubits"], layered_gates(40), precision="complex128", checkpoint_every=16)
    h = 1e-4
    plus = params.repeat_interleave(P, dim=0)
    minus = plus.clone()
    idx = torch.arange(P, device=params.device).repeat(B)
    rows = torch.arange(plus.shape[0], device=params.device)
    plus[rows, idx] += h
    minus[rows, idx] -= h
    with torch.no_grad():
        fd = ((fdc.fidelity_loss(plus, psi0, tgt) - fdc.fidelity_loss(minus, psi0, tgt)) / (2 * h)).reshape(B, P)
    scale = float(fd.abs().max())
    fd_err = {prec: float((grad_of(prec) - fd).abs().max()) / scale for prec in ("complex128", "complex64")}
    return {"value": 64 / (ms * 1e-3), "unit": "parameter-set gradients/s", "ms_per_step": ms,
            "batch": 64, "params_per_set": 80, "layout": [1, 12], "dtype": "c64",
            "step": "forward (80 gates as 40 fused Rx + cd layers) + overlap + adjoint sweep (40 fused layers: "
                    "both gradients and the inverse gates), checkpoints every 16 gates; both sweeps replayed from "
                    "CUDA graphs",
            "eager": {"value": 64 / (ms_eager * 1e-3), "ms_per_step": ms_eager,
                      "how": "the same step launching kernel by kernel from Python"},
            "adjoint_vs_central_differences": {"h": h, "max_rel_err": fd_err, "target": 1e-6,
                                               "how": "max |adjoint - FD| / max |FD| over all 64 x 80 "
                                                      "gradients; FD of the complex128 forward"}}


def husimi_readout(args):
    """Husimi Q of the mode of [1, 10] and [1, 12] (N = 1024, 4096; two slices): the
    overlap route as one fused pass per output row (cvdvGetHusimiQ), kernel time and
    wall time including the N^2 read-back."""
    import numpy as np
    import torch
    from cvdv_b200 import CudaCvdv, _lib
    L = _lib.load()
    out = {"unit": "ms"}
    for qubits in ([1, 10], [1, 12]):
        rng = np.random.default_rng(1)
        n = sum(qubits)
        psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
        sim = CudaCvdv(qubits, check_errors=True)
        sim.initFromArray(psi / np.linalg.norm(psi))
        sim.getHusimiQ(1)
        L.cvdvSetTiming(sim.ctx, 1)
        _lib.kernel_stats(sim.ctx)
        reps = max(3, min(args.steps, 5))
        t0 = time.perf_counter()
        for _ in range(reps):
            sim.getHusimiQ(1)
        wall = (time.perf_counter() - t0) / reps
        st = _lib.kernel_stats(sim.ctx)
        L.cvdvSetTiming(sim.ctx, 0)
        out[f"N={1 << qubits[1]}"] = {"kernel_ms": (st["phase_space"][0] + st["fft_pass"][0]) / reps,
                                      "wall_ms": wall * 1e3, "launches": (st["phase_space"][1] + st["fft_pass"][1]) / reps}
        del sim
        torch.cuda.empty_cache()
    return out


def diagonal_runs(args):
    """A standalone diagonal run on two modes [14, 14] (2^28 complex128 amplitudes;
    [12, 12] for --workload small): a bilinear phase, a shear and a cubic phase that
    no transform, sequence or row program absorbs run as one k_diag pass (each
    register's phases from one table, the bilinear term's sincos per amplitude)."""
    import torch
    from cvdv_b200 import CudaCvdv, _lib
    from cvdv_b200.separable import SeparableState
    L = _lib.load()
    mq = 14 if args.workload == "full" else 12
    sep = SeparableState([mq, mq])
    sep.setCoherent(0, 0.5 + 0.2j)
    sep.setFock(1, 1)
    sim = CudaCvdv([mq, mq], check_errors=True)
    sim.initStateVector(sep)

    def run():
        sim.q1q2(0, 1, 0.1)
        sim.sheer(0, 0.05)
        sim.phaseCubic(1, 0.01)
        L.cvdvFlush(sim.ctx)

    run()
    sim.synchronize()
    stream = torch.cuda.ExternalStream(L.cvdvGetStream(sim.ctx))
    reps = max(3, min(args.steps, 10))
    for _ in range(args.warmup):
        run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        run()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    L.cvdvSetTiming(sim.ctx, 1)
    _lib.kernel_stats(sim.ctx)
    run()
    st = _lib.kernel_stats(sim.ctx)
    L.cvdvSetTiming(sim.ctx, 0)
    state_bytes = 16 << (2 * mq)
    diag_ms, n = st["diag"]
    out = {"unit": "ms", "amplitudes": 1 << (2 * mq), "ms_per_run": ms, "diag_launches": n,
           "table_builds": st["table"][1], "table_ms": st["table"][0],
           "achieved_gbs": 2 * state_bytes / (diag_ms / max(n, 1) * 1e-3) / 1e9 if n else None}
    del sim
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the one-circuit and 200-layer accuracy legs (profiler runs)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched-circuits and variational-gradient measurements")
    ap.add_argument("--workload", default="full", choices=["full", "small"],
                    help="small: 10 qubit registers + the 2^14 mode (2^24 amplitudes), and the two-mode "
                         "network at [12, 12], for ncu")
    ap.add_argument("--extra", default=None, choices=["c3", "c4", "c5", "husimi", "diag"],
                    help="run only that extra measurement (one GPU) and print its JSON, for profiling")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_init()
    try:
        if args.extra:
            fn = {"c3": gaussian_c3, "c4": batched_c4, "c5": variational_c5, "husimi": husimi_readout,
                  "diag": diagonal_runs}[args.extra]
            print(json.dumps({"extra": args.extra, **fn(args)}), flush=True)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_gpu(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
