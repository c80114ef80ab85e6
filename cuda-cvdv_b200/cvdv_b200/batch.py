"""Batched independent circuits of uneven layouts.

``BatchedCircuits`` runs many independent instances -- each a layout
``[1]*Q + [m]`` (Q one-qubit registers, a mode of 2^m points, m = 8..14) with
its own gate list in the ``CudaCvdv`` vocabulary -- in one state array.  Stage
s applies every instance's s-th gate in ONE persistent launch
(``cvdvBatchRunStage``): the host compiles each gate, once, into tasks -- a
row program for gates on the mode (the reference decompositions of
src/cuda/gates.cu: transforms, parity and phase polynomials) or a 2x2 gate on
a qubit bit -- and the stages can be captured in one CUDA graph and replayed.

Supported gates: ``h``, ``rx``, ``ry``, ``rz`` (qubit registers), ``d``,
``cd``, ``s``, ``r``, ``sheer``, ``ftQ2P``, ``ftP2Q`` (the mode).  Decompositions
follow the single-instance path exactly (thresholds 1e-12 / 1e-15, rint for the
rotation's quarter turns, dropped global phases), so every instance matches
``CudaCvdv`` running the same gates.

Tuning: ``autotune()`` times candidates on the compiled batch: the persistent
grid size, the pair-gate chunk (the 2x2-gate tasks' shape), and, per mode
length 2^m of the batch, the row tasks' amplitudes per thread 2^logE -- which
is both the radix schedule of their transforms (radix-8, 16 or 32 Stockham
stages) and the rows a CTA holds (512 2^logE / 2^m) -- by coordinate descent
over the mode lengths, largest total work first.  The result is kept per
(mode length, precision) in ``row_loge``.
"""

from __future__ import annotations

import ctypes
import math
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .cudaCvdv import PRECISIONS, CvdvError

PHASE_DTYPE = np.dtype([("a1", "f8"), ("b1", "f8"), ("a2", "f8"), ("b2", "f8"), ("a3", "f8"), ("g0", "f8"),
                        ("h0", "f8"), ("scale", "f8"), ("tw", "i4"), ("ctrlBit", "i4")])
PROGRAM_DTYPE = np.dtype([("nOps", "i4"), ("op", "i4", (15,)), ("phase", PHASE_DTYPE, (8,))])
TASK_DTYPE = np.dtype([("stateOffset", "i8"), ("kind", "i4"), ("n", "i4"), ("logRow", "i4"), ("first", "i4"),
                       ("count", "i4"), ("bit", "i4"), ("program", "i4"), ("logE", "i4"), ("m", "f8", (8,))])

OP_DIAG, OP_FWD, OP_INV, OP_PARITY = 0, 1, 2, 3
SQRT2 = math.sqrt(2.0)
THREADS = 512


def loge_options(m: int, prec: int) -> List[int]:
    """Amplitudes per thread (log2) a row task of 2^m points can use: a row fits the
    512 threads, and complex128 rows at most 16 per thread (shared memory)."""
    top = 5 if prec == 1 else 4
    return [e for e in (3, 4, 5) if e <= top and e <= m and m - e <= 9]


def default_loge(m: int, prec: int) -> int:
    return 5 if (prec == 1 and m >= 13) else 4


def struct_sizes() -> Tuple[int, int, int]:
    s = (ctypes.c_int * 3)()
    _lib.load().cvdvBatchStructSizes(s)
    return int(s[0]), int(s[1]), int(s[2])


class _Phase:
    """Accumulates diagonal terms of one run: scale * exp(i [tw theta_j + g0 + Z h0 + ...])."""

    def __init__(self) -> None:
        self.c = dict(a1=0.0, b1=0.0, a2=0.0, b2=0.0, a3=0.0, g0=0.0, h0=0.0)
        self.scale = 1.0
        self.tw = 0
        self.ctrl = -1

    def poly(self, power: int, coeff: float, ctrl: int = -1) -> None:
        if ctrl >= 0:
            if self.ctrl not in (-1, ctrl):
                raise ValueError("one control bit per diagonal run")
            self.ctrl = ctrl
            self.c[f"b{power}"] += coeff
        else:
            self.c[f"a{power}"] += coeff

    def record(self) -> np.void:
        r = np.zeros((), dtype=PHASE_DTYPE)
        for k, v in self.c.items():
            r[k] = v
        r["scale"] = self.scale
        r["tw"] = self.tw
        r["ctrlBit"] = self.ctrl
        return r


def _ft_global(N: int, sign: int) -> float:
    m = ((N - 1) * (N - 1)) % (4 * N)
    return sign * math.pi * m / (2.0 * N)


class _RowProgram:
    """Ops of one mode gate; consecutive diagonal terms merge into one phase."""

    def __init__(self, N: int) -> None:
        self.N = N
        self.ops: List[int] = []
        self.phases: List[_Phase] = []

    def _diag(self) -> _Phase:
        if not self.ops or self.ops[-1] != OP_DIAG:
            self.ops.append(OP_DIAG)
            self.phases.append(_Phase())
        return self.phases[-1]

    def poly(self, power: int, coeff: float, ctrl: int = -1) -> None:
        self._diag().poly(power, coeff, ctrl)

    def ft(self, sign: int) -> None:  # FtQ2P (+1) / FtP2Q (-1), src/cuda/gates.cu:19-122
        self._diag().tw += sign
        self.ops.append(OP_FWD if sign > 0 else OP_INV)
        ph = self._diag()
        ph.tw += sign
        ph.scale /= math.sqrt(self.N)
        ph.c["g0"] += _ft_global(self.N, sign)

    def parity(self) -> None:
        self.ops.append(OP_PARITY)

    def rotation_small(self, th: float) -> None:  # gates.cu:572-584
        if abs(th) < 1e-15:
            return
        t, s = math.tan(th / 2.0), math.sin(th)
        self.poly(2, -0.5 * t)
        self.ft(1)
        self.poly(2, -0.5 * s)
        self.ft(-1)
        self.poly(2, -0.5 * t)

    def record(self) -> np.void:
        if len(self.ops) > 15 or len(self.phases) > 8:
            raise ValueError("gate program too long")
        r = np.zeros((), dtype=PROGRAM_DTYPE)
        r["nOps"] = len(self.ops)
        r["op"][: len(self.ops)] = self.ops
        for i, p in enumerate(self.phases):
            r["phase"][i] = p.record()
        return r


def _mode_program(name: str, args: tuple, N: int, ctrl_bit: int) -> _RowProgram:
    P = _RowProgram(N)
    if name == "d":  # gates.cu:124-161
        a = complex(args[0])
        if abs(a.imag) > 1e-12:
            P.poly(1, SQRT2 * a.imag)
        if abs(a.real) > 1e-12:
            P.ft(1)
            P.poly(1, -SQRT2 * a.real)
            P.ft(-1)
    elif name == "cd":  # gates.cu:163-204
        a = complex(args[0])
        if abs(a.imag) > 1e-12:
            P.poly(1, SQRT2 * a.imag, ctrl_bit)
        if abs(a.real) > 1e-12:
            P.ft(1)
            P.poly(1, -SQRT2 * a.real, ctrl_bit)
            P.ft(-1)
    elif name == "sheer":
        P.poly(2, float(args[0]))
    elif name == "s":  # gates.cu:394-421
        r = float(args[0])
        a, b, s = math.exp(0.5 * r), math.exp(-0.5 * r), math.sqrt(abs(math.exp(r) - 1.0))
        sg = 1.0 if r >= 0 else -1.0
        P.ft(1)
        P.poly(2, -0.5 * a * s)
        P.ft(-1)
        P.poly(2, 0.5 * b * s * sg)
        P.ft(1)
        P.poly(2, 0.5 * b * s)
        P.ft(-1)
        P.poly(2, -0.5 * a * s * sg)
    elif name == "r":  # gates.cu:316-348 (rint on the quarter turns)
        theta = float(args[0])
        theta0 = float(np.rint(theta / (math.pi / 2.0))) * (math.pi / 2.0)
        qt = int(np.rint(theta0 / (math.pi / 2.0))) % 4
        if qt == 1:
            P.ft(1)
        elif qt == 2:
            P.parity()
        elif qt == 3:
            P.ft(-1)
        P.rotation_small(theta - theta0)
    elif name == "ftQ2P":
        P.ft(1)
    elif name == "ftP2Q":
        P.ft(-1)
    else:
        raise ValueError(f"unsupported mode gate {name!r}")
    return P


def _qubit_matrix(name: str, args: tuple) -> Optional[np.ndarray]:
    """2x2 matrix (row-major) of a qubit gate, None for Rz (diagonal, run as a phase)."""
    if name == "h":
        h = 1.0 / math.sqrt(2.0)
        return np.array([h, h, h, -h], dtype=np.complex128)
    th = float(args[-1]) if name in ("rx", "ry") else 0.0
    c, s = math.cos(th / 2.0), math.sin(th / 2.0)
    if name == "rx":  # gates.cuh:63-92
        return np.array([c, -1j * s, -1j * s, c])
    if name == "ry":
        return np.array([c, -s, s, c], dtype=np.complex128)
    return None


class BatchedCircuits:
    QUBIT_GATES = ("h", "rx", "ry", "rz")

    def __init__(self, instances: Sequence[Dict[str, Any]], precision: str = "complex64",
                 pair_chunk: int = 4096, grid: int = 148, row_loge: Optional[Dict[int, int]] = None) -> None:
        """instances: dicts with ``qubits`` ([1]*Q + [m]) and ``gates`` [(name, args)];
        row_loge: amplitudes per thread (log2) of the row tasks per mode length m
        (default 4, or 5 for complex64 modes of 2^13 and 2^14 points)."""
        self.prec = PRECISIONS[precision]
        self.cdtype = torch.complex128 if self.prec == 0 else torch.complex64
        self.instances = list(instances)
        self.grid = grid
        self.pair_chunk = pair_chunk
        self.row_loge: Dict[int, int] = dict(row_loge or {})
        for m, e in self.row_loge.items():
            if e not in loge_options(m, self.prec):
                raise ValueError(f"row_loge[{m}] = {e}: choose from {loge_options(m, self.prec)}")
        max_log = 14 if self.prec == 1 else 13
        self.offsets = []
        off = 0
        for inst in self.instances:
            q = inst["qubits"]
            if any(x != 1 for x in q[:-1]) or not (8 <= q[-1] <= max_log):
                raise ValueError(f"layout {q}: one-qubit registers and a mode of 2^8..2^{max_log} points")
            self.offsets.append(off)
            off += 1 << sum(q)
        self.total = off
        self.n_stages = max(len(i["gates"]) for i in self.instances)
        self.states = torch.zeros(self.total, dtype=self.cdtype, device="cuda")
        self._L = _lib.load()
        self._graph = None
        self._compile()

    # ---------------------------------------------------------------- compile
    def _compile(self) -> None:
        progs: List[np.void] = []
        stage_tasks: List[List[np.void]] = [[] for _ in range(self.n_stages)]
        for i, inst in enumerate(self.instances):
            q = inst["qubits"]
            n, m = sum(q), q[-1]
            mode = len(q) - 1
            logE = self.row_loge.get(m, default_loge(m, self.prec))
            rows_per_task = max(1, THREADS // ((1 << m) >> logE))
            for s, (name, args) in enumerate(inst["gates"]):
                if name in self.QUBIT_GATES:
                    reg = args[0]
                    bit = n - 1 - reg  # one-qubit register r holds flat bit n-1-r
                    M = _qubit_matrix(name, args)
                    if M is None:  # Rz: diag(e^{-i t/2}, e^{i t/2}) as a row phase
                        P = _RowProgram(1 << m)
                        ph = P._diag()
                        ph.ctrl = bit
                        ph.c["h0"] = -0.5 * float(args[-1])
                        stage_tasks[s] += self._row_tasks(i, n, m, len(progs), rows_per_task, logE)
                        progs.append(P.record())
                    else:
                        pairs = 1 << (n - 1)
                        for first in range(0, pairs, self.pair_chunk):
                            t = np.zeros((), dtype=TASK_DTYPE)
                            t["stateOffset"], t["kind"], t["n"], t["logRow"] = self.offsets[i], 1, n, m
                            t["first"], t["count"], t["bit"] = first, min(self.pair_chunk, pairs - first), bit
                            t["m"] = np.stack([M.real, M.imag], axis=1).reshape(-1)
                            stage_tasks[s].append(t)
                else:
                    if args[0] != mode:
                        raise ValueError("mode gates act on the last register")
                    ctrl = -1
                    if name == "cd":
                        ctrl = n - 1 - args[1]
                        args = (args[3],)
                    else:
                        args = tuple(args[1:])
                    P = _mode_program(name, args, 1 << m, ctrl)
                    stage_tasks[s] += self._row_tasks(i, n, m, len(progs), rows_per_task, logE)
                    progs.append(P.record())
        self.n_programs = len(progs)
        prog_arr = np.array(progs, dtype=PROGRAM_DTYPE) if progs else np.zeros(1, dtype=PROGRAM_DTYPE)
        self._progs = torch.from_numpy(prog_arr.view(np.uint8).copy()).cuda()
        nfft = [int(np.isin(pr["op"][: pr["nOps"]], (OP_FWD, OP_INV)).sum()) for pr in progs]

        def cost(t: np.void) -> int:
            """Work of a task: amplitudes, times the transforms' log2 length for row programs."""
            if int(t["kind"]) == 0:
                m = int(t["logRow"])
                return (int(t["count"]) << m) * (2 + nfft[int(t["program"])] * m)
            return int(t["count"]) * 4

        self._tasks = []
        for tl in stage_tasks:
            # the CTAs take tasks round-robin: largest first, so the long row programs
            # start in the first wave instead of trailing the stage
            tl = sorted(tl, key=cost, reverse=True)
            arr = np.array(tl, dtype=TASK_DTYPE) if tl else np.zeros(0, dtype=TASK_DTYPE)
            self._validate(arr)
            self._tasks.append((torch.from_numpy(arr.view(np.uint8).copy()).cuda(), len(arr)))

    def _row_tasks(self, i: int, n: int, m: int, prog: int, per: int, logE: int) -> List[np.void]:
        out = []
        rows = 1 << (n - m)
        for first in range(0, rows, per):
            t = np.zeros((), dtype=TASK_DTYPE)
            t["stateOffset"], t["kind"], t["n"], t["logRow"] = self.offsets[i], 0, n, m
            t["first"], t["count"], t["program"], t["logE"] = first, min(per, rows - first), prog, logE
            out.append(t)
        return out

    def _validate(self, arr: np.ndarray) -> None:
        """Every task stays inside its instance (checked before anything runs on the GPU)."""
        for t in arr:
            size = 1 << int(t["n"])
            if t["stateOffset"] < 0 or t["stateOffset"] + size > self.total:
                raise CvdvError("task outside the batch array")
            if t["kind"] == 0:
                if (int(t["first"]) + int(t["count"])) << int(t["logRow"]) > size:
                    raise CvdvError("row task outside its instance")
                if int(t["logE"]) not in loge_options(int(t["logRow"]), self.prec):
                    raise CvdvError("row task shape the stage kernel does not take")
                if int(t["count"]) > THREADS // ((1 << int(t["logRow"])) >> int(t["logE"])):
                    raise CvdvError("row task larger than a CTA")
                if not (0 <= t["program"] < self.n_programs):
                    raise CvdvError("row task program index out of range")
            else:
                if not (0 <= t["bit"] < t["n"]) or int(t["first"]) + int(t["count"]) > size // 2:
                    raise CvdvError("pair task outside its instance")

    # ---------------------------------------------------------------- run
    def set_initial(self, states: Sequence[torch.Tensor]) -> None:
        for off, psi in zip(self.offsets, states):
            self.states[off: off + psi.numel()].copy_(psi.reshape(-1).to(self.cdtype))

    def state(self, i: int) -> torch.Tensor:
        n = sum(self.instances[i]["qubits"])
        return self.states[self.offsets[i]: self.offsets[i] + (1 << n)]

    def _launch_all(self) -> None:
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        for tasks, nt in self._tasks:
            code = self._L.cvdvBatchRunStage(ctypes.c_void_p(self.states.data_ptr()), self.prec,
                                             ctypes.c_void_p(tasks.data_ptr()), nt,
                                             ctypes.c_void_p(self._progs.data_ptr()), self.grid, stream)
            if code:
                raise CvdvError(_lib.last_error(None)[1])

    def run(self, graph: bool = False) -> None:
        """All stages, in order; with graph=True the launches are captured once and replayed."""
        if not graph:
            self._launch_all()
            return
        if self._graph is None:
            self._launch_all()  # first call sets kernel attributes outside the capture
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    self._launch_all()
            self._graph = g
            return  # the capture itself does not run: the warm-up call above was the run
        self._graph.replay()

    def _time(self, reps: int) -> float:
        self._launch_all()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            self._launch_all()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    def autotune(self, grids: Sequence[int] = (148, 296), chunks: Sequence[int] = (2048, 8192),
                 reps: int = 3, tune_rows: bool = True) -> Tuple[int, int]:
        """Time every (grid, pair chunk) pair on the compiled batch and keep the
        fastest; then, per mode length (largest total work first), every row-task
        shape loge_options(m) with the others fixed (coordinate descent), keeping
        the fastest in row_loge.  The states are saved and restored around the
        timing runs.  Returns (grid, pair chunk); self.tuning records every trial."""
        saved = self.states.clone()
        self.tuning = {"grid_chunk": [], "row_loge": []}
        best = None
        for chunk in chunks:
            self.pair_chunk = chunk
            self._compile()
            for grid in grids:
                self.grid = grid
                ms = self._time(reps)
                self.tuning["grid_chunk"].append((grid, chunk, ms))
                if best is None or ms < best[0]:
                    best = (ms, grid, chunk)
        best_ms, self.grid, self.pair_chunk = best
        if tune_rows:
            work: Dict[int, int] = {}
            for inst in self.instances:
                m = inst["qubits"][-1]
                work[m] = work.get(m, 0) + (1 << sum(inst["qubits"]))
            for m in sorted(work, key=lambda k: -work[k]):
                keep = self.row_loge.get(m, default_loge(m, self.prec))
                for e in loge_options(m, self.prec):
                    if e == keep:
                        continue
                    self.row_loge[m] = e
                    self._compile()
                    ms = self._time(reps)
                    self.tuning["row_loge"].append((m, e, ms))
                    if ms < best_ms:
                        best_ms, keep = ms, e
                self.row_loge[m] = keep
        self._compile()
        self._graph = None
        self.states.copy_(saved)
        return self.grid, self.pair_chunk


def random_instances(seed: int = 4, count: int = 512, gates: int = 50, m_range=(8, 14),
                     q_range=(1, 3)) -> List[Dict[str, Any]]:
    """Seeded uneven circuits: Q ~ U{q_range} qubits, mode 2^m, m ~ U{m_range}; gates uniform from
    {H, Rx, Rz, cd, d, s, r}, angles ~ U[0, 2pi), beta, alpha ~ (X + iY)/sqrt2 with X, Y ~ N(0, 1),
    r ~ U[0, 0.5]; qubit gates and cd controls on a uniform qubit register.  Start: qubits |0>,
    mode vacuum."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        Q = int(rng.integers(q_range[0], q_range[1] + 1))
        m = int(rng.integers(m_range[0], m_range[1] + 1))
        qubits = [1] * Q + [m]
        mode = Q
        gl = []
        for _ in range(gates):
            g = int(rng.integers(7))
            if g == 0:
                gl.append(("h", (int(rng.integers(Q)), 0)))
            elif g == 1:
                gl.append(("rx", (int(rng.integers(Q)), 0, float(rng.uniform(0, 2 * math.pi)))))
            elif g == 2:
                gl.append(("rz", (int(rng.integers(Q)), 0, float(rng.uniform(0, 2 * math.pi)))))
            elif g == 3:
                beta = complex(rng.standard_normal(), rng.standard_normal()) / math.sqrt(2.0)
                gl.append(("cd", (mode, int(rng.integers(Q)), 0, beta)))
            elif g == 4:
                alpha = complex(rng.standard_normal(), rng.standard_normal()) / math.sqrt(2.0)
                gl.append(("d", (mode, alpha)))
            elif g == 5:
                gl.append(("s", (mode, float(rng.uniform(0, 0.5)))))
            else:
                gl.append(("r", (mode, float(rng.uniform(0, 2 * math.pi)))))
        init = [("setZero", ())] * Q + [("setFock", (0,))]
        out.append(dict(qubits=qubits, gates=gl, init=init))
    return out
