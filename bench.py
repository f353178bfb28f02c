"""Benchmark: second-order Trotter evolution of the XXZ chain on one B200.

Workload (the Trotter configuration of the reference's state-vector path):
XXZ chain N=28, open boundary, J=1, Delta=0.5, on-site fields h_i ~ U[-1,1]
(seed 42), Neel initial state, Strang splitting S2(dt) = S1(dt/2) then
reversed S1(dt/2) with S1 = [Rz fields; per bond Rxx, Ryy, Rzz]
(218 gate applications per step), dt = 0.05, 200 steps, <Z_i> recorded every
10 steps (21 records); complex64 amplitudes, FP64 reductions.

One bench step = one whole 200-step evolution from the initial state,
43,600 gate applications.  metric = gate applications per second (whole job).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs an independent replica (the path does
not shard: one state per GPU); value = all ranks' gate applications / the
max over ranks of the device time.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "smoq.jl_b200"))

N_QUBITS = 28
DT = 0.05
STEPS = 200
RECORD_EVERY = 10
J, DELTA = 1.0, 0.5
SEED = 42
GATES_PER_STEP = 2 * (N_QUBITS + 3 * (N_QUBITS - 1))  # 218
GATE_APPS = STEPS * GATES_PER_STEP                    # 43,600 per bench step
WORKLOAD = "xxz_chain_trotter2_n28_c64_200steps"


def rz(t):
    return np.diag([np.exp(-0.5j * t), np.exp(0.5j * t)])


def rpp(P, t):
    PP = np.kron(P, P)
    return np.cos(t / 2) * np.eye(4) - 1j * np.sin(t / 2) * PP


X = np.array([[0, 1], [1, 0]], complex)
Y = np.array([[0, -1j], [1j, 0]], complex)
Z = np.array([[1, 0], [0, -1]], complex)


def s1_gates(N, tau):
    """S1(tau) as (1-based indices, U): Rz(2 h_i tau) on every site, then per bond
    Rxx(2 J tau), Ryy(2 J tau), Rzz(2 J Delta tau)."""
    h = np.random.default_rng(SEED).uniform(-1, 1, size=N)
    g = [([i + 1], rz(2 * h[i] * tau)) for i in range(N)]
    for i in range(1, N):
        g += [([i, i + 1], rpp(X, 2 * J * tau)), ([i, i + 1], rpp(Y, 2 * J * tau)),
              ([i, i + 1], rpp(Z, 2 * J * DELTA * tau))]
    return g


def neel_index(N):
    return sum(1 << (k - 1) for k in range(1, N + 1, 2))


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(ms, dist, device):
    """The slowest replica's device time: every rank passes its own CUDA-event time
    and gets back the maximum (the job finishes when its slowest rank does)."""
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, ranks, ms):
    """Whole-job throughput of independent replicas: all ranks' units over the
    slowest rank's time (weak scaling: the work per rank is fixed)."""
    return ranks * units_per_rank / (ms * 1e-3)


class Clocks:
    """nvidia-smi sampler during the timed region."""

    def __init__(self, device):
        self.device = device
        self.p = None
        # the raw samples go to $SMOQ_CLOCKS_DIR when set (kept as evidence), else to a temp file
        d = os.environ.get("SMOQ_CLOCKS_DIR")
        self.path = os.path.join(d, f"clocks_rank{device}.csv") if d and os.path.isdir(d) else \
            os.path.join(tempfile.gettempdir(), f"smoq_clocks_{os.getpid()}_{device}.csv")

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        for ln in open(self.path):
            c = [x.strip() for x in ln.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx = float(c[2])
            except ValueError:
                continue
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], c[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


ENGINE_KERNELS = {0: ("tile_pass_kernel<float>", "tile_pass_xxz_n28_c64.json"),
                  2: ("stage_kernel<float>", None),
                  3: ("smoq_pass_e0 (compiled per pass)", "compiled_pass_xxz_n28_c64.json")}


def resolve_engine(S, engine):
    """the fused-pass engine a Trotter plan runs: the option, or the library's auto
    choice (compiled pass kernels when NVRTC loads, else shared-memory sweeps)"""
    if engine >= 0:
        return engine
    return 3 if S.jit_available() else 0


def ncu_traffic(engine):
    name = ENGINE_KERNELS[engine][1]
    if name is None:
        return None
    p = os.path.join(ROOT, "profiles", name)
    if os.path.exists(p):
        try:
            return float(json.load(open(p))["traffic_bytes_per_launch"])
        except Exception:
            return None
    return None


def cpu_baseline_sample(n_gates=12, N=N_QUBITS):
    """The oracle (CPU restatement of the reference's loops, one thread) on the
    first n_gates of one Strang step at full N, complex128."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    gl = s1_gates(N, DT / 2)
    both = gl + gl[::-1]
    sample = both[:n_gates]
    arr = O.make_gates([([q for q in idx], U) for idx, U in sample])
    psi = O.zero_state(N, neel_index(N))
    t0 = O.wtime()
    O.trotter_step(psi, arr, len(sample), N)
    dt = O.wtime() - t0
    return len(sample) / dt, dt


def cpu_model():
    """the host CPU's model name (for the CPU baseline's record)"""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip() + f" ({os.cpu_count()} logical cores)"
    except OSError:
        pass
    return None


def reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    n_gates = 8
    for _ in range(args.warmup):
        cpu_baseline_sample(n_gates)
    rates, tot = [], 0.0
    for _ in range(args.steps):
        r, t = cpu_baseline_sample(n_gates)
        rates.append(r)
        tot += t
    v = float(np.mean(rates))
    line = {"impl": "reference", "metric": "gate_apps_per_s", "value": v, "unit": "gate-apps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * GATE_APPS / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": WORKLOAD, "N": N_QUBITS, "dtype_reference": "complex128",
                       "sample": f"first {n_gates} gates of one Strang step at N=28 per step"},
            "cpu_baseline": {"value": v, "unit": "gate-apps/s", "cores": 1, "kind": "port", "cpu_model": cpu_model(),
                             "sample": f"{n_gates} of the 218 gate applications of one step at N=28, complex128, "
                                       "single thread (the reference's kernels are single-threaded per state)"},
            "e2e": {"value": v, "unit": "gate-apps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def _events(torch, stream):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return e0, e1


def default_geometry_record(S, local, N, gates, neel, tsteps, gate_apps, steps, peak):
    """The headline evolution on a second context whose plan keeps the default fused-pass
    geometry (tile 13, low bits 5; SMOQ_OPT_AUTOTUNE 2: the per-pass kernel variants are
    still tuned): gate-apps/s over `steps` evolutions and the per-pass HBM fraction, beside
    the geometry the autotuner chose for the headline (fewer passes, more gates each)."""
    import torch
    ctx = S.Context(local)
    try:
        ctx.set_option(S._lib.OPT_TILE_BITS_C64, 13)
        ctx.set_option(S._lib.OPT_LOW_BITS_C64, 5)
        ctx.set_option(S._lib.OPT_AUTOTUNE, 2)
        plan = S.TrotterPlan(ctx, N, gates, order=2, dtype=S.C64)
        st = S.CuState(ctx, N, S.C64, basis=None)
        stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))

        def step():
            st.set_basis(neel)
            return plan.run(st, tsteps, RECORD_EVERY)
        for _ in range(2):
            step()
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        ctx.set_option(S._lib.OPT_USE_GRAPHS, 0)
        ctx.set_option(S._lib.OPT_KERNEL_TIMING, 1)
        ctx.reset_counters()
        step()
        ctx.synchronize()
        kc = ctx.counters()
        avg_ms = kc["tile_ms"] / max(1, kc["tile_passes"])
        achieved = kc["tile_bytes"] / max(1, kc["tile_passes"]) / (avg_ms * 1e-3) / 1e9
        st.close()
        plan.close()
        return {"tile_bits_c64": 13, "low_bits_c64": 5, "autotune": "variants only",
                "value": gate_apps * steps / (ms * 1e-3), "unit": "gate-apps/s", "ms_per_step": ms / steps,
                "tile_passes_per_step": kc["tile_passes"], "avg_launch_ms": avg_ms,
                "roofline_achieved_gbs": achieved, "roofline_frac": achieved / peak}
    finally:
        ctx.close()


def vqe_measure(ctx, steps, warmup, B=8):
    """VQE gradient throughput on the gradient configuration: TFIM N=24, 12 layers of
    [Ry all; Rz all; CZ ladder] (852 gates, 576 parameters).  Batched complex64
    adjoint gradients (B parameter sets per call) against the complex128 adjoint
    and the plain complex128 path (one kernel per gate, one reduction per
    Hamiltonian term, parameter-shift gradient: 2 x 576 energies per gradient);
    the plain path is timed on one parameter's two shifted energies and scaled to
    576 parameters.  Energy error: complex64 against complex128 of the same
    parameters."""
    import torch
    import pysmoq as S
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", torch.cuda.current_device()))
    N, L = 24, 12
    ops, idx = [], 1
    for _ in range(L):
        rot, idx = S.single_qubit_rotation_layer(N, idx, gates=("ry", "rz"))
        ops += rot + S.entangling_layer(N, "chain", "cz")
    circ = S.ParameterizedCircuit(N, ops)
    P = circ.n_params
    thetas = np.random.default_rng(SEED).uniform(0, 2 * np.pi, size=(B, P))
    H = S.PauliSum.tfim(N)
    res = {}
    for name, dt in (("c64", S.C64), ("c128", S.C128)):
        for _ in range(max(1, warmup)):
            S.energy_and_gradient(ctx, circ, H, thetas[:1], dtype=dt)
        e0, e1 = _events(torch, stream)
        e0.record(stream)
        for _ in range(steps):
            E, G = S.energy_and_gradient(ctx, circ, H, thetas, dtype=dt)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        res[name] = (B * steps / (ms * 1e-3), E, G)

    def plain_energy(theta):
        st = S.CuState(ctx, N, S.C128, basis=0)
        S.apply_circuit(st, circ, theta, fused=False)
        e = -sum(S.expect_corr(st, i, i + 1, N, "zz") for i in range(1, N)) - \
            sum(S.expect_local(st, i, N, "x") for i in range(1, N + 1))
        st.close()
        return e

    plain_energy(thetas[0])
    e0, e1 = _events(torch, stream)
    e0.record(stream)
    th = thetas[0].copy()
    th[0] += np.pi / 2
    ep = plain_energy(th)
    th[0] -= np.pi
    em = plain_energy(th)
    e1.record(stream)
    e1.synchronize()
    pair_ms = e0.elapsed_time(e1)
    plain_gps = 1.0 / (P * pair_ms * 1e-3)
    ps0 = (ep - em) / 2
    return {"workload": "vqe_tfim_n24_hea12_576params", "N": N, "layers": L, "params": P, "gates": len(ops),
            "batch": B, "calls": steps, "gradient": "adjoint",
            "c64_adjoint_gradients_per_s": res["c64"][0],
            "c128_adjoint_gradients_per_s": res["c128"][0],
            "plain_c128_ps_gradients_per_s": plain_gps,
            "plain_c128_sample": "two shifted energies of one parameter, one kernel per gate and one reduction per "
                                 "term; scaled to 576 parameters",
            "speedup_c64_adjoint_vs_plain_c128_ps": res["c64"][0] / plain_gps,
            "speedup_c64_adjoint_vs_c128_adjoint": res["c64"][0] / res["c128"][0],
            "energy_abs_err_c64_vs_c128": float(np.max(np.abs(res["c64"][1] - res["c128"][1]))),
            "grad_max_abs_err_c64_vs_c128": float(np.max(np.abs(res["c64"][2] - res["c128"][2]))),
            "plain_ps_vs_adjoint_param0": float(abs(ps0 - res["c128"][2][0, 0]))}


# The reference's own expectation-value benchmark
# (SmoQ.jl_benchmarks/benchmark_expectation_values/bench_smoq.jl:17-37, 82-85): 4 brickwork
# layers [H on even qubits; Ry(ANGLES_RY[q]) on all; CNOT on (q, q+1) for odd q; S on odd
# qubits; Rx(ANGLES_RX[q]) on all; CZ on (q, q+1) for even q] from |0...0>, then <X>, <Y>, <Z>
# of every qubit and <XX>, <YY>, <ZZ> of every bond, complex128.  Its published wall times
# (timing_smoq.txt:10-14, a laptop, single-threaded kernels).
PUBLISHED_EXPECTATION_S = {20: 0.483826, 24: 11.048547}
_ANG_RY = [np.pi / d for d in (4, 3, 6, 5, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26)]
_ANG_RX = [np.pi / d for d in (5, 7, 4, 9, 3, 11, 6, 13, 8, 10, 12, 14, 15, 17, 16, 19, 18, 20, 21, 22, 23, 24, 25, 26)]


def published_comparison(ctx, runs=5):
    """the reference's expectation benchmark at N=20 and N=24 on the GPU, CUDA events around
    circuit + 6N-3 observables (the observables come back to the host inside the region);
    against the reference's own published seconds"""
    import torch
    import pysmoq as S
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", torch.cuda.current_device()))
    out = {}
    for N, ref_s in PUBLISHED_EXPECTATION_S.items():
        g = S.gate
        ops = []
        for _ in range(4):
            ops += [g("h", q) for q in range(2, N + 1, 2)]
            ops += [g("ry", q, angle=_ANG_RY[q - 1]) for q in range(1, N + 1)]
            ops += [g("cnot", [q, q + 1]) for q in range(1, N, 2)]
            ops += [g("s", q) for q in range(1, N + 1, 2)]
            ops += [g("rx", q, angle=_ANG_RX[q - 1]) for q in range(1, N + 1)]
            ops += [g("cz", [q, q + 1]) for q in range(2, N, 2)]
        circ = S.ParameterizedCircuit(N, ops)
        st = S.CuState(ctx, N, S.C128, basis=0)
        times = []
        for r in range(runs + 1):
            e0, e1 = _events(torch, stream)
            e0.record(stream)
            st.set_basis(0)
            S.apply_circuit(st, circ, np.zeros(1))
            obs = S.measure_all_observables_state_vector(st, N, 1)
            e1.record(stream)
            e1.synchronize()
            if r:  # the first run plans and warms up
                times.append(e0.elapsed_time(e1) * 1e-3)
        st.close()
        t = float(np.median(times))
        out[f"n{N}"] = {"gpu_s": t, "reference_published_s": ref_s, "speedup": ref_s / t, "gates": len(ops),
                        "observables": int(obs.size)}
    return {"workload": "reference expectation benchmark: 4 brickwork layers + all X/Y/Z and XX/YY/ZZ, complex128",
            "source": "SmoQ.jl_benchmarks/benchmark_expectation_values/timing_smoq.txt:10-14 (laptop)",
            "runs": out}


def vqe_workload(args):
    """the VQE gradient figures as their own line (see vqe_measure)"""
    import pysmoq as S
    ctx = S.Context(0)
    if args.engine >= 0:
        ctx.set_option(S._lib.OPT_ENGINE, args.engine)
    r = vqe_measure(ctx, args.steps, args.warmup)
    line = {"metric": "vqe_gradients_per_s", "value": r["c64_adjoint_gradients_per_s"], "unit": "gradients/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * r["batch"] / r["c64_adjoint_gradients_per_s"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {k: r[k] for k in ("workload", "N", "layers", "params", "gates", "batch", "gradient")}}
    line.update({k: v for k, v in r.items() if k not in line["config"]})
    print(json.dumps(line))
    ctx.close()
    return 0


def lib_trotter_gates(S, N, bonds, fields, dt):
    """the library's closed-form Trotter gates (smoq_precompute_trotter_gates) of bonds
    (i, j, Jxx, Jyy, Jzz) and fields (idx, hx, hy, hz), 1-based sites"""
    params = S.HamiltonianParams(N, [S.CouplingTerm(*b) for b in bonds], [],
                                 [S.FieldTerm(*f) for f in fields])
    return S.precompute_trotter_gates_bitwise(params, dt)


def vqe_jobs_workload(args):
    print(json.dumps(vqe_jobs_line(args)))
    return 0


def vqe_jobs_line(args):
    """Batched uneven circuits: 256 circuits, N ~ U{10..20}, depth ~ U{4..16} layers of
    [Ry all; Rz all; CZ ladder] (seeded), TFIM H = -sum ZZ - sum X each, one energy +
    adjoint gradient per circuit, through smoq_energy_grad_jobs.  metric =
    full gradients per second (one gradient = all of one circuit's parameters).
    The jobs run in order on the library stream."""
    import torch
    import pysmoq as S
    ctx = S.Context(0)
    rng = np.random.default_rng(SEED)
    jobs, nparams = [], 0
    for _ in range(256):
        N = int(rng.integers(10, 21))
        L = int(rng.integers(4, 17))
        ops, idx = [], 1
        for _ in range(L):
            rot, idx = S.single_qubit_rotation_layer(N, idx, gates=("ry", "rz"))
            ops += rot + S.entangling_layer(N, "chain", "cz")
        circ = S.ParameterizedCircuit(N, ops)
        theta = rng.uniform(0, 2 * np.pi, size=circ.n_params)
        jobs.append((circ, S.PauliSum.tfim(N), theta))
        nparams += circ.n_params
    res = {}
    for name, dt in (("c64", S.C64), ("c128", S.C128)):
        for _ in range(max(1, args.warmup)):
            S.energy_and_gradient_jobs(ctx, jobs[:32], dtype=dt)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            E, G = S.energy_and_gradient_jobs(ctx, jobs, dtype=dt)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        res[name] = (len(jobs) * args.steps / sec, E, G, sec)
    err_e = float(np.max(np.abs(res["c64"][1] - res["c128"][1])))
    err_g = float(max(np.max(np.abs(a - b)) for a, b in zip(res["c64"][2], res["c128"][2])))
    line = {"metric": "vqe_gradients_per_s", "value": res["c64"][0], "unit": "gradients/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * res["c64"][3] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": "vqe_256_uneven_circuits_n10_20_depth4_16", "circuits": len(jobs),
                       "params_total": nparams, "gradient": "adjoint",
                       "timing": "host wall clock around the call (returns after all jobs synchronised)"},
            "c128_gradients_per_s": res["c128"][0],
            "param_gradients_per_s_c64": nparams * args.steps / res["c64"][3],
            "energy_abs_err_c64_vs_c128": err_e, "grad_max_abs_err_c64_vs_c128": err_g}
    ctx.close()
    return line
    return 0


def mcwf_workload(args):
    print(json.dumps(mcwf_line(args)))
    return 0


def mcwf_line(args):
    """Batched MCWF: TFIM N=16 (J = h = 1, first-order Trotter, 31 gates per step),
    jumps sqrt(0.1) sigma- and sqrt(0.05) sigma_z on every qubit, dt = 0.01, 500
    steps, 4096 trajectories from |0...0>, complex64 amplitudes with FP64 norms and
    sums, trajectory means of <Z_i> and <Z_i Z_{i+1}> every 10 steps.  metric =
    trajectory-steps per second.  CPU baseline: the oracle's quantum-jump rule
    (complex128, the reference's per-trajectory loops) on all host cores, timed on
    a trajectory subset."""
    import torch
    import pysmoq as S
    ctx = S.Context(0)
    if args.engine >= 0:
        ctx.set_option(S._lib.OPT_ENGINE, args.engine)
    N, dt, steps, B, rec = 16, 0.01, 500, 4096, 10
    bonds = [(i, i + 1, 0.0, 0.0, 1.0) for i in range(1, N)]
    fields = [(i, 1.0, 0.0, 0.0) for i in range(1, N + 1)]
    gates = lib_trotter_gates(S, N, bonds, fields, dt)
    jumps = [S.JumpOperator("sigma_minus", q, 0.1) for q in range(1, N + 1)] + \
            [S.JumpOperator("sigma_z", q, 0.05) for q in range(1, N + 1)]
    plan = S.TrotterPlan(ctx, N, gates, order=1, dtype=S.C64)
    st = S.CuState(ctx, N, S.C64, B, basis=0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    for w in range(max(1, args.warmup)):
        st.set_basis(0)
        S.mcwf_run(plan, st, jumps, dt, 1000 + w, 50, rec)
    e0, e1 = _events(torch, stream)
    e0.record(stream)
    for k in range(args.steps):
        st.set_basis(0)
        res = S.mcwf_run(plan, st, jumps, dt, 2026 + k, steps, rec)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    value = B * steps * args.steps / (ms * 1e-3)
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        arr, n = O.precompute_trotter_gates(bonds, fields, dt)
        ncpu = os.cpu_count() or 1
        ntr = 2 * ncpu
        oj = [(0, q, 0.1) for q in range(1, N + 1)] + [(2, q, 0.05) for q in range(1, N + 1)]
        t0 = time.perf_counter()
        O.mcwf_run(N, arr, n, O.make_jumps(oj), len(oj), dt, 7, 0, ntr, 20, 10, nthreads=ncpu)
        sec = time.perf_counter() - t0
        cpu = {"value": ntr * 20 / sec, "unit": "trajectory-steps/s", "cores": ncpu, "kind": "port",
               "sample": f"{ntr} trajectories x 20 steps of the same configuration, complex128, {sec:.1f} s"}
    line = {"metric": "mcwf_trajectory_steps_per_s", "value": value, "unit": "trajectory-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": "mcwf_tfim_n16_4096traj_500steps", "N": N, "trajectories": B, "dt": dt,
                       "trotter_steps": steps, "record_every": rec, "jump_ops": len(jumps),
                       "state_bytes": (1 << N) * 8 * B},
            "jumps_per_trajectory_mean": float(np.mean(res["jumps"])),
            "z_mean_final": float(np.mean(res["z_mean"][-1])),
            "reference_published": "N=16 1000 trajectories x 200 steps (dephasing only, dt 0.05) 397.29 s "
                                   "= 503 trajectory-steps/s on a laptop (output.log:449)",
            "cpu_baseline": cpu}
    st.close()
    plan.close()
    ctx.close()
    return line


def qrc_workload(args):
    print(json.dumps(qrc_line(args)))
    return 0


def qrc_line(args):
    """Quantum reservoir computing, the bitwise MCWF loop: two XXZ rails of L=6
    qubits (N=12; rail bonds Jxx = Jyy = 1, Jzz = 0.5; rungs 0.7, 0.7, 0.3; x field
    0.5 and seeded z fields), dt = 0.1, 5 Trotter steps per input, 100 seeded
    inputs in [0, 1] (:batch window, :traceout_rail_1 reset), 4096 trajectories,
    the 84 ladder features after every input.  metric = trajectory-inputs per
    second through smoq_qrc_run (host inputs in, host feature means out: the
    value is end to end).  CPU baseline: the oracle's restatement of the loop
    (complex128, trajectories over all host cores) on a trajectory subset."""
    import torch
    import pysmoq as S
    ctx = S.Context(0)
    L, T, B, sub, dt = 6, args.inputs, args.trajectories, 5, 0.1
    rng = np.random.default_rng(2026)
    bonds = [(r * L + s + 1, r * L + s + 2, 1.0, 1.0, 0.5) for r in range(2) for s in range(L - 1)]
    bonds += [(s + 1, L + s + 1, 0.7, 0.7, 0.3) for s in range(L)]
    fields = [(q + 1, 0.5, 0.0, float(rng.uniform(-1, 1))) for q in range(2 * L)]
    gates = lib_trotter_gates(S, 2 * L, bonds, fields, dt)
    u = rng.uniform(0, 1, T)
    padded = np.concatenate([np.zeros(L), u])
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    res = {}
    for name, dt_ in (("c64", S.C64), ("c128", S.C128)):
        plan = S.TrotterPlan(ctx, 2 * L, gates, order=1, dtype=dt_)
        for w in range(max(1, args.warmup)):
            S.run_mcwf_simulation(None, None, plan, padded, L, 2, T, 256, n_substeps=sub, seed=100 + w)
        e0, e1 = _events(torch, stream)
        walls = []
        e0.record(stream)
        for k in range(args.steps):
            t0 = time.perf_counter()
            X = S.run_mcwf_simulation(None, None, plan, padded, L, 2, T, B, n_substeps=sub, seed=2026 + k)
            walls.append(time.perf_counter() - t0)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        res[name] = (B * T * args.steps / (ms * 1e-3), ms / args.steps, B * T * args.steps / sum(walls), X,
                     [round(w * 1e3, 1) for w in walls])
        plan.close()
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        arr, n = O.precompute_trotter_gates(bonds, fields, dt)
        ncpu = os.cpu_count() or 1
        ntr, ti = 4 * ncpu, min(20, T)
        t0 = time.perf_counter()
        O.qrc_run(L, arr, n, u[:ti], ntr, n_substeps=sub, seed=7, nthreads=ncpu)
        sec = time.perf_counter() - t0
        cpu = {"value": ntr * ti / sec, "unit": "trajectory-inputs/s", "cores": ncpu, "kind": "port",
               "sample": f"{ntr} trajectories x {ti} inputs of the same configuration, complex128, {sec:.1f} s"}
    X64, X128 = res["c64"][3], res["c128"][3]
    line = {"metric": "qrc_trajectory_inputs_per_s", "value": res["c64"][0], "unit": "trajectory-inputs/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["c64"][1],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": f"qrc_xxz_ladder_L6_{B}traj_{T}inputs", "L": L, "N": 2 * L, "trajectories": B,
                       "inputs": T, "n_substeps": sub, "features": S.qrc_n_ops(L), "encoding": "batch",
                       "reset": "traceout_rail_1", "state_bytes_per_trajectory": (1 << (2 * L)) * 8},
            "e2e": {"value": res["c64"][2], "unit": "trajectory-inputs/s",
                    "h2d_bytes_per_step": int(padded.nbytes), "d2h_bytes_per_step": int(X64.nbytes)},
            "e2e_ms_per_call": res["c64"][4],
            "c128_trajectory_inputs_per_s": res["c128"][0],
            "feature_mean_abs_diff_c64_vs_c128": float(np.mean(np.abs(X64 - X128))),
            "gpu_launches": args.steps, "cpu_baseline": cpu}
    ctx.close()
    return line


def _op_fp32_per_amp(o):
    """FP32 FMA-pipe instructions per amplitude of one fused op, from its matrix: per
    output amplitude each nonzero coefficient costs 4 (general complex), 2 (real or
    imaginary) or 0 (+-1, +-i: a copy or a swap of parts)"""
    c, k, nq = o["c"], o["kind"], o["nq"]
    dim = 1 << nq
    if k in (5, 6):                       # per-state scale, real byte tables: 2 real multiplies
        return 2.0
    M = np.zeros((dim, dim), complex)
    if k == 0:
        M = c[:4].reshape(2, 2)
    elif k == 1:
        M = c[:16].reshape(4, 4)
    elif k == 2:
        M[0, 0], M[0, 3], M[3, 0], M[3, 3] = c[0], c[1], c[2], c[3]
        M[1, 1], M[1, 2], M[2, 1], M[2, 2] = c[4], c[5], c[6], c[7]
    elif k == 3:
        for r in range(dim):
            M[r, o["perm"][r]] = c[r]
    elif k == 4:
        M = np.diag(c[:dim])
    else:
        return 0.0

    def cost(z):
        if z == 0:
            return 0
        if (z.imag == 0 and abs(z.real) == 1) or (z.real == 0 and abs(z.imag) == 1):
            return 0
        return 2 if (z.imag == 0 or z.real == 0) else 4
    return sum(cost(z) for z in M.reshape(-1)) / dim


def plan_fp32_per_amp(S, N, ops, dtype, engine):
    """sum over the planned passes of the FP32 instructions per amplitude (host planner;
    for engine 3 an upper bound: the compiled kernels fold the stage diagonals)"""
    tb, lb = (13, 5) if dtype == S.C64 else (12, 4)
    plan = S.debug_plan(N, ops, dtype=dtype, tile_bits=tb, low_bits=lb, engine=max(0, engine))
    return sum(_op_fp32_per_amp(o) for p in plan for o in p["ops"]), len(plan)


def bandwidth_workload(args):
    """32 GiB single-state sweeps: N=32 complex64 and N=31 complex128, 20 layers of
    [Rx, Ry, Rz on every qubit (seeded angles); Rzz on a seeded random perfect
    matching], fused passes; every pass timed with CUDA events.  Reported against
    the HBM roofline (2 state sizes per pass) and the FP32 roofline (the planned
    ops' FMA-pipe instructions per amplitude; 148 SMs x 128 lanes x the clock)."""
    import time as _t
    import torch
    import pysmoq as S
    peak, peak_kind = measured_peak()
    sm_mhz = 1965.0
    fp32_peak = 148 * 128 * sm_mhz * 1e6  # FMA-pipe instructions / s
    out = {}
    for N, dt, name in ((32, S.C64, "n32_c64"), (31, S.C128, "n31_c128")):
        rng = np.random.default_rng(SEED)
        ops = []
        for _ in range(20):
            for g in ("rx", "ry", "rz"):
                ops += [S.gate(g, q, angle=float(rng.uniform(0, 2 * np.pi))) for q in range(1, N + 1)]
            perm = rng.permutation(N) + 1
            ops += [S.gate("rzz", [int(perm[2 * i]), int(perm[2 * i + 1])], angle=float(rng.uniform(0, 2 * np.pi)))
                    for i in range(N // 2)]
        circ = S.ParameterizedCircuit(N, ops)
        engines = [args.engine] if args.engine >= 0 else ([-1, 3] if dt == S.C64 and S.jit_available() else [-1])
        for eng in engines:
            ctx = S.Context(0)
            if eng >= 0:
                ctx.set_option(S._lib.OPT_ENGINE, eng)
            st = S.CuState(ctx, N, dt, basis=0)
            t0 = _t.perf_counter()
            S.apply_circuit(st, circ, np.zeros(1))  # first call: plans (and compiles, engine 3), first touch
            first_s = _t.perf_counter() - t0
            ctx.set_option(S._lib.OPT_KERNEL_TIMING, 1)
            ctx.reset_counters()
            st.set_basis(0)
            S.apply_circuit(st, circ, np.zeros(1))
            c = ctx.counters()
            ctx.set_option(S._lib.OPT_KERNEL_TIMING, 0)
            masks = [1 << q for q in range(N)] + [3 << q for q in range(N - 1)]
            obs = S.expect_zstrings(st, masks[:32])
            gbs = c["tile_bytes"] / (c["tile_ms"] * 1e-3) / 1e9
            eng_run = eng if eng >= 0 else 0   # one-shot sequences: auto = shared-memory sweeps
            instr, npass = plan_fp32_per_amp(S, N, ops, dt, eng_run)
            fp32_rate = instr * float(1 << N) / (c["tile_ms"] * 1e-3)
            out[f"{name}_engine{eng_run}"] = {
                "gates": len(ops), "passes": c["tile_passes"], "ms": c["tile_ms"], "first_call_s": first_s,
                "gate_apps_per_s": len(ops) / (c["tile_ms"] * 1e-3), "hbm_gbs": gbs, "hbm_frac": gbs / peak,
                "fp32_instr_per_amp": instr, "fp32_frac": fp32_rate / fp32_peak,
                "norm": float(S.get_norm(st)), "z1": float(obs[0, 0])}
            st.close()
            ctx.close()
    head = out.get("n32_c64_engine0") or next(iter(out.values()))
    line = {"metric": "hbm_gbs_per_sweep", "value": head["hbm_gbs"], "unit": "GB/s", "n_gpus": 1,
            "steps": 1, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64", "data": "synthetic",
            "config": {"workload": "random_rxryrz_rzz_depth20_32GiB", "engine": args.engine},
            "peak": peak, "peak_kind": peak_kind, "fp32_peak_instr_per_s": fp32_peak, "runs": out}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-vqe", action="store_true", help="skip the VQE gradient sub-record of the default line")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the short C4b / MCWF / QRC sub-records of the default line")
    ap.add_argument("--autotune", type=int, default=-1,
                    help="compiled pass kernels: per-pass variant tuning (-1 library default = on, 0 off, 1 on)")
    # smaller cases of the same kernel (profiling, sweeps); the defaults are the workload
    ap.add_argument("--n-qubits", type=int, default=N_QUBITS)
    ap.add_argument("--trotter-steps", type=int, default=STEPS)
    ap.add_argument("--tile-bits", type=int, default=0, help="complex64 tile width (0 = library default)")
    ap.add_argument("--low-bits", type=int, default=0, help="complex64 contiguous low qubits per tile segment (0 = default)")
    ap.add_argument("--engine", type=int, default=-1, help="fused-pass engine (-1 = library default)")
    ap.add_argument("--jit-buffers", type=int, default=1, help="compiled pass kernels: tile buffers per CTA (1, 2)")
    ap.add_argument("--jit-groups", type=int, default=2, help="compiled pass kernels: register groups per thread (1, 2)")
    ap.add_argument("--trajectories", type=int, default=4096, help="qrc workload: trajectories")
    ap.add_argument("--inputs", type=int, default=100, help="qrc workload: length of the input series")
    ap.add_argument("--workload", default="trotter", choices=["trotter", "vqe", "vqe_jobs", "mcwf", "bandwidth", "qrc"],
                    help="trotter: the headline line; vqe / bandwidth: the gradient and 32 GiB sweep figures")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "vqe":
        return vqe_workload(args)
    if args.workload == "bandwidth":
        return bandwidth_workload(args)
    if args.workload == "vqe_jobs":
        return vqe_jobs_workload(args)
    if args.workload == "mcwf":
        return mcwf_workload(args)
    if args.workload == "qrc":
        return qrc_workload(args)

    ws, rank, local = dist_env()
    import torch
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    import build as _b
    if rank == 0 and not os.path.exists(_b.LIB):
        _b.build_cuda()
    if ws > 1:
        dist.barrier()
    import pysmoq as S

    ctx = S.Context(local)
    eng = resolve_engine(S, args.engine)
    if args.tile_bits:
        ctx.set_option(S._lib.OPT_TILE_BITS_C64, args.tile_bits)
    if args.low_bits:
        ctx.set_option(S._lib.OPT_LOW_BITS_C64, args.low_bits)
    if args.engine >= 0:
        ctx.set_option(S._lib.OPT_ENGINE, args.engine)
    if args.jit_buffers != 1:
        ctx.set_option(S._lib.OPT_JIT_BUFFERS, args.jit_buffers)
    if args.jit_groups != 2:
        ctx.set_option(S._lib.OPT_JIT_GROUPS, args.jit_groups)
    if args.autotune >= 0:
        ctx.set_option(S._lib.OPT_AUTOTUNE, args.autotune)
    N = args.n_qubits
    tsteps = args.trotter_steps
    gate_apps = tsteps * 2 * (N + 3 * (N - 1))
    workload = WORKLOAD if (N, tsteps) == (N_QUBITS, 200) else f"xxz_chain_trotter2_n{N}_c64_{tsteps}steps"
    gl = s1_gates(N, DT / 2)
    gates = [S.FastTrotterGate(idx, U) for idx, U in gl]
    plan = S.TrotterPlan(ctx, N, gates, order=2, dtype=S.C64)
    st = S.CuState(ctx, N, S.C64, basis=None)
    neel = neel_index(N)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))

    def device_step():
        st.set_basis(neel)                      # make_initial_psi on the device
        return plan.run(st, tsteps, RECORD_EVERY)

    # e2e input: the initial state in pinned host memory (what a caller holding
    # psi on the host passes), uploaded every step; output: the <Z> records.
    host_psi = torch.zeros(1 << N, dtype=torch.complex64, pin_memory=True)
    host_psi[neel] = 1.0
    hp = host_psi.numpy()

    def e2e_step():
        S.lib.smoq_state_upload(st.h, hp.ctypes.data_as(S._lib.C.c_void_p), hp.nbytes)
        return plan.run(st, tsteps, RECORD_EVERY)

    def timed(fn, k):
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize(local)
        ctx.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        e1.synchronize()
        ctx.synchronize()
        ms = e0.elapsed_time(e1)
        if ws > 1:
            ms = max_over_ranks(ms, dist, f"cuda:{local}")
        return ms

    for _ in range(args.warmup):
        rec = device_step()
    tune = ctx.tune_report()
    if tune:
        sys.stderr.write(tune)
    # the plan's fused-pass geometry: the autotuner's choice, else the options
    geom = (args.tile_bits or 13, args.low_bits or 5, None)
    for line in tune.splitlines():
        if line.startswith("-> geometry tile"):
            w = line.split()
            geom = (int(w[3]), int(w[5]), None if w[7] == "-1" else int(w[7]))
    ctx.reset_counters()
    clocks = Clocks(local)
    clocks.start()
    ms = timed(device_step, args.steps)
    clk = clocks.stop()
    launches = ctx.counters()["launches"]
    rec = device_step()
    # sanity of the result: the Neel state's <Z> at t=0 and bounded magnetisation after
    assert np.allclose(rec[0, 0, :], [(-1.0 if (neel >> k) & 1 else 1.0) for k in range(N)], atol=1e-6)
    assert np.all(np.abs(rec) <= 1 + 1e-5)

    # roofline of the dominant kernel: the fused tile pass, timed per launch with
    # CUDA events on the library's stream (graphs off so every launch is bracketed)
    for _ in range(1):
        e2e_step()
    ctx.set_option(S._lib.OPT_USE_GRAPHS, 0)
    ctx.set_option(S._lib.OPT_KERNEL_TIMING, 1)
    ctx.reset_counters()
    timed(device_step, 1)
    kc = ctx.counters()
    ctx.set_option(S._lib.OPT_KERNEL_TIMING, 0)
    ctx.set_option(S._lib.OPT_USE_GRAPHS, 1)
    passes = kc["tile_passes"]
    avg_ms = kc["tile_ms"] / max(1, passes)
    bytes_per_launch = kc["tile_bytes"] / max(1, passes)
    achieved = bytes_per_launch / (avg_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()

    # e2e through the C ABI with host buffers
    e2e_ms = timed(e2e_step, args.steps)

    # the same evolution with the default geometry, when the autotuner chose another
    default_geom = None
    if rank == 0 and ws == 1 and not args.tile_bits and not args.low_bits and args.autotune != 0 \
            and geom != (13, 5, None):
        try:
            default_geom = default_geometry_record(S, local, N, gates, neel, tsteps, gate_apps, args.steps, peak)
        except Exception as ex:  # a sub-record never costs the headline line
            default_geom = {"error": f"{type(ex).__name__}: {ex}"}

    per_rank_apps = gate_apps * args.steps
    value = whole_job_rate(per_rank_apps, ws, ms)
    e2e_value = whole_job_rate(per_rank_apps, ws, e2e_ms)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and N == N_QUBITS:
        r, t = cpu_baseline_sample(12)
        cpu = {"value": r, "unit": "gate-apps/s", "cores": 1, "kind": "port",
               "sample": f"first 12 of the 218 gate applications of one Strang step at N=28, complex128, "
                         f"single thread, {t:.1f} s (oracle restating the reference's loops)",
               "cpu_model": cpu_model()}

    # the gradient figures of the metric's second half (VQE gradients/s, complex64
    # adjoint against the plain complex128 path, energy error), every rank
    vqe = None
    if not args.no_vqe and N == N_QUBITS:
        try:  # (no collectives inside: a rank that fails here fails alone)
            vqe = vqe_measure(ctx, steps=2, warmup=1)
        except Exception as ex:  # a sub-record never costs the headline line
            vqe = {"error": f"{type(ex).__name__}: {ex}"}
    published = None
    if not args.no_vqe and N == N_QUBITS and rank == 0:
        try:
            published = published_comparison(ctx)
        except Exception as ex:
            published = {"error": f"{type(ex).__name__}: {ex}"}
    # short runs of the other workloads (one timed step each, no CPU baselines), so the
    # default line carries their figures too; the full runs are --workload vqe_jobs,
    # mcwf and qrc
    extras = None
    if rank == 0 and ws == 1 and not args.no_extras and N == N_QUBITS:
        extras = {}
        sub = argparse.Namespace(steps=1, warmup=1, engine=-1, no_cpu_baseline=True, trajectories=4096,
                                 inputs=100)
        keep = ("metric", "value", "unit", "ms_per_step", "c128_gradients_per_s", "energy_abs_err_c64_vs_c128",
                "c128_trajectory_inputs_per_s", "e2e", "jumps_per_trajectory_mean")
        for name, fn in (("vqe_jobs", vqe_jobs_line), ("mcwf", mcwf_line), ("qrc", qrc_line)):
            try:
                r = fn(sub)
                extras[name] = {k: r[k] for k in keep if k in r}
                extras[name]["workload"] = r["config"]["workload"]
            except Exception as ex:  # a sub-record never costs the headline line
                extras[name] = {"error": f"{type(ex).__name__}: {ex}"}

    if rank == 0:
        line = {"metric": "gate_apps_per_s", "value": value, "unit": "gate-apps/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
                "data": "synthetic",
                "config": {"workload": workload, "N": N, "dt": DT, "trotter_steps": tsteps,
                           "tile_bits_c64": geom[0], "low_bits_c64": geom[1], "fusion_depth": geom[2],
                           "engine": eng,
                           "record_every": RECORD_EVERY, "gate_apps_per_step": gate_apps,
                           "state_bytes": (1 << N) * 8, "l2_policy": "inputs larger than L2 (2 GiB state)",
                           "parallelism": "replicas" if ws > 1 else "single_gpu",
                           "autotune": args.autotune != 0,
                           "tuned_variants": {v: tune.count("-> " + v) for v in ("v0", "v1", "v2", "v3", "v4", "v5")
                                              if tune.count("-> " + v)},
                           "tile_passes_per_step": passes, "hbm_gbs_effective":
                               2.0 * (1 << N) * 8 * passes / (ms / args.steps * 1e-3) / 1e9},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": ncu_traffic(eng), "peak_kind": peak_kind,
                             "kernel": ENGINE_KERNELS[eng][0], "avg_launch_ms": avg_ms,
                             "algorithmic_bytes_per_launch": bytes_per_launch,
                             # per pass launch: with the autotuner's geometry a pass may carry
                             # more gates (fewer passes per evolution); the same kernels' fraction
                             # at the default geometry, measured in this run, sits beside it
                             "geometry": f"tile {geom[0]}, low bits {geom[1]}",
                             "default_geometry_frac": (default_geom or {}).get("roofline_frac")},
                "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": "gate-apps/s", "h2d_bytes_per_step": int(hp.nbytes),
                        "d2h_bytes_per_step": int(8 * N * (tsteps // RECORD_EVERY + 1))},
                "gpu_launches": int(launches),
                "clocks": clk,
                "default_geometry": default_geom,
                "vqe": vqe,
                "published_comparison": published,
                "other_workloads": extras}
        print(json.dumps(line))
    st.close()
    plan.close()
    ctx.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
