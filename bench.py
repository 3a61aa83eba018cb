"""Benchmark: energy + gradient evaluations per second of the variational
hot path at n = 3 (two heavy particles + two electrons, four Y^+Y terms),
K = 4000 seeded synthetic ECGs, FP64, one GPU per rank.

One step = one EnergyIB evaluation through the fused adjoint pass: all
K(K+1)/2 pair elements of H and S, the LDL^H factorisation of H - lambda~ S,
inverse iteration to the lowest root (EIGVAL_TOLERANCE 1e-12, warm-started
from the previous step's eigenvector as Glob_LastEigvector is), and the
gradient with respect to all K * 12 nonlinear parameters.  Between steps the
parameters move by a seeded relative perturbation of 1e-6, as an optimiser's
steps move them, so every step is a new evaluation.  `value` times that with
the parameters already on the device; `e2e` adds, every step, the
host->device copy of the parameters (pinned host memory) and the
device->host copy of the gradient.  The plain drop-in (derivatives
materialised in Glob_D, then contracted) is timed beside it.  Before timing,
the energy of the unperturbed basis is checked against the oracle's value
stored in tests/golden/bench_k4000.json (which also holds lambda~).

--impl reference times the CPU restatement of the reference (the oracle:
OpenMP over pairs, LDLHF's parallel branch with the threads as ranks, all
host threads) on the same steps: one full, unscaled EnergyIB per step.

Multi-GPU: every rank evaluates its own replica (independent bases, no
collective on the data path); value = total evaluations / max-over-ranks
time.
"""
import argparse
import json
import os
import platform
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "atom-mol-nonbo_b200"))

METRIC = "energy+gradient evals/s at n=3,K=4000 (adjoint vs plain GPU); ECG pairs/s"
CONFIG_INDEX = 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--K", type=int, default=None, help="override the basis size (testing only)")
    ap.add_argument("--tol", type=float, default=1e-12,
                    help="GHEPIIS tolerance (EIGVAL_TOLERANCE); negative: iterate until the residual stops "
                         "decreasing, once below |tol| (src/linalg.f90:1900-1906)")
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--cpu-baseline", type=int, default=1)
    ap.add_argument("--candidates", type=int, default=1, help="also time the batched-candidate configuration")
    ap.add_argument("--large", type=int, default=1, help="also run the K=10000 step (Li-like n=3 and five-particle n=4)")
    ap.add_argument("--large-K", type=int, default=10000)
    ap.add_argument("--composite", type=int, default=1,
                    help="also time one new function's energy + gradient at K: plain, adjoint, batched")
    ap.add_argument("--cand-K", type=int, default=2000)
    ap.add_argument("--expc", type=int, default=1, help="also time the expectation-value pass")
    ap.add_argument("--expc-K", type=int, default=4000)
    ap.add_argument("--only-expc", type=int, default=0, help="time only the expectation-value pass (profiling)")
    ap.add_argument("--lam", type=float, default=None,
                    help="use this lambda~ instead of the stored one or a search (profiling runs)")
    ap.add_argument("--factor-mode", type=int, default=0,
                    help="whole-matrix LDL^H: 0 persistent tile kernel (default), 1 one launch per panel step")
    ap.add_argument("--ref-max-iter", type=int, default=None,
                    help="MaxIter of the reference arm's GHEPIIS (default 20, the reference's)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
class Dist:
    """torch.distributed for the barrier and the max-over-ranks time only."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as td
            td.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.td = td

    def barrier(self):
        if self.world > 1:
            self.td.barrier()

    def max(self, x):
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.td.destroy_process_group()


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        # the raw samples go to ECG_BENCH_CLOCKS_DIR when it is set, else to a temporary file
        out = os.environ.get("ECG_BENCH_CLOCKS_DIR")
        if out:
            self.path = os.path.join(out, f"clocks_rank{device}.csv")
        else:
            import tempfile
            self.path = os.path.join(tempfile.gettempdir(), f"ecg_bench_clocks_{os.getpid()}_{device}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def setup_problem(K, rank):
    from ecg_b200 import synth
    sysm, params = synth.config_basis(CONFIG_INDEX, K=K)
    if rank:  # independent replica per rank
        cfg = synth.CONFIGS[CONFIG_INDEX]
        params = synth.random_basis(sysm.n, K, cfg["seed"] + 7919 * rank)
    return sysm, params, synth.SYSTEMS[synth.CONFIGS[CONFIG_INDEX]["system"]]["e_floor"]


# lambda~ = CURRENT_ENERGY * INVITPARAMETER (src/main.f90:52), with the
# INVITPARAMETER of the reference's example inputs (1.000001).
INVIT_PARAMETER = 1.000001
# Parameter sets the steps cycle through: relative perturbations of 1e-6 of
# every parameter (seeded), the size of a late optimiser step.
NSETS, PERTURB, PERTURB_SEED = 8, 1e-6, 2002
TOL_E = 1e-10


def load_fixture(K):
    """The stored oracle energy and lambda~ of the workload at this K."""
    path = os.path.join(ROOT, "tests", "golden", f"bench_k{K}.json")
    return json.load(open(path)) if os.path.exists(path) else None


def perturbed_sets(params, rank=0):
    rng = np.random.default_rng(PERTURB_SEED + 7919 * rank)
    return [np.ascontiguousarray(params * (1.0 + PERTURB * rng.uniform(-1.0, 1.0, params.shape)))
            for _ in range(NSETS)]


def find_shift(ctx, K, e_floor):
    """lambda~ for the benchmark: converge to the lowest root from a lower
    bound of the spectrum (the current energy of an optimisation), then
    lambda~ = E * INVITPARAMETER."""
    ctx.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
    E, err, it = ctx.energy_ia(1, K, e_floor, -1e-12, max_iter=200, specif_norm=0)
    E2, err2, it2 = ctx.energy_ia(1, K, E * INVIT_PARAMETER, -1e-12, max_iter=50, specif_norm=0)
    return E2 * INVIT_PARAMETER, E2


def flush_l2(buf):
    """Write a buffer larger than L2 on the default device (torch)."""
    if buf is not None:
        buf.add_(1.0)


def run_ours(args, dist):
    import ctypes as C

    import torch

    from ecg_b200 import Context, probe_fp64_peak, probe_fp64_tensor_peak
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import opcount

    dev = dist.local
    torch.cuda.set_device(dev)
    K = args.K or 4000
    sysm, params, e_floor = setup_problem(K, dist.rank)
    T = sysm.T
    pairs = K * (K + 1) // 2
    fx = load_fixture(K) if dist.rank == 0 else None
    ctx = Context(sysm, K, max_nfo=K if args.plain_steps > 0 else 0, device=dev)
    ctx.set_factor_mode(args.factor_mode)
    ctx.set_params(params)
    if args.lam is not None:
        lam = args.lam
    elif fx is not None:
        lam = fx["lambda_tilde"]
    else:
        lam, _ = find_shift(ctx, K, e_floor)
    ones = np.ones(K, dtype=np.complex128)
    # ---- the energy of the unperturbed basis against the stored oracle value
    check = None
    if fx is not None and args.lam is None:
        ctx.set_vectors(K, last_eigvec=ones)
        Ec, errc, itc = ctx.energy_ia(1, K, lam, 1e-12, specif_norm=0)
        check = {"energy_gpu": Ec, "energy_oracle": fx["energy_oracle"], "abs_diff": abs(Ec - fx["energy_oracle"]),
                 "tol": TOL_E, "error_code": int(errc), "iterations": int(itc),
                 "source": "tests/golden/bench_k4000.json (oracle EnergyIAM, start vector of ones)"}
        assert abs(Ec - fx["energy_oracle"]) <= TOL_E, check
    ctx.set_vectors(K, last_eigvec=ones)
    sets = perturbed_sets(params, dist.rank)
    sets_dev = [torch.from_numpy(p.ravel()).to(f"cuda:{dev}") for p in sets]
    l2buf = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")  # 256 MB > L2

    def one(step, adjoint=True, want_grad=False):
        ctx.set_params_device(sets_dev[step % NSETS].data_ptr(), 1, K)
        fn = ctx.energy_ib_adjoint if adjoint else ctx.energy_ib
        return fn(0, K, lam, args.tol, max_iter=20, want_grad=want_grad)

    # ---- device-resident timing --------------------------------------
    step = 0
    for _ in range(args.warmup):
        one(step)
        step += 1
    ctx.set_timing(True)
    clocks = ClockSampler(dev)
    clocks.start()
    launches0 = ctx.launch_count()
    stage = np.zeros(4)
    total_ms, iters, codes = 0.0, [], []
    dist.barrier()
    torch.cuda.synchronize()
    for _ in range(args.steps):
        flush_l2(l2buf)
        torch.cuda.synchronize()
        ctx.timer_start()
        E, _, err, it = one(step)
        total_ms += ctx.timer_stop()
        step += 1
        stage += ctx.stage_ms()
        iters.append(it)
        codes.append(err)
    torch.cuda.synchronize()
    dist.barrier()
    launches = ctx.launch_count() - launches0
    clk = clocks.stop()
    tuning = ctx.tuning()
    ms_step = dist.max(total_ms) / args.steps
    value = dist.sum(args.steps) / (dist.max(total_ms) / 1e3)

    # ---- end-to-end through the public API with host buffers ------------
    pins = []
    for p in sets:
        t = torch.empty(p.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = p
        pins.append(t)
    gpin = torch.empty(K * sysm.npt, dtype=torch.float64, pin_memory=True)
    g_np = gpin.numpy()
    h0, d0 = ctx.io_bytes()
    e2e_ms = 0.0
    dist.barrier()
    for _ in range(args.steps):
        flush_l2(l2buf)
        torch.cuda.synchronize()
        ctx.timer_start()
        ctx.set_params(pins[step % NSETS].numpy())
        e = C.c_double()
        it = C.c_int()
        st = ctx.lib.ecg_energy_ib_adjoint(ctx.h, 0, K, 1, lam, args.tol, 20, C.byref(e),
                                           g_np.ctypes.data_as(C.POINTER(C.c_double)), C.byref(it))
        e2e_ms += ctx.timer_stop()
        step += 1
        assert st >= 0
    h1, d1 = ctx.io_bytes()
    e2e_value = dist.sum(args.steps) / (dist.max(e2e_ms) / 1e3)

    # ---- plain drop-in beside it ---------------------------------------
    plain = None
    if args.plain_steps > 0:
        one(step, adjoint=False)
        step += 1
        pms = 0.0
        pstage = np.zeros(4)
        for _ in range(args.plain_steps):
            flush_l2(l2buf)
            torch.cuda.synchronize()
            ctx.timer_start()
            Ep, _, _, _ = one(step, adjoint=False)
            pms += ctx.timer_stop()
            step += 1
            pstage += ctx.stage_ms()
        pms = dist.max(pms) / args.plain_steps
        plain = {"value": dist.sum(1) / (pms / 1e3), "ms_per_step": pms, "E": Ep,
                 "stages_ms": dict(zip(["pairs_hs_and_derivs", "ldlh", "invit", "contract"],
                                       (pstage / args.plain_steps).round(4).tolist()))}

    # ---- rooflines: every stage, the dominant one as `roofline` -----------
    st = stage / args.steps
    names = ["pairs_hs", "ldlh", "invit", "adjoint"]
    peak_fma = probe_fp64_peak(dev)
    peak_tc = probe_fp64_tensor_peak(dev)
    counts = opcount.pair_counts(sysm.n, T)
    adj_flop = counts["adjoint"]["total"] * pairs
    hs_flop = counts["reference_energy"]["total"] * pairs
    ldl_flop = 4.0 / 3.0 * K ** 3
    invit_bytes = 32.0 * K * K * max(np.mean(iters), 1) + 32.0 * K * K  # iterations + the Rayleigh quotient
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"hbm_gbs": 6650.0, "fallback": True}
    traffic = {}
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath))
    fma_src = "measured in this run: register FMA loop over all SMs (MEASURED_PEAKS.json has no FP64 entry)"
    tc_src = ("measured in this run: register mma.sync.m8n8k4.f64 loop over all SMs "
              "(MEASURED_PEAKS.json has no FP64 entry)")
    hbm_src = "MEASURED_PEAKS.json hbm_gbs" + (" (fallback)" if peaks.get("fallback") else "")

    def roof(bound, work, ms, peak, unit, kern, src, tkey):
        ach = work / (ms * 1e-3) / (1e12 if unit == "TFLOP/s" else 1e9)
        return {"bound": bound, "achieved": ach, "peak": peak, "unit": unit, "frac": ach / peak,
                "traffic": traffic.get(tkey), "kernel": kern, "peak_source": src,
                "algorithmic": work, "algorithmic_unit": "flop" if unit == "TFLOP/s" else "byte"}

    stage_roof = {
        "pairs_hs": roof("fp64", hs_flop, st[0], peak_fma, "TFLOP/s",
                         "k_pair_energy<3> (+ k_pair_diag, k_prep): one launch per step", fma_src, "pairs_hs"),
        "ldlh": roof("tensor", ldl_flop, st[1], peak_tc, "TFLOP/s",
                     "LDL^H factorisation, one CUDA-graph launch per step: the persistent tile kernel "
                     "k_ldl_persist (trailing updates and panel rows on the FP64 tensor cores, the diagonal "
                     "chain on its own CTA) between k_ldl_mirror and k_ldl_linv + k_ldl_mn", tc_src, "ldlh"),
        "invit": roof("hbm", invit_bytes, st[2], peaks["hbm_gbs"], "GB/s",
                      "inverse iterations (k_hemv, k_fwd_coop, k_bwd_coop) + Rayleigh quotient", hbm_src, "invit"),
        "adjoint": roof("fp64", adj_flop, st[3], peak_fma, "TFLOP/s",
                        "k_adjoint<3> + k_adjoint_final<3>: one launch each per step", fma_src, "adjoint"),
    }
    dom_name = names[int(np.argmax(st))]
    roof_line = dict(stage_roof[dom_name])
    per_stage_tf = {k: round(v["achieved"], 3) for k, v in stage_roof.items() if v["unit"] == "TFLOP/s"}

    line = {
        "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": f"synthetic: seeded ECG basis (seed {1002}), two heavy particles + two electrons",
        "config": {"workload": f"EnergyIB (adjoint) n=3 K={K} T={T}: H,S + LDL^H + inverse iteration + gradient",
                   "K": K, "n": sysm.n, "T": T, "tol": args.tol, "max_iter": 20, "lambda_tilde": lam,
                   "invit_parameter": INVIT_PARAMETER,
                   "l2": "H,S are 2 x 256 MB (> 126 MB L2) and a 256 MB buffer is written between steps",
                   "parallelism": f"replicas x{dist.world}"},
        "pairs_per_s": pairs * value, "pair_terms_per_s": pairs * T * value,
        "energy": E, "energy_check": check, "invit_iters": float(np.mean(iters)),
        "invit_iters_per_step": [int(i) for i in iters], "error_codes": np.bincount(codes, minlength=3).tolist(),
        "steps_perturbation": f"{NSETS} parameter sets, relative perturbation {PERTURB:g} (seed {PERTURB_SEED}), "
                              "cycled; warm start from the previous step's eigenvector",
        "stages_ms": dict(zip(names, st.round(4).tolist())),
        "stage_tflops": per_stage_tf,
        "stage_rooflines": stage_roof,
        "plain_gpu": plain,
        "adjoint_speedup_vs_plain": (value / plain["value"]) if plain else None,
        "e2e": {"value": e2e_value, "unit": "evals/s", "h2d_bytes_per_step": (h1 - h0) // args.steps,
                "d2h_bytes_per_step": (d1 - d0) // args.steps},
        "gpu_launches": int(launches),
        "autotune": tuning,
        "roofline": roof_line,
        "clocks": clk,
    }
    if args.cpu_baseline and dist.rank == 0:
        line["cpu_baseline"] = cpu_sample(sysm, sets, lam, K, args.tol, max(1, int(np.ceil(np.mean(iters)))),
                                          warmup=1, steps=2)
    ctx.close()
    if args.composite:
        comp = run_composite(args, dev, dist.rank, lam)
        comp["full_gradient"] = {"adjoint_ms": ms_step, "plain_ms": plain["ms_per_step"] if plain else None,
                                 "speedup": (plain["ms_per_step"] / ms_step) if plain else None}
        line["composite"] = comp
    if args.large:
        line["large_k10000"] = run_large(args, dev, dist.rank)
    if args.candidates:
        line["candidates"] = run_candidates(args, dev, dist.rank, cpu=bool(args.cpu_baseline and dist.rank == 0))
    if args.expc:
        line["expectation_values"] = run_expc(args, dev, dist.rank, cpu=bool(args.cpu_baseline and dist.rank == 0))
    return line


# ---------------------------------------------------------------------------
def cpu_sample(sysm, sets, lam, K, tol, max_iter, warmup=1, steps=2, start=0):
    """Time the oracle on full, unscaled EnergyIB evaluations of the
    workload (all K(K+1)/2 pair terms with derivatives and StoreHSD into
    Glob_D, GHEPIIS with LDLHF's parallel branch when linalg_setparam would
    pick it, the gradient contraction), all host threads, warm-started like
    the GPU steps.  Returns the cpu_baseline object (value in evals/s)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    threads = orc.host_threads()
    orc.set_threads(threads)
    orc.set_ldlhf_mode(-1)
    o = orc.Oracle(sysm, K, max_nfo=K)
    o.last[:K] = 1.0
    times, its, Es = [], [], []
    for s in range(start, start + warmup + steps):
        o.set_params(sets[s % len(sets)])
        t0 = time.perf_counter()
        E, g, err, it = o.energy_ib(0, K, lam, tol, max_iter=max_iter)
        dt = time.perf_counter() - t0
        if s >= start + warmup:
            times.append(dt)
            its.append(it)
            Es.append(E)
    t = float(np.mean(times))
    par = (threads >= 8 and K > 5000) or (threads >= 16 and K > 3000)
    return {"value": 1.0 / t, "unit": "evals/s", "cores": threads, "kind": "port",
            "sample": (f"oracle (C restatement, {threads} OpenMP threads): {steps} full unscaled EnergyIB "
                       f"evaluations at K={K} after {warmup} warm-up, GHEPIIS Tol {tol:g} MaxIter {max_iter}, "
                       f"LDLHF {'parallel' if par else 'serial'} branch"),
            "seconds_per_eval": t, "seconds": [round(x, 3) for x in times], "invit_iters": its,
            "energies": Es, "cpu": platform.processor() or platform.machine()}


def run_composite(args, dev, rank, lam):
    """Energy + gradient of one new basis function at K = 4000 (n = 3, T = 4):
    the evaluation the optimisation of a newly added function repeats
    (BasisEnlI's DRMNG loop, src/workproc.f90:4137-4170; OptCycleI): the
    first K-1 functions of the seed-1002 basis are fixed and factorised, the
    candidate is function K.  Three ways, all through the C ABI with host
    buffers:
      plain     per candidate ecg_set_params + ecg_energy_ib(K-1, K): row K
                with derivatives into Glob_D, GHEPIIS(K, K) on the base
                factor, the Glob_D contraction (the reference's sequence);
      adjoint   per candidate ecg_set_params + ecg_energy_ib_adjoint(K-1, K);
      batched   ecg_eval_candidates_grad for 256 candidates at once (bordered
                Schur-complement inverse iteration for all candidates, the
                fused adjoint pass over their rows).
    Candidates follow GenerateTrialParam's rule from the base functions."""
    from ecg_b200 import Context, synth
    K = args.K or 4000
    K0 = K - 1
    sysm, params = synth.config_basis(CONFIG_INDEX, K=K)
    base = params[:K0]
    B = 256
    cands = synth.candidates(base, B, 3002 + 7919 * rank)
    tol = args.tol
    with Context(sysm, K, max_nfo=1, device=dev) as ctx:
        ctx.set_params(base)
        ctx.set_vectors(K0, last_eigvec=np.ones(K0, dtype=np.complex128))
        E0, err0, it0 = ctx.energy_ia(1, K0, lam, tol, max_iter=50)
        _, x = ctx.vectors(K)
        start = x.copy()
        start[K0] = 0.0
        out = {"workload": f"energy + gradient of function K={K} (n=3, T=4) against a fixed, factorised base of "
                           f"{K0}; {B} candidates (GenerateTrialParam rule), tol {tol:g}",
               "base_energy": E0}
        nsing = 16
        for mode in ("plain", "adjoint"):
            fn = ctx.energy_ib if mode == "plain" else ctx.energy_ib_adjoint
            ctx.set_params(cands[:1], first=K)
            ctx.set_vectors(K, last_eigvec=start)
            fn(K0, K, lam, tol)  # warm-up (graphs, workspaces)
            ms, its = 0.0, []
            for j in range(nsing):
                ctx.set_vectors(K, last_eigvec=start)
                ctx.timer_start()
                ctx.set_params(cands[j:j + 1], first=K)
                Ej, gj, ej, itj = fn(K0, K, lam, tol)
                ms += ctx.timer_stop()
                its.append(itj)
            out[mode] = {"ms_per_eval": ms / nsing, "evals_per_s": nsing / (ms / 1e3),
                         "invit_iters": float(np.mean(its)), "sample": nsing}
        ctx.set_vectors(K, last_eigvec=start)
        ctx.eval_candidates_grad(K0, cands, lam, tol)  # warm-up
        reps, ms = 3, 0.0
        for _ in range(reps):
            ctx.set_vectors(K, last_eigvec=start)
            ctx.timer_start()
            E, err, it, ra, g = ctx.eval_candidates_grad(K0, cands, lam, tol)
            ms += ctx.timer_stop()
        ms /= reps
        out["batched"] = {"ms_per_call": ms, "candidates_per_call": B, "ms_per_eval": ms / B,
                          "evals_per_s": B / (ms / 1e3), "codes": np.bincount(err, minlength=3).tolist(),
                          "iterations": np.bincount(it).tolist()}
        # the batched results against the one-call adjoint path on a few candidates
        diffs = []
        for j in range(4):
            if err[j] != 0:
                continue
            ctx.set_params(cands[j:j + 1], first=K)
            ctx.set_vectors(K, last_eigvec=start)
            Ej, gj, ej, _ = ctx.energy_ib_adjoint(K0, K, lam, tol)
            diffs.append((abs(Ej - E[j]), float(np.max(np.abs(gj - g[j])) / np.max(np.abs(gj)))))
        out["batched_vs_single"] = {"max_abs_dE": max(d[0] for d in diffs) if diffs else None,
                                    "max_rel_dgrad": max(d[1] for d in diffs) if diffs else None}
    out["speedup_batched_vs_plain"] = out["plain"]["ms_per_eval"] / out["batched"]["ms_per_eval"]
    out["speedup_adjoint_vs_plain"] = out["plain"]["ms_per_eval"] / out["adjoint"]["ms_per_eval"]
    return out


def run_large(args, dev, rank):
    """The largest workload, K = 10000: one full energy + gradient step (H, S build,
    LDL^H, inverse iteration at Tol 1e-12, fused adjoint gradient) for the
    Li-like n = 3 system (six Y^+Y terms) and for the five-particle n = 4
    system (heavy particle + four electrons, 14 terms), mass-scaled seeded
    bases.  lambda~ = E * INVITPARAMETER from a first solve."""
    from ecg_b200 import Context, synth
    K = args.large_K
    out = {}
    for key, idx in (("n3_li_like", 4), ("n4_five_particles", "4n4")):
        cfg = synth.CONFIG4_N4 if idx == "4n4" else synth.CONFIGS[idx]
        sysm, params = synth.config_basis(idx, K=K)
        if rank:
            params = synth.random_basis(sysm.n, K, cfg["seed"] + 7919 * rank,
                                        row_scale=synth.reduced_mass_scale(sysm.masses))
        e_floor = synth.SYSTEMS[cfg["system"]]["e_floor"]
        with Context(sysm, K, device=dev) as ctx:
            ctx.set_factor_mode(args.factor_mode)
            ctx.set_params(params)
            ctx.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
            E0, err0, it0 = ctx.energy_ia(1, K, e_floor, -1e-12, max_iter=300, specif_norm=0)
            lam = E0 * INVIT_PARAMETER
            ctx.energy_ia(1, K, lam, 1e-12, max_iter=50, specif_norm=0)
            ctx.set_timing(True)
            ctx.energy_ib_adjoint(0, K, lam, 1e-12)  # warm-up (graphs, workspaces)
            reps, ms, st, its = 2, 0.0, np.zeros(4), []
            for _ in range(reps):
                ctx.timer_start()
                E, g, err, it = ctx.energy_ib_adjoint(0, K, lam, 1e-12)
                ms += ctx.timer_stop()
                st += ctx.stage_ms()
                its.append(int(it))
            ctx.set_timing(False)
        out[key] = {"n": sysm.n, "T": sysm.T, "K": K, "ms_per_step": ms / reps,
                    "stages_ms": dict(zip(["pairs_hs", "ldlh", "invit", "adjoint"], (st / reps).round(3).tolist())),
                    "energy": E, "error_code": int(err), "invit_iters": its, "lambda_tilde": lam,
                    "search": {"E0": E0, "code": int(err0), "iters": int(it0)},
                    "grad_norm": float(np.linalg.norm(g)),
                    "ldlh_tflops": 4.0 / 3.0 * K ** 3 / (st[1] / reps * 1e-3) / 1e12}
    return out


def run_candidates(args, dev, rank, cpu=True):
    """The batched configuration: the BasisEnlI trial loop with K = 2000
    existing functions (seed 1003) and 256 candidates per call, drawn by
    GenerateTrialParam's rule (synth.candidates).  Times ecg_eval_candidates
    (all candidates in one call) against one candidate per call
    (ecg_set_params + ecg_energy_ia(K+1, K+1), the reference's sequence),
    both with host buffers, plus the oracle's trial loop on a bounded sample."""
    from ecg_b200 import Context, synth
    cfg = synth.CONFIGS[3]
    K0, B = args.cand_K, cfg["candidates"]
    sysm, params = synth.config_basis(3, K=K0)
    if rank:
        params = synth.random_basis(sysm.n, K0, cfg["seed"] + 7919 * rank)
    cands = synth.candidates(params, B, cfg["seed"])
    e_floor = synth.SYSTEMS[cfg["system"]]["e_floor"]
    with Context(sysm, K0 + 1, device=dev) as ctx:
        ctx.set_params(params)
        ctx.set_vectors(K0, last_eigvec=np.ones(K0, dtype=np.complex128))
        E0, _, _ = ctx.energy_ia(1, K0, e_floor, -1e-12, max_iter=200)
        lam = E0 * INVIT_PARAMETER
        ctx.set_vectors(K0, last_eigvec=np.ones(K0, dtype=np.complex128))
        Eb, errb, _ = ctx.energy_ia(1, K0, lam, 1e-12)
        _, x = ctx.vectors(K0 + 1)
        start = x.copy()
        start[K0] = 0.0
        launches0 = ctx.launch_count()
        for _ in range(max(1, args.warmup // 2)):
            ctx.set_vectors(K0 + 1, last_eigvec=start)
            ctx.eval_candidates(K0, cands, lam, 1e-12)
        ms, nrep = 0.0, 3
        for _ in range(nrep):
            ctx.set_vectors(K0 + 1, last_eigvec=start)
            ctx.timer_start()
            E, err, it, _ = ctx.eval_candidates(K0, cands, lam, 1e-12)
            ms += ctx.timer_stop()
        ms /= nrep
        n1, ms1 = 16, 0.0
        single = []
        for j in range(n1):
            ctx.set_params(cands[j:j + 1], first=K0 + 1)
            ctx.set_vectors(K0 + 1, last_eigvec=start)
            ctx.timer_start()
            Ej, ej, _ = ctx.energy_ia(K0 + 1, K0 + 1, lam, 1e-12)
            ms1 += ctx.timer_stop()
            single.append(abs(Ej - E[j]) if (ej == 0 and err[j] == 0) else 0.0)
    out = {"workload": f"BasisEnlI trial loop n=3 K={K0} + {B} candidates (T={sysm.T}), tol 1e-12",
           "batched_cand_per_s": B / (ms / 1e3), "ms_per_batch": ms,
           "single_cand_per_s": n1 / (ms1 / 1e3), "ms_per_single": ms1 / n1,
           "batched_speedup": (B / ms) / (n1 / ms1),
           "max_abs_dE_batched_vs_single": float(max(single)),
           "codes": np.bincount(err, minlength=3).tolist(), "iterations": np.bincount(it).tolist(),
           "best_E": float(np.min(np.where(err == 0, E, np.inf))), "base_E": Eb}
    if cpu:
        out["cpu_baseline"] = cpu_candidates(sysm, params, cands, K0)
    return out


def cpu_candidates(sysm, params, cands, K0, Kp=600, ntrial=8):
    """The oracle's sequential trial loop (all host threads) on a sample: a
    base of K' functions, ntrial candidates, scaled to K by (K/K')^2 (one
    trial is the row K of H, S, the bordered LDLHF row and O(K^2) inverse
    iterations)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    threads = orc.host_threads()
    orc.set_threads(threads)
    o = orc.Oracle(sysm, Kp + 1)
    o.set_params(params[:Kp])
    o.last[:Kp] = 1.0
    E0, _, _ = o.energy_ia(1, Kp, -1.2, -1e-12, max_iter=200)
    lam = E0 * INVIT_PARAMETER
    o.last[:Kp] = 1.0
    o.energy_ia(1, Kp, lam, 1e-12)
    start = np.zeros(Kp + 1, dtype=np.complex128)
    start[:Kp] = o.last[:Kp]
    t0 = time.perf_counter()
    o.trial_loop(Kp, cands[:ntrial], lam, 1e-12, start)
    t = (time.perf_counter() - t0) / ntrial * (K0 / Kp) ** 2
    return {"value": 1.0 / t, "unit": "candidates/s", "cores": threads, "kind": "port",
            "sample": f"oracle trial loop, {ntrial} candidates on a base of K'={Kp}, scaled by (K/K')^2"}


def run_expc(args, dev, rank, cpu=True):
    """The expectation-value pass of ExpectationValuesG (SymmAdaptMethod 1:
    MatrixElementsForExpcVals for every pair and Y^+Y term, weighted by the
    eigenvector) at n = 3, T = 4 on the first K functions of the seed-1002
    basis, with the eigenvector of the 'G' solve.  Timed through the C ABI
    with the eigenvector in host memory (copied in every call) and the
    6np+9 sums and bounds copied back."""
    from ecg_b200 import Context, synth
    K = args.expc_K
    sysm, params = synth.config_basis(CONFIG_INDEX, K=K)
    if rank:
        params = synth.random_basis(sysm.n, K, synth.CONFIGS[CONFIG_INDEX]["seed"] + 7919 * rank)
    with Context(sysm, K, method="G", device=dev) as ctx:
        ctx.set_params(params)
        E, err, _ = ctx.energy_ga(1, K, which=1, want_vector=True)
        c, _ = ctx.vectors(K)
        for _ in range(max(1, min(args.warmup, 2))):
            ctx.expectation_values(K, E, c)
        reps = max(1, min(args.steps, 3))
        ms = 0.0
        l0 = ctx.launch_count()
        for _ in range(reps):
            ctx.timer_start()
            d = ctx.expectation_values(K, E, c)
            ms += ctx.timer_stop()
        launches = (ctx.launch_count() - l0) // reps
        ms /= reps
    terms = K * (K + 1) // 2 * sysm.T
    out = {"workload": f"ExpectationValuesG pass n=3 K={K} T={sysm.T} (SymmAdaptMethod 1), eigenvector of the "
                       f"'G' solve (E = {E:.12f})",
           "pair_terms_per_s": terms / (ms / 1e3), "ms_per_pass": ms, "gpu_launches_per_pass": int(launches),
           "S": d["S"], "H_minus_E": d["H"] - E, "rel_err_bound_H": abs(d["H_e"] / d["H"])}
    if cpu:
        out["cpu_baseline"] = cpu_expc(sysm, params, terms)
    return out


def cpu_expc(sysm, params, terms, Kp=300):
    """The oracle's expectation-value loop (all host threads) over the first
    K' functions, scaled to the full pair count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    threads = orc.host_threads()
    orc.set_threads(threads)
    o = orc.Oracle(sysm, Kp)
    o.set_params(params[:Kp])
    o.compute_mat_elem(1, Kp, 0.0, method="G")
    c = np.ones(Kp, dtype=np.complex128)
    t0 = time.perf_counter()
    o.expectation_values(Kp, c, -1.0)
    t = time.perf_counter() - t0
    sample = Kp * (Kp + 1) // 2 * sysm.T
    return {"value": sample / t, "unit": "pair terms/s", "cores": threads, "kind": "port",
            "sample": f"oracle ExpectationValuesG loop over K'={Kp} functions ({sample} pair terms)",
            "ms_per_pass_scaled": t * terms / sample * 1e3}


def run_reference(args, dist):
    """The reference arm: the oracle's EnergyIB on the host cores, one full,
    unscaled evaluation per step, on the GPU arm's workload (same basis,
    lambda~, perturbed parameter sets and warm starts, Tol 1e-12 and
    MaxIter 20 as the reference's inputs set them; --ref-max-iter caps the
    iterations instead)."""
    if dist.rank != 0:
        return None
    K = args.K or 4000
    sysm, params, e_floor = setup_problem(K, 0)
    fx = load_fixture(K)
    if args.lam is not None:
        lam = args.lam
    elif fx is not None:
        lam = fx["lambda_tilde"]
    else:
        lam = e_floor
    mi = args.ref_max_iter or 20
    sets = perturbed_sets(params, 0)
    t0 = time.perf_counter()
    cb = cpu_sample(sysm, sets, lam, K, args.tol, int(mi), warmup=args.warmup, steps=args.steps)
    wall = time.perf_counter() - t0
    v = cb["value"]
    return {"metric": METRIC, "value": v, "unit": "evals/s", "impl": "reference", "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic: seeded ECG basis (seed 1002), perturbed sets (seed {PERTURB_SEED})",
            "config": {"workload": f"EnergyIB n=3 K={K} T={sysm.T} on the host CPU, one full evaluation per step",
                       "K": K, "n": sysm.n, "T": sysm.T, "tol": args.tol, "max_iter": int(mi), "lambda_tilde": lam,
                       "parallelism": "OpenMP over pairs; LDLHF parallel branch with the threads as ranks"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "invit_iters_per_step": cb["invit_iters"], "seconds_per_step": cb["seconds"], "wall_s": wall,
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    dist = Dist()
    try:
        if args.only_expc and args.impl == "ours":
            import torch
            torch.cuda.set_device(dist.local)
            line = {"expectation_values": run_expc(args, dist.local, dist.rank, cpu=bool(args.cpu_baseline))}
        else:
            line = run_reference(args, dist) if args.impl == "reference" else run_ours(args, dist)
        if dist.rank == 0 and line is not None:
            print(json.dumps(line))
    finally:
        dist.close()


if __name__ == "__main__":
    main()
