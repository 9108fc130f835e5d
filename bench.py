"""Benchmark of the TPB sigma hot path on B200 (one JSON line on rank 0).

A step is one sigma = H*C over the whole determinant space of the workload (default: norb=32,
10+10 electrons, 20,000 x 20,000 strings = 400M determinants, seeded synthetic integrals and
strings as the reference's molecular inputs would give them).  `value` is sigma GDets/s with the
vectors resident in HBM (the library's internal sign convention, no conversion passes); `e2e`
is the same through the reference-facing C ABI call sbd_tpb_sigma with host buffers (H2D of C,
sign conversions, D2H of sigma inside the timed region).  Multi-GPU runs are replicas (the
path has no data exchange on one node in this build): every rank solves its own copy and
`value` is the aggregate.  `--impl reference` times the reference's own CPU sigma (compiled
unchanged under oracle/_ref) on a bounded sample of the same workload with all host threads.

The line also carries `strings` (a 2,000,000-line string file parsed, sorted and de-duplicated on
the GPU, beside the reference's LoadAlphaDets on the host) and `carryover`: the carry-over string selection (sbd_tpb_carryover_strings,
the step after the solve in the reference's sbd::tpb::diag) on an FP64 vector of the workload,
with the roofline of its pass over W and the CPU restatement timed on a sample of rows.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload sci32]
                    [--precision mixed|fp64] [--impl ours|reference] [--no-solve] [--no-carryover]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sbd-pub_b200", "python"))

METRIC = "sigma GDets/s; time to 1e-6 Ha: mixed+learned vs plain FP64, 1 B200"
REF_BENCH = os.path.join(ROOT, "oracle", "_ref", "ref_bench")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="sci32")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-solve", action="store_true", help="skip the time-to-solution solves")
    ap.add_argument("--cpu-sample-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU reference sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end pass")
    ap.add_argument("--no-carryover", action="store_true", help="skip the carry-over measurement")
    ap.add_argument("--davidson-cycle", action="store_true",
                    help="only run one Davidson cycle (8 sigma steps, final FP64 sigma) on the workload "
                         "and print its time; the command the Davidson launch-list profile is taken on")
    return ap.parse_args()


def run_davidson_cycle(args, local):
    import sbd_tpb
    import synth
    prob = synth.make_problem(args.workload)
    h = sbd_tpb.Handle(local)
    h.set_problem(prob)
    prec = sbd_tpb.MIXED if args.precision == "mixed" else sbd_tpb.FP64
    t0 = time.perf_counter()
    r = h.davidson(sbd_tpb.default_params(max_it=1, max_nb=8, eps=1e-12, precision=prec), want_vector=False)
    dt = time.perf_counter() - t0
    print(json.dumps({"workload": args.workload, "precision": args.precision, "sigma_steps": r["iterations"],
                      "seconds": dt, "ms_per_step": 1e3 * dt / max(1, r["iterations"]),
                      "energy": r["energy"]}), flush=True)
    h.close()


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def replica_throughput(pg, ms_local, dets_local, world, device="cpu"):
    """Whole-job throughput of `world` replicas that each processed dets_local determinants in
    ms_local device milliseconds: the slowest replica's time (all_reduce MAX) and the aggregate
    GDets/s over it.  pg is torch.distributed (or None for one process)."""
    import torch
    ms_max = ms_local
    if pg is not None:
        t = torch.tensor([ms_local], dtype=torch.float64, device=device)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_max = float(t.item())
    return ms_max, world * dets_local / (ms_max * 1e-3) / 1e9


def cpu_reference_sigma(prob_name, seconds_target, reps=1, threads=None):
    """Time the reference's CPU sigma (oracle/_ref/ref_bench) on the first `amax` alpha strings x
    all beta strings of the workload; amax is sized so the sample takes ~seconds_target."""
    import synth
    if not os.path.exists(REF_BENCH):
        return None
    L, n, cnt = synth.CONFIGS[prob_name]
    h1, eri, core = synth.synthetic_hamiltonian(L)
    strs = synth.sample_strings(L, n, cnt)
    env = dict(os.environ)
    threads = threads or os.cpu_count()
    env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory() as tmp:
        fd, fa = os.path.join(tmp, "fcidump.txt"), os.path.join(tmp, "a.txt")
        synth.write_fcidump(fd, L, 2 * n, h1, eri, core)
        synth.write_strings(fa, strs, L)

        def run(amax, reps_):
            out = subprocess.run([REF_BENCH, "--fcidump", fd, "--adetfile", fa, "--amax", str(amax),
                                  "--reps", str(reps_)], capture_output=True, text=True, env=env,
                                 check=True).stdout
            kv = dict(tok.split("=", 1) for tok in out.split())
            return int(kv["ndet"]), [float(x) for x in kv["sigma_s"].split(",")], float(kv["helper_s"])

        amax = max(2, min(len(strs), 16))
        ndet, ts, _ = run(amax, 1)
        per_det = max(ts[0], 1e-4) / ndet
        amax = int(min(len(strs), max(2, seconds_target / per_det / len(strs))))
        ndet, ts, helper_s = run(amax, reps)
    return dict(ndet=ndet, amax=amax, sigma_s=ts, helper_s=helper_s, threads=threads,
                nstrings=len(strs))


def run_reference(args, world, rank):
    if rank != 0:
        return
    import synth
    L, n, cnt = synth.CONFIGS[args.workload]
    if not os.path.exists(REF_BENCH):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_bench not built "
                          "(needs the reference checkout at build time)"}))
        return
    per_step = max(1.0, args.cpu_sample_seconds / max(1, args.steps))
    r = cpu_reference_sigma(args.workload, per_step, reps=args.warmup + args.steps)
    ts = r["sigma_s"][args.warmup:]
    t = sum(ts)
    val = r["ndet"] * len(ts) / t / 1e9
    sample = (f"first {r['amax']} of {r['nstrings']} alpha strings x all {r['nstrings']} beta "
              f"strings ({r['ndet']} determinants) per step, reference sbd::mult (tpb/mult.h:625-881)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": val, "unit": "GDets/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / len(ts),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": f"{args.workload}: norb={L}, {n}+{n} electrons, "
                                        f"{cnt} x {cnt} strings", "sample": sample},
        "cpu_baseline": {"value": val, "unit": "GDets/s", "cores": r["threads"], "kind": "reference",
                         "sample": sample},
        "e2e": {"value": val, "unit": "GDets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def end_to_end(h, x, N, dt, esz, world):
    import torch
    xh = torch.empty(N, dtype=dt, pin_memory=True)
    xh.copy_(x.cpu())
    yh = torch.empty(N, dtype=dt, pin_memory=True)
    xn, yn = xh.numpy(), yh.numpy()
    h.sigma(xn, yn)
    torch.cuda.synchronize()
    steps = 5
    te = time.perf_counter()
    for _ in range(steps):
        h.sigma(xn, yn)
    e2e_s = (time.perf_counter() - te) / steps
    return {"value": world * N / e2e_s / 1e9, "unit": "GDets/s", "h2d_bytes_per_step": N * esz,
            "d2h_bytes_per_step": N * esz, "api": "sbd_tpb_sigma / sbd_tpb_sigma_f32 (host buffers)"}


def train_preconditioner(device):
    """The learned preconditioner, trained on pairs from FP64 Davidson runs on the two smaller
    configurations (12-orbital full CI, 24-orbital 4000 x 4000 selected CI): first along the
    diagonal solver's trajectories, then two rounds along the learned solver's own trajectories
    (each round adds its pairs and retrains)."""
    import sbd_tpb
    import synth
    t0 = time.perf_counter()
    pc = sbd_tpb.Precond(device, seed=2024)
    hs = []
    for name in ("fci12", "sci24"):
        hh = sbd_tpb.Handle(device)
        hh.set_problem(synth.make_problem(name))
        hs.append(hh)
    t_collect = t_train = 0.0
    for rnd in range(3):
        tc = time.perf_counter()
        for hh in hs:
            pc.collect(hh, sbd_tpb.default_params(max_it=30, max_nb=10, eps=1e-8,
                                                  preconditioner=0 if rnd == 0 else 1),
                       samples_per_step=1 << 15)
        t_collect += time.perf_counter() - tc
        tt = time.perf_counter()
        loss = pc.train(epochs=3 if rnd == 0 else 2, batch=8192, lr=1e-3)
        t_train += time.perf_counter() - tt
    for hh in hs:
        hh.close()
    lt, dt = pc.evaluate(0)
    return pc, {"collect_s": t_collect, "train_s": t_train, "rounds": 3,
                "pairs": pc.num_samples(0), "final_batch_loss": loss,
                "train_error_learned_over_diagonal": lt / dt if dt > 0 else None}


def carryover_measure(h, prob, cpu_sample=True):
    """Carry-over selection on an FP64 vector of the workload's size held in HBM: per-call times of
    the pass over W (CUDA events) and of the whole call for types 1 (dominant strings) and 3
    (singles of the determinants above a cutoff).  The pass reads W once (8 bytes per
    determinant) and writes per-string sums: its roofline is HBM bandwidth."""
    import torch

    import sbd_tpb
    N = prob.ndet
    g = torch.Generator(device=f"cuda:{h.device}").manual_seed(99)
    W = torch.randn(N, dtype=torch.float64, device=f"cuda:{h.device}", generator=g)
    W /= torch.linalg.vector_norm(W)
    out = {}
    # cutoff at half the mean weight 1/N: about half the determinants of a random vector pass it
    for name, kind, thr in (("dominant", sbd_tpb.CARRYOVER_DOMINANT, 0.01),
                            ("cutoff_singles", sbd_tpb.CARRYOVER_CUTOFF_SINGLES, 0.5 / N)):
        for _ in range(3):
            r = h.carryover(W, kind, 0.0, thr, mem=sbd_tpb.DEVICE)
        ts = []
        for _ in range(5):
            r = h.carryover(W, kind, 0.0, thr, mem=sbd_tpb.DEVICE)
            ts.append(h.last_carryover_ms())
        ts = np.array(ts)
        pass_ms = float(np.median(ts[:, 0]))
        pk = peaks()
        gbs = N * 8 / (pass_ms * 1e-3) / 1e9
        out[name] = {"pass_ms": pass_ms, "call_ms": float(np.median(ts[:, 1])), "threshold": thr,
                     "strings_out": [len(r["astr"]), len(r["bstr"])],
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
                                  "frac": gbs / pk["hbm_gbs"], "algorithmic_bytes": N * 8}}
    if cpu_sample:
        # the CPU restatement (oracle, one thread) of the same pass on the first rows of W
        import pyoracle
        na, nb = len(prob.astr), len(prob.bstr)
        rows = max(1, min(na, int(2e7) // nb))
        w = W[: rows * nb].cpu().numpy()
        t0 = time.perf_counter()
        pyoracle.string_weights(w, rows, nb)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": rows * nb / dt / 1e9, "unit": "GDets/s", "cores": 1, "kind": "port",
                               "sample": f"per-string weights of the first {rows} alpha rows x {nb} "
                                         f"(orc_string_weights, tpb/rdmat.h:11-61, 138-188)"}
        out["gpu_pass_gdets"] = N / (out["dominant"]["pass_ms"] * 1e-3) / 1e9
    del W
    torch.cuda.empty_cache()
    return out


def strings_measure(h, args, cpu_sample=True):
    """String-file parsing (sbd_tpb_read_strings): a text file of 2,000,000 lines drawn with
    repetition from the workload's strings (as a sampled-string file of the sample-based loop
    holds them), parsed, sorted and de-duplicated on the GPU; beside it the reference's own
    LoadAlphaDets on the same file, on the host cores (oracle/_ref/ref_bench --parse)."""
    import synth
    L, n, cnt = synth.CONFIGS[args.workload]
    pool = synth.sample_strings(L, n, cnt)
    rng = np.random.default_rng(5)
    vals = np.asarray(pool, np.uint64)[rng.integers(0, len(pool), size=2_000_000)]
    bits = ((vals[:, None] >> np.arange(L - 1, -1, -1, dtype=np.uint64)) & 1).astype(np.uint8) + ord("0")
    text = np.concatenate([bits, np.full((len(vals), 1), ord("\n"), np.uint8)], axis=1).tobytes()
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "strings.txt")
        with open(path, "wb") as f:
            f.write(text)
        for _ in range(2):
            h.read_strings(path, L)
        dev, wall = [], []
        for _ in range(5):
            t0 = time.perf_counter()
            got = h.read_strings(path, L)
            wall.append(time.perf_counter() - t0)
            dev.append(h.last_parse_ms())
        out = {"lines": len(vals), "bytes": len(text), "unique": int(len(got)),
               "device_ms": float(np.median(dev)), "call_ms": 1e3 * float(np.median(wall)),
               "note": "device_ms: host-to-device copy of the file from pinned memory, newline index, "
                       "parse, sort, unique (CUDA events); call_ms adds reading the file from disk"}
        if cpu_sample and os.path.exists(REF_BENCH):
            env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count()))
            r = subprocess.run([REF_BENCH, "--parse", path, "--norb", str(L), "--reps", "2"], capture_output=True,
                               text=True, env=env, check=True).stdout
            kv = dict(tok.split("=", 1) for tok in r.split())
            ts = [float(x) for x in kv["parse_s"].split(",")]
            out["cpu_baseline"] = {"value_ms": 1e3 * min(ts), "cores": 1, "kind": "reference",
                                   "sample": "the same file through the reference's LoadAlphaDets "
                                             "(basic/makedeterminants.h:160-186, serial)",
                                   "unique": int(kv["nstrings"])}
    return out


def time_to_solution(h, args):
    """Wall time of whole Davidson solves from the HF start: the FP64 reference answer (residual
    1e-6), then plain FP64, mixed precision and mixed precision + learned preconditioner, all to
    residual 1e-4 (energy error ~ residual^2, far below 1e-6 Ha)."""
    import torch

    import sbd_tpb
    out = {}

    def solve(name, runs=2, **kw):
        # each compared solve runs twice and the faster wall time is reported (both are listed):
        # a step synchronises with the host two or three times, and on a host shared with other
        # jobs single solves were seen up to 40 % slower than the same solve run again
        p = sbd_tpb.default_params(max_it=40, max_nb=8, **kw)
        times = []
        for _ in range(runs):
            torch.cuda.synchronize()
            ts = time.perf_counter()
            r = h.davidson(p, want_vector=False)
            times.append(time.perf_counter() - ts)
        out[name] = {"seconds": min(times), "seconds_runs": times, "sigma_steps": r["iterations"],
                     "energy": r["energy"], "residual": r["residual"], "converged": r["converged"],
                     "eps": kw.get("eps"), "learned_steps": r["learned_steps"],
                     "fallback_steps": r["fallback_steps"]}

    solve("fp64_reference", runs=1, eps=1e-6, precision=sbd_tpb.FP64)
    solve("fp64", eps=1e-4, precision=sbd_tpb.FP64)
    solve("mixed", eps=1e-4, precision=sbd_tpb.MIXED)
    pc, train = train_preconditioner(h.device)
    h.set_preconditioner(pc)
    solve("mixed_learned", eps=1e-4, precision=sbd_tpb.MIXED, preconditioner=sbd_tpb.PRECOND_LEARNED)
    h.set_preconditioner(None)
    pc.close()
    e_ref = out["fp64_reference"]["energy"]
    for k in ("fp64", "mixed", "mixed_learned"):
        out[k]["abs_energy_error_vs_fp64_reference"] = abs(out[k]["energy"] - e_ref)
    out["learned_training"] = train
    out["speedup_mixed_vs_fp64"] = out["fp64"]["seconds"] / out["mixed"]["seconds"]
    out["speedup_mixed_learned_vs_fp64"] = out["fp64"]["seconds"] / out["mixed_learned"]["seconds"]
    out["note"] = ("training (pairs from the 12- and 24-orbital problems) is timed separately and not "
                   "part of the solve times; seconds = the faster of seconds_runs (two runs of each "
                   "compared solve)")
    return out


def run_ours(args, world, rank, local, pg):
    import torch

    import sbd_tpb
    import synth
    torch.cuda.set_device(local)
    L, n, cnt = synth.CONFIGS[args.workload]
    prob = synth.make_problem(args.workload)
    N = prob.ndet
    h = sbd_tpb.Handle(local)
    t0 = time.time()
    h.set_problem(prob, build=False)
    t1 = time.time()
    h.build_tables()
    t_tables = time.time() - t1
    dt = torch.float32 if args.precision == "mixed" else torch.float64
    esz = 4 if dt == torch.float32 else 8
    gen = torch.Generator(device=f"cuda:{local}").manual_seed(1234 + rank)
    x = torch.randn(N, dtype=dt, device=f"cuda:{local}", generator=gen)
    x /= torch.linalg.vector_norm(x)
    y = torch.empty_like(x)
    stream = torch.cuda.ExternalStream(h.stream(), device=f"cuda:{local}")

    def barrier():
        if pg is not None:
            pg.barrier()

    for _ in range(args.warmup):
        h.sigma_device(x, y)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = h.kernel_launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            h.sigma_device(x, y)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms_total = ev0.elapsed_time(ev1)
    launches = h.kernel_launches() - launches0
    barrier()
    ms_max, value = replica_throughput(pg, ms_total, N * args.steps, world, device=f"cuda:{local}")
    ms_step = ms_max / args.steps

    # per-kernel times of the same sigma (separate pass: reading them synchronises each call)
    kern = []
    for _ in range(max(3, min(args.steps, 10))):
        h.sigma_device(x, y)
        kern.append(h.last_sigma_kernels())
    kern = np.array(kern).mean(axis=0)
    # algorithmic bytes of each pass: 3 N s (alpha: read C, write sigma, write C^T; beta: read
    # C^T, sigma read-modify-write) plus its sigma-program tables read once
    def table_bytes(singles, doubles):
        ns, nd = int(h.table(singles)[1].size), int(h.table(doubles)[1].size)
        return ns * (4 + esz + 4) + nd * (4 + esz) + 8 * (len(prob.astr) + 1)
    bytes_alpha = 3 * N * esz + table_bytes(0, 1)
    bytes_beta = 3 * N * esz + table_bytes(2, 3)
    # third timed kernel: the alpha-beta term (sparse kernel, or the dense gather/contract/scatter)
    names = ["sigma_block_kernel<alpha>", "sigma_block_kernel<beta>", "alpha_beta_term"][:len(kern)]
    # sparse alpha-beta: sigma rows of alpha strings with singles read-modified-written, their
    # singles' C rows read once
    bytes_ab = 2 * N * esz + table_bytes(0, 2) // 4
    per = [bytes_alpha, bytes_beta, bytes_ab][:len(kern)]
    dom = int(np.argmax(kern))
    pk = peaks()
    achieved = per[dom] / (kern[dom] * 1e-3) / 1e9
    # DRAM bytes per determinant of each pass from the ncu capture at 10^8 determinants (FP32,
    # profiles/sigma_kernels_sci28_fp32.md), scaled to this workload's determinants
    traffic_per_det = {"sigma_block_kernel<alpha>": 17.69, "sigma_block_kernel<beta>": 12.60}
    traffic = (traffic_per_det[names[dom]] * N / 1e9
               if dt == torch.float32 and names[dom] in traffic_per_det else None)
    roofline = {"kernel": names[dom], "bound": "hbm", "achieved": achieved,
                "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                "traffic": traffic, "traffic_unit": "GB per launch",
                "traffic_source": "ncu capture at 1e8 determinants scaled by determinants" if traffic else None,
                "peak_source": "measured" if not pk.get("fallback") else "fallback",
                "kernel_ms": {names[i]: float(kern[i]) for i in range(len(kern))},
                "algorithmic_bytes": {names[i]: int(per[i]) for i in range(len(kern))}}

    # end to end through the reference-facing C ABI: host buffers, copies and sign passes timed
    e2e = None
    if not args.no_e2e:
        e2e = end_to_end(h, x, N, dt, esz, world)

    solve = None
    if not args.no_solve and world == 1:
        del x, y
        torch.cuda.empty_cache()
        solve = time_to_solution(h, args)

    strings = None
    if not args.no_carryover and world == 1:
        strings = strings_measure(h, args, cpu_sample=rank == 0 and not args.no_cpu)

    carry = None
    if not args.no_carryover and world == 1:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        carry = carryover_measure(h, prob, cpu_sample=rank == 0 and not args.no_cpu)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        r = cpu_reference_sigma(args.workload, args.cpu_sample_seconds)
        if r is not None:
            t = sum(r["sigma_s"]) / len(r["sigma_s"])
            cpu = {"value": r["ndet"] / t / 1e9, "unit": "GDets/s", "cores": r["threads"],
                   "kind": "reference",
                   "sample": f"first {r['amax']} of {r['nstrings']} alpha x all beta strings "
                             f"({r['ndet']} dets), one reference sbd::mult (tpb/mult.h:625-881)"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GDets/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 vectors, f64 accumulate" if dt == torch.float32 else "f64",
            "data": "synthetic (seeded integrals 1729, strings 137)",
            "config": {"workload": f"{args.workload}: norb={L}, {n}+{n} electrons, {cnt} x {cnt} strings",
                       "determinants": N, "precision": args.precision,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (vector of %.2f GB)" % (N * esz / 1e9),
                       "tables_s": t_tables, "setup_s": t1 - t0},
            "gpu_launches": launches, "clocks": clocks.summary(), "roofline": roofline, "e2e": e2e,
            "cpu_baseline": cpu, "time_to_solution": solve, "carryover": carry, "strings": strings,
        }
        print(json.dumps(line), flush=True)
    h.close()


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.davidson_cycle:
            run_davidson_cycle(args, local)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
