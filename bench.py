"""Throughput of the BRP4 per-template search on B200.

Workload: the batched bank search at N = 2^22 (one 2^22-sample float32 series
at 128 us with 3 injected binary pulsars, 512 circular-orbit templates with
production search parameters, bank-wide toplist of 100), seeded synthetic
data.  A step is one pass of the search path over the whole bank.

Reported (one JSON line, rank 0):
  value      templates/s over all ranks, device-resident inputs, one captured
             CUDA graph per step, L2 flushed between steps (CUDA events on the
             bank's stream, max over ranks)
  e2e        the same metric through the public API (Bank.submit / Bank.wait)
             with the series copied from pinned host memory every step,
             candidates copied back and folded into the bank-wide toplist on
             the host; one step's upload and fold overlap its neighbours'
             kernels
  roofline   the dominant kernel's algorithmic bytes / its device time, and
             its ncu DRAM bytes / its device time
  plain      templates/s of the step-by-step per-template pipeline, same GPU
  cpu_baseline  the reference CPU path over the whole bank once (rank 0, N = 1)

`--impl reference` times the reference's own CPU implementation of the path
(oracle/_ref: src/science.cpp resampling, the harmonic summing restatement,
select) with scipy's float32 real FFT standing in for FFTW, over all host
cores, on the same bank: its templates come from the reference's own compiled
search_parameters (src/workload.cpp:108-125), and each timed step searches the
whole 512-template bank (a rotating sample of it only when the steps would not
fit REF_TIMED_BUDGET_S).  The reference process loads none of this
repository's CUDA library.
"""
import argparse
import datetime
import hashlib
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "boinc-einstein-bpr4-v3d_b200")
for _p in (ROOT, PKG_DIR):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

N = 1 << 22
TEMPLATES = 512
CAPACITY = 8192
METRIC = "orbital templates/s at N=2^22 on 1 B200 (batched bank search)"
UNIT = "templates/s"
L2_FLUSH_BYTES = 512 << 20
REF_TIMED_BUDGET_S = 240.0  # bound of the reference arm's timed region (all steps)
# Algorithmic HBM bytes per template (per kernel) at length n: pass 1 gathers the
# series (4n) and writes the four-step intermediate (4n); pass 2 reads it (4n) and
# writes the power spectrum (2n); harmonic summing reads the power spectrum (2n).
ALGO_BYTES = {"pass1": 8, "pass2": 6, "harmonic": 2}


def parse():
    a = argparse.ArgumentParser()
    a.add_argument("--gpus", type=int, default=1)
    a.add_argument("--steps", type=int, default=40)
    a.add_argument("--warmup", type=int, default=3)
    a.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    a.add_argument("--templates", type=int, default=TEMPLATES)
    a.add_argument("--no-cpu-baseline", action="store_true")
    a.add_argument("--no-plain", action="store_true")
    a.add_argument("--no-tune", action="store_true", help="skip the autotuner (default kernels)")
    a.add_argument("--plan", default=None,
                   help="pass1,pass2,group,chains: use this configuration instead of the autotuner")
    a.add_argument("--toplist-rows", type=int, default=100,
                   help="device toplist pre-filter rows per level (0: return every candidate)")
    a.add_argument("--same-device", action="store_true",
                   help="every rank on device 0 (the multi-rank flow on one GPU; needs --dist-backend gloo)")
    a.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                   help="process-group backend of the multi-rank run (the search has no data-path collective)")
    a.add_argument("--workload", default="bank", choices=["bank", "mixed-radix", "uneven"],
                   help="bank: N=2^22, 512 templates (the headline); mixed-radix: N=3*2^21, 128 templates; "
                        "uneven: 1024 templates over N in {2^20, 3*2^20, 2^22} (1 GPU, documentation runs)")
    return a.parse_args()


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_traffic():
    """Per-template DRAM bytes of each kernel from the committed ncu summary
    (profiles/traffic.txt: lines `kernel bytes_per_template`), if present."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    out = {}
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and not line.startswith("#"):
                    out[parts[0]] = float(parts[1])
    except OSError:
        pass
    return out


# ------------------------------------------------------------------ workload
def workload(total_templates, search=None):
    from brp_b200 import synth
    return synth.bank_workload("bank-2^22", [N], [total_templates], [3], seed=3, search=search)


def workload_name(templates):
    return "bank search, N=2^22, %d templates per GPU, 3 injected pulsars" % templates


def reference_search():
    """The reference's own search_parameters (oracle/_ref, compiled from
    src/workload.cpp), else the oracle's restatement of it."""
    from oracle import oracle as O
    return O.ref_search_parameters if O.ref_available() else O.search_parameters


# --------------------------------------------------------------- CPU baseline
_W = {}


def _cpu_init(series):
    from oracle import oracle as O
    import scipy.fft  # noqa: F401
    _W["x"] = series
    _W["O"] = O
    O.ref() if O.ref_available() else O.lib()


def _cpu_search(pbytes):
    """One template through the reference CPU path: (resampled series, candidates)."""
    import scipy.fft
    O = _W["O"]
    p = O.Params.from_buffer_copy(pbytes)
    x = _W["x"]
    if O.ref_available():
        r = O.ref_resample(x, p)
    else:
        r = O.resample(x, p)
    X = scipy.fft.rfft(r, workers=1)  # float32 FFT, the FFTW stand-in
    n = p.n
    P = ((X.real[: n // 2].astype(np.float64) ** 2 + X.imag[: n // 2].astype(np.float64) ** 2)
         * float(np.float32(1.0) / np.float32(n))).astype(np.float32)
    P[0] = 0
    S = O.ref_harmonic(P, p) if O.ref_available() else O.harmonic(P, p)
    return r[: p.steps], O.select(S, p)


def _cpu_template(pbytes):
    """One template through the reference CPU path; returns the candidate count."""
    return len(_cpu_search(pbytes)[1])


def _cpu_check(pbytes):
    """The reference CPU path's answer for one template, for the parity check:
    (SHA-1 of the resampled samples below `steps`, candidate list)."""
    import hashlib
    r, c = _cpu_search(pbytes)
    return hashlib.sha1(r.tobytes()).hexdigest(), c


def cpu_pool(series, cores):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    return ctx.Pool(cores, initializer=_cpu_init, initargs=(series,))


def time_cpu(pool, templates, sample, start=0):
    """Seconds for `sample` templates (from `start`, wrapping) over the pool."""
    blobs = [bytes(templates[(start + k) % len(templates)]) for k in range(sample)]
    t0 = time.perf_counter()
    pool.map(_cpu_template, blobs, chunksize=1)
    return time.perf_counter() - t0


def time_cpu_one_core(pool, templates, reps=3):
    """Seconds per template on one host core (one worker process, scipy FFT
    with one thread): the median of `reps` templates."""
    times = []
    for k in range(reps):
        t0 = time.perf_counter()
        pool.apply(_cpu_template, (bytes(templates[k % len(templates)]),))
        times.append(time.perf_counter() - t0)
    return statistics.median(times)


def reference_check(B, bank, pool, templates, orbits, sample, resampled_sha1):
    """The reference's CPU path (its compiled resampling and harmonic sum, the
    float32 FFT stand-in, select) on the first `sample` bank templates against
    the bank's own full candidate lists for them (toplist pre-filter off):
    template 0's resampled samples bit for bit (through brp::GPU's snapshot),
    candidate (bin, level) keys equal except within 1e-5 relative of the
    level's threshold (the FFTs differ by rounding), the largest relative power
    difference of the shared keys, and the (bin, harmonics, template) order of
    the final toplists folded from the two sets of lists."""
    ref = pool.map(_cpu_check, [bytes(templates[k]) for k in range(sample)], chunksize=1)
    bank.set_toplist_filter(0)
    flat, offs, counts, status = bank.run_flat(B.Bank.params_array(templates[:sample]))
    gpu = [flat[offs[t]:offs[t + 1]].copy() for t in range(sample)]
    differ = near_threshold = 0
    worst = 0.0
    for t in range(sample):
        thr = templates[t].threshold
        kg = {(int(b), int(l)): float(v) for b, l, v in zip(gpu[t]["bin"], gpu[t]["level"], gpu[t]["power"])}
        c = ref[t][1]
        kr = {(int(b), int(l)): float(v) for b, l, v in zip(c["bin"], c["level"], c["power"])}
        for k in set(kg) ^ set(kr):
            differ += 1
            v = kg.get(k, kr.get(k))
            near_threshold += abs(v - thr[k[1]]) <= 1e-5 * thr[k[1]]
        for k in set(kg) & set(kr):
            worst = max(worst, abs(kg[k] - kr[k]) / max(abs(kr[k]), 1e-30))
    tops = []
    for lists in (gpu, [np.asarray(r[1]).view(B.CANDIDATE) for r in ref]):
        top = B.Toplist().fold(templates[:sample], orbits[:sample], lists).final()
        tops.append(list(zip(top["bin"].tolist(), top["harmonics"].tolist(), top["period"].tolist())))
    return {"templates": sample, "status_words_clear": not bool(np.any(status)),
            "resampled_template0_bit_exact": ref[0][0] == resampled_sha1,
            "candidates_gpu": int(sum(len(c) for c in gpu)), "candidates_reference": int(sum(len(r[1]) for r in ref)),
            "candidates_differ": differ, "candidates_differ_away_from_threshold": differ - int(near_threshold),
            "max_power_rel_diff_shared": worst, "toplist_rows": len(tops[0]),
            "toplist_row_order_equal": tops[0] == tops[1]}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_kind():
    from oracle import oracle as O
    return "reference" if O.ref_available() else "port"


# ------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi samples every 100 ms; only the samples whose timestamps fall
    inside the timed region (begin() .. end()) are summarised."""
    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.proc = None
        self.t0 = self.t1 = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(device_index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.5)  # the sampler's start-up, before the timed region
        except Exception:
            self.proc = None

    def begin(self):
        self.t0 = datetime.datetime.now()

    def end(self):
        self.t1 = datetime.datetime.now()

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.2)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            return None
        rows = []
        for line in out.strip().splitlines():
            r = [x.strip() for x in line.split(",")]
            if len(r) < 9:
                continue
            try:
                ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f")
                rows.append((ts, float(r[1]), float(r[2]), r[5:9]))
            except ValueError:
                continue
        inside = [r for r in rows if self.t0 and self.t1 and self.t0 <= r[0] <= self.t1]
        use = inside or rows
        if not use:
            return None
        sm = [r[1] for r in use]
        mx = max(r[2] for r in use)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in use for i in range(4) if r[3][i].lower() == "active"})
        loaded = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": reasons, "samples": len(use),
                "window": "timed region" if inside else "whole run (no sample inside the timed region)"}


# --------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    """The reference's CPU path on the bench bank, all host cores, rank 0 only.
    Each timed step searches the per-GPU bank (all args.templates templates;
    at N > 1 the first args.templates of the N-GPU bank), unless K such steps
    would exceed REF_TIMED_BUDGET_S, in which case each step searches a
    rotating sample of it (stated in config.workload).  Warm-up steps search
    one template per worker."""
    if rank != 0:
        return
    wl = workload(args.templates * world, search=reference_search())
    bank = wl.templates[:args.templates]
    cores = host_cores()
    pool = cpu_pool(wl.series[0], cores)
    warm = [time_cpu(pool, bank, cores, k * cores) for k in range(max(args.warmup, 1))]
    rate = cores / min(warm)  # templates/s, from the fastest warm-up step
    per_step = len(bank)
    if args.steps * per_step / rate > REF_TIMED_BUDGET_S:
        per_step = max(cores, int(REF_TIMED_BUDGET_S * rate / args.steps) // cores * cores)
    times = [time_cpu(pool, bank, per_step, k * per_step) for k in range(args.steps)]
    pool.close()
    total = sum(times)
    value = per_step * args.steps / total
    kind = reference_kind()
    name = workload_name(args.templates)
    if per_step < len(bank):
        name += " (reference: a rotating sample of %d of the %d templates per step)" % (per_step, len(bank))
    elif world > 1:
        name += " (reference: the first %d of the %d templates per step)" % (len(bank), len(wl.templates))
    sample = "%d templates of the N=2^22 bank per step over %d processes (scipy float32 rfft for FFTW)" % (
        per_step, cores)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": name, "n": N, "templates_per_gpu": args.templates,
                       "templates_per_step": per_step, "templates": "reference search_parameters (%s)" % kind,
                       "parallelism": "%d host processes, one template each at a time" % cores},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- CUDA arm
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.same_device:
        local = 0  # the ranks share one GPU; their kernels never wait on one another
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload != "bank":
        return run_other_workload(args)

    total_templates = args.templates * world
    wl = workload(total_templates)
    from brp_b200 import shard
    begin, end = shard.shard_range(total_templates, rank, world)
    my_templates = wl.templates[begin:end]
    count = len(my_templates)

    # The CPU pool is started before the first GPU call (spawned workers).
    pool = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        pool = cpu_pool(wl.series[0], host_cores())

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        if args.dist_backend == "nccl":
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    import brp_b200 as B

    bank = B.Bank([N], [N], count, CAPACITY, device=local)
    series = torch.from_numpy(wl.series[0]).pin_memory()
    x_host = series.numpy()
    stream = torch.cuda.ExternalStream(bank.stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    tarr = B.Bank.params_array(my_templates)
    orbits = np.asarray(wl.orbits[begin:end], np.float64)
    outbuf = np.empty(count * CAPACITY, B.CANDIDATE)
    all_tarr = B.Bank.params_array(wl.templates) if world > 1 else tarr
    all_orbits = np.asarray(wl.orbits, np.float64)

    def e2e_step():
        bank.set_series(0, x_host)
        return bank.run_flat(tarr, out=outbuf)

    def e2e_fold_step():
        # the public API end to end: series upload, search of this rank's shard,
        # candidate lists to the host, bank-wide toplist (gathered to rank 0)
        bank.set_series(0, x_host)
        return shard.search_and_fold(bank, tarr, begin, all_tarr, all_orbits, out=outbuf)

    def e2e_pipelined(steps):
        # The same work per step through the asynchronous half of the API: step
        # k + 1's series upload (pinned memory, the copy stream, into the buffer
        # step k does not read) crosses PCIe while step k's kernels run, and
        # step k's candidate download is followed by step k + 1's submit before
        # step k's toplist fold on the host.
        bank.set_series(0, x_host)
        bank.submit(tarr)
        for k in range(steps):
            if k + 1 < steps:
                bank.set_series(0, x_host)
            flat, offs, counts, status = bank.wait(out=outbuf)
            if k + 1 < steps:
                bank.submit(tarr)
            B.Toplist().fold(tarr, orbits, flat, counts)

    # autotune the kernel configuration and templates per launch on this bank
    # (untimed), then warm up through the public API (captures the graph)
    plan = None
    if args.plan:
        p1, p2, grp, ch = (int(v) for v in args.plan.split(","))
        bank.configure(N, pass1=p1, pass2=p2, group=grp, chains=ch)
        plan = {str(N): {"pass1": p1, "pass2": p2, "group": grp, "chains": ch, "ms": None}}
    elif not args.no_tune:
        from brp_b200 import tune
        bank.set_series(0, x_host)
        res = tune.autotune(bank, my_templates, use_cache=False)
        plan = {str(n): {k: r[k] for k in ("pass1", "pass2", "group", "chains", "ms")} for n, r in res.items()}
        if os.environ.get("BRP_BENCH_VERBOSE"):
            print(json.dumps({"tuning": {str(n): r.get("tried") for n, r in res.items()}}), file=sys.stderr)
    bank.set_toplist_filter(args.toplist_rows)  # candidates that can reach the toplist
    for _ in range(max(args.warmup, 3)):
        flat, offs, counts, status = e2e_step()
    d2h = 4 * count * (3 if args.toplist_rows else 2) + 8 * (count + 1) + 16 * len(flat)
    h2d = 4 * N + 108 * count + 8 * count

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # --- device throughput (value)
    clocks = Clocks(local)
    barrier()
    clocks.begin()
    step_ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bank.launch()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    barrier()
    clocks.end()
    clock = clocks.stop()
    dev_ms = sum(step_ms)
    launches_per_step = bank.kernels_per_run  # of the graph just timed

    # --- end to end through the public API (series H2D + candidates D2H + toplist)
    barrier()
    t0 = time.perf_counter()
    if world == 1:
        e2e_pipelined(args.steps)
    else:
        for _ in range(args.steps):
            e2e_fold_step()
    torch.cuda.synchronize()
    e2e_ms = 1000 * (time.perf_counter() - t0)
    barrier()

    # per-kernel device time of one eager replay (roofline)
    kernel_ms, launches = bank.profile()

    if dist:
        t = torch.tensor([dev_ms, e2e_ms], dtype=torch.float64,
                         device="cuda" if args.dist_backend == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms, e2e_ms = t.tolist()

    # the spectrum error of this build on the bench workload: one template's
    # power against an FP64 FFT of the same padded series
    accuracy = resampled_sha1 = None
    if rank == 0:
        accuracy, resampled_sha1 = spectrum_error(B, wl, my_templates[0])

    # plain per-template pipeline on the same GPU (comparator)
    plain = None
    if rank == 0 and not args.no_plain:
        plain = time_plain(B, wl, my_templates[:8])

    cpu = None
    if pool is not None:
        # the reference arm's step: the whole bank once over every host core
        cores = host_cores()
        time_cpu(pool, wl.templates, cores)
        secs = time_cpu(pool, wl.templates, count)
        one = time_cpu_one_core(pool, wl.templates)
        cpu = {"value": count / secs, "unit": UNIT, "cores": cores, "kind": reference_kind(),
               "sample": "the whole %d-template N=2^22 bank once over %d processes (scipy float32 rfft for FFTW)"
                         % (count, cores),
               "one_core_value": 1.0 / one}
        # parity of this run against the reference's CPU path over the whole
        # bank (untimed); a failure of the check is reported in the line
        try:
            accuracy["vs_reference_cpu"] = reference_check(B, bank, pool, my_templates, orbits, count,
                                                           resampled_sha1)
        except Exception as e:
            accuracy["vs_reference_cpu"] = {"error": "%s: %s" % (type(e).__name__, e)}
        pool.close()

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peak, peak_kind = load_peaks()
    per_launch = {k: kernel_ms[k] / max(launches[k], 1) for k in ("pass1", "pass2", "harmonic")}
    top_kernel = max(per_launch, key=lambda k: kernel_ms[k])
    group = count / max(launches[top_kernel], 1)
    algo = ALGO_BYTES[top_kernel] * N * group
    achieved = algo / (per_launch[top_kernel] * 1e-3) / 1e9
    traffic = measured_traffic().get(top_kernel)
    traffic_launch = traffic * group if traffic else None
    achieved_dram = traffic_launch / (per_launch[top_kernel] * 1e-3) / 1e9 if traffic else None
    value = total_templates * args.steps / (dev_ms / 1000)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "bank search, N=2^22, %d templates per GPU, 3 injected pulsars" % args.templates,
                   "n": N, "templates_per_gpu": count, "candidate_capacity": CAPACITY,
                   "toplist_prefilter_rows": args.toplist_rows,
                   "l2": "flushed between steps (%d MiB write)" % (L2_FLUSH_BYTES >> 20),
                   "parallelism": "template shards, %d rank(s)" % world,
                   "plan": plan},
        "e2e": {"value": total_templates * args.steps / (e2e_ms / 1000), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "hbm", "kernel": top_kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic_launch,
                     "achieved_dram": achieved_dram, "frac_dram": achieved_dram / peak if traffic else None,
                     "algorithmic_bytes_per_launch": algo, "templates_per_launch": group,
                     "note": "achieved/frac: algorithmic bytes %dn per template (pass 1 counts its 4n series "
                             "gather, which the 16 MiB series shared by every template serves from L2); "
                             "achieved_dram/frac_dram: ncu DRAM bytes of the same launch (profiles/traffic.txt) "
                             "over its live duration" % ALGO_BYTES[top_kernel]},
        "kernel_ms_per_step": kernel_ms, "kernel_launches_per_step": launches,
        "algorithmic_gbs_all_kernels": 16 * N * count / (sum(kernel_ms[k] for k in ALGO_BYTES) * 1e-3) / 1e9,
        "clocks": clock,
    }
    if accuracy:
        line["accuracy"] = accuracy
    if plain:
        line["plain"] = plain
        line["batched_vs_plain"] = value / world / plain["templates_per_s"]
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_other_workload(args):
    """The mixed-radix and uneven banks on one GPU: device time of the captured
    graph (L2 flushed between steps), end to end through the public API
    (series H2D, graph, candidates D2H, toplist fold per length class in bank
    order), algorithmic HBM bytes 16 n per template over all kernels."""
    from brp_b200 import synth, tune
    import torch
    import brp_b200 as B
    wl = synth.config4() if args.workload == "mixed-radix" else synth.config5()
    count = len(wl.templates)
    bank = B.Bank(wl.n, [len(x) for x in wl.series], count, CAPACITY)
    hosts = [torch.from_numpy(x).pin_memory().numpy() for x in wl.series]
    for s, x in enumerate(hosts):
        bank.set_series(s, x)
    if args.plan:  # single-length workloads: a fixed configuration (e.g. the tensor-core pass 1)
        p1, p2, grp, ch = (int(v) for v in args.plan.split(","))
        bank.configure(wl.n[0], pass1=p1, pass2=p2, group=grp, chains=ch)
        plan = {str(wl.n[0]): {"pass1": p1, "pass2": p2, "group": grp, "chains": ch, "ms": None}}
    else:
        res = tune.autotune(bank, wl.templates, wl.series_of, use_cache=False)
        plan = {str(n): {k: r[k] for k in ("pass1", "pass2", "group", "chains", "ms")} for n, r in res.items()}
    tarr = B.Bank.params_array(wl.templates)
    so = np.asarray(wl.series_of, np.uint32)
    orbits = np.asarray(wl.orbits, np.float64)
    out = np.empty(count * CAPACITY, B.CANDIDATE)
    classes = sorted(set(int(v) for v in wl.series_of))
    members = {s: np.flatnonzero(so == s) for s in classes}
    class_params = {s: B.Bank.params_array([wl.templates[t] for t in members[s]]) for s in classes}

    def fold(flat, offs, counts):
        tops = {}
        for s in classes:  # one toplist per series, its templates in bank order
            idx = members[s]
            if len(idx) and idx[-1] - idx[0] + 1 == len(idx):  # contiguous in the bank
                cand = flat[offs[idx[0]]:offs[idx[-1] + 1]]
            else:
                cand = np.concatenate([flat[offs[t]:offs[t + 1]] for t in idx]) if len(idx) else flat[:0]
            tops[s] = B.Toplist().fold(class_params[s], orbits[idx], cand, counts[idx])
        return tops

    def e2e_step():
        for s, x in enumerate(hosts):
            bank.set_series(s, x)
        return fold(*bank.run_flat(tarr, so, out=out)[:3])

    def e2e_pipelined(steps):
        # as e2e_step per step, with step k + 1's uploads during step k's kernels
        # and step k's folds during step k + 1's (Bank.submit / Bank.wait)
        for s, x in enumerate(hosts):
            bank.set_series(s, x)
        bank.submit(tarr, so)
        for k in range(steps):
            if k + 1 < steps:
                for s, x in enumerate(hosts):
                    bank.set_series(s, x)
            flat, offs, counts, status = bank.wait(out=out)
            if k + 1 < steps:
                bank.submit(tarr, so)
            fold(flat, offs, counts)

    bank.set_toplist_filter(args.toplist_rows)  # candidates that can reach the toplist
    for _ in range(max(args.warmup, 3)):
        e2e_step()
    stream = torch.cuda.ExternalStream(bank.stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    clocks = Clocks(0)
    clocks.begin()
    step_ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bank.launch()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    clocks.end()
    clock = clocks.stop()
    launches_per_step = bank.kernels_per_run  # of the graph just timed
    t0 = time.perf_counter()
    e2e_pipelined(args.steps)
    torch.cuda.synchronize()
    e2e_ms = 1000 * (time.perf_counter() - t0)
    kernel_ms, launches = bank.profile()
    dev_ms = sum(step_ms)
    algo = sum(16 * wl.n[s] for s in wl.series_of)
    print(json.dumps({
        "metric": "orbital templates/s (%s bank on 1 B200)" % args.workload, "value": count * args.steps / (dev_ms / 1e3),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl.name, "lengths": list(wl.n),
                   "templates_per_length": [int(len(members.get(s, []))) for s in range(len(wl.n))],
                   "candidate_capacity": CAPACITY, "toplist_prefilter_rows": args.toplist_rows,
                   "l2": "flushed between steps (%d MiB write)" % (L2_FLUSH_BYTES >> 20),
                   "plan": plan},
        "e2e": {"value": count * args.steps / (e2e_ms / 1e3), "unit": UNIT},
        "gpu_launches": launches_per_step * args.steps,
        "algorithmic_hbm_gbs": algo / (dev_ms / args.steps * 1e-3) / 1e9,
        "kernel_ms_per_step": kernel_ms, "kernel_launches_per_step": launches, "clocks": clock}), flush=True)
    bank.close()


def spectrum_error(B, wl, p):
    """Relative RMS of the GPU power spectrum against numpy's FP64 real FFT of
    the GPU's own padded series (isolates the FFT and power arithmetic)."""
    g = B.GPU(p, wl.series[0], 256, 0, 1, stockham=True, packed=True)
    g.set_template(p)
    g.run()
    s = g.snapshot()
    g.close()
    X = np.fft.rfft(s.resampled.astype(np.float64))
    P = (X.real[: p.n // 2] ** 2 + X.imag[: p.n // 2] ** 2) / p.n
    P[0] = 0
    err = float(np.sqrt(np.sum((s.power - P) ** 2) / np.sum(P ** 2)))
    sha = hashlib.sha1(np.ascontiguousarray(s.resampled[: p.steps]).tobytes()).hexdigest()
    return {"power_rel_rms_vs_fp64": err, "template": "bank template 0", "bar": 2e-6}, sha


def time_plain(B, wl, templates):
    """Device time per template of the step-by-step pipeline (batch 1), and of
    the fused pipeline run one template at a time through brp::GPU."""
    out = {}
    for name, plain in (("templates_per_s", True), ("fused_single_templates_per_s", False)):
        g = B.GPU(templates[0], wl.series[0], 256, 0, 1, stockham=True, packed=True, plain=plain)
        ms = []
        for k, p in enumerate(templates):
            g.set_template(p)
            t = g.run()
            if k >= 2:
                ms.append(sum(t.stage_ms))
        g.close()
        out[name] = 1000.0 / statistics.mean(ms)
    return out


if __name__ == "__main__":
    main()
