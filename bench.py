"""bench.py -- output GB/s of the rocRAND host-API generation path on B200.

Workload (one "step"): the plain single-generator sweep at n = 2^28 values per call --
every generator family built so far x {raw uint32, uniform fp32/fp64/fp16, normal fp32/fp64,
log-normal fp32, Poisson lambda in {0.5, 10, 1000}} at seed 0xdeadbeef -- each call one
rocrand_generate_* through the C ABI into a resident device buffer.  Outputs (0.5-2 GiB per
call) are larger than L2, so no flush is needed between calls.

value  = total output bytes / device time of the K timed steps (CUDA events, max over ranks);
e2e    = the same sweep through the same C ABI with the output copied to pinned host memory
         inside the timed region (what a host caller gets);
roofline = the dominant kernel's achieved write GB/s against the measured HBM copy peak;
cpu_baseline = the reference's own host generators (oracle/_ref, compiled from the reference
         sources) on this host's cores, on a bounded sample of the same sweep.

--impl reference runs only the reference's CPU host generators on the same workload.
Multi-GPU (torchrun): each rank fills its own slice [r*n, (r+1)*n) of every stream through
rocrand_b200_set_output_position (rank_stream), no data-path collective; weak scaling.
MT19937 and MTGP32 have no position: rank r uses seed 0xdeadbeef + r instead (an
independent stream of the same size).
"""

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from ctypes import c_size_t, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

SEED = 0xDEADBEEF
FALLBACK_HBM_GBS = 6650.0

# Generator families in the sweep (rocrand_rng_type values), in the order they were built.
SWEEP_GENERATORS = [("philox4x32_10", 404), ("xorwow", 401), ("mrg32k3a", 402), ("lfsr113", 406),
                    ("mt19937", 407), ("threefry4x32_20", 410), ("mtgp32", 403), ("mrg31k3p", 405),
                    ("threefry2x32_20", 408), ("threefry2x64_20", 409), ("threefry4x64_20", 411)]
# The quasi-random workload: Sobol32 and scrambled Sobol64, 1 / 64 / 1000 dimensions x 2^20
# points at offset 4096, uniform fp64 and normal fp32 (dimension-major output).
QUASI_GENERATORS = [("sobol32", 501), ("scrambled_sobol64", 505)]
QUASI_DIMS = [1, 64, 1000]
QUASI_DISTS = [("uniform_double", None), ("normal", (0.0, 1.0))]
NO_OFFSET = {407, 403}  # MT19937, MTGP32: set_offset is a TYPE_ERROR
PORT_SEEDED = {407}  # host streams seeded by the C port (the reference's host seeding is slow)
STATEFUL = {401, 402, 405, 406}
TWO_WORD = {"uniform_double", "normal", "normal_double", "log_normal", "log_normal_double"}

# DRAM traffic of a launch from one ncu capture of the kernel on a smaller case (summaries in
# profiles/): the state it reads is a fixed amount per launch, and every output byte is
# written once (at the capture's size part of the output was still in L2 when the kernel
# ended and was written back after it), so a launch of B output bytes moves read + B.
NCU_TRAFFIC = {
    ("mt19937", "normal_double"): (20.53e6, "profiles/mt_fill_normal_double_n2p24.md"),
    ("mtgp32", "normal_double"): (2.26e6, "profiles/mtgp_fill_normal_double_n2p24.md"),
    ("philox4x32_10", "uniform"): (0.01e6, "profiles/philox_fill_fast_uniform_n2p26.md"),
    ("philox4x32_10", "normal_double"): (0.05e6, "profiles/philox_fill_fast_normal_double_n2p24.md"),
    ("mtgp32", "uint"): (2.2e6, "profiles/mtgp_fill_uint_n2p24.md"),
}


# Warp instructions per output value of each sweep kernel (sm__inst_executed.sum / n) from one
# ncu capture of the sweep at n = 2^24 (profiles/sweep_instructions_n2p24.md); the issue bound
# of a kernel is these instructions at 4 per SM per clock.  Filled from that capture.
NCU_INST_SOURCE = "profiles/sweep_instructions_n2p24.md"
NCU_INST = {
    ("philox4x32_10", "uint"): 0.3647,
    ("philox4x32_10", "uniform"): 0.4155,
    ("philox4x32_10", "uniform_double"): 0.8292,
    ("philox4x32_10", "uniform_half"): 0.2744,
    ("philox4x32_10", "normal[0.0, 1.0]"): 1.6415,
    ("philox4x32_10", "normal_double[0.0, 1.0]"): 4.2097,
    ("philox4x32_10", "log_normal[0.0, 1.0]"): 1.9227,
    ("philox4x32_10", "poisson[0.5]"): 0.6473,
    ("philox4x32_10", "poisson[10.0]"): 0.6482,
    ("philox4x32_10", "poisson[1000.0]"): 0.6567,
    ("xorwow", "uint"): 0.3291,
    ("xorwow", "uniform"): 0.3970,
    ("xorwow", "uniform_double"): 0.6548,
    ("xorwow", "uniform_half"): 0.2766,
    ("xorwow", "normal[0.0, 1.0]"): 1.5476,
    ("xorwow", "normal_double[0.0, 1.0]"): 3.9299,
    ("xorwow", "log_normal[0.0, 1.0]"): 1.8289,
    ("xorwow", "poisson[0.5]"): 0.6151,
    ("xorwow", "poisson[10.0]"): 0.6155,
    ("xorwow", "poisson[1000.0]"): 0.6190,
    ("mrg32k3a", "uint"): 1.2554,
    ("mrg32k3a", "uniform"): 1.2395,
    ("mrg32k3a", "uniform_double"): 1.2139,
    ("mrg32k3a", "uniform_half"): 0.7507,
    ("mrg32k3a", "normal[0.0, 1.0]"): 2.4856,
    ("mrg32k3a", "normal_double[0.0, 1.0]"): 4.6174,
    ("mrg32k3a", "log_normal[0.0, 1.0]"): 2.7668,
    ("mrg32k3a", "poisson[0.5]"): 1.5675,
    ("mrg32k3a", "poisson[10.0]"): 1.5679,
    ("mrg32k3a", "poisson[1000.0]"): 1.5714,
    ("lfsr113", "uint"): 0.7690,
    ("lfsr113", "uniform"): 0.8394,
    ("lfsr113", "uniform_double"): 1.5347,
    ("lfsr113", "uniform_half"): 0.4895,
    ("lfsr113", "normal[0.0, 1.0]"): 1.9692,
    ("lfsr113", "normal_double[0.0, 1.0]"): 4.7683,
    ("lfsr113", "log_normal[0.0, 1.0]"): 2.2505,
    ("lfsr113", "poisson[0.5]"): 1.0531,
    ("lfsr113", "poisson[10.0]"): 1.0535,
    ("lfsr113", "poisson[1000.0]"): 1.0570,
    ("mt19937", "uint"): 0.8396,
    ("mt19937", "uniform"): 0.9146,
    ("mt19937", "uniform_double"): 1.3757,
    ("mt19937", "uniform_half"): 0.6749,
    ("mt19937", "normal[0.0, 1.0]"): 2.2219,
    ("mt19937", "normal_double[0.0, 1.0]"): 4.9500,
    ("mt19937", "log_normal[0.0, 1.0]"): 2.5032,
    ("mt19937", "poisson[0.5]"): 1.1601,
    ("mt19937", "poisson[10.0]"): 1.1608,
    ("mt19937", "poisson[1000.0]"): 1.1660,
    ("threefry4x32_20", "uint"): 1.1911,
    ("threefry4x32_20", "uniform"): 1.2614,
    ("threefry4x32_20", "uniform_double"): 2.5036,
    ("threefry4x32_20", "uniform_half"): 0.6872,
    ("threefry4x32_20", "normal[0.0, 1.0]"): 2.4985,
    ("threefry4x32_20", "normal_double[0.0, 1.0]"): 5.7965,
    ("threefry4x32_20", "log_normal[0.0, 1.0]"): 2.7797,
    ("threefry4x32_20", "poisson[0.5]"): 1.4929,
    ("threefry4x32_20", "poisson[10.0]"): 1.4938,
    ("threefry4x32_20", "poisson[1000.0]"): 1.5023,
    ("mtgp32", "uint"): 1.1253,
    ("mtgp32", "uniform"): 1.1956,
    ("mtgp32", "uniform_double"): 2.9434,
    ("mtgp32", "uniform_half"): 0.8387,
    ("mtgp32", "normal[0.0, 1.0]"): 2.4131,
    ("mtgp32", "normal_double[0.0, 1.0]"): 5.4471,
    ("mtgp32", "log_normal[0.0, 1.0]"): 2.6944,
    ("mtgp32", "poisson[0.5]"): 1.7156,
    ("mtgp32", "poisson[10.0]"): 1.7160,
    ("mtgp32", "poisson[1000.0]"): 1.7199,
    ("mrg31k3p", "uint"): 1.4998,
    ("mrg31k3p", "uniform"): 1.4685,
    ("mrg31k3p", "uniform_double"): 1.4363,
    ("mrg31k3p", "uniform_half"): 0.8748,
    ("mrg31k3p", "normal[0.0, 1.0]"): 2.6685,
    ("mrg31k3p", "normal_double[0.0, 1.0]"): 4.8044,
    ("mrg31k3p", "log_normal[0.0, 1.0]"): 2.9497,
    ("mrg31k3p", "poisson[0.5]"): 1.7848,
    ("mrg31k3p", "poisson[10.0]"): 1.7852,
    ("mrg31k3p", "poisson[1000.0]"): 1.7887,
    ("threefry2x32_20", "uint"): 1.2033,
    ("threefry2x32_20", "uniform"): 1.2814,
    ("threefry2x32_20", "uniform_double"): 2.5471,
    ("threefry2x32_20", "uniform_half"): 0.6955,
    ("threefry2x32_20", "normal[0.0, 1.0]"): 2.6073,
    ("threefry2x32_20", "normal_double[0.0, 1.0]"): 5.9723,
    ("threefry2x32_20", "log_normal[0.0, 1.0]"): 2.8886,
    ("threefry2x32_20", "poisson[0.5]"): 1.4889,
    ("threefry2x32_20", "poisson[10.0]"): 1.4899,
    ("threefry2x32_20", "poisson[1000.0]"): 1.4983,
    ("threefry2x64_20", "uint"): 1.2759,
    ("threefry2x64_20", "uniform"): 2.6118,
    ("threefry2x64_20", "uniform_double"): 2.6899,
    ("threefry2x64_20", "uniform_half"): 0.7368,
    ("threefry2x64_20", "normal[0.0, 1.0]"): 2.6313,
    ("threefry2x64_20", "normal_double[0.0, 1.0]"): 6.1530,
    ("threefry2x64_20", "log_normal[0.0, 1.0]"): 2.9126,
    ("threefry2x64_20", "poisson[0.5]"): 2.9953,
    ("threefry2x64_20", "poisson[10.0]"): 2.9963,
    ("threefry2x64_20", "poisson[1000.0]"): 3.0074,
    ("threefry4x64_20", "uint"): 1.2798,
    ("threefry4x64_20", "uniform"): 2.6001,
    ("threefry4x64_20", "uniform_double"): 2.6783,
    ("threefry4x64_20", "uniform_half"): 0.7388,
    ("threefry4x64_20", "normal[0.0, 1.0]"): 2.6241,
    ("threefry4x64_20", "normal_double[0.0, 1.0]"): 6.1164,
    ("threefry4x64_20", "log_normal[0.0, 1.0]"): 2.9053,
    ("threefry4x64_20", "poisson[0.5]"): 3.0316,
    ("threefry4x64_20", "poisson[10.0]"): 3.0327,
    ("threefry4x64_20", "poisson[1000.0]"): 3.0437,
}


def ncu_traffic(gname, dist, out_bytes):
    """(DRAM bytes per launch, source) scaled from the capture, or (None, None)."""
    read, source = NCU_TRAFFIC.get((gname, dist), (None, None))
    if read is None:
        return None, None
    return int(read + out_bytes), "%s: state read %.2f MB per launch + the output written once" % (source, read / 1e6)


OUTPUT_KIND = {"uint": 0, "uniform": 4, "uniform_double": 5, "uniform_half": 6, "normal": 7,
               "normal_double": 8, "log_normal": 10, "poisson": 13, "char": 1, "short": 2}


def rank_stream(gtype, dist, rank, n):
    """(seed, output position or None) giving rank `rank` the outputs [rank*n, (rank+1)*n) of
    the stream of seed SEED: every generator with a position (counter and stateful engines,
    rocrand_b200_set_output_position) continues that one stream at output rank*n; MT19937
    and MTGP32, which have no position, take seed SEED + rank instead."""
    if gtype in NO_OFFSET:
        return SEED + rank, None
    return SEED, rank * n
SWEEP_DISTS = [
    ("uint", None), ("uniform", None), ("uniform_double", None), ("uniform_half", None),
    ("normal", (0.0, 1.0)), ("normal_double", (0.0, 1.0)), ("log_normal", (0.0, 1.0)),
    ("poisson", (0.5,)), ("poisson", (10.0,)), ("poisson", (1000.0,)),
]
ELEM = {"uint": 4, "uniform": 4, "uniform_double": 8, "uniform_half": 2, "normal": 4,
        "normal_double": 8, "log_normal": 4, "poisson": 4, "char": 1, "short": 2}
ENTRY = {"uint": "rocrand_generate", "uniform": "rocrand_generate_uniform",
         "uniform_double": "rocrand_generate_uniform_double",
         "uniform_half": "rocrand_generate_uniform_half", "normal": "rocrand_generate_normal",
         "normal_double": "rocrand_generate_normal_double",
         "log_normal": "rocrand_generate_log_normal", "poisson": "rocrand_generate_poisson"}


def call_args(dist, params):
    if params is None:
        return []
    if dist in ("normal", "log_normal"):
        return [ctypes.c_float(params[0]), ctypes.c_float(params[1])]
    if dist in ("normal_double", "log_normal_double"):
        return [ctypes.c_double(params[0]), ctypes.c_double(params[1])]
    return [ctypes.c_double(params[0])]


def stream_offset(dist, first_value):
    """Engine offset that starts a stream slice at output `first_value` (aligned outputs):
    inputs per output = iw/ow of the distribution."""
    per = {"uniform_double": 2.0, "normal_double": 2.0, "log_normal_double": 2.0,
           "uniform_half": 0.5, "char": 0.25, "short": 0.5}.get(dist, 1.0)
    return int(first_value * per)


def measured_peak():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to print its first sample: wait for it so the
            # timed region is covered from its start.
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def select_calls(only):
    """The sweep's calls, optionally filtered by "gen:dist[:param],..." (e.g. the single
    kernel an ncu capture looks at)."""
    calls = [(gname, gtype, d, p) for gname, gtype in SWEEP_GENERATORS for d, p in SWEEP_DISTS]
    if not only:
        return calls
    keep = []
    for item in only.split(","):
        parts = item.split(":")
        for c in calls:
            if c[0] == parts[0] and c[2] == parts[1] and (
                    len(parts) < 3 or (c[3] is not None and float(parts[2]) == c[3][0])):
                keep.append(c)
    if not keep:
        raise SystemExit("--only matched no call: %s" % only)
    return keep


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ------------------------------------------------------------------------------------
# our arm


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import rocrand_b200 as rb
    lib = rb.load_library()

    n = args.n
    calls = select_calls(args.only)
    max_bytes = max(ELEM[d] for _, _, d, _ in calls) * n
    out = torch.empty(max_bytes, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    gens = {}
    for gname, gtype, d, p in calls:
        g = c_void_p()
        rb.check_rocrand(lib.rocrand_create_generator(ctypes.byref(g), gtype))
        seed, pos = rank_stream(gtype, d, rank, n)
        rb.check_rocrand(lib.rocrand_set_seed(g, seed))
        if pos is not None and pos > 0:
            rb.check_rocrand(lib.rocrand_b200_set_output_position(g, OUTPUT_KIND[d], pos))
        rb.check_rocrand(lib.rocrand_set_stream(g, c_void_p(stream.cuda_stream)))
        gens[(gname, d, p)] = g

    def one_call(c, ptr):
        gname, gtype, d, p = c
        st = getattr(lib, ENTRY[d])(gens[(gname, d, p)], c_void_p(ptr), c_size_t(n), *call_args(d, p))
        if st != 0:
            raise rb.RocRandError(st)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        for c in calls:
            one_call(c, out.data_ptr())
    barrier()

    sampler = ClockSampler(local)
    sampler.start()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(len(calls) + 1)] for _ in range(args.steps)]
    barrier()
    for s in range(args.steps):
        evs[s][0].record(stream)
        for i, c in enumerate(calls):
            one_call(c, out.data_ptr())
            evs[s][i + 1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    step_ms = [evs[s][0].elapsed_time(evs[s][-1]) for s in range(args.steps)]
    per_call_ms = [[evs[s][i].elapsed_time(evs[s][i + 1]) for i in range(len(calls))] for s in range(args.steps)]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    step_bytes = sum(ELEM[d] * n for _, _, d, _ in calls)
    value = step_bytes * world * args.steps / (total_ms * 1e-3) / 1e9

    # per-kernel rooflines: achieved write GB/s against the smaller of the measured HBM peak
    # and the kernel's issue bound (NCU_INST at the sampled clock); the dominant kernel is the
    # call with the largest device time in the step
    mean_call = [statistics.mean(per_call_ms[s][i] for s in range(args.steps)) for i in range(len(calls))]
    peak, peak_kind = measured_peak()

    def kernel_roof(i):
        gname, _, d, p = calls[i]
        b = ELEM[d] * n
        gbs = b / (mean_call[i] * 1e-3) / 1e9
        iss, iss_src = issue_bound(gname, d + ("" if p is None else str(list(p))), ELEM[d], n,
                                   clocks.get("sm_mhz"))
        bound = "issue" if iss is not None and iss < peak else "hbm"
        lim = min(peak, iss) if iss is not None else peak
        return {"kernel": "%s %s%s" % (gname, d, "" if calls[i][3] is None else list(calls[i][3])),
                "bytes": b, "gbs": gbs, "hbm_frac": gbs / peak,
                "issue_gbs": iss, "issue_frac": (gbs / iss) if iss else None, "bound": bound,
                "frac": gbs / lim, "issue_source": iss_src}

    roofs = [kernel_roof(i) for i in range(len(calls))]
    dom = max(range(len(calls)), key=lambda i: mean_call[i])
    ns = [i for i, c in enumerate(calls) if c[0] == "philox4x32_10" and c[2] == "uniform"]

    # e2e through the same C ABI with pinned host output, copies inside the timed region
    e2e_steps = 0 if args.sweep_only else max(1, min(args.steps, 3))
    host = torch.empty(max_bytes if e2e_steps else 1, dtype=torch.uint8, pin_memory=True)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    d2h = 0
    for _ in range(e2e_steps):
        for c in calls:
            one_call(c, out.data_ptr())
            nb = ELEM[c[2]] * n
            host[:nb].copy_(out[:nb], non_blocking=True)
            d2h += nb
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = step_bytes * world * e2e_steps / (e2e_ms * 1e-3) / 1e9 if e2e_steps else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.sweep_only:
        cpu = cpu_baseline_sample(args.cpu_n, calls)

    quasi = config1 = None
    if rank == 0 and world == 1 and not args.sweep_only:
        config1 = config1_leg(lib)
        if not args.no_quasi:
            del out
            torch.cuda.empty_cache()
            out = None
            quasi = quasi_leg(lib, max(3, min(args.steps, 10)))

    refk = None
    if rank == 0 and world == 1 and not args.sweep_only and not args.no_ref_kernels:
        if out is not None:
            del out
            out = None
        torch.cuda.empty_cache()
        refk = ref_kernels_leg(lib, calls, n, mean_call, 3)

    batched = serving = None
    if rank == 0 and world == 1 and not args.no_batched and not args.sweep_only:
        del out
        torch.cuda.empty_cache()
        batched = batched_leg(lib, not args.quick_batched)
        torch.cuda.empty_cache()
        serving = serving_leg(lib, args.full_configs)

    for g in gens.values():
        lib.rocrand_destroy_generator(g)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()

    if rank != 0:
        return
    dr = roofs[dom]
    dom_bytes = dr["bytes"]
    line = {
        "metric": "output GB/s of rocrand_generate_* (bit-exact vs reference host generators)",
        "value": round(value, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32/f32/f64/f16 outputs, int32 engine arithmetic",
        "data": "synthetic: seeded generator streams (seed 0xdeadbeef), no input data",
        "config": {
            "workload": "plain single-generator sweep, n=2^28 values per call, %d generator families x %d "
                        "distributions" % (len(SWEEP_GENERATORS), len(SWEEP_DISTS)),
            "n_per_call": n,
            "bytes_per_step_per_gpu": step_bytes,
            "l2": "outputs 0.5-2 GiB per call > 126 MB L2; no flush needed",
            "parallelism": "replica shards: rank r fills stream slice [r*n, (r+1)*n)",
            "families": ",".join(g for g, _ in SWEEP_GENERATORS),
        },
        "roofline": {
            "bound": dr["bound"],
            "kernel": dr["kernel"],
            "achieved": round(dr["gbs"], 1),
            "peak": round(min(peak, dr["issue_gbs"]) if dr["issue_gbs"] else peak, 1),
            "unit": "GB/s",
            "frac": round(dr["frac"], 4),
            "hbm_peak": peak,
            "hbm_frac": round(dr["hbm_frac"], 4),
            "issue_frac": round(dr["issue_frac"], 4) if dr["issue_frac"] else None,
            "peak_source": ("HBM: %s copy bandwidth (MEASURED_PEAKS.json); issue: %s" % (
                peak_kind, dr["issue_source"])) if peak_kind == "measured" else "fallback 6650 GB/s",
            "traffic": ncu_traffic(calls[dom][0], calls[dom][2], dom_bytes)[0],
            "traffic_source": ncu_traffic(calls[dom][0], calls[dom][2], dom_bytes)[1],
            "algorithmic_bytes_per_launch": dom_bytes,
            "headline_kernel": ("philox4x32_10 uniform fp32 2^28: %.1f GB/s = %.3f of HBM peak" % (
                roofs[ns[0]]["gbs"], roofs[ns[0]]["hbm_frac"])) if ns else None,
            "config1": config1,
            "quasi_gbs": quasi["gbs"] if quasi else None,
            "vs_reference_kernels": ({k: refk[k] for k in ("speedup", "min_kernel_speedup", "ours_gbs", "ref_gbs",
                                                           "identical_bit_exact_outputs")}
                                     if refk and "speedup" in refk else refk),
        },
        "e2e": {"value": round(e2e_value, 2) if e2e_value else None, "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": step_bytes,
                "how": "same C-ABI calls + D2H copy of every output to pinned host memory, %d steps" % e2e_steps},
        "gpu_launches": len(calls) * args.steps,
        "clocks": clocks,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    # every kernel (device ms, fraction of its governing bound, that bound) and the full
    # comparison with the reference's kernels go to a details file beside the bench; the line
    # keeps their summaries, so that it stays short enough to be kept whole
    per_kernel = {r["kernel"]: [round(mean_call[i], 4), round(r["frac"], 3), r["bound"]] for i, r in enumerate(roofs)}
    details_path = os.path.join(HERE, "bench_details.json")
    try:
        with open(details_path, "w") as fh:
            json.dump({"per_kernel": per_kernel, "reference_kernels": refk}, fh, indent=1)
        line["details"] = os.path.basename(details_path)
    except OSError:
        line["details"] = None
    fracs = sorted(v[1] for v in per_kernel.values())
    slowest = sorted(per_kernel.items(), key=lambda kv: -kv[1][0])[:6]
    line["per_kernel_summary"] = {
        "kernels": len(per_kernel), "frac_min": fracs[0], "frac_median": fracs[len(fracs) // 2],
        "bound_counts": {b: sum(1 for v in per_kernel.values() if v[2] == b) for b in ("hbm", "issue")},
        "slowest_ms_frac_bound": {k: v for k, v in slowest}}
    if refk is not None:
        line["reference_kernels"] = {k: v for k, v in refk.items()
                                     if k not in ("per_kernel_ms_ours_ref_ratio", "ref_normals_outside_host_bound")}
        outside = refk.get("ref_normals_outside_host_bound") or {}
        if outside:
            line["reference_kernels"]["ref_normals_outside_host_bound_max"] = max(outside.values())
    if quasi is not None:
        line["quasi"] = quasi
    if batched is not None:
        line["batched_fill"] = batched
    if serving is not None:
        line["serving"] = serving
    print(json.dumps(line))


def quasi_leg(lib, reps, only=""):
    """The quasi-random workload: Sobol32 and scrambled Sobol64, 1 / 64 / 1000 dimensions x
    2^20 points per dimension at offset 4096, uniform fp64 and normal fp32, dimension-major.
    Each case: one generator, 2 untimed calls, then `reps` calls timed with CUDA events on
    its stream (every call continues the sequence).  Output GB/s per case and over all."""
    import torch
    import rocrand_b200 as rb
    stream = torch.cuda.current_stream()
    out = torch.empty(max(QUASI_DIMS) * (1 << 20) * 8, dtype=torch.uint8, device="cuda")
    res, tot_b, tot_ms = {}, 0, 0.0
    for gname, gtype in QUASI_GENERATORS:
        for dims in QUASI_DIMS:
            for d, p in QUASI_DISTS:
                if only and only != "%s:%s:%d" % (gname, d, dims):
                    continue
                g = c_void_p()
                rb.check_rocrand(lib.rocrand_create_generator(ctypes.byref(g), gtype))
                rb.check_rocrand(lib.rocrand_set_quasi_random_generator_dimensions(g, dims))
                rb.check_rocrand(lib.rocrand_set_offset(g, 4096))
                rb.check_rocrand(lib.rocrand_set_stream(g, c_void_p(stream.cuda_stream)))
                n = dims << 20
                fn = getattr(lib, ENTRY[d])

                def call():
                    st = fn(g, c_void_p(out.data_ptr()), c_size_t(n), *call_args(d, p))
                    if st != 0:
                        raise rb.RocRandError(st)

                for _ in range(2):
                    call()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                for _ in range(reps):
                    call()
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / reps
                lib.rocrand_destroy_generator(g)
                b = n * ELEM[d]
                res["%s/%s/d%d" % (gname, "f64" if d == "uniform_double" else "nf32", dims)] = round(
                    b / (ms * 1e-3) / 1e9, 1)
                tot_b += b
                tot_ms += ms
    del out
    return {"gbs": round(tot_b / (tot_ms * 1e-3) / 1e9, 1) if tot_ms else None, "cases": res,
            "workload": "2^20 points/dim, offset 4096, %d calls each" % reps}


def config1_leg(lib):
    """The small reference case: Philox4x32-10, seed 1234, offset 0, uniform fp32, 2^24 values
    into a 256-byte aligned buffer -- its SHA-256 against the digest recorded from the
    reference's own host generator, and its device time."""
    import hashlib
    import torch
    import rocrand_b200 as rb
    n = 1 << 24
    with open(os.path.join(HERE, "tests", "golden", "full_digests.json")) as f:
        want = json.load(f).get("philox/uniform/seed1234/2^24", {}).get("sha256")
    stream = torch.cuda.current_stream()
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    g = c_void_p()
    rb.check_rocrand(lib.rocrand_create_generator(ctypes.byref(g), 404))
    rb.check_rocrand(lib.rocrand_set_stream(g, c_void_p(stream.cuda_stream)))
    times = []
    for _ in range(6):
        rb.check_rocrand(lib.rocrand_set_seed(g, 1234))  # every call writes the same values
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rb.check_rocrand(lib.rocrand_generate_uniform(g, c_void_p(out.data_ptr()), c_size_t(n)))
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    lib.rocrand_destroy_generator(g)
    got = hashlib.sha256(out.cpu().numpy().view("u1").data).hexdigest()
    ms = statistics.median(times[1:])
    return {"bit_exact_vs_reference": got == want, "ms": round(ms, 4),
            "gbs": round(4 * n / (ms * 1e-3) / 1e9, 1)}


REF_GPU_PATH = os.path.join(HERE, "oracle", "_ref", "librocrand_ref_gpu.so")
BIT_EXACT = {"uint", "uniform", "uniform_double", "uniform_half", "poisson"}


def ref_kernels_leg(lib, calls, n, ours_ms, reps):
    """The reference's own device kernels on the same B200: its sources compiled for sm_100a
    (oracle/_ref/librocrand_ref_gpu.so, built by oracle/Makefile.ref gpu), the same sweep
    through its own rocrand_generate_* entry points, each call timed with CUDA events like
    ours.  Per kernel: our time and the reference's; bit-exact outputs of the first call on
    fresh generators are compared byte for byte."""
    import torch
    import rocrand_b200 as rb
    if not os.path.exists(REF_GPU_PATH):
        return {"unavailable": "oracle/_ref/librocrand_ref_gpu.so not built"}
    ref = rb.load_library(REF_GPU_PATH)
    stream = torch.cuda.current_stream()
    nbytes = max(ELEM[d] for _, _, d, _ in calls) * n
    a = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    b = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    per, same, compared, ours_tot, ref_tot = {}, 0, 0, 0.0, 0.0
    ulps = {}
    for i, (gname, gtype, d, p) in enumerate(calls):
        gens, fns = [], []
        for L, buf in ((lib, a), (ref, b)):
            g = c_void_p()
            rb.check_rocrand(L.rocrand_create_generator(ctypes.byref(g), gtype))
            rb.check_rocrand(L.rocrand_set_seed(g, SEED))
            rb.check_rocrand(L.rocrand_set_stream(g, c_void_p(stream.cuda_stream)))
            fn = getattr(L, ENTRY[d])
            # first call on a fresh generator: the outputs compared below
            rb.check_rocrand(fn(g, c_void_p(buf.data_ptr()), c_size_t(n), *call_args(d, p)))
            gens.append((L, g))
            fns.append((fn, buf))
        torch.cuda.synchronize()
        nb = ELEM[d] * n
        if d in BIT_EXACT:
            compared += 1
            same += int(torch.equal(a[:nb], b[:nb]))
        elif d in ("normal", "normal_double"):
            # share of the reference kernel's normals farther than the host-parity bound (4 ulp
            # fp32, 2 ulp fp64) from ours, which are within it of the reference's host output:
            # the reference's kernels use the fast __sincosf / sincospi device functions
            it, tol = (torch.int32, 4) if d == "normal" else (torch.int64, 2)
            x, y = a[:nb].view(it), b[:nb].view(it)
            far = ((x >= 0) != (y >= 0)) | ((x - y).abs() > tol)
            ulps["%s %s" % (gname, d)] = round(float(far.sum().item()) / (nb // (4 if d == "normal" else 8)), 6)
        ms = []
        for (L, g), (fn, buf) in zip(gens, fns):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                rb.check_rocrand(fn(g, c_void_p(buf.data_ptr()), c_size_t(n), *call_args(d, p)))
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1) / reps)
            L.rocrand_destroy_generator(g)
        key = "%s %s%s" % (gname, d, "" if p is None else list(p))
        per[key] = [round(ms[0], 4), round(ms[1], 4), round(ms[1] / ms[0], 2)]
        ours_tot += ms[0]
        ref_tot += ms[1]
    del a, b
    torch.cuda.empty_cache()
    step_bytes = sum(ELEM[d] * n for _, _, d, _ in calls)
    ratios = sorted(v[2] for v in per.values())
    return {"ours_gbs": round(step_bytes / (ours_tot * 1e-3) / 1e9, 1),
            "ref_gbs": round(step_bytes / (ref_tot * 1e-3) / 1e9, 1),
            "speedup": round(ref_tot / ours_tot, 2),
            "min_kernel_speedup": ratios[0], "median_kernel_speedup": ratios[len(ratios) // 2],
            "identical_bit_exact_outputs": "%d of %d" % (same, compared),
            "ref_normals_outside_host_bound": ulps,
            "per_kernel_ms_ours_ref_ratio": per}


def issue_bound(gname, dist_key, elem, n, clock_mhz):
    """(GB/s that the instruction issue rate allows, source) for one sweep kernel: warp
    instructions per output value from the ncu capture in NCU_INST, issued at most 4 per SM
    per clock on 148 SMs at the sampled SM clock; (None, None) where no capture exists."""
    per_value = NCU_INST.get((gname, dist_key))
    if per_value is None or not clock_mhz:
        return None, None
    secs = per_value * n / (148 * 4 * clock_mhz * 1e6)
    return elem * n / secs / 1e9, "%s: %.3f warp instructions per value" % (NCU_INST_SOURCE, per_value)


# ------------------------------------------------------------------------------------
# reference host generators (CPU)


def splitmix64(i):
    """SplitMix64 output for input i (Steele, Lea and Flood 2014; the mixing constants as
    published by Vigna): the seeds of the batched-fill generators."""
    m = (1 << 64) - 1
    z = (i + 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


def _entry_args(d, p0, p1):
    """(entry point, trailing arguments) of the plain call for batch distribution d."""
    if d == 1:
        return "rocrand_generate_uniform", []
    if d == 3:
        return "rocrand_generate_normal", [ctypes.c_float(p0), ctypes.c_float(p1)]
    if d == 4:
        return "rocrand_generate_poisson", [ctypes.c_double(p0)]
    if d == 2:
        return "rocrand_generate_uniform_double", []
    return "rocrand_generate", []


def batched_leg(lib, full):
    """Batched fill: 4096 Philox4x32-10 + 4096 XORWOW fresh generators (seed_i = splitmix64(i),
    offset 0), sizes log-uniform in [2^10, 2^24] (numpy PCG64 seed 42), 50% uniform fp32 /
    30% normal fp32 / 20% Poisson lambda=4; one persistent launch replayed from a CUDA graph
    versus one plain call per generator (set_seed + generate, so every pass writes the same
    values).  With --quick-batched a quarter of the requests (1024 + 1024)."""
    import numpy as np
    import torch
    import rocrand_b200 as rb
    per = 4096 if full else 1024
    count = 2 * per
    rs = np.random.Generator(np.random.PCG64(42))
    sizes = np.exp(rs.uniform(np.log(2.0 ** 10), np.log(2.0 ** 24), count)).astype(np.int64)
    u = rs.random(count)
    dists = np.where(u < 0.5, 1, np.where(u < 0.8, 3, 4))
    types = [rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10] * per + [rb.ROCRAND_RNG_PSEUDO_XORWOW] * per
    seeds = [splitmix64(i) for i in range(count)]
    offs, total = [], 0
    for n in sizes:
        offs.append(total)
        total += (int(n) * 4 + 511) // 512 * 512
    out = torch.zeros(total, dtype=torch.uint8, device="cuda")
    base = out.data_ptr()
    stream = torch.cuda.current_stream()
    reqs = (rb.BatchRequest * count)()
    params = {1: (0.0, 0.0), 3: (0.0, 1.0), 4: (4.0, 0.0)}
    for k in range(count):
        p0, p1 = params[int(dists[k])]
        reqs[k] = rb.BatchRequest(types[k], int(dists[k]), seeds[k], 0, p0, p1, base + offs[k], int(sizes[k]))
    byte_count = int(sizes.sum()) * 4

    def checksum():
        # two sums over 1 GiB slices (no temporary larger than a slice's int64 widening)
        torch.cuda.synchronize()
        a = b = 0
        words = out.view(torch.int32)
        step = 1 << 28
        for i in range(0, words.numel(), step):
            w = words[i:i + step]
            a += int(w.sum(dtype=torch.int64).item())
            b += int((w.to(torch.int64) * ((i // step) % 7 + 1)).sum().item())
        return a, b

    def timed(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    # plain: one generator per request, re-seeded every pass (the XORWOW arena re-initialises)
    gens = []
    for k in range(count):
        g = ctypes.c_void_p()
        rb.check_rocrand(lib.rocrand_create_generator(ctypes.byref(g), types[k]))
        rb.check_rocrand(lib.rocrand_set_stream(g, c_void_p(stream.cuda_stream)))
        gens.append(g)
    calls = [(gens[k], seeds[k], getattr(lib, _entry_args(int(dists[k]), *params[int(dists[k])])[0]),
              c_void_p(base + offs[k]), c_size_t(int(sizes[k])),
              _entry_args(int(dists[k]), *params[int(dists[k])])[1]) for k in range(count)]

    def plain_pass():
        for g, seed, fn, ptr, n, extra in calls:
            lib.rocrand_set_seed(g, seed)
            fn(g, ptr, n, *extra)

    plain_ms = timed(plain_pass, 2)
    # the plain pass's bytes kept for a byte comparison when the device has room for a copy,
    # else two checksums of them
    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # earlier legs' cached blocks back to the device first
    free_bytes, _ = torch.cuda.mem_get_info()
    keep = out.clone() if free_bytes > out.numel() + (8 << 30) else None
    plain_sum = checksum() if keep is None else None
    out.zero_()
    rb.check_rocrand(lib.rocrand_b200_autotune_batch(c_void_p(stream.cuda_stream)))
    plan = c_void_p()
    rb.check_rocrand(lib.rocrand_b200_create_batch_plan(ctypes.byref(plan), reqs, count,
                                                        c_void_p(stream.cuda_stream)))
    batch_ms = timed(lambda: lib.rocrand_b200_execute_batch_plan(plan, 1, c_void_p(stream.cuda_stream)), 5)
    torch.cuda.synchronize()
    if keep is not None:
        step = 1 << 30  # slices, so that the comparison's temporary stays at 1 GiB
        identical = all(bool(torch.equal(out[i:i + step], keep[i:i + step])) for i in range(0, out.numel(), step))
    else:
        identical = plain_sum == checksum()
    compared  = "bytes" if keep is not None else "checksums"
    del keep
    lib.rocrand_b200_destroy_batch_plan(plan)
    for g in gens:
        lib.rocrand_destroy_generator(g)
    del out
    return {"requests": count, "bytes_per_pass": byte_count,
            "batched_gbs": round(byte_count / (batch_ms * 1e-3) / 1e9, 1),
            "plain_gbs": round(byte_count / (plain_ms * 1e-3) / 1e9, 1),
            "speedup": round(plain_ms / batch_ms, 2), "batched_ms": round(batch_ms, 3),
            "plain_ms": round(plain_ms, 3), "identical_outputs": identical,
            "compared": compared,
            "graph_replay": True, "autotuned": True,
            "sizes": "log-uniform [2^10, 2^24], PCG64 seed 42",
            "mix": "50% uniform fp32 / 30% normal fp32 / 20% Poisson 4"}


def serving_rates(lib, types):
    """Per-request costs of plain calls, for the bound of the batched/plain ratio: the device
    throughput of each (generator, dtype) at 2^24 values, and the wall time per call of
    back-to-back tiny calls on one stream (the launch floor a per-request server pays)."""
    import torch
    import rocrand_b200 as rb
    stream = torch.cuda.current_stream()
    buf = torch.empty(8 << 24, dtype=torch.uint8, device="cuda")
    entries = {0: "rocrand_generate", 1: "rocrand_generate_uniform", 2: "rocrand_generate_uniform_double"}
    bw, floor = {}, None
    for t in types:
        g = c_void_p()
        rb.check_rocrand(lib.rocrand_create_generator(ctypes.byref(g), t))
        rb.check_rocrand(lib.rocrand_set_stream(g, c_void_p(stream.cuda_stream)))
        for d, fname in entries.items():
            fn = getattr(lib, fname)
            n = 1 << 24
            for _ in range(2):
                fn(g, c_void_p(buf.data_ptr()), c_size_t(n))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(5):
                fn(g, c_void_p(buf.data_ptr()), c_size_t(n))
            e1.record(stream)
            torch.cuda.synchronize()
            bw[(t, d)] = n * (8 if d == 2 else 4) / (e0.elapsed_time(e1) / 5 * 1e-3)
        if t == types[0]:
            fn = lib.rocrand_generate_uniform
            for _ in range(50):
                fn(g, c_void_p(buf.data_ptr()), c_size_t(256))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(1000):
                fn(g, c_void_p(buf.data_ptr()), c_size_t(256))
            torch.cuda.synchronize()
            floor = (time.perf_counter() - t0) / 1000
        lib.rocrand_destroy_generator(g)
    del buf
    return bw, floor


def serving_leg(lib, full):
    """Serving: Poisson arrivals at 1k-50k req/s over 64 handles (16 each of Philox,
    XORWOW, MRG32k3a, Sobol32; states resident), sizes log-uniform in [2^8, 2^26], dtypes
    uniform over fp32 / fp64 / uint32, a 64 GB output budget; the continuous-batching server
    and the plain per-request server replay the same trace.  Also a saturated trace (every
    request at t=0).  Requests per trace: 10^5 at 50k req/s, 2000 for the saturated trace,
    max(10^4, one second of arrivals) otherwise, so that each p99 rests on 100 or more
    requests (10^5 at every rate with --full-configs).  For the saturated trace the report includes the bound of the
    batched/plain ratio that the mix allows: sum over requests of max(launch floor, device
    time) / sum of device times (serving_rates)."""
    import numpy as np
    import rocrand_b200 as rb
    types = [rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10, rb.ROCRAND_RNG_PSEUDO_XORWOW,
             rb.ROCRAND_RNG_PSEUDO_MRG32K3A, rb.ROCRAND_RNG_QUASI_SOBOL32]
    budget = 64 << 30
    rates = [1000, 5000, 10000, 20000, 50000, None]
    bw, floor = serving_rates(lib, types)
    results = {}
    for mode in ("batched", "plain"):
        server = c_void_p()
        rb.check_rocrand(lib.rocrand_b200_server_create(ctypes.byref(server), budget, 3,
                                                        1 if mode == "plain" else 0))
        handles = []
        htype = []
        for t in types:
            for k in range(16):
                h = ctypes.c_uint()
                rb.check_rocrand(lib.rocrand_b200_server_add_generator(server, t, splitmix64(len(handles)),
                                                                       ctypes.byref(h)))
                handles.append(h.value)
                htype.append(t)
        for rate in rates:
            rs = np.random.Generator(np.random.PCG64(7))
            n = 100000 if (full or rate == 50000) else (2000 if rate is None else max(10000, rate))
            gaps = rs.exponential(1.0 / rate, n) if rate else np.zeros(n)
            arrivals = np.cumsum(gaps) if rate else gaps
            hidx = rs.integers(0, len(handles), n)
            dts = rs.integers(0, 3, n)  # uint32, fp32, fp64
            sizes = np.exp(rs.uniform(np.log(2.0 ** 8), np.log(2.0 ** 26), n)).astype(np.int64)
            items = (rb.TraceItem * n)()
            nbytes = 0
            dev_s = plain_s = 0.0
            for i in range(n):
                items[i] = rb.TraceItem(float(arrivals[i]), handles[hidx[i]], int(dts[i]), 0.0, 0.0,
                                        int(sizes[i]))
                b = int(sizes[i]) * (8 if dts[i] == 2 else 4)
                nbytes += b
                t_dev = b / bw[(htype[hidx[i]], int(dts[i]))]
                dev_s += t_dev
                plain_s += max(floor, t_dev)
            lat = (ctypes.c_double * n)()
            wall = ctypes.c_double()
            rb.check_rocrand(lib.rocrand_b200_server_run_trace(server, items, n, lat, ctypes.byref(wall)))
            l = np.ctypeslib.as_array(lat)
            key = "saturated" if rate is None else "%d_req_s" % rate
            ent = results.setdefault(key, {"requests": n})
            ent[mode] = {"gbs": round(nbytes / wall.value / 1e9, 1),
                         "p50_ms": round(float(np.percentile(l, 50)) * 1e3, 3),
                         "p99_ms": round(float(np.percentile(l, 99)) * 1e3, 3), "wall_s": round(wall.value, 3)}
            if rate is None:
                ent["ratio_bound"] = round(plain_s / dev_s, 3)
                ent["kernel_time_s"] = round(dev_s, 3)
        rb.check_rocrand(lib.rocrand_b200_server_destroy(server))
    for v in results.values():
        if "batched" in v and "plain" in v:
            v["gbs_ratio"] = round(v["batched"]["gbs"] / v["plain"]["gbs"], 3)
            if "ratio_bound" in v:
                v["of_bound"] = round(v["gbs_ratio"] / v["ratio_bound"], 3)
    return {"budget_bytes": budget, "handles": 64, "streams": 3, "launch_floor_us": round(floor * 1e6, 2),
            "sizes": "log-uniform [2^8, 2^26]", "dtypes": "uint32/fp32/fp64", "rates": results}


def _ref_lib():
    from oracle import pyorc
    if os.path.exists(pyorc.REF_PATH):
        return pyorc.CLib("ref"), "reference"
    return pyorc.CLib("orc"), "port"


_SEEDED = {}  # host generators per (call, threads, size): created, seeded and warmed once


def cpu_sample(n_per_call, calls, threads):
    """Runs every call of the sweep on the reference's host generators, n_per_call values
    each, split over `threads` host threads, each its own generator on its own slice of the
    stream (an offset slice; MT19937 and MTGP32, which have no offset, a seed of their own).
    The generators are created, seeded and run once untimed the first time a call is sampled
    (the host generators seed their 131072 or 8192 engines on the first call), and later
    samples continue their streams, so the timed region is steady-state generation, as on the
    GPU.  The reference's host MT19937 spends minutes seeding its 8192 generators, so those
    are the C port's.  Returns (bytes, seconds, kind)."""
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor
    from oracle import pyorc
    ref_lib, kind = _ref_lib()
    total_bytes = 0
    t_all = 0.0
    for gname, gtype, d, p in calls:
        lib = pyorc.CLib("orc") if gtype in PORT_SEEDED else ref_lib
        suffix, dt, _ = pyorc.DISTS[d]
        buf = np.empty(n_per_call + 64, dtype=dt)
        base = (-buf.ctypes.data // buf.itemsize) % (64 // buf.itemsize)
        view = buf[base:base + n_per_call]
        chunk = (n_per_call // threads) // 64 * 64
        bounds = [(i * chunk, (i + 1) * chunk if i < threads - 1 else n_per_call) for i in range(threads)]
        fn = lib.fn(suffix)
        args = pyorc.dist_args(d, p if p is not None else ())
        key = (gtype, threads, n_per_call)  # one set of generators per family

        def work(i, gens, out):
            a, b = bounds[i]
            return fn(gens[i], c_void_p(out[a:b].ctypes.data), c_size_t(b - a), *args)

        if key not in _SEEDED:
            gens = []
            for i, (a, b) in enumerate(bounds):
                g = lib.create(gtype)
                if gtype in NO_OFFSET:
                    lib.set_seed(g, SEED + i)
                else:
                    lib.set_seed(g, SEED)
                    lib.set_offset(g, a)
                gens.append(g)
            with ThreadPoolExecutor(threads) as ex:
                assert all(s == 0 for s in ex.map(lambda i: work(i, gens, view), range(threads)))
            _SEEDED[key] = gens
        gens = _SEEDED[key]
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            sts = list(ex.map(lambda i: work(i, gens, view), range(threads)))
        t_all += time.perf_counter() - t0
        assert all(s == 0 for s in sts), sts
        total_bytes += n_per_call * buf.itemsize
    return total_bytes, t_all, kind


def cpu_baseline_sample(n_per_call, calls):
    threads = os.cpu_count() or 1
    nb, secs, kind = cpu_sample(n_per_call, calls, threads)
    one_n = max(1 << 16, n_per_call // 16)
    nb1, secs1, _ = cpu_sample(one_n, calls, 1)
    return {"value": round(nb / secs / 1e9, 3), "unit": "GB/s", "cores": threads, "kind": kind,
            "value_1core": round(nb1 / secs1 / 1e9, 4),
            "sample": "same sweep at n=%d values per call (1 core: n=%d) vs 2^28 on the GPU; "
                      "%d host threads, each its own host generator on a disjoint offset slice" % (
                          n_per_call, one_n, threads)}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    calls = select_calls(args.only)
    threads = os.cpu_count() or 1
    # each step a bounded sample of the sweep (2^23 values per call, 1/32 of the GPU's 2^28),
    # so that the default 20 + 5 steps end within a few minutes; the first sample of each
    # call creates and warms its generators untimed
    step_n = args.cpu_n
    for _ in range(args.warmup):
        cpu_sample(step_n, calls, threads)
    nb = 0
    secs = 0.0
    kind = None
    for _ in range(args.steps):
        b, s, kind = cpu_sample(step_n, calls, threads)
        nb += b
        secs += s
    value = nb / secs / 1e9
    line = {
        "impl": "reference",
        "metric": "output GB/s of rocrand_generate_* (bit-exact vs reference host generators)",
        "value": round(value, 3),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(secs / args.steps * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32/f32/f64/f16 outputs, int32 engine arithmetic",
        "data": "synthetic: seeded generator streams (seed 0xdeadbeef), no input data",
        "config": {"workload": "plain single-generator sweep, n=2^28 values per call (sampled)",
                   "families": ",".join(g for g, _ in SWEEP_GENERATORS), "n_per_call_sampled": step_n},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": kind,
                         "sample": "n=%d values per call per step, %d threads" % (step_n, threads)},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 28)
    ap.add_argument("--cpu-n", type=int, default=1 << 23)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", default="", help="gen:dist[:param],... subset of the sweep")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-fill and serving legs")
    ap.add_argument("--no-quasi", action="store_true", help="skip the quasi-random (Sobol) leg")
    ap.add_argument("--quasi-only", action="store_true",
                    help="only the quasi-random leg (--only sobol32:normal:64 picks one case), --steps calls each")
    ap.add_argument("--no-ref-kernels", action="store_true",
                    help="skip timing the reference's own device kernels (oracle/_ref gpu build)")
    ap.add_argument("--sweep-only", action="store_true",
                    help="only the timed sweep (no e2e, CPU, config-1, quasi, batched or serving legs): "
                         "the form profiled under ncu")
    ap.add_argument("--full-configs", action="store_true", help="serving with 10^5 requests per rate")
    ap.add_argument("--quick-batched", action="store_true",
                    help="batched-fill leg on 1024 + 1024 generators instead of 4096 + 4096")
    args = ap.parse_args()
    if args.quasi_only:
        # the quasi-random leg alone (one case with --only gen:dist:dims), for profiling
        import torch
        import rocrand_b200 as rb
        torch.cuda.set_device(0)
        print(json.dumps(quasi_leg(rb.load_library(), args.steps, args.only)))
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
