"""Groth16 prove benchmark on B200 (BN254), one JSON line on stdout.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload poseidon2048|poseidon4096|matmul32]

Metric: Groth16 prove milliseconds for a 2^20-constraint circuit (the poseidon
circuit with 2048 hashes at sparse density: 899,072 constraints padded to 2^20
rows, 903,169 variables padded to 2^20 columns), lower is better.  A "step" is
one full prove (SpMV, the 7-transform quotient chain, 4 G1 MSMs and 1 G2 MSM)
of a fresh seeded witness on resident keys.

  value     device time per prove (CUDA events on the prover's stream), witness
            already in HBM; K proves timed back to back; with N GPUs every rank
            proves independently (replicas) and value = max-over-ranks time / (N K).
  e2e       the same through the C ABI from pinned host memory: witness upload,
            prove, raw-proof download, blinding with seeded r, s, proof download.
  roofline  the dominant kernel (MSM bucket accumulation) in Fq-multiplications/s
            against the instruction-issue ceiling of the product (SMs x 4 warp
            instructions per cycle x 32 lanes x SM clock / instructions per
            product); HBM bytes of the same kernel against the measured copy
            bandwidth beside it.
  cpu_baseline  one single-threaded prove of the same circuit, key and witness by
            the reference's own CPU prover (oracle/_ref: libff/libfqfft built from
            the reference sources, one thread as the reference's bench runs it),
            in its own process; its raw proof is compared with the GPU's.

--impl reference runs the reference CPU prover alone on the host cores: the
circuit built by the reference's own Poseidon gadget from the same seeded
preimages, its own CPU setup, then m = min(cores, steps) single-threaded
processes proving and blinding together (groth16.prove.total); value = T_max / m
ms per proof (the reference bench's m / T_max throughput).  That arm loads
nothing of this repository's library.
Inputs (all > 126 MB L2 per prove: keys ~7 GB, witness 32 MB) are synthetic and
seeded: circuit, witness and toxic waste come from seeded generators.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nkr-zkp_b200"))

WORKLOADS = {
    "poseidon512": ("poseidon", 512, 2),
    "poseidon2048": ("poseidon", 2048, 2),
    "poseidon4096": ("poseidon", 4096, 2),
    "matmul32": ("matmul", 32, 0),
}
METRIC = "Groth16 prove ms @2^20 constraints (bit-exact)"
# DRAM read + write bytes per (point, digit) entry of the G1 accumulation kernel,
# from an ncu capture at 2^18 points (a 2^20 capture would hold ~6 GB of keys on
# the device); traffic grows with entries (one random base gather per entry)
TRAFFIC_PER_ENTRY = (439.882752e6 + 20.989440e6) / 3932125   # 117.2 B per entry
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of k_acc_l1_g1 on the "
                  "2^18-point uniform G1 MSM of --mode kernels (3,932,125 entries), 117.2 B "
                  "per entry, scaled by this launch's entries")
# Thread instructions per 52-bit-limb Fq product in the lazily reduced form the G1
# accumulation runs: ncu smsp__inst_executed.sum x 32 over the products of
# nkr_b200_bench_mul's variant 4 (6,603,139,584 warp instructions for
# 148 x 16 x 256 threads x 256 x 4 = 620,756,992 products).
INSTR_PER_PRODUCT = 6603139584 * 32 / 620756992   # 340.4
# Pipe counters of k_acc_l1_g1 from one ncu launch (2^18-point uniform G1 MSM of
# --mode kernels; profiles/k_acc_l1_g1_msm_2_18.md); percentages of peak.
ACC_NCU = {"issue_active_pct": 59.27, "fp64_pipe_pct": 40.11, "alu_pipe_pct": 56.05,
           "fmaheavy_pipe_pct": 18.69, "warps_active_per_sm": 10.68, "registers": 168,
           "stall_per_issue": {"wait": 0.75, "not_selected": 0.75, "math_pipe_throttle": 0.66,
                               "long_scoreboard": 0.55},
           "source": "ncu --metrics ... -k regex:k_acc_l1_g1 -c 1, --clock-control none"}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")

    def start(self):
        """Starts sampling every 50 ms and returns once the first sample is written,
        so that even a short timed region that follows is sampled."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            self.out.flush()
            if os.path.getsize(self.out.name) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def replica_ms_per_proof(total_ms, proofs, world, dist=None, device="cpu"):
    """Whole-job milliseconds per proof of `world` independent replicas that each
    proved `proofs` times in `total_ms`: the slowest rank's time over all ranks'
    proofs (one MAX all-reduce, the only collective of the replica path)."""
    if dist is not None:
        import torch
        t = torch.tensor([float(total_ms)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    return total_ms / (proofs * world)


def _measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def _uniform_fr(n, rng):
    """n uniform Fr values (4 x u64 each, < r, taken as Montgomery limbs)"""
    import numpy as np
    r_limbs = [0x43e1f593f0000001, 0x2833e84879b97091, 0xb85045b68181585d, 0x30644e72e131a029]
    out = np.empty((n, 4), np.uint64)
    filled = 0
    while filled < n:
        k = n - filled
        cand = rng.integers(0, 2**64, size=(k, 4), dtype=np.uint64, endpoint=False)
        cand[:, 3] &= np.uint64((1 << 62) - 1)
        less = np.zeros(k, bool)
        equal = np.ones(k, bool)
        for i in range(3, -1, -1):
            less |= equal & (cand[:, i] < np.uint64(r_limbs[i]))
            equal &= cand[:, i] == np.uint64(r_limbs[i])
        good = cand[less]
        out[filled:filled + good.shape[0]] = good
        filled += good.shape[0]
    return out


def _seeded_toxic(seed):
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    rng = np.random.default_rng(seed)
    # uniform Fr elements as Montgomery limbs (rejection of values >= r)
    r = 21888242871839275222246405745257275088548364400416034343698204186575808495617
    out = []
    while len(out) < 5:
        v = int.from_bytes(rng.bytes(32), "little") & ((1 << 254) - 1)
        if 0 < v < r:
            out.append(np.frombuffer(v.to_bytes(32, "little"), np.uint64).copy())
    return out


def _save_circuit(d, c):
    """The circuit's CSR arrays and witness as .npy files a spawned process reloads."""
    import numpy as np
    np.save(os.path.join(d, "shape.npy"), np.array([c.rows, c.cols, c.public_inputs], np.uint64))
    np.save(os.path.join(d, "witness.npy"), c.witness)
    for k in range(3):
        np.save(os.path.join(d, f"row_ptr{k}.npy"), c.row_ptr[k])
        np.save(os.path.join(d, f"col_idx{k}.npy"), c.col_idx[k])
        np.save(os.path.join(d, f"values{k}.npy"), c.values[k])


def _load_circuit(d):
    from types import SimpleNamespace
    import numpy as np
    rows, cols, pub = (int(v) for v in np.load(os.path.join(d, "shape.npy")))
    return SimpleNamespace(
        rows=rows, cols=cols, public_inputs=pub, witness=np.load(os.path.join(d, "witness.npy")),
        row_ptr=[np.load(os.path.join(d, f"row_ptr{k}.npy")) for k in range(3)],
        col_idx=[np.load(os.path.join(d, f"col_idx{k}.npy")) for k in range(3)],
        values=[np.load(os.path.join(d, f"values{k}.npy")) for k in range(3)])


def _ref_prove_process(circ_dir, pk_path, blind, barrier, results, idx):
    """One reference CPU prove in its own spawned, single-threaded process
    (OMP_NUM_THREADS=1 as the reference's bench runs it, scripts/bench/runner.py:
    458-467).  Only oracle/_ref (the reference's CPU path built from its sources)
    is loaded.  Circuit, witness and proving key load before the barrier, untimed;
    the timer covers CpuBackend::prove (backends/cpu/src/backend.cpp:156-201) and,
    with blind, the reference's blind_proof after it (groth16.prove.total of
    app/prove.cpp:70-88).  Puts (idx, seconds, raw proof bytes or None)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    try:
        c = _load_circuit(circ_dir)
        ref = O.Ref()
        h = ref.prover(c, pk_path)
        if barrier is not None:
            barrier.wait(timeout=900)
        t0 = time.perf_counter()
        if blind:
            ref.prover_prove_blind(h, c.witness)
            raw = None
        else:
            g1, g2 = ref.prover_prove(h, c.witness)
            raw = g1.tobytes() + g2.tobytes()
        dt = time.perf_counter() - t0
        ref.prover_close(h)
        results.put((idx, dt, raw))
    except Exception as e:  # reported by the parent
        results.put((idx, None, repr(e)))


def _spawn_ref_proves(circ_dir, pk_path, m, blind):
    """m concurrent single-threaded reference proves started together; returns
    the per-process prove seconds (and the raw proofs without blinding)."""
    import multiprocessing as mp
    os.environ["OMP_NUM_THREADS"] = "1"
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(m) if m > 1 else None
    results = ctx.Queue()
    procs = [ctx.Process(target=_ref_prove_process,
                         args=(circ_dir, pk_path, blind, barrier, results, i)) for i in range(m)]
    for p in procs:
        p.start()
    out = [results.get(timeout=1800) for _ in range(m)]
    for p in procs:
        p.join(timeout=60)
    bad = [o for o in out if o[1] is None]
    if bad:
        raise RuntimeError(f"reference prove failed: {bad[0][2]}")
    return sorted(out)


def _ref_workload(ref, workload):
    """The bench workload built by the reference's own Poseidon gadget and
    R1CSManager from the seeded preimages (identical to the repository's
    generator output; tests/test_generator.py pins that)."""
    kind, param, dens = WORKLOADS[workload]
    if kind != "poseidon":
        return None
    return ref.poseidon_circuit_seeded(param, dens, 1)


def _config(kind, param, dens, rows, cols, world):
    return {"workload": f"groth16-prove {kind} count={param} density="
                        f"{['full', 'hybrid', 'sparse'][dens]} ({rows} constraints, "
                        f"{cols} variables padded)",
            "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (keys, witness); no flush"}


DTYPE = "bn254 Fr/Fq (exact modular arithmetic)"


def run_reference(args):
    """--impl reference: the reference's own CPU prover (oracle/_ref) on the same
    2^20 workload, every host core busy, measured as the reference's bench
    measures concurrent proves (scripts/bench/metrics.py:73-77: m proves started
    together, throughput m / T_max), reported as ms per proof = T_max / m.  This
    process and its workers load nothing of this repository's library."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (needs the "
                          "reference source tree at build time)"}))
        return
    t_setup = time.perf_counter()
    ref = O.Ref()
    c = _ref_workload(ref, args.workload)
    if c is None:
        print(json.dumps({"impl": "reference", "unavailable": f"--impl reference builds poseidon "
                          f"workloads only (asked: {args.workload})"}))
        return
    kind, param, dens = WORKLOADS[args.workload]
    d = tempfile.mkdtemp()
    pk_path = os.path.join(d, "pk.bin")
    # the reference CPU setup (backend.cpp:41-154; its own unseeded toxic waste)
    ref.cpu_setup(c, pk_path, os.path.join(d, "vk.bin"))
    _save_circuit(d, c)
    cores = len(os.sched_getaffinity(0))
    try:
        import psutil
        mem_cap = int(psutil.virtual_memory().available // (3 << 30))  # ~1.2 GB per process at 2^20
    except ImportError:
        mem_cap = cores
    m = max(1, min(cores, args.steps, mem_cap))
    setup_s = time.perf_counter() - t_setup
    t0 = time.perf_counter()
    out = _spawn_ref_proves(d, pk_path, m, blind=True)
    wall = time.perf_counter() - t0
    secs = [o[1] for o in out]
    t_max_ms = max(secs) * 1e3
    ms_per_proof = t_max_ms / m
    sample = (f"{m} concurrent single-threaded reference proves (CpuBackend::prove + blind_proof, "
              f"the CLI's groth16.prove.total) of the full workload, one process per core, "
              f"started together; value = T_max / m (metrics.py:73-77)")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(ms_per_proof, 3), "unit": "ms",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_per_proof, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": DTYPE,
        "data": "synthetic (seeded circuit and witness; the reference setup's own toxic waste)",
        "config": _config(kind, param, dens, c.rows, c.cols, world),
        "proofs_timed": m, "t_max_ms": round(t_max_ms, 1),
        "latency_ms_median": round(statistics.median(secs) * 1e3, 1),
        "warmup_note": "no warm-up proves: each process loads its circuit and key untimed before "
                       "the common start; a CPU prove has no device state to warm",
        "setup_s": round(setup_s, 1), "wall_s": round(wall, 1),
        "cpu_baseline": {"value": round(ms_per_proof, 3), "unit": "ms", "cores": m,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": round(ms_per_proof, 3), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def cpu_baseline_single(r1, pk, raw_gpu):
    """The GPU line's CPU baseline: one single-threaded reference CPU prove
    (oracle/_ref) of the same circuit, key and witness, in a spawned process.
    Returns (ms, raw proofs equal)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available():
        return None
    d = tempfile.mkdtemp()
    pk_path = os.path.join(d, "pk.bin")
    O.write_proving_key(pk_path, pk)
    _save_circuit(d, r1)
    out = _spawn_ref_proves(d, pk_path, 1, blind=False)
    _, secs, raw = out[0]
    same = raw == raw_gpu
    return secs * 1e3, same


def run_b200(args):
    import numpy as np
    import torch
    import nkr_b200 as nk

    world, rank, local = _dist()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    device = local
    kind, param, dens = WORKLOADS[args.workload]

    # ---- inputs: circuit, seeded setup, resident key ---------------------------
    r1 = nk.generate(kind, param, dens, seed=1 + rank)
    ctx = nk.Context(device)
    pk, _vk = nk.setup(ctx, r1, _seeded_toxic(77))
    # prepare from host keys (upload, normalisation, window copies, tables): the
    # first one on a context also runs the MSM-window and NTT-tile autotuners for
    # its sizes; the later ones are key loads of a tuned process (median of two)
    prep_ms = []
    for i in range(3):
        be = nk.Backend(ctx)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        be.prepare(r1, pk)
        prep_ms.append((time.perf_counter() - t0) * 1e3)
        if i < 2:
            be.free()
    want_cpu = rank == 0 and world == 1 and not args.no_cpu_baseline
    if not want_cpu:
        del pk
    key_gb = be.device_bytes() / 2**30
    # a few distinct seeded witnesses for the same circuit, resident in HBM
    nwit = 4
    wits_host = [r1.witness] + [nk.generate(kind, param, dens, seed=100 + rank * 10 + i).witness
                                for i in range(nwit - 1)]
    wits_dev = [torch.from_numpy(w.view(np.int64).reshape(-1)).to(f"cuda:{device}") for w in wits_host]
    wits_pin = []
    for w in wits_host:
        t = torch.from_numpy(w.view(np.int64).reshape(-1)).pin_memory()
        wits_pin.append(t)
    torch.cuda.synchronize(device)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(device)

    # ---- device-timed proves -----------------------------------------------------
    for i in range(args.warmup):
        be.prove(None, witness_ptr=wits_dev[i % nwit].data_ptr())
    barrier()
    clocks = ClockSampler(device)
    clocks.start()
    launches0 = nk.launch_count()
    print(f"[bench] library launches before the timed region: {launches0}", file=sys.stderr)
    stage = []
    t0 = time.perf_counter()
    for i in range(args.steps):
        be.prove(None, witness_ptr=wits_dev[i % nwit].data_ptr())
        stage.append(be.stage_times())
    barrier()
    wall = time.perf_counter() - t0
    launches = nk.launch_count() - launches0
    print(f"[bench] launches in the timed region: {launches} ({launches // args.steps} per prove)",
          file=sys.stderr)
    clk = clocks.stop()
    value = replica_ms_per_proof(sum(s["total_ms"] for s in stage), args.steps, world, dist,
                                 f"cuda:{device}")

    # ---- end to end through the C ABI from pinned host memory -------------------
    rs = _seeded_toxic(5)[:2]
    e2e = []
    for i in range(args.warmup + args.steps):
        t1 = time.perf_counter()
        raw = be.prove(None, witness_ptr=wits_pin[i % nwit].data_ptr())
        be.blind(raw, rs[0], rs[1])
        if i >= args.warmup:
            e2e.append((time.perf_counter() - t1) * 1e3)
    e2e_ms = replica_ms_per_proof(sum(e2e), len(e2e), world, dist, f"cuda:{device}")
    # witness; the blinding's upload: raw proof (576 B) + r, s as canonical scalars
    # and their GLV halves (240 B); downloads: raw proof, then the proof (384 B)
    h2d = r1.cols * 32 + 576 + 240
    d2h = 576 + 384

    # ---- the same circuit over a witness without repeated values ----------------
    # The witness MSMs sum the bases of equal witness values once (the benchmark
    # witness repeats 829 values over 731 K variables); proves over seeded uniform
    # values (all distinct; not a satisfying witness, which a prove does not check)
    # show the cost when nothing repeats.
    rng = np.random.default_rng(1234 + rank)
    uni = torch.from_numpy(_uniform_fr(r1.cols, rng).view(np.int64).reshape(-1)).to(f"cuda:{device}")
    for _ in range(2):
        be.prove(None, witness_ptr=uni.data_ptr())
    uni_ms = []
    for _ in range(5):
        be.prove(None, witness_ptr=uni.data_ptr())
        uni_ms.append(be.stage_times()["total_ms"])
    del uni

    # ---- roofline of the dominant kernel (MSM bucket accumulation) ---------------
    peaks = _measured_peaks()
    # The product roof is the instruction-issue ceiling of the 52-bit-limb Fq product
    # the G1 accumulation runs: every SM issues 4 warp instructions per cycle and one
    # product costs INSTR_PER_PRODUCT thread instructions (ncu), so no kernel built
    # from these products exceeds SMs x 4 x 32 x f_sm / INSTR_PER_PRODUCT products/s.
    # The best register-resident microbenchmark of the same product (itself at ~60%
    # issue) is reported beside it.
    peak_int, _ = ctx.bench_mul(1)
    peak_fp64, _ = ctx.bench_mul(1 | (4 << 8))  # the lazily reduced FP64 form
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    f_sm = (clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0) * 1e6
    issue_peak = sms * 4 * 32 * f_sm / INSTR_PER_PRODUCT
    mb = nk.MsmBases(ctx, 1, be._keep["a_query"]) if hasattr(be, "_keep") and be._keep else None
    roof = None
    if mb is not None:
        accs = []
        for i in range(3):
            mb.run(wits_host[i % nwit])
            accs.append(mb.stats())
        st = accs[-1]
        acc_ms = statistics.median(a["acc_ms"] for a in accs)
        muls = st["entries"] * 10.0  # mixed XYZZ add = 8M + 2S per (point, digit) entry
        achieved = muls / (acc_ms * 1e-3)
        # algorithmic HBM bytes of the launch: one 64 B affine base + 4 B entry per entry,
        # plus the task bucket ids and bucket / partial writes (128 B each)
        algo_bytes = st["entries"] * (64 + 4) + st["tasks"] * 2 * 128
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        # DRAM bytes per entry from an ncu capture of this kernel at 2^18, scaled to
        # this launch's entries
        traffic = round(st["entries"] * TRAFFIC_PER_ENTRY) if TRAFFIC_PER_ENTRY else None
        roof = {"bound": "int", "kernel": "k_acc_l1_g1 (G1 bucket accumulation; operator-level MSM "
                                          "over the A query and the workload's witness, no class path)",
                "achieved": round(achieved / 1e9, 2), "peak": round(issue_peak / 1e9, 2),
                "unit": "G Fq-mul/s", "frac": round(achieved / issue_peak, 3),
                "peak_source": f"instruction-issue ceiling of the FP64-limb Fq product: {sms} SMs "
                               f"x 4 warp instructions/cycle x 32 x {f_sm / 1e6:.0f} MHz (SM clock "
                               f"sampled in the timed region) / {INSTR_PER_PRODUCT:.1f} instructions "
                               f"per product (ncu on nkr_b200_bench_mul); no FLOP or integer peak "
                               f"in MEASURED_PEAKS.json applies",
                "microbench": {"int_cios": round(peak_int / 1e9, 2),
                               "fp64_52bit": round(peak_fp64 / 1e9, 2),
                               "frac_of_best": round(achieved / max(peak_int, peak_fp64), 3),
                               "note": "register-resident product chains (nkr_b200_bench_mul), "
                                       "issue active ~60% themselves"},
                "ncu": ACC_NCU,
                "units_per_launch": {"entries": st["entries"], "fq_muls": muls,
                                     "window_bits": st["window_bits"], "windows": st["windows"],
                                     "buckets": st["buckets"]},
                "launch_ms": round(acc_ms, 4),
                "hbm": {"achieved": round(algo_bytes / (acc_ms * 1e-3) / 1e9, 1),
                        "peak": hbm_peak, "unit": "GB/s",
                        "frac": round(algo_bytes / (acc_ms * 1e-3) / 1e9 / hbm_peak, 4),
                        "algorithmic_bytes": algo_bytes, "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
                "traffic": traffic, "traffic_unit": "bytes per launch",
                "traffic_source": TRAFFIC_SOURCE}
        mb.free()

    # ---- CPU baseline (rank 0, N = 1 only) --------------------------------------
    cpu = None
    if want_cpu:
        g1, g2 = nk.raw_to_arrays(be.prove(wits_host[0]))
        raw_gpu = np.stack([x[:8] for x in g1]).tobytes() + g2[:16].tobytes()
        got = cpu_baseline_single(r1, pk, raw_gpu)
        del pk
        if got is not None:
            ms, same = got
            cpu = {"value": round(ms, 1), "unit": "ms", "cores": 1, "kind": "reference",
                   "sample": f"one single-threaded reference CPU prove (oracle/_ref: "
                             f"CpuBackend::prove, backends/cpu/src/backend.cpp:156-201) of the "
                             f"same {r1.rows}-constraint circuit, key and witness, in its own "
                             f"process; circuit and key load untimed",
                   "raw_proof_equal_to_gpu": bool(same)}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    s_med = {k: round(statistics.median(s[k] for s in stage), 3) for k in stage[0]
             if not k.endswith(("_start_ms", "l1_end_ms", "fixup_end_ms", "reduce_first_end_ms"))}
    # each MSM's phases in the concurrent prove: level-1 start / end, fix-ups end,
    # first reduction level end, MSM end (ms from the prove's start)
    timeline = {m: [round(statistics.median(s[f"msm_{m}_{ph}_ms"] for s in stage), 3)
                    for ph in ("l1_start", "l1_end", "fixup_end", "reduce_first_end", "end")]
                for m in ("a", "b_g1", "b_g2", "l", "h")}
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(wall * 1e3 / args.steps, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": DTYPE,
        "arith": "Fr and Fq in 8 x 32-bit limbs on the integer pipe; the G1 MSMs' Fq in "
                 "5 x 52-bit limbs on the FP64 pipe",
        "data": "synthetic (seeded circuit, witness and toxic waste)",
        "config": _config(kind, param, dens, r1.rows, r1.cols, world),
        "key_device_gib": round(key_gb, 2),
        "stages_ms_median": s_med,
        "prove_ms_distinct_witness": {"value": round(statistics.median(uni_ms), 3),
                                      "note": "median of 5 device-timed proves of the same circuit "
                                              "over seeded uniform Fr values (no repeated values)"},
        "msm_timeline_ms_median": {"phases": ["l1_start", "l1_end", "fixup_end",
                                              "reduce_first_end", "end"], **timeline},
        "prepare_ms": {"first": round(prep_ms[0], 1),
                       "tuned": round(statistics.median(prep_ms[1:]), 1)},
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk,
        "roofline": roof,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# batched form: 64 proofs of uneven size, batched vs plain sequential
# ---------------------------------------------------------------------------

def batch_mix(count=64, seed=4):
    """The uneven mix: matmul size 16..64 or poseidon count 64..2048 (log-uniform),
    hybrid density, sizes and kinds drawn from one seed."""
    import numpy as np
    rng = np.random.default_rng(seed)
    mix = []
    for i in range(count):
        if rng.random() < 0.5:
            mix.append(("matmul", int(rng.integers(16, 65)), 1, 10_000 + i))
        else:
            mix.append(("poseidon", int(2 ** rng.integers(6, 12)), 1, 10_000 + i))
    return mix


def _pinned_copy(torch, arr):
    import numpy as np
    t = torch.empty(arr.size, dtype=torch.int64, pin_memory=True)
    t.numpy()[:] = np.ascontiguousarray(arr).reshape(-1).view(np.int64)
    return t


def _prepare_keys(ctx, nk, specs, key_of):
    """One prepared key per distinct circuit (GPU setup with seeded toxic waste)."""
    keys = {}
    for spec in specs:
        kid = key_of(spec)
        if kid in keys:
            continue
        kind, param, dens, seed = spec
        r1 = nk.generate(kind, param, dens, seed=seed)
        pk, _ = nk.setup(ctx, r1, _seeded_toxic(seed))
        be = nk.Backend(ctx)
        be.prepare(r1, pk)
        keys[kid] = be
    return keys


def run_batch(args):
    import torch
    import nkr_b200 as nk
    t_setup = time.perf_counter()
    ctx = nk.Context(0)
    mix = batch_mix()
    # poseidon circuits depend only on the count; a matmul circuit on its seed
    key_of = lambda s: (s[0], s[1]) if s[0] == "poseidon" else (s[0], s[1], s[3])  # noqa: E731
    keys = _prepare_keys(ctx, nk, mix, key_of)
    bes, pins, rows = [], [], []
    for kind, param, dens, seed in mix:
        r1 = nk.generate(kind, param, dens, seed=seed)
        bes.append(keys[key_of((kind, param, dens, seed))])
        pins.append(_pinned_copy(torch, r1.witness))
        rows.append(r1.rows)
    ptrs = [t.data_ptr() for t in pins]
    setup_s = time.perf_counter() - t_setup
    clocks = ClockSampler(0)
    # warm-up: slots, graphs and the tuner's size classes
    first = [bytes(be.prove(None, witness_ptr=p)) for be, p in zip(bes, ptrs)]
    for _ in range(args.warmup):
        out = nk.prove_batch(bes, witness_ptrs=ptrs)
        out_l = nk.prove_batch(bes, witness_ptrs=ptrs, lists=True)
    assert [bytes(o) for o in out] == first, "batched proofs differ from the plain proves"
    assert [bytes(o) for o in out_l] == first, "cross-proof batched proofs differ from the plain proves"
    clocks.start()
    seq, bat, lst = [], [], []
    launches0 = nk.launch_count()
    for _ in range(args.steps):
        t = time.perf_counter()
        got = [bytes(be.prove(None, witness_ptr=p)) for be, p in zip(bes, ptrs)]
        seq.append(time.perf_counter() - t)
        assert got == first
        t = time.perf_counter()
        out = nk.prove_batch(bes, witness_ptrs=ptrs)
        bat.append(time.perf_counter() - t)
        assert [bytes(o) for o in out] == first
        t = time.perf_counter()
        out = nk.prove_batch(bes, witness_ptrs=ptrs, lists=True)
        lst.append(time.perf_counter() - t)
        assert [bytes(o) for o in out] == first
    launches = (nk.launch_count() - launches0) // max(args.steps, 1)
    clk = clocks.stop()
    n = len(mix)
    seq_pps = n / statistics.median(seq)
    bat_pps = n / statistics.median(bat)
    lst_pps = n / statistics.median(lst)
    hist = {}
    for r in rows:
        hist[f"2^{r.bit_length() - 1}"] = hist.get(f"2^{r.bit_length() - 1}", 0) + 1
    line = {
        "metric": "batched Groth16 proofs/s, 64 uneven proofs (bit-exact)", "value": round(bat_pps, 2),
        "unit": "proofs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "dtype": "bn254 (exact modular; u32 limbs, G1 MSM in 52-bit FP64 limbs)",
        "data": "synthetic (seeded circuits, witnesses and toxic waste)",
        "config": {"workload": "64 proofs: matmul s in [16, 64] or poseidon count 2^6..2^11, "
                               "hybrid density, seed 4", "domains": dict(sorted(hist.items())),
                   "distinct_keys": len(keys), "witness": "pinned host memory, uploaded per proof"},
        "plain_sequential": {"value": round(seq_pps, 2), "unit": "proofs/s",
                             "path": "nkr_b200_prove one proof at a time (upload, prove, download)"},
        "speedup_vs_plain": round(bat_pps / seq_pps, 3),
        "cross_proof_lists": {"value": round(lst_pps, 2), "unit": "proofs/s",
                              "speedup_vs_plain": round(lst_pps / seq_pps, 3),
                              "path": "nkr_b200_prove_batch_lists: per wave one launch per NTT "
                                      "pass, quotient step and level-1 accumulation over all "
                                      "proofs (device work lists)"},
        "e2e": {"value": round(bat_pps, 2), "unit": "proofs/s",
                "h2d_bytes_per_step": sum(t.numel() * 8 for t in pins),
                "d2h_bytes_per_step": 576 * n},
        "gpu_launches": launches, "clocks": clk, "setup_s": round(setup_s, 1),
        "key_device_gib": round(sum(be.device_bytes() for be in keys.values()) / 2**30, 2),
    }
    print(json.dumps(line))
    for be in keys.values():
        be.free()
    ctx.close()


# ---------------------------------------------------------------------------
# serving form: Poisson stream over 6 resident keys, server vs plain FIFO
# ---------------------------------------------------------------------------

SERVE_KEYS = [("matmul", 32, 0), ("matmul", 64, 0), ("poseidon", 256, 2), ("poseidon", 4096, 2),
              ("sql-aggregate", 1 << 10, 2), ("sql-aggregate", 1 << 14, 2)]


def _percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
    return xs[k]


def run_serve(args):
    import threading
    import numpy as np
    import torch
    import nkr_b200 as nk
    t_setup = time.perf_counter()
    ctx = nk.Context(0)
    keys = SERVE_KEYS[:args.serve_keys]
    bes, wits = [], []
    for j, (kind, param, dens) in enumerate(keys):
        r1 = nk.generate(kind, param, dens, seed=20 + j)
        pk, _ = nk.setup(ctx, r1, _seeded_toxic(20 + j))
        be = nk.Backend(ctx)
        be.prepare(r1, pk)
        del pk
        bes.append(be)
        # matmul circuits depend on their seed: one witness; the others take fresh ones
        ws = [r1.witness] if kind == "matmul" else [
            r1.witness, nk.generate(kind, param, dens, seed=40 + j).witness]
        wits.append([_pinned_copy(torch, w) for w in ws])
    setup_s = time.perf_counter() - t_setup
    # plain service times per key (also the warm-up of slot 0 of every key)
    expect, service = [], []
    for be, ws in zip(bes, wits):
        expect.append([bytes(be.prove(None, witness_ptr=w.data_ptr())) for w in ws])
        t = time.perf_counter()
        be.prove(None, witness_ptr=ws[0].data_ptr())
        service.append(time.perf_counter() - t)
    mean_s = sum(service) / len(service)
    n_req = args.serve_requests

    def stream(load, seed):
        """Poisson arrivals at `load` x the plain path's capacity (one request per
        mean plain service time at load 1), keys uniform, seeded."""
        rng = np.random.default_rng(seed)
        lam = load / mean_s
        arrivals = np.cumsum(rng.exponential(1.0 / lam, n_req))
        which = rng.integers(0, len(keys), n_req)
        wsel = [int(rng.integers(0, len(wits[k]))) for k in which]
        return lam, arrivals, which, wsel

    def replay(arrivals, submit, wait_all):
        t0 = time.perf_counter()
        handles = []
        for i in range(n_req):
            d = arrivals[i] - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            handles.append(submit(i, t0))
        res = wait_all(handles)
        return res, time.perf_counter() - t0

    # plain arm: one request at a time in arrival order (FIFO), the same arrivals
    def plain_arm(arrivals, which, wsel):
        done = [None] * n_req
        q, cv = [], threading.Condition()

        def worker():
            for i in range(n_req):
                with cv:
                    while not q:
                        cv.wait()
                    j, t0 = q.pop(0)
                k = which[j]
                raw = bytes(bes[k].prove(None, witness_ptr=wits[k][wsel[j]].data_ptr()))
                done[j] = (raw, (time.perf_counter() - t0 - arrivals[j]) * 1e3)
        th = threading.Thread(target=worker)
        th.start()

        def submit(i, t0):
            with cv:
                q.append((i, t0))
                cv.notify()
            return i
        res, wall = replay(arrivals, submit, lambda h: (th.join(), done)[1])
        return res, wall

    def server_arm(arrivals, which, wsel, ageing):
        sv = nk.Server(ctx, max_inflight=args.serve_inflight, max_slots_per_key=4)
        sv.set_ageing(ageing)
        ids = [sv.add_key(be) for be in bes]

        def submit(i, t0):
            k = which[i]
            return sv.submit(ids[k], witness_ptr=wits[k][wsel[i]].data_ptr())

        def wait_all(handles):
            out = []
            for h in handles:
                raw, lat, _ = sv.wait(h)
                out.append((bytes(raw), lat))
            return out
        res, wall = replay(arrivals, submit, wait_all)
        slots = [sv.slots(i) for i in ids]
        aged = sv.stats()["aged"]
        sv.close()
        return res, wall, slots, aged

    clocks = ClockSampler(0)
    # server warm-up: slots and graphs of every key
    server_arm_warm = nk.Server(ctx, max_inflight=args.serve_inflight, max_slots_per_key=4)
    wids = [server_arm_warm.add_key(be) for be in bes]
    for _ in range(2):
        hs = [server_arm_warm.submit(wids[k], witness_ptr=wits[k][0].data_ptr())
              for k in range(len(keys)) for _ in range(4)]
        for h in hs:
            server_arm_warm.wait(h)
    server_arm_warm.close()
    clocks.start()
    launches0 = nk.launch_count()
    ok = True

    def summary(res, wall):
        lat = [x[1] for x in res]
        return {"proofs_per_s": round(n_req / wall, 2), "p50_ms": round(_percentile(lat, 50), 2),
                "p99_ms": round(_percentile(lat, 99), 2)}

    def exact(res, which, wsel):
        return all(res[i][0] == expect[which[i]][wsel[i]] for i in range(n_req))

    # the offered load below capacity: latency; the server with and without ageing
    lam, arrivals, which, wsel = stream(args.serve_load, 5)
    plain, plain_wall = plain_arm(arrivals, which, wsel)
    srv, srv_wall, slots, aged = server_arm(arrivals, which, wsel, args.serve_age)
    srv0, srv0_wall, _, _ = server_arm(arrivals, which, wsel, 0.0)
    ok = ok and exact(plain, which, wsel) and exact(srv, which, wsel) and exact(srv0, which, wsel)
    # saturation: offered load above the plain path's capacity, so each arm runs
    # at its own throughput
    lam_sat, arr_s, which_s, wsel_s = stream(args.serve_sat_load, 6)
    plain_s, plain_s_wall = plain_arm(arr_s, which_s, wsel_s)
    srv_s, srv_s_wall, _, aged_s = server_arm(arr_s, which_s, wsel_s, args.serve_age)
    ok = ok and exact(plain_s, which_s, wsel_s) and exact(srv_s, which_s, wsel_s)
    clk = clocks.stop()
    line = {
        "metric": "served Groth16 proofs/s and latency, Poisson stream over 6 resident keys",
        "value": round(n_req / srv_s_wall, 2), "unit": "proofs/s", "n_gpus": 1,
        "higher_is_better": True, "dtype": DTYPE, "bit_exact": ok,
        "data": "synthetic (seeded circuits, witnesses, toxic waste and arrivals)",
        "config": {"workload": "keys " + ", ".join(f"{k} {p}" for k, p, _ in keys),
                   "requests_per_arm": n_req,
                   "plain_service_ms": [round(x * 1e3, 2) for x in service],
                   "max_inflight": args.serve_inflight, "slots_used": slots,
                   "ageing_factor": args.serve_age},
        "saturation": {"offered_load": args.serve_sat_load, "arrival_rate_per_s": round(lam_sat, 2),
                       "server": dict(summary(srv_s, srv_s_wall), aged=aged_s),
                       "plain_fifo": summary(plain_s, plain_s_wall),
                       "speedup_vs_plain": round(plain_s_wall / srv_s_wall, 3)},
        "below_capacity": {"offered_load": args.serve_load, "arrival_rate_per_s": round(lam, 2),
                           "server": dict(summary(srv, srv_wall), aged=aged),
                           "server_no_ageing": summary(srv0, srv0_wall),
                           "plain_fifo": summary(plain, plain_wall)},
        "gpu_launches": nk.launch_count() - launches0, "clocks": clk, "setup_s": round(setup_s, 1),
        "key_device_gib": round(sum(be.device_bytes() for be in bes) / 2**30, 2),
    }
    print(json.dumps(line))
    for be in bes:
        be.free()
    ctx.close()


# ---------------------------------------------------------------------------
# standalone kernels: NTT, G1 / G2 MSM at the operator sizes
# ---------------------------------------------------------------------------

FR_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617
_FR_LIMBS = [(FR_MOD >> (64 * i)) & (2**64 - 1) for i in range(4)]


def _uniform_fr(n, rng):
    """n uniform Fr elements as 4 x u64 limbs (read as Montgomery representations):
    254-bit candidates, values >= r rejected."""
    import numpy as np
    out = np.empty((n, 4), np.uint64)
    filled = 0
    while filled < n:
        k = n - filled
        cand = rng.integers(0, 2**64, size=(k, 4), dtype=np.uint64)
        cand[:, 3] &= np.uint64((1 << 62) - 1)
        less = np.zeros(k, bool)
        equal = np.ones(k, bool)
        for i in range(3, -1, -1):
            less |= equal & (cand[:, i] < np.uint64(_FR_LIMBS[i]))
            equal &= cand[:, i] == np.uint64(_FR_LIMBS[i])
        good = cand[less]
        out[filled:filled + len(good)] = good
        filled += len(good)
    return out


def _sparse_witness_scalars(n, rng):
    """The sparse-witness mix: 10% uniform Fr, 30% zero, 60% drawn uniformly from
    {zero, one, a small value < 2^16}, shuffled (Montgomery limbs)."""
    import numpy as np
    r_mont = pow(2, 256, FR_MOD)
    small_tab = np.array([[(v * r_mont % FR_MOD >> (64 * i)) & (2**64 - 1) for i in range(4)]
                          for v in range(1 << 16)], dtype=np.uint64)
    out = np.zeros((n, 4), np.uint64)
    n_uni, n_zero = n // 10, (3 * n) // 10
    out[:n_uni] = _uniform_fr(n_uni, rng)
    rest = n - n_uni - n_zero
    cat = rng.integers(0, 3, rest)
    vals = np.where(cat == 0, 0, np.where(cat == 1, 1, rng.integers(0, 1 << 16, rest)))
    out[n_uni + n_zero:] = small_tab[vals]
    return out[rng.permutation(n)]


FQ_MOD = 21888242871839275222246405745257275088696311157297823662689037894645226208583
# affine generators of G1 = (1, 2) and of the G2 subgroup (x = x0 + x1 u, y = y0 + y1 u)
G2_GEN = (10857046999023057135944570762232829481370756359578518086990519993285655852781,
          11559732032986387107991004021392285783925812861821192530917403151452391805634,
          8495653923123431417604973247489272438418190587263600148770280649306958101930,
          4082367875863433681332203403145435568316851327593401208105741076214120093531)


def _generator_jac(group):
    """The group's generator in the libff Jacobian layout (Montgomery Fq limbs, Z = 1)."""
    import numpy as np
    coords = (1, 2, 1) if group == 1 else G2_GEN + (1, 0)
    return np.array([(v * pow(2, 256, FQ_MOD) % FQ_MOD >> (64 * i)) & (2**64 - 1)
                     for v in coords for i in range(4)], dtype=np.uint64)


def _limb_ints(a):
    return [int.from_bytes(row.tobytes(), "little") for row in a]


def run_kernels(args):
    """One JSON line: device time, work rate and a self-check of every standalone op."""
    import numpy as np
    import torch
    import nkr_b200 as nk
    ctx = nk.Context(0)
    dev = "cuda:0"
    rng = np.random.default_rng(11)
    peaks = _measured_peaks()
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    fr_peak, _ = ctx.bench_mul(0)
    fq_peak = max(ctx.bench_mul(1)[0], ctx.bench_mul(1 | (4 << 8))[0])
    clocks = ClockSampler(0)
    clocks.start()
    launches0 = nk.launch_count()
    rows = []
    r_inv = pow(2, -256, FR_MOD)

    want = None if args.cases == "all" else set(args.cases.split(","))

    def selected(name):
        return want is None or name in want

    # (i) NTT: FFT, iFFT, cosetFFT, icosetFFT at 2^16, 2^20, 2^24
    for logn in (16, 20, 24):
        if not selected(f"ntt.{logn}"):
            continue
        n = 1 << logn
        host = _uniform_fr(n, rng)
        x = torch.from_numpy(host.view(np.int64).reshape(-1)).to(dev)
        work = torch.empty_like(x)
        out = torch.empty_like(x)
        back = torch.empty_like(x)
        stream = torch.cuda.current_stream().cuda_stream  # the copies below run on it
        shape = ctx.tune_ntt(n)  # builds the size's tables and tunes its tile shape
        for op, name, inv_op in ((0, "fft", 1), (1, "ifft", 0), (2, "coset_fft", 3), (3, "icoset_fft", 2)):
            ts = []
            for it in range(args.warmup + args.steps):
                work.copy_(x)
                ms = ctx.ntt_device(op, work.data_ptr(), out.data_ptr(), n, stream, timed=True)
                if it >= args.warmup:
                    ts.append(ms)
            # round trip: the inverse op brings the input back bit for bit
            work.copy_(out)
            ctx.ntt_device(inv_op, work.data_ptr(), back.data_ptr(), n, stream)
            torch.cuda.synchronize()
            ok = bool(torch.equal(back, x))
            ms = statistics.median(ts)
            muls = (n // 2) * logn + (n if op != 0 else 0)  # butterflies + the coset / 1/N scale
            byts = 2 * 32 * n * 2  # one transform read + write, one permuting read + write
            rows.append({"op": f"ntt.{name}", "n": f"2^{logn}", "ms": round(ms, 4),
                         "G_fr_mul_per_s": round(muls / ms / 1e6, 2),
                         "frac_fr_mul_peak": round(muls / (ms * 1e-3) / fr_peak, 3),
                         "GB_per_s": round(byts / ms / 1e6, 1),
                         "frac_hbm": round(byts / (ms * 1e-3) / 1e9 / hbm_peak, 3),
                         "tile": {"max_stages_per_pass": shape[0], "butterflies_per_thread": shape[1]},
                         "check": "inverse round trip bit-exact" if ok else "ROUND TRIP FAILED"})
        del x, work, out, back

    # (ii)-(iv) MSM: bases k_i G from the library's scalar multiplication; the result
    # must equal (sum_i s_i k_i) G computed by that independent double-and-add path
    def msm_case(group, logn, mix):
        n = 1 << logn
        gen = _GEN[group]
        w = 12 if group == 1 else 24
        ks = _uniform_fr(n, rng)
        bases = ctx.group_op(group, 2, np.tile(gen, (n, 1)), ks)
        scal = _uniform_fr(n, rng) if mix == "uniform" else _sparse_witness_scalars(n, rng)
        t_mont = sum(a * b for a, b in zip(_limb_ints(scal), _limb_ints(ks))) * r_inv % FR_MOD
        want = ctx.group_op(group, 2, gen.reshape(1, w),
                            np.array([[(t_mont >> (64 * i)) & (2**64 - 1) for i in range(4)]],
                                     dtype=np.uint64))[0]
        mb = nk.MsmBases(ctx, group, bases)
        del bases
        sd = torch.from_numpy(scal.view(np.int64).reshape(-1)).to(dev)
        torch.cuda.synchronize()  # the MSM runs on the library's own stream
        ts, accs = [], []
        for it in range(args.warmup + args.steps):
            got, ms = mb.run(None, scalars_ptr=sd.data_ptr())
            if it >= args.warmup:
                ts.append(ms)
                accs.append(mb.stats()["acc_ms"])
        st = mb.stats()
        mb.free()
        ok = bool(np.array_equal(got, want))
        ms, acc_ms = statistics.median(ts), statistics.median(accs)
        per_entry = 10 if group == 1 else 28  # mixed XYZZ add: 8M + 2S; Fq2 product = 3 Fq
        muls = st["entries"] * per_entry
        byts = n * (64 * group + 32)
        return {"op": f"msm.g{group}.{mix}", "n": f"2^{logn}", "ms": round(ms, 4),
                "window_bits": st["window_bits"], "windows": st["windows"], "entries": st["entries"],
                "acc_ms": round(acc_ms, 4), "G_fq_mul_per_s_acc": round(muls / acc_ms / 1e6, 2),
                "phases_ms": {k: round(st[k], 4) for k in ("sort_ms", "acc_ms", "fixup_ms",
                                                            "reduce_first_ms", "reduce_levels_ms")},
                "frac_fq_mul_peak_acc": round(muls / (acc_ms * 1e-3) / fq_peak, 3),
                "G_fq_mul_per_s_whole": round(muls / ms / 1e6, 2),
                "GB_per_s_algorithmic": round(byts / ms / 1e6, 1),
                "check": "equals (sum s_i k_i) G" if ok else "MISMATCH"}

    _GEN = {1: _generator_jac(1), 2: _generator_jac(2)}
    for group, logn, mix in [(1, 16, "uniform"), (1, 16, "sparse"), (1, 20, "uniform"),
                             (1, 20, "sparse"), (1, 22, "uniform"), (1, 22, "sparse"),
                             (2, 18, "uniform"), (1, 18, "uniform")]:
        # the 2^18 G1 case is the small profiling case (run only when named)
        if (want is None and (group, logn) != (1, 18)) or \
                (want is not None and f"msm.g{group}.{mix}.{logn}" in want):
            rows.append(msm_case(group, logn, mix))
    clk = clocks.stop()
    line = {
        "metric": "standalone NTT and MSM kernels: device ms per op (bit-exact self-checks)",
        "value": None, "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": False, "dtype": "bn254 (exact modular)",
        "data": "synthetic (seeded uniform Fr; bases k_i G with seeded k_i)",
        "peaks": {"fr_mul_per_s": round(fr_peak / 1e9, 2), "fq_mul_per_s": round(fq_peak / 1e9, 2),
                  "hbm_gbs": hbm_peak, "unit_mul": "G/s"},
        "ops": rows, "all_checks_pass": all(not r["check"].isupper() for r in rows),
        "gpu_launches": nk.launch_count() - launches0, "clocks": clk,
    }
    print(json.dumps(line))
    ctx.close()


# verification: circuits with few (sql-aggregate 1024: 4) and many (matmul 32: 3072)
# public inputs
VERIFY_WORKLOADS = [("sql-aggregate", 1024, 2), ("matmul", 32, 0)]


def _uniform_fr_rows(rng, n):
    """n uniform Fr elements (Montgomery limbs), rejection of values >= r"""
    import numpy as np
    r = 21888242871839275222246405745257275088548364400416034343698204186575808495617
    out = np.zeros((n, 4), np.uint64)
    k = 0
    while k < n:
        v = int.from_bytes(rng.bytes(32), "little") & ((1 << 254) - 1)
        if v < r:
            out[k] = np.frombuffer(v.to_bytes(32, "little"), np.uint64)
            k += 1
    return out


def run_verify(args):
    """Groth16 verification throughput: nkr_b200_verify_batch over batches of valid
    proofs (one raw proof blinded with many seeded r, s) against the reference's
    own verify (common/src/protocol.cpp:96-108, oracle/_ref) on one host core."""
    import numpy as np
    import nkr_b200 as nk
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    ctx = nk.Context(0)
    n = args.verify_batch
    rng = np.random.default_rng(12)
    rows_out = []
    for kind, param, dens in VERIFY_WORKLOADS:
        r1 = nk.generate(kind, param, dens, seed=1)
        pk, vkp = nk.setup(ctx, r1, _seeded_toxic(77))
        be = nk.Backend(ctx)
        be.prepare(r1, pk)
        del pk
        raw = be.prove(r1.witness)
        # distinct blinded proofs, tiled to the batch (every copy is verified in full)
        nd = min(n, args.verify_distinct)
        rs = _uniform_fr_rows(rng, 2 * nd).reshape(nd, 2, 4)
        uniq = np.stack([np.frombuffer(bytes(be.blind(raw, r, s)), np.uint64) for r, s in rs])
        proofs = np.ascontiguousarray(np.tile(uniq, (-(-n // nd), 1))[:n])
        pub = np.ascontiguousarray(r1.witness[1:1 + r1.public_inputs])
        publics = np.ascontiguousarray(np.broadcast_to(pub, (n,) + pub.shape))
        vk = nk.VerifyingKey(ctx, vkp["alpha_g1_beta_g2"], vkp["gamma_g2"], vkp["delta_g2"], vkp["ic"])
        for _ in range(args.warmup):
            ok = vk.verify_batch(publics, proofs)
        assert ok.all(), "a valid proof was rejected"
        clocks = ClockSampler(0)
        clocks.start()
        ts = []
        for _ in range(args.steps):
            t = time.perf_counter()
            vk.verify_batch(publics, proofs)
            ts.append(time.perf_counter() - t)
        clk = clocks.stop()
        gpu_ps = n / statistics.median(ts)
        # the reference verifier on one host core, a bounded sample of the same proofs
        ref_ps = None
        if not args.no_cpu_baseline:
            import oracle as O
            if O.ref_available():
                ref = O.Ref()
                with tempfile.TemporaryDirectory() as d:
                    vk_path = os.path.join(d, "vk.bin")
                    ref.write_vk(vkp, vk_path)
                    done, t0 = 0, time.perf_counter()
                    while done < 50 and time.perf_counter() - t0 < 10.0:
                        pth = os.path.join(d, "p.bin")
                        pr = proofs[done]
                        O.write_proof(pth, pr[0:12], pr[12:36], pr[36:48])
                        assert ref.verify(vk_path, pub, pth)
                        done += 1
                    ref_ps = done / (time.perf_counter() - t0)
        rows_out.append({"workload": f"{kind} {param} ({r1.rows} constraints, "
                                     f"{r1.public_inputs} public inputs)",
                         "batch": n, "distinct_proofs": nd, "proofs_per_s": round(gpu_ps, 1),
                         "ms_per_batch": round(statistics.median(ts) * 1e3, 3),
                         "reference_cpu_1core_proofs_per_s": None if ref_ps is None else round(ref_ps, 2),
                         "clocks": clk})
        vk.free()
        be.free()
    line = {
        "metric": "Groth16 verifications/s, batched (reference verdicts)", "value": rows_out[0]["proofs_per_s"],
        "unit": "proofs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "dtype": "bn254 (exact modular; u32 limbs)",
        "data": "synthetic (seeded circuits, witnesses, toxic waste, r and s)",
        "config": {"workloads": rows_out,
                   "path": "nkr_b200_verify_batch from host memory (proof and public-input "
                           "upload, vk_x, Miller loop, final exponentiation, verdict download)"},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="poseidon2048", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="prove", choices=["prove", "batch", "serve", "kernels", "verify"],
                    help="prove: the 2^20 prove (default line); batch: 64 uneven proofs batched vs "
                         "plain; serve: Poisson requests over resident keys, server vs plain FIFO")
    ap.add_argument("--cases", default="all",
                    help="kernels mode: comma-separated subset, e.g. ntt.20,msm.g1.uniform.18 "
                         "(ntt.{16,20,24}; msm.g1.{uniform,sparse}.{16,18,20,22}; msm.g2.uniform.18)")
    ap.add_argument("--verify-batch", type=int, default=32768)
    ap.add_argument("--verify-distinct", type=int, default=4096)
    ap.add_argument("--serve-keys", type=int, default=6)
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-load", type=float, default=0.8)
    ap.add_argument("--serve-sat-load", type=float, default=1.5)
    ap.add_argument("--serve-age", type=float, default=0.5)
    ap.add_argument("--serve-inflight", type=int, default=8)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "batch":
        run_batch(args)
    elif args.mode == "serve":
        run_serve(args)
    elif args.mode == "kernels":
        run_kernels(args)
    elif args.mode == "verify":
        run_verify(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
