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
            against this GPU's measured Montgomery-product throughput; HBM bytes
            of the same kernel against the measured copy bandwidth beside it.
  cpu_baseline  the reference's own CPU prover (oracle/_ref, libff/libfqfft, one
            thread as the reference runs it) on a bounded sample (poseidon 128,
            2^16 constraints), scaled linearly to 2^20 constraints.

--impl reference runs the reference CPU prover alone on the host cores (one
process per core, each proving the 2^16 sample; ms per 2^20-equivalent proof).
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
REF_SAMPLE = ("poseidon", 128, 2)  # 2^16 constraints
TRAFFIC_PER_ENTRY = (390.744064e6 + 48.899328e6) / 3373063  # k_acc_l1<Fq>, 2^18 capture


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

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


def _measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


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


def cpu_baseline_reference(sample=REF_SAMPLE):
    """Reference CPU prover on the bounded sample; returns (ms at 2^20 scale, description)."""
    import numpy as np  # noqa: F401
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import nkr_b200 as nk
    import oracle as O
    kind, param, dens = sample
    r1 = nk.generate(kind, param, dens, seed=1)
    d = tempfile.mkdtemp()
    if O.ref_available():
        ref = O.Ref()
        ref.cpu_setup(r1, os.path.join(d, "pk"), os.path.join(d, "vk"))
        h = ref.prover(r1, os.path.join(d, "pk"))
        t0 = time.perf_counter()
        ref.prover_prove(h, r1.witness)
        dt = time.perf_counter() - t0
        ref.prover_close(h)
        kind_s = "reference"
    else:
        orc = O.Oracle()
        pk = {}
        # oracle port: random bases suffice for timing
        gen1, gen2 = orc.g1_generator(), orc.g2_generator()
        import numpy as np
        rng = np.random.default_rng(3)
        k = O.random_fr(1, rng)[0]
        p1, p2 = orc.mul_affine(1, gen1, k), orc.mul_affine(2, gen2, k)
        for name, n, g in (("a_query", r1.cols, p1), ("b_g1_query", r1.cols, p1),
                           ("b_g2_query", r1.cols, p2), ("l_query", r1.cols, p1),
                           ("h_query", r1.rows, p1)):
            pk[name] = np.tile(g, (n, 1))
        for name, g in (("alpha_g1", p1), ("beta_g1", p1), ("delta_g1", p1), ("beta_g2", p2),
                        ("delta_g2", p2)):
            pk[name] = g
        t0 = time.perf_counter()
        orc.prove(r1, pk, r1.witness, threads=1)
        dt = time.perf_counter() - t0
        kind_s = "port"
    scale = (1 << 20) / r1.rows
    return dt * 1e3 * scale, kind_s, (f"{kind} count={param} density=sparse ({r1.rows} constraints), "
                                      f"one single-threaded prove {dt:.2f} s, scaled x{scale:.0f} "
                                      "(linear in constraints) to 2^20")


def _ref_worker(args):
    kind, param, dens, pk_path = args
    sys.path.insert(0, os.path.join(ROOT, "nkr-zkp_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import nkr_b200 as nk
    import oracle as O
    r1 = nk.generate(kind, param, dens, seed=1)
    ref = O.Ref()
    h = ref.prover(r1, pk_path)
    t0 = time.perf_counter()
    ref.prover_prove(h, r1.witness)
    return time.perf_counter() - t0


def run_reference(args):
    """--impl reference: the reference CPU prover with every host core busy."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import nkr_b200 as nk
    import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (needs the "
                          "reference source tree at build time)"}))
        return
    cores = os.cpu_count() or 1
    kind, param, dens = REF_SAMPLE
    r1 = nk.generate(kind, param, dens, seed=1)
    d = tempfile.mkdtemp()
    O.Ref().cpu_setup(r1, os.path.join(d, "pk"), os.path.join(d, "vk"))
    ctx = mp.get_context("spawn")
    scale = (1 << 20) / r1.rows
    with ctx.Pool(cores) as pool:
        job = [(kind, param, dens, os.path.join(d, "pk"))] * cores
        for _ in range(args.warmup):
            pool.map(_ref_worker, job)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            pool.map(_ref_worker, job)
        wall = time.perf_counter() - t0
    ms_per_proof = wall * 1e3 / (args.steps * cores) * scale
    line = {
        "impl": "reference", "metric": METRIC, "value": round(ms_per_proof, 3), "unit": "ms",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(wall * 1e3 / args.steps, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "bn254 (u32 limbs, exact)",
        "data": "synthetic (seeded circuit, witness and toxic waste)",
        "config": {"workload": "groth16-prove poseidon count=2048 density=sparse (2^20 constraints)",
                   "sample": f"{kind} count={param} sparse ({r1.rows} constraints) per process, "
                             f"{cores} processes, scaled x{scale:.0f} to 2^20"},
        "cpu_baseline": {"value": round(ms_per_proof, 3), "unit": "ms", "cores": cores,
                         "kind": "reference",
                         "sample": f"{cores} concurrent single-threaded reference proves of the "
                                   f"2^16 sample per step, scaled linearly to 2^20"},
        "e2e": {"value": round(ms_per_proof, 3), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


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
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
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
    dev_ms = sum(s["total_ms"] for s in stage)
    if dist is not None:
        t = torch.tensor([dev_ms], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = float(t.item())
    value = dev_ms / (args.steps * world)

    # ---- end to end through the C ABI from pinned host memory -------------------
    rs = _seeded_toxic(5)[:2]
    e2e = []
    for i in range(args.warmup + args.steps):
        t1 = time.perf_counter()
        raw = be.prove(None, witness_ptr=wits_pin[i % nwit].data_ptr())
        be.blind(raw, rs[0], rs[1])
        if i >= args.warmup:
            e2e.append((time.perf_counter() - t1) * 1e3)
    e2e_ms = sum(e2e) / len(e2e)
    if dist is not None:
        t = torch.tensor([sum(e2e)], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item()) / (len(e2e) * world)
    h2d = r1.cols * 32 + 576 + 64
    d2h = 576 + 384

    # ---- roofline of the dominant kernel (MSM bucket accumulation) ---------------
    peaks = _measured_peaks()
    muls_peak, _ = ctx.bench_mul(1)
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
        # DRAM bytes per entry from an ncu capture of this kernel at 2^18 (read + write
        # 439.6 MB over 3,373,063 entries), scaled to this launch's entries
        traffic = round(st["entries"] * TRAFFIC_PER_ENTRY)
        roof = {"bound": "int", "kernel": "k_acc_l1<Fq> (G1 bucket accumulation)",
                "achieved": round(achieved / 1e9, 2), "peak": round(muls_peak / 1e9, 2),
                "unit": "G Fq-mul/s", "frac": round(achieved / muls_peak, 3),
                "peak_source": "measured: nkr_b200_bench_mul register-resident Montgomery products "
                               "(MEASURED_PEAKS.json has no integer peak)",
                "units_per_launch": {"entries": st["entries"], "fq_muls": muls,
                                     "window_bits": st["window_bits"], "windows": st["windows"],
                                     "buckets": st["buckets"]},
                "launch_ms": round(acc_ms, 4),
                "hbm": {"achieved": round(algo_bytes / (acc_ms * 1e-3) / 1e9, 1),
                        "peak": hbm_peak, "unit": "GB/s",
                        "frac": round(algo_bytes / (acc_ms * 1e-3) / 1e9 / hbm_peak, 4),
                        "algorithmic_bytes": algo_bytes, "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
                "traffic": traffic, "traffic_unit": "bytes per launch",
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum at 2^18, "
                                  "130.3 B per entry, scaled by entries"}
        mb.free()

    # ---- CPU baseline (rank 0, N = 1 only) --------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ms, kind_s, sample = cpu_baseline_reference()
        cpu = {"value": round(ms, 1), "unit": "ms", "cores": 1, "kind": kind_s, "sample": sample}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    s_med = {k: round(statistics.median(s[k] for s in stage), 3) for k in stage[0]}
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(wall * 1e3 / args.steps, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "bn254 (u32 limbs, exact)",
        "data": "synthetic (seeded circuit, witness and toxic waste)",
        "config": {"workload": f"groth16-prove {kind} count={param} density="
                               f"{['full', 'hybrid', 'sparse'][dens]} ({r1.rows} constraints, "
                               f"{r1.cols} variables padded)",
                   "parallelism": f"replicas x{world}", "key_device_gib": round(key_gb, 2),
                   "l2": "inputs larger than L2 (keys, witness); no flush"},
        "stages_ms_median": s_med,
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk,
        "roofline": roof,
        "cpu_baseline": cpu,
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
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
