#!/usr/bin/env python
"""Benchmark of the mapping hot path on B200.

Default workload (the metric's batched form): the mixed-length nucleotide workload at full
size -- a 100 Mbp reference (41 % GC, 45 % of it mutated repeat copies) and a read set of 10M
Illumina-like reads of 35, 50, 75, 100 and 150 bp, mapped with `storm-nucleotide -i 15 -M 1
-z 100 -t 100` and three weight-10 spaced seeds.  The read set is drawn in independent chunks
of 100,000 reads (storm_b200.synth.reads_chunk); one step maps one chunk, a different chunk
every step, with the reference and its index resident in HBM.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--cfg 0..4 --scale s]

value        reads/s, device-resident: the chunk's packed reads in HBM before the timed region,
             results left in HBM; CUDA events on the mapping stream, max over ranks.
e2e          reads/s through the resident front end (storm_b200.pipeline.ResidentMapper): the
             chunk's FASTQ file in, its SAM file out -- parsing, tag sort, host->device copies,
             mapping, device->host copies and SAM formatting inside the timed region.
roofline     the dominant kernel against the chip (integer issue rate at the sampled clock, or
             the measured HBM bandwidth); every stage's fraction is in `stages`.
cpu_baseline the reference's own OpenMP/AVX2 build (oracle/_ref) on this host's cores, on a
             bounded sample (the first reads of each length of a chunk), index resident.
parity_vs_reference  chunk 0 mapped through the same front end, per read length, against the
             digests of the reference's own SAM for that chunk (tests/golden/scale_digests.json).

--impl reference times the reference (oracle/_ref/storm-nucleotide-resident: its stock command
line run once per request with its reference and indexes kept in memory) on the same chunks,
each step the first reads of each length of the step's chunk.
Multi-GPU (torchrun): each rank maps its own chunks (weak scaling), no collective on the data
path; time = max over ranks.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from storm_b200 import synth  # noqa: E402

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_PATH = os.path.join(ROOT, "profiles", "traffic.json")
DIGESTS_PATH = os.path.join(ROOT, "tests", "golden", "scale_digests.json")
FALLBACK_HBM_GBS = 6650.0  # measured on this pool's B200s before MEASURED_PEAKS.json existed
SMS = 148
REF_SAMPLE_PER_LENGTH = 80  # reference arm: reads of each length per step


def log(*a):
    print(*a, file=sys.stderr, flush=True)


DEFAULT_SEEDS = {0: "####--#-#--##--####;#####--###-#-###;###-##-#######",
                 1: "####----##--##-####;####-###--#----####;####-####-####"}


def workload_name(cfg, scale):
    names = {0: "nucleotide 1 Mbp, 100k x 50 bp, -i 3", 1: "colour 10 Mbp (20 % repeats), 2M x 50 colours, -i 7",
             2: "mixed-length nucleotide 100 Mbp (45 % repeats), 10M x 35-150 bp, -i 15, three w10 seeds",
             3: "served -O chain, 100 Mbp (45 % repeats), 35-150 bp", 4: "large 3.1 Gbp in 24 sequences, 100 bp, -i 20"}
    return names[cfg] + ("" if scale == 1.0 else " (scale %g)" % scale)


def headline_config(a, w):
    """The workload identity, the same in both arms (the per-step samples are reported apart)."""
    return {"workload": workload_name(a.cfg, a.scale), "reference_codes": sum(w["ref_sizes"]),
            "reads_total": w["reads"], "read_lengths": w["lengths"] if isinstance(w["lengths"], list) else [w["lengths"]],
            "args": " ".join(w["args"]), "parallelism": "dp%d (reads)" % a.gpus,
            "l2": "inputs larger than L2 (the index alone is 1.2 GB) and a 512 MB write between timed steps"}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 5 + k and s[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ------------------------------------------------------------------------------ inputs

def work_dir(cfg, scale, rank=0):
    d = os.path.join(tempfile.gettempdir(), "storm_bench_c%d_s%g_r%d" % (cfg, scale, rank))
    os.makedirs(d, exist_ok=True)
    return d


def chunked_inputs(a, w, chunks, rank=0):
    """Reference FASTA and the FASTQ of each chunk index in `chunks` (made once, cached)."""
    d = work_dir(a.cfg, a.scale, rank)
    ref = os.path.join(d, "ref.fa")
    genome = None
    if not os.path.exists(ref + ".done"):
        genome = synth.genome_of(w)
        synth.write_fasta(ref, genome)
        open(ref + ".done", "w").write("ok")
    paths = {}
    for c in chunks:
        p = os.path.join(d, "chunk%d.fq" % c)
        if not os.path.exists(p + ".done"):
            if genome is None:
                genome = synth.genome_of(w)
            seqs, quals = synth.reads_chunk(w, genome, c)
            synth.write_fastq(p, seqs, quals)
            open(p + ".done", "w").write("ok")
        paths[c] = p
    return ref, paths, d


def whole_inputs(a, w, rank=0):
    """Reference FASTA + the whole read set (the workloads mapped whole per step)."""
    d = work_dir(a.cfg, a.scale, rank)
    ref, reads = os.path.join(d, "ref.fa"), os.path.join(d, "reads.fq")
    if not os.path.exists(os.path.join(d, "done")):
        genome = synth.genome_of(w)
        synth.write_fasta(ref, genome)
        model = synth.ReadModel(**w.get("model", {}))
        if w["mode"] == "colour":
            pr, cols, q = synth.simulate_colour_reads(genome, w["reads"], w["lengths"], w["read_seed"] + 1000 * rank,
                                                      model)
            synth.write_colour_fastq(reads, pr, cols, q)
        else:
            seqs, quals = synth.simulate_nucleotide_reads(genome, w["reads"], w["lengths"], w["read_seed"] + 1000 * rank,
                                                          model)
            synth.write_fastq(reads, seqs, quals)
        open(os.path.join(d, "done"), "w").write("ok")
    return ref, reads, d


def fastq_records(path):
    with open(path, "rb") as f:
        while True:
            rec = [f.readline() for _ in range(4)]
            if not rec[0]:
                return
            yield rec


def per_length_sample(path, d, per_length, tag):
    """FASTQ files of the first `per_length` reads of each length of `path`, in file order
    (None: all of them); returns [(length, file, count)]."""
    out = {}
    for rec in fastq_records(path):
        L = len(rec[1].rstrip(b"\n"))
        o = out.setdefault(L, [])
        if per_length is None or len(o) < per_length:
            o.append(b"".join(rec))
    res = []
    for L in sorted(out):
        p = os.path.join(d, "%s_len%d.fq" % (tag, L))
        with open(p, "wb") as f:
            f.writelines(out[L])
        res.append((L, p, len(out[L])))
    return res


# ------------------------------------------------------------------------------ peaks

def hbm_peak():
    if os.path.exists(PEAKS_PATH):
        try:
            return float(json.load(open(PEAKS_PATH))["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback 6.65 TB/s (earlier measurement on this pool)"


def issue_ceiling(sm_mhz):
    """32-bit integer lane instructions per second the chip can issue: SMs x 4 warp
    instructions per clock x 32 lanes x the sampled SM clock."""
    return SMS * 4 * 32 * sm_mhz * 1e6


def stage_rooflines(st, n_reads, max_len, sm_mhz, index_info=None):
    """Per-stage achieved work rates and fractions from (summed) step statistics.

    sw_filter   10 integer operations per band cell (L * (2 min(I,15) + 1) cells per candidate),
                two 16-bit cells per 32-bit lane instruction: peak = 2 x the issue ceiling.
    full_align  GCUPS on the band cells it computed ((2I + 1) per row it ran), and the same
                10-operation cell count against the 32-bit issue ceiling.
    hit_gather  8 B per seed lookup + 4 B per index position read + L/4 B of read per strand +
                4 B per candidate diagonal written, against the HBM peak.
    index_build per seed N/4 + 4 (N - span + 1) + 4 (4^w + 1) + 4 * 4^w bytes, against HBM."""
    hbm, hbm_src = hbm_peak()
    ceil = issue_ceiling(sm_mhz)
    out = {}
    if st["ms_filter"] > 0:
        ach = 10.0 * st["filter_band_cells"] / (st["ms_filter"] * 1e-3)
        out["sw_filter"] = {"ms": st["ms_filter"], "bound": "int", "achieved": ach / 1e12, "peak": 2 * ceil / 1e12,
                            "unit": "T int-ops/s", "frac": ach / (2 * ceil),
                            "band_gcups": st["filter_band_cells"] / (st["ms_filter"] * 1e-3) / 1e9,
                            "cell_updates_per_s": st["filter_cells"] / (st["ms_filter"] * 1e-3)}
    if st["ms_align"] > 0:
        ach = 10.0 * st["align_cells"] / (st["ms_align"] * 1e-3)
        out["full_align"] = {"ms": st["ms_align"], "bound": "int", "achieved": ach / 1e12, "peak": ceil / 1e12,
                             "unit": "T int-ops/s", "frac": ach / ceil, "aligned": st["aligned"],
                             "gcups": st["align_cells"] / (st["ms_align"] * 1e-3) / 1e9}
    if st["ms_gather"] > 0:
        gb = st["seed_lookups"] * 8 + st["hit_positions"] * 4 + n_reads * 2 * (max_len / 4) + st["candidates"] * 4
        ach = gb / (st["ms_gather"] * 1e-3) / 1e9
        out["hit_gather"] = {"ms": st["ms_gather"], "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                             "frac": ach / hbm, "bytes": gb}
    out["replay"] = {"ms": st["ms_replay"]}
    if index_info:
        ms, nbytes = index_info
        ach = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        out["index_build"] = {"ms": ms, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                              "bytes": nbytes}
    out["_peak_sources"] = {"int": "issue ceiling: %d SMs x 4 warp-inst/clk x 32 lanes x %.0f MHz (sampled)" % (SMS, sm_mhz),
                            "hbm": hbm_src}
    return out


def index_bytes(seeds, sizes):
    """Algorithmic bytes of building every seed's index of every sequence."""
    tot = 0
    for s in seeds.split(";"):
        pat = s.split(":")[0]
        wgt = pat.count("#") + pat.count("1")
        span = len(pat)
        for n in sizes:
            tot += n / 4 + 4 * (n - span + 1) + 4 * (4 ** wgt + 1) + 4 * 4 ** wgt
    return tot


# ------------------------------------------------------------------------------ reference arm

def run_reference_resident(w, ref, plan, d, threads, warmup, log_setup=True):
    """Setup (reference loads + index build, once per read length), then every step of `plan`
    [(chunk, [(length, file, count)])] maps its per-length sample files, one stock run each.
    Returns (setup seconds, [(reads, seconds)] of the timed steps, of the warm-up steps)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from resident import ResidentReference
    colour = w["mode"] == "colour"
    out = os.path.join(d, "ref_out")
    os.makedirs(out, exist_ok=True)

    def args(path, k):
        return ["-g", ref, "-r", path, "-o", os.path.join(out, "s%d.sam" % k), "-v", "0"] + list(w["args"])

    steps = []
    with ResidentReference(colour, threads=threads, cwd=d) as rr:
        t0 = time.perf_counter()
        # one run per read length on one read: the loads (padding per length) and the index
        # build, the work the resident process does once
        for L, path, _ in plan[0][1]:
            one = os.path.join(d, "one_len%d.fq" % L)
            with open(path, "rb") as f, open(one, "wb") as o:
                o.writelines([f.readline() for _ in range(4)])
            rr.run(args(one, 0))
        setup = time.perf_counter() - t0
        if log_setup:
            log("reference: setup (reference loads, index build) %.1f s" % setup)
        for c, samples in plan:
            secs = sum(rr.run(args(path, j)) for j, (L, path, _) in enumerate(samples))
            steps.append((sum(n for _, _, n in samples), secs))
    return setup, steps[warmup:], steps[:warmup]


def reference_arm(a, w):
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from resident import binary
    if not os.path.exists(binary(w["mode"] == "colour")):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (the reference's sources were absent)"}))
        return
    if a.cfg != 2:
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm is defined for the default workload"}))
        return
    chunks = list(range(a.warmup + a.steps))
    ref, paths, d = chunked_inputs(a, w, chunks)
    plan = [(c, per_length_sample(paths[c], d, REF_SAMPLE_PER_LENGTH, "refsample%d" % c)) for c in chunks]
    setup, steps, _ = run_reference_resident(w, ref, plan, d, threads, a.warmup)
    reads = sum(n for n, _ in steps)
    secs = sum(s for _, s in steps)
    value = reads / secs
    sample = ("each step: the first %d reads of each length of the step's chunk (%d reads), the reference's "
              "stock command line run once per length with its reference and index resident (setup %.1f s, "
              "untimed)" % (REF_SAMPLE_PER_LENGTH, steps[0][0] if steps else 0, setup))
    line = {"metric": "mapped reads/sec", "value": value, "unit": "reads/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1000 * secs / max(1, a.steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/int16/int32", "data": "synthetic", "impl": "reference",
            "config": headline_config(a, w), "sample": sample,
            "cpu_baseline": {"value": value, "unit": "reads/s", "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "includes": "read file in, SAM file out (the stock command line per length)"},
            "reference_setup_s": setup}
    print(json.dumps(line))


# ------------------------------------------------------------------------------ headline arm

def mixed_arm(a, w):
    """The workloads whose read set is drawn in chunks (mixed-length, large): one chunk per
    step, reference and index resident."""
    import ctypes

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    from storm_b200 import api, build, host, pipeline
    build.build()
    per_rank = a.warmup + a.steps
    chunks = [rank * per_rank + k for k in range(per_rank)]
    t0 = time.perf_counter()
    ref_path, paths, d = chunked_inputs(a, w, sorted(set(chunks + [0])), rank)
    log("rank %d: inputs ready in %.1f s" % (rank, time.perf_counter() - t0))

    p, seeds, *_ = pipeline.parse_options(w["args"])
    seeds = seeds or DEFAULT_SEEDS[0]
    prm = api.params(colour=0, device=local, **p)
    reference = host.Reference(ref_path, 0)
    mapper = api.Mapper(prm, seeds)
    reference.add_to(mapper)
    t0 = time.perf_counter()
    mapper.build_index()
    mapper.sync()
    index_cold_ms = mapper.stats()["ms_index"]
    mapper.build_index()  # again: the first build also grows the memory pool
    mapper.sync()
    index_ms = mapper.stats()["ms_index"]
    log("rank %d: index built in %.1f ms (device; first build %.1f ms), %.2f s wall"
        % (rank, index_ms, index_cold_ms, time.perf_counter() - t0))

    sets = {c: host.ReadSet(paths[c], 0) for c in chunks}
    max_len = max(s.max_len for s in sets.values())
    tbs = ((max_len + prm.allowed_indels + 1) // 2 + 7) & ~7
    t0 = time.perf_counter()
    if a.tuning:
        mapper.set_tuning(**{k: int(v) for k, v in (kv.split("=") for kv in a.tuning.split(","))})
        tuning = mapper.tuning()
    else:
        tuning = mapper.autotune(sets[chunks[0]].batch(), sample=a.tune_sample)
    tune_s = time.perf_counter() - t0
    log("rank %d: tuning %s (%.1f s)" % (rank, tuning, tune_s))

    # device-resident inputs of every step, uploaded before the timed region
    dev_in = {}
    for c in chunks:
        b = sets[c].batch()
        dc = torch.from_numpy(b.codes).to(dev)
        dl = torch.from_numpy(b.levels).to(dev)
        dn = torch.from_numpy(b.lengths.copy()).to(dev)
        dev_in[c] = (dc, dl, dn, api.Reads(b.n, dc.data_ptr(), b.codes.shape[1], dl.data_ptr(), b.levels.shape[1],
                                             dn.data_ptr(), None))
    nmax = max(s.n for s in sets.values())
    d_hits = torch.empty(nmax * 4 * ctypes.sizeof(api.Hit), dtype=torch.uint8, device=dev)
    d_tb = torch.empty(nmax * 4 * tbs, dtype=torch.uint8, device=dev)
    d_mapped = torch.empty(nmax, dtype=torch.uint8, device=dev)
    ostruct = api.Results(d_hits.data_ptr(), d_tb.data_ptr(), tbs, d_mapped.data_ptr())
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    for c in chunks[:a.warmup]:
        mapper.map_device(dev_in[c][3], ostruct, stream.cuda_stream)
    torch.cuda.synchronize()

    ms_steps, stats, mapped_total, reads_total = [], [], 0, 0
    with ClockSampler(local) as clk:
        for c in chunks[a.warmup:]:
            flush.fill_(1)
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            mapper.map_device(dev_in[c][3], ostruct, stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms_steps.append(e0.elapsed_time(e1))
            stats.append(mapper.stats())
            mapped_total += int(d_mapped[:sets[c].n].sum().item())
            reads_total += sets[c].n
    torch.cuda.synchronize()
    t_local = sum(ms_steps)
    t_max, reads_all = t_local, float(reads_total)
    if dist:
        t = torch.tensor([t_local], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
        n_all = torch.tensor([reads_total], dtype=torch.float64, device=dev)
        dist.all_reduce(n_all)
        reads_all = float(n_all.item())
    value = reads_all / (t_max / 1000.0)
    clocks = clk.summary()
    del dev_in
    mapper.close()

    # end to end through the resident front end: FASTQ file in, SAM file out, per chunk
    res_mapper = pipeline.ResidentMapper(ref_path, w["args"], colour=0, default_seeds=seeds, device=local)
    res_mapper.mapper.set_tuning(**tuning)
    e2e_chunks = chunks[a.warmup:a.warmup + max(1, min(a.steps, a.e2e_steps))]
    res_mapper.map_file(paths[chunks[0]], os.path.join(d, "warm.sam"))  # warm-up (buffers, page cache)
    e2e_s, h2d, d2h = [], 0, 0
    for c in e2e_chunks:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        res_mapper.map_file(paths[c], os.path.join(d, "e2e_%d.sam" % c))
        e2e_s.append(time.perf_counter() - t0)
        s = sets[c]
        h2d += s.codes.nbytes + s.levels.nbytes + s.lengths.nbytes
        d2h += s.n * (4 * ctypes.sizeof(api.Hit) + 4 * tbs + 1)
    e2e_t = sum(e2e_s)
    if dist:
        t = torch.tensor([e2e_t], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = float(t.item())
    e2e_reads = sum(sets[c].n for c in e2e_chunks) * world
    e2e = {"value": e2e_reads / e2e_t, "unit": "reads/s", "h2d_bytes_per_step": int(h2d / len(e2e_chunks)),
           "d2h_bytes_per_step": int(d2h / len(e2e_chunks)), "steps": len(e2e_chunks),
           "includes": "read FASTQ file -> parse + tag sort -> host-to-device -> map -> device-to-host -> SAM file",
           "api": "storm_b200.pipeline.ResidentMapper.map_file"}

    parity = batching = cpu = None
    if rank == 0:
        parity = check_parity(a, res_mapper, paths, d)
        if a.cfg == 2:  # reads of several lengths
            batching = batched_vs_plain(res_mapper, sets[chunks[a.warmup]], tbs, api)
            batching["command_line"] = cli_batching(ref_path, paths[chunks[a.warmup]], d, w)
    res_mapper.close()
    if rank == 0 and world == 1 and not a.no_cpu_baseline and a.cfg == 2:
        cpu = cpu_baseline_leg(a, w)

    if rank == 0:
        agg = {k: sum(s[k] for s in stats) for k in stats[0] if k != "ms_index"}
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        stages = stage_rooflines(agg, reads_total, max_len, sm_mhz, (index_ms, index_bytes(seeds, w["ref_sizes"])))
        stages["index_build"]["first_build_ms"] = index_cold_ms
        per_step = {k: v for k, v in stages.items() if not k.startswith("_")}
        dom = max(("sw_filter", "full_align", "hit_gather"), key=lambda k: per_step.get(k, {}).get("ms", 0))
        traffic = None
        if os.path.exists(TRAFFIC_PATH) and dom == "sw_filter" and agg.get("passes") and (a.cfg, a.scale) == (2, 1.0):
            per_cell = json.load(open(TRAFFIC_PATH)).get("mixed_100M", {}).get(dom, {}).get("bytes_per_cell_update")
            if per_cell:  # measured on a small case, scaled to the mean launch of the timed steps
                traffic = per_cell * agg["filter_cells"] / agg["passes"]
        roof = {"kernel": dom, "bound": per_step[dom]["bound"], "achieved": per_step[dom]["achieved"],
                "peak": per_step[dom]["peak"], "unit": per_step[dom]["unit"], "frac": per_step[dom]["frac"],
                "traffic": traffic,
                "peak_source": stages["_peak_sources"]["int" if per_step[dom]["bound"] == "int" else "hbm"]}
        for k, v in per_step.items():
            if "ms" in v and k != "index_build":  # the index is built once, before the steps
                v["ms_per_step"] = v["ms"] / len(stats)
        line = {"metric": "mapped reads/sec", "value": value, "unit": "reads/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": t_max / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u8/int16/int32", "data": "synthetic",
                "config": headline_config(a, w),
                "sample": "each step: one chunk of %d reads (chunk = step index + %d x rank), reference and index "
                          "resident" % (synth.CHUNK_READS, per_rank),
                "tuning": tuning, "tuning_s": round(tune_s, 2),
                "mapped_fraction": mapped_total / max(1, reads_total),
                "gpu_launches": int(sum(s["kernels"] for s in stats)),
                "cuda_graph": {"passes": int(agg["passes"]), "graph_passes": int(agg["graph_passes"])},
                "roofline": roof, "stages": stages, "clocks": clocks, "e2e": e2e, "cpu_baseline": cpu,
                "parity_vs_reference": parity, "batching": batching,
                "counts_per_step": {k: int(agg[k] / len(stats)) for k in
                                    ("candidates", "filter_passed", "aligned", "seed_lookups", "hit_positions",
                                     "filter_cells", "filter_band_cells", "align_cells")}}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


PARITY_CASE = {2: "mixed_100M_chunk0", 4: "large_3G_10k"}


def check_parity(a, res_mapper, paths, d):
    """The workload's at-scale parity case through the resident front end against the digests
    of the reference's own runs: for the mixed-length workload chunk 0, one run per read length,
    and the mixed run's records against the per-length ones; for the large one its 10k-read
    sample, one run."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import scale_cases
    case = PARITY_CASE.get(a.cfg)
    digests = json.load(open(DIGESTS_PATH)) if os.path.exists(DIGESTS_PATH) else {}
    if case not in digests:
        return {"case": case, "checked": False, "why": "no reference digests for the case"}
    ref_d = digests[case]
    pd = os.path.join(d, "parity")
    os.makedirs(pd, exist_ok=True)
    if scale_cases.CASES[case]["kind"] == "single":
        w, _, reads = scale_cases.make_inputs(case, pd)
        sam, un = os.path.join(pd, "all.sam"), os.path.join(pd, "all.un.fq")
        res_mapper.map_file(reads, sam, un)
        h, nrec = scale_cases.digest_sam(sam)
        exp = ref_d["runs"]["all"]
        return {"case": case, "checked": True, "runs": 1, "records": nrec,
                "identical": h == exp["sam_sha256"] and scale_cases.digest_file(un) == exp["unmapped_fastq_sha256"]}
    ok, runs, bodies = True, 0, []
    for L, path, n in per_length_sample(paths[0], pd, None, "chunk0"):
        sam = os.path.join(pd, "len%d.sam" % L)
        un = os.path.join(pd, "len%d.un.fq" % L)
        res_mapper.map_file(path, sam, un)
        h, nrec = scale_cases.digest_sam(sam)
        exp = ref_d["runs"].get("len%d" % L)
        ok &= exp is not None and h == exp["sam_sha256"] and scale_cases.digest_file(un) == exp["unmapped_fastq_sha256"]
        runs += 1
        with open(sam, "rb") as f:
            bodies.append(b"".join(x for x in f if not x.startswith(b"@")))
    mixed = os.path.join(pd, "mixed.sam")
    res_mapper.map_file(paths[0], mixed)
    with open(mixed, "rb") as f:
        mixed_body = b"".join(x for x in f if not x.startswith(b"@"))
    return {"case": case, "checked": True, "runs": runs, "identical": bool(ok and runs == len(ref_d["runs"])),
            "mixed_run_equals_per_length_runs": mixed_body == b"".join(bodies)}


def batched_vs_plain(res_mapper, reads, tbs, api):
    """One chunk: one mapping call over every read length (the batched form) against one call
    per length (the plain per-batch path the reference implies), host buffers in and out for
    both, best of two after a warm-up; and whether both give the same records."""
    import numpy as np
    m = res_mapper.mapper
    batch = reads.batch()
    L = reads.lengths
    cuts = [0] + [int(i) for i in np.nonzero(np.diff(L))[0] + 1] + [reads.n]
    buckets = [api.ReadBatch(batch.codes[x:y], batch.lengths[x:y], batch.levels[x:y]) for x, y in zip(cuts, cuts[1:])]
    whole = m.map(batch, tbs)
    for b in buckets:
        m.map(b, tbs)
    tb_, tp_ = [], []
    for _ in range(2):
        t0 = time.perf_counter()
        parts = [m.map(b, tbs) for b in buckets]
        tp_.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        whole = m.map(batch, tbs)
        tb_.append(time.perf_counter() - t0)
    hits = np.concatenate([p.hits for p in parts])
    mapped = np.concatenate([p.mapped for p in parts])
    live = np.repeat(mapped != 0, 4)
    same = bool(np.array_equal(mapped != 0, whole.mapped != 0) and hits[live].tobytes() == whole.hits[live].tobytes())
    return {"reads": int(reads.n), "batched_ms": 1000 * min(tb_), "plain_per_length_ms": 1000 * min(tp_),
            "plain_calls": len(buckets), "batched_over_plain": min(tp_) / min(tb_), "same_records": same}


def cli_batching(ref_path, reads_path, d, w):
    """The drop-in command line on one chunk, wall clock, file in and SAM out: one run over the
    mixed-length file, against one run per read length (what the reference needs: it maps one
    read length per run, reads_data.c:418-426); every run loads the reference, builds the index
    and starts the device."""
    from storm_b200 import build
    exe = os.path.join(build.BIN_DIR, "storm-nucleotide")
    cd = os.path.join(d, "cli")
    os.makedirs(cd, exist_ok=True)

    def run(path, tag):
        t0 = time.perf_counter()
        p = subprocess.run([exe, "-g", ref_path, "-r", path, "-o", os.path.join(cd, tag + ".sam"), "-v", "0"]
                           + list(w["args"]), capture_output=True)
        if p.returncode:
            raise RuntimeError("command line failed: %s" % p.stderr[-500:])
        return time.perf_counter() - t0

    run(reads_path, "warm")
    mixed = run(reads_path, "mixed")
    per = [run(path, "len%d" % L) for L, path, _ in per_length_sample(reads_path, cd, None, "cli")]
    return {"mixed_run_s": mixed, "per_length_runs_s": sum(per), "runs": len(per),
            "mixed_over_per_length": sum(per) / mixed}


def cpu_baseline_leg(a, w):
    """The reference on this host's cores on a bounded sample: the first reads of each length
    of one chunk, index resident (its setup is reported, not counted)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from resident import binary
    if not os.path.exists(binary(False)):
        return None
    ref, paths, d = chunked_inputs(a, w, [a.warmup])
    plan = [(a.warmup, per_length_sample(paths[a.warmup], d, REF_SAMPLE_PER_LENGTH, "cpusample"))]
    setup, _, warm = run_reference_resident(w, ref, plan, d, os.cpu_count() or 1, 1, log_setup=False)
    n, secs = warm[0]
    return {"value": n / secs, "unit": "reads/s", "cores": os.cpu_count(), "kind": "reference",
            "sample": "the first %d reads of each length of chunk %d (%d reads), stock command line per length, "
                      "reference and index resident (setup %.1f s, not counted)" % (REF_SAMPLE_PER_LENGTH, a.warmup,
                                                                                    n, setup)}


# ------------------------------------------------------------------------------ other workloads

def whole_set_arm(a, w):
    """Workloads mapped whole per step (colour, small nucleotide, large): every read of the
    set, both strands, index build included, device-resident results."""
    import ctypes

    import torch
    from storm_b200 import api, build, host, pipeline
    build.build()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ref_path, reads_path, d = whole_inputs(a, w)
    colour = 1 if w["mode"] == "colour" else 0
    p, seeds, *_ = pipeline.parse_options(w["args"])
    seeds = seeds or DEFAULT_SEEDS[colour]
    prm = api.params(colour=colour, device=local, **p)
    reads = host.ReadSet(reads_path, colour)
    reference = host.Reference(ref_path, colour)
    n = reads.n
    tbs = ((reads.max_len + prm.allowed_indels + 1) // 2 + 7) & ~7
    mapper = api.Mapper(prm, seeds)
    reference.add_to(mapper)
    mapper.build_index()
    batch = reads.batch()
    if a.tuning:
        mapper.set_tuning(**{k: int(v) for k, v in (kv.split("=") for kv in a.tuning.split(","))})
        tuning = mapper.tuning()
    else:
        tuning = mapper.autotune(batch, sample=a.tune_sample)
    d_codes = torch.from_numpy(batch.codes).to(dev)
    d_levels = torch.from_numpy(batch.levels).to(dev) if batch.levels is not None else None
    d_len = torch.from_numpy(batch.lengths.copy()).to(dev)
    d_fl = torch.from_numpy(batch.first_levels).to(dev) if batch.first_levels is not None else None
    d_hits = torch.empty(n * 4 * ctypes.sizeof(api.Hit), dtype=torch.uint8, device=dev)
    d_tb = torch.empty(n * 4 * tbs, dtype=torch.uint8, device=dev)
    d_mapped = torch.empty(n, dtype=torch.uint8, device=dev)
    rstruct = api.Reads(n, d_codes.data_ptr(), batch.codes.shape[1], d_levels.data_ptr() if d_levels is not None else None,
                        batch.levels.shape[1] if batch.levels is not None else 0, d_len.data_ptr(),
                        d_fl.data_ptr() if d_fl is not None else None)
    ostruct = api.Results(d_hits.data_ptr(), d_tb.data_ptr(), tbs, d_mapped.data_ptr())
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    def step():
        mapper.build_index()
        mapper.map_device(rstruct, ostruct, stream.cuda_stream)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    ms, stats = [], []
    with ClockSampler(local) as clk:
        for _ in range(a.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            stats.append(mapper.stats())
    clocks = clk.summary()
    mapper.close()
    value = n * a.steps / (sum(ms) / 1000.0)
    res_mapper = pipeline.ResidentMapper(ref_path, w["args"], colour=colour, default_seeds=seeds, device=local)
    res_mapper.mapper.set_tuning(**tuning)
    res_mapper.map_file(reads_path, os.path.join(d, "warm.sam"))
    t0 = time.perf_counter()
    res_mapper.map_file(reads_path, os.path.join(d, "e2e.sam"))
    e2e_s = time.perf_counter() - t0
    res_mapper.close()
    st = stats[-1]
    stages = stage_rooflines(st, n, reads.max_len, clocks.get("sm_mhz") or 1965.0,
                             (st["ms_index"], index_bytes(seeds, w["ref_sizes"])))
    per = {k: v for k, v in stages.items() if not k.startswith("_")}
    dom = max(("sw_filter", "full_align", "hit_gather"), key=lambda k: per.get(k, {}).get("ms", 0))
    line = {"metric": "mapped reads/sec", "value": value, "unit": "reads/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": sum(ms) / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8/int16/int32", "data": "synthetic",
            "config": dict(headline_config(a, w), step="index build (all seeds) + map every read, both strands"),
            "tuning": tuning, "gpu_launches": int(sum(s["kernels"] for s in stats)),
            "cuda_graph": {"passes": int(sum(s["passes"] for s in stats)),
                           "graph_passes": int(sum(s["graph_passes"] for s in stats))},
            "roofline": {"kernel": dom, **{k: per[dom][k] for k in ("bound", "achieved", "peak", "unit", "frac")},
                         "traffic": None},
            "stages": stages, "clocks": clocks,
            "e2e": {"value": n / e2e_s, "unit": "reads/s", "h2d_bytes_per_step": int(batch.codes.nbytes),
                    "d2h_bytes_per_step": int(n * (4 * ctypes.sizeof(api.Hit) + 4 * tbs + 1)),
                    "includes": "read FASTQ file -> SAM file through storm_b200.pipeline.ResidentMapper (index resident)"}}
    print(json.dumps(line))


def serving_arm(a, w):
    """The served -O chain: the workload's reads split into batches of log-uniform sizes (1k to
    1M reads, scaled), arriving as a Poisson process (seed 7).  The same batches first go through
    the plain per-batch path (each chain step mapped with stormgpu_map, the unmapped reads
    picked on the host, one batch at a time); then the server takes them as they arrive
    (continuous batching).  Reports the served reads/s, the plain reads/s, p50/p99 batch
    latency, and checks that both give the same records."""
    import numpy as np

    from storm_b200 import api, build, host, pipeline
    build.build()
    ref_path, reads_path, d = whole_inputs(a, w)
    p, _, *_ = pipeline.parse_options(w["args"])
    prm = api.params(colour=0, **p)
    chain = w["chain"]
    reads = host.ReadSet(reads_path, 0)
    reference = host.Reference(ref_path, 0)
    rng = np.random.default_rng(7)
    perm = rng.permutation(reads.n)
    lo, hi = max(1, int(1000 * a.scale)), max(2, int(1000000 * a.scale))
    batches, k = [], 0
    while k < reads.n:
        size = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        idx = np.sort(perm[k:k + size])
        k += size
        batches.append(api.ReadBatch(reads.codes[idx], reads.lengths[idx], reads.levels[idx]))
    tbs = ((reads.max_len + prm.allowed_indels + 1) // 2 + 7) & ~7
    total = sum(b.n for b in batches)
    mappers = []
    for seeds in chain:
        m = api.Mapper(prm, seeds)
        reference.add_to(m)
        m.build_index()
        mappers.append(m)
    tuning = mappers[0].autotune(api.ReadBatch(reads.codes, reads.lengths, reads.levels), sample=a.tune_sample)
    for m in mappers[1:]:
        m.set_tuning(**tuning)

    def plain(batch):
        n = batch.n
        out = api.MapResults(n, tbs)
        step = np.full(n, 255, np.uint8)
        ids, cur = np.arange(n), batch
        for s, m in enumerate(mappers):
            if cur.n == 0:
                break
            res = m.map(cur, tbs)
            got = np.nonzero(res.mapped != 0)[0]
            o = ids[got]
            for q in range(4):
                out.hits[4 * o + q] = res.hits[4 * got + q]
                out.tb[4 * o + q] = res.tb[4 * got + q]
            out.mapped[o] = 1
            step[o] = s
            keep = np.nonzero(res.mapped == 0)[0]
            ids = ids[keep]
            cur = api.ReadBatch(cur.codes[keep], cur.lengths[keep], cur.levels[keep])
        return out, step

    plain(batches[0])
    t0 = time.perf_counter()
    ref_out = [plain(b) for b in batches]
    t_plain = time.perf_counter() - t0
    for m in mappers:
        m.close()
    plain_rate = total / t_plain
    srv = api.Server(prm, chain, slots=3, budget_bytes=48 << 30)
    reference.add_to_server(srv)
    srv.set_tuning(**tuning)
    srv.build()
    srv.poll(srv.submit(batches[0], tbs))

    def serve(arrivals):
        tickets = [None] * len(batches)
        start = time.perf_counter()

        def submitter():
            for i, b in enumerate(batches):
                dt = start + arrivals[i] - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                tickets[i] = srv.submit(b, tbs)

        th = threading.Thread(target=submitter)
        th.start()
        lat, outs = [], []
        for i in range(len(batches)):
            while tickets[i] is None:
                time.sleep(0.0005)
            res, step, ms = srv.poll(tickets[i])
            lat.append(ms)
            outs.append((res, step))
        el = time.perf_counter() - start
        th.join()
        return el, lat, outs

    t_served, _, outs = serve(np.zeros(len(batches)))
    cap = total / t_served
    gaps = rng.exponential(total / (0.8 * cap) / len(batches), size=len(batches))
    _, lat, outs2 = serve(np.concatenate([[0.0], np.cumsum(gaps[:-1])]))
    srv.close()
    same = True
    for (res, step), (pres, pstep) in list(zip(outs, ref_out)) + list(zip(outs2, ref_out)):
        live = np.repeat(pres.mapped != 0, 4)
        same &= bool(np.array_equal(step, pstep) and np.array_equal(res.mapped != 0, pres.mapped != 0) and
                     res.hits[live].tobytes() == pres.hits[live].tobytes())
    served_rate = total / t_served
    line = {"metric": "served reads/sec (3-step -O chain, continuous batching)", "value": served_rate,
            "unit": "reads/s", "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8/int16/int32", "data": "synthetic",
            "config": {"tuning": tuning, "workload": workload_name(a.cfg, a.scale), "reads": total,
                       "batches": len(batches), "batch_sizes": [b.n for b in batches], "chain": chain,
                       "args": " ".join(w["args"]),
                       "arrivals": "capacity: all batches at once; latency: Poisson at 80 % of capacity", "slots": 3},
            "serving": {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                        "plain_reads_per_s": plain_rate, "served_over_plain": served_rate / plain_rate,
                        "same_records": same},
            "e2e": {"value": served_rate, "unit": "reads/s",
                    "h2d_bytes_per_step": int(sum(b.codes.nbytes + b.levels.nbytes + b.lengths.nbytes for b in batches)),
                    "d2h_bytes_per_step": int(sum(b.n * (4 * 28 + 4 * tbs + 2) for b in batches)),
                    "includes": "host buffers in, every chain step, results out"}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cfg", type=int, default=2)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=5, help="chunks timed end to end")
    ap.add_argument("--tune-sample", type=int, default=8000, help="reads the autotuner times each setting on")
    ap.add_argument("--tuning", default="", help="launch parameters name=value,... instead of the autotuner")
    a = ap.parse_args()
    w = synth.workload(a.cfg, a.scale)
    rank = int(os.environ.get("RANK", "0"))
    if a.impl == "reference":
        if rank == 0:
            reference_arm(a, w)
        return
    if a.cfg in (2, 4):
        mixed_arm(a, w)
    elif a.cfg == 3:
        if rank == 0:
            serving_arm(a, w)
    elif rank == 0:
        whole_set_arm(a, w)


if __name__ == "__main__":
    main()
