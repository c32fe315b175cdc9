"""Write tests/golden/scale_digests.json: the reference's own outputs on the at-scale parity
cases of tests/scale_cases.py, as SHA-256 digests (the SAM without its @PG line, the -O FASTQ)
with record counts, the digest of the inputs and the reference's run times here.

The reference is the one compiled from its sources into oracle/_ref (make -C oracle ref):
its stock command line through the resident driver (oracle/ref_resident.c: reference and
indexes kept between the runs of a case), or the stock binary itself for a case of one run.
The GPU box regenerates the same inputs from the same seeds and compares digests.

    python tests/golden/make_scale_digests.py [case ...]      (default: every case)
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import scale_cases  # noqa: E402
from resident import ResidentReference, binary, reference_env  # noqa: E402

OUT = os.path.join(HERE, "scale_digests.json")


def run_case(name: str, work: str):
    c = scale_cases.CASES[name]
    d = os.path.join(work, name)
    os.makedirs(d, exist_ok=True)
    w, ref, reads = scale_cases.make_inputs(name, d)
    colour = w["mode"] == "colour"
    plan = scale_cases.runs(name, w, reads, d)
    for _, _, _, sam, un in plan:          # outputs of an earlier attempt must not feed a chain
        for p in (sam, un):
            if os.path.exists(p):
                os.remove(p)
    entry = {"case": c, "inputs_sha256_16": scale_cases.inputs_digest(ref, reads),
             "reads_per_length": scale_cases.sample_sizes(reads), "threads": os.cpu_count(), "runs": {}}
    t0 = time.time()
    if c["kind"] == "single":
        lab, src, seeds, sam, un = plan[0]
        args = scale_cases.command_args(w, seeds, src, sam, un, ref)
        t = time.time()
        subprocess.run([binary(colour, resident=False)] + args + ["-N", str(os.cpu_count())], check=True,
                       cwd=d, env=reference_env())
        secs = {lab: time.time() - t}
    else:
        secs = {}
        with ResidentReference(colour, cwd=d) as rr:
            for lab, src, seeds, sam, un in plan:
                if scale_cases.skip_run(src):
                    continue
                secs[lab] = rr.run(scale_cases.command_args(w, seeds, src, sam, un, ref))
    for lab, src, seeds, sam, un in plan:
        if lab not in secs:
            continue
        h, n = scale_cases.digest_sam(sam)
        entry["runs"][lab] = {"sam_sha256": h, "records": n, "unmapped_fastq_sha256": scale_cases.digest_file(un),
                              "seconds": round(secs[lab], 3)}
    entry["total_seconds"] = round(time.time() - t0, 1)
    return entry


def main(argv):
    names = argv or list(scale_cases.CASES)
    work = os.environ.get("STORM_SCALE_WORK") or tempfile.mkdtemp(prefix="storm_scale_")
    for name in names:
        print("case %s in %s" % (name, work), flush=True)
        entry = run_case(name, work)
        data = json.load(open(OUT)) if os.path.exists(OUT) else {}
        data[name] = entry
        json.dump(data, open(OUT, "w"), indent=1, sort_keys=True)
        print("  done in %.0f s" % entry["total_seconds"], flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
