"""Client of oracle/_ref/storm-*-resident (ref_resident.c): the reference's stock command line
run once per request in one long-lived process that keeps the reference sequences and their
indexes between runs.  Test and measurement infrastructure only: the parity fixtures and the
benchmark's reference arm use it; the product never does."""
from __future__ import annotations

import os
import subprocess

REF_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref")


def binary(colour: bool, resident: bool = True) -> str:
    name = ("storm-color" if colour else "storm-nucleotide") + ("-resident" if resident else "")
    return os.path.join(REF_DIR, name)


def reference_env():
    # the reference's colour-space SEQ field reads heap bytes it never set
    # (hit_map.c:243-251); a fixed fill byte for fresh allocations makes it deterministic
    return dict(os.environ, MALLOC_PERTURB_="255")


class ResidentReference:
    """One resident reference process.  run(args) maps with the stock options `args` (the
    program name excluded; give -o so that standard output stays free for the protocol) and
    returns the run's wall time in seconds, timed inside the process around the stock main()."""

    def __init__(self, colour: bool, threads: int | None = None, cwd: str | None = None):
        self.colour = colour
        self.threads = threads or os.cpu_count() or 1
        self.p = subprocess.Popen([binary(colour)], stdin=subprocess.PIPE, stdout=subprocess.PIPE,
                                  cwd=cwd, env=reference_env(), text=True, bufsize=1)

    def run(self, args) -> float:
        argv = [binary(colour=self.colour, resident=False)] + list(args) + ["-N", str(self.threads)]
        if any("\t" in a or "\n" in a for a in argv):
            raise ValueError("arguments may not hold tabs or newlines")
        self.p.stdin.write("\t".join(argv) + "\n")
        self.p.stdin.flush()
        line = self.p.stdout.readline()
        if not line.startswith("done "):
            raise RuntimeError("resident reference ended (exit %s) on %s" % (self.p.poll(), " ".join(argv)))
        _, rc, secs = line.split()
        if int(rc) != 0:
            raise RuntimeError("reference run returned %s: %s" % (rc, " ".join(argv)))
        return float(secs)

    def close(self):
        if self.p.poll() is None:
            self.p.stdin.close()
            self.p.wait(timeout=60)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
