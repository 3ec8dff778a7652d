"""Time the reference's own time loop (forced-dns-sm.py + particles.py, unmodified apart from the
driver parameters) on this machine's host cores.

The reference is a Python script that runs at import; like make_golden.py this reads its source
from the reference checkout, substitutes N, T (= nsteps dt) and Nprtcl, seeds np.random, and
execs it single-rank with the mpi4py / h5py stand-ins of _standin/ (mpi4py and an MPI launcher
are not installed here), with NUMBA_NUM_THREADS = the host's core count.  The loop prints
"step i in time t" before step i (F:574), where t is the wall time of step i - 1 (its RK4 stages
and end-of-step epilogue, F:582-620); step 0 also pays numba's compilation, so it is reported but
left out of the median.  Nothing of the reference enters the repository; the script needs the
reference checkout and runs by hand:

    python tests/golden/time_reference.py <reference_dir> [--N 256] [--nprtcl 1000000] [--steps 4]

(the reference directory may also come from $LD_REFERENCE_DIR).  It prints one JSON line.
"""
import argparse
import contextlib
import io
import json
import os
import pathlib
import re
import statistics
import sys
import tempfile
import time

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import STANDIN, _patched_source  # noqa: E402


class _Tee(io.StringIO):
    """Collects the script's stdout with the host time of every write."""

    def __init__(self):
        super().__init__()
        self.stamps = []

    def write(self, s):
        self.stamps.append((time.perf_counter(), s))
        return super().write(s)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("reference_dir", nargs="?", default=os.environ.get("LD_REFERENCE_DIR"))
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--nprtcl", type=int, default=1_000_000)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    if not a.reference_dir:
        raise SystemExit("usage: time_reference.py <reference_dir>  (or set LD_REFERENCE_DIR)")
    ref_dir = pathlib.Path(a.reference_dir)
    cores = os.cpu_count() or 1
    os.environ["NUMBA_NUM_THREADS"] = str(cores)
    src = _patched_source(ref_dir, a.N, a.steps, a.nprtcl, a.seed, run=True)
    for m in ("particles", "mpi4py", "h5py"):
        sys.modules.pop(m, None)
    sys.path[:0] = [str(STANDIN), str(ref_dir)]
    tmp = tempfile.mkdtemp(prefix="ld_reftime_")
    ns = {"__name__": "__reference__", "__file__": str(pathlib.Path(tmp) / "forced-dns-sm.py")}
    out = _Tee()
    old = os.getcwd()
    t0 = time.perf_counter()
    try:
        os.chdir(tmp)
        with contextlib.redirect_stdout(out):
            exec(compile(src, "forced-dns-sm.py", "exec"), ns)
    finally:
        os.chdir(old)
    total = time.perf_counter() - t0
    steps = {}
    for m in re.finditer(r"step (\d+) in time ([0-9.eE+-]+)", out.getvalue()):
        steps[int(m.group(1))] = float(m.group(2))
    # the print before step i times step i - 1
    per_step = [steps[i] for i in sorted(steps) if i >= 1]
    clean = per_step[1:]
    res = {"what": "reference forced-dns-sm.py + particles.py time loop (RK4, n field, cosine droplets), "
                   "single rank with stand-in mpi4py, NUMBA_NUM_THREADS=cores",
           "N": a.N, "nprtcl": a.nprtcl, "cores": cores, "steps_run": a.steps,
           "s_per_step": per_step, "s_per_step_median_after_first": statistics.median(clean) if clean else None,
           "wall_s_total": total, "host": os.uname().nodename}
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
