"""Generate the golden vectors under tests/golden/ by running the reference itself.

The reference (forced-dns-sm.py + particles.py) is a script that runs at import.  This generator
reads its source text from the reference checkout, substitutes the driver parameters
(N, T, Nprtcl) and inserts ``np.random.seed(seed)`` after the numpy import, then ``exec``s it
in a fresh namespace inside a scratch directory (the script writes its npz outputs relative to
the working directory).  ``mpi4py`` and ``h5py`` are replaced by the single-rank stand-ins in
``_standin/`` (neither is installed here); numba runs with one thread so the racy scatter of
particles.py:26-34 is deterministic.

Two runs are made per case with the same seed:
  * ``init`` - the evolve call at forced-dns-sm.py:766 is replaced by ``pass``, so the namespace
    holds the initial field (F:691-736) and the initial droplets (P:91-96); the reference's own
    functions (rfft_mpi, irfft_mpi, forcing, full_RHS, e3d_to_e1d, stb.interp_cosine, ...) are
    then called on that state to record per-function input/output pairs;
  * ``run``  - T = nsteps*dt, so evolve_and_save (F:556-627) advances nsteps RK4 steps.

Only the recorded arrays are written (``*.npz``); no reference source enters the repository.
This script needs the reference checkout and is run by hand in the build container:

    NUMBA_NUM_THREADS=1 python tests/golden/make_golden.py <reference_dir>

The reference checkout is the first argument, or the environment variable LD_REFERENCE_DIR.
"""
import contextlib
import io
import os
import pathlib
import re
import sys
import tempfile

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
STANDIN = HERE / "_standin"


def _patched_source(ref_dir, N, nsteps, nprtcl, seed, run):
    src = (pathlib.Path(ref_dir) / "forced-dns-sm.py").read_text()

    def sub(pattern, repl):
        nonlocal src
        new, n = re.subn(pattern, repl, src, count=1, flags=re.M)
        if n != 1:
            raise RuntimeError(f"pattern not found in reference: {pattern!r}")
        src = new

    sub(r"^import numpy as np\s*$", f"import numpy as np\nnp.random.seed({seed})")
    sub(r"^N = 256\s*$", f"N = {N}")
    sub(r"^T = 40\s*$", f"T = {nsteps}*dt")
    sub(r"^Nprtcl = 0\s*$", f"Nprtcl = {nprtcl}")
    if not run:
        sub(r"^evolve_and_save\(t,u,n\)\s*$", "pass")
    return src


def run_reference(ref_dir, N, nsteps, nprtcl, seed, run):
    """Exec the patched reference script; return its module namespace."""
    os.environ.setdefault("NUMBA_NUM_THREADS", "1")
    src = _patched_source(ref_dir, N, nsteps, nprtcl, seed, run)
    old_path, old_cwd = list(sys.path), os.getcwd()
    for m in ("particles", "mpi4py", "h5py"):
        sys.modules.pop(m, None)
    sys.path[:0] = [str(STANDIN), str(ref_dir)]
    tmp = tempfile.mkdtemp(prefix="ld_golden_")
    ns = {"__name__": "__reference__", "__file__": str(pathlib.Path(tmp) / "forced-dns-sm.py")}
    try:
        os.chdir(tmp)
        with contextlib.redirect_stdout(io.StringIO()):
            exec(compile(src, "forced-dns-sm.py", "exec"), ns)
    finally:
        os.chdir(old_cwd)
        sys.path[:] = old_path
    return ns


def record_functions(ns, seed):
    """Per-function input/output pairs on the initial state of an ``init`` run."""
    out = {}
    N, Nf = ns["N"], ns["Nf"]
    rng = np.random.default_rng(seed + 1000)
    # operators (F:123-141)
    for key in ("kint", "dealias", "normalize", "invlap"):
        out[f"op_{key}"] = np.asarray(ns[key])
    out["N"] = N
    out["nu"] = ns["nu"]
    out["dt"] = ns["dt"]
    out["f0"] = ns["f0"]
    out["tps"] = ns["tps"]
    out["tf"] = ns["tf"]
    out["g"] = ns["g"]
    out["shell_no"] = np.asarray(ns["shell_no"])
    # initial physical field and droplets (F:691-736, P:91-96)
    out["init_u"] = np.asarray(ns["u"]).copy()
    out["init_n"] = np.asarray(ns["n"]).copy()
    stb = ns["stb"]
    out["init_coord"] = stb.coord.copy()
    out["init_prtclid"] = stb.prtclid.copy()
    out["prt_factor"] = stb.factor
    out["prt_growthfactor"] = stb.growthfactor
    # rfft_mpi / irfft_mpi (F:201-213) on seeded random data
    a = rng.standard_normal((N, N, N))
    fa = np.zeros((N, N, Nf), np.complex128)
    out["fft_in"] = a
    out["fft_out"] = ns["rfft_mpi"](a.copy(), fa).copy()
    b = (rng.standard_normal((N, N, Nf)) + 1j * rng.standard_normal((N, N, Nf)))
    ub = np.zeros((N, N, N))
    out["ifft_in"] = b
    out["ifft_out"] = ns["irfft_mpi"](b.copy(), ub).copy()
    # the spectral state evolve_and_save starts from (F:567-569)
    uk = np.zeros((3, N, N, Nf), np.complex128)
    for c in range(3):
        uk[c] = ns["rfft_mpi"](out["init_u"][c].copy(), np.zeros((N, N, Nf), np.complex128)) * ns["dealias"]
    out["uk0"] = uk.copy()
    # forcing (F:239-275) and the shell spectrum it builds (F:232-233, F:243-245)
    fk = np.zeros_like(uk)
    out["forcing_fk"] = np.asarray(ns["forcing"](uk.copy(), fk)).copy()
    out["forcing_ek_arr"] = np.asarray(ns["ek_arr"]).copy()
    # cosine interpolation (P:435-511) of the 7 fields [u, u, n] at the initial droplets
    if stb.coord.shape[0] > 0:
        fields = np.concatenate((out["init_u"], out["init_u"] * 0.5, out["init_n"][None]), axis=0)
        coord = stb.coord.copy()
        coord[:, :3] %= ns["L"]
        out["interp_coord"] = coord.copy()
        out["interp_out"] = stb.interp_cosine(coord, fields).copy()
    return out


def main(ref_dir):
    ref_dir = pathlib.Path(ref_dir)
    cases = [
        # name, N, nsteps, nprtcl, seed
        ("N16", 16, 2, 64, 7),
        ("N32", 32, 2, 256, 11),
    ]
    for name, N, nsteps, nprtcl, seed in cases:
        ns0 = run_reference(ref_dir, N, nsteps, nprtcl, seed, run=False)
        rec = record_functions(ns0, seed)
        # the full RHS (F:287-332) on the initial state: velocity, n-field and droplet parts
        uk0 = rec["uk0"].copy()
        stb = ns0["stb"]
        n0 = np.ones((N, N, N))
        coord = stb.coord.copy()
        ku, kn, kp, sump = ns0["full_RHS"](0.0, uk0.copy(), n0.copy(), coord.copy(), coord.copy(), stb)
        rec["rhs_ku"] = np.asarray(ku).copy()
        rec["rhs_kn"] = np.asarray(kn).copy()
        rec["rhs_kp"] = np.asarray(kp).copy()
        rec["rhs_prtclid"] = stb.prtclid.copy()
        rec["rhs_coord_in"] = coord
        rec["rhs_fc"] = np.asarray(ns0["fc"]).copy()
        rec["rhs_interpmat"] = stb.interpmat.copy()
        # nsteps of the reference's own time loop (F:556-627)
        ns1 = run_reference(ref_dir, N, nsteps, nprtcl, seed, run=True)
        rec["nsteps"] = nsteps
        rec["run_uk"] = np.asarray(ns1["uk"]).copy()
        rec["run_n"] = np.asarray(ns1["n"]).copy()
        rec["run_coord"] = ns1["stb"].coord.copy()
        rec["run_prtclid"] = ns1["stb"].prtclid.copy()
        if N > 16:
            # the per-function pairs are pinned at N=16; larger cases keep the time-loop pins only
            for key in [k for k in rec if k.startswith(("fft_", "ifft_", "op_", "forcing_fk"))]:
                del rec[key]
        path = HERE / f"ref_{name}.npz"
        np.savez_compressed(path, **rec)
        print(f"wrote {path} ({path.stat().st_size/1e6:.2f} MB)")


def reference_dir(argv=None):
    """The reference checkout: the first argument, else $LD_REFERENCE_DIR; no default."""
    argv = sys.argv[1:] if argv is None else argv
    d = argv[0] if argv else os.environ.get("LD_REFERENCE_DIR")
    if not d:
        raise SystemExit("usage: make_golden.py <reference_dir>  (or set LD_REFERENCE_DIR)")
    return d


if __name__ == "__main__":
    main(reference_dir())
