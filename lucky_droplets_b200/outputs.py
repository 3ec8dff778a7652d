"""Output and restart files with the reference's names and keys (forced-dns-sm.py save(),
F:419-460; load_npz, F:374-407).

On one rank the reference writes, in its output directory:
  Fields_k_0.npz       uk, vk, wk: the spectral velocity, (N, N, N/2+1) complex, (kx, ky, kz)
  Energy_spectrum.npz  ek: shell spectrum (N/2+1)
  Flux_spectrum.npz    Pik: flux spectrum, the reversed cumulative sum of the shell transfer
  <droplet dir>/state_0.npz  pos, vel, mass, prtclid, umat (droplets; mass only where droplets
                       carry one)
  <n dir>/n_0.npz      n: the droplet number-density field, where one is advanced
With P ranks every rank writes its own slab: Fields_k_{r}.npz holds the spectra of the ky
slab r (shape (N, N/P, N/2+1), ky = r N/P .. (r+1) N/P - 1; F:158, F:446) and n_{r}.npz the
physical n of the x slab r (shape (N/P, N, N); F:150, F:449-450).  load_npz (F:374-407) reads
such a checkpoint back on any rank count: it counts the Fields files and takes ky plane j from
slab j // (N/P) at index j % (N/P).  read_fields / read_n here do the same for one GPU, which
holds every slab.
The writers here take host arrays; ForcedDNS.save/.load move the device state.
"""
import pathlib

import numpy as np


def reference_dirs(save_path, t, wg="", sts=0.0, stb=None):
    """The reference's directory names for an output at time t (F:439-440, F:453): the field
    directory time_{t:.1f} and, with droplets, the droplet directory below it."""
    root = pathlib.Path(save_path) / f"time_{t:.1f}"
    drop = root / (f"{wg}_stb_{stb:.3f}_sts_{sts:.3f}" if stb is not None else f"{wg}_sts_{sts:.3f}")
    return root, drop


def write_outputs(dirpath, uk_full, ek, pik, state=None, n=None, n_dir=None, rank=0, slabs=1):
    """Write the reference's files into dirpath (created); returns the written paths.

    slabs = P > 1 writes the checkpoint a P-rank run leaves: Fields_k_{r}.npz and n_{r}.npz for
    every slab r (P must divide N); `rank` is then ignored."""
    d = pathlib.Path(dirpath)
    d.mkdir(parents=True, exist_ok=True)
    uk_full = np.asarray(uk_full)
    N = uk_full.shape[1]
    if slabs < 1 or N % slabs:
        raise ValueError(f"{slabs} slabs do not divide N = {N}")
    Np = N // slabs
    ranks = [rank] if slabs == 1 else list(range(slabs))
    paths = []
    for r in ranks:
        sl = slice(0, N) if slabs == 1 else slice(r * Np, (r + 1) * Np)
        paths.append(d / f"Fields_k_{r}.npz")
        np.savez_compressed(paths[-1], uk=uk_full[0][:, sl], vk=uk_full[1][:, sl], wk=uk_full[2][:, sl])
    paths += [d / "Energy_spectrum.npz", d / "Flux_spectrum.npz"]
    np.savez_compressed(paths[-2], ek=np.asarray(ek))
    np.savez_compressed(paths[-1], Pik=np.asarray(pik))
    if n is not None:
        nd = pathlib.Path(n_dir) if n_dir is not None else d
        nd.mkdir(parents=True, exist_ok=True)
        n = np.asarray(n)
        for r in ranks:
            sl = slice(0, N) if slabs == 1 else slice(r * Np, (r + 1) * Np)
            paths.append(nd / f"n_{r}.npz")
            np.savez_compressed(paths[-1], n=n[sl])
    if state is not None:
        sd = pathlib.Path(state.pop("dir", d))
        sd.mkdir(parents=True, exist_ok=True)
        paths.append(sd / f"state_{rank}.npz")
        np.savez_compressed(paths[-1], **{k: np.asarray(v) for k, v in state.items()})
    return paths


class CheckpointError(ValueError):
    """A restart directory that does not hold a complete, consistent checkpoint."""


def _slab_files(d, stem):
    """The slab files stem_0.npz .. stem_{P-1}.npz of a checkpoint directory, in slab order."""
    d = pathlib.Path(d)
    if not d.is_dir():
        raise CheckpointError(f"no checkpoint directory {d}")
    found = {}
    for f in d.iterdir():
        name = f.name
        if name.startswith(stem + "_") and name.endswith(".npz"):
            idx = name[len(stem) + 1:-4]
            if idx.isdigit():
                found[int(idx)] = f
    if not found:
        raise CheckpointError(f"no {stem}_<slab>.npz in {d}")
    P = len(found)
    if sorted(found) != list(range(P)):
        raise CheckpointError(f"{stem} slabs of {d} are not 0..{P - 1}: {sorted(found)}")
    return [found[r] for r in range(P)]


def _load(path, keys):
    try:
        with np.load(path) as f:
            missing = [k for k in keys if k not in f.files]
            if missing:
                raise CheckpointError(f"{path.name} lacks {missing}")
            return [f[k] for k in keys]
    except CheckpointError:
        raise
    except Exception as e:  # truncated or corrupt archives
        raise CheckpointError(f"cannot read {path}: {type(e).__name__}: {e}") from e


def read_fields(dirpath):
    """(3, N, N, N/2+1) spectral velocity from the Fields_k_{slab}.npz files of a checkpoint
    written by any number of ranks: the ky slabs are put back in order (load_npz, F:374-407)."""
    parts = [np.stack(_load(f, ["uk", "vk", "wk"])) for f in _slab_files(dirpath, "Fields_k")]
    N, Nf = parts[0].shape[1], parts[0].shape[3]
    for f, a in zip(_slab_files(dirpath, "Fields_k"), parts):
        if a.ndim != 4 or a.shape[1] != N or a.shape[3] != Nf or a.shape[2] != parts[0].shape[2]:
            raise CheckpointError(f"{f.name}: slab shape {a.shape[1:]} does not match {parts[0].shape[1:]}")
    uk = np.concatenate(parts, axis=2)
    if uk.shape[2] != N or Nf != N // 2 + 1:
        raise CheckpointError(f"slabs give a ({N}, {uk.shape[2]}, {Nf}) spectrum, not ({N}, {N}, {N // 2 + 1})")
    return uk


def read_n(dirpath):
    """(N, N, N) number density from the n_{slab}.npz files of a checkpoint (x slabs in order,
    load_npz F:391-396)."""
    files = _slab_files(dirpath, "n")
    parts = [_load(f, ["n"])[0] for f in files]
    n = np.concatenate(parts, axis=0)
    if n.ndim != 3 or not (n.shape[0] == n.shape[1] == n.shape[2]):
        raise CheckpointError(f"n slabs give shape {n.shape}, not (N, N, N)")
    return n


def flux_from_transfer(transfer):
    """Pik_arr of F:428: the reversed cumulative sum of the shell transfer."""
    t = np.asarray(transfer)
    return np.cumsum(t[::-1])[::-1]
