"""Output and restart files with the reference's names and keys (forced-dns-sm.py save(),
F:419-460; load of the spectral fields, F:374-407).

On one rank the reference writes, in its output directory:
  Fields_k_0.npz       uk, vk, wk: the spectral velocity, (N, N, N/2+1) complex, (kx, ky, kz)
  Energy_spectrum.npz  ek: shell spectrum (N/2+1)
  Flux_spectrum.npz    Pik: flux spectrum, the reversed cumulative sum of the shell transfer
  <droplet dir>/state_0.npz  pos, vel, mass, prtclid, umat (droplets; mass only where droplets
                       carry one)
  <n dir>/n_0.npz      n: the droplet number-density field, where one is advanced
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


def write_outputs(dirpath, uk_full, ek, pik, state=None, n=None, n_dir=None, rank=0):
    """Write the reference's files into dirpath (created); returns the written paths."""
    d = pathlib.Path(dirpath)
    d.mkdir(parents=True, exist_ok=True)
    uk_full = np.asarray(uk_full)
    paths = [d / f"Fields_k_{rank}.npz", d / "Energy_spectrum.npz", d / "Flux_spectrum.npz"]
    np.savez_compressed(paths[0], uk=uk_full[0], vk=uk_full[1], wk=uk_full[2])
    np.savez_compressed(paths[1], ek=np.asarray(ek))
    np.savez_compressed(paths[2], Pik=np.asarray(pik))
    if n is not None:
        nd = pathlib.Path(n_dir) if n_dir is not None else d
        nd.mkdir(parents=True, exist_ok=True)
        paths.append(nd / f"n_{rank}.npz")
        np.savez_compressed(paths[-1], n=np.asarray(n))
    if state is not None:
        sd = pathlib.Path(state.pop("dir", d))
        sd.mkdir(parents=True, exist_ok=True)
        paths.append(sd / f"state_{rank}.npz")
        np.savez_compressed(paths[-1], **{k: np.asarray(v) for k, v in state.items()})
    return paths


def read_fields(dirpath, rank=0):
    """(3, N, N, N/2+1) spectral velocity from Fields_k_<rank>.npz."""
    f = np.load(pathlib.Path(dirpath) / f"Fields_k_{rank}.npz")
    return np.stack([f["uk"], f["vk"], f["wk"]])


def flux_from_transfer(transfer):
    """Pik_arr of F:428: the reversed cumulative sum of the shell transfer."""
    t = np.asarray(transfer)
    return np.cumsum(t[::-1])[::-1]
