"""Empty stand-in for ``h5py``: the reference imports it (forced-dns-sm.py:8) but its only
users, ``load_hdf5``/``save_hdf5``, are never called on the path the golden generator runs."""
