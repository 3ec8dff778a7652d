"""Single-rank stand-in for ``mpi4py`` used only to run the reference scripts in-process
when generating golden vectors (tests/golden/make_golden.py).

It implements the subset of ``MPI.COMM_WORLD`` that forced-dns-sm.py and particles.py call,
for a world of size 1:

* ``Alltoall`` / ``Alltoallv`` / ``Neighbor_alltoall`` / ``Neighbor_alltoallv`` copy the send
  buffer into the receive buffer flat (with one rank every block goes to itself; the graph made
  at particles.py:84 has two self-edges and each halo request comes back in the order it left);
* ``allreduce`` / ``allgather`` are the identity / a one-element list;
* ``Create_graph`` returns the communicator itself; ``Barrier`` does nothing; ``Abort`` raises.
"""
import numpy as _np


def _buf(b):
    # [array, datatype] or [array, counts, displs, datatype] or a bare array
    if isinstance(b, (list, tuple)):
        return b[0]
    return b


class _Comm:
    def Get_size(self):
        return 1

    def Get_rank(self):
        return 0

    def Barrier(self):
        return None

    def Abort(self, code=1):
        raise RuntimeError("MPI Abort called (stand-in)")

    def allreduce(self, x, op=None):
        return x

    def allgather(self, x):
        return [x]

    def _copy(self, send, recv):
        s = _np.asarray(_buf(send)).ravel()
        r = _buf(recv)
        rv = r.reshape(-1)
        n = min(s.size, rv.size)
        rv[:n] = s[:n]

    def Alltoall(self, send, recv):
        self._copy(send, recv)

    def Alltoallv(self, send, recv):
        self._copy(send, recv)

    def Neighbor_alltoall(self, send, recv):
        self._copy(send, recv)

    def Neighbor_alltoallv(self, send, recv):
        self._copy(send, recv)

    def Create_graph(self, index, edges, reorder=False):
        return self


class _MPI:
    COMM_WORLD = _Comm()
    DOUBLE = "double"
    DOUBLE_COMPLEX = "double_complex"
    SUM = "sum"
    MIN = "min"
    MAX = "max"


MPI = _MPI()
