"""Single-rank stand-in for ``mpi4py.MPI``.

Test infrastructure only: ``tests/golden/make_golden.py`` puts this package on
``sys.path`` so that the upstream qttools package (which imports ``mpi4py`` at
module import time) can be imported in a process with no MPI installation. Every
collective is the identity on one rank.
"""

import numpy as _np

SUM = "sum"
PROD = "prod"
MAX = "max"
MIN = "min"
LAND = "land"
IN_PLACE = object()


def Get_library_version() -> str:
    return "single-rank shim"


class Request:
    def Wait(self):
        return None

    @staticmethod
    def Waitall(reqs):
        return None


def _copy(sendbuf, recvbuf):
    if sendbuf is IN_PLACE:
        return
    s = sendbuf[0] if isinstance(sendbuf, (list, tuple)) else sendbuf
    r = recvbuf[0] if isinstance(recvbuf, (list, tuple)) else recvbuf
    _np.copyto(_np.asarray(r).reshape(-1), _np.asarray(s).reshape(-1))


class Intracomm:
    rank = 0
    size = 1

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def Get_info(self):
        return {}

    def Split(self, color=0, key=0):
        return Intracomm()

    def Barrier(self):
        return None

    barrier = Barrier

    def Allreduce(self, sendbuf, recvbuf, op=SUM):
        _copy(sendbuf, recvbuf)

    def Allgather(self, sendbuf, recvbuf):
        _copy(sendbuf, recvbuf)

    def Alltoall(self, sendbuf, recvbuf):
        _copy(sendbuf, recvbuf)

    def Bcast(self, buf, root=0):
        return None

    def bcast(self, obj, root=0):
        return obj

    def allgather(self, obj):
        return [obj]

    def gather(self, obj, root=0):
        return [obj]

    def allreduce(self, obj, op=SUM):
        return obj

    def Ibcast(self, buf, root=0):
        return Request()


Comm = Intracomm
COMM_WORLD = Intracomm()
