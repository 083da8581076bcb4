"""Single-rank stand-in for ``mpi4py.util.pkl5`` (fixture generation only)."""


def Intracomm(comm):
    return comm
