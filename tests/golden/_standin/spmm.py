"""Stand-in for realworld/spmm.py: dense product with the SciPy CSR."""


def spmm(A, X):
    return A @ X
