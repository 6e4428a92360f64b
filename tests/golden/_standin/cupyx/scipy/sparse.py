"""Stand-in: cupyx.scipy.sparse.csr_matrix is SciPy's CSR (with a .get() that returns itself)."""
import scipy.sparse as _sp


class csr_matrix(_sp.csr_matrix):
    def get(self):
        return _sp.csr_matrix(self)
