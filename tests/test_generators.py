"""Generator contracts that the parity and bench workloads rely on (CPU only)."""
import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import structural_rank

from mumblebee_b200 import generators as G


def test_exppow_free_block_has_full_structural_rank():
    """Free columns have a zero Hessian block, so δH + BᵀB is definite on them only if B's free
    block has full column rank.  The generator gives every free column an entry in a row of its
    own; at the full n = 20000 size (4000 free columns, m = 5000, 0.1% density) the random pattern
    alone leaves five single-entry free columns sharing a row."""
    pb = G.exppow(seed=0)
    B = sp.csc_matrix(pb["B"])
    assert B.shape == (5000, 20000)
    f0 = 3 * (3000 + 1000)
    assert pb["kinds"][4000] == G.CONE_FREE and pb["sizes"][4000] == 4000
    assert structural_rank(B[:, f0:f0 + 4000].tocsr()) == 4000
    assert np.all(np.diff(B.indptr) > 0)
    assert np.isfinite(pb["g"]).all() and np.isfinite(pb["f"]).all()


def test_exppow_is_seeded():
    a = G.exppow(nexp=20, npow=10, nfree=15, npos=15, m=40, density=0.05, seed=3)
    b = G.exppow(nexp=20, npow=10, nfree=15, npos=15, m=40, density=0.05, seed=3)
    assert (sp.csc_matrix(a["B"]) != sp.csc_matrix(b["B"])).nnz == 0
    np.testing.assert_array_equal(a["f"], b["f"])
