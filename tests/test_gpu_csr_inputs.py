"""CSR counts at the C-ABI boundary: the device-side checks and the
per-gene statistics read the rows as 16-byte pieces, so rows that start
and end anywhere inside a piece, empty rows, and an array whose last piece
ends past nnz must give exactly what the element-by-element definitions
give; malformed CSR input must be rejected with the library's message
(the reference's own entry points assume well-formed matrices from R).
"""
import numpy as np
import pytest

from devil_b200 import synthetic

pytestmark = pytest.mark.gpu

INVALID = "invalid CSR"


def _small(seed=5, G=40, n=1500):
    return synthetic.make("plain_sparse", seed=seed, G=G, n=n)


def _fit(dv, rowptr, col, val, n, X):
    return dv.fit_devil((rowptr, col, val, n), X, overdispersion="MOM", size_factors="normed_sum")


def _rows_with(P, k, at_least=3):
    """Rows with at least `at_least` entries, spread over the matrix."""
    cnt = np.diff(P.rowptr)
    rows = np.flatnonzero(cnt >= at_least)
    return rows[np.linspace(0, len(rows) - 1, k).astype(int)]


@pytest.mark.parametrize("kind", ["unsorted", "duplicate", "too_large", "negative"])
def test_malformed_cell_indices_rejected(dv, kind):
    P = _small()
    for g in _rows_with(P, 3):  # first, middle and last eligible rows
        col = P.col.copy()
        a = int(P.rowptr[g])
        if kind == "unsorted":
            col[a], col[a + 1] = col[a + 1], col[a]
        elif kind == "duplicate":
            col[a + 2] = col[a + 1]
        elif kind == "too_large":
            col[a + 1] = P.n
        else:
            col[a] = -1
        with pytest.raises(dv.DevilError, match=INVALID):
            _fit(dv, P.rowptr, col, P.val, P.n, P.X)


def test_malformed_row_pointers_rejected(dv):
    P = _small()
    rp = P.rowptr.copy()
    g = len(rp) // 2
    rp[g] = rp[g + 1] + 1  # a row that ends before it starts
    with pytest.raises(dv.DevilError, match=INVALID):
        _fit(dv, rp, P.col, P.val, P.n, P.X)


@pytest.mark.parametrize("shift", [0, 1, 3, 5, 7])
def test_gene_statistics_at_every_row_alignment(dv, orc, shift):
    """theta_0 (from the per-gene sums) and the fit agree with the oracle
    when every row boundary moves by `shift` entries: leading empty rows
    and a prefix row change where each row starts within its piece, and
    dropping entries at the end leaves nnz at every residue mod 8."""
    P = _small(seed=11 + shift)
    # a first row of `shift` counts in the first cells, then an empty row
    lead_col = np.arange(shift, dtype=np.int32)
    lead_val = np.full(shift, 2, dtype=P.val.dtype)
    cut = shift  # drop the last `cut` entries of the last row
    last = len(P.rowptr) - 2
    keep = P.rowptr[-1] - min(cut, int(P.rowptr[-1] - P.rowptr[last]))
    col = np.concatenate([lead_col, P.col[:keep]])
    val = np.concatenate([lead_val, P.val[:keep]])
    rp = np.concatenate([[0, shift, shift], P.rowptr[1:] + shift]).astype(np.int64)
    rp[-1] = len(col)
    rp = np.minimum(rp, len(col))
    csr = (rp, col, val, P.n)
    Y = np.zeros((len(rp) - 1, P.n))
    for g in range(len(rp) - 1):
        Y[g, col[rp[g]:rp[g + 1]]] = val[rp[g]:rp[g + 1]]
    # (given size factors: a draw this small leaves cells without counts)
    off = np.log(P.sf_true)
    th = dv.estimate_dispersion(csr, off)
    np.testing.assert_allclose(th, orc.estimate_dispersion(Y, off), rtol=1e-12)
    fit = dv.fit_devil(csr, P.X, overdispersion="MOM", size_factors=P.sf_true)
    assert np.isfinite(fit["beta"][2:]).all()
