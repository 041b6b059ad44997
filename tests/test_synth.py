"""The synthetic generator is deterministic, hits its density and has canonical CSR rows."""

import numpy as np

from cusingler_b200 import synth


def test_deterministic_and_worker_independent():
    w1, r1, q1 = synth.custom_dataset(300, 100, 2000, 5, 0.08, seed=11, workers=1)
    w2, r2, q2 = synth.custom_dataset(300, 100, 2000, 5, 0.08, seed=11, workers=2)
    for a, b in ((r1, r2), (q1, q2)):
        assert np.array_equal(a.data, b.data) and np.array_equal(a.indices, b.indices)
        assert np.array_equal(a.indptr, b.indptr) and np.array_equal(a.labels, b.labels)


def test_density_and_canonical_rows():
    w, ref, qry = synth.custom_dataset(2000, 10, 5000, 6, 0.06, seed=2, workers=1)
    dens = ref.nnz / (ref.n_rows * ref.n_cols)
    assert 0.045 < dens < 0.075
    assert (ref.data > 0).all()
    for r in range(0, ref.n_rows, 97):
        cols = ref.indices[ref.indptr[r]:ref.indptr[r + 1]]
        assert (np.diff(cols) > 0).all()
