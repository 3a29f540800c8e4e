"""The blocked Gauss-Jordan step structure of the coarse inverse
(peridigm_b200/csrc/k_coarse.cu), restated in oracle/oracle.py, against
numpy's inverse: SPD matrices whose order is below one block, a multiple of
the block, and ragged (the last block narrower), with the production block
width 64 and a narrow one; the symmetric form (tiles on and above the
diagonal only, tile side a multiple of the block) on the same cases. The GPU kernels are checked through
|Ac^-1 Ac - I| in tests/test_gpu_coarse.py."""
import numpy as np
import pytest

from oracle import oracle as O


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, n))
    return B @ B.T / n + np.diag(rng.uniform(0.5, 2.0, n))


@pytest.mark.parametrize("n,bk", [(40, 64), (128, 64), (300, 64), (375, 64), (97, 16)])
def test_blocked_gauss_jordan_inverts(n, bk):
    A = _spd(n, n + bk)
    Ai = O.gauss_jordan_blocked(A, bk=bk)
    ref = np.linalg.inv(A)
    assert np.abs(Ai - ref).max() <= 1e-10 * np.abs(ref).max()
    assert np.abs(Ai @ A - np.eye(n)).max() <= 1e-10


@pytest.mark.parametrize("n,bk,tile", [(40, 64, 128), (128, 64, 128), (300, 64, 128), (375, 64, 128),
                                       (97, 16, 32), (200, 16, 64), (300, 128, 128), (401, 128, 128)])
def test_symmetric_gauss_jordan_inverts(n, bk, tile):
    A = _spd(n, n + bk + tile)
    Ai = O.gauss_jordan_sym_blocked(A, bk=bk, tile=tile)
    ref = np.linalg.inv(A)
    assert np.isfinite(Ai).all()
    assert np.abs(Ai - ref).max() <= 1e-10 * np.abs(ref).max()
    assert np.abs(Ai - Ai.T).max() == 0.0
    assert np.abs(Ai @ A - np.eye(n)).max() <= 1e-10
