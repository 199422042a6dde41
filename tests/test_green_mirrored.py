"""The mirrored Green tabulation (a quarter of the work) equals the plain restatement of
Green_3D (Green.f90:1-80); the reference arm of the benchmark tabulates its 512^3 table with it."""
import numpy as np
import pytest


@pytest.mark.parametrize("n,soft,rng_,gs", [(16, 4.0, 0.0, 0.5), (24, 3.5, 7.0, 0.5), (40, 4.0, 0.0, 0.25)])
def test_green_mirrored_equals_plain(oracle_lib, n, soft, rng_, gs):
    from oracle import oracle as O
    A = O.green(n, soft, rng_, gs)
    B = O.green_mirrored(n, soft, rng_, gs)
    assert np.max(np.abs(A - B)) <= 1e-7 * np.max(np.abs(A))
