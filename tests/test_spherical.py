"""Real solid harmonics over the Cartesians (felizjueves_b200/spherical.py):
the reference's own table (eri/density_fit/kernel_eri3.py aux_harmonics,
l = 0..6) to 1e-14; orthonormality of a one-centre shell normalised as its
(l, 0, 0) component; the block-diagonal transform's layout."""

import math

import numpy as np
import pytest

from conftest import golden
from felizjueves_b200 import spherical
from felizjueves_b200.shell import Basis, Shell, primitive_norm


@pytest.mark.parametrize("l", range(7))
def test_harmonics_match_reference(l):  # noqa: E741
    g = golden("harmonics.npz")
    assert np.abs(spherical.harmonics(l) - g[f"l{l}"]).max() <= 1e-14


@pytest.mark.parametrize("l", range(4))
def test_one_centre_shell_is_orthonormal(oracle_lib, l):  # noqa: E741
    """A shell whose (l, 0, 0) component is normalised maps to 2l+1
    orthonormal spherical functions: T^T S T = 1."""
    from oracle import one_electron
    a = 0.9
    B = Basis((Shell(l, (0.3, -0.2, 0.1), [a], [primitive_norm(l, a)]),))
    S = one_electron.matrices(B, [])[0]
    T = spherical.transform(B)
    assert abs(S[0, 0] - 1.0) <= 1e-14
    assert np.abs(T.T @ S @ T - np.eye(2 * l + 1)).max() <= 1e-13


def test_transform_layout():
    B = Basis((Shell(0, (0, 0, 0), [1.0], [1.0]), Shell(2, (0, 0, 1), [1.0], [1.0]),
               Shell(1, (0, 1, 0), [1.0], [1.0]), Shell(3, (1, 0, 0), [1.0], [1.0])))
    T = spherical.transform(B)
    assert T.shape == (1 + 6 + 3 + 10, 1 + 5 + 3 + 7) and spherical.n_spherical(B) == 16
    assert T[0, 0] == 1.0 and np.array_equal(T[7:10, 6:9], np.eye(3))
    assert np.array_equal(T[1:7, 1:6], spherical.harmonics(2).T)
    with pytest.raises(ValueError):
        spherical.harmonics(-1)
    assert math.isclose(spherical.harmonics(2)[0, 1], math.sqrt(3.0))  # xy of m = -2
