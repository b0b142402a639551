"""The streamed DF build's aux blocking (DFEngine.aux_blocks), host only:
consecutive shell ranges that cover the aux basis once, each within the
requested function count unless one shell alone exceeds it."""

import types

import pytest

from felizjueves_b200 import configs
from felizjueves_b200.df import DFEngine


@pytest.mark.parametrize("limit", [1, 15, 40, 384, 10 ** 6])
def test_aux_blocks_cover_the_basis(limit):
    w = configs.cluster(2, 5)
    aux = configs.aux_basis(w)
    blocks = DFEngine.aux_blocks(types.SimpleNamespace(aux=aux), limit)
    assert blocks[0][0] == 0 and blocks[0][2] == 0
    assert blocks[-1][1] == len(aux.shells) and blocks[-1][3] == aux.n_ao
    for (s0, s1, p0, p1), nxt in zip(blocks, blocks[1:] + [None]):
        assert s0 < s1 and p0 == aux.offsets[s0]
        assert p1 - p0 == sum(aux.shells[s].n_cart for s in range(s0, s1))
        assert p1 - p0 <= limit or s1 == s0 + 1
        if nxt is not None:
            assert nxt[0] == s1 and nxt[2] == p1
