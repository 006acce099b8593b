"""Configuration generation, host side: the generator's block function
against the published Philox4x32-10 known-answer vectors (Random123), and
the committed over-relaxation fixture against GLU's own OR_lattice."""
import numpy as np
import pytest

from glu_b200 import update

# Philox4x32-10 known-answer vectors (Random123 distribution, kat_vectors)
KAT = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
       ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
       ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
        (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    assert update.philox4x32_10(ctr, key) == want


def test_or_fixture_is_glus(reference, lat400):
    dims = tuple(int(d) for d in lat400["dims"])
    reference.setup(dims)
    reference.put_links(lat400["links"])
    reference.overrelax(2)
    assert np.array_equal(reference.get_links(), lat400["or2_links"])


def test_unit_config():
    U = update.unit_config((2, 2, 2, 2))
    assert U.shape == (16, 4, 3, 3)
    assert np.array_equal(U[3, 2], np.eye(3))
