"""Full-size (2M-parcel) properties that need no oracle run: exact tiling, symmetric touches, plain == filtered."""
import numpy as np
import pytest

import gsj
from gsj import gen

pytestmark = pytest.mark.gpu
BOX = (-119.0, 33.0, -117.0, 35.0)


@pytest.fixture(scope="module")
def big(engine):
    ps = gen.layer_parcels(2_000_000, BOX, seed=0)
    return engine.upload_polygons(ps), ps


def test_self_join_full_size(engine, big):
    L, ps = big
    plain = engine.join(L, L, want_area=True, want_relate=True, upper=True, refine_mode=gsj.GSJ_REFINE_PLAIN)
    filt = engine.join(L, L, want_area=True, want_relate=True, upper=True, refine_mode=gsj.GSJ_REFINE_FILTERED)
    i, j = np.lexsort(plain.pairs.T[::-1]), np.lexsort(filt.pairs.T[::-1])
    assert np.array_equal(plain.pairs[i], filt.pairs[j])      # 0 pair diffs between the two variants
    assert np.array_equal(plain.code[i], filt.code[j]) and np.array_equal(plain.area[i], filt.area[j])
    diag = plain.pairs[:, 0] == plain.pairs[:, 1]
    assert diag.sum() == L.info["n"]
    assert abs(plain.area[diag].sum() - 4.0) < 1e-9            # parcels tile the 2 x 2 degree box
    assert np.abs(plain.area[~diag]).max() < 1e-15             # neighbours only touch
    ii = plain.code[~diag] & 3                                  # interiors never meet off the diagonal
    assert (ii == 0).all()
