"""The oracle-side square scene (oracle/square_scene.py, used by the CPU
baseline and the reference arm of bench.py so that they need no product
library) equals the product builder's scene widened to FP64, record by
record."""
import numpy as np
import pytest

import numi_cloth as nc
import oracle_py as op
import square_scene


@pytest.mark.parametrize("side,fruits", [(24, 6), (48, 64)])
def test_oracle_square_scene_equals_product(side, fruits):
    prod = nc.square_scene(side=side, fruitCount=fruits)
    want = op.from_abi(prod)
    got = square_scene.build(side=side, fruit_count=fruits)
    for name in ("particles", "distances", "bends", "grips", "fruits", "pairs"):
        a, b = getattr(got, name), getattr(want, name)
        assert a.dtype == b.dtype and len(a) == len(b), name
        assert a.tobytes() == b.tobytes(), name
    for field, _ in op.Params._fields_:
        assert np.array_equal(np.asarray(getattr(got.params, field)), np.asarray(getattr(want.params, field))), field
    cfg = nc.substep_configs(prod, 3)
    assert square_scene.substeps(got, 3).tobytes() == op.substeps_from_configs(cfg).tobytes()
