"""rocrand_b200_set_output_position: a generator positioned at output r*n writes outputs
[r*n, (r+1)*n) of the stream one fresh generator writes in one call -- the slice a rank of a
multi-GPU job fills, with no communication.  Checked for the stateful engines (where the
offset cannot place two-value distributions) and the counter engines, across the 131072-
engine rotation, against one long call of the same library (itself pinned to the reference
by the parity tests)."""

import ctypes

import numpy as np
import pytest

import rocrand_b200 as rb
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu

OUTPUT = {"uint": 0, "uniform": 4, "uniform_double": 5, "normal": 7, "normal_double": 8,
          "log_normal": 10, "poisson": 13}
GENERATORS = {"xorwow": 401, "mrg32k3a": 402, "mrg31k3p": 405, "lfsr113": 406, "philox": 404,
              "threefry4x32": 410, "threefry2x64": 409}


@pytest.mark.parametrize("name", sorted(GENERATORS))
@pytest.mark.parametrize("dist,params", [("uniform_double", []), ("normal", [0.0, 1.0]),
                                         ("normal_double", [0.0, 1.0]), ("uint", []),
                                         ("poisson", [10.0])])
def test_slices_equal_one_long_call(lib, name, dist, params):
    rng = GENERATORS[name]
    seed = 0x5EED + rng
    n = 2 * 131072 + 6  # crosses the engine rotation, a multiple of every output width
    ranks = 3
    g = gu.create(lib, rng, seed)
    try:
        st, whole = gu.device_generate(lib, g, dist, ranks * n, params, 0)
    finally:
        lib.rocrand_destroy_generator(g)
    assert st == 0
    for r in range(ranks):
        g = gu.create(lib, rng, seed)
        try:
            assert lib.rocrand_b200_set_output_position(g, OUTPUT[dist], r * n) == 0
            st, part = gu.device_generate(lib, g, dist, n, params, 0)
            assert st == 0
            # and the next call continues the same stream
            st2, more = gu.device_generate(lib, g, dist, 1000, params, 0)
            assert st2 == 0
        finally:
            lib.rocrand_destroy_generator(g)
        want = whole[r * n:(r + 1) * n]
        assert np.array_equal(part.view(np.uint8), want.view(np.uint8)), (name, dist, r)
        if r < ranks - 1:
            assert np.array_equal(more.view(np.uint8), whole[(r + 1) * n:(r + 1) * n + 1000].view(np.uint8))


def test_position_errors(lib):
    g = gu.create(lib, rb.ROCRAND_RNG_PSEUDO_MT19937, 1)
    try:
        assert lib.rocrand_b200_set_output_position(g, 0, 0) == rb.ROCRAND_STATUS_TYPE_ERROR
    finally:
        lib.rocrand_destroy_generator(g)
    g = gu.create(lib, rb.ROCRAND_RNG_PSEUDO_XORWOW, 1)
    try:
        # normal outputs come in pairs: an odd index is not a vector boundary
        assert lib.rocrand_b200_set_output_position(g, OUTPUT["normal"], 7) == \
            rb.ROCRAND_STATUS_LENGTH_NOT_MULTIPLE
        assert lib.rocrand_b200_set_output_position(g, 99, 0) == rb.ROCRAND_STATUS_OUT_OF_RANGE
        assert lib.rocrand_b200_set_output_position(g, OUTPUT["uint"], 12345) == 0
    finally:
        lib.rocrand_destroy_generator(g)
    assert lib.rocrand_b200_set_output_position(None, 0, 0) == rb.ROCRAND_STATUS_NOT_CREATED
