"""Host generators (rocrand_create_generator_host / _host_blocking, rocrand.cpp:118-160).

Their outputs land in host memory and equal, bit for bit, those of the device generator of
the same type making the same calls with its output at the same alignment; the device
generators are checked against the oracle elsewhere.  Every generator type, every output
type it supports, several misalignments and call sequences that continue a stream.
"""

import ctypes
from ctypes import c_size_t, c_void_p

import numpy as np
import pytest

import rocrand_b200 as rb
from oracle import pyorc
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu

TYPES = {"philox": 404, "threefry2x32": 408, "threefry4x64": 411, "xorwow": 401, "mrg32k3a": 402,
         "mrg31k3p": 405, "lfsr113": 406, "mt19937": 407, "mtgp32": 403, "sobol32": 501,
         "scrambled_sobol64": 505}
CALLS = [("uniform", 1000, (), 1), ("uint", 70001, (), 0), ("normal_double", 4097, (0.5, 2.0), 1),
         ("poisson", 3000, (12.0,), 3), ("uniform_half", 777, (), 5), ("log_normal", 5000, (0.0, 0.5), 2),
         ("ulonglong", 999, (), 1)]


def _host_generate(lib, g, dist, n, params, mis):
    suffix, dt, _ = pyorc.DISTS[dist]
    isz = np.dtype(dt).itemsize
    raw = np.zeros((n + 1024 // isz + 16) * isz, dtype=np.uint8)
    base = (-raw.ctypes.data) % 512
    view = raw[base + mis * isz: base + (mis + n) * isz]
    fn = getattr(lib, "rocrand_" + suffix)
    st = fn(g, c_void_p(view.ctypes.data), c_size_t(n), *pyorc.dist_args(dist, params))
    return st, view.view(dt).copy()


@pytest.mark.parametrize("blocking", [0, 1])
@pytest.mark.parametrize("name", sorted(TYPES))
def test_host_generator_equals_device(lib, name, blocking):
    rng = TYPES[name]
    h = c_void_p()
    create = lib.rocrand_create_generator_host_blocking if blocking else lib.rocrand_create_generator_host
    assert create(ctypes.byref(h), rng) == 0
    d = gu.create(lib, rng)
    try:
        if rng < 500:
            assert lib.rocrand_set_seed(h, 0xC0FFEE) == lib.rocrand_set_seed(d, 0xC0FFEE) == 0
        else:
            assert lib.rocrand_set_quasi_random_generator_dimensions(h, 3) == 0
            assert lib.rocrand_set_quasi_random_generator_dimensions(d, 3) == 0
        for dist, n, params, mis in CALLS:
            if rng >= 500:
                n -= n % 3
            sh, vh = _host_generate(lib, h, dist, n, params, mis)
            sd, vd = gu.device_generate(lib, d, dist, n, params, mis)
            assert sh == sd, (dist, sh, sd)
            if sh == 0:
                assert np.array_equal(vh.view(np.uint8), vd.view(np.uint8)), dist
    finally:
        lib.rocrand_destroy_generator(h)
        lib.rocrand_destroy_generator(d)
