"""This library against the reference's own device kernels on the same B200.

oracle/Makefile.ref gpu compiles the reference's sources for sm_100a into
oracle/_ref/librocrand_ref_gpu.so (its host-API generators with their device kernels, test
infrastructure only).  The small reference case -- Philox4x32-10, seed 1234, uniform fp32,
2^24 values -- must be byte-identical across this library, the reference's kernel and the
digest recorded from the reference's host generator; and for every pseudo-random generator
the bit-exact outputs of a call sequence (sizes, misalignments, width changes) must equal the
reference kernels' outputs.  The reference's kernels are the pin for MT19937, whose host
emulation in the reference differs from its own kernels on some unaligned calls.
"""

import ctypes
import hashlib
import json
import os
import zlib

import numpy as np
import pytest

import rocrand_b200 as rb
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "librocrand_ref_gpu.so")

PSEUDO = {"philox": 404, "threefry2x32": 408, "threefry2x64": 409, "threefry4x32": 410,
          "threefry4x64": 411, "xorwow": 401, "mrg32k3a": 402, "mrg31k3p": 405, "lfsr113": 406,
          "mt19937": 407, "mtgp32": 403}


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_GPU):
        pytest.skip("oracle/_ref/librocrand_ref_gpu.so not built (make -C oracle -f Makefile.ref gpu)")
    return rb.load_library(REF_GPU)


def _run(L, rng, seed, calls):
    """The calls on a fresh generator of library L; numpy outputs."""
    import torch
    g = ctypes.c_void_p()
    assert L.rocrand_create_generator(ctypes.byref(g), rng) == 0
    try:
        assert L.rocrand_set_seed(g, seed) == 0
        outs = []
        for dist, n, params, mis in calls:
            st, vals = gu.device_generate(L, g, dist, n, params, mis)
            assert st == 0, (rng, dist, st)
            outs.append(vals)
        torch.cuda.synchronize()
        return outs
    finally:
        L.rocrand_destroy_generator(g)


def test_config1_three_way(lib, ref):
    with open(os.path.join(ROOT, "tests", "golden", "full_digests.json")) as f:
        want = json.load(f)["philox/uniform/seed1234/2^24"]["sha256"]
    calls = [("uniform", 1 << 24, [], 0)]
    ours = _run(lib, 404, 1234, calls)[0]
    theirs = _run(ref, 404, 1234, calls)[0]
    assert hashlib.sha256(ours.view(np.uint8).tobytes()).hexdigest() == want
    assert np.array_equal(ours.view(np.uint32), theirs.view(np.uint32))


@pytest.mark.parametrize("name", sorted(PSEUDO))
def test_bit_exact_outputs_equal_reference_kernels(lib, ref, name):
    rs = np.random.default_rng(zlib.crc32(name.encode()))
    seed = int(rs.integers(0, 2**63))
    calls = [("uint", (1 << 20) + 3, [], 1), ("uniform", 77, [], 0), ("short", 12345, [], 3),
             ("uniform_double", (1 << 18) + 1, [], 0), ("poisson", 50001, [10.0], 2),
             ("uniform_half", 999, [], 1), ("char", 4099, [], 5), ("poisson", 3000, [1000.0], 0),
             ("uint", 1 << 21, [], 0)]
    ours = _run(lib, PSEUDO[name], seed, calls)
    theirs = _run(ref, PSEUDO[name], seed, calls)
    for (dist, n, _, _), a, b in zip(calls, ours, theirs):
        assert a.shape == b.shape
        bad = np.nonzero(a.view(np.uint8) != b.view(np.uint8))[0]
        assert bad.size == 0, (name, dist, n, int(bad[0]))
