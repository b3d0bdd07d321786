"""The package's Python mirror of the reference binding (rocrand_b200.PRNG / QRNG, after
python/rocrand/rocrand/rocrand.py:148-357) generating on the GPU.

The generate cases the reference's own suite runs against its binding
(python/rocrand/tests/rocrand_test.py: every generator type, numpy arrays and device
buffers, generate / uniform / normal / lognormal / poisson, the `size` argument and its
errors) are exercised here through the mirror, and every bit-exact output is compared with
the oracle making the same calls.
"""

import numpy as np
import pytest

import rocrand_b200 as rb
from oracle import pyorc

pytestmark = pytest.mark.gpu

PRNGS = [rb.ROCRAND_RNG_PSEUDO_XORWOW, rb.ROCRAND_RNG_PSEUDO_MRG32K3A, rb.ROCRAND_RNG_PSEUDO_MTGP32,
         rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10, rb.ROCRAND_RNG_PSEUDO_MRG31K3P, rb.ROCRAND_RNG_PSEUDO_LFSR113,
         rb.ROCRAND_RNG_PSEUDO_MT19937, rb.ROCRAND_RNG_PSEUDO_THREEFRY2_32_20,
         rb.ROCRAND_RNG_PSEUDO_THREEFRY4_32_20]
QRNGS = [rb.ROCRAND_RNG_QUASI_SOBOL32, rb.ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL32,
         rb.ROCRAND_RNG_QUASI_SOBOL64, rb.ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL64]


@pytest.fixture(scope="module")
def orc():
    return pyorc.CLib("orc")


@pytest.mark.parametrize("rng", PRNGS)
def test_prng_numpy_outputs_equal_oracle(orc, rng):
    seed, n = 0xC0FFEE, 10007
    gen = rb.PRNG(rng, seed=seed)
    outs = [gen.generate(np.empty(n, dtype=np.uint32)), gen.uniform(np.empty(n, dtype=np.float32)),
            gen.uniform(np.empty(n, dtype=np.float64)), gen.poisson(np.empty(n, dtype=np.uint32), 12.5)]
    calls = [("uint", n, [], 0), ("uniform", n, [], 0), ("uniform_double", n, [], 0),
             ("poisson", n, [12.5], 0)]
    ref = pyorc.run_sequence(orc, rng, seed, None, calls)
    for (d, _, _, _), got, (st, exp) in zip(calls, outs, ref):
        assert st == 0
        assert np.array_equal(got.view(np.uint8), exp.view(np.uint8)), (rng, d)


@pytest.mark.parametrize("rng", PRNGS + QRNGS)
def test_device_tensors_and_size(rng):
    import torch
    gen = rb.QRNG(rng, ndim=2) if rng in QRNGS else rb.PRNG(rng, seed=7)
    x = torch.zeros(4096, dtype=torch.float32, device="cuda")
    gen.uniform(x, size=2048)  # a size within the buffer: only the first 2048 are written
    torch.cuda.synchronize()
    assert bool((x[:2048] > 0).all()) and bool((x[:2048] <= 1).all())
    assert bool((x[2048:] == 0).all())
    with pytest.raises(ValueError):
        gen.uniform(x, size=8192)
    y = torch.empty(4096, dtype=torch.float64, device="cuda")
    gen.normal(y, 0.0, 1.0)
    torch.cuda.synchronize()
    assert abs(float(y.mean())) < 0.2 and 0.8 < float(y.std()) < 1.2
    z = torch.empty(4096, dtype=torch.float32, device="cuda")
    gen.lognormal(z, 0.0, 0.5)
    torch.cuda.synchronize()
    assert bool((z > 0).all())


@pytest.mark.parametrize("rng", QRNGS)
def test_qrng_numpy_outputs_equal_oracle(orc, rng):
    dims, n = 3, 3 * 4001
    gen = rb.QRNG(rng, ndim=dims)
    got = gen.uniform(np.empty(n, dtype=np.float64))
    st, exp = pyorc.run_sequence(orc, rng, None, None, [("uniform_double", n, [], 0)], dims=dims)[0]
    assert st == 0 and np.array_equal(got.view(np.uint8), exp.view(np.uint8))
    # a size that is not a multiple of the dimensions is the reference's LENGTH_NOT_MULTIPLE
    with pytest.raises(rb.RocRandError) as e:
        gen.uniform(np.empty(10, dtype=np.float64))
    assert e.value.value == rb.ROCRAND_STATUS_LENGTH_NOT_MULTIPLE
