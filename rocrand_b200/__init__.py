"""rocrand_b200 -- B200-native random-number library with rocRAND's host C ABI.

The product is ``librocrand.so`` (built from ``csrc/``): the reference's C entry points
(rocrand_create_generator, rocrand_set_*, rocrand_generate_*) implemented in C++ over
hand-written sm_100a kernels.  This module is the Python host-side mirror of the
reference's ctypes binding (python/rocrand/rocrand/rocrand.py: ``RNG``, ``PRNG``, ``QRNG``,
``RocRandError``, same method names and argument meaning) and the loader every test and
benchmark goes through.  Arrays are torch CUDA tensors (device memory) or numpy arrays
(copied through a device tensor, as the reference binding does for host arrays).

There is no CPU fallback: if ``librocrand.so`` is missing, importing the loader raises.
"""

import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_size_t, c_uint, c_uint16, c_ulonglong, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librocrand.so")

# Status codes, generator types and orderings (library/include/rocrand/rocrand.h:59-126).
ROCRAND_STATUS_SUCCESS = 0
ROCRAND_STATUS_VERSION_MISMATCH = 100
ROCRAND_STATUS_NOT_CREATED = 101
ROCRAND_STATUS_ALLOCATION_FAILED = 102
ROCRAND_STATUS_TYPE_ERROR = 103
ROCRAND_STATUS_OUT_OF_RANGE = 104
ROCRAND_STATUS_LENGTH_NOT_MULTIPLE = 105
ROCRAND_STATUS_DOUBLE_PRECISION_REQUIRED = 106
ROCRAND_STATUS_LAUNCH_FAILURE = 107
ROCRAND_STATUS_INTERNAL_ERROR = 108

ROCRAND_RNG_PSEUDO_DEFAULT = 400
ROCRAND_RNG_PSEUDO_XORWOW = 401
ROCRAND_RNG_PSEUDO_MRG32K3A = 402
ROCRAND_RNG_PSEUDO_MTGP32 = 403
ROCRAND_RNG_PSEUDO_PHILOX4_32_10 = 404
ROCRAND_RNG_PSEUDO_MRG31K3P = 405
ROCRAND_RNG_PSEUDO_LFSR113 = 406
ROCRAND_RNG_PSEUDO_MT19937 = 407
ROCRAND_RNG_PSEUDO_THREEFRY2_32_20 = 408
ROCRAND_RNG_PSEUDO_THREEFRY2_64_20 = 409
ROCRAND_RNG_PSEUDO_THREEFRY4_32_20 = 410
ROCRAND_RNG_PSEUDO_THREEFRY4_64_20 = 411
ROCRAND_RNG_QUASI_DEFAULT = 500
ROCRAND_RNG_QUASI_SOBOL32 = 501
ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL32 = 502
ROCRAND_RNG_QUASI_SOBOL64 = 504
ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL64 = 505

ROCRAND_ORDERING_PSEUDO_BEST = 100
ROCRAND_ORDERING_PSEUDO_DEFAULT = 101
ROCRAND_ORDERING_PSEUDO_SEEDED = 102
ROCRAND_ORDERING_PSEUDO_LEGACY = 103
ROCRAND_ORDERING_PSEUDO_DYNAMIC = 104
ROCRAND_ORDERING_QUASI_DEFAULT = 201

ROCRAND_STATUS = {
    0: ("ROCRAND_STATUS_SUCCESS", "Success"),
    100: ("ROCRAND_STATUS_VERSION_MISMATCH", "Header file and linked library version do not match"),
    101: ("ROCRAND_STATUS_NOT_CREATED", "Generator was not created using rocrand_create_generator"),
    102: ("ROCRAND_STATUS_ALLOCATION_FAILED", "Memory allocation failed during execution"),
    103: ("ROCRAND_STATUS_TYPE_ERROR", "Generator type is wrong"),
    104: ("ROCRAND_STATUS_OUT_OF_RANGE", "Argument out of range"),
    105: ("ROCRAND_STATUS_LENGTH_NOT_MULTIPLE", "Length requested is not a multiple of dimension"),
    106: ("ROCRAND_STATUS_DOUBLE_PRECISION_REQUIRED", "GPU does not have double precision"),
    107: ("ROCRAND_STATUS_LAUNCH_FAILURE", "Kernel launch failure"),
    108: ("ROCRAND_STATUS_INTERNAL_ERROR", "Internal library error"),
}

# (name, argtypes) of every exported function; the half parameters travel as their 16 bits.
_G = c_void_p
class BatchRequest(ctypes.Structure):
    """rocrand_b200_request (include/rocrand_b200.h): one plain call of a batched fill."""
    _fields_ = [("rng_type", c_int), ("distribution", c_int), ("seed", ctypes.c_ulonglong),
                ("offset", ctypes.c_ulonglong), ("param0", ctypes.c_double),
                ("param1", ctypes.c_double), ("output", c_void_p), ("n", c_size_t)]


class TraceItem(ctypes.Structure):
    """rocrand_b200_trace_item (include/rocrand_b200.h): one timed request of a trace."""
    _fields_ = [("arrival_seconds", ctypes.c_double), ("handle", ctypes.c_uint),
                ("distribution", c_int), ("param0", ctypes.c_double),
                ("param1", ctypes.c_double), ("n", c_size_t)]


# batch distributions of rocrand_b200_request
B200_DIST_UINT, B200_DIST_UNIFORM_FLOAT, B200_DIST_UNIFORM_DOUBLE, B200_DIST_NORMAL_FLOAT, \
    B200_DIST_POISSON = range(5)

_SIGNATURES = [
    ("rocrand_b200_generate_batch", [c_void_p, c_size_t, c_void_p]),
    ("rocrand_b200_create_batch_plan", [POINTER(c_void_p), c_void_p, c_size_t, c_void_p]),
    ("rocrand_b200_execute_batch_plan", [c_void_p, c_int, c_void_p]),
    ("rocrand_b200_destroy_batch_plan", [c_void_p]),
    ("rocrand_b200_autotune_batch", [c_void_p]),
    ("rocrand_b200_get_batch_tile", [c_int, c_int, c_void_p]),
    ("rocrand_b200_server_create", [POINTER(c_void_p), c_size_t, ctypes.c_uint, c_int]),
    ("rocrand_b200_server_destroy", [c_void_p]),
    ("rocrand_b200_server_add_generator", [c_void_p, c_int, ctypes.c_ulonglong, c_void_p]),
    ("rocrand_b200_server_submit", [c_void_p, ctypes.c_uint, c_int, ctypes.c_double, ctypes.c_double,
                                    c_size_t, c_void_p]),
    ("rocrand_b200_server_wait", [c_void_p, ctypes.c_ulonglong, c_void_p, c_void_p]),
    ("rocrand_b200_server_release", [c_void_p, ctypes.c_ulonglong]),
    ("rocrand_b200_server_run_trace", [c_void_p, c_void_p, c_size_t, c_void_p, c_void_p]),
    ("rocrand_b200_set_output_position", [_G, c_int, c_ulonglong]),
    ("rocrand_create_generator", [POINTER(c_void_p), c_int]),
    ("rocrand_create_generator_host", [POINTER(c_void_p), c_int]),
    ("rocrand_create_generator_host_blocking", [POINTER(c_void_p), c_int]),
    ("rocrand_destroy_generator", [_G]),
    ("rocrand_generate", [_G, c_void_p, c_size_t]),
    ("rocrand_generate_long_long", [_G, c_void_p, c_size_t]),
    ("rocrand_generate_char", [_G, c_void_p, c_size_t]),
    ("rocrand_generate_short", [_G, c_void_p, c_size_t]),
    ("rocrand_generate_uniform", [_G, c_void_p, c_size_t]),
    ("rocrand_generate_uniform_double", [_G, c_void_p, c_size_t]),
    ("rocrand_generate_uniform_half", [_G, c_void_p, c_size_t]),
    ("rocrand_generate_normal", [_G, c_void_p, c_size_t, c_float, c_float]),
    ("rocrand_generate_normal_double", [_G, c_void_p, c_size_t, c_double, c_double]),
    ("rocrand_generate_normal_half", [_G, c_void_p, c_size_t, c_uint16, c_uint16]),
    ("rocrand_generate_log_normal", [_G, c_void_p, c_size_t, c_float, c_float]),
    ("rocrand_generate_log_normal_double", [_G, c_void_p, c_size_t, c_double, c_double]),
    ("rocrand_generate_log_normal_half", [_G, c_void_p, c_size_t, c_uint16, c_uint16]),
    ("rocrand_generate_poisson", [_G, c_void_p, c_size_t, c_double]),
    ("rocrand_initialize_generator", [_G]),
    ("rocrand_set_stream", [_G, c_void_p]),
    ("rocrand_set_seed", [_G, c_ulonglong]),
    ("rocrand_set_offset", [_G, c_ulonglong]),
    ("rocrand_set_ordering", [_G, c_int]),
    ("rocrand_set_quasi_random_generator_dimensions", [_G, c_uint]),
    ("rocrand_get_version", [POINTER(c_int)]),
]


class _Uint4(ctypes.Structure):
    _fields_ = [("x", c_uint), ("y", c_uint), ("z", c_uint), ("w", c_uint)]


_lib = None


def load_library(path=None):
    """Loads librocrand.so with argument types for every entry point (raises if absent)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError("librocrand.so not built at %s (run __graft_entry__.build())" % p)
    lib = ctypes.CDLL(p)
    for name, args in _SIGNATURES:
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = c_int
    if hasattr(lib, "rocrand_set_seed_uint4"):
        lib.rocrand_set_seed_uint4.argtypes = [_G, _Uint4]
        lib.rocrand_set_seed_uint4.restype = c_int
    if path is None:
        _lib = lib
    return lib


class RocRandError(Exception):
    """Run-time rocRAND error (same text as the reference binding)."""

    def __init__(self, value):
        super().__init__(value)
        self.value = value

    def __str__(self):
        v, s = ROCRAND_STATUS.get(self.value, (str(self.value), "Unknown error"))
        return "{} ({})".format(s, v)


def check_rocrand(status):
    if status != ROCRAND_STATUS_SUCCESS:
        raise RocRandError(status)


def get_version():
    v = c_int(0)
    check_rocrand(load_library().rocrand_get_version(ctypes.byref(v)))
    return v.value


def _half_bits(x):
    import numpy as np
    return int(np.array([x], dtype=np.float16).view(np.uint16)[0])


class RNG:
    """Generator base class (python/rocrand/rocrand/rocrand.py:148-357)."""

    def __init__(self, rngtype, offset=None, stream=None):
        self._lib = load_library()
        self._gen = c_void_p()
        check_rocrand(self._lib.rocrand_create_generator(ctypes.byref(self._gen), rngtype))
        self._offset = 0
        if offset is not None:
            self.offset = offset
        self._stream = None
        if stream is not None:
            self.stream = stream

    def __del__(self):
        gen = getattr(self, "_gen", None)
        if gen is not None and gen.value:
            self._lib.rocrand_destroy_generator(gen)
            self._gen = None

    @property
    def handle(self):
        return self._gen

    @property
    def offset(self):
        return self._offset

    @offset.setter
    def offset(self, offset):
        check_rocrand(self._lib.rocrand_set_offset(self._gen, c_ulonglong(offset)))
        self._offset = offset

    @property
    def stream(self):
        return self._stream

    @stream.setter
    def stream(self, stream):
        """A torch.cuda.Stream, a raw cudaStream_t int, or None for the default stream."""
        raw = getattr(stream, "cuda_stream", stream)
        check_rocrand(self._lib.rocrand_set_stream(self._gen, c_void_p(raw or 0)))
        self._stream = stream

    def _generate(self, fn, ary, size, *args):
        import torch
        if size is None:
            size = ary.numel() if isinstance(ary, torch.Tensor) else ary.size
        if isinstance(ary, torch.Tensor):
            if not ary.is_cuda:
                raise TypeError("device tensor expected")
            if size > ary.numel():
                raise ValueError("requested size is greater than ary")
            check_rocrand(fn(self._gen, c_void_p(ary.data_ptr()), c_size_t(size), *args))
            return ary
        import numpy as np
        if not isinstance(ary, np.ndarray):
            raise TypeError("unsupported type {}".format(type(ary)))
        if size > ary.size:
            raise ValueError("requested size is greater than ary")
        dev = torch.empty(size * ary.itemsize, dtype=torch.uint8, device="cuda")
        check_rocrand(fn(self._gen, c_void_p(dev.data_ptr()), c_size_t(size), *args))
        ary.reshape(-1).view(np.uint8)[: size * ary.itemsize] = dev.cpu().numpy()
        return ary

    @staticmethod
    def _dtype_name(ary):
        return str(ary.dtype).replace("torch.", "")

    def generate(self, ary, size=None):
        d = self._dtype_name(ary)
        fns = {"uint32": "rocrand_generate", "int32": "rocrand_generate",
               "uint64": "rocrand_generate_long_long", "int64": "rocrand_generate_long_long",
               "uint8": "rocrand_generate_char", "int8": "rocrand_generate_char",
               "uint16": "rocrand_generate_short", "int16": "rocrand_generate_short"}
        if d not in fns:
            raise TypeError("unsupported type {}".format(d))
        return self._generate(getattr(self._lib, fns[d]), ary, size)

    def uniform(self, ary, size=None):
        d = self._dtype_name(ary)
        fns = {"float32": "rocrand_generate_uniform", "float64": "rocrand_generate_uniform_double",
               "float16": "rocrand_generate_uniform_half"}
        if d not in fns:
            raise TypeError("unsupported type {}".format(d))
        return self._generate(getattr(self._lib, fns[d]), ary, size)

    def _normal_like(self, ary, mean, stddev, size, names):
        d = self._dtype_name(ary)
        if d == "float32":
            return self._generate(getattr(self._lib, names[0]), ary, size, c_float(mean), c_float(stddev))
        if d == "float64":
            return self._generate(getattr(self._lib, names[1]), ary, size, c_double(mean), c_double(stddev))
        if d == "float16":
            return self._generate(getattr(self._lib, names[2]), ary, size,
                                  c_uint16(_half_bits(mean)), c_uint16(_half_bits(stddev)))
        raise TypeError("unsupported type {}".format(d))

    def normal(self, ary, mean, stddev, size=None):
        return self._normal_like(ary, mean, stddev, size, ("rocrand_generate_normal",
                                                           "rocrand_generate_normal_double",
                                                           "rocrand_generate_normal_half"))

    def lognormal(self, ary, mean, stddev, size=None):
        return self._normal_like(ary, mean, stddev, size, ("rocrand_generate_log_normal",
                                                           "rocrand_generate_log_normal_double",
                                                           "rocrand_generate_log_normal_half"))

    def poisson(self, ary, lmbd, size=None):
        d = self._dtype_name(ary)
        if d not in ("uint32", "int32"):
            raise TypeError("unsupported type {}".format(d))
        return self._generate(self._lib.rocrand_generate_poisson, ary, size, c_double(lmbd))


class PRNG(RNG):
    """Pseudo-random generator (python/rocrand/rocrand/rocrand.py:359-441)."""

    DEFAULT = ROCRAND_RNG_PSEUDO_DEFAULT
    XORWOW = ROCRAND_RNG_PSEUDO_XORWOW
    MRG32K3A = ROCRAND_RNG_PSEUDO_MRG32K3A
    MTGP32 = ROCRAND_RNG_PSEUDO_MTGP32
    PHILOX4_32_10 = ROCRAND_RNG_PSEUDO_PHILOX4_32_10
    MRG31K3P = ROCRAND_RNG_PSEUDO_MRG31K3P
    LFSR113 = ROCRAND_RNG_PSEUDO_LFSR113
    MT19937 = ROCRAND_RNG_PSEUDO_MT19937
    THREEFRY2_32_20 = ROCRAND_RNG_PSEUDO_THREEFRY2_32_20
    THREEFRY2_64_20 = ROCRAND_RNG_PSEUDO_THREEFRY2_64_20
    THREEFRY4_32_20 = ROCRAND_RNG_PSEUDO_THREEFRY4_32_20
    THREEFRY4_64_20 = ROCRAND_RNG_PSEUDO_THREEFRY4_64_20

    def __init__(self, rngtype=DEFAULT, seed=None, offset=None, stream=None):
        super().__init__(rngtype, offset=offset, stream=stream)
        self._seed = None
        if seed is not None:
            self.seed = seed

    @property
    def seed(self):
        return self._seed

    @seed.setter
    def seed(self, seed):
        check_rocrand(self._lib.rocrand_set_seed(self._gen, c_ulonglong(seed)))
        self._seed = seed


class QRNG(RNG):
    """Quasi-random generator (python/rocrand/rocrand/rocrand.py:444-510)."""

    DEFAULT = ROCRAND_RNG_QUASI_DEFAULT
    SOBOL32 = ROCRAND_RNG_QUASI_SOBOL32
    SCRAMBLED_SOBOL32 = ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL32
    SOBOL64 = ROCRAND_RNG_QUASI_SOBOL64
    SCRAMBLED_SOBOL64 = ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL64

    def __init__(self, rngtype=DEFAULT, ndim=None, offset=None, stream=None):
        super().__init__(rngtype, offset=offset, stream=stream)
        self._ndim = 1
        if ndim is not None:
            self.ndim = ndim

    @property
    def ndim(self):
        return self._ndim

    @ndim.setter
    def ndim(self, ndim):
        check_rocrand(self._lib.rocrand_set_quasi_random_generator_dimensions(self._gen, c_uint(ndim)))
        self._ndim = ndim
