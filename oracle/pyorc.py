"""pyorc -- Python driver of the CPU oracle libraries.  TEST INFRASTRUCTURE ONLY.

Drives, through the same call sequence:
  * ``liborc.so``      -- the C restatement of the reference host generators (orc_* API);
  * ``_ref/librocrand_ref.so`` -- the reference's own sources compiled by Makefile.ref, used
    through its host generators (rocrand_create_generator_host_blocking), when present.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference legs may
import this module, and only as the checker or the timed CPU baseline.

Alignment matters for parity: the reference derives its head/tail split from the output
address (vectors of 8 to 32 bytes), so every generate call here takes ``mis`` and places
the host output (mis * element size) mod 64 bytes past a 64-byte boundary.
"""

import ctypes
import os
import subprocess
from ctypes import c_double, c_float, c_size_t, c_uint16, c_ulonglong, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_PATH = os.path.join(HERE, "liborc.so")
REF_PATH = os.path.join(HERE, "_ref", "librocrand_ref.so")

# dist name -> (entry-point suffix, numpy dtype, parameter kind)
DISTS = {
    "uint": ("generate", np.uint32, None),
    "ulonglong": ("generate_long_long", np.uint64, None),
    "char": ("generate_char", np.uint8, None),
    "short": ("generate_short", np.uint16, None),
    "uniform": ("generate_uniform", np.float32, None),
    "uniform_double": ("generate_uniform_double", np.float64, None),
    "uniform_half": ("generate_uniform_half", np.float16, None),
    "normal": ("generate_normal", np.float32, "f"),
    "normal_double": ("generate_normal_double", np.float64, "d"),
    "normal_half": ("generate_normal_half", np.float16, "h"),
    "log_normal": ("generate_log_normal", np.float32, "f"),
    "log_normal_double": ("generate_log_normal_double", np.float64, "d"),
    "log_normal_half": ("generate_log_normal_half", np.float16, "h"),
    "poisson": ("generate_poisson", np.uint32, "lambda"),
}


def build_orc():
    """Builds liborc.so in place (gcc, a few seconds)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "liborc.so"])


def half_bits(x):
    return int(np.array([x], dtype=np.float16).view(np.uint16)[0])


def dist_args(dist, params):
    kind = DISTS[dist][2]
    if kind is None:
        return []
    if kind == "f":
        return [c_float(params[0]), c_float(params[1])]
    if kind == "d":
        return [c_double(params[0]), c_double(params[1])]
    if kind == "h":
        return [c_uint16(half_bits(params[0])), c_uint16(half_bits(params[1]))]
    return [c_double(params[0])]


class CLib:
    """One oracle library.  ``kind`` is "orc" (the C restatement) or "ref" (the reference
    build, host generators)."""

    def __init__(self, kind="orc", path=None):
        self.kind = kind
        self.prefix = "orc_" if kind == "orc" else "rocrand_"
        p = path or (ORC_PATH if kind == "orc" else REF_PATH)
        if kind == "orc" and path is None and not os.path.exists(p):
            build_orc()
        self.lib = ctypes.CDLL(p)
        for fn in ("set_seed", "set_offset"):
            f = getattr(self.lib, self.prefix + fn)
            f.argtypes = [c_void_p, c_ulonglong]

    def set_libm_ulps(self, log_ulps, trig_ulps=0):
        """Oracle only: moves the host library's log and sin/cos results of the fp64 normal
        transforms (and the inverse-erf normal's log) by these many ulps (0, 0 restores)."""
        self.lib.orc_set_libm_ulps(ctypes.c_int(log_ulps), ctypes.c_int(trig_ulps))

    def fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def create(self, rng_type):
        g = c_void_p()
        create = "orc_create" if self.kind == "orc" else "rocrand_create_generator_host_blocking"
        st = getattr(self.lib, create)(ctypes.byref(g), rng_type)
        if st != 0:
            raise RuntimeError("create(%d) -> status %d" % (rng_type, st))
        return g

    def destroy(self, g):
        self.fn("destroy" if self.kind == "orc" else "destroy_generator")(g)

    def set_seed(self, g, seed):
        return self.fn("set_seed")(g, c_ulonglong(seed))

    def set_offset(self, g, offset):
        return self.fn("set_offset")(g, c_ulonglong(offset))

    def set_dimensions(self, g, dims):
        name = "set_dimensions" if self.kind == "orc" else "set_quasi_random_generator_dimensions"
        return self.fn(name)(g, ctypes.c_uint(dims))

    def set_ordering(self, g, order):
        name = "set_ordering"
        return self.fn(name)(g, ctypes.c_int(order))

    def generate(self, g, dist, n, params=(), mis=0):
        """Returns (status, values) for one generate call with the output placed at
        (mis * itemsize) mod 64 bytes past a 64-byte boundary."""
        suffix, dt, _ = DISTS[dist]
        isz = np.dtype(dt).itemsize
        buf = np.zeros(n + 128 // isz + 16, dtype=dt)
        base = buf.ctypes.data
        want = (mis * isz) % 64
        off = 0
        while (base + off * isz) % 64 != want:
            off += 1
        view = buf[off:off + n]
        st = self.fn(suffix)(g, c_void_p(view.ctypes.data), c_size_t(n), *dist_args(dist, params))
        return st, view.copy()


def run_sequence(lib, rng_type, seed, offset, calls, dims=None, ordering=None):
    """Creates a generator, applies seed/offset(/dims), runs ``calls`` = list of
    (dist, n, params, mis) and returns the list of (status, values)."""
    g = lib.create(rng_type)
    try:
        if seed is not None:
            lib.set_seed(g, seed)
        if dims is not None:
            lib.set_dimensions(g, dims)
        if offset is not None:
            lib.set_offset(g, offset)
        if ordering is not None:
            lib.set_ordering(g, ordering)
        return [lib.generate(g, d, n, p, m) for (d, n, p, m) in calls]
    finally:
        lib.destroy(g)
