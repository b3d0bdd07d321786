"""Call sequences recorded in the golden fixtures (see make_golden.py).

A case is {"rng": type, "seed": s, "offset": o, "calls": [[dist, n, params, mis], ...]}.
``mis`` places the output (mis * element size) mod 64 bytes past a 64-byte boundary, which
selects the reference's head/tail split.  Sequences of several calls pin continuity.
"""

PSEUDO_DISTS = [
    ("uint", []), ("ulonglong", []), ("char", []), ("short", []), ("uniform", []), ("uniform_double", []),
    ("uniform_half", []), ("normal", [0.5, 2.0]), ("normal_double", [-1.0, 0.5]),
    ("normal_half", [1.0, 2.0]), ("log_normal", [0.2, 0.7]), ("log_normal_double", [0.1, 0.4]),
    ("log_normal_half", [0.0, 0.5]), ("poisson", [0.5]), ("poisson", [10.0]),
    ("poisson", [1000.0]), ("poisson", [5000.5]),
]


def _seq(dist, params):
    return [[dist, 1000, params, 0], [dist, 37, params, 1], [dist, 4099, params, 3],
            [dist, 1, params, 2], [dist, 0, params, 0], [dist, 257, params, 5]]


def pseudo_cases(rng, seeds_offsets, extra=()):
    out = []
    for seed, offset in seeds_offsets:
        for dist, params in PSEUDO_DISTS:
            out.append({"rng": rng, "seed": seed, "offset": offset, "calls": _seq(dist, params)})
    out.extend(extra)
    return out


# Philox / ThreeFry: the vector at j % 262144 == 0 comes from thread 0 of the reference
# grid, which the head moved by ceil(head/ow)*iw instead of head: pin that with a call
# whose vector count is a multiple of 262144 (char: 16 per vector, 13 head elements).
_STRIDE_CORNER = [
    {"rng": 404, "seed": 77, "offset": 0,
     "calls": [["char", 13 + 262144 * 16 + 5, [], 3], ["short", 7 + 262144 * 8 + 3, [], 1],
               ["normal", 3 + 262144 * 4 + 1, [0.0, 1.0], 1]]},
]

def _tf_corner(rng):
    return [{"rng": rng, "seed": 77, "offset": 5,
             "calls": [["char", 13 + 262144 * 16 + 5, [], 3], ["normal", 3 + 262144 * 4 + 1, [0.0, 1.0], 1],
                       ["uniform_double", 1 + 262144 * 2 + 1, [], 1]]}]


_SO = [(1234, 0), (0xdeadbeefcafe, 12345)]

# Stateful engines: the head/tail slot is vec_n % 131072; pin a call whose vector count is
# a multiple of the engine count (the head/tail thread is then slot 0).
def _st_corner(rng):
    return [{"rng": rng, "seed": 99, "offset": 131072 * 3 + 17,
             "calls": [["normal", 1 + 131072 * 2 * 2 + 1, [0.0, 1.0], 1],
                       ["short", 1 + 131072 * 2 + 1, [], 1], ["char", 3 + 131072 * 4 + 2, [], 1],
                       ["uniform_double", 5, [], 0]]}]


_SO_ST = [(1234, 0), (0xdeadbeefcafe, 123456789)]


def quasi_cases(rng):
    """Sobol: dimension-major output, n a multiple of dims; a non-multiple call pins the
    LENGTH_NOT_MULTIPLE status."""
    out = []
    for dims, offset in ((1, 0), (64, 4096), (3, 77)):
        for dist, params in PSEUDO_DISTS:
            out.append({"rng": rng, "seed": None, "offset": offset, "dims": dims,
                        "calls": [[dist, dims * 1000, params, 0], [dist, dims * 37, params, 1],
                                  [dist, dims * 4099, params, 3], [dist, dims * 2 + 1, params, 0],
                                  [dist, dims * 257, params, 5]]})
    return out

# MT19937: generator state is 8192 x 624 words and every (re)seed of the reference host
# generator jumps all 8192 of them (minutes on a CPU), so each seed gets one long sequence
# instead of one case per distribution.  It crosses rounds, changes input width (the
# reference skips to the next unused slot group) and ends calls mid-round.  Calls served
# from the state left by the previous call ("short" calls, mt19937.hpp:973-1005) are kept
# aligned and a multiple of the vector width: the reference's host emulation of that kernel
# shares one extra-unit flag across its eight emulated lanes (mt19937.hpp:404-430), so its
# head/tail values there differ from its device kernel, which the library follows.
_MT_ELEMS = {"uint": (4, 1, 1), "uniform": (4, 1, 1), "char": (1, 1, 4), "short": (2, 1, 2),
             "uniform_half": (2, 1, 2), "uniform_double": (8, 2, 1), "normal": (4, 2, 2),
             "log_normal": (4, 2, 2), "normal_double": (8, 4, 2), "log_normal_double": (8, 4, 2),
             "normal_half": (2, 1, 2), "log_normal_half": (2, 1, 2), "poisson": (4, 1, 1)}


def _mt_check(calls):
    """Asserts that no short call of the sequence needs the extra head/tail unit."""
    stride, start, prev = 65536, 0, 0
    for dist, n, _, mis in calls:
        if dist == "ulonglong":
            continue  # TYPE_ERROR before any state change (mt19937.hpp:1044-1050)
        tsize, iw, ow = _MT_ELEMS[dist]
        full = stride * (78 // iw)
        if prev != iw and start > 0:
            used = (start + stride - 1) // stride * prev
            start = (used + iw - 1) // iw * stride
            start = 0 if start >= full else start
        head = min(n, (ow - mis % ow) % ow)
        tail = (n - head) % ow
        total = (n - head) // ow + (1 if head or tail else 0)
        short = start > 0 and start + total <= full
        assert not (short and (head or tail)), (dist, n, mis)
        start, prev = (start + total) % full, iw
    return calls


_MT_CALLS = _mt_check([
    ["uint", 1000, [], 0], ["uniform", 4096, [], 0], ["normal", 5002, [0.5, 2.0], 0],
    ["char", 4100, [], 0], ["uniform_double", 778, [], 0], ["normal_double", 1000, [-1.0, 0.5], 0],
    ["poisson", 3000, [10.0], 0], ["uint", 5200000, [], 0], ["normal", 70000, [0.0, 1.0], 0],
    ["normal", 4200001, [0.0, 1.0], 1], ["uniform_half", 11000003, [], 0],
    ["poisson", 100, [1000.0], 0], ["log_normal", 10, [0.2, 0.7], 0], ["uint", 0, [], 0],
    ["char", 21000003, [], 3], ["log_normal_double", 2, [0.1, 0.4], 0],
    ["normal_half", 5111808 * 2 + 7, [1.0, 2.0], 1], ["poisson", 4000, [5000.5], 0],
    ["log_normal_half", 4, [0.0, 0.5], 0], ["short", 2002, [], 0],
    ["log_normal", 10223617, [0.2, 0.7], 1], ["ulonglong", 8, [], 0],
    ["poisson", 2555904 + 12345, [0.5], 0], ["uniform", 65536 * 78, [], 0],
])

CASES = {
    "philox": pseudo_cases(404, [(1234, 0), (0xdeadbeef, 12345), (0xAAAAAAAAAAA, 2**40 + 3)],
                           _STRIDE_CORNER),
    "threefry2x32": pseudo_cases(408, _SO, _tf_corner(408)),
    "threefry2x64": pseudo_cases(409, _SO, _tf_corner(409)),
    "threefry4x32": pseudo_cases(410, _SO, _tf_corner(410)),
    "threefry4x64": pseudo_cases(411, _SO, _tf_corner(411)),
    "xorwow": pseudo_cases(401, _SO_ST, _st_corner(401)),
    "mrg32k3a": pseudo_cases(402, _SO_ST + [(0, 7)], _st_corner(402)),
    "mrg31k3p": pseudo_cases(405, _SO_ST, _st_corner(405)),
    "lfsr113": pseudo_cases(406, _SO_ST, _st_corner(406)),
    "mtgp32": pseudo_cases(403, [(1234, None), (0xdeadbeefcafe, None)],
                           [{"rng": 403, "seed": 5, "offset": None,
                             "calls": [["uint", 131072 * 3 + 77, [], 0], ["normal", 1 + 131072 * 4 + 1, [0.0, 1.0], 1],
                                       ["char", 3 + 256 * 4 * 7, [], 1], ["uniform_double", 256 * 512, [], 0]]}]),
    "mt19937": [{"rng": 407, "seed": 1234, "offset": None, "calls": _MT_CALLS},
                {"rng": 407, "seed": 0xdeadbeefcafe, "offset": None,
                 "calls": _mt_check(_MT_CALLS[::-1])}],
    "sobol32": quasi_cases(501),
    "scrambled_sobol32": quasi_cases(502),
    "sobol64": quasi_cases(504),
    "scrambled_sobol64": quasi_cases(505),
}
