"""Inputs of the shader prediction vectors (spec_intra.json, spec_mc.json),
shared by the generator (make_golden.py) and the test (tests/test_oracle.py):
planes of pseudo-random bytes from a 64-bit xorshift, so the inputs are
reproduced exactly from a seed on any machine and only the seeds and the
expected outputs' digests are committed."""
import hashlib

import numpy as np

INTRA_PLANE = (72, 80)          # rows, cols
MC_PLANE = (48, 64)
INTRA_SIZES = (4, 8, 16, 32)
INTRA_MODES = (0, 1, 2, 9, 3, 7)
INTRA_POS = ((0, 0), (24, 0), (0, 16), (40, 32))   # (x, y): no edges, left, above, both


def plane_bytes(seed, shape):
    """xorshift64 stream; a smooth ramp under the noise keeps the filters'
    outputs away from the clip limits most of the time."""
    x = (seed * 0x9E3779B97F4A7C15 + 1) & 0xFFFFFFFFFFFFFFFF
    n = shape[0] * shape[1]
    out = np.empty(n, np.uint8)
    for i in range(n):
        x ^= (x << 13) & 0xFFFFFFFFFFFFFFFF
        x ^= x >> 7
        x ^= (x << 17) & 0xFFFFFFFFFFFFFFFF
        r, c = divmod(i, shape[1])
        base = (r * 3 + c * 2) % 160 + 40
        out[i] = (base + (x >> 58) - 32) & 0xFF
    return out.reshape(shape)


def digest(arr):
    return hashlib.sha256(np.ascontiguousarray(arr, np.uint8).tobytes()).hexdigest()[:24]


def intra_cases():
    k = 0
    for n in INTRA_SIZES:
        for mode in INTRA_MODES:
            for (x, y) in INTRA_POS:
                yield {"seed": 1000 + k, "n": n, "mode": mode, "x": x, "y": y}
                k += 1


def mc_cases():
    rng = np.random.default_rng(7)   # only picks the cases; the picks are committed
    k = 0
    for fy in range(8):
        for fx in range(8):
            ix, iy = (int(v) for v in rng.integers(-6, 7, 2))
            yield {"seed": 2000 + k, "mvx": ix * 8 + fx, "mvy": iy * 8 + fy}
            k += 1
    for mvx, mvy in ((-563, 3), (557, -5), (6, -445), (-1, 421), (-700, -650), (645, 602), (-3, -4), (9, 11)):
        yield {"seed": 2000 + k, "mvx": mvx, "mvy": mvy}
        k += 1
