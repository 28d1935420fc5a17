"""Host-side keys of the JAX Threefry-2x32 stream PyGFMC draws from.

PyGFMC takes ``jax.random.PRNGKey`` keys; this engine takes the same two
uint32 words (a ``jax.random.PRNGKey(s)`` converted with ``np.asarray``, or
:func:`PRNGKey` here) and derives every sub-stream exactly as jax does with
the partitionable Threefry (the default since jax 0.5):

* ``split(key, n)[i] == fold_in(key, i) == threefry2x32(key, (0, i))``
* ``bits(key, (n,))[i]`` = ``y0 ^ y1`` of ``threefry2x32(key, (0, i))``
  (32-bit), ``y0 << 32 | y1`` (64-bit)

so walkers drawn here and runs keyed here reproduce PyGFMC's.
"""
import numpy as np

_ROT = ((13, 15, 26, 6), (17, 29, 16, 24))


def threefry2x32(k0, k1, c0, c1):
    """Threefry-2x32 (20 rounds) over broadcast uint32 arrays."""
    with np.errstate(over="ignore"):
        k0 = np.asarray(k0, dtype=np.uint32)
        k1 = np.asarray(k1, dtype=np.uint32)
        ks = (k0, k1, k0 ^ k1 ^ np.uint32(0x1BD11BDA))
        x0 = np.asarray(c0, dtype=np.uint32) + ks[0]
        x1 = np.asarray(c1, dtype=np.uint32) + ks[1]
        for i in range(5):
            for r in _ROT[i % 2]:
                x0 = x0 + x1
                x1 = (x1 << np.uint32(r)) | (x1 >> np.uint32(32 - r))
                x1 = x1 ^ x0
            x0 = x0 + ks[(i + 1) % 3]
            x1 = x1 + ks[(i + 2) % 3] + np.uint32(i + 1)
    return x0, x1


def as_key(key):
    """A key as a uint32 array of shape (2,) (accepts jax keys, lists, arrays)."""
    k = np.asarray(key)
    if k.shape != (2,) or not np.issubdtype(k.dtype, np.integer):
        raise ValueError("rng_key must be a legacy Threefry key: two uint32 words, "
                         f"got shape {k.shape} dtype {k.dtype}")
    if np.any(k < 0) or np.any(k > 0xFFFFFFFF):
        raise ValueError("rng_key words must be uint32 values")
    return k.astype(np.uint32)


def PRNGKey(seed):
    """jax.random.PRNGKey(seed) for an integer seed: [seed >> 32, seed & 0xFFFFFFFF]."""
    seed = int(seed)
    return np.array([(seed >> 32) & 0xFFFFFFFF, seed & 0xFFFFFFFF], dtype=np.uint32)


def split(key, num=2):
    key = as_key(key)
    i = np.arange(num, dtype=np.uint32)
    y0, y1 = threefry2x32(key[0], key[1], np.zeros(num, np.uint32), i)
    return np.stack([y0, y1], axis=1)


def fold_in(key, data):
    key = as_key(key)
    y0, y1 = threefry2x32(key[0], key[1], 0, np.uint32(int(data) & 0xFFFFFFFF))
    return np.array([y0, y1], dtype=np.uint32)


def bits32(key, n):
    key = as_key(key)
    y0, y1 = threefry2x32(key[0], key[1], np.zeros(n, np.uint32), np.arange(n, dtype=np.uint32))
    return y0 ^ y1


def bits64(key, n):
    key = as_key(key)
    y0, y1 = threefry2x32(key[0], key[1], np.zeros(n, np.uint32), np.arange(n, dtype=np.uint32))
    return (y0.astype(np.uint64) << np.uint64(32)) | y1.astype(np.uint64)


def uniform(key, dtype=np.float64):
    """jax.random.uniform(key) (a scalar in [0, 1))."""
    if np.dtype(dtype) == np.float64:
        b = bits64(key, 1)[0] >> np.uint64(12)
        return float(np.array(b | np.uint64(0x3FF0000000000000)).view(np.float64) - 1.0)
    b = bits32(key, 1)[0] >> np.uint32(9)
    return float(np.array(b | np.uint32(0x3F800000)).view(np.float32) - np.float32(1.0))


def randint(key, shape, minval, maxval, x64=True):
    """jax.random.randint: two draws combined through 2**nbits % span."""
    n = int(np.prod(shape))
    k1, k2 = split(key, 2)
    span_i = int(maxval) - int(minval)
    if span_i <= 0:
        return np.full(shape, int(minval), dtype=np.int64 if x64 else np.int32)
    if x64:
        hi, lo = bits64(k1, n), bits64(k2, n)
        span = np.uint64(span_i)
        mult = (2 ** 32 % span_i) ** 2 % span_i
        off = ((hi % span) * np.uint64(mult) + (lo % span)) % span
        return (int(minval) + off.astype(np.int64)).reshape(shape)
    hi, lo = bits32(k1, n), bits32(k2, n)
    span = np.uint32(span_i)
    mult = (2 ** 16 % span_i) ** 2 % span_i
    with np.errstate(over="ignore"):
        off = ((hi % span) * np.uint32(mult) + (lo % span)) % span
    return (int(minval) + off.astype(np.int64)).reshape(shape).astype(np.int32)


def permutation(key, x):
    """jax.random.permutation of a 1-D array: rounds of a stable sort by
    fresh 32-bit keys (3 ln(n) / ln(2**32 - 1) rounds, rounded up)."""
    x = np.asarray(x).copy()
    rounds = int(np.ceil(3 * np.log(max(1, x.size)) / np.log(np.iinfo(np.uint32).max)))
    key = as_key(key)
    for _ in range(rounds):
        key, sub = split(key, 2)
        x = x[np.argsort(bits32(sub, x.size), kind="stable")]
    return x


def permutation_rows(keys, base):
    """One :func:`permutation` of ``base`` per key (vectorised over keys)."""
    keys = np.asarray(keys, dtype=np.uint32)
    n, size = keys.shape[0], np.asarray(base).size
    rounds = int(np.ceil(3 * np.log(max(1, size)) / np.log(np.iinfo(np.uint32).max)))
    out = np.broadcast_to(np.asarray(base), (n, size)).copy()
    cur = keys.copy()
    for _ in range(rounds):
        nk0, nk1 = threefry2x32(cur[:, 0], cur[:, 1], 0, 0)
        s0, s1 = threefry2x32(cur[:, 0], cur[:, 1], 0, 1)
        y0, y1 = threefry2x32(s0[:, None], s1[:, None], 0, np.arange(size, dtype=np.uint32)[None, :])
        order = np.argsort(y0 ^ y1, axis=1, kind="stable")
        out = np.take_along_axis(out, order, axis=1)
        cur = np.stack([nk0, nk1], axis=1)
    return out
