"""Order-independent digest of a match set, for comparing pair sets too large
to hold twice (the 50M x 50M crossmatch has ~35M pairs).

Each pair (idA, idB) is mixed into one 64-bit word by the splitmix64
finaliser (Steele, Lea & Flood 2014) applied to idA and then to the mixed idA
xor idB; the digest is the count, the sum (mod 2^64) and the xor of those
words.  Two sets with the same digest are equal up to a collision of all
three, which a missing, extra or altered pair makes astronomically unlikely.
The result does not depend on the order of the pairs, so sets produced by
different kernels (or by the oracle) can be compared without sorting.

Plain numpy and no relative imports: this file also loads by path, without
the package (and so without its CUDA library).
"""
import numpy as np

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_G = np.uint64(0x9E3779B97F4A7C15)


def _mix(x):
    x = x + _G
    x = (x ^ (x >> np.uint64(30))) * _M1
    x = (x ^ (x >> np.uint64(27))) * _M2
    return x ^ (x >> np.uint64(31))


def pairset_digest(pairs, chunk=1 << 22):
    """{"count", "sum", "xor"} of an [n, 2] int64 array of (idA, idB) pairs;
    sum and xor as 16-digit hex strings."""
    p = np.asarray(pairs).reshape(-1, 2)
    total = np.uint64(0)
    acc_x = np.uint64(0)
    with np.errstate(over="ignore"):
        for k in range(0, len(p), chunk):
            q = p[k:k + chunk].view(np.uint64) if p.dtype == np.int64 else p[k:k + chunk].astype(np.int64).view(np.uint64)
            h = _mix(_mix(q[:, 0]) ^ q[:, 1])
            total = total + np.add.reduce(h, dtype=np.uint64)
            acc_x = acc_x ^ np.bitwise_xor.reduce(h)
    return {"count": int(len(p)), "sum": "%016x" % int(total), "xor": "%016x" % int(acc_x)}


def inputs_fingerprint(objs, stride=997):
    """A cheap fingerprint of a catalog (every stride-th record, sha256), to tell
    whether a regenerated synthetic catalog is the one a digest was made from."""
    import hashlib
    a = np.ascontiguousarray(objs[::stride])
    return hashlib.sha256(a.tobytes()).hexdigest()[:32] + ":%d" % len(objs)
