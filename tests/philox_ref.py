"""Philox4x32-10 (Salmon, Moraes, Dror and Shaw, SC 2011) and the sampler's uniform and Box-Muller
steps in plain Python/numpy: the CPU reference of gpop_sample_states (test infrastructure)."""
import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    x0, x1, x2, x3 = ctr
    k0, k1 = key
    for r in range(10):
        if r:
            k0 = (k0 + W0) & MASK
            k1 = (k1 + W1) & MASK
        p0 = M0 * x0
        p1 = M1 * x2
        x0, x1, x2, x3 = ((p1 >> 32) ^ x1 ^ k0) & MASK, p1 & MASK, ((p0 >> 32) ^ x3 ^ k1) & MASK, p0 & MASK
    return x0, x1, x2, x3


def unit53(a, b):
    return float((((a << 21) | (b >> 11)) + 1)) * 2.0 ** -53


def normals(i, seed):
    k = (seed & MASK, (seed >> 32) & MASK)
    z = []
    for b in range(3):
        o = philox4x32_10((i & MASK, b, (i >> 32) & MASK, 0), k)
        u1, u2 = unit53(o[0], o[1]), unit53(o[2], o[3])
        rad = np.sqrt(-2.0 * np.log(u1))
        z += [rad * np.cos(2.0 * np.pi * u2), rad * np.sin(2.0 * np.pi * u2)]
    return np.array(z)
