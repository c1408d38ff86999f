"""Host restatement of the engine's active-Brownian random stream (test
infrastructure): Philox4x32-10 (Salmon, Moraes, Dror and Shaw, SC'11) keyed
by the system seed, counter {particle id, step lo, step hi, 0 | 1}, two 53-bit
uniforms per draw and Box-Muller, three standard normals per particle and
step, as normals3 in activechi4_b200/csrc/acg_device.cuh.  The transcendental
functions are numpy's, so values agree with the device's to a few ulp."""
import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)
SEED_XOR = 0x5DEECE66D  # the engine's Brownian stream: the system seed ^ this


def philox4x32(c0, c1, c2, c3, k0, k1):
    c = [np.asarray(x, dtype=np.uint64) & MASK for x in (c0, c1, c2, c3)]
    k0, k1 = int(k0) & 0xFFFFFFFF, int(k1) & 0xFFFFFFFF
    for _ in range(10):
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c = [hi1 ^ c[1] ^ np.uint64(k0), lo1, hi0 ^ c[3] ^ np.uint64(k1), lo0]
        k0 = (k0 + W0) & 0xFFFFFFFF
        k1 = (k1 + W1) & 0xFFFFFFFF
    return c


def u53(a, b):
    m = ((a << np.uint64(32)) | b) >> np.uint64(11)
    return (m.astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)


def normals(seed, step, n):
    """[n][3] standard normals of particles 0..n-1 at `step`."""
    s = int(seed) ^ SEED_XOR
    k0, k1 = s & 0xFFFFFFFF, (s >> 32) & 0xFFFFFFFF
    ids = np.arange(n, dtype=np.uint64)
    st0, st1 = int(step) & 0xFFFFFFFF, (int(step) >> 32) & 0xFFFFFFFF
    a = philox4x32(ids, st0, st1, 0, k0, k1)
    b = philox4x32(ids, st0, st1, 1, k0, k1)
    r1, t1 = np.sqrt(-2.0 * np.log(u53(a[0], a[1]))), 6.283185307179586 * u53(a[2], a[3])
    r2, t2 = np.sqrt(-2.0 * np.log(u53(b[0], b[1]))), 6.283185307179586 * u53(b[2], b[3])
    return np.stack([r1 * np.cos(t1), r1 * np.sin(t1), r2 * np.cos(t2)], axis=1)
