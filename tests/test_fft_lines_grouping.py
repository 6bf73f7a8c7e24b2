"""Index algebra of the FFT-pass chain's line transform (fft_lines in
maos_b200/csrc/shwfs_gen.cuh), restated on the CPU in float64: the radix-2
decimation-in-time stages taken two at a time -- a thread's four points
k0 + {0, h, 2h, 3h} with stage st's butterflies, then stage st+1's, and one
lone radix-2 stage first when log2 N is odd -- touch every point of a line
once per step, stay inside the line, and give the stage-by-stage transform
exactly (the same operations on every point, in the same order), which is
numpy's FFT (forward) or N times its inverse.  No GPU."""
import numpy as np
import pytest


def _bitrev(k, logn):
    return int(format(k, f"0{logn}b")[::-1], 2)


def _twiddles(n):
    return np.exp(-2j * np.pi * np.arange(n // 2) / n)


def _stagewise(x, direction):
    n = len(x)
    logn = n.bit_length() - 1
    tw = _twiddles(n)
    a = np.array([x[_bitrev(k, logn)] for k in range(n)], dtype=complex)
    for st in range(logn):
        half = 1 << st
        for j in range(n // 2):
            grp, pos = j >> st, j & (half - 1)
            k0 = grp * 2 * half + pos
            k1 = k0 + half
            w = tw[pos << (logn - 1 - st)]
            if direction > 0:
                w = np.conj(w)
            u, t = a[k0], a[k1] * w
            a[k0], a[k1] = u + t, u - t
    return a


def _paired(x, direction):
    n = len(x)
    logn = n.bit_length() - 1
    tw = _twiddles(n)
    a = np.array([x[_bitrev(k, logn)] for k in range(n)], dtype=complex)

    def bfly(u, v, w):
        t = v * w
        return u + t, u - t

    st = 0
    if logn & 1:
        w0 = tw[0] if direction < 0 else np.conj(tw[0])
        for j in range(n // 2):
            a[2 * j], a[2 * j + 1] = bfly(a[2 * j], a[2 * j + 1], w0)
        st = 1
    while st < logn:
        h = 1 << st
        seen = np.zeros(n, dtype=int)
        for j in range(n // 4):
            grp, pos = j >> st, j & (h - 1)
            k0 = grp * 4 * h + pos
            idx = (k0, k0 + h, k0 + 2 * h, k0 + 3 * h)
            assert max(idx) < n
            seen[list(idx)] += 1
            w1 = tw[pos << (logn - 1 - st)]
            w2 = tw[pos << (logn - 2 - st)]
            w3 = tw[(pos + h) << (logn - 2 - st)]
            if direction > 0:
                w1, w2, w3 = np.conj(w1), np.conj(w2), np.conj(w3)
            x0, x1, x2, x3 = (a[i] for i in idx)
            x0, x1 = bfly(x0, x1, w1)  # stage st
            x2, x3 = bfly(x2, x3, w1)
            x0, x2 = bfly(x0, x2, w2)  # stage st + 1
            x1, x3 = bfly(x1, x3, w3)
            for i, v in zip(idx, (x0, x1, x2, x3)):
                a[i] = v
        assert (seen == 1).all()
        st += 2
    return a


@pytest.mark.parametrize("n", [64, 128, 256])
@pytest.mark.parametrize("direction", [-1, 1])
def test_paired_stages_equal_stagewise_transform(n, direction):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    a, b = _stagewise(x, direction), _paired(x, direction)
    assert np.array_equal(a, b)
    ref = np.fft.fft(x) if direction < 0 else np.fft.ifft(x) * n
    assert np.abs(a - ref).max() < 1e-12 * n
