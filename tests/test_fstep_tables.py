"""Host-side arithmetic of the station-block F-step's shared-memory tables.

The kernel (difx_b200/csrc/gx_fstep_sb.cu) takes the stride-256 radix-16
twiddles W_4096^(r m), m < 256, as the product of two 15 x 16 rows
(B[r][m mod 16] = W_4096^(r (m mod 16)), A[r][m / 16] = W_256^(r (m / 16)))
and decodes 8-bit VDIF codes (format_vdif.c: level = (b - 128) / 3.3) by
fma(x, hi, x * lo) with 1/3.3 = hi + lo when the host finds that equal to the
level table.  These tests restate both in numpy: the factorised twiddle stays
within a few FP32 ulps of the exact one, and the two-term FMA reproduces every
entry of the reference's table.  They also check the index arithmetic of the
phase-cal sums the kernel forms: the exchange-buffer pad slots it parks them
in, and the one bin a thread's samples share.
"""
import numpy as np


def _w(n, k):
    return np.exp(-2j * np.pi * np.asarray(k, dtype=np.float64) / n)


def _c64(z):
    """Complex value rounded to FP32 parts, as the device table holds it."""
    return np.asarray(z).astype(np.complex64)


def _cmul32(a, b):
    """FP32 complex product with the device's rounding (one rounding per product and per sum)."""
    ar, ai = np.float32(a.real), np.float32(a.imag)
    br, bi = np.float32(b.real), np.float32(b.imag)
    re = np.float32(np.float32(ar * br) - np.float32(ai * bi))
    im = np.float32(np.float32(ar * bi) + np.float32(ai * br))
    return np.complex64(re + 1j * im)


def test_stride256_twiddle_rows_factorisation():
    worst = 0.0
    for r in range(1, 16):
        for m in range(256):
            a = _c64(_w(256, r * (m >> 4)))
            b = _c64(_w(4096, r * (m & 15)))
            got = _cmul32(b, a)
            err = abs(complex(got) - _w(4096, r * m))
            worst = max(worst, err)
    # one FP32 rounding of each factor and of the product: a few 2^-24
    assert worst < 4 * 2.0 ** -23, worst


def test_stride16_rows_are_the_table_section():
    # entry (r - 1) 16 + m of the stride-16 pass is W_256^(r m), which is also
    # W_F^(r m F / 256) of the F-point table for every F the kernel takes
    for F in (512, 1024, 2048, 4096, 8192):
        for r in range(1, 16):
            for m in range(16):
                assert abs(_w(256, r * m) - _w(F, r * m * F // 256)) < 1e-12


def _two_term_levels(off):
    hi = np.float32(1.0 / 3.3)
    lo = np.float32(1.0 / 3.3 - float(hi))
    b = np.arange(256)
    x = (b - off).astype(np.float32)
    xlo = (x * lo).astype(np.float32)
    # fma(x, hi, xlo): x * hi is exact in float64 (8-bit x 24-bit), and the sum
    # spans under 53 bits, so one rounding to FP32 is the fused result
    return (x.astype(np.float64) * np.float64(hi) + xlo.astype(np.float64)).astype(np.float32)


def test_8bit_levels_by_two_term_fma_match_table():
    b = np.arange(256)
    table = ((b - 128.0) / 3.3).astype(np.float32)     # format_vdif.c lut8bit, FP64 then FP32
    np.testing.assert_array_equal(_two_term_levels(128.0), table)


def test_8bit_symmetric_offset_keeps_table():
    # the kernel forms x as float(2^23 + b) - (2^23 + offset); with the 127.5
    # offset that bias is not an FP32 value, so the host leaves the table on
    bias = 8388608.0 + 127.5
    assert float(np.float32(bias)) != bias
    assert float(np.float32(8388608.0 + 128.0)) == 8388608.0 + 128.0


def test_phase_cal_pad_slots_are_free():
    # The exchange buffer holds element i of a transform at pad(i) = i + i // 16
    # (F + F / 16 entries); thread j parks its phase-cal sum at 17 j + 16,
    # j < F / 16.  Those slots must lie inside the buffer and never be an
    # element position, so the transform's stores and loads cannot touch them.
    for F in (512, 1024, 2048, 4096, 8192):
        used = {i + i // 16 for i in range(F)}
        slots = {17 * j + 16 for j in range(F // 16)}
        assert len(slots) == F // 16
        assert not (used & slots)
        assert max(slots) < F + F // 16 and max(used) < F + F // 16


def test_phase_cal_bins_of_a_thread():
    # Sample j + (F / 16) t of a block whose first sample is absolute sample S
    # falls in bin (S + j) mod nbins for every t when nbins divides F / 16.
    rng = np.random.default_rng(5)
    for F in (512, 4096, 8192):
        NT = F // 16
        for nbins in [d for d in (1, 2, 4, 8, 16, 32, 64, 128, 256, 512) if NT % d == 0]:
            S = int(rng.integers(0, 2**40))
            for j in rng.integers(0, NT, 8):
                bins = {(S + int(j) + NT * t) % nbins for t in range(16)}
                assert bins == {(S + int(j)) % nbins}
