"""Operand rounding of the tensor-core X-step forms, measured by emulation on
the CPU: the visibilities V = X X^H of 64 inputs over 2000 FFT blocks of
seeded noise spectra (a common signal of correlation 0.05, scaled to an
r.m.s. of 8 as the X-step's default operand scales do) with the operands
rounded as each form rounds them -- FP16 once, FP16 hi + lo (the split form,
hi*hi + hi*lo + lo*hi), FP8 E4M3 once, E4M3 hi + lo -- products accumulated
in FP64, so that the figures are the operand rounding alone.  Metrics as the
GPU parity tests use them: per record (one input pair over the channels)
mean|V - V64| / mean|V64|, and per visibility |V - V64| over the larger of
|V64| and its record's mean |V64|.

The E4M3 figures are why the tensor-core X-step offers no FP8 form: one E4M3
rounding per operand misses the 1e-3 visibility bound by more than an order
of magnitude, and even a hi + lo pair of E4M3 values (the same three
products per term as split FP16) is further from the FP64 result than single
FP16."""
import numpy as np
import pytest


def e4m3(x):
    """Round to FP8 E4M3 (1 sign, 4 exponent, 3 mantissa bits, bias 7; no
    infinities, largest finite 448; subnormals down to 2^-9), nearest even,
    saturating."""
    a = np.abs(x)
    e = np.floor(np.log2(np.where(a > 0, a, 1.0)))
    e = np.maximum(e, -6.0)                         # subnormal range shares the smallest exponent
    q = np.exp2(e - 3.0)                            # spacing at that exponent
    r = np.round(a / q) * q                         # np.round: half to even
    r = np.minimum(r, 448.0)
    return np.sign(x) * r


def fp16(x):
    return x.astype(np.float16).astype(np.float64)


def forms(X):
    """Operand pairs (A, B) whose products sum to each form's V."""
    h16 = fp16(X.real) + 1j * fp16(X.imag)
    l16 = fp16(X.real - h16.real) + 1j * fp16(X.imag - h16.imag)
    h8 = e4m3(X.real) + 1j * e4m3(X.imag)
    l8 = e4m3(X.real - h8.real) + 1j * e4m3(X.imag - h8.imag)
    return {
        "fp16": [(h16, h16)],
        "fp16_hilo": [(h16, h16), (h16, l16), (l16, h16)],
        "e4m3": [(h8, h8)],
        "e4m3_hilo": [(h8, h8), (h8, l8), (l8, h8)],
    }


def measure(seed=7, ni=64, k=2000, nchan=16, rho=0.05):
    rng = np.random.default_rng(seed)
    common = rng.standard_normal((nchan, 1, k)) + 1j * rng.standard_normal((nchan, 1, k))
    own = rng.standard_normal((nchan, ni, k)) + 1j * rng.standard_normal((nchan, ni, k))
    X = (np.sqrt(rho) * common + np.sqrt(1 - rho) * own) * (8.0 / np.sqrt(2.0))
    V64 = np.einsum("cik,cjk->cij", X, X.conj())
    iu = np.triu_indices(ni)
    ref = V64[:, iu[0], iu[1]]                      # [channel, pair]
    recmean = np.mean(np.abs(ref), axis=0)          # per record (pair)
    out = {}
    for name, terms in forms(X).items():
        V = sum(np.einsum("cik,cjk->cij", a, b.conj()) for a, b in terms)[:, iu[0], iu[1]]
        d = np.abs(V - ref)
        out[name] = {"record": float(np.max(np.mean(d, axis=0) / recmean)),
                     "visibility": float(np.max(d / np.maximum(np.abs(ref), recmean[None, :])))}
    return out


@pytest.mark.parametrize("seed", [7])
def test_operand_rounding_of_the_forms(seed):
    m = measure(seed)
    for name, v in m.items():
        print(f"\n{name}: worst record {v['record']:.2e}, worst visibility {v['visibility']:.2e}")
    # split FP16 far inside the bounds the GPU tests use; single FP16 within 1e-3 per record
    assert m["fp16_hilo"]["visibility"] < 1e-5 and m["fp16_hilo"]["record"] < 1e-6
    assert m["fp16"]["record"] < 1e-3
    # E4M3: a single rounding misses 1e-3 per visibility by more than 10x, and
    # its hi + lo split stays behind single FP16
    assert m["e4m3"]["visibility"] > 1e-2
    assert m["e4m3_hilo"]["record"] > m["fp16"]["record"]
