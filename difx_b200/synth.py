"""Seeded synthetic VDIF station streams for correlation jobs.

Each station's stream per recorded band is

    x_k(u) = sqrt(rho) * c_k(u) + sqrt(1 - rho) * n_k(u)

where n_k is independent unit Gaussian noise and c_k is one common
unit-variance Gaussian signal (one per band) advanced by the station's
geometric delay tau_k(t) and carrying the matching fringe phase
exp(+2 pi i f_LO tau_k) on its positive frequencies.  That is the inverse of
the correlator's corrections (the correlator reads station data at
t - tau(t) and multiplies by exp(-2 pi i f_LO tau), mpifxcorr/src/mode.cpp:
674-675, 933-955), the same convention as the reference's own simulator
(applications/datasim/src/subband.cpp:866-918).  The delay is applied per
chunk (integer sample shift plus an FFT fractional shift); the fringe phase
per sample.

Quantisation: 2-bit at +-0.98 sigma into codes 0..3 (decoded by the VDIF
tables to -3.3359, -1, +1, +3.3359), 1-bit by sign, 8-bit as
round(128 + 16 x) clipped to 0..255 (sigma = 16 counts).

Frames are VDIF with 32-byte headers; a seeded fraction of frames can be
marked invalid (header word 0 bit 31), which the correlator blanks.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Tuple

import numpy as np

from .jobfiles import JobSpec, VDIF_HEADER_BYTES

_CHUNK = 16384
_PAD = 256


def _common_signal(seed: int, band: int, first: int, count: int, is_complex: bool) -> np.ndarray:
    """Common (sky) signal samples [first, first+count) of one band; chunk-seeded
    so that any window is reproducible."""
    g = 65536
    c0 = first // g
    c1 = (first + count - 1) // g
    parts = []
    for c in range(c0, c1 + 1):
        rng = np.random.default_rng([seed, 7, band, c & 0x7FFFFFFF, (c >> 31) & 0xFFFF])
        if is_complex:
            v = (rng.standard_normal(g) + 1j * rng.standard_normal(g)) / np.sqrt(2.0)
        else:
            v = rng.standard_normal(g)
        parts.append(v)
    s = np.concatenate(parts)
    off = first - c0 * g
    return s[off:off + count]


def _delay_us(coeffs: np.ndarray, t: np.ndarray) -> np.ndarray:
    return coeffs[0] + coeffs[1] * t + coeffs[2] * t * t


def station_band_signal(spec: JobSpec, station: int, band: int, lofreq_mhz: float,
                        first_sample: int, nsamples: int, rho: float, seed: int) -> np.ndarray:
    """Float samples (real, or complex for complex sampling) of one station/band."""
    fs = spec.samples_per_second
    coeffs = spec.delay_models()[station]
    out = np.empty(nsamples, dtype=np.complex128 if spec.is_complex else np.float64)
    nfft = _CHUNK + 2 * _PAD
    freqs = np.fft.fftfreq(nfft, d=1.0 / fs)  # Hz
    for c0 in range(0, nsamples, _CHUNK):
        n = min(_CHUNK, nsamples - c0)
        u0 = first_sample + c0
        tmid = (u0 + n / 2.0) / fs
        d = _delay_us(coeffs, np.array([tmid]))[0] * 1e-6 * fs  # samples
        di = int(np.floor(d))
        df = d - di
        win = _common_signal(seed, band, u0 + di - _PAD, nfft, spec.is_complex)
        W = np.fft.fft(win)
        # advance by df samples: s(u + df)
        W *= np.exp(2j * np.pi * freqs * df / fs)
        if not spec.is_complex:
            # analytic signal: keep positive frequencies (doubled), drop negative
            W[freqs < 0] = 0.0
            W[1:nfft // 2] *= 2.0
        a = np.fft.ifft(W)[_PAD:_PAD + n]
        t = (u0 + np.arange(n)) / fs
        tau_s = _delay_us(coeffs, t) * 1e-6
        ph = np.exp(2j * np.pi * np.mod(lofreq_mhz * 1e6 * tau_s, 1.0))
        v = a * ph
        out[c0:c0 + n] = v if spec.is_complex else v.real
    rng = np.random.default_rng([seed, 11, station, band, first_sample & 0x7FFFFFFF])
    if spec.is_complex:
        noise = (rng.standard_normal(nsamples) + 1j * rng.standard_normal(nsamples)) / np.sqrt(2.0)
    else:
        noise = rng.standard_normal(nsamples)
    return np.sqrt(rho) * out + np.sqrt(1.0 - rho) * noise


def quantise(x: np.ndarray, nbits: int) -> np.ndarray:
    """Real array -> integer codes (uint8)."""
    if nbits == 1:
        return (x >= 0).astype(np.uint8)
    if nbits == 2:
        t = 0.98
        c = np.where(x < -t, 0, np.where(x < 0, 1, np.where(x < t, 2, 3)))
        return c.astype(np.uint8)
    if nbits == 4:
        return np.clip(np.floor(x * 2.95 + 8.0), 0, 15).astype(np.uint8)
    if nbits == 8:
        return np.clip(np.round(128.0 + 16.0 * x), 0, 255).astype(np.uint8)
    raise ValueError(f"unsupported nbits {nbits}")


def pack_timesamples(codes: np.ndarray, nbits: int) -> np.ndarray:
    """codes [T, nsub] (nsub = bands, or 2*bands interleaved re/im) -> bytes [T*nsub*nbits/8].

    Sub-sample j of a time sample occupies bits j*nbits.. of that sample's
    little-endian bit field (VDIF channel order, LSB first)."""
    T, nsub = codes.shape
    if nbits == 8:
        return codes.reshape(-1).astype(np.uint8)
    spb = 8 // nbits
    flat = codes.reshape(-1, spb).astype(np.uint16)
    shifts = (np.arange(spb) * nbits).astype(np.uint16)
    return np.bitwise_or.reduce(flat << shifts, axis=1).astype(np.uint8)


def vdif_header(spec: JobSpec, seconds: int, framenum: int, invalid: bool, station: int,
                validity: int = -1) -> bytes:
    """VDIF header words 0-7.  Muxed streams (spec.mux_threads > 0) carry the
    EDV4 fields of a multiplexed frame (vdifio.h:272-297): extended version 4,
    mask length = threads, validity mask in words 6-7 (one bit per thread;
    validity < 0: all threads present)."""
    nb = spec.nbands
    log2n = int(np.ceil(np.log2(nb))) if nb > 1 else 0
    w = np.zeros(8, dtype=np.uint32)
    w[0] = (seconds & 0x3FFFFFFF) | ((1 << 31) if invalid else 0)
    w[1] = (framenum & 0xFFFFFF) | (0 << 24)
    w[2] = ((spec.framebytes // 8) & 0xFFFFFF) | (log2n << 24)
    w[3] = ((1 << 31) if spec.is_complex else 0) | ((spec.nbits - 1) << 26) | (station & 0xFFFF)
    if spec.mux_threads > 0:
        mt = spec.mux_threads
        mask = ((1 << mt) - 1) if validity < 0 else validity
        w[4] = (4 << 24) | (mt << 16)
        w[5] = 0xACABFEED
        w[6] = mask & 0xFFFFFFFF
        w[7] = (mask >> 32) & 0xFFFFFFFF
    return w.tobytes()


def edv4_masks(spec: JobSpec, station: int, seed: int, first_frame: int, nframes: int) -> np.ndarray:
    """Validity mask of each muxed frame: all threads present, except a seeded
    fraction spec.edv4_partial_frac of frames with one to three threads absent."""
    mt = spec.mux_threads
    full = (1 << mt) - 1
    out = np.full(nframes, full, dtype=np.int64)
    if spec.edv4_partial_frac <= 0 or mt <= 0:
        return out
    rng = np.random.default_rng([seed, 19, station])
    n = first_frame + nframes
    partial = rng.random(n) < spec.edv4_partial_frac
    drops = rng.integers(0, mt, size=(n, 3))
    ndrop = rng.integers(1, 4, size=n)
    for f in range(nframes):
        af = first_frame + f
        if partial[af]:
            m = full
            for k in range(ndrop[af]):
                m &= ~(1 << int(drops[af, k]))
            out[f] = m
    return out


@dataclasses.dataclass
class StationStream:
    """Whole VDIF frames of one station covering [first_frame, first_frame+nframes)."""
    station: int
    first_frame: int
    nframes: int
    data: np.ndarray          # uint8 [nframes*framebytes]
    invalid: np.ndarray       # bool [nframes]


def make_station_stream(spec: JobSpec, station: int, first_frame: int, nframes: int,
                        rho: float = 0.05, seed: int = 1, invalid_frac: float = 0.0,
                        fill_frac: float = 0.0) -> StationStream:
    """Generate VDIF frames [first_frame, first_frame+nframes) (frame 0 starts at the scan start)."""
    spec.validate()
    fsamp = spec.frame_samples
    first = first_frame * fsamp
    n = nframes * fsamp
    cols = []
    for sbi in spec.station_sb(station):
        sb = spec.subbands[sbi]
        for pi_ in range(len(spec.pols)):
            # the common signal of a subband is the same at every station recording it
            band = sbi * len(spec.pols) + pi_
            lo = sb.freq_mhz
            x = station_band_signal(spec, station, band, lo, first, n, rho, seed)
            if spec.is_complex:
                cols.append(quantise(x.real, spec.nbits))
                cols.append(quantise(x.imag, spec.nbits))
            else:
                cols.append(quantise(x, spec.nbits))
    codes = np.stack(cols, axis=1)  # [n, nsub]
    payload = pack_timesamples(codes, spec.nbits).reshape(nframes, spec.payload_bytes)
    rng = np.random.default_rng([seed, 13, station])
    # draw per absolute frame so a window's flags do not depend on the window
    allflags = rng.random(first_frame + nframes)
    invalid = allflags[first_frame:] < invalid_frac
    fillflags = np.random.default_rng([seed, 17, station]).random(first_frame + nframes)[first_frame:] < fill_frac
    fps = int(round(spec.frames_per_second))
    masks = edv4_masks(spec, station, seed, first_frame, nframes)
    out = np.empty((nframes, spec.framebytes), dtype=np.uint8)
    for f in range(nframes):
        af = first_frame + f
        sec = spec.start_seconds + af // fps
        hdr = vdif_header(spec, sec, af % fps, bool(invalid[f]), station, int(masks[f]))
        out[f, :VDIF_HEADER_BYTES] = np.frombuffer(hdr, dtype=np.uint8)
        out[f, VDIF_HEADER_BYTES:] = payload[f]
        if fillflags[f]:
            out[f, VDIF_HEADER_BYTES:VDIF_HEADER_BYTES + 8] = np.frombuffer(
                np.uint64(0x1122334411223344).tobytes(), dtype=np.uint8)
    return StationStream(station, first_frame, nframes, out.reshape(-1), invalid | fillflags)


@dataclasses.dataclass
class SubintInput:
    """What one Core slot receives for one subint (core.h processslot)."""
    scan: int
    sec: int
    ns: int
    data: List[np.ndarray]       # per station raw bytes (whole frames)
    control: List[np.ndarray]    # per station int32 [3 + flaglength]: scan, sec, ns, valid flags


def subint_window(spec: JobSpec, station: int, sub_start_ns: int) -> Tuple[int, int]:
    """Frames [first, first+count) a station must supply for a subint starting
    sub_start_ns after the scan start (covers the delay range plus one frame)."""
    coeffs = spec.delay_models()[station]
    t0 = sub_start_ns * 1e-9
    t1 = t0 + spec.subint_ns * 1e-9
    ts = np.linspace(t0, t1, 65)
    tau = _delay_us(coeffs, ts) * 1e-6
    clock = (spec.clock_us[station] if station < len(spec.clock_us) else 0.0) * 1e-6
    lo = t0 - tau.max() - clock - 2e-6
    hi = t1 - tau.min() - clock + spec.fftchannels / spec.samples_per_second + 2e-6
    fdur = spec.frame_samples / spec.samples_per_second
    f0 = int(np.floor(lo / fdur)) - 1
    f1 = int(np.ceil(hi / fdur)) + 1
    return f0, f1 - f0


def frame_time_ns(spec: JobSpec, frame: int) -> Tuple[int, int]:
    """(sec, ns) after scan start of the first sample of a frame."""
    fps = int(round(spec.frames_per_second))
    sec = frame // fps
    ns = int(round((frame % fps) * 1e9 / fps))
    return sec, ns


def valid_flags(spec: JobSpec, bad_blocks: Optional[np.ndarray] = None) -> np.ndarray:
    """Per-block valid flags packed 30 per int32 (mpifxcorr.h FLAGS_PER_INT)."""
    nb = spec.blocks_per_send
    nwords = nb // 30 + (1 if nb % 30 else 0)
    w = np.zeros(nwords, dtype=np.int64)
    ok = np.ones(nb, dtype=bool)
    if bad_blocks is not None:
        ok[np.asarray(bad_blocks, dtype=np.int64)] = False
    for b in range(nb):
        if ok[b]:
            w[b // 30] |= (1 << (b % 30))
    return w.astype(np.int32)


def build_subint(spec: JobSpec, streams: List[StationStream], sub_start_ns: int,
                 bad_blocks: Optional[List[np.ndarray]] = None) -> SubintInput:
    """Slice each station's stream to the window the subint needs."""
    data, control = [], []
    for s, st in enumerate(streams):
        f0, nf = subint_window(spec, s, sub_start_ns)
        if f0 < st.first_frame or f0 + nf > st.first_frame + st.nframes:
            raise ValueError(f"station {s} stream does not cover frames {f0}..{f0 + nf}")
        a = (f0 - st.first_frame) * spec.framebytes
        data.append(st.data[a:a + nf * spec.framebytes])
        sec, ns = frame_time_ns(spec, f0)
        flags = valid_flags(spec, bad_blocks[s] if bad_blocks else None)
        control.append(np.concatenate([np.array([0, sec, ns], dtype=np.int32), flags]))
    sec = sub_start_ns // 1_000_000_000
    ns = sub_start_ns % 1_000_000_000
    return SubintInput(0, int(sec), int(ns), data, control)


def streams_for_job(spec: JobSpec, sub_starts_ns: List[int], rho: float = 0.05, seed: int = 1,
                    invalid_frac: float = 0.0, fill_frac: float = 0.0) -> List[StationStream]:
    out = []
    for s in range(spec.nstations):
        lo, hi = None, None
        for t in sub_starts_ns:
            f0, nf = subint_window(spec, s, t)
            lo = f0 if lo is None else min(lo, f0)
            hi = f0 + nf if hi is None else max(hi, f0 + nf)
        out.append(make_station_stream(spec, s, lo, hi - lo, rho=rho, seed=seed,
                                       invalid_frac=invalid_frac, fill_frac=fill_frac))
    return out


def make_station_stream_tiled(spec: JobSpec, station: int, first_frame: int, nframes: int, tile_frames: int,
                              rho: float = 0.05, seed: int = 1, invalid_frac: float = 0.0) -> StationStream:
    """Like make_station_stream, but only the first `tile_frames` frames are
    synthesised from the signal model; their payloads repeat over the rest of
    the window.  Headers (seconds, frame number, invalid bit per absolute
    frame) are written for every frame.  Used for benchmark-size inputs,
    where the throughput does not depend on the sample values."""
    tile_frames = max(1, min(tile_frames, nframes))
    base = make_station_stream(spec, station, first_frame, tile_frames, rho=rho, seed=seed, invalid_frac=0.0)
    fb = spec.framebytes
    tile = base.data.reshape(tile_frames, fb)
    reps = (nframes + tile_frames - 1) // tile_frames
    out = np.tile(tile, (reps, 1))[:nframes].copy()
    fps = int(round(spec.frames_per_second))
    af = first_frame + np.arange(nframes, dtype=np.int64)
    rng = np.random.default_rng([seed, 13, station])
    invalid = rng.random(first_frame + nframes)[first_frame:] < invalid_frac
    hdr = out[:, :VDIF_HEADER_BYTES].view(np.uint32).reshape(nframes, 8)
    sec = (spec.start_seconds + af // fps).astype(np.uint32)
    hdr[:, 0] = (sec & np.uint32(0x3FFFFFFF)) | np.where(invalid, np.uint32(1 << 31), np.uint32(0))
    hdr[:, 1] = (af % fps).astype(np.uint32) & np.uint32(0xFFFFFF)
    return StationStream(station, first_frame, nframes, out.reshape(-1), invalid)
