"""Seeded multi-thread VDIF streams for the multiplexer tests (test
infrastructure): single-thread frames of several threads in time order, with
frames dropped, marked invalid, duplicated, swapped within a window, replaced
by fill-pattern frames, and frames of a thread nobody asked for."""
import struct

import numpy as np

FILL = 0x11223344


def header(seconds, frame, thread, nbits, frame_bytes, invalid=False, epoch=40, station=0x4142, cplx=False,
           log2chans=0):
    w0 = (seconds & 0x3FFFFFFF) | (int(invalid) << 31)
    w1 = (frame & 0xFFFFFF) | (epoch << 24)
    w2 = ((frame_bytes // 8) & 0xFFFFFF) | (log2chans << 24)   # version 0
    w3 = (station & 0xFFFF) | ((thread & 1023) << 16) | ((nbits - 1) << 26) | (int(cplx) << 31)
    return struct.pack("<8I", w0, w1, w2, w3, 0, 0, 0, 0)


def stream(thread_ids, nframes, frame_bytes, fps, nbits, seed, start_sec=1000, start_frame=0, invalid_frac=0.0,
           drop_frac=0.0, dup_frac=0.0, swap_frac=0.0, fill_frac=0.0, stray_frac=0.0, cplx=False, chans=1):
    """Bytes of nframes frame times of every thread (chans channels each, a
    power of two), perturbed as asked."""
    lc = chans.bit_length() - 1
    rng = np.random.default_rng(seed)
    payload = frame_bytes - 32
    frames = []
    for n in range(nframes):
        fn = start_frame + n
        sec, fr = start_sec + fn // fps, fn % fps
        for t in thread_ids:
            if rng.random() < drop_frac:
                continue
            body = rng.integers(0, 256, payload, dtype=np.uint8).tobytes()
            inv = rng.random() < invalid_frac
            frames.append(header(sec, fr, t, nbits, frame_bytes, inv, cplx=cplx, log2chans=lc) + body)
            if rng.random() < dup_frac:   # a second copy with other samples: the first must win
                frames.append(header(sec, fr, t, nbits, frame_bytes, False, cplx=cplx, log2chans=lc) +
                              rng.integers(0, 256, payload, dtype=np.uint8).tobytes())
            if rng.random() < stray_frac:
                frames.append(header(sec, fr, 1000, nbits, frame_bytes, False, cplx=cplx, log2chans=lc) + body)
    for i in range(len(frames) - 1):
        if rng.random() < swap_frac:
            frames[i], frames[i + 1] = frames[i + 1], frames[i]
    for i in range(len(frames)):
        if rng.random() < fill_frac:
            frames[i] = struct.pack("<I", FILL) * (frame_bytes // 4)
    return b"".join(frames)


def corner_turn(payloads, nbits, cplx=False):
    """Restatement of the output payload of one complete output frame: time
    sample s of thread k at slot k of P (threads rounded up to a power of two)
    slots of B = nbits x (1|2) bits, samples LSB first; padding slots zero."""
    nt = len(payloads)
    P = 1
    while P < nt:
        P *= 2
    B = nbits * (2 if cplx else 1)
    ids = len(payloads[0])
    nsamp = ids * 8 // B
    out_bits = np.zeros(nsamp * P * B, np.uint8)
    for k, p in enumerate(payloads):
        bits = np.unpackbits(np.frombuffer(p, np.uint8), bitorder="little").reshape(nsamp, B)
        out_bits.reshape(nsamp, P, B)[:, k, :] = bits
    return np.packbits(out_bits, bitorder="little").tobytes()
