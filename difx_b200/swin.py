"""Reader for DIFX/SWIN binary visibility records.

The format is the one Visibility::writeSWIN writes
(mpifxcorr/src/visibility.cpp:781-960, header in appendSWINHeaderBuffered
1205-1234): per record a 74-byte little-endian header -- sync word
0xFF00FF00, header version 1, baseline number (256 * (telescope1 + 1) +
telescope2 + 1), MJD, seconds of day (centre of the integration), config
index, source index, freq index, polarisation pair, pulsar bin, weight,
u, v, w (metres) -- followed by nchan complex64 channels.
"""
from __future__ import annotations

from typing import Callable, List, Tuple, Union

import numpy as np

SYNC_WORD = 0xFF00FF00
HEADER = np.dtype([("sync", "<u4"), ("version", "<i4"), ("baseline", "<i4"), ("mjd", "<i4"), ("seconds", "<f8"),
                   ("config", "<i4"), ("source", "<i4"), ("freq", "<i4"), ("pol", "S2"), ("bin", "<i4"),
                   ("weight", "<f8"), ("uvw", "<f8", (3,))])
assert HEADER.itemsize == 74


def read_records(path: str, nchan: Union[int, Callable[[int], int]]) -> List[Tuple[np.void, np.ndarray]]:
    """All records of a SWIN file as (header, complex64 channels); nchan is the
    channel count of every record, or a function of the record's freq index."""
    raw = np.fromfile(path, dtype=np.uint8)
    out = []
    pos = 0
    while pos < raw.size:
        if raw.size - pos < HEADER.itemsize:
            raise ValueError(f"{path}: truncated header at byte {pos}")
        h = raw[pos:pos + HEADER.itemsize].view(HEADER)[0]
        if int(h["sync"]) != SYNC_WORD:
            raise ValueError(f"{path}: bad sync word at byte {pos}")
        n = nchan(int(h["freq"])) if callable(nchan) else int(nchan)
        pos += HEADER.itemsize
        data = raw[pos:pos + 8 * n].view(np.complex64).copy()
        if data.size != n:
            raise ValueError(f"{path}: truncated record at byte {pos}")
        pos += 8 * n
        out.append((h, data))
    return out
